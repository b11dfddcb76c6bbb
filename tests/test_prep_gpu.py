"""GNN_descent's input preparation on the device (pybind.cu:19-61): the FP16
base, the centroid and the power-of-ten factor equal the reference's own
output (golden fixture) and the oracle's, whether the base comes from host
memory or streams from an fvecs file that the device parses; norms are the
exact squared norms of the FP16 rows."""
import os

import numpy as np
import pytest

from tagore_b200 import synth

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
PREP = os.path.join(HERE, "golden", "golden_prep.npz")


def outputs(st):
    n, dim = st.st.n, st.st.dim
    half = st.download(2).reshape(n, dim)
    center = st.download(6)
    norms = st.download(8)
    return half, center, norms, st.st.norm_factor


def test_golden_prep_both_paths(capi, tmp_path):
    g = np.load(PREP)
    base = g["base"]
    path = tmp_path / "golden.fvecs"
    synth.write_fvecs(str(path), base)
    for st in (capi.gnn_descent_file(path, 16, 1), capi.gnn_descent_host(base, 16, 1)):
        half, center, norms, _ = outputs(st)
        st.free()
        assert np.array_equal(half.reshape(-1).view(np.uint16), g["data_half"])
        assert np.array_equal(center.view(np.uint16), g["center_half"])
        h = half.astype(np.float32)
        assert np.allclose(norms, (h * h).sum(1), rtol=1e-6)


@pytest.mark.parametrize("kind,n,dim", [("sift", 150_000, 128), ("gist", 20_000, 960),
                                        ("deep", 70_001, 100)])
def test_file_ingest_equals_host_path_and_oracle(capi, orc, tmp_path, kind, n, dim):
    base, _ = synth.mixture(kind, n, dim, 16, 71)
    path = tmp_path / "b.fvecs"
    synth.write_fvecs(str(path), base)
    a = capi.gnn_descent_file(path, 8, 1)
    b = capi.gnn_descent_host(base, 8, 1)
    oa, ob = outputs(a), outputs(b)
    a.free()
    b.free()
    for x, y in zip(oa[:3], ob[:3]):
        assert np.array_equal(x.view(np.uint8), y.view(np.uint8))
    assert oa[3] == ob[3]
    half, center, factor = orc.host_prep(base)
    assert np.array_equal(oa[0].view(np.uint16), half.view(np.uint16))
    assert np.array_equal(oa[1].view(np.uint16), center.view(np.uint16))
    assert np.float32(oa[3]) == np.float32(factor)


def test_bad_record_is_an_io_error(capi, tmp_path):
    base, _ = synth.mixture("sift", 100_000, 16, 4, 72)
    path = tmp_path / "bad.fvecs"
    synth.write_fvecs(str(path), base)
    raw = bytearray(path.read_bytes())
    rec = 4 * (16 + 1)
    raw[rec * 77_777:rec * 77_777 + 4] = (15).to_bytes(4, "little")   # one record claims dim 15
    path.write_bytes(bytes(raw))
    with pytest.raises(capi.TagoreError, match="vector 77777"):
        capi.gnn_descent_file(path, 8, 1)
    path.write_bytes(bytes(raw[:-3]))                                 # not whole records
    with pytest.raises(capi.TagoreError):
        capi.gnn_descent_file(path, 8, 1)
