"""tagore_pruning_cfs_noalloc against tagore_pruning_cfs.

The static-scratch variant must give the same pruned rows and entry point as
the allocating entry point, call after call (its scratch is reused, so a
second call in a row catches state left over from the first), and must not
draw on the device's default memory pool. Collected last so that it also runs
after everything else has used the device.
"""
import numpy as np
import pytest

from tagore_b200 import synth

pytestmark = pytest.mark.gpu

N, DIM, K = 6000, 64, 32


@pytest.fixture(scope="module")
def knn(capi):
    base, _ = synth.mixture("sift", N, DIM, 24, 31)
    st = capi.gnn_descent_host(base, K, 6, mode=capi.KNN_CHOSEN)
    bufs = st.buffers()
    st.free()
    return bufs


def fresh(capi, bufs):
    s = capi.State.alloc(N, DIM, K)
    for i, (name, _) in enumerate(capi.BUFFERS[:8]):
        s.upload(i, bufs[name])
    return s


def pool_high_water():
    """Peak bytes in use in device 0's default memory pool since the last reset."""
    from cuda.bindings import driver as drv
    err, = drv.cuInit(0)
    assert err == drv.CUresult.CUDA_SUCCESS
    err, pool = drv.cuDeviceGetDefaultMemPool(0)
    assert err == drv.CUresult.CUDA_SUCCESS
    attr = drv.CUmemPool_attribute
    err, cur = drv.cuMemPoolGetAttribute(pool, attr.CU_MEMPOOL_ATTR_USED_MEM_CURRENT)
    assert err == drv.CUresult.CUDA_SUCCESS
    return pool, int(cur)


def reset_high(pool):
    from cuda.bindings import driver as drv
    err, = drv.cuMemPoolSetAttribute(pool, drv.CUmemPool_attribute.CU_MEMPOOL_ATTR_USED_MEM_HIGH,
                                     drv.cuuint64_t(0))
    assert err == drv.CUresult.CUDA_SUCCESS


def read_high(pool):
    from cuda.bindings import driver as drv
    err, v = drv.cuMemPoolGetAttribute(pool, drv.CUmemPool_attribute.CU_MEMPOOL_ATTR_USED_MEM_HIGH)
    assert err == drv.CUresult.CUDA_SUCCESS
    return int(v)


CALLS = [("path", "dist", 24, 64, 1.0), ("path", "dist", 24, 64, 1.0),
         ("2-hop", "angle", 16, 64, 0.5), ("path", "dist", 32, 96, 1.2)]


def test_noalloc_matches_allocating_entry_calls_in_a_row(capi, knn):
    pool, _ = pool_high_water()
    for mode, metric, fd, topm, thre in CALLS:
        ref = fresh(capi, knn)
        ep_ref = capi.pruning_cfs(ref, fd, mode, metric, topm=topm, thre=thre)
        exp = {i: ref.download(i) for i in (0, 1, 4, 5)}
        ref.free()
        got = fresh(capi, knn)
        _, before = pool_high_water()
        reset_high(pool)
        ep = capi.pruning_cfs_noalloc(got, fd, mode, metric, topm=topm, thre=thre)
        assert read_high(pool) <= before, "the no-allocation prune drew on the memory pool"
        assert ep == ep_ref
        for i, a in exp.items():
            assert np.array_equal(got.download(i), a), (mode, metric, fd, capi.BUFFERS[i][0])
        got.free()


def test_noalloc_rejections(capi, knn):
    big = capi.State.alloc(40000, DIM, K)  # about 31 MB of temporaries at FINAL_DEGREE 32
    with pytest.raises(capi.TagoreError) as e:
        capi.pruning_cfs_noalloc(big, 32, "path", "dist")
    assert e.value.code == capi.TAGORE_EINVAL and "static scratch" in str(e.value)
    big.free()
    s = fresh(capi, knn)
    with pytest.raises(capi.TagoreError) as e:
        capi.pruning_cfs_noalloc(s, 16, "1-hop", "rank")
    assert e.value.code == capi.TAGORE_EINVAL
    s.free()
