"""tagore_pruning_cfs_noalloc against tagore_pruning_cfs and the oracle.

The static-scratch variant must give the same pruned rows and entry point as
the allocating entry point, call after call (its scratch is reused, so a
second call in a row catches state left over from the first), and must make
no allocation. The library counts every allocation it makes (its memory pool
and pinned host buffers) in tagore_allocation_count(); the count must not move
across a no-allocation call. The device's default memory pool is watched as a
second guard. Collected last so that it also runs after everything else has
used the device.
"""
import numpy as np
import pytest

from oracle import oracle as orc
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


def default_pool():
    from cuda.bindings import driver as drv
    err, = drv.cuInit(0)
    assert err == drv.CUresult.CUDA_SUCCESS
    err, pool = drv.cuDeviceGetDefaultMemPool(0)
    assert err == drv.CUresult.CUDA_SUCCESS
    return pool


def pool_attr(pool, name):
    from cuda.bindings import driver as drv
    err, v = drv.cuMemPoolGetAttribute(pool, getattr(drv.CUmemPool_attribute, name))
    assert err == drv.CUresult.CUDA_SUCCESS
    return int(v)


def reset_high(pool):
    from cuda.bindings import driver as drv
    err, = drv.cuMemPoolSetAttribute(pool, drv.CUmemPool_attribute.CU_MEMPOOL_ATTR_USED_MEM_HIGH,
                                     drv.cuuint64_t(0))
    assert err == drv.CUresult.CUDA_SUCCESS


CALLS = [("path", "dist", 24, 64, 1.0), ("path", "dist", 24, 64, 1.0),
         ("2-hop", "angle", 16, 64, 0.5), ("path", "dist", 32, 96, 1.2)]


def test_noalloc_matches_allocating_entry_calls_in_a_row(capi, knn):
    pool = default_pool()
    L = capi.lib()
    for mode, metric, fd, topm, thre in CALLS:
        ref = fresh(capi, knn)
        ep_ref = capi.pruning_cfs(ref, fd, mode, metric, topm=topm, thre=thre)
        exp = {i: ref.download(i) for i in (0, 1, 4, 5)}
        ref.free()
        got = fresh(capi, knn)
        before = pool_attr(pool, "CU_MEMPOOL_ATTR_USED_MEM_CURRENT")
        reset_high(pool)
        allocs = L.tagore_allocation_count()
        ep = capi.pruning_cfs_noalloc(got, fd, mode, metric, topm=topm, thre=thre)
        assert L.tagore_allocation_count() == allocs, "the no-allocation prune allocated"
        assert pool_attr(pool, "CU_MEMPOOL_ATTR_USED_MEM_HIGH") <= before, \
            "the no-allocation prune drew on the default memory pool"
        assert ep == ep_ref
        for i, a in exp.items():
            assert np.array_equal(got.download(i), a), (mode, metric, fd, capi.BUFFERS[i][0])
        got.free()


def test_allocation_count_sees_the_allocating_entry(capi, knn):
    """The counter is live: the allocating prune moves it."""
    L = capi.lib()
    s = fresh(capi, knn)
    allocs = L.tagore_allocation_count()
    capi.pruning_cfs(s, 24, "path", "dist", topm=64)
    assert L.tagore_allocation_count() > allocs
    s.free()


def test_noalloc_rows_equal_the_oracle(capi, knn):
    n = N
    buf = orc.Buffers(knn["graph"].reshape(n, K), knn["nei_distance"].reshape(n, K),
                      knn["data"].reshape(n, DIM), knn["center"], knn["reverse_graph"],
                      knn["reverse_distance"], knn["reverse_num"], knn["hybrid_list"])
    ep_c = orc.prune_cfs(buf, 24, "path", "dist", topm=64, thre=1.0)
    for _ in range(2):
        got = fresh(capi, knn)
        ep = capi.pruning_cfs_noalloc(got, 24, "path", "dist", topm=64, thre=1.0)
        assert ep == ep_c
        assert np.array_equal(got.download(0), buf.graph)
        assert np.array_equal(got.download(5), buf.reverse_num)
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
