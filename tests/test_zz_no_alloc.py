"""The allocation-free entry point (wl_sumcheck_abc_prove_noalloc), for callers that cannot
allocate device memory: called through the C ABI twice in a row, it must return exactly the
proof of the allocating entry point (wl_sumcheck_abc_prove_device) for the same device inputs,
and reject sizes beyond its fixed scratch. Collected last so a failure here comes after every
other test has run; it also passes alone in a fresh process."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

P = 0x7F000001


def _inputs(log_n, seed):
    import torch
    rng = np.random.default_rng(seed)
    a = rng.integers(0, P, 1 << log_n, dtype=np.uint64)
    b = rng.integers(0, P, 1 << log_n, dtype=np.uint64)
    c = (a * b) % P
    return [torch.from_numpy(x.astype(np.uint32).view(np.int32)).cuda() for x in (a, b, c)]


def _device_memory_state():
    """Free device memory (cudaMemGetInfo) and the bytes in use in the device's default
    stream-ordered pool (where cudaMallocAsync allocates): an allocation of either kind
    changes one of them."""
    import torch
    from cuda.bindings import driver as drv
    free, _ = torch.cuda.mem_get_info(0)
    assert drv.cuInit(0)[0] == drv.CUresult.CUDA_SUCCESS
    err, dev = drv.cuDeviceGet(0)
    assert err == drv.CUresult.CUDA_SUCCESS
    err, pool = drv.cuDeviceGetDefaultMemPool(dev)
    assert err == drv.CUresult.CUDA_SUCCESS
    err, used = drv.cuMemPoolGetAttribute(pool, drv.CUmemPool_attribute.CU_MEMPOOL_ATTR_USED_MEM_CURRENT)
    assert err == drv.CUresult.CUDA_SUCCESS
    return free, int(used)


@pytest.mark.parametrize("log_n,skips", [(12, 3), (14, 2), (9, 4)])
def test_noalloc_matches_allocating_entry_point(wl, ctx, log_n, skips):
    import torch
    consts, _ = wl.generate_workload(2)
    p16 = consts[148:296]
    a, b, c = _inputs(log_n, 40 + log_n)
    ref, _ = wl.sumcheck_abc_prove(ctx, p16, log_n, skips, a, b, c, device=True)
    before = [t.clone() for t in (a, b, c)]
    torch.cuda.synchronize()
    for call in range(2):
        mem0 = _device_memory_state()
        got = wl.sumcheck_abc_prove_noalloc(p16, log_n, skips, a, b, c)
        torch.cuda.synchronize()
        assert np.array_equal(got, ref)
        if call == 1:  # warm call: no device allocation of any kind
            assert _device_memory_state() == mem0
    assert all(torch.equal(x, y) for x, y in zip((a, b, c), before))  # inputs untouched


def test_noalloc_rejects_a_capturing_stream(wl):
    """The prover waits for its stream between rounds, which graph capture cannot hold: a
    stream under capture is refused before any work is queued."""
    import torch
    consts, _ = wl.generate_workload(2)
    a, b, c = _inputs(10, 2)
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    st = None
    with torch.cuda.stream(s):
        g.capture_begin()
        try:
            st = wl.sumcheck_abc_prove_noalloc(consts[148:296], 10, 3, a, b, c, stream=s.cuda_stream)
        except wl.ProverError as e:
            st = e.status
        finally:
            g.capture_end()
    assert st == 1  # WL_E_INVALID_ARG


def test_noalloc_rejects_sizes_beyond_scratch(wl):
    consts, _ = wl.generate_workload(2)
    a, b, c = _inputs(15, 1)
    with pytest.raises(wl.ProverError) as e:
        wl.sumcheck_abc_prove_noalloc(consts[148:296], 15, 3, a, b, c)
    assert e.value.status == 7  # WL_E_SCRATCH_LIMIT
