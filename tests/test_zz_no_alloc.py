"""The allocation-free batch entry point (ntt_batch_run_noalloc) against the
allocating one (ntt_batch_submit) through the C ABI.  Needs a B200.

Self-contained (preloads its own tables), so it passes alone in a fresh
process as well as after the other tests.
"""
import ctypes

import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nb(torch_cuda):
    import ntt_b200
    f = ntt_b200._lib.ntt_batch_run_noalloc
    f.argtypes = [ctypes.POINTER(ntt_b200.Job), ctypes.c_int, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return ntt_b200


def run_noalloc(nb, jobs, stream=None):
    arr, keep = nb._job_array(jobs)
    st = nb._lib.ntt_batch_run_noalloc(arr, len(jobs), stream)
    return st


def test_noalloc_matches_allocating_entry_point_twice(torch_cuda, nb):
    torch = torch_cuda
    from ntt_b200 import mixes
    jobs = mixes.ragged_mix(seed=41, count=30, logn=range(12, 18), limbs=(1, 6), bits=(30, 31),
                            ops=((nb.OP_FORWARD, 2), (nb.OP_INVERSE, 2), (nb.OP_MULTIPLY, 1)))
    for j in jobs:
        nb.tables_preload(j.logN, j.moduli)
    g = torch.Generator(device="cuda")
    g.manual_seed(7)
    for call in range(2):  # two calls in a row on the same scratch
        data = [mixes.uniform_device(torch, j, g) for j in jobs]
        opnd = [mixes.uniform_device(torch, j, g) if j.op == nb.OP_MULTIPLY else None
                for j in jobs]
        ref = [x.clone() for x in data]
        torch.cuda.synchronize()
        st = run_noalloc(nb, [(j.op, j.logN, j.moduli, x, a) for j, x, a in zip(jobs, data, opnd)])
        assert st == 0, nb._lib.ntt_last_error()
        nb.batch_submit([(j.op, j.logN, j.moduli, x, a) for j, x, a in zip(jobs, ref, opnd)])
        torch.cuda.synchronize()
        for i, (x, r) in enumerate(zip(data, ref)):
            assert torch.equal(x, r), f"call {call} job {i}"


def test_noalloc_back_to_back_on_one_stream_allocates_nothing(torch_cuda, nb):
    """Two calls queued on one stream with no wait between them (the second
    call's descriptor upload is ordered behind the first kernel), each
    checked against the allocating entry point; the device's free memory is
    the same before and after (the calls allocate nothing)."""
    torch = torch_cuda
    from ntt_b200 import mixes
    jobs = mixes.ragged_mix(seed=43, count=24, logn=range(12, 18), limbs=(1, 5), bits=(30, 31),
                            ops=((nb.OP_FORWARD, 2), (nb.OP_INVERSE, 2), (nb.OP_MULTIPLY, 1)))
    for j in jobs:
        nb.tables_preload(j.logN, j.moduli)
    g = torch.Generator(device="cuda")
    g.manual_seed(11)
    sets = []
    for _ in range(2):
        data = [mixes.uniform_device(torch, j, g) for j in jobs]
        opnd = [mixes.uniform_device(torch, j, g) if j.op == nb.OP_MULTIPLY else None
                for j in jobs]
        sets.append((data, opnd, [x.clone() for x in data]))
    warm = [mixes.uniform_device(torch, j, g) for j in jobs]
    s = torch.cuda.Stream()
    # the same job list once first, so that the one-time set-up (the scratch's
    # address, and the kernels' code if the driver loads it lazily) is done
    st = run_noalloc(nb, [(j.op, j.logN, j.moduli, x, a)
                          for j, x, a in zip(jobs, warm, sets[0][1])], s.cuda_stream)
    assert st == 0, nb._lib.ntt_last_error()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for data, opnd, _ in sets:  # queued back to back, no synchronisation in between
        st = run_noalloc(nb, [(j.op, j.logN, j.moduli, x, a)
                              for j, x, a in zip(jobs, data, opnd)], s.cuda_stream)
        assert st == 0, nb._lib.ntt_last_error()
    s.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    for k, (data, opnd, ref) in enumerate(sets):
        nb.batch_submit([(j.op, j.logN, j.moduli, x, a) for j, x, a in zip(jobs, ref, opnd)])
        torch.cuda.synchronize()
        for i, (x, r) in enumerate(zip(data, ref)):
            assert torch.equal(x, r), f"call {k} job {i}"


def test_noalloc_refuses_a_capturing_stream(torch_cuda, nb):
    torch = torch_cuda
    from ntt_b200 import mixes
    pool = mixes.prime_pool(12, 30, 4)
    nb.tables_preload(12, pool[:1])
    x = torch.zeros(1, 1 << 12, dtype=torch.int32, device="cuda")
    s = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    torch.cuda.synchronize()
    with torch.cuda.stream(s):
        graph.capture_begin()
        st = run_noalloc(nb, [(nb.OP_FORWARD, 12, pool[:1], x, None)], s.cuda_stream)
        graph.capture_end()
    assert nb.STATUS_NAMES[st] == "NTT_ERR_UNSUPPORTED"
    assert "capturing" in nb._lib.ntt_last_error().decode()
    del graph


def test_noalloc_limits(torch_cuda, nb):
    torch = torch_cuda
    from ntt_b200 import mixes
    pool = mixes.prime_pool(12, 31, 300)
    nb.tables_trim()
    x = torch.zeros(1, 1 << 12, dtype=torch.int32, device="cuda")
    # tables that were never preloaded: refused, nothing launched
    st = run_noalloc(nb, [(nb.OP_FORWARD, 12, [pool[-1]], x, None)])
    assert nb.STATUS_NAMES[st] == "NTT_ERR_NOT_READY"
    # more tiles than the scratch holds: refused before any device work
    many = [pool[0]] * (4096 + 1)
    st = run_noalloc(nb, [(nb.OP_FORWARD, 12, many, 0x1000, None)])
    assert nb.STATUS_NAMES[st] == "NTT_ERR_UNSUPPORTED"
    assert "4096" in nb._lib.ntt_last_error().decode()
