"""Bit-exact parity of the CUDA path with the CPU oracle (needs a B200).

Every call goes through the C ABI (libntt_b200.so via ntt_b200).  The oracle
restates the reference's cpu_ntt_butterfly / cpu_intt_butterfly
(src/v04_montgomery.cu:742-784); the forward output is compared in the
Montgomery domain, as the reference's --verify does after from_mont
(v04:1081-1087).  Integer work: the bar is exact equality.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from twiddle_ref import device_tables

pytestmark = pytest.mark.gpu
THREADS = os.cpu_count() or 4


@pytest.fixture(scope="module")
def nb(torch_cuda):
    import ntt_b200
    return ntt_b200


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()


def host(t):
    return t.cpu().numpy().view(np.uint32)


def moduli_set(logN, limbs, bits):
    start = 974258177 if bits == "baseline" else (int(2 ** 29.5) if bits == 30 else int(2 ** 30.5))
    return O.ascending_primes(logN, limbs, start)


def roundtrip_check(torch, nb, logN, mods, x, plan=None):
    T = O.LimbTables(logN, mods)
    p = plan or nb.Plan(logN, mods)
    d = dev(torch, x)
    p.forward(d)
    torch.cuda.synchronize()
    f = host(d)
    assert np.array_equal(f, T.forward_mont(x, THREADS)), "forward mismatch"
    p.inverse(d)
    torch.cuda.synchronize()
    expect = np.stack([x[i] % np.uint32(q) for i, (q, _) in enumerate(mods)])
    assert np.array_equal(host(d), expect), "inverse mismatch"
    assert p.check() == 0  # no bounded wait expired on the device"


def test_config1_baseline_moduli(torch_cuda, nb):
    """2^16 x 16 limbs, the 16 ascending primes from 974258177, seeded input."""
    mods = moduli_set(16, 16, "baseline")
    roundtrip_check(torch_cuda, nb, 16, mods, O.uniform_limbs(16, [q for q, _ in mods], 1234))
    # the reference's own input generator (fill_random, seed 1234 per limb)
    roundtrip_check(torch_cuda, nb, 16, mods, O.fill_random_ref_compatible(16, [q for q, _ in mods]))


def test_reference_verify_config(torch_cuda, nb):
    """The reference's --verify case: default_moduli (7 of them 31-bit)."""
    mods = O.REFERENCE_DEFAULT_MODULI
    roundtrip_check(torch_cuda, nb, 16, mods, O.fill_random_ref_compatible(16, [q for q, _ in mods]))


@pytest.mark.parametrize("logN", [12, 13, 14, 15, 16, 17])
@pytest.mark.parametrize("limbs", [1, 4, 16, 32, 64])
@pytest.mark.parametrize("bits", [30, 31])
def test_sweep(torch_cuda, nb, logN, limbs, bits):
    """Config 2: logN 12..17 x limbs {1,4,16,32,64} x 30/31-bit ascending primes."""
    mods = moduli_set(logN, limbs, bits)
    x = O.uniform_limbs(logN, [q for q, _ in mods], logN * 1000 + limbs * 10 + bits)
    roundtrip_check(torch_cuda, nb, logN, mods, x)


@pytest.mark.parametrize("logN", list(range(1, 12)))
def test_small_sizes(torch_cuda, nb, logN):
    mods = moduli_set(logN, 3, 30) + moduli_set(logN, 2, 31)
    x = O.uniform_limbs(logN, [q for q, _ in mods], logN)
    x[0, 0] = 0xFFFFFFFF  # forward reduces any uint32 input, like mont_mul(x, r2)
    roundtrip_check(torch_cuda, nb, logN, mods, x)


@pytest.mark.parametrize("schedule", [0, 1], ids=["direct", "staged"])
def test_every_compiled_config(torch_cuda, nb, schedule):
    """Every compiled configuration under both schedules, 30/31-bit moduli,
    several polynomials per launch (the staged schedule prefetches across
    limbs of one cluster's chunk)."""
    cfgs = nb.kernel_configs()
    for idx, c in enumerate(cfgs):
        for bits in (30, 31):
            mods = moduli_set(c.logN, 3, bits)
            p = nb.Plan(c.logN, mods)
            p.force_config(idx, idx)
            p.set_schedule(schedule)
            x = O.uniform_limbs(c.logN, [q for q, _ in mods], idx)
            roundtrip_check(torch_cuda, nb, c.logN, mods, x, plan=p)
            polys = 5
            xs = np.stack([O.uniform_limbs(c.logN, [q for q, _ in mods], 100 * idx + k)
                           for k in range(polys)])
            d = dev(torch_cuda, xs)
            p.forward_many(d, polys)
            p.inverse_many(d, polys)
            torch_cuda.cuda.synchronize()
            assert np.array_equal(host(d).reshape(xs.shape), xs)
            assert p.check() == 0


@pytest.mark.parametrize("logN", [5, 12, 16, 17])
def test_device_twiddle_tables(torch_cuda, nb, logN):
    """The device-generated Shoup tables equal the oracle's tables (with the
    stage-0 fold constants in entries 0 and 1)."""
    torch = torch_cuda
    mods = moduli_set(logN, 3, 30) + moduli_set(logN, 2, 31)
    p = nb.Plan(logN, mods)
    fptr, iptr, qptr = p.tables()
    N, L = 1 << logN, len(mods)
    ef, ei = device_tables(O.LimbTables(logN, mods))
    assert np.array_equal(_read_device(torch, fptr, L * N * 2).reshape(L, N, 2), ef)
    assert np.array_equal(_read_device(torch, iptr, L * N * 2).reshape(L, N, 2), ei)
    assert np.array_equal(_read_device(torch, qptr, L), np.array([q for q, _ in mods], np.uint32))


def _read_device(torch, ptr, words):
    """Copy `words` uint32 from a raw device address (cudaMemcpy D2H)."""
    import ctypes
    torch.cuda.synchronize()
    rt = ctypes.CDLL("libcudart.so.12")
    rt.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    out = np.empty(words, dtype=np.uint32)
    assert rt.cudaMemcpy(out.ctypes.data, ptr, words * 4, 2) == 0  # cudaMemcpyDeviceToHost
    return out


def test_many_polys_with_stride(torch_cuda, nb):
    torch = torch_cuda
    logN, limbs, polys = 16, 5, 3
    mods = moduli_set(logN, limbs, 30)
    N = 1 << logN
    stride = limbs * N + 64  # padded rows, still a multiple of 4 words
    x = np.zeros((polys, stride), np.uint32)
    for p_ in range(polys):
        x[p_, :limbs * N] = O.uniform_limbs(logN, [q for q, _ in mods], 7 + p_).reshape(-1)
    x[:, limbs * N:] = 0xABCDEF01
    d = dev(torch, x)
    P = nb.Plan(logN, mods)
    P.forward_many(d, polys, stride)
    torch.cuda.synchronize()
    out = host(d).reshape(polys, stride)
    T = O.LimbTables(logN, mods)
    for p_ in range(polys):
        assert np.array_equal(out[p_, :limbs * N].reshape(limbs, N),
                              T.forward_mont(x[p_, :limbs * N].reshape(limbs, N), THREADS))
    assert (out[:, limbs * N:] == 0xABCDEF01).all()  # padding untouched
    P.inverse_many(d, polys, stride)
    torch.cuda.synchronize()
    assert np.array_equal(host(d).reshape(polys, stride), x)


def test_streams_and_batched_equals_alone(torch_cuda, nb):
    torch = torch_cuda
    logN, limbs = 15, 8
    mods = moduli_set(logN, limbs, 31)
    P = nb.Plan(logN, mods)
    xs = [O.uniform_limbs(logN, [q for q, _ in mods], 50 + k) for k in range(4)]
    alone = []
    for x in xs:
        d = dev(torch, x)
        P.forward(d)
        alone.append(host(d))
    s = torch.cuda.Stream()
    big = dev(torch, np.stack(xs))
    with torch.cuda.stream(s):
        P.forward_many(big, 4, 0, stream=s)
    s.synchronize()
    assert np.array_equal(host(big), np.stack(alone))


def test_full_size_properties(torch_cuda, nb):
    """Largest sweep case (2^17 x 64 limbs, 32 MiB): linearity of the forward
    transform and the roundtrip identity, checked without the oracle."""
    torch = torch_cuda
    logN, limbs = 17, 64
    mods = moduli_set(logN, limbs, 31)
    q = np.array([m[0] for m in mods], np.uint64)[:, None]
    P = nb.Plan(logN, mods)
    a = O.uniform_limbs(logN, q[:, 0], 1)
    b = O.uniform_limbs(logN, q[:, 0], 2)
    s = ((a.astype(np.uint64) + b) % q).astype(np.uint32)
    da, db, ds = dev(torch, a), dev(torch, b), dev(torch, s)
    for t in (da, db, ds):
        P.forward(t)
    torch.cuda.synchronize()
    fa, fb, fs = host(da), host(db), host(ds)
    assert np.array_equal(((fa.astype(np.uint64) + fb) % q).astype(np.uint32), fs)
    P.inverse(da)
    torch.cuda.synchronize()
    assert np.array_equal(host(da), a)


def test_dropin_launchers_match_reference_tables(torch_cuda, nb):
    """launch_ntt / launch_intt with the reference's Montgomery-form tables
    (v04:947-967 uploads) and LC phase triples give the plan's results."""
    torch = torch_cuda
    for logN, mods in ((16, O.REFERENCE_DEFAULT_MODULI), (12, moduli_set(12, 4, 30)),
                       (8, moduli_set(8, 2, 31))):
        T = O.LimbTables(logN, mods)
        tw, itw = T.mont_tables()
        x = O.fill_random_ref_compatible(logN, T.q)
        d = dev(torch, x)
        tw_d, itw_d = dev(torch, tw), dev(torch, itw)
        q_d, qi_d = dev(torch, T.q), dev(torch, T.q_inv)
        r2_d, di_d = dev(torch, T.r2), dev(torch, T.degree_inv_mont)
        ph = nb.default_transform(logN) if logN >= 10 else None
        nb.launch_ntt(d, tw_d, q_d, qi_d, r2_d, len(mods), logN,
                      ph.ntt_phase1 if ph else None, ph.ntt_phase2 if ph else None)
        torch.cuda.synchronize()
        assert np.array_equal(host(d), T.forward_mont(x, THREADS))
        nb.launch_intt(d, itw_d, q_d, qi_d, di_d, len(mods), logN,
                       ph.intt_phase1 if ph else None, ph.intt_phase2 if ph else None)
        torch.cuda.synchronize()
        assert np.array_equal(host(d), x)
    nb.shim_cache_clear()


def test_dropin_tables_rewritten_in_place(torch_cuda, nb):
    """A caller that rewrites its tables and moduli at the same addresses gets
    the new moduli's results on the next call (the reference reads its tables
    at every launch); one changed table word alone is picked up too; a
    modulus outside the Montgomery range is reported by shim_check."""
    torch = torch_cuda
    logN = 13
    mods_a, mods_b = moduli_set(logN, 4, 30), moduli_set(logN, 4, 31)
    Ta, Tb = O.LimbTables(logN, mods_a), O.LimbTables(logN, mods_b)
    bufs = None
    for T in (Ta, Tb, Ta):
        tw, itw = T.mont_tables()
        arrays = (tw, itw, T.q, T.q_inv, T.r2, T.degree_inv_mont)
        if bufs is None:
            bufs = [dev(torch, a) for a in arrays]
        else:  # same addresses, new contents
            for b, a in zip(bufs, arrays):
                b.copy_(dev(torch, a))
        tw_d, itw_d, q_d, qi_d, r2_d, di_d = bufs
        x = O.uniform_limbs(logN, T.q, 7)
        d = dev(torch, x)
        nb.launch_ntt(d, tw_d, q_d, qi_d, r2_d, 4, logN, None, None)
        torch.cuda.synchronize()
        assert np.array_equal(host(d), T.forward_mont(x, THREADS))
        nb.launch_intt(d, itw_d, q_d, qi_d, di_d, 4, logN, None, None)
        torch.cuda.synchronize()
        assert np.array_equal(host(d), x)
    nb.shim_check()
    # one table word changed (entry 5 of limb 2 set to entry 6's value): the
    # forward must follow the edited table, entry by entry
    tw, _ = Ta.mont_tables()
    tw = tw.copy()
    tw[2, 5] = tw[2, 6]
    bufs[0].copy_(dev(torch, tw))
    x = O.uniform_limbs(logN, Ta.q, 8)
    d = dev(torch, x)
    nb.launch_ntt(d, bufs[0], bufs[2], bufs[3], bufs[4], 4, logN, None, None)
    torch.cuda.synchronize()
    got = host(d)
    assert np.array_equal(got[[0, 1, 3]], Ta.forward_mont(x, THREADS)[[0, 1, 3]])
    assert not np.array_equal(got[2], Ta.forward_mont(x, THREADS)[2])
    # a modulus above the range: reported, not silently used
    q_bad = Ta.q.copy()
    q_bad[1] = (1 << 31) + 11
    bufs[2].copy_(dev(torch, q_bad))
    nb.launch_ntt(d, bufs[0], bufs[2], bufs[3], bufs[4], 4, logN, None, None)
    with pytest.raises(nb.NttError) as e:
        nb.shim_check()
    assert e.value.name == "NTT_ERR_MODULUS_RANGE"
    nb.shim_check()  # the record was cleared
    nb.shim_cache_clear()


def test_reference_v04_gpu_output(torch_cuda, nb):
    """Third reference: the reference's own launch_ntt / launch_intt, built
    unchanged for sm_100a (oracle/_ref), on the same inputs."""
    R = O.ref_lib()
    if R is None:
        pytest.skip("reference harness not built")
    torch = torch_cuda
    mods = O.REFERENCE_DEFAULT_MODULI
    T = O.LimbTables(16, mods)
    tw, itw = T.mont_tables()
    x = O.fill_random_ref_compatible(16, T.q)
    ref_d, ours = dev(torch, x), dev(torch, x)
    tw_d, itw_d = dev(torch, tw), dev(torch, itw)
    q_d, qi_d = dev(torch, T.q), dev(torch, T.q_inv)
    r2_d, di_d = dev(torch, T.r2), dev(torch, T.degree_inv_mont)
    assert R.ref_gpu_launch_ntt16(ref_d.data_ptr(), tw_d.data_ptr(), q_d.data_ptr(),
                                  qi_d.data_ptr(), r2_d.data_ptr(), 16) == 0
    P = nb.Plan(16, mods)
    P.forward(ours)
    torch.cuda.synchronize()
    assert np.array_equal(host(ref_d), host(ours))
    assert R.ref_gpu_launch_intt16(ref_d.data_ptr(), itw_d.data_ptr(), q_d.data_ptr(),
                                   qi_d.data_ptr(), di_d.data_ptr(), 16) == 0
    P.inverse(ours)
    torch.cuda.synchronize()
    assert np.array_equal(host(ref_d), host(ours))
    assert np.array_equal(host(ours), x)


def test_error_paths(torch_cuda, nb):
    torch = torch_cuda
    mods = moduli_set(16, 2, 30)
    P = nb.Plan(16, mods)
    d = torch.zeros(2 * (1 << 16) + 4, dtype=torch.int32, device="cuda")
    with pytest.raises(nb.NttError) as e:
        P.forward(d.data_ptr() + 4)  # 4-byte offset: not 16-byte aligned
    assert e.value.name == "NTT_ERR_MISALIGNED"
    with pytest.raises(nb.NttError) as e:
        P.forward(None)
    assert e.value.name == "NTT_ERR_INVALID_ARGUMENT"
    P.forward_many(d, 0)  # empty batch is a no-op
    info = P.info
    assert info.logN == 16 and info.limbs == 2 and info.cluster_ctas >= 1
