"""The C ABI without a GPU: the library loads, exports every declared entry
point, and its host-side precompute matches the oracle and the reference's
error behaviour (status codes where the reference exits)."""
import os
import re

import numpy as np
import pytest

import ntt_b200 as nb
from oracle import oracle as O

INCLUDE = os.path.join(os.path.dirname(__file__), "..", "include")


def declared_symbols():
    names = set()
    for fn in os.listdir(INCLUDE):
        if fn.endswith(".h"):
            src = open(os.path.join(INCLUDE, fn)).read()
            names |= set(re.findall(r"^NTT_API [^(]*?\b(ntt\w+)\(", src, re.M))
    return sorted(names)


def test_every_declared_symbol_is_exported():
    syms = declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(nb._lib, s), s


def test_version_and_status_strings():
    assert nb.version() == 100
    for code in nb.STATUS_NAMES:
        assert nb._lib.ntt_status_string(code)


def test_default_moduli_is_reference_list():
    assert [tuple(m) for m in nb.default_moduli()] == O.REFERENCE_DEFAULT_MODULI


def test_default_transform_matches_default_launch_config():
    t = nb.default_transform(16)
    assert t.ntt_phase1.as_tuple() == (7, 4, 4) and t.intt_phase2.as_tuple() == (7, 4, 4)
    assert t.ntt_phase2.as_tuple() == (9, 3, 0) and t.intt_phase1.as_tuple() == (9, 3, 0)
    t = nb.default_transform(12)
    assert t.ntt_phase1.as_tuple() == (3, 3, 4)
    with pytest.raises(nb.NttError) as e:
        nb.default_transform(9)  # static_assert(LogN >= 10) in the reference
    assert e.value.name == "NTT_ERR_UNSUPPORTED"


@pytest.mark.parametrize("logN", [1, 10, 16, 17])
def test_modulus_runtime_matches_oracle(logN):
    for q, g in O.REFERENCE_DEFAULT_MODULI[:6] if logN <= 16 else O.ascending_primes(17, 4, 1 << 30):
        rt = nb.modulus_runtime(logN, (q, g))
        st, ort = O.modulus_runtime(logN, q, g)
        assert st == 0
        assert tuple(getattr(rt, n) for n, _ in rt._fields_) == ort.as_tuple()


def test_modulus_errors_mirror_reference_exits():
    with pytest.raises(nb.NttError) as e:
        nb.modulus_runtime(16, (974258177 + 2, 3))
    assert e.value.name == "NTT_ERR_MODULUS"
    with pytest.raises(nb.NttError) as e:
        nb.modulus_runtime(16, (974258177, 1))
    assert e.value.name == "NTT_ERR_ROOT"
    with pytest.raises(nb.NttError) as e:  # even q: fails the congruence, as in v04
        nb.modulus_runtime(4, (64, 3))
    assert e.value.name == "NTT_ERR_MODULUS"
    with pytest.raises(nb.NttError) as e:  # composite q == 1 mod 2N
        nb.modulus_runtime(4, (33 * 32 + 1, 3))
    assert e.value.name in ("NTT_ERR_MODULUS_RANGE", "NTT_ERR_ROOT")
    with pytest.raises(nb.NttError) as e:  # 32-bit prime: beyond the 2^31 bound
        q = next(q for q in range((1 << 31) + 1, (1 << 32), 1 << 17) if O.is_prime_u32(q))
        nb.modulus_runtime(16, (q, O.smallest_generator(q)))
    assert e.value.name == "NTT_ERR_MODULUS_RANGE"


@pytest.mark.parametrize("logN", [2, 9, 16])
def test_twiddle_table_matches_oracle(logN):
    q, g = O.ascending_primes(logN, 1, int(2 ** 30.5))[0]
    _, rt = O.modulus_runtime(logN, q, g)
    assert np.array_equal(nb.twiddle_table(logN, q, rt.psi), O.twiddle_table(logN, q, rt.psi))


@pytest.mark.parametrize("logN,count,start", [(16, 16, 974258177), (17, 8, int(2 ** 29.5)),
                                              (12, 64, int(2 ** 30.5))])
def test_find_moduli_matches_oracle(logN, count, start):
    got = [tuple(m) for m in nb.find_moduli(logN, count, start)]
    assert got == O.ascending_primes(logN, count, start)


def test_config_catalogue_covers_every_size():
    cfgs = nb.kernel_configs()
    assert {c.logN for c in cfgs} == set(range(10, 18))
    for c in cfgs:
        assert c.threads in (32, 64, 128, 256, 512, 1024)
        assert c.smem_bytes <= 227 * 1024
        assert c.cluster_ctas in (1, 2, 4, 8, 16)
        assert c.polys_per_job in (1, 2)
        assert c.exchange in (0, 1)
        if c.exchange:  # split: one phase-1 pass per column, 2 or 3 phase-2 passes
            assert c.k1a == c.r1 == c.words_log2 and c.polys_per_job == 1
            k2c = c.logN - c.r1 - c.k2a - c.k2b
            assert 1 <= c.k2a <= c.words_log2 and 1 <= c.k2b <= c.words_log2
            assert 0 <= k2c <= c.words_log2
    assert any(c.polys_per_job == 2 for c in cfgs)
    assert {c.logN for c in cfgs if c.exchange} >= {15, 16, 17}


def test_plan_without_device_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with pytest.raises(nb.NttError) as e:
        nb.Plan(12, O.ascending_primes(12, 2, 1 << 29))
    assert e.value.name in ("NTT_ERR_CUDA", "NTT_ERR_OUT_OF_MEMORY")


def test_invalid_plan_arguments():
    with pytest.raises(nb.NttError) as e:
        nb.Plan(18, [(974258177, 3)])
    assert e.value.name == "NTT_ERR_UNSUPPORTED"
    with pytest.raises(nb.NttError) as e:
        nb.Plan(16, [])
    assert e.value.name == "NTT_ERR_INVALID_ARGUMENT"
    bad = nb.default_transform(16)
    bad.ntt_phase2.radix_stages = 8  # 7 + 8 != 16
    with pytest.raises(nb.NttError) as e:
        nb.Plan(16, [(974258177, 3)], bad)
    assert e.value.name == "NTT_ERR_INVALID_ARGUMENT"


def test_batch_job_validation_without_device():
    """Job-level checks run before any device call (status codes, no exit)."""
    mods = [(m.qi, m.primitive_root) for m in nb.find_moduli(12, 2, 1 << 29)]
    cases = [
        ((7, 12, mods, 0x1000, None), "NTT_ERR_INVALID_ARGUMENT"),    # unknown op
        ((nb.OP_FORWARD, 11, mods, 0x1000, None), "NTT_ERR_UNSUPPORTED"),
        ((nb.OP_FORWARD, 18, mods, 0x1000, None), "NTT_ERR_UNSUPPORTED"),
        ((nb.OP_FORWARD, 12, [], 0x1000, None), "NTT_ERR_INVALID_ARGUMENT"),
        ((nb.OP_FORWARD, 12, mods, 0x1004, None), "NTT_ERR_MISALIGNED"),
        ((nb.OP_MULTIPLY, 12, mods, 0x1000, None), "NTT_ERR_INVALID_ARGUMENT"),
        ((nb.OP_MULTIPLY, 12, mods, 0x1000, 0x2008), "NTT_ERR_MISALIGNED"),
    ]
    for job, name in cases:
        with pytest.raises(nb.NttError) as e:
            nb.Batch([job])
        assert e.value.name == name, job
    with pytest.raises(nb.NttError) as e:
        nb.Batch([(nb.OP_FORWARD, 12, mods, 0x1000, None)], cluster_ctas=4)
    assert e.value.name == "NTT_ERR_INVALID_ARGUMENT"


def test_ragged_mix_is_seeded():
    from ntt_b200 import mixes
    a = mixes.ragged_mix(seed=3, count=50, logn=range(12, 17), limbs=(1, 48))
    b = mixes.ragged_mix(seed=3, count=50, logn=range(12, 17), limbs=(1, 48))
    assert [(j.op, j.logN, j.moduli) for j in a] == [(j.op, j.logN, j.moduli) for j in b]
    for j in a:
        assert 12 <= j.logN <= 16 and 1 <= j.limbs <= 48
        qs = [q for q, _ in j.moduli]
        assert qs == sorted(qs) and len(set(qs)) == len(qs)
        for q, g in j.moduli:
            assert (q - 1) % (2 << j.logN) == 0 and (1 << 29) < q < (1 << 30)
    assert len({tuple(j.moduli) for j in a}) > 40  # chains differ between polynomials


def test_server_and_batch_without_device_fail_cleanly():
    with pytest.raises(nb.NttError) as e:
        nb.Server(hbm_budget_bytes=1 << 20)
    assert e.value.name in ("NTT_ERR_CUDA", "NTT_ERR_OUT_OF_MEMORY")
    with pytest.raises(nb.NttError) as e:
        nb.Server(streams=-1)
    assert e.value.name == "NTT_ERR_INVALID_ARGUMENT"
    assert nb.tables_device_bytes() == 0


@pytest.mark.parametrize("logN,count,start", [(12, 3, 1 << 59), (16, 4, 1 << 60), (17, 2, 3 << 60)])
def test_find_moduli64_matches_oracle(logN, count, start):
    got = [tuple(m) for m in nb.find_moduli64(logN, count, start)]
    assert got == O.primes64(logN, count, start)
    for q, g in got:
        assert q < 1 << 62 and (q - 1) % (2 << logN) == 0


def test_plan64_validation_without_device():
    import torch
    mods = O.primes64(12, 1, 1 << 59)
    cases = [([(mods[0][0] + 2, 3)], "NTT_ERR_MODULUS"),          # not 1 mod 2N
             ([((1 << 62) + (2 << 12) + 1, 3)], None),             # >= 2^62 (and maybe not 1 mod 2N)
             ([(mods[0][0], 1)], "NTT_ERR_ROOT")]                  # 1 is a residue
    for m, want in cases:
        with pytest.raises(nb.NttError) as e:
            nb.Plan64(12, m)
        if want:
            assert e.value.name == want
        elif torch.cuda.is_available():
            assert e.value.name in ("NTT_ERR_MODULUS", "NTT_ERR_MODULUS_RANGE")
    with pytest.raises(nb.NttError) as e:
        nb.Plan64(18, mods)
    assert e.value.name == "NTT_ERR_UNSUPPORTED"


def test_new_entry_points_validate_before_device_work():
    """Argument checks of the RNS steps, the spectrum product, compressed
    plans and the small-kernel knob run before any CUDA call (no GPU
    needed): NULL plans, unknown plan flags, compressed tables below logN 15."""
    import ctypes
    lib = nb._lib
    null = ctypes.c_void_p(0)
    calls = {
        "ntt_forward_skip": lambda: lib.ntt_forward_skip(null, null, 1, 0, 0, 1, null),
        "ntt_forward_sub_scale": lambda: lib.ntt_forward_sub_scale(null, null, 1, 0, null, 0, 0, 0,
                                                                   null, null, null),
        "ntt_inverse_scaled_range": lambda: lib.ntt_inverse_scaled_range(null, null, 1, 0, 0, 1,
                                                                         null, null),
        "ntt_multiply_spectrum_many": lambda: lib.ntt_multiply_spectrum_many(null, null, null, 1, 0,
                                                                             null),
        "ntt_plan_set_small_kernel": lambda: lib.ntt_plan_set_small_kernel(null, 0),
    }
    for name, call in calls.items():
        assert nb.STATUS_NAMES[call()] == "NTT_ERR_INVALID_ARGUMENT", name
    m = [(974258177, 3)]
    arr, n = nb._moduli_array(m)
    h = ctypes.c_void_p()
    st = lib.ntt_plan_create_ex(16, arr, n, None, 0x80, ctypes.byref(h))
    assert nb.STATUS_NAMES[st] == "NTT_ERR_INVALID_ARGUMENT"  # unknown flag
    mods14 = O.ascending_primes(14, 1, 1 << 29)
    with pytest.raises(nb.NttError) as e:
        nb.Plan(14, mods14, compressed_twiddles=True)
    assert e.value.name == "NTT_ERR_UNSUPPORTED"
