"""The CPU oracle pinned against the reference's own code.

Checks oracle/ntt_oracle.c (the C restatement) against the golden fixtures
produced by the reference's compiled host functions (tests/golden/), against
the reference harness itself when it is built, and against independent
known-answer checks (direct O(N^2) evaluation, schoolbook negacyclic product).
"""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.uint32).tobytes()).hexdigest()


@pytest.mark.parametrize("case", [c for c in GOLD["cases"] if "sha256" in c], ids=lambda c: c["name"])
def test_oracle_matches_reference_digests(case):
    logN, mods = case["logN"], [tuple(m) for m in case["moduli"]]
    T = O.LimbTables(logN, mods)
    assert [list(r.as_tuple()) for r in T.rt] == case["runtime"]
    x = O.fill_random_ref_compatible(logN, T.q, 1234)
    f = T.forward(x, threads=8)
    fm = T.forward_mont(x, threads=8)
    rt = T.inverse(f, threads=8)
    s = case["sha256"]
    assert sha(x) == s["input"]
    assert sha(T.psi_tab) == s["twiddles"]
    assert sha(T.inv_tab) == s["inv_twiddles"]
    assert sha(f) == s["ntt"]
    assert sha(fm) == s["ntt_mont"]
    assert sha(rt) == s["roundtrip"]
    assert np.array_equal(rt, x)  # the CPU roundtrip is the identity
    smp = case["samples"]
    assert x[0, :8].tolist() == smp["input_limb0"]
    assert f[0, :8].tolist() == smp["ntt_limb0"]
    assert f[-1, :8].tolist() == smp["ntt_limb_last"]


@pytest.mark.parametrize("case", [c for c in GOLD["cases"] if "full" in c], ids=lambda c: c["name"])
def test_oracle_matches_reference_small_vectors(case):
    logN, (q, g) = case["logN"], tuple(case["moduli"][0])
    T = O.LimbTables(logN, [(q, g)])
    full = case["full"]
    x = np.array([full["input"]], dtype=np.uint32)
    assert O.fill_random_ref_compatible(logN, [q], 1234)[0].tolist() == full["input"]
    assert T.psi_tab[0].tolist() == full["twiddles"]
    assert T.inv_tab[0].tolist() == full["inv_twiddles"]
    assert T.forward(x)[0].tolist() == full["ntt"]
    assert T.forward_mont(x)[0].tolist() == full["ntt_mont"]
    assert T.inverse(T.forward(x))[0].tolist() == full["roundtrip"]


def test_survey_known_answers():
    """Values recorded when the reference was first run in this container."""
    st, rt = O.modulus_runtime(16, 974258177, 3)
    assert st == 0
    assert (rt.psi, rt.psi_inv, rt.degree_inv, rt.q_inv, rt.r2) == (
        478732885, 718772821, 974243311, 974258175, 850126382)
    assert int(O.twiddle_table(16, 974258177, rt.psi)[1]) == 756671896
    x = O.fill_random_ref_compatible(16, [974258177], 1234)
    assert x[0, :4].tolist() == [186589390, 484852896, 606094552, 796785790]


@pytest.mark.parametrize("logN", [1, 2, 3, 5, 7, 9])
@pytest.mark.parametrize("start", [int(2 ** 29.5), int(2 ** 30.5)])
def test_oracle_equals_direct_evaluation(logN, start):
    (q, g), = O.ascending_primes(logN, 1, start)
    T = O.LimbTables(logN, [(q, g)])
    x = O.uniform_limbs(logN, [q], 11)
    assert np.array_equal(T.forward(x)[0], O.ntt_direct(x[0], logN, q, T.rt[0].psi))


@pytest.mark.parametrize("logN", [3, 6, 10])
def test_oracle_negacyclic_product(logN):
    """INTT(NTT(a) * NTT(b)) equals the schoolbook product mod (X^N + 1, q)."""
    (q, g), = O.ascending_primes(logN, 1, int(2 ** 29.5))
    T = O.LimbTables(logN, [(q, g)])
    a = O.uniform_limbs(logN, [q], 1)
    b = O.uniform_limbs(logN, [q], 2)
    fa, fb = T.forward(a), T.forward(b)
    prod = (fa.astype(np.uint64) * fb.astype(np.uint64) % np.uint64(q)).astype(np.uint32)
    c = T.inverse(prod)
    N = 1 << logN
    for k in sorted({0, 1, N // 2, N - 1}):
        assert c[0, k] == O.negacyclic_coeff(a[0], b[0], logN, q, k)


def test_oracle_error_codes():
    # q != 1 mod 2N  (the reference exits, v04:685-689)
    assert O.modulus_runtime(16, 974258177 + 2, 3)[0] == 1
    # a non-generator gives a psi that is not a primitive 2N-th root (v04:703-707)
    assert O.modulus_runtime(16, 974258177, 1)[0] == 2


def test_oracle_against_reference_harness():
    R = O.ref_lib()
    if R is None:
        pytest.skip("reference harness not built (needs the reference checkout)")
    for logN in (11, 13, 17):
        mods = O.ascending_primes(logN, 3, int(2 ** 30.5))
        T = O.LimbTables(logN, mods)
        x = O.uniform_limbs(logN, T.q, 3)
        ref = x.copy()
        R.ref_cpu_transform_limbs(O._ptr(ref), logN, 3, O._ptr(T.q), O._ptr(T.psi_tab), None, 3)
        assert np.array_equal(ref, T.forward(x))
        ref2 = ref.copy()
        R.ref_cpu_transform_limbs(O._ptr(ref2), logN, 3, O._ptr(T.q), O._ptr(T.inv_tab),
                                  O._ptr(T.degree_inv), 3)
        assert np.array_equal(ref2, T.inverse(ref))


@pytest.mark.parametrize("logN", [1, 4, 9])
def test_oracle64_matches_definition_and_roundtrips(logN):
    """The 64-bit restatement (CT / GS loops with 128-bit products) equals the
    O(N^2) evaluation of the bit-reversed negacyclic transform, and the
    inverse undoes it."""
    mods = O.primes64(logN, 3, (1 << 61) + 12345)
    T = O.LimbTables64(logN, mods)
    rng = np.random.default_rng(logN)
    x = np.stack([rng.integers(0, int(q), 1 << logN, dtype=np.uint64) for q in T.q])
    f = T.forward(x)
    assert np.array_equal(f, T.direct(x))
    assert np.array_equal(T.inverse(f), x)
