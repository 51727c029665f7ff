"""Python side of the CPU oracle (test infrastructure only).

Loads ``oracle/liboracle.so`` (the C restatement in ``ntt_oracle.c``) and, when
it has been built, ``oracle/_ref/libntt_ref.so`` (the reference's own v04
translation unit, see ``ref_harness.cu``).  Only tests/, the smoke check and
bench.py's CPU-baseline leg import this module; the product never does.

Besides thin wrappers it holds independent pure-Python helpers the tests use
to build moduli chains (deterministic Miller-Rabin for 32-bit integers and the
smallest-generator search) -- the reference hard-codes its moduli
(src/ntt_config.h:75-94) and has no such search.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB: Optional[ctypes.CDLL] = None
_REF: Optional[ctypes.CDLL] = None

_u32p = ctypes.POINTER(ctypes.c_uint32)


class ModulusRuntime(ctypes.Structure):
    """Field order of ModulusRuntime (src/v04_montgomery.cu:17-26)."""

    _fields_ = [(n, ctypes.c_uint32) for n in (
        "qi", "primitive_root", "q_inv", "r2", "psi", "psi_inv", "omega", "degree_inv")]

    def as_tuple(self):
        return tuple(getattr(self, n) for n, _ in self._fields_)


def _ptr(a: np.ndarray):
    assert a.dtype == np.uint32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_u32p)


def ref_root() -> str:
    """The reference checkout: $NTT_REF_ROOT when set, else its location in
    the build container (absent on machines that only run the prebuilt
    harness)."""
    return os.environ.get("NTT_REF_ROOT", "/root/reference")


def build() -> None:
    """Compile liboracle.so (and the reference harness when the reference
    checkout is present)."""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    if os.path.isdir(os.path.join(ref_root(), "src")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF_ROOT={ref_root()}"], check=True)


def lib() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        for name in ("oracle_pow_mod",):
            getattr(L, name).restype = ctypes.c_uint32
            getattr(L, name).argtypes = [ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint32]
        for name in ("oracle_add_mod", "oracle_sub_mod", "oracle_mul_mod", "oracle_from_mont"):
            getattr(L, name).restype = ctypes.c_uint32
            getattr(L, name).argtypes = [ctypes.c_uint32] * 3
        for name in ("oracle_mont_q_inv", "oracle_mont_r2"):
            getattr(L, name).restype = ctypes.c_uint32
            getattr(L, name).argtypes = [ctypes.c_uint32]
        L.oracle_to_mont.restype = ctypes.c_uint32
        L.oracle_to_mont.argtypes = [ctypes.c_uint32, ctypes.c_uint32]
        L.oracle_mont_mul.restype = ctypes.c_uint32
        L.oracle_mont_mul.argtypes = [ctypes.c_uint32] * 4
        L.oracle_bit_reverse.restype = ctypes.c_uint32
        L.oracle_bit_reverse.argtypes = [ctypes.c_uint32, ctypes.c_int]
        L.oracle_modulus_runtime.restype = ctypes.c_int
        L.oracle_modulus_runtime.argtypes = [ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32,
                                             ctypes.POINTER(ModulusRuntime)]
        L.oracle_twiddle_table.argtypes = [ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32, _u32p]
        L.oracle_ntt.argtypes = [_u32p, ctypes.c_int, ctypes.c_uint32, _u32p]
        L.oracle_intt.argtypes = [_u32p, ctypes.c_int, ctypes.c_uint32, _u32p, ctypes.c_uint32]
        L.oracle_ntt_direct.argtypes = [_u32p, _u32p, ctypes.c_int, ctypes.c_uint32,
                                        ctypes.c_uint32]
        L.oracle_negacyclic_coeff.restype = ctypes.c_uint32
        L.oracle_negacyclic_coeff.argtypes = [_u32p, _u32p, ctypes.c_int, ctypes.c_uint32,
                                              ctypes.c_size_t]
        L.oracle_fill_random.restype = ctypes.c_int
        L.oracle_fill_random.argtypes = [_u32p, ctypes.c_size_t, ctypes.c_uint32,
                                         ctypes.c_uint32]
        L.oracle_transform_limbs.restype = ctypes.c_int
        L.oracle_transform_limbs.argtypes = [_u32p, ctypes.c_int, ctypes.c_int, _u32p, _u32p,
                                             _u32p, ctypes.c_int]
        _LIB = L
    return _LIB


def ref_lib() -> Optional[ctypes.CDLL]:
    """The reference's own compiled functions, or None when not built."""
    global _REF
    if _REF is None:
        path = os.path.join(HERE, "_ref", "libntt_ref.so")
        if not os.path.exists(path):
            return None
        R = ctypes.CDLL(path)
        R.ref_modulus_runtime.argtypes = [ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32, _u32p]
        R.ref_twiddle_table.argtypes = [ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32, _u32p]
        R.ref_fill_random.argtypes = [_u32p, ctypes.c_size_t, ctypes.c_uint32]
        R.ref_to_mont.restype = ctypes.c_uint32
        R.ref_to_mont.argtypes = [ctypes.c_uint32, ctypes.c_uint32]
        R.ref_from_mont.restype = ctypes.c_uint32
        R.ref_from_mont.argtypes = [ctypes.c_uint32] * 3
        R.ref_cpu_ntt.argtypes = [_u32p, ctypes.c_int, ctypes.c_uint32, _u32p]
        R.ref_cpu_intt.argtypes = [_u32p, ctypes.c_int, ctypes.c_uint32, _u32p, ctypes.c_uint32]
        R.ref_cpu_transform_limbs.argtypes = [_u32p, ctypes.c_int, ctypes.c_int, _u32p, _u32p,
                                              _u32p, ctypes.c_int]
        for n in ("ref_gpu_launch_ntt16", "ref_gpu_launch_intt16"):
            getattr(R, n).restype = ctypes.c_int
            getattr(R, n).argtypes = [ctypes.c_void_p] * 5 + [ctypes.c_size_t]
        R.ref_gpu_time16.restype = ctypes.c_int
        R.ref_gpu_time16.argtypes = ([ctypes.c_void_p] * 8 + [ctypes.c_size_t, ctypes.c_int,
                                     ctypes.c_int] + [ctypes.POINTER(ctypes.c_float)] * 2)
        _REF = R
    return _REF


# ---------------------------------------------------------------------------
# scalar helpers and per-limb precompute
# ---------------------------------------------------------------------------

def modulus_runtime(logN: int, q: int, g: int):
    """(status, ModulusRuntime) -- make_modulus_runtime (v04:681-718) with a
    status code instead of std::exit (1: q != 1 mod 2N, 2: bad root)."""
    out = ModulusRuntime()
    st = lib().oracle_modulus_runtime(logN, q, g, ctypes.byref(out))
    return st, out


def twiddle_table(logN: int, q: int, psi: int) -> np.ndarray:
    out = np.empty(1 << logN, dtype=np.uint32)
    lib().oracle_twiddle_table(logN, q, psi, _ptr(out))
    return out


def to_mont_array(x: np.ndarray, q: int) -> np.ndarray:
    r = (1 << 32) % q
    return ((x.astype(np.uint64) * np.uint64(r)) % np.uint64(q)).astype(np.uint32)


def from_mont_array(x: np.ndarray, q: int) -> np.ndarray:
    rinv = pow(1 << 32, -1, q)
    return ((x.astype(np.uint64) % np.uint64(q)) * np.uint64(rinv) % np.uint64(q)).astype(np.uint32)


class LimbTables:
    """Host tables for one (logN, moduli) configuration, as the reference's
    main() builds them (v04:892-916)."""

    def __init__(self, logN: int, moduli: Sequence[tuple]):
        self.logN = logN
        self.N = 1 << logN
        self.moduli = [(int(q), int(g)) for q, g in moduli]
        self.rt = []
        L = len(self.moduli)
        self.q = np.array([q for q, _ in self.moduli], dtype=np.uint32)
        self.psi_tab = np.empty((L, self.N), dtype=np.uint32)
        self.inv_tab = np.empty((L, self.N), dtype=np.uint32)
        for i, (q, g) in enumerate(self.moduli):
            st, rt = modulus_runtime(logN, q, g)
            if st != 0:
                raise ValueError(f"invalid modulus/root ({q}, {g}) for logN={logN}: status {st}")
            self.rt.append(rt)
            lib().oracle_twiddle_table(logN, q, rt.psi, _ptr(self.psi_tab[i]))
            lib().oracle_twiddle_table(logN, q, rt.psi_inv, _ptr(self.inv_tab[i]))
        self.degree_inv = np.array([r.degree_inv for r in self.rt], dtype=np.uint32)
        self.q_inv = np.array([r.q_inv for r in self.rt], dtype=np.uint32)
        self.r2 = np.array([r.r2 for r in self.rt], dtype=np.uint32)
        self.degree_inv_mont = np.array(
            [(int(d) * ((1 << 32) % q)) % q for d, (q, _) in zip(self.degree_inv, self.moduli)],
            dtype=np.uint32)

    def mont_tables(self):
        """Montgomery-form copies, as uploaded to the device (v04:910-914)."""
        tw = np.stack([to_mont_array(self.psi_tab[i], q) for i, (q, _) in enumerate(self.moduli)])
        itw = np.stack([to_mont_array(self.inv_tab[i], q) for i, (q, _) in enumerate(self.moduli)])
        return tw, itw

    def forward(self, a: np.ndarray, threads: int = 1) -> np.ndarray:
        """Limb-major a[limb, N] -> cpu_ntt_butterfly per limb (normal domain,
        bit-reversed order)."""
        out = np.ascontiguousarray(a, dtype=np.uint32).copy()
        lib().oracle_transform_limbs(_ptr(out), self.logN, len(self.moduli), _ptr(self.q),
                                     _ptr(self.psi_tab), None, threads)
        return out

    def inverse(self, a: np.ndarray, threads: int = 1) -> np.ndarray:
        out = np.ascontiguousarray(a, dtype=np.uint32).copy()
        lib().oracle_transform_limbs(_ptr(out), self.logN, len(self.moduli), _ptr(self.q),
                                     _ptr(self.inv_tab), _ptr(self.degree_inv), threads)
        return out

    def forward_mont(self, a: np.ndarray, threads: int = 1) -> np.ndarray:
        """What the v04 GPU forward writes: the CPU NTT in Montgomery form
        (the --verify path compares after from_mont, v04:1081-1087)."""
        f = self.forward(a, threads)
        return np.stack([to_mont_array(f[i], q) for i, (q, _) in enumerate(self.moduli)])

    def inverse_from_mont(self, a_mont: np.ndarray, threads: int = 1) -> np.ndarray:
        """The v04 GPU INTT contract: Montgomery-domain input, normal output."""
        a = np.stack([from_mont_array(a_mont[i], q) for i, (q, _) in enumerate(self.moduli)])
        return self.inverse(a, threads)


def fill_random_ref_compatible(logN: int, moduli_q: Sequence[int], seed: int = 1234) -> np.ndarray:
    """The reference's input: fill_random per limb, re-seeded with `seed` for
    every limb (v04:786-797, v04:932-934)."""
    N = 1 << logN
    out = np.empty((len(moduli_q), N), dtype=np.uint32)
    for i, q in enumerate(moduli_q):
        lib().oracle_fill_random(_ptr(out[i]), N, int(q), seed)
    return out


def uniform_limbs(logN: int, moduli_q: Sequence[int], seed: int) -> np.ndarray:
    """Fast seeded uniform [0, q) coefficients per limb (numpy PCG64)."""
    rng = np.random.default_rng(seed)
    N = 1 << logN
    q = np.asarray(moduli_q, dtype=np.uint64)[:, None]
    return rng.integers(0, q, size=(len(moduli_q), N), dtype=np.uint64).astype(np.uint32)


def ntt_direct(a: np.ndarray, logN: int, q: int, psi: int) -> np.ndarray:
    out = np.empty(1 << logN, dtype=np.uint32)
    lib().oracle_ntt_direct(_ptr(np.ascontiguousarray(a, dtype=np.uint32)), _ptr(out), logN, q, psi)
    return out


def negacyclic_coeff(a: np.ndarray, b: np.ndarray, logN: int, q: int, k: int) -> int:
    a = np.ascontiguousarray(a, dtype=np.uint32)
    b = np.ascontiguousarray(b, dtype=np.uint32)
    return int(lib().oracle_negacyclic_coeff(_ptr(a), _ptr(b), logN, q, k))


# ---------------------------------------------------------------------------
# moduli chains (pure Python, independent of the product's own search)
# ---------------------------------------------------------------------------

def is_prime_u32(n: int) -> bool:
    if n < 2:
        return False
    for p in (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37):
        if n % p == 0:
            return n == p
    d, s = n - 1, 0
    while d % 2 == 0:
        d //= 2
        s += 1
    for a in (2, 7, 61):  # deterministic for n < 4,759,123,141
        x = pow(a, d, n)
        if x in (1, n - 1):
            continue
        for _ in range(s - 1):
            x = x * x % n
            if x == n - 1:
                break
        else:
            return False
    return True


def _factor_distinct(n: int):
    f, p = [], 2
    while p * p <= n:
        if n % p == 0:
            f.append(p)
            while n % p == 0:
                n //= p
        p += 1 if p == 2 else 2
    if n > 1:
        f.append(n)
    return f


def smallest_generator(q: int) -> int:
    fs = _factor_distinct(q - 1)
    g = 2
    while True:
        if all(pow(g, (q - 1) // f, q) != 1 for f in fs):
            return g
        g += 1


def ascending_primes(logN: int, count: int, start: int):
    """The first `count` primes q >= start with q == 1 (mod 2N), ascending,
    each with its smallest generator."""
    step = 2 << logN
    q = start + ((1 - start) % step)
    out = []
    while len(out) < count:
        if q >= 1 << 31:
            raise ValueError("ran out of 31-bit primes")
        if is_prime_u32(q):
            out.append((q, smallest_generator(q)))
        q += step
    return out


# The reference's default_moduli() (src/ntt_config.h:75-94), restated as data.
REFERENCE_DEFAULT_MODULI = [
    (974258177, 3), (1081212929, 6), (1196556289, 7), (993263617, 5),
    (989986817, 3), (1074266113, 5), (1168900097, 5), (1010565121, 7),
    (957349889, 6), (1073872897, 7), (1209139201, 31), (994705409, 3),
    (998244353, 3), (1073479681, 11), (1158676481, 3), (1016463361, 38),
]


# ---- 64-bit words (oracle for the 64-bit variant) ----------------------------

_u64p = ctypes.POINTER(ctypes.c_uint64)


def _p64(a: np.ndarray):
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_u64p)


def _lib64():
    L = lib()
    if not getattr(L, "_sig64", False):
        L.oracle_mul_mod64.restype = ctypes.c_uint64
        L.oracle_mul_mod64.argtypes = [ctypes.c_uint64] * 3
        L.oracle_pow_mod64.restype = ctypes.c_uint64
        L.oracle_pow_mod64.argtypes = [ctypes.c_uint64] * 3
        L.oracle_tables64.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_uint64, _u64p, _u64p,
                                      _u64p]
        L.oracle_ntt64.argtypes = [_u64p, ctypes.c_int, ctypes.c_uint64, _u64p]
        L.oracle_intt64.argtypes = [_u64p, ctypes.c_int, ctypes.c_uint64, _u64p, ctypes.c_uint64]
        L.oracle_ntt_direct64.argtypes = [_u64p, _u64p, ctypes.c_int, ctypes.c_uint64,
                                          ctypes.c_uint64]
        L._sig64 = True
    return L


class LimbTables64:
    """Per-limb 64-bit tables and the CPU transforms of the 64-bit variant:
    forward_mont (CPU NTT, then x * 2^64 mod q) and its inverse."""

    def __init__(self, logN: int, moduli: Sequence):
        L = _lib64()
        self.logN, self.moduli = logN, [(int(q), int(g)) for q, g in moduli]
        N = 1 << logN
        self.q = np.array([q for q, _ in self.moduli], dtype=np.uint64)
        self.psi_tab = np.zeros((len(moduli), N), dtype=np.uint64)
        self.inv_tab = np.zeros((len(moduli), N), dtype=np.uint64)
        self.degree_inv = []
        for i, (q, g) in enumerate(self.moduli):
            di = ctypes.c_uint64()
            L.oracle_tables64(logN, q, g, _p64(self.psi_tab[i]), _p64(self.inv_tab[i]),
                              ctypes.byref(di))
            self.degree_inv.append(di.value)
        self.psi = [pow(g, (q - 1) // (2 * N), q) for q, g in self.moduli]

    def forward(self, a: np.ndarray) -> np.ndarray:
        out = np.ascontiguousarray(a, dtype=np.uint64).copy()
        for i, (q, _) in enumerate(self.moduli):
            _lib64().oracle_ntt64(_p64(out[i]), self.logN, q, _p64(self.psi_tab[i]))
        return out

    def inverse(self, a: np.ndarray) -> np.ndarray:
        out = np.ascontiguousarray(a, dtype=np.uint64).copy()
        for i, (q, _) in enumerate(self.moduli):
            _lib64().oracle_intt64(_p64(out[i]), self.logN, q, _p64(self.inv_tab[i]),
                                   self.degree_inv[i])
        return out

    def direct(self, a: np.ndarray) -> np.ndarray:
        out = np.zeros_like(a, dtype=np.uint64)
        for i, (q, _) in enumerate(self.moduli):
            row = np.ascontiguousarray(a[i], dtype=np.uint64)
            _lib64().oracle_ntt_direct64(_p64(row), _p64(out[i]), self.logN, q, self.psi[i])
        return out

    def forward_mont(self, a: np.ndarray) -> np.ndarray:
        f = self.forward(a)
        return np.stack([np.array([(int(v) << 64) % q for v in f[i]], dtype=np.uint64)
                         for i, (q, _) in enumerate(self.moduli)])

    def to_mont(self, a: np.ndarray) -> np.ndarray:
        return np.stack([np.array([(int(v) << 64) % q for v in a[i]], dtype=np.uint64)
                         for i, (q, _) in enumerate(self.moduli)])


def primes64(logN: int, count: int, start: int):
    """Ascending primes q >= start, q == 1 mod 2N, q < 2^62, each with its
    smallest quadratic non-residue (Miller-Rabin with the first 12 primes as
    bases: deterministic below 3.3e24)."""
    def is_prime(n):
        if n < 2:
            return False
        bases = (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37)
        for p in bases:
            if n % p == 0:
                return n == p
        d, s = n - 1, 0
        while d % 2 == 0:
            d //= 2
            s += 1
        for a in bases:
            x = pow(a, d, n)
            if x in (1, n - 1):
                continue
            for _ in range(s - 1):
                x = x * x % n
                if x == n - 1:
                    break
            else:
                return False
        return True
    step = 2 << logN
    q = ((max(start, 2) - 2) // step + 1) * step + 1
    out = []
    while len(out) < count:
        if is_prime(q):
            g = 2
            while pow(g, (q - 1) // 2, q) != q - 1:
                g += 1
            out.append((q, g))
        q += step
    return out
