"""Index maps of every compiled fused-kernel and split-kernel configuration,
checked on the CPU.

tests/emu/libntt_emu.so runs the device kernels' pass functions
(ntt_b200/csrc/ntt_core.cuh) thread by thread on the host.  Each
configuration, with staged (bulk-copied) and direct (global-memory) input,
must reproduce the oracle bit for bit (forward and inverse, 30- and 31-bit
moduli), never access out of bounds, cover the stage buffer and every
written word exactly once, read only its own warp's words after a warp
barrier, and keep warp-wide shared-memory bank conflicts at most 4-way.
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O
from twiddle_ref import COMP_MIN_LOGN, compressed_tables, device_tables

EMU_DIR = os.path.join(os.path.dirname(__file__), "emu")


@pytest.fixture(scope="module")
def emu():
    subprocess.run(["make", "-s", "-C", EMU_DIR], check=True, capture_output=True)
    E = ctypes.CDLL(os.path.join(EMU_DIR, "libntt_emu.so"))
    E.emu_transform.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    E.emu_last_error.restype = ctypes.c_char_p
    return E


def configs():
    # parsed from the same X-list the library compiles
    import re
    src = open(os.path.join(os.path.dirname(__file__), "..", "ntt_b200", "csrc", "configs.h")).read()
    body = src.split("#define NTTB_CFG_ALL")[0]
    return [tuple(int(v) for v in m) for m in
            re.findall(r"X\((\d+), (\d+), (\d+), (\d+), (\d+), (\d+), (\d+)\)", body)]


@pytest.mark.parametrize("idx,cfg", list(enumerate(configs())), ids=lambda v: str(v))
@pytest.mark.parametrize("bits", [30, 31])
@pytest.mark.parametrize("direct", [0, 2], ids=["staged", "direct"])
def test_config_matches_oracle(emu, idx, cfg, bits, direct):
    if cfg[6] > 1 and direct == 0:
        pytest.skip("several polynomials per job: no staged form (its staged entry is the direct run)")
    c = (ctypes.c_int * 9)()
    emu.emu_config(idx, c)
    assert tuple(c)[:7] == cfg
    logN = cfg[0]
    start = int(2 ** 29.5) if bits == 30 else int(2 ** 30.5)
    mods = O.ascending_primes(logN, 2, start)
    T = O.LimbTables(logN, mods)
    fwd, inv = device_tables(T)
    x = O.uniform_limbs(logN, T.q, 100 + idx)
    x[0, :4] = [0, 1, T.q[0] - 1, 0xFFFFFFFF]  # edge values (forward reduces any uint32)
    d = x.copy()
    st = (ctypes.c_double * 2)()
    rc = emu.emu_transform(idx, 1 | direct, d.ctypes.data, fwd.ctypes.data, T.q.ctypes.data, 2, st)
    assert rc == 0, emu.emu_last_error().decode()
    assert np.array_equal(d, T.forward_mont(x))
    assert st[0] <= 4  # worst warp-wide bank conflict degree
    rc = emu.emu_transform(idx, 0 | direct, d.ctypes.data, inv.ctypes.data, T.q.ctypes.data, 2, st)
    assert rc == 0, emu.emu_last_error().decode()
    expect = x.copy()
    expect[0, 3] = 0xFFFFFFFF % T.q[0]
    assert np.array_equal(d, expect)


@pytest.mark.parametrize("idx,cfg", [(i, c) for i, c in enumerate(configs())
                                     if c[0] >= COMP_MIN_LOGN], ids=lambda v: str(v))
@pytest.mark.parametrize("bits", [30, 31])
def test_compressed_twiddles_match_oracle(emu, idx, cfg, bits):
    """The compressed-table butterflies (two Shoup factors in the last four
    stages, aligned and unaligned index paths) over every configuration of
    logN >= 15: bit-exact against the oracle, in bounds, exactly-once."""
    logN = cfg[0]
    start = int(2 ** 29.5) if bits == 30 else int(2 ** 30.5)
    mods = O.ascending_primes(logN, 2, start)
    T = O.LimbTables(logN, mods)
    fwd, inv = compressed_tables(T)
    assert fwd.shape[1] == 3 * (1 << logN) // 16 + 16
    x = O.uniform_limbs(logN, T.q, 300 + idx)
    x[1, :3] = [0, T.q[1] - 1, 0xFFFFFFFF]
    d = x.copy()
    st = (ctypes.c_double * 2)()
    rc = emu.emu_transform(idx, 1 | 4, d.ctypes.data, fwd.ctypes.data, T.q.ctypes.data, 2, st)
    assert rc == 0, emu.emu_last_error().decode()
    assert np.array_equal(d, T.forward_mont(x))
    rc = emu.emu_transform(idx, 0 | 4, d.ctypes.data, inv.ctypes.data, T.q.ctypes.data, 2, st)
    assert rc == 0, emu.emu_last_error().decode()
    expect = x.copy()
    expect[1, 2] = 0xFFFFFFFF % T.q[1]
    assert np.array_equal(d, expect)


def test_compressed_tables_factor_the_full_ones():
    """Every entry of the last four stages is its base entry times its
    unit-step factor (mod q): the identity the compressed layout rests on."""
    for logN in (15, 16, 17):
        mods = O.ascending_primes(logN, 1, int(2 ** 30.5))
        T = O.LimbTables(logN, mods)
        q = T.q[0]
        N = 1 << logN
        for tab in (T.psi_tab[0], T.inv_tab[0]):
            for p in range(4):
                h, f = N >> (p + 1), 16 >> p
                j = np.arange(N >> (p + 1), dtype=np.uint64)
                base = tab[h + (j // f) * f].astype(np.uint64)
                lsb = tab[(j % f)].astype(np.uint64)
                assert np.array_equal((base * lsb) % np.uint64(q), tab[h + j].astype(np.uint64))


def split_configs():
    # the split list in NTTB_SPLIT_ALL order (NTTB_SPLIT_N16, then NTTB_SPLIT_REST)
    import re
    src = open(os.path.join(os.path.dirname(__file__), "..", "ntt_b200", "csrc", "configs.h")).read()
    out = []
    for name in ("NTTB_SPLIT_N16", "NTTB_SPLIT_REST"):
        body = src.split(f"#define {name}(S)")[1].split("#define")[0]
        out += [tuple(int(v) for v in m)
                for m in re.findall(r"S\((\d+), (\d+), (\d+), (\d+), (\d+)\)", body)]
    return out


@pytest.mark.parametrize("idx,cfg", list(enumerate(split_configs())), ids=lambda v: str(v))
@pytest.mark.parametrize("bits", [30, 31])
@pytest.mark.parametrize("compressed", [False, True], ids=["full", "compressed"])
def test_split_config_matches_oracle(emu, idx, cfg, bits, compressed):
    """The split kernels' passes (split_geo.cuh) run thread by thread: phase 1
    in place in global memory, the cluster barrier between steps, the phase-2
    passes in the work buffer.  Bit-exact against the oracle, every access in
    bounds, every word of each pass and phase written exactly once, warp-local
    reads after warp barriers, bank conflicts at most 4-way; full and
    compressed twiddle tables."""
    emu.emu_split_config.argtypes = [ctypes.c_int, ctypes.c_void_p]
    emu.emu_split_transform.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                        ctypes.c_void_p]
    assert emu.emu_num_split() == len(split_configs())
    c = (ctypes.c_int * 7)()
    emu.emu_split_config(idx, c)
    assert tuple(c)[:5] == cfg
    logN = cfg[0]
    start = int(2 ** 29.5) if bits == 30 else int(2 ** 30.5)
    mods = O.ascending_primes(logN, 2, start)
    T = O.LimbTables(logN, mods)
    fwd, inv = compressed_tables(T) if compressed else device_tables(T)
    x = O.uniform_limbs(logN, T.q, 500 + idx)
    x[0, :3] = [0, T.q[0] - 1, 0xFFFFFFFF]
    d = x.copy()
    st = (ctypes.c_double * 2)()
    mode = 4 if compressed else 0
    rc = emu.emu_split_transform(idx, 1 | mode, d.ctypes.data, fwd.ctypes.data, T.q.ctypes.data, 2, st)
    assert rc == 0, emu.emu_last_error().decode()
    assert np.array_equal(d, T.forward_mont(x))
    assert st[0] <= 4
    rc = emu.emu_split_transform(idx, mode, d.ctypes.data, inv.ctypes.data, T.q.ctypes.data, 2, st)
    assert rc == 0, emu.emu_last_error().decode()
    expect = x.copy()
    expect[0, 2] = 0xFFFFFFFF % T.q[0]
    assert np.array_equal(d, expect)
    assert st[0] <= 4
