"""Index maps of every compiled fused-kernel configuration, checked on the CPU.

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
from twiddle_ref import device_tables

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
