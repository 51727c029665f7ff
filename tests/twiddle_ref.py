"""Device twiddle-table layout built from the oracle's tables (test helper).

The product's device tables (ntt_b200/csrc/twiddle.cu) hold, per limb, N
(w, w') pairs: w = psi^bitrev(i) (forward) or psi^-bitrev(i) (inverse), w' its
Shoup companion floor(w * 2^32 / q), with entries 0 and 1 replaced by the
constants folded into limb stage 0:
  forward  [0] = R mod q, [1] = psi^bitrev(1) * R   (R = 2^32: Montgomery form)
  inverse  [0] = c = N^-1 * R^-1, [1] = psi^-bitrev(1) * c
For logN >= 10 entry i is stored at slot tw_slot(i) below: the blocks of the
last four stages are interleaved: stage logN-1-p (p = 0..3) starts at
H = N / 2^(p+1) and its entry H + j sits at H + (j % F) * N/32 + j // F with
F = 16 / 2^p.
This module rebuilds that layout from the oracle so the CPU emulator and the
GPU table check have an independent expected value.
"""
import numpy as np

PERM_MIN_LOGN = 10


def tw_slot(i: int, logN: int) -> int:
    if logN < PERM_MIN_LOGN:
        return i
    N = 1 << logN
    for p in range(4):
        h, f = N >> (p + 1), 16 >> p
        if i >= h:
            return h + ((i - h) % f) * (N // 32) + (i - h) // f
    return i


def _pair(w: int, q: int):
    return (w % q, ((w % q) << 32) // q)


def device_tables(T):
    """T: oracle.LimbTables -> (fwd_pairs, inv_pairs), each uint32[L, N, 2]."""
    L, N = T.psi_tab.shape
    fwd = np.empty((L, N, 2), dtype=np.uint32)
    inv = np.empty((L, N, 2), dtype=np.uint32)
    for l, (q, _) in enumerate(T.moduli):
        qq = np.uint64(q)
        w = T.psi_tab[l].astype(np.uint64)
        fwd[l, :, 0] = w
        fwd[l, :, 1] = ((w << np.uint64(32)) // qq).astype(np.uint32)
        w = T.inv_tab[l].astype(np.uint64)
        inv[l, :, 0] = w
        inv[l, :, 1] = ((w << np.uint64(32)) // qq).astype(np.uint32)
        R = (1 << 32) % q
        Rinv = pow(R, q - 2, q)
        c = int(T.degree_inv[l]) * Rinv % q
        fwd[l, 0] = _pair(R, q)
        fwd[l, 1] = _pair(int(T.psi_tab[l, 1]) * R, q)
        inv[l, 0] = _pair(c, q)
        inv[l, 1] = _pair(int(T.inv_tab[l, 1]) * c, q)
    slots = np.array([tw_slot(i, T.logN) for i in range(N)])
    pf, pi = np.empty_like(fwd), np.empty_like(inv)
    pf[:, slots] = fwd
    pi[:, slots] = inv
    return pf, pi


COMP_MIN_LOGN = 15


def compressed_tables(T):
    """The compressed layout (arith.cuh, tw_comp_*) of T's device tables:
    uint32[L, 3N/16 + 16, 2] per direction -- entries 0 .. N/16-1 as in the
    full table (folded 0 and 1 included), then for p = 3, 2, 1, 0 the base
    block of stage logN-1-p (entry H + m F, H = N / 2^(p+1), F = 16 / 2^p,
    m < N/32), then the unit-step factors psi^(+-bitrev(c)), c < 16, with
    factor 0 = 1 (never folded)."""
    fwd_s, inv_s = device_tables(T)
    L, N = T.psi_tab.shape
    logN = T.logN
    slots = np.array([tw_slot(i, logN) for i in range(N)])
    fwd, inv = fwd_s[:, slots], inv_s[:, slots]  # natural order, folds kept
    idx = list(range(N // 16))
    for p in (3, 2, 1, 0):
        h, f = N >> (p + 1), 16 >> p
        idx += [h + m * f for m in range(N // 32)]
    out = []
    for full, tab in ((fwd, T.psi_tab), (inv, T.inv_tab)):
        c = np.empty((L, len(idx) + 16, 2), dtype=np.uint32)
        c[:, :len(idx)] = full[:, idx]
        for l, (q, _) in enumerate(T.moduli):
            for k in range(16):
                c[l, len(idx) + k] = _pair(int(tab[l, k]), q)
        out.append(c)
    return out[0], out[1]
