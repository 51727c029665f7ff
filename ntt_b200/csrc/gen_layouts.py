"""Generate layouts_gen.h: the shared-memory work-buffer layout of every
compiled fused-kernel configuration (configs.h).

The work buffer uses an additive bank-spreading layout
    phys(l) = l + C1*(l >> A1) + C2*(l >> A2)
(monotone, hence injective; additive over disjoint bit sets, so per-register
addresses stay base + immediate).  One layout serves every pass of a
configuration: each pass rewrites in place exactly the words it read, so its
read and write layouts must agree (a different write layout would overwrite
words other threads have not read yet).  This script searches A1, C1, A2, C2
over the lane patterns of all register passes (reads count double), of both
scatters' writes (as the writer's lane bits land in the receiving CTA; bits
that select a different CTA are dropped) and of the warp-chunk slab moves:
among the layouts with at most 1/8 of pads and no access worse than 4-way
bank-conflicted, it minimises their weighted wavefronts plus instructions,
then the worst conflict, then the size.  A pass whose registers
hold runs of 2 or 4 consecutive words uses 64- / 128-bit shared-memory
accesses when the layout keeps those runs aligned (C1, C2 multiples of the
run and A1, A2 at least its log2), which the search weighs against the
scalar accesses' conflicts.

The lane patterns mirror PassLayout / Geometry in ntt_core.cuh; the header
records them and ntt_core.cuh static_asserts that they agree.

    python ntt_b200/csrc/gen_layouts.py      # rewrites layouts_gen.h
"""
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))


def configs():
    """Distinct (N, CL, R1, EB, K1A, K2A) of configs.h: the layout of a slab
    does not depend on the polynomials per job (NP, the 7th field)."""
    src = open(os.path.join(HERE, "configs.h")).read().split("#define NTTB_CFG_ALL")[0]
    out = []
    for m in re.findall(r"X\((\d+), (\d+), (\d+), (\d+), (\d+), (\d+), (\d+)\)", src):
        g = tuple(int(v) for v in m[:6])
        if g not in out:
            out.append(g)
    return out


def pass_regs(MB, PLO, KB, EB, WM):
    XB = EB - KB
    free = [p for p in range(MB) if not (PLO <= p < PLO + KB) and not (WM >> p) & 1]
    return set(range(PLO, PLO + KB)) | set(free[:XB])


def pass_lanes(MB, PLO, KB, EB, WM):
    reg = pass_regs(MB, PLO, KB, EB, WM)
    rest = [p for p in range(MB) if p not in reg and not (WM >> p) & 1]
    return rest[:5]


def run_bits(reg):
    v = 0
    while v in reg:
        v += 1
    return v


def geometry(N, CL, R1, EB, K1A, K2A):
    g = dict(N=N, CL=CL, R1=R1, EB=EB, K1A=K1A, K2A=K2A)
    R2 = N - R1
    MB = N - CL
    S1 = R2 - CL
    TB = MB - EB
    K1B, K2B = R1 - K1A, R2 - K2A
    WB = TB - 5
    WARP2 = K2B > 0 and (R1 - CL) >= WB
    WM1 = 0  # phase 1 keeps a CTA barrier (coalesced strided accesses)
    WM2 = (((1 << WB) - 1) << (MB - WB)) if WARP2 else 0
    g.update(R2=R2, MB=MB, S1=S1, K1B=K1B, K2B=K2B)
    args = {"P1A": (MB - K1A, K1A, WM1), "P1B": (S1, max(K1B, 1), WM1),
            "P2A": (R2 - K2A, K2A, WM2), "P2B": (0, max(K2B, 1), WM2)}
    for n, (plo, kb, wm) in args.items():
        g[n] = pass_lanes(MB, plo, kb, EB, wm)
        g[n + "_run"] = run_bits(pass_regs(MB, plo, kb, EB, wm))
    g["EB"] = EB
    return g


def f_lam_pos(g, p):
    """lambda1 bit -> lambda2 bit of the forward scatter (None: selects the CTA)."""
    if p < g["S1"]:
        return p
    if p < g["S1"] + g["R1"] - g["CL"]:
        return p + g["CL"]
    return None


def i_lam_pos(g, p):
    """lambda2 bit -> lambda1 bit of the inverse scatter (None: selects the CTA)."""
    if p < g["S1"]:
        return p
    if p < g["R2"]:
        return None
    return p - g["CL"]


def phys(l, a1, c1, a2, c2):
    return l + c1 * (l >> a1) + c2 * (l >> a2)


def conflicts(pos, lay):
    """Scalar access: the most distinct words one bank serves for the warp."""
    pos = [p for p in pos if p is not None]
    cnt = {}
    for l in range(1 << len(pos)):
        lam = sum(((l >> i) & 1) << p for i, p in enumerate(pos))
        b = phys(lam, *lay) & 31
        cnt[b] = cnt.get(b, 0) + 1
    return max(cnt.values()) if cnt else 1


def aligned(lay, v):
    """Every aligned run of v lambdas maps to an aligned run of v words."""
    a1, c1, a2, c2 = lay
    return all(c % v == 0 and (c == 0 or (1 << a) % v == 0) for a, c in ((a1, c1), (a2, c2)))


def vec_width(run, lay):
    """The access width the kernels use (ntt_core.cuh smem_vec): 4 words
    when the pass owns runs of 4 and the layout keeps them aligned, else 2,
    else 1."""
    if run >= 2 and aligned(lay, 4):
        return 4
    if run >= 1 and aligned(lay, 2):
        return 2
    return 1


def vec_wavefronts(pos, lay, v):
    """(wavefronts of one warp instruction, worst per-phase degree) of a
    v-word access: the warp runs in 32/v-lane phases (lane-id order), each
    v-word chunk occupies a group of v banks, and a phase costs as many
    wavefronts as the most distinct chunks one group serves."""
    lanes_per_phase = 32 // v
    lb = lanes_per_phase.bit_length() - 1
    total, worst = 0, 0
    for ph in range(v):
        cnt = {}
        for l in range(lanes_per_phase):
            lane = (ph << lb) | l
            lam = sum(((lane >> i) & 1) << p for i, p in enumerate(pos))
            chunk = phys(lam, *lay) // v
            g = chunk % (32 // v)
            cnt.setdefault(g, set()).add(chunk)
        d = max(len(c) for c in cnt.values())
        total += d
        worst = max(worst, d)
    return total, worst


def pattern_cost(pos, run, words, lay):
    """(worst degree, wavefronts + instructions) of one pass's accesses."""
    v = vec_width(run, lay)
    if v == 1:
        d = conflicts(pos, lay)
        return d, words * (d + 1)
    wf, worst = vec_wavefronts(pos, lay, v)
    return worst, (words // v) * (wf + 1)


def search(MB, passes, scalar_pats, chunk_words):
    """passes: (lane positions, run bits, words per thread, weight);
    scalar_pats: (positions, weight) of the scalar scatter writes.  Among the
    layouts whose worst conflict is at most 4-way: the least weighted
    wavefronts + instructions of every access (the warp-chunk slab moves
    included: vector when the layout keeps 4-word runs aligned), then the
    worst conflict, then the size."""
    best = None
    cs = [1, 2, 3, 4, 5, 6, 7, 8, 12, 16, 20, 24, 28, 32, 36, 40]
    top = (1 << MB) - 1
    cands = [(a1, c1, MB, 0) for a1 in range(MB) for c1 in cs]
    cands += [(a1, c1, a2, c2) for a1 in range(MB) for c1 in cs
              for a2 in range(a1 + 1, MB) for c2 in cs]
    for lay in cands:
        # at most 1/8 of the slab in pads: the work buffer of the 2^16
        # configurations stays within the 5 CTAs per SM their registers allow
        if phys(top, *lay) + 1 > (top + 1) * 9 // 8:
            continue
        worst, cost = 1, 0
        for pos, run, words, w in passes:
            d, c = pattern_cost(pos, run, words, lay)
            worst, cost = max(worst, d), cost + w * c
        for pos, w in scalar_pats:
            d = conflicts(pos, lay)
            worst, cost = max(worst, d), cost + w * 32 * (d + 1)
        chunk = ([2, 3, 4, 5, 6], 2) if aligned(lay, 4) else ([0, 1, 2, 3, 4], 0)
        d, c = pattern_cost(chunk[0], chunk[1], chunk_words, lay)
        worst, cost = max(worst, d), cost + 2 * c
        if worst > 4:  # the bound the emulator test holds every layout to
            continue
        key = (cost, worst, phys(top, *lay) + 1)
        if best is None or key < best[0]:
            best = (key, lay)
    (deg, total, size), lay = best
    return lay, size


# Layouts kept by measurement on B200 where the cost model's choice was slower:
# the forward default (2^16, 8-CTA cluster, R1 = 8) runs 0.250 ms per 64 x 16
# limbs with its scalar layout, 0.262 ms with the vector-aligned one the model
# prefers (6, 4, 13, 0) and 0.264 ms with (5, 4, 13, 0), whose 128-bit
# accesses are conflict-free but whose 64-bit phase-2 accesses are 2-way.
MEASURED = {(16, 3, 8, 5, 3, 4): (5, 1, 13, 0)}


def layout(g):
    key = (g["N"], g["CL"], g["R1"], g["EB"], g["K1A"], g["K2A"])
    if key in MEASURED:
        lay = MEASURED[key]
        return lay, phys((1 << g["MB"]) - 1, *lay) + 1
    fw = g["P1B"] if g["K1B"] > 0 else g["P1A"]  # forward scatter writer
    iw = g["P2A"]                                 # inverse scatter writer
    E = 1 << g["EB"]
    passes = [(g[n], g[n + "_run"], E, 2) for n in ("P1A", "P1B", "P2A", "P2B")]
    scat = [([f_lam_pos(g, p) for p in fw], 1), ([i_lam_pos(g, p) for p in iw], 1)]
    return search(g["MB"], passes, scat, E)


def mask(pos):
    return sum(1 << p for p in pos)


# ---------------------------------------------------------------------------
# Split (L2-exchange) configurations: phase 1 is one register pass per column
# in global memory (no shared memory); phase 2 runs two or three register
# passes over the CTA's contiguous rows in the work buffer.  The first phase-2
# pass reads global memory with its lanes on the 5 lowest bits (its extra
# register bits are the lowest free positions from bit 5 up); the others
# follow PassLayout's rule.  Mirrors SplitGeo in split_kernel.cuh.
# ---------------------------------------------------------------------------

def split_configs():
    src = open(os.path.join(HERE, "configs.h")).read()
    src = src.split("// Split configurations")[1].split("#include")[0]
    out = []
    for m in re.findall(r"S\((\d+), (\d+), (\d+), (\d+), (\d+)\)", src):
        g = tuple(int(v) for v in m)
        if g not in out:
            out.append(g)
    return out


def split_passes(N, CL, EB, K2A, K2B):
    MB, R2 = N - CL, N - EB
    K2C = R2 - K2A - K2B
    lo_a, lo_b = R2 - K2A, R2 - K2A - K2B
    # first pass: explicit extras from bit 5 up
    extra = [p for p in range(5, MB) if not (lo_a <= p < lo_a + K2A)][:EB - K2A]
    reg_a = set(range(lo_a, lo_a + K2A)) | set(extra)
    lanes_a = [p for p in range(MB) if p not in reg_a][:5]
    out = [("P2A", lanes_a, run_bits(reg_a), False)]
    out.append(("P2B", pass_lanes(MB, lo_b, K2B, EB, 0), run_bits(pass_regs(MB, lo_b, K2B, EB, 0)), True))
    if K2C > 0:
        out.append(("P2C", pass_lanes(MB, 0, K2C, EB, 0), run_bits(pass_regs(MB, 0, K2C, EB, 0)), True))
    return MB, out


def split_layout(cfg):
    N, CL, EB, K2A, K2B = cfg
    MB, ps = split_passes(*cfg)
    E = 1 << EB
    best = None
    cs = [1, 2, 3, 4, 5, 6, 7, 8, 12, 16, 20, 24, 28, 32, 36, 40]
    top = (1 << MB) - 1
    cands = [(a1, c1, MB, 0) for a1 in range(MB) for c1 in cs]
    cands += [(a1, c1, a2, c2) for a1 in range(MB) for c1 in cs
              for a2 in range(a1 + 1, MB) for c2 in cs]
    for lay in cands:
        # up to 1/4 of pads: 5 CTAs of 256 threads still fit an SM's shared
        # memory (the split kernels hold one buffer per CTA)
        if phys(top, *lay) + 1 > (top + 1) * 5 // 4:
            continue
        worst, cost = 1, 0
        for name, pos, run, both in ps:  # the first pass only stores
            d, c = pattern_cost(pos, run, E, lay)
            worst, cost = max(worst, d), cost + (2 if both else 1) * c
        chunk = ([2, 3, 4, 5, 6], 2) if aligned(lay, 4) else ([0, 1, 2, 3, 4], 0)
        d, c = pattern_cost(chunk[0], chunk[1], E, lay)
        worst, cost = max(worst, d), cost + 2 * c
        key = (worst, cost, phys(top, *lay) + 1)
        if best is None or key < best[0]:
            best = (key, lay)
    (deg, cost, size), lay = best
    return lay, size, ps


def main():
    lines = [
        "// GENERATED by gen_layouts.py from configs.h -- do not edit.",
        "// Per configuration: the work-buffer bank-spreading layout (A1, C1, A2, C2,",
        "// size in words) and the lane masks the search assumed (checked against",
        "// PassLayout by static_assert in ntt_core.cuh).",
        "#pragma once",
        "#include <cstdint>",
        "",
        "namespace nttb {",
        "",
        "template <int N, int CL, int R1, int EB, int K1A, int K2A>",
        "struct LayoutTable;",
        "",
    ]
    for cfg in configs():
        g = geometry(*cfg)
        (a1, c1, a2, c2), size = layout(g)
        lines.append("template <>")
        lines.append("struct LayoutTable<%d, %d, %d, %d, %d, %d> {" % cfg)
        lines.append(f"    static constexpr int XW[5] = {{{a1}, {c1}, {a2}, {c2}, {size}}};")
        for name in ("P1A", "P1B", "P2A", "P2B"):
            lines.append(f"    static constexpr uint32_t lanes_{name} = 0x{mask(g[name]):x}u;")
        lines.append("};")
        lines.append("")
    lines += ["template <int N, int CL, int EB, int K2A, int K2B>", "struct SplitLayoutTable;", ""]
    for cfg in split_configs():
        (a1, c1, a2, c2), size, ps = split_layout(cfg)
        lines.append("template <>")
        lines.append("struct SplitLayoutTable<%d, %d, %d, %d, %d> {" % cfg)
        lines.append(f"    static constexpr int XW[5] = {{{a1}, {c1}, {a2}, {c2}, {size}}};")
        for name, pos, run, both in ps:
            lines.append(f"    static constexpr uint32_t lanes_{name} = 0x{mask(pos):x}u;")
        lines.append("};")
        lines.append("")
    lines.append("}  // namespace nttb")
    path = os.path.join(HERE, "layouts_gen.h")
    open(path, "w").write("\n".join(lines) + "\n")
    print("wrote", path)


if __name__ == "__main__":
    main()
