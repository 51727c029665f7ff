"""Generate layouts_gen.h: the shared-memory work-buffer layout of every
compiled fused-kernel configuration (configs.h).

The work buffer uses an additive bank-spreading layout
    phys(l) = l + C1*(l >> A1) + C2*(l >> A2)
(monotone, hence injective; additive over disjoint bit sets, so per-register
addresses stay base + immediate).  One layout serves every pass of a
configuration: each pass rewrites in place exactly the words it read, so its
read and write layouts must agree (a different write layout would overwrite
words other threads have not read yet).  This script searches A1, C1, A2, C2
minimising the worst warp-wide bank conflict over the lane patterns of all
register passes (reads count double) and of both scatters' writes (as the
writer's lane bits land in the receiving CTA; bits that select a different
CTA are dropped), then the layout size.

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


def pass_lanes(MB, PLO, KB, EB, WM):
    XB = EB - KB
    free = [p for p in range(MB) if not (PLO <= p < PLO + KB) and not (WM >> p) & 1]
    reg = set(range(PLO, PLO + KB)) | set(free[:XB])
    rest = [p for p in range(MB) if p not in reg and not (WM >> p) & 1]
    return rest[:5]


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
    g["P1A"] = pass_lanes(MB, MB - K1A, K1A, EB, WM1)
    g["P1B"] = pass_lanes(MB, S1, max(K1B, 1), EB, WM1)
    g["P2A"] = pass_lanes(MB, R2 - K2A, K2A, EB, WM2)
    g["P2B"] = pass_lanes(MB, 0, max(K2B, 1), EB, WM2)
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
    pos = [p for p in pos if p is not None]
    cnt = {}
    for l in range(1 << len(pos)):
        lam = sum(((l >> i) & 1) << p for i, p in enumerate(pos))
        b = phys(lam, *lay) & 31
        cnt[b] = cnt.get(b, 0) + 1
    return max(cnt.values()) if cnt else 1


def search(MB, patterns):
    best = None
    cs = [1, 2, 3, 4, 5, 6, 7, 8, 12, 16]
    top = (1 << MB) - 1
    cands = [(a1, c1, MB, 0) for a1 in range(MB) for c1 in cs]
    cands += [(a1, c1, a2, c2) for a1 in range(MB) for c1 in cs
              for a2 in range(a1 + 1, MB) for c2 in cs]
    for lay in cands:
        degs = [conflicts(p, lay) * w for p, w in patterns]
        key = (max(degs), sum(degs), phys(top, *lay) + 1)
        if best is None or key < best[0]:
            best = (key, lay)
    (deg, total, size), lay = best
    return lay, size


def layout(g):
    fw = g["P1B"] if g["K1B"] > 0 else g["P1A"]  # forward scatter writer
    iw = g["P2A"]                                 # inverse scatter writer
    pats = [(g[n], 2) for n in ("P1A", "P1B", "P2A", "P2B")]
    pats += [([f_lam_pos(g, p) for p in fw], 1), ([i_lam_pos(g, p) for p in iw], 1)]
    return search(g["MB"], pats)


def mask(pos):
    return sum(1 << p for p in pos)


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
    lines.append("}  // namespace nttb")
    path = os.path.join(HERE, "layouts_gen.h")
    open(path, "w").write("\n".join(lines) + "\n")
    print("wrote", path)


if __name__ == "__main__":
    main()
