"""CPU restatement of one cell-based 3-D APR pass (test infrastructure).

Restates, per NNPS cell in cell order, the reference's
  * KERNEL_APR_condition3D_cell (functions_APR.cuh:270-403): the first
    record whose target level M exceeds its level log(m_ref/m)/log(8) by
    >= 0.75 is marked to split (apr_cond 1, the cell flags +1); otherwise the
    last record exceeding M by more than 0.3 is a merge candidate, its family
    (blood_index) is searched within search_kappa * h over the cells
    ceil(2 h / h_ref) around it, the search gives up when a member has M == 1,
    and the member of largest index is marked (apr_cond -1, the cell flags -1);
  * Cell_index (functions_APR_etc.cuh:5-20): +1, +2, ... and -1, -2, ...;
  * KERNEL_cell_APR_3D (functions_APR.cuh:406-652), split: eight children
    from k_num_part + num_buffer + 8 * number, octants with the x sign
    slowest, x +- 0.25 cbrt(m / rho), m / 8, vol / 8, h / 2 (h_change);
and, where the reference's 3-D merge is commented out, its active 2-D merge
(KERNEL_cell_APR_2D, functions_APR.cuh:119-186) in 3-D: in the cell that
holds the marked member, a complete family of eight (i_type 1, same family,
in the cells around the marked member, which is the family's largest index)
is summed -- m, vol, and 1/8 of positions, velocities and pressure -- into a
copy of the marked member written at num_part2 + number, with h = h_ref
cbrt(m / m_ref); the members become dummies.

The condition and the split are checked against the reference's own kernels
compiled for the host (oracle/ref_apr_shim.cpp, tests/test_oracle.py); the
merge has no runnable counterpart in the reference, so that part of this
restatement is parity unpinned.  Input is a sorted state (the records after
NNPS with g_str / g_end, as sph_download + sph_nnps_export give them) with
per-record target levels and families (sph_apr_state).
"""
import numpy as np

f32 = np.float32


def bin_axis(v, vmin, vmax, n):
    if vmax == vmin:
        return np.zeros(np.shape(v), np.int64)
    t = np.floor(f32(f32(f32(v) - f32(vmin)) / f32(f32(vmax) - f32(vmin))) * f32(n))
    return np.clip(np.minimum(t, n - 1), 0, None).astype(np.int64)


def _grid(p):
    return ((p.getf("x_min"), p.getf("x_max"), p.geti("NI")), (p.getf("y_min"), p.getf("y_max"), p.geti("NJ")),
            (p.getf("z_min"), p.getf("z_max"), p.geti("NK")))


def zone_target(P, g_idx, p):
    """Target level per record: apr_max_level for fluid (p_type 1, active)
    whose cell lies within ceil(apr_zone / dcell) cells of a marker's cell."""
    NI, NJ, NK = p.geti("NI"), p.geti("NJ"), p.geti("NK")
    NC = p.geti("num_cells")
    lvl = int(p.apr_max_level)
    target = np.zeros(len(P), np.float32)
    if lvl <= 0:
        return target
    reach = int(np.ceil(p.apr_zone / float(f32(p.getf("dcell")))))
    zone = np.zeros((NK, NJ, NI), bool)
    mk = (P["p_type"] >= 1000) & (P["i_type"] < 3)
    ci = [bin_axis(P[a][mk], *g) for a, g in zip(("x", "y", "z"), _grid(p))]
    for a, b, c in zip(*ci):
        zone[max(c - reach, 0):c + reach + 1, max(b - reach, 0):b + reach + 1, max(a - reach, 0):a + reach + 1] = True
    zone = zone.ravel()
    k = np.asarray(g_idx, np.int64)
    ok = (P["i_type"] < 3) & (P["p_type"] == 1) & (k >= 0) & (k < NC)
    ok[ok] = zone[k[ok]]
    target[ok] = f32(lvl)
    return target


def level(m_ref, m):
    """log(m_ref / m) / log(8.0): a float logarithm over the double log(8)."""
    return f32(float(np.log(f32(f32(m_ref) / f32(m)))) / np.log(8.0))


def _cells_around(P, j, p):
    (x0, x1, NI), (y0, y1, NJ), (z0, z1, NK) = _grid(p)
    ic, jc, kc = (int(bin_axis(P[a][j], lo, hi, nn)) for a, (lo, hi, nn) in zip(("x", "y", "z"), _grid(p)))
    rng = int(np.ceil(f32(f32(2.0) * f32(P["h"][j])) / f32(P["h_ref"][j])))
    for dz in range(-rng, rng + 1):
        for dy in range(-rng, rng + 1):
            for dx in range(-rng, rng + 1):
                a, b, c = ic + dx, jc + dy, kc + dz
                if a < 0 or a > NI - 1 or b < 0 or b > NJ - 1 or c < 0 or c > NK - 1:
                    continue
                yield a + NI * b + NI * NJ * c


def condition(P, g_str, g_end, p, target, family):
    """apr_cond per record and flag per cell (+1 split, -1 merge, 0)."""
    NC = p.geti("num_cells")
    cond = np.zeros(len(P), np.int32)
    flag = np.zeros(NC, np.int32)
    skappa = f32(p.getf("search_kappa"))
    for k in range(NC):
        s, e = int(g_str[k]), int(g_end[k])
        if s < 0 or e <= s:
            continue
        merge_index, blood, merge = 0, 0, False
        split = False
        for j in range(s, e):
            d = f32(f32(target[j]) - level(P["m_ref"][j], P["m"][j]))
            if d >= 0.75:
                cond[j] = 1
                flag[k] = 1
                split = True
                break
            elif d < -0.3:
                merge_index, blood, merge = j, int(family[j]), True
        if split or not merge:
            continue
        xi = np.array([P["x"][merge_index], P["y"][merge_index], P["z"][merge_index]], np.float32)
        search = f32(skappa * f32(P["h"][merge_index]))
        gave_up = False
        for kk in _cells_around(P, merge_index, p):
            if g_str[kk] < 0:
                continue
            for j in range(int(g_str[kk]), int(g_end[kk])):
                d2 = f32(f32(f32(f32(xi[0] - P["x"][j]) ** 2) + f32(f32(xi[1] - P["y"][j]) ** 2)) +
                         f32(f32(xi[2] - P["z"][j]) ** 2))
                r = f32(float(np.sqrt(d2)) + 1e-20)
                if not r < search:
                    continue
                if P["i_type"][j] == 1 and family[j] == blood:
                    if target[j] == 1.0:
                        gave_up = True
                        break
                    if j > merge_index:
                        merge_index = j
            if gave_up:
                break
        if gave_up:
            continue
        cond[merge_index] = -1
        flag[k] = -1
    return cond, flag


def family_members(P, p, g_str, g_end, family, j, blood):
    """Active (i_type 1) members of family `blood` in the cells around record j."""
    out = []
    for kk in _cells_around(P, j, p):
        if g_str[kk] < 0:
            continue
        out += [i for i in range(int(g_str[kk]), int(g_end[kk])) if P["i_type"][i] == 1 and family[i] == blood]
    return out


def merge_record(P, p, g_str, g_end, family, cond, k):
    """The record cell k merges: its first marked member, when that member's
    family is complete (eight active members around it) and it is the
    family's member of largest index; else -1."""
    s, e = int(g_str[k]), int(g_end[k])
    js = [j for j in range(s, e) if cond[j] == -1]
    if not js:
        return -1
    j = js[0]
    blood = int(family[j])
    if blood == 0:
        return -1
    members = family_members(P, p, g_str, g_end, family, j, blood)
    return j if len(members) == 8 and max(members) == j else -1


def merge_cells(flag, cond, g_str, g_end, P, p, family):
    """The merging cells of a pass: those holding a marked member (apr_cond -1)
    whose family merges in this pass, so that the free records at the tail
    go to merges that happen.  The reference numbers every cell whose
    condition asked to merge (Cell_index on its flags), whose slots stay
    unused when the cell holds no marked member or the family is incomplete;
    its 3-D merge is commented out, and with few free records left that
    numbering would hand every slot to cells that do not merge."""
    out = np.where(flag > 0, flag, 0).astype(np.int32)
    for k in range(len(flag)):
        if flag[k] > 0 or g_str[k] < 0:
            continue
        if merge_record(P, p, g_str, g_end, family, cond, k) >= 0:
            out[k] = -1
    return out


def numbering(flag):
    """Cell_index: +1, +2, ... for splitting cells, -1, -2, ... for merging cells."""
    num = np.zeros(len(flag), np.int32)
    pos = neg = 0
    for k, f in enumerate(flag):
        if f > 0:
            pos += 1
            num[k] = pos
        elif f < 0:
            neg += 1
            num[k] = -neg
    return num, pos, neg


def execute(P, g_str, g_end, p, target, family, cond, num, first_free):
    """Split and merge with the capacity rule of the CUDA pass (children
    while they fit, then merged records at the tail while they stay past the
    children, both in cell order); returns
    (records, target, family, cells split, families merged)."""
    n = len(P)
    pos = int((num > 0).sum())
    neg = int((num < 0).sum())
    nfree = n - first_free
    max_split = max(0, min(pos, (nfree - 8) // 8))
    min_slot = first_free + 8 * (max_split + 1) if max_split > 0 else first_free
    Q = P.copy()
    T = np.array(target, np.float32, copy=True)
    F = np.array(family, np.int32, copy=True)
    h_change = p.geti("h_change")
    merged = 0
    for k in range(len(num)):
        q = int(num[k])
        s, e = int(g_str[k]), int(g_end[k])
        if q == 0 or s < 0 or e <= s:
            continue
        if q > 0:
            if q > max_split:
                continue
            js = [j for j in range(s, e) if not (P["p_type"][j] != 1 and target[j] > 2.0) and cond[j] == 1]
            if not js:
                continue
            j = js[0]
            d = np.cbrt(f32(f32(P["m"][j]) / f32(P["rho"][j])), dtype=np.float32)
            for o in range(8):
                dst = first_free + 8 * q + o
                Q[dst] = P[j]
                T[dst] = target[j]
                F[dst] = family[j]
                sx = 0.25 if o < 4 else -0.25
                sy = 0.25 if (o & 2) == 0 else -0.25
                sz = 0.25 if (o & 1) == 0 else -0.25
                Q["x"][dst] = f32(float(P["x"][j]) + sx * float(d))
                Q["y"][dst] = f32(float(P["y"][j]) + sy * float(d))
                Q["z"][dst] = f32(float(P["z"][j]) + sz * float(d))
                Q["m"][dst] = f32(0.125 * float(P["m"][j]))
                Q["vol"][dst] = f32(0.125 * float(P["vol"][j]))
                if h_change:
                    Q["h"][dst] = f32(0.5 * float(P["h"][j]))
            Q["i_type"][j] = 3
            continue
        if n + q < min_slot:
            continue
        j = merge_record(P, p, g_str, g_end, family, cond, k)
        if j < 0:
            continue
        members = family_members(P, p, g_str, g_end, family, j, int(family[j]))
        acc = {f: f32(0) for f in ("m", "vol", "x", "y", "z", "ux", "uy", "uz", "pres")}
        for i in members:
            acc["m"] = f32(acc["m"] + P["m"][i])
            acc["vol"] = f32(acc["vol"] + P["vol"][i])
            for f in ("x", "y", "z", "ux", "uy", "uz", "pres"):
                acc[f] = f32(float(acc[f]) + 0.125 * float(P[f][i]))
        dst = n + q
        Q[dst] = P[j]
        T[dst] = target[j]
        F[dst] = family[j]
        for i in members:
            Q["i_type"][i] = 3
        Q["i_type"][dst] = 1
        for f in ("m", "vol", "x", "y", "z", "ux", "uy", "uz", "pres"):
            Q[f][dst] = acc[f]
        if h_change:
            Q["h"][dst] = f32(f32(P["h_ref"][j]) * np.cbrt(f32(acc["m"] / f32(P["m_ref"][j])), dtype=np.float32))
        merged += 1
    return Q, T, F, max_split, merged


def apr_pass(P, g_idx, g_str, g_end, p, family=None):
    """One pass on a sorted state.  family None: the first pass (index + 1).
    Returns (records, target, family, cells split, cells that asked, families merged)."""
    NC = p.geti("num_cells")
    if family is None:
        family = np.arange(1, len(P) + 1, dtype=np.int32)
    target = zone_target(P, g_idx, p)
    cond, flag = condition(P, g_str, g_end, p, target, family)
    num, pos, neg = numbering(merge_cells(flag, cond, g_str, g_end, P, p, family))
    first_free = int(g_str[NC]) if g_str[NC] >= 0 else len(P)
    Q, T, F, ns, nm = execute(P, g_str, g_end, p, target, family, cond, num, first_free)
    return Q, T, F, ns, pos, nm


def split(P, g_str, g_end, p, g_idx=None):
    """First pass on a sorted state: (records, cells split, cells that asked)."""
    if g_idx is None:
        g_idx = np.full(len(P), p.geti("num_cells"), np.int64)
        for k in range(p.geti("num_cells")):
            if g_str[k] >= 0:
                g_idx[g_str[k]:g_end[k]] = k
    Q, _, _, ns, pos, _ = apr_pass(P, g_idx, g_str, g_end, p)
    return Q, ns, pos
