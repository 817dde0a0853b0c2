"""CPU restatement of the APR splitting pass (test infrastructure).

Follows the same rules as urban-sph_a100_b200/csrc/apr.cu, which restates
the reference's cell-based 3-D APR (functions_APR.cuh:270-652,
functions_APR_etc.cuh:5-20): per NNPS cell in cell order the first fluid
particle whose target level exceeds log8(m_ref/m) by >= 0.75 splits into
eight children in free dummy records.  Input is the sorted state the CUDA
path holds before the pass (sph_download + sph_nnps_export).
"""
import numpy as np


def bin_axis(v, vmin, vmax, n):
    f = np.float32
    if vmax == vmin:
        return np.zeros(len(v), np.int64)
    t = np.floor(f((f(v) - f(vmin)) / f(f(vmax) - f(vmin))) * f(n))
    return np.clip(np.minimum(t, n - 1), 0, None).astype(np.int64)


def split(P, g_str, g_end, p):
    """Returns (expected records after the pass, cells split, cells that asked)."""
    NI, NJ, NK = p.geti("NI"), p.geti("NJ"), p.geti("NK")
    NC = p.geti("num_cells")
    lim = [(p.getf("x_min"), p.getf("x_max"), NI), (p.getf("y_min"), p.getf("y_max"), NJ),
           (p.getf("z_min"), p.getf("z_max"), NK)]
    reach = int(np.ceil(p.apr_zone / float(np.float32(p.getf("dcell")))))
    zone = np.zeros((NK, NJ, NI), bool)
    mk = (P["p_type"] >= 1000) & (P["i_type"] < 3)
    ci = [bin_axis(P[a][mk], *lim[k]) for k, a in enumerate(("x", "y", "z"))]
    for a, b, c in zip(*ci):
        zone[max(c - reach, 0):c + reach + 1, max(b - reach, 0):b + reach + 1, max(a - reach, 0):a + reach + 1] = True
    zone = zone.ravel()
    picks = []
    lvl_max = p.apr_max_level
    for k in range(NC - 1):
        if not zone[k] or g_str[k] < 0:
            continue
        for j in range(g_str[k], g_end[k]):
            if P["p_type"][j] != 1 or P["i_type"][j] >= 3:
                continue
            level = np.log(float(P["m_ref"][j]) / float(P["m"][j])) / np.log(8.0)
            if lvl_max - level >= 0.75:
                picks.append(j)
                break
    first_free = int(g_str[NC]) if g_str[NC] >= 0 else len(P)   # the dummy segment
    nfree = len(P) - first_free
    cells = min(len(picks), nfree // 8)
    Q = P.copy()
    h_change = p.geti("h_change")
    f = np.float32
    for q, j in enumerate(picks[:cells]):
        d = f(0.25) * np.cbrt(f(P["m"][j]) / f(P["rho"][j]), dtype=f)
        for o in range(8):
            dst = first_free + 8 * q + o
            Q[dst] = P[j]
            sx = d if o < 4 else -d
            sy = d if (o & 2) == 0 else -d
            sz = d if (o & 1) == 0 else -d
            Q["x"][dst] = f(P["x"][j]) + sx
            Q["y"][dst] = f(P["y"][j]) + sy
            Q["z"][dst] = f(P["z"][j]) + sz
            Q["m"][dst] = f(0.125) * P["m"][j]
            Q["vol"][dst] = f(0.125) * P["vol"][j]
            if h_change:
                Q["h"][dst] = f(0.5) * P["h"][j]
        Q["i_type"][j] = 3
    return Q, cells, len(picks)
