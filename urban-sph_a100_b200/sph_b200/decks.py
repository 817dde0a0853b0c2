"""Seeded synthetic particle decks in the reference's part1 layout.

The reference ships no input decks (its ./input/*.txt files are absent), so
every case here is generated.  Each deck is a ``part1`` record array as
c_initial_inner_outer_particle_single (functions_NNPS.cuh:196-373) leaves it
before upload, plus the solver parameters.

* ``caseh_mini``  -- a small deck laid out in the reference's own hard-wired
  Case-H coordinates (buffer planes L2/L3/L_left/L_right at
  functions_NNPS.cuh:4-11, IB cube faces at functions_PREP.cuh:958-963), so
  that the unmodified reference host build and this project see the same
  geometry.  It exercises every particle class of the step: fluid, inlet,
  outlet and periodic-y buffers, floor walls, moving walls, free-slip ceiling,
  IBM markers and MOST wall-layer particles.  Records are shuffled so the sort
  does real work.
* ``canyon``      -- the urban-canyon workload: a 2.4 x 1.2 x 0.6 m channel at
  dx = 0.01 m (240 x 120 x 60 = 1,728,000 fluid particles), floor walls,
  free-slip ceiling, periodic-y side buffers, inlet/outlet buffers, a 0.1 m
  IBM cube at x = 0.6 m, neutral MOST log-law inflow with u* = 0.3 m/s and
  z0 = 0.01 m, a seeded 5 % uniform velocity perturbation and Cs = 0.12.
  ``scale`` shrinks every extent for small cases.
* ``cube_array`` -- staggered 4 x 4 array of 0.1 m cubes (IBM) in a
  4.8 x 2.4 x 0.8 m channel with two-level APR near the faces.
* ``thermal_mini`` -- ``caseh_mini`` with the conduction, Boussinesq and
  concentration switches on and varied temperature / concentration fields.
* ``cavity``, ``tgv_box``, ``ensemble`` -- the batched-ensemble workload:
  lid-driven cavities and Taylor-Green boxes of 20k-200k particles with Re in
  [100, 2000], seeded.
"""
import numpy as np

from .layout import BUFFER_PERIODIC_GHOST, PART1
from .params import CASEH_PROFILE_U, CASEH_PROFILE_Z, default_params, domain_setup, set_profile

SEED = 20261203


def _records(x, y, z):
    P = np.zeros(len(x), dtype=PART1)
    P["x"], P["y"], P["z"] = x, y, z
    P["i_type"] = 1
    return P


def _grid(xs, ys, zs):
    X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
    return X.ravel(), Y.ravel(), Z.ravel()


def _assign_buffers(P, l2, l3, l_left, l_right, l4=1e30):
    """Buffer classes of functions_NNPS.cuh:254-279 for p_type 1 and -1."""
    sel = (P["p_type"] == 1) | (P["p_type"] == -1)
    y, x = P["y"].astype(np.float64), P["x"].astype(np.float64)
    left = sel & (y < l_left)
    right = sel & ~left & (y > l_right)
    outlet = sel & ~left & ~right & (x >= l3 - 1e-6) & (x < l4 - 1e-6)
    inlet = sel & ~left & ~right & ~outlet & (x < l2 - 1e-6)
    for mask, code in ((left, 3), (right, 4), (outlet, 2), (inlet, 1)):
        P["buffer_type"][mask] = code
        P["i_type"][mask] = 2


def _common_fields(P, dx, h_coeff=1.5, rho=1.225):
    P["h"] = np.float32(h_coeff * dx)
    P["h_ref"] = P["h"]
    P["rho"] = np.float32(rho)
    P["m"] = np.float32(rho * dx ** 3)
    P["m_ref"] = P["m"]
    P["vol"] = np.float32(dx ** 3)
    P["temp"] = np.float32(300.0)


def caseh_mini(dx=0.0412, nx=24, ny=12, nz=7, seed=SEED, shuffle=True, **pkw):
    """Small deck in the reference's hard-wired Case-H coordinates."""
    rng = np.random.default_rng(seed)
    f = np.float32
    xs = np.arange(nx) * dx
    # a quarter-spacing offset keeps every particle off the buffer planes
    # y = +-0.412, so each periodic partner (y +- 0.824) is an interior particle
    ys = (np.arange(-ny, ny) + 0.25) * dx
    parts = []
    # fluid
    fx, fy, fz = _grid(xs, ys, (np.arange(nz) + 0.5) * dx)
    Pf = _records(fx, fy, fz)
    Pf["p_type"] = 1
    parts.append(Pf)
    # floor walls (3 layers) with a moving patch in the top layer
    wx, wy, wz = _grid(xs, ys, -(np.arange(3) + 0.5) * dx)
    Pw = _records(wx, wy, wz)
    Pw["p_type"] = 0
    mov = (Pw["x"] >= xs[-3] - 1e-6) & (np.abs(Pw["z"] + 0.5 * dx) < 1e-6)
    Pw["p_type"][mov] = 9
    parts.append(Pw)
    # free-slip ceiling (3 layers)
    cx, cy, cz = _grid(xs, ys, (nz + np.arange(3) + 0.5) * dx)
    Pc = _records(cx, cy, cz)
    Pc["p_type"] = -1
    parts.append(Pc)
    # IBM markers on the faces of the reference's IB cube
    x0, x1, y0, y1, z0, z1 = 0.764, 0.836, -0.036, 0.036, 0.0, 0.152
    gx, gy, gz = np.linspace(x0, x1, 4), np.linspace(y0, y1, 4), np.linspace(z0, z1, 5)
    mk = []
    for xv in (x0, x1):
        a, b, c = _grid([xv], gy, gz); mk.append((a, b, c))
    for yv in (y0, y1):
        a, b, c = _grid(gx, [yv], gz); mk.append((a, b, c))
    for zv in (z0, z1):
        a, b, c = _grid(gx, gy, [zv]); mk.append((a, b, c))
    Pm = _records(np.concatenate([m[0] for m in mk]), np.concatenate([m[1] for m in mk]),
                  np.concatenate([m[2] for m in mk]))
    Pm["p_type"] = 1000
    parts.append(Pm)
    # outlet island around the reference's L3 = 13.304 (probe plane 13.296)
    ox = np.concatenate([13.296 - np.arange(3) * dx, 13.304 + np.arange(3) * dx])
    qx, qy, qz = _grid(ox, ys, (np.arange(3) + 0.5) * dx)
    Po = _records(qx, qy, qz)
    Po["p_type"] = 1
    parts.append(Po)

    P = np.concatenate(parts)
    _common_fields(P, dx)
    _assign_buffers(P, 0.028, 13.304, -0.412, 0.412)
    fluidlike = (P["p_type"] == 1) | (P["p_type"] == -1)
    zt, ut = np.array(CASEH_PROFILE_Z), np.array(CASEH_PROFILE_U)
    u = np.interp(np.maximum(P["z"].astype(np.float64), 0.0), zt, ut)
    u = u * (1.0 + 0.05 * rng.uniform(-1, 1, len(P)))
    P["ux"] = np.where(fluidlike, u, 0.0).astype(f)
    P["uy"] = np.where(fluidlike, 0.05 * rng.uniform(-1, 1, len(P)) * u, 0.0).astype(f)
    P["uz"] = np.where(fluidlike, 0.05 * rng.uniform(-1, 1, len(P)) * u, 0.0).astype(f)
    P["pres"] = rng.uniform(-0.5, 0.5, len(P)).astype(f)
    P["k_turb"] = np.where(fluidlike, 0.1 + 0.05 * rng.uniform(0, 1, len(P)), 0.0).astype(f)
    P["vis_t"] = np.where(fluidlike, 1e-5 * rng.uniform(0, 1, len(P)), 0.0).astype(f)
    most = (P["p_type"] == 1) & (P["buffer_type"] == 0) & (P["z"] < dx) & (P["x"] < 5.0)
    P["MOST_buffer"][most] = 1
    # Wall-layer air stays at the surface temperature: with the reference's
    # hard-wired MOST_z0 = 1 m (Parameters.cuh:114) and z = dx/2 the Newton
    # branch of KERNEL_MOST_boundary3D diverges to NaN in the reference itself,
    # so step decks use the neutral branch; the Newton branch is covered by a
    # separate wall-layer case at atmospheric heights.
    if shuffle:
        P = P[rng.permutation(len(P))]
    p = default_params(**pkw)
    domain_setup(p, P)
    return P, p


def thermal_mini(con=1, bouss=1, concn=1, seed=11, nx=12, ny=6, nz=5):
    """caseh_mini with conduction, Boussinesq buoyancy and concentration
    switched on: a varied temperature (300 K +- 4 K) and concentration field
    and 20 concentration sources.  Moving walls (p_type 9) become fixed walls:
    the reference gives p_type 9 zero conductivity and heat capacity
    (functions_PPE.cuh:233-234), so its temperature rate there is 0/0."""
    P, p = caseh_mini(nx=nx, ny=ny, nz=nz)
    rng = np.random.default_rng(seed)
    P["p_type"][P["p_type"] == 9] = 0
    P["temp"] = (300.0 + 4.0 * np.sin(7.0 * P["x"]) * np.cos(5.0 * P["z"])
                 + rng.uniform(-0.5, 0.5, len(P))).astype(np.float32)
    P["concn"] = rng.uniform(0.0, 1.0, len(P)).astype(np.float32)
    P["source"][rng.choice(len(P), 20, replace=False)] = 1
    p.seti("con_solve", con)
    p.seti("boussinesq_solve", bouss)
    p.seti("concn_solve", concn)
    return P, p


# the reference's built-in corium table (functions_PROP.cuh:67-70): enthalpy
# [J/kg] against temperature [K], the one htoT reads with prop_table = 0
CORIUM_H = np.array([-554932, 215789, 757894, 905263, 1268421], np.float32)
CORIUM_T = np.array([280, 1537, 2300, 2450, 2650], np.float32)


def enthalpy_mini(seed=11):
    """thermal_mini with the energy equation in enthalpy (enthalpy_eqn = 1)
    and every record's enthalpy on the corium table at its temperature: the
    reference reads no enthalpy from its decks and keeps its
    temperature-to-enthalpy kernel commented out, so the caller sets it."""
    P, p = thermal_mini(1, 1, 1, seed=seed)
    P["enthalpy"] = np.interp(P["temp"].astype(np.float64), CORIUM_T, CORIUM_H).astype(np.float32)
    p.enthalpy_eqn = 1
    return P, p


# two-material property tables for prop_table = 1 (slot 0: walls, |p_type|
# 0; slot 1: fluid and the p_type -1 wall layer), h ascending, with
# breakpoints inside the enthalpy range of enthalpy_mini so that htoT meets
# inner segments and both extrapolated ends
TABLE_WALL = dict(T=[297.0, 300.0, 305.0, 2400.0], h=[-542600.0, -541800.0, -541000.0, 900000.0],
                  k=[1.5, 1.6, 1.7, 2.5], cp=[480.0, 490.0, 500.0, 600.0], mu=[0.0, 0.0, 0.0, 0.0])
TABLE_FLUID = dict(T=[250.0, 290.0, 299.0, 301.5, 304.0, 2650.0],
                   h=[-560000.0, -546000.0, -543500.0, -542000.0, -540500.0, 1268421.0],
                   k=[2.0, 2.1, 2.2, 2.3, 2.4, 3.0], cp=[500.0, 510.0, 515.0, 520.0, 530.0, 560.0],
                   mu=[4e-3, 3.9e-3, 3.8e-3, 3.7e-3, 3.6e-3, 1e-3])


def enthalpy_tables_mini(seed=11):
    """enthalpy_mini with vii[prop_table] = 1 and the two-material tables
    (a PropTables for sph_set_prop_tables): htoT reads table |p_type|."""
    from .layout import PropTables
    P, p = enthalpy_mini(seed=seed)
    p.seti("prop_table", 1)
    return P, p, PropTables.from_columns([TABLE_WALL, TABLE_FLUID])


def with_headroom(P, p, frac):
    """Appends int(frac * len(P)) free dummy records (i_type 3), the room the
    reference reserves for buffer and APR particles (ISPH.cuh:116)."""
    nd = int(frac * len(P))
    D = np.zeros(nd, dtype=PART1)
    D["i_type"] = 3
    D["x"], D["y"], D["z"] = P["x"][0], P["y"][0], P["z"][0]
    D["h"] = D["h_ref"] = P["h"][0]
    D["m"] = D["m_ref"] = P["m"][0]
    D["rho"] = P["rho"][0]
    D["vol"] = P["vol"][0]
    Q = np.concatenate([P, D])
    domain_setup(p, Q)
    return Q, p


def canyon(scale=1.0, dx=0.01, seed=SEED, ustar=0.3, z0=0.01, cs=0.12, dt=2e-4, **pkw):
    """Urban-canyon deck: 2.4 x 1.2 x 0.6 m at dx (scaled by ``scale``)."""
    rng = np.random.default_rng(seed)
    f = np.float32
    nx, ny, nz = (int(round(240 * scale)), int(round(120 * scale)), int(round(60 * scale)))
    nx, ny, nz = max(nx, 16), max(ny, 12), max(nz, 8)
    xs = (np.arange(nx) + 0.5) * dx
    ys = (np.arange(ny) + 0.5) * dx - 0.5 * ny * dx
    zs = (np.arange(nz) + 0.5) * dx
    parts = []
    fx, fy, fz = _grid(xs, ys, zs)
    Pf = _records(fx, fy, fz); Pf["p_type"] = 1; parts.append(Pf)
    wx, wy, wz = _grid(xs, ys, -(np.arange(3) + 0.5) * dx)
    Pw = _records(wx, wy, wz); Pw["p_type"] = 0; parts.append(Pw)
    cx, cy, cz = _grid(xs, ys, (nz + np.arange(3) + 0.5) * dx)
    Pc = _records(cx, cy, cz); Pc["p_type"] = -1; parts.append(Pc)
    # IBM cube: edge = 10 dx at full scale, centred at x = 0.25 L, y = 0
    edge = max(4, int(round(10 * scale))) * dx
    cxm = 0.25 * nx * dx
    bx0, bx1, by0, by1, bz0, bz1 = cxm - edge / 2, cxm + edge / 2, -edge / 2, edge / 2, 0.0, edge
    nm = int(round(edge / dx)) + 1
    gx, gy, gz = np.linspace(bx0, bx1, nm), np.linspace(by0, by1, nm), np.linspace(bz0, bz1, nm)
    mk = []
    for xv in (bx0, bx1):
        mk.append(_grid([xv], gy, gz))
    for yv in (by0, by1):
        mk.append(_grid(gx, [yv], gz))
    for zv in (bz0, bz1):
        mk.append(_grid(gx, gy, [zv]))
    Pm = _records(*[np.concatenate([m[k] for m in mk]) for k in range(3)])
    Pm["p_type"] = 1000
    parts.append(Pm)
    P = np.concatenate(parts)
    _common_fields(P, dx)
    l2 = 3 * dx
    l3 = (nx - 3) * dx
    l_left = ys[3] - 0.5 * dx
    l_right = l_left + (ny - 6) * dx
    _assign_buffers(P, l2, l3, l_left, l_right)
    fluidlike = (P["p_type"] == 1) | (P["p_type"] == -1)
    zz = P["z"].astype(np.float64)
    ulog = np.where(zz > z0, ustar / 0.4 * np.log(np.maximum(zz, z0) / z0), 0.0)
    ux = ulog * (1.0 + 0.05 * rng.uniform(-1, 1, len(P)))
    P["ux"] = np.where(fluidlike, ux, 0.0).astype(f)
    P["uy"] = np.where(fluidlike, 0.05 * ulog * rng.uniform(-1, 1, len(P)), 0.0).astype(f)
    P["uz"] = np.where(fluidlike, 0.05 * ulog * rng.uniform(-1, 1, len(P)), 0.0).astype(f)
    most = (P["p_type"] == 1) & (P["buffer_type"] == 0) & (P["z"] < dx)
    P["MOST_buffer"][most] = 1
    p = default_params(dt=dt, **pkw)
    p.cs_sgs = cs
    p.l2, p.l3, p.l_left, p.l_right = l2, l3, l_left, l_right
    p.outlet_probe_dx = 0.5 * dx
    for k, v in enumerate((bx0, bx1, by0, by1, bz0, bz1)):
        p.ib_box[k] = v
    p.most_z0, p.most_z0h = z0, 0.1 * z0
    zt = np.linspace(0.5 * dx, nz * dx, 24)
    set_profile(p, zt, ustar / 0.4 * np.log(np.maximum(zt, z0) / z0))
    p.setf("u_limit", 20.0)
    p.setf("time_end", 1e9)
    domain_setup(p, P)
    return P, p


def _cube_markers(bx0, bx1, by0, by1, bz0, bz1, dx):
    nm = int(round((bx1 - bx0) / dx)) + 1
    gx, gy, gz = np.linspace(bx0, bx1, nm), np.linspace(by0, by1, nm), np.linspace(bz0, bz1, nm)
    mk = []
    for xv in (bx0, bx1):
        mk.append(_grid([xv], gy, gz))
    for yv in (by0, by1):
        mk.append(_grid(gx, [yv], gz))
    for zv in (bz0, bz1):
        mk.append(_grid(gx, gy, [zv]))
    return [np.concatenate([m[k] for m in mk]) for k in range(3)]


def cube_array(scale=1.0, dx=0.01, seed=SEED, ustar=0.3, z0=0.01, cs=0.12, dt=2e-4, edge=0.1, pitch=0.3,
               apr=False, apr_zone=0.1, headroom=None, stable_dT=0.0, fill_obstacles=True, **pkw):
    """Staggered array of 0.1 m cubes at 0.3 m pitch in a 4.8 x 2.4 x 0.8 m
    channel at dx (extents scaled by ``scale``; 4 x 4 cubes at full size),
    IBM markers on every face, floor walls, free-slip ceiling, periodic-y
    and inlet/outlet buffers, log-law inflow.  With ``apr`` the deck carries
    free dummy records and the parameters for two-level APR (children at
    dx / 2) of fluid within ``apr_zone`` of a marker.  ``stable_dT`` warms
    the wall-layer air above the surface; the default 0 keeps MOST neutral
    (with a temperature difference its Obukhov-length iteration at these
    wall-layer heights gives NaN, as the reference's does).  Returns
    (P, params, boxes) with boxes an (ncube, 6) array for sph_set_ib_boxes."""
    rng = np.random.default_rng(seed)
    f = np.float32
    # the 4.8 x 2.4 x 0.8 m channel (times scale) at spacing dx
    nx, ny, nz = (int(round(4.8 * scale / dx)), int(round(2.4 * scale / dx)), int(round(0.8 * scale / dx)))
    nx, ny, nz = max(nx, 40), max(ny, 24), max(nz, 16)
    xs = (np.arange(nx) + 0.5) * dx
    ys = (np.arange(ny) + 0.5) * dx - 0.5 * ny * dx
    zs = (np.arange(nz) + 0.5) * dx
    Lx, Ly = nx * dx, ny * dx
    # cube array: columns from x = 0.25 Lx, staggered rows, inside the core in y
    ncx = max(1, min(4, int((0.6 * Lx) // pitch)))
    ncy = max(1, min(4, int((0.7 * Ly) // pitch)))
    boxes = []
    for a in range(ncx):
        for b in range(ncy):
            cx = 0.25 * Lx + a * pitch
            cy = (b - 0.5 * (ncy - 1)) * pitch + (0.5 * pitch if a % 2 else 0.0)
            if abs(cy) + 0.5 * edge > 0.5 * Ly - 4 * dx:
                cy -= pitch
            boxes.append((cx - edge / 2, cx + edge / 2, cy - edge / 2, cy + edge / 2, 0.0, edge))
    boxes = np.array(boxes)
    parts = []
    fx, fy, fz = _grid(xs, ys, zs)
    # as in the canyon deck, fluid particles fill the obstacles: the IBM forcing
    # holds them at rest (removing them leaves voids without a boundary row)
    inside = np.zeros(len(fx), bool)
    if not fill_obstacles:
        for bx0, bx1, by0, by1, bz0, bz1 in boxes:
            inside |= (fx > bx0) & (fx < bx1) & (fy > by0) & (fy < by1) & (fz < bz1)
    Pf = _records(fx[~inside], fy[~inside], fz[~inside]); Pf["p_type"] = 1; parts.append(Pf)
    wx, wy, wz = _grid(xs, ys, -(np.arange(3) + 0.5) * dx)
    Pw = _records(wx, wy, wz); Pw["p_type"] = 0; parts.append(Pw)
    cx_, cy_, cz_ = _grid(xs, ys, (nz + np.arange(3) + 0.5) * dx)
    Pc = _records(cx_, cy_, cz_); Pc["p_type"] = -1; parts.append(Pc)
    for bx in boxes:
        Pm = _records(*_cube_markers(*bx, dx)); Pm["p_type"] = 1000; parts.append(Pm)
    P = np.concatenate(parts)
    _common_fields(P, dx)
    l2 = 3 * dx
    l3 = (nx - 3) * dx
    l_left = ys[3] - 0.5 * dx
    l_right = l_left + (ny - 6) * dx
    _assign_buffers(P, l2, l3, l_left, l_right)
    fluidlike = (P["p_type"] == 1) | (P["p_type"] == -1)
    zz = P["z"].astype(np.float64)
    ulog = np.where(zz > z0, ustar / 0.4 * np.log(np.maximum(zz, z0) / z0), 0.0)
    P["ux"] = np.where(fluidlike, ulog * (1.0 + 0.05 * rng.uniform(-1, 1, len(P))), 0.0).astype(f)
    P["uy"] = np.where(fluidlike, 0.05 * ulog * rng.uniform(-1, 1, len(P)), 0.0).astype(f)
    P["uz"] = np.where(fluidlike, 0.05 * ulog * rng.uniform(-1, 1, len(P)), 0.0).astype(f)
    most = (P["p_type"] == 1) & (P["buffer_type"] == 0) & (P["z"] < dx)
    P["MOST_buffer"][most] = 1
    P["temp"][most] = f(300.0 + stable_dT)
    # the wall-layer particles sit at z = dx / 2: the MOST roughness length must
    # lie below them for the Obukhov-length Newton iteration to exist
    p = default_params(dt=dt, **pkw)
    p.cs_sgs = cs
    p.l2, p.l3, p.l_left, p.l_right = l2, l3, l_left, l_right
    p.outlet_probe_dx = 0.5 * dx
    for k, v in enumerate(boxes[0]):
        p.ib_box[k] = v
    p.most_z0, p.most_z0h = min(z0, 0.1 * dx), 0.01 * dx
    zt = np.linspace(0.5 * dx, nz * dx, 24)
    set_profile(p, zt, ustar / 0.4 * np.log(np.maximum(zt, z0) / z0))
    p.setf("u_limit", 20.0)
    p.setf("time_end", 1e9)
    if not apr:
        domain_setup(p, P)
        return P, p, boxes
    p.apr_max_level = 1
    p.apr_zone = apr_zone
    p.seti("h_change", 1)
    near = np.zeros(len(P), bool)
    fl = P["p_type"] == 1
    for bx0, bx1, by0, by1, bz0, bz1 in boxes:
        d = np.sqrt(np.maximum(np.maximum(bx0 - P["x"], P["x"] - bx1), 0) ** 2 +
                    np.maximum(np.maximum(by0 - P["y"], P["y"] - by1), 0) ** 2 +
                    np.maximum(P["z"] - bz1, 0) ** 2)
        # the pass marks whole NNPS cells within ceil(zone / dcell) cells of a marker cell
        near |= fl & (d <= apr_zone + 2.5 * 1.65 * dx)
    frac = headroom if headroom is not None else 7.2 * near.sum() / len(P)
    P, p = with_headroom(P, p, frac)
    return P, p, boxes


def most_column(dx=1.0, n=6, nz=5, seed=SEED, **pkw):
    """Wall-layer deck at atmospheric heights (z = 1.5 .. 5.5 m above walls)
    where the reference's MOST Newton branch (functions_MOST.cuh:217-247,
    hard-wired z0 = 1 m) converges: stable and unstable wall-layer air."""
    rng = np.random.default_rng(seed)
    f = np.float32
    xs = (np.arange(n) + 0.5) * dx
    fx, fy, fz = _grid(xs, xs, (np.arange(nz) + 1.5) * dx)
    Pf = _records(fx, fy, fz); Pf["p_type"] = 1
    wx, wy, wz = _grid(xs, xs, (0.5 - np.arange(3)) * dx)
    Pw = _records(wx, wy, wz); Pw["p_type"] = 0
    P = np.concatenate([Pf, Pw])
    _common_fields(P, dx)
    fl = P["p_type"] == 1
    zz = P["z"].astype(np.float64)
    u = np.where(fl, 0.3 / 0.4 * np.log(np.maximum(zz, 1.0) / 0.5), 0.0)
    P["ux"] = (u * (1 + 0.05 * rng.uniform(-1, 1, len(P)))).astype(f)
    P["uy"] = (0.1 * u * rng.uniform(-1, 1, len(P))).astype(f)
    most = fl & (P["z"] < 2.0 * dx)
    P["MOST_buffer"][most] = 1
    P["temp"][most] = (300.0 + rng.uniform(-3.0, 3.0, most.sum())).astype(f)
    P = P[rng.permutation(len(P))]
    p = default_params(**pkw)
    p.setf("dt", 1e-3)
    domain_setup(p, P)
    return P, p


def _box_case(n, dx, re, lid, seed, ppe_kw):
    """Cube of n^3 fluid particles inside 3 wall layers; lid-driven (top
    layers moving at U = 1 m/s in x) or a Taylor-Green initial field in a
    walled box.  Dynamic viscosity from Re = rho U L / mu."""
    rng = np.random.default_rng(seed)
    f = np.float32
    L = n * dx
    c = (np.arange(n) + 0.5) * dx
    fx, fy, fz = _grid(c, c, c)
    Pf = _records(fx, fy, fz); Pf["p_type"] = 1
    w = (np.arange(-3, n + 3) + 0.5) * dx
    wx, wy, wz = _grid(w, w, w)
    inside = (wx > 0) & (wx < L) & (wy > 0) & (wy < L) & (wz > 0) & (wz < L)
    Pw = _records(wx[~inside], wy[~inside], wz[~inside]); Pw["p_type"] = 0
    if lid:
        Pw["p_type"][Pw["z"] > L] = 9
    P = np.concatenate([Pf, Pw])
    _common_fields(P, dx)
    fl = P["p_type"] == 1
    if not lid:
        k = 2 * np.pi / L
        x, y, z = (P[a].astype(np.float64) for a in ("x", "y", "z"))
        P["ux"] = np.where(fl, np.sin(k * x) * np.cos(k * y) * np.cos(k * z), 0.0).astype(f)
        P["uy"] = np.where(fl, -np.cos(k * x) * np.sin(k * y) * np.cos(k * z), 0.0).astype(f)
    P = P[rng.permutation(len(P))]
    p = default_params(dt=0.1 * dx, turbulence="Laminar", open_boundary=0, **ppe_kw)
    p.visc_fluid = 1.225 * 1.0 * L / re
    p.boundary_velocity = 1.0
    p.l2, p.l3, p.l_left, p.l_right = -1e9, 1e9, -1e9, 1e9
    p.setf("u_limit", 20.0)
    p.setf("time_end", 1e9)
    domain_setup(p, P)
    return P, p


def cavity(n=30, dx=0.01, re=1000.0, seed=SEED, **kw):
    """Lid-driven cavity: n^3 fluid particles, lid speed 1 m/s."""
    return _box_case(n, dx, re, True, seed, kw)


def tgv_box(n=30, dx=0.01, re=1000.0, seed=SEED, **kw):
    """Taylor-Green initial field in a walled box (the reference's NNPS has
    no triply periodic mode)."""
    return _box_case(n, dx, re, False, seed, kw)


def tgv_periodic(n=64, h_coeff=1.3, kernel="Wendland6", rho=1000.0, nu=1e-3, u0=1.0, seed=SEED, shuffle=True, **kw):
    """Triply periodic Taylor-Green vortex: n^3 particles cell-centred in the
    unit cube (dx = 1/n, h = h_coeff dx), u = U0 sin x cos y cos z,
    v = -U0 cos x sin y cos z, w = 0 with the coordinates mapped to
    [0, 2 pi), density rho, kinematic viscosity nu, dt = 0.1 dx / U0
    (CFL 0.1), and the Taylor-Green pressure of that field.  Three layers of
    periodic ghosts (buffer_type 7) surround the cube, enough for the kernel
    support kappa h = 2.6 dx."""
    rng = np.random.default_rng(seed)
    f = np.float32
    dx = 1.0 / n
    c = (np.arange(-3, n + 3) + 0.5) * dx
    x, y, z = _grid(c, c, c)
    P = _records(x, y, z)
    P["p_type"] = 1
    ghost = (x < 0) | (x > 1) | (y < 0) | (y > 1) | (z < 0) | (z > 1)
    P["buffer_type"][ghost] = BUFFER_PERIODIC_GHOST
    _common_fields(P, dx, h_coeff=h_coeff, rho=rho)
    k = 2 * np.pi
    xd, yd, zd = x.astype(np.float64), y.astype(np.float64), z.astype(np.float64)
    P["ux"] = (u0 * np.sin(k * xd) * np.cos(k * yd) * np.cos(k * zd)).astype(f)
    P["uy"] = (-u0 * np.cos(k * xd) * np.sin(k * yd) * np.cos(k * zd)).astype(f)
    P["pres"] = (rho * u0 * u0 / 16.0 * (np.cos(2 * k * xd) + np.cos(2 * k * yd)) * (np.cos(2 * k * zd) + 2.0)).astype(f)
    if shuffle:
        P = P[rng.permutation(len(P))]
    p = default_params(dt=0.1 * dx / u0, kernel=kernel, turbulence="Laminar", open_boundary=0, noslip=0, **kw)
    p.visc_fluid = nu * rho
    p.rho_air = rho
    p.l2, p.l3, p.l_left, p.l_right = -1e9, 1e9, -1e9, 1e9
    for a, v in enumerate((0.0, 1.0, 0.0, 1.0, 0.0, 1.0)):
        p.periodic_box[a] = v
    p.partner_tol = 1e-3 * dx
    p.setf("u_limit", 20.0 * u0)
    p.setf("time_end", 1e9)
    domain_setup(p, P)
    return P, p


def ensemble(ncase=64, nmin=20000, nmax=200000, dx=0.01, seed=SEED, **kw):
    """Seeded ensemble: case k has N_k ~ U[nmin, nmax] fluid particles (cube
    edge round(N_k^(1/3)) at dx), Re ~ U[100, 2000]; even k lid-driven
    cavity, odd k Taylor-Green box.  Returns [(P, params, meta)]."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(ncase):
        nk = int(rng.integers(nmin, nmax + 1))
        edge = int(round(nk ** (1.0 / 3.0)))
        re = float(rng.uniform(100.0, 2000.0))
        lid = k % 2 == 0
        P, p = (cavity if lid else tgv_box)(n=edge, dx=dx, re=re, seed=seed + k, **kw)
        out.append((P, p, {"kind": "cavity" if lid else "taylor-green", "edge": edge, "re": re,
                           "target_fluid": nk, "particles": len(P)}))
    return out


def nnps_stress(seed=SEED):
    """Small Case-H deck made hard for the cell sort and the lists: scattered
    dummy records (i_type 3), one cell crowded with 150 particles (longer
    than the 64-entry insertion sort), duplicated positions (zero-distance
    pairs) and records on the domain maximum (clamped cell index)."""
    rng = np.random.default_rng(seed)
    P, p = caseh_mini(nx=12, ny=6, nz=5, seed=seed)
    P = P.copy()
    fl = np.where((P["p_type"] == 1) & (P["i_type"] == 1))[0]
    pick = rng.permutation(fl)
    crowd, dup, edge = pick[:150], pick[150:170], pick[170:180]
    # crowd: inside a box a fifth of a cell wide around one fluid particle
    c = pick[200]
    dcell = p.getf("dcell")
    for a in ("x", "y", "z"):
        P[a][crowd] = (P[a][c] + rng.uniform(0.0, 0.2 * dcell, len(crowd))).astype(np.float32)
    # duplicates of other fluid particles
    src = pick[300:320]
    for a in ("x", "y", "z"):
        P[a][dup] = P[a][src]
    # on the domain maximum of each axis (not the last record, which find_minmax skips)
    for a in ("x", "y", "z"):
        P[a][edge[:3]] = P[a][:-1].max()
    # scattered dummies
    dum = rng.choice(len(P) - 1, len(P) // 20, replace=False)
    P["i_type"][dum] = 3
    domain_setup(p, P)
    return P, p


def describe(P):
    counts = {}
    for name, mask in (("fluid", P["p_type"] == 1), ("wall", P["p_type"] == 0),
                       ("moving", P["p_type"] == 9), ("freeslip", P["p_type"] == -1),
                       ("marker", P["p_type"] >= 1000)):
        counts[name] = int(mask.sum())
    return counts
