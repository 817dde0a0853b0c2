// CPU restatement of the reference ISPH step -- TEST INFRASTRUCTURE ONLY.
//
// This is the oracle the CUDA path is checked against.  It restates, in plain
// serial C++, every kernel SOPHIA_single_ISPH (ISPH_Calc.cuh:4-214) launches,
// following each kernel's formula, operand order and float/double promotion
// so that, instantiated with Real = float, it reproduces the reference host
// build (oracle/_ref) bit for bit; with Real = double it is the plain-FP64
// form.  Differences from the reference, all deliberate:
//   * race-free: KERNEL_PPE3D and the ghost read of KERNEL_Neumann_boundary3D
//     see the pre-launch state (Jacobi semantics) instead of racing;
//   * neighbours are visited through explicit per-particle lists built by the
//     reference's own cell loop (same order, same FP32 distance test), and the
//     radius predicates are always evaluated in FP32 from the FP32 positions
//     (the reference's precision), so both precisions see identical lists;
//   * particles with i_type >= 3 (dummies) are not processed by the Neumann
//     pass (the reference runs it on them with meaningless positions);
//   * the converged pressure solves (BiCGSTAB, pinned row) are new work with
//     no reference counterpart;
//   * with the property tables, a record whose |p_type| has no table of two
//     entries keeps its value in htoT / Ttoh (the reference reads past its
//     ten-entry k_table_index there, e.g. for the IBM markers in its
//     conversion kernels).
// Beyond the step it restates the energy conversions of functions_ENERGY.cuh
// (Ttoh / htoT on the records), pinned to the reference's kernels on the
// built-in corium table and on property tables its read_table loaded.
// Nothing here is linked into the product library.

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <math.h>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <functional>
#include <numeric>
#include <type_traits>
#include <vector>

#include "sph_isph.h"

namespace {

// ---- parameter accessors (function_init.cuh:84-163) ------------------------
struct P {
    const sph_params &p;
    int kernel_type() const { return p.vii[3]; }
    int time_type() const { return p.vii[4]; }
    int freq_filt() const { return p.vii[8]; }
    int fp_solve() const { return p.vii[12]; }
    int fv_solve() const { return p.vii[13]; }
    int fg_solve() const { return p.vii[14]; }
    int con_solve() const { return p.vii[15]; }
    int enthalpy_eqn() const { return p.enthalpy_eqn; }
    int prop_table() const { return p.vii[2]; }
    int boussinesq() const { return p.vii[16]; }
    int kgc_solve() const { return p.vii[17]; }
    int turb() const { return p.vii[18]; }
    int concn_solve() const { return p.vii[19]; }
    int NI() const { return p.vii[24]; }
    int NJ() const { return p.vii[25]; }
    int NK() const { return p.vii[26]; }
    int num_cells() const { return p.vii[28]; }
    int n() const { return p.vii[32]; }
    int noslip() const { return p.vii[34]; }
    float kappa() const { return p.vif[0]; }
    float dt() const { return p.vif[2]; }
    float u_limit() const { return p.vif[5]; }
    float xmin() const { return p.vif[9]; }
    float xmax() const { return p.vif[10]; }
    float ymin() const { return p.vif[11]; }
    float ymax() const { return p.vif[12]; }
    float zmin() const { return p.vif[13]; }
    float zmax() const { return p.vif[14]; }
    float skappa() const { return p.vif[17]; }
    float dcell() const { return p.vif[18]; }
    float dt_structure() const { return p.vif[20]; }
};

const double PI_REF = 3.141592653;      // Parameters.cuh:32
const double GRAV = 9.810;              // Parameters.cuh:34
// thermal constants, Parameters.cuh:120-131 (Air_cp is an int literal there)
const double SOLID_CP = 900.0;
const int AIR_CP = 1005;
const double SOLID_K = 1.0;
const double AIR_K = 0.025;
const double SOLID_RHO = 2300.0;
const double TEMPB = 300.0;

// ---- kernel functions, functions_KNL.cuh:2-103 and :326-369 -----------------
template <class Real>
Real calc_tmpA(const P &q, Real tH) {
    const int kt = q.kernel_type();
    const float kap = q.kappa();
    Real tA = 0.0;
    if (kt == 0) tA = 1.0 / (std::pow(PI_REF, 1.5) * std::pow(tH, 3));
    else if (kt == 1) tA = 3.0 / (359.0 * PI_REF * std::pow(tH, 3));
    else if (kt == 2) tA = 315.0 / (208.0 * PI_REF * std::pow(tH, 3));
    else if (kt == 3) tA = 3.342253804929802 / (kap * tH) / (kap * tH) / (kap * tH);
    else if (kt == 4) tA = 4.923856051905513 / (kap * tH) / (kap * tH) / (kap * tH);
    else if (kt == 5) tA = 6.788953041263660 / (kap * tH) / (kap * tH) / (kap * tH);
    return tA;
}

template <class Real>
Real calc_wij(const P &q, Real tA, Real tH, Real rr) {
    const int kt = q.kernel_type();
    const float kap = q.kappa();
    Real tR = rr / tH / kap, wij = 0.0;
    if (kt == 0) {
        wij = tA * std::exp(-std::pow(2.0 * tR, 2));
    } else if (kt == 1) {
        if (tR < 0.5) wij = tA * (std::pow(3.0 - 2.0 * tR, 5) - 6.0 * std::pow(2.0 - 2.0 * tR, 5) + 15.0 * std::pow(1.0 - 2.0 * tR, 5));
        else if (0.5 <= tR && tR < 1) wij = tA * (std::pow(3.0 - 2.0 * tR, 5) - 6.0 * std::pow(2.0 - 2.0 * tR, 5));
        else if (1 <= tR && tR < 1.5) wij = tA * (std::pow(3.0 - 2.0 * tR, 5));
    } else if (kt == 2) {
        wij = (tR < 1) * tA * (2.0 / 3.0 - 9.0 / 2.0 * std::pow(tR, 2) + 19.0 / 3.0 * std::pow(tR, 3) - 5.0 / 2.0 * std::pow(tR, 4));
    } else if (kt == 3) {
        wij = (tR < 1) * tA * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) * (1 + 4 * tR);
    } else if (kt == 4) {
        wij = (tR < 1) * tA * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) * (1 + 6 * tR + 11.666666666666666 * tR * tR);
    } else if (kt == 5) {
        wij = (tR < 1) * tA * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) * (1 + 8 * tR + 25 * tR * tR + 32 * tR * tR * tR);
    }
    return wij;
}

template <class Real>
Real calc_dwij(const P &q, Real tA, Real tH, Real rr) {
    const int kt = q.kernel_type();
    const float kap = q.kappa();
    Real tR = rr / tH / kap, dwij = 0.0;
    if (kt == 0) {
        dwij = (1.0 / tH) * tA * (-2.0) * 2.0 * tR * std::exp(-std::pow(2.0 * tR, 2));
    } else if (kt == 1) {
        if (tR < 0.5) dwij = (1.0 / tH) * tA * (-5.0 * std::pow(3.0 - 2.0 * tR, 4) + 30.0 * std::pow(2.0 - 2.0 * tR, 4) - 75.0 * std::pow(1.0 - 2.0 * tR, 4));
        else if (0.5 <= tR && tR < 1.0) dwij = (1.0 / tH) * tA * (-5.0 * std::pow(3.0 - 2.0 * tR, 4) + 30.0 * std::pow(2.0 - 2.0 * tR, 4));
        else if (1.0 <= tR && tR < 1.5) dwij = (1.0 / tH) * tA * (-5.0 * std::pow(3.0 - 2.0 * tR, 4));
    } else if (kt == 2) {
        dwij = (tR < 1) * (1.0 / tH) * tA * (-9.0 / 2.0 * 2 * tR + 19.0 / 3.0 * 3.0 * std::pow(tR, 2) - 5.0 / 2.0 * 4.0 * std::pow(tR, 3));
    } else if (kt == 3) {
        dwij = (tR < 1) * (1 / (kap * tH)) * tA * (-20 * tR * (1 - tR) * (1 - tR) * (1 - tR));
    } else if (kt == 4) {
        dwij = (tR < 1) * (1 / (kap * tH)) * tA * (-18.666666666666668 * tR * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) * (5 * tR + 1));
    } else if (kt == 5) {
        dwij = (tR < 1) * (1 / (kap * tH)) * tA * (-22 * tR * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) * (16 * tR * tR + 7 * tR + 1));
    }
    return dwij;
}

// Wendland-6 shape with the kernel_type normalisation, functions_KNL.cuh:339-369
template <class Real>
Real calc_wij_pressure(const P &q, Real tA, Real tH, Real rr) {
    const float kap = q.kappa();
    Real tR = rr / tH / kap;
    return (tR < 1) * tA * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) * (1 + 8 * tR + 25 * tR * tR + 32 * tR * tR * tR);
}
template <class Real>
Real calc_dwij_pressure(const P &q, Real tA, Real tH, Real rr) {
    const float kap = q.kappa();
    Real tR = rr / tH / kap;
    return (tR < 1) * (1 / (kap * tH)) * tA * (-22 * tR * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) * (16 * tR * tR + 7 * tR + 1));
}

// viscosity2, functions_PROP.cuh:121-131 (the temperature argument is unused)
template <class Real>
Real viscosity2(const sph_params &p, int p_type) {
    Real vis;
    if (p_type == 1) vis = (float)p.visc_fluid;
    else if (p_type == 0) vis = (float)p.visc_wall;
    else if (p_type == 1000) vis = (float)p.visc_marker;
    else vis = (float)p.visc_fluid;
    return vis;
}

// ---- particle state -----------------------------------------------------------
template <class Real>
struct State {
    int n = 0;
    std::vector<int> i_type, buffer_type, most, p_type, ncell, source;
    std::vector<Real> x, y, z, ux, uy, uz, m, h, temp, pres, pres0, rho, flt_s, enthalpy, concn,
        concentration, k_turb, e_turb, eli, vol, m_ref, h_ref, vis_t, fbx, fby, fbz, fmx, fmy,
        hmz, f1, f2, f3;
    void resize(int nn) {
        n = nn;
        for (auto *v : {&i_type, &buffer_type, &most, &p_type, &ncell, &source}) v->assign(n, 0);
        for (auto *v : reals()) v->assign(n, Real(0));
    }
    std::vector<std::vector<Real> *> reals() {
        return {&x, &y, &z, &ux, &uy, &uz, &m, &h, &temp, &pres, &pres0, &rho, &flt_s, &enthalpy,
                &concn, &concentration, &k_turb, &e_turb, &eli, &vol, &m_ref, &h_ref, &vis_t,
                &fbx, &fby, &fbz, &fmx, &fmy, &hmz, &f1, &f2, &f3};
    }
};

template <class Real>
struct P2State {
    std::vector<Real> rho_ref, SR, x0, y0, z0, ux0, uy0, uz0, temp0, concn0, enthalpy0;
    void resize(int n) {
        for (auto *v : {&rho_ref, &SR, &x0, &y0, &z0, &ux0, &uy0, &uz0, &temp0, &concn0, &enthalpy0})
            v->assign(n, Real(0));
    }
};

// interp2 (functions_PROP.cuh:8-41) over n >= 2 points, in the reference's
// Real arithmetic: linear inside the table, the end segments extended
// outside it.  Each segment's slope multiplies the distance from its left
// point, except past the last point, where the reference measures from the
// last point and adds its value (:16-21; equal in exact arithmetic, not in
// rounding).  The reference's search loop also tests the pair (n-1, n), one
// entry past the table, but only for an x it cannot bracket, which a table
// with increasing x_data does not leave (NaN x leaves its result unset;
// here it is the last value).
template <class Real>
static Real interp2(const Real *xd, const Real *yd, int n, Real x) {
    auto seg = [&](int a, int at) {
        Real y = yd[a + 1] - yd[a];
        y /= (xd[a + 1] - xd[a]);
        y *= (x - xd[at]);
        y += yd[at];
        return y;
    };
    const int e = n - 1;
    if (xd[e] < x) return seg(e - 1, e);
    if (x <= xd[0]) return seg(0, 0);
    for (int a = 0; a < e; ++a)
        if (xd[a] < x && x <= xd[a + 1]) return seg(a, a);
    return yd[e];
}

// htoT (functions_PROP.cuh:43-67): with prop_table = 0 the built-in corium
// table, with prop_table = 1 table |p_type| of the property tables (the
// device copies k_Tab_h / k_Tab_T at k_table_index, k_table_size).  A slot
// without a table of two entries leaves the temperature as it was (the
// library refuses such a step before it runs).
template <class Real>
struct PropTables {
    bool set = false;
    Real h[SPH_TABLE_SIZE] = {}, T[SPH_TABLE_SIZE] = {};
    int index[SPH_TABLE_SLOTS] = {}, size[SPH_TABLE_SLOTS] = {};
};
template <class Real>
static Real htoT(Real h, int p_type, bool prop_table, const PropTables<Real> &tab, Real keep) {
    static const Real xd[5] = {Real(-554932), Real(215789), Real(757894), Real(905263), Real(1268421)};
    static const Real yd[5] = {Real(280), Real(1537), Real(2300), Real(2450), Real(2650)};
    if (!prop_table) return interp2<Real>(xd, yd, 5, h);
    const int t = p_type < 0 ? -p_type : p_type;
    if (t >= SPH_TABLE_SLOTS || tab.size[t] < 2) return keep;
    return interp2<Real>(tab.h + tab.index[t], tab.T + tab.index[t], tab.size[t], h);
}

// Ttoh (functions_PROP.cuh:69-93): the inverse lookup, T to h, on the same
// tables (the built-in corium pairs with the columns swapped, or table
// |p_type| with k_Tab_T as x and k_Tab_h as y)
template <class Real>
static Real Ttoh(Real T, int p_type, bool prop_table, const PropTables<Real> &tab, Real keep) {
    static const Real xd[5] = {Real(280), Real(1537), Real(2300), Real(2450), Real(2650)};
    static const Real yd[5] = {Real(-554932), Real(215789), Real(757894), Real(905263), Real(1268421)};
    if (!prop_table) return interp2<Real>(xd, yd, 5, T);
    const int t = p_type < 0 ? -p_type : p_type;
    if (t >= SPH_TABLE_SLOTS || tab.size[t] < 2) return keep;
    return interp2<Real>(tab.T + tab.index[t], tab.h + tab.index[t], tab.size[t], T);
}

template <class Real>
struct P3State {
    std::vector<Real> ftx, fty, ftz, ft, fpx, fpy, fpz, dtemp, dconcn, denthalpy, nx, ny, nz, gxx, gyy, gzz, gxy,
        gyz, gzx;
    void reset(int n) {
        for (auto *v : {&ftx, &fty, &ftz, &ft, &fpx, &fpy, &fpz, &dtemp, &dconcn, &denthalpy, &nx, &ny, &nz, &gxx,
                        &gyy, &gzz, &gxy, &gyz, &gzx})
            v->assign(n, Real(0));
    }
};

// ---- cell helpers ----------------------------------------------------------
// binning formula, functions_NNPS.cuh:890-898
inline int bin_axis(float v, float vmin, float vmax, int N) {
    if (vmax == vmin) return 0;
    float t = std::floor((v - vmin) / (vmax - vmin) * N);
    int c = (int)((t < (float)(N - 1)) ? t : (float)(N - 1));
    return c < 0 ? 0 : c;
}
// search formula, functions_PPE.cuh:52-59
inline int search_axis(float v, float vmin, float vmax, float dcell, int N) {
    if (vmax == vmin) return 0;
    float t = std::floor((v - vmin) / dcell);
    int c = (int)((t < (float)(N - 1)) ? t : (float)(N - 1));
    return c < 0 ? 0 : c;
}
inline float d2f(float xi, float yi, float zi, float xj, float yj, float zj) {
    return (xi - xj) * (xi - xj) + (yi - yj) * (yi - yj) + (zi - zj) * (zi - zj);
}

template <class Real>
struct Oracle {
    sph_params prm;
    int prec;
    State<Real> S1, S;      // dev_P1, dev_SP1
    P2State<Real> S2;       // dev_SP2 (P2 keeps only rho_ref between steps)
    std::vector<Real> p2_rho_ref;
    P3State<Real> S3;
    PropTables<Real> tab;               // k_Tab_h / k_Tab_T, k_table_index / k_table_size
    std::vector<float> xf, yf, zf, hf;   // FP32 positions / h, sorted (NNPS precision)
    std::vector<int> g_idx, p_idx, g_str, g_end;
    std::vector<int64_t> nb_off;
    std::vector<int> nb;                 // canonical list: r < kappa*max(hi,hj)
    std::vector<int64_t> nm_off;         // Neumann candidate list (2h, ghost node)
    std::vector<int> nm;
    bool built = false;
    int count = 0;
    float time = 0.f;
    float us_update = 0.f;        // u* of the recycling probe (a device global there)
    int pin_row = -1;
    std::vector<int> pins;
    std::vector<int> comp_of;     // rank-one component of each fluid row (-1: none)
    std::vector<int> comp_size;
    int stop_after = 1000;   // debugging: phases of step() to run

    P q() const { return P{prm}; }
    int n() const { return prm.vii[32]; }

    // -------------------------------------------------------------------------
    void upload(const sph_part1 *A, int nn) {
        S1.resize(nn);
        for (int i = 0; i < nn; ++i) {
            const sph_part1 &r = A[i];
            S1.i_type[i] = r.i_type; S1.buffer_type[i] = r.buffer_type; S1.most[i] = r.MOST_buffer;
            S1.p_type[i] = r.p_type; S1.ncell[i] = r.ncell; S1.source[i] = r.source;
            S1.x[i] = r.x; S1.y[i] = r.y; S1.z[i] = r.z; S1.ux[i] = r.ux; S1.uy[i] = r.uy; S1.uz[i] = r.uz;
            S1.m[i] = r.m; S1.h[i] = r.h; S1.temp[i] = r.temp; S1.pres[i] = r.pres; S1.pres0[i] = r.pres0;
            S1.rho[i] = r.rho; S1.flt_s[i] = r.flt_s; S1.enthalpy[i] = r.enthalpy; S1.concn[i] = r.concn;
            S1.concentration[i] = r.concentration; S1.k_turb[i] = r.k_turb; S1.e_turb[i] = r.e_turb;
            S1.eli[i] = r.eli; S1.vol[i] = r.vol; S1.m_ref[i] = r.m_ref; S1.h_ref[i] = r.h_ref;
            S1.vis_t[i] = r.vis_t; S1.fbx[i] = r.fbx; S1.fby[i] = r.fby; S1.fbz[i] = r.fbz;
            S1.fmx[i] = r.fmx; S1.fmy[i] = r.fmy; S1.hmz[i] = r.hmz; S1.f1[i] = r.float1;
            S1.f2[i] = r.float2; S1.f3[i] = r.float3;
        }
        xf.resize(nn); yf.resize(nn); zf.resize(nn); hf.resize(nn);
        for (int i = 0; i < nn; ++i) { xf[i] = A[i].x; yf[i] = A[i].y; zf[i] = A[i].z; hf[i] = A[i].h; }
        S2.resize(nn);
        p2_rho_ref.assign(nn, Real(0));
        S3.reset(nn);
        count = prm.vii[27];
        time = prm.vif[3];
        built = false;
    }

    // KERNEL_set_ncell, functions_NNPS.cuh:943-955 (FP32 as the reference)
    void set_ncell(State<Real> &A) {
        for (int i = 0; i < n(); ++i) {
            if (A.i_type[i] == 3) continue;
            float h0 = (float)A.h_ref[i], h = hf[i];
            A.ncell[i] = (int)(1.0 * std::ceil(float(2) / float(h0 / h)));
        }
    }

    // hash + stable sort + reorder + lists, ISPH_Calc.cuh:23-45
    void nnps() {
        const P Q = q();
        const int N = n();
        set_ncell(S1);
        std::vector<int> key(N);
        for (int i = 0; i < N; ++i) {
            if (S1.i_type[i] == 3) { key[i] = Q.num_cells(); continue; }
            int ic = bin_axis(xf[i], Q.xmin(), Q.xmax(), Q.NI());
            int jc = bin_axis(yf[i], Q.ymin(), Q.ymax(), Q.NJ());
            int kc = bin_axis(zf[i], Q.zmin(), Q.zmax(), Q.NK());
            key[i] = ic + Q.NI() * jc + Q.NI() * Q.NJ() * kc;
        }
        std::vector<int> order(N);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return key[a] < key[b]; });
        g_idx.resize(N); p_idx.resize(N);
        g_str.assign(Q.num_cells() + 1, -1);
        g_end.assign(Q.num_cells() + 1, 0);
        for (int s = 0; s < N; ++s) { g_idx[s] = key[order[s]]; p_idx[s] = order[s]; }
        for (int s = 0; s < N; ++s) {
            if (s == 0 || g_idx[s] != g_idx[s - 1]) {
                g_str[g_idx[s]] = s;
                if (s > 0) g_end[g_idx[s - 1]] = s;
            }
        }
        if (N > 0) g_end[g_idx[N - 1]] = N;
        // reorder (P1 <- SP1 at step 0, ISPH_Calc.cuh:45)
        State<Real> T = S1;
        std::vector<float> txf = xf, tyf = yf, tzf = zf, thf = hf;
        auto perm_i = [&](std::vector<int> &dst, const std::vector<int> &src) { for (int s = 0; s < N; ++s) dst[s] = src[order[s]]; };
        auto perm_r = [&](std::vector<Real> &dst, const std::vector<Real> &src) { for (int s = 0; s < N; ++s) dst[s] = src[order[s]]; };
        perm_i(S1.i_type, T.i_type); perm_i(S1.buffer_type, T.buffer_type); perm_i(S1.most, T.most);
        perm_i(S1.p_type, T.p_type); perm_i(S1.ncell, T.ncell); perm_i(S1.source, T.source);
        auto dr = S1.reals(); auto sr = T.reals();
        for (size_t k = 0; k < dr.size(); ++k) perm_r(*dr[k], *sr[k]);
        for (int s = 0; s < N; ++s) { xf[s] = txf[order[s]]; yf[s] = tyf[order[s]]; zf[s] = tzf[order[s]]; hf[s] = thf[order[s]]; }
        std::vector<Real> rr = p2_rho_ref;
        for (int s = 0; s < N; ++s) p2_rho_ref[s] = rr[order[s]];
        build_lists();
        built = true;
    }

    template <class F>
    void cell_loop(int ic, int jc, int kc, int nc, F f) const {
        const P Q = q();
        for (int z = -nc; z <= nc; z++)
            for (int y = -nc; y <= nc; y++)
                for (int x = -nc; x <= nc; x++) {
                    int k = (ic + x) + Q.NI() * (jc + y) + Q.NI() * Q.NJ() * (kc + z);
                    if (ic + x < 0 || ic + x > Q.NI() - 1 || jc + y < 0 || jc + y > Q.NJ() - 1 || kc + z < 0 || kc + z > Q.NK() - 1) continue;
                    if (g_str[k] == -1) continue;
                    for (int j = g_str[k]; j < g_end[k]; j++) f(j);
                }
    }

    void search_cell(float x, float y, float z, int &ic, int &jc, int &kc) const {
        const P Q = q();
        ic = search_axis(x, Q.xmin(), Q.xmax(), Q.dcell(), Q.NI());
        jc = search_axis(y, Q.ymin(), Q.ymax(), Q.dcell(), Q.NJ());
        kc = search_axis(z, Q.zmin(), Q.zmax(), Q.dcell(), Q.NK());
    }

    // rows are independent: a counting pass and a filling pass, each over
    // rows in parallel, give the same list as one serial pass
    void build_lists() {
        const P Q = q();
        const int N = n();
        nb_off.assign(N + 1, 0);
        auto visit = [&](int i, auto &&emit) {
            if (S1.i_type[i] == 3) return;   // not in any cell, never a neighbour
            int ic, jc, kc;
            search_cell(xf[i], yf[i], zf[i], ic, jc, kc);
            cell_loop(ic, jc, kc, S1.ncell[i], [&](int j) {
                float tdist = std::sqrt(d2f(xf[i], yf[i], zf[i], xf[j], yf[j], zf[j]));
                if (tdist < Q.skappa() * std::fmax(hf[i], hf[j])) emit(j);
            });
        };
#pragma omp parallel for schedule(dynamic, 1024)
        for (int i = 0; i < N; ++i) {
            int64_t c = 0;
            visit(i, [&](int) { ++c; });
            nb_off[i + 1] = c;
        }
        for (int i = 0; i < N; ++i) nb_off[i + 1] += nb_off[i];
        nb.assign((size_t)nb_off[N], 0);
#pragma omp parallel for schedule(dynamic, 1024)
        for (int i = 0; i < N; ++i) {
            int64_t e = nb_off[i];
            visit(i, [&](int j) { nb[(size_t)e++] = j; });
        }
    }

    // ---- passes ----------------------------------------------------------------
    // KERNEL_clc_gradient_correction_3D, functions_KNL.cuh:216-324
    void gradient_correction(State<Real> &A) {
        const P Q = q();
        for (int i = 0; i < n(); ++i) {
            if (A.i_type[i] == 3) { set_identity(i); continue; }
            int ptype_i = A.p_type[i];
            Real hi = A.h[i];
            Real tmp_A = calc_tmpA(Q, hi);
            Real xi = A.x[i], yi = A.y[i], zi = A.z[i];
            Real txx = 0, tyy = 0, tzz = 0, txy = 0, tyz = 0, tzx = 0;
            for (int64_t e = nb_off[i]; e < nb_off[i + 1]; ++e) {
                int j = nb[e];
                float tdf = std::sqrt(d2f(xf[i], yf[i], zf[i], xf[j], yf[j], zf[j]));
                if (!(tdf > 0 && tdf < Q.skappa() * hf[i])) continue;
                Real xj = A.x[j], yj = A.y[j], zj = A.z[j];
                int ptype_j = A.p_type[j];
                Real tdist = std::sqrt((xi - xj) * (xi - xj) + (yi - yj) * (yi - yj) + (zi - zj) * (zi - zj));
                Real tdwij = calc_dwij(Q, tmp_A, hi, tdist);
                Real mj = A.m[j], rhoj = A.rho[j];
                Real mtd = mj * tdwij;
                Real rtd = 1.0 / (rhoj * tdist);
                Real a = -mtd * (xi - xj) * (xi - xj); a *= rtd;
                Real b = -mtd * (yi - yj) * (xi - xj); b *= rtd;
                Real c = -mtd * (yi - yj) * (yi - yj); c *= rtd;
                Real d = -mtd * (xi - xj) * (zi - zj); d *= rtd;
                Real e2 = -mtd * (yi - yj) * (zi - zj); e2 *= rtd;
                Real f = -mtd * (zi - zj) * (zi - zj); f *= rtd;
                txx += a * (ptype_j == 1); txy += b * (ptype_j == 1); tyy += c * (ptype_j == 1);
                tzx += d * (ptype_j == 1); tyz += e2 * (ptype_j == 1); tzz += f * (ptype_j == 1);
            }
            Real det = txx * (tyy * tzz - tyz * tyz);
            det -= txy * (txy * tzz - tyz * tzx);
            det += tzx * (txy * tyz - tyy * tzx);
            if ((std::abs(det) > DBL_EPSILON) && (ptype_i == 1)) {
                Real r = 1.0 / det;
                S3.gxx[i] = (tyy * tzz - tyz * tyz) * r;
                S3.gxy[i] = (tzx * tyz - txy * tzz) * r;
                S3.gzx[i] = (txy * tyz - tzx * tyy) * r;
                S3.gyy[i] = (txx * tzz - tzx * tzx) * r;
                S3.gyz[i] = (tzx * txy - txx * tyz) * r;
                S3.gzz[i] = (txx * tyy - txy * txy) * r;
            } else {
                set_identity(i);
            }
        }
    }
    void set_identity(int i) {
        S3.gxx[i] = 1; S3.gxy[i] = 0; S3.gzx[i] = 0; S3.gyy[i] = 1; S3.gyz[i] = 0; S3.gzz[i] = 1;
    }

    // KERNEL_clc_prep3D, functions_PREP.cuh:287-488 (SSM and DDF branches)
    void prep(State<Real> &A, int tcount, Real tdt) {
        const P Q = q();
        std::vector<Real> new_vis = A.vis_t, new_k = A.k_turb, new_e = A.e_turb, new_flt = A.flt_s;
        for (int i = 0; i < n(); ++i) {
            if (A.i_type[i] > 2 || A.p_type[i] >= 1000 || A.p_type[i] <= 0) continue;
            Real mi = A.m[i], rhoi = A.rho[i];
            Real ki = std::fmax(A.k_turb[i], 0.0);
            Real nui = A.vis_t[i];
            Real gc11 = S3.gxx[i], gc12 = S3.gxy[i], gc22 = S3.gyy[i], gc23 = S3.gyz[i], gc31 = S3.gzx[i], gc33 = S3.gzz[i];
            Real xi = A.x[i], yi = A.y[i], zi = A.z[i], uxi = A.ux[i], uyi = A.uy[i], uzi = A.uz[i];
            Real hi = A.h[i];
            Real tmp_A = calc_tmpA(Q, hi);
            Real tmp_flt = 0, tmp_SR = 0, tmp_sigma = 0, tvis_t = 0;
            Real st11 = 0, st12 = 0, st22 = 0, st23 = 0, st31 = 0, st33 = 0;
            for (int64_t e = nb_off[i]; e < nb_off[i + 1]; ++e) {
                int j = nb[e];
                float tdf = std::sqrt(d2f(xf[i], yf[i], zf[i], xf[j], yf[j], zf[j]));
                if (!(tdf < Q.skappa() * hf[i])) continue;
                Real xj = A.x[j], yj = A.y[j], zj = A.z[j], uxj = A.ux[j], uyj = A.uy[j], uzj = A.uz[j];
                Real mj = A.m[j], rhoj = A.rho[j];
                int ptypej = A.p_type[j];
                Real tdist = std::sqrt((xi - xj) * (xi - xj) + (yi - yj) * (yi - yj) + (zi - zj) * (zi - zj)) + 1e-20;
                Real tmp_wij = calc_wij(Q, tmp_A, hi, tdist);
                Real tmp_dwij = calc_dwij(Q, tmp_A, hi, tdist);
                Real tdwx = tmp_dwij * (xi - xj) / tdist;
                Real tdwy = tmp_dwij * (yi - yj) / tdist;
                Real tdwz = tmp_dwij * (zi - zj) / tdist;
                if ((tcount % Q.freq_filt()) == 0) tmp_flt += mj / rhoj * tmp_wij;
                if (Q.fv_solve() != 0 && Q.turb() != 0) {
                    tmp_sigma += tdist * tdist * tmp_wij * mj / rhoj;
                    if (ptypej == 1) {
                        Real tdwxc = gc11 * tdwx + gc12 * tdwy + gc31 * tdwz;
                        Real tdwyc = gc12 * tdwx + gc22 * tdwy + gc23 * tdwz;
                        Real tdwzc = gc31 * tdwx + gc23 * tdwy + gc33 * tdwz;
                        st11 += mj / rhoj * (uxj - uxi) * tdwxc;
                        st12 += 0.5 * mj / rhoj * ((uxj - uxi) * tdwyc + (uyj - uyi) * tdwxc);
                        st22 += mj / rhoj * (uyj - uyi) * tdwyc;
                        st23 += 0.5 * mj / rhoj * ((uyj - uyi) * tdwzc + (uzj - uzi) * tdwyc);
                        st31 += 0.5 * mj / rhoj * ((uxj - uxi) * tdwzc + (uzj - uzi) * tdwxc);
                        st33 += mj / rhoj * (uzj - uzi) * tdwzc;
                    }
                }
            }
            if (Q.fv_solve() != 0 && Q.turb() != 0) {
                tmp_SR = 2 * (st11 * st11 + st22 * st22 + st33 * st33 + 2 * st12 * st12 + 2 * st31 * st31 + 2 * st23 * st23);
                tmp_SR = std::sqrt(tmp_SR);
                S2.SR[i] = tmp_SR;
                tmp_sigma = 0.3333 * tmp_sigma;
                tmp_sigma = std::sqrt(tmp_sigma);
                Real tmp_cl = (tmp_sigma > hi) ? tmp_sigma : hi;
                if (Q.turb() == 4) {
                    tvis_t = prm.cs_sgs * prm.cs_sgs * tmp_cl * tmp_cl * tmp_SR;
                    if (A.buffer_type[i] != 1) new_vis[i] = tvis_t;
                } else if (Q.turb() == 5) {
                    Real pp = nui * tmp_SR * tmp_SR;
                    Real b = 0.0;
                    Real eps = 0.93 * ki * std::sqrt(ki) / tmp_cl;     // Ce_sgs, Parameters.cuh:133
                    Real dk = pp + b - eps + Real(0);
                    ki += dk * tdt;
                    ki = (ki > 1e-4) ? ki : (Real)1e-4;
                    tvis_t = 0.1 * tmp_cl * std::sqrt(ki);               // Ck_sgs, Parameters.cuh:132
                    if (A.buffer_type[i] != 1) { new_vis[i] = tvis_t; new_k[i] = ki; new_e[i] = eps; }
                }
            }
            if (tcount == 0) S2.rho_ref[i] = A.rho[i];
            if ((tcount % Q.freq_filt()) == 0) new_flt[i] = tmp_flt;
        }
        A.vis_t = new_vis; A.k_turb = new_k; A.e_turb = new_e; A.flt_s = new_flt;
    }

    // KERNEL_boundary3D, functions_BC.cuh:100-190
    void boundary(State<Real> &A) {
        const P Q = q();
        std::vector<Real> nux = A.ux, nuy = A.uy, nuz = A.uz;
        for (int i = 0; i < n(); ++i) {
            if (A.i_type[i] > 2) continue;
            int pti = A.p_type[i];
            if (pti > 0) continue;
            Real hi = A.h[i];
            Real tmp_A = calc_tmpA(Q, hi);
            Real xi = A.x[i], yi = A.y[i], zi = A.z[i], uxi = A.ux[i];
            Real tx = 0, ty = 0, tz = 0, flt = 1.0e-10;
            for (int64_t e = nb_off[i]; e < nb_off[i + 1]; ++e) {
                int j = nb[e];
                float tdf = std::sqrt(d2f(xf[i], yf[i], zf[i], xf[j], yf[j], zf[j]));
                if (!(tdf < Q.skappa() * hf[i])) continue;
                Real xj = A.x[j], yj = A.y[j], zj = A.z[j];
                Real tdist = std::sqrt((xi - xj) * (xi - xj) + (yi - yj) * (yi - yj) + (zi - zj) * (zi - zj)) - 1e-20;
                Real twij = calc_wij(Q, tmp_A, hi, tdist);
                int ptj = A.p_type[j];
                if (Q.noslip() == 1 && (ptj > 0) & (ptj != 9)) {
                    tx += A.ux[j] * twij; ty += A.uy[j] * twij; tz += A.uz[j] * twij; flt += twij;
                }
            }
            (void)uxi;
            if (Q.noslip() == 1 && (pti == 0 || pti == 9)) {
                nux[i] = 2 * A.ux[i] * (pti == 9) - tx / flt;
                nuy[i] = 2 * A.uy[i] * (pti == 9) - ty / flt;
                nuz[i] = 2 * A.uz[i] * (pti == 9) - tz / flt;
            }
        }
        A.ux = nux; A.uy = nuy; A.uz = nuz;
    }

    // KERNEL_MOST_boundary3D, functions_MOST.cuh:151-322 (float as written)
    static float clampf(float v, float lo, float hi) { return std::fmax(lo, std::fmin(v, hi)); }
    static double psi_m(float zeta) {
        if (zeta < 0.0f) {
            float xx = sqrtf(sqrtf(1.0f - 16.0f * zeta));
            return M_PI * 0.5f - 2.0f * atanf(xx) + logf((1.0f + xx) * (1.0f + xx) * (1.0f + xx * xx) * 0.125f);
        }
        return -5.0f * zeta;
    }
    static double psi_h(float zeta) {
        if (zeta < 0.0f) return 2.0f * logf(0.5f * (1.0f + sqrtf(1.0f - 16.0f * zeta)));
        return -5.0f * zeta;
    }
    static double Phi_m(float L, float zz, float z0) { return logf(zz / z0) - psi_m(zz / L) + psi_m(z0 / L); }
    static double Phi_h(float L, float zz, float z0h) { return logf(zz / z0h) - psi_h(zz / L) + psi_h(z0h / L); }

    void most(State<Real> &A, int tcount, float tdt) {
        const P Q = q();
        for (int i = 0; i < n(); ++i) {
            if (A.most[i] != 1) continue;
            Real xi = A.x[i], yi = A.y[i], zi = A.z[i], uxi = A.ux[i], uyi = A.uy[i];
            Real tempi = A.temp[i], rhoi = A.rho[i], mi = A.m[i];
            Real space = A.h[i] / 1.5;                       // h_coeff, Parameters.cuh:68
            float z0 = (float)prm.most_z0, z0h = (float)prm.most_z0h;
            float u_star = 0.0, theta_star = 0.0, OB_length;
            float theta_surface;
            if (tdt * tcount >= prm.t_start && tdt * tcount < prm.t_con_t) theta_surface = prm.t_ini + tdt * tcount * (prm.t_con - prm.t_ini) / (prm.t_con_t - prm.t_start);
            else if (tdt * tcount < prm.t_start) theta_surface = prm.t_ini;
            else theta_surface = prm.t_con;
            float ws = sqrtf((float)(uxi * uxi + uyi * uyi));
            ws = clampf(ws, 0.001, 100.0);
            float ziF = (float)zi, tempiF = (float)tempi;
            float Ri_b = (GRAV / tempiF) * (tempiF - theta_surface) * ziF / (ws * ws + 1e-10);
            if (std::abs(Ri_b) > 1e-3) {
                OB_length = ziF / Ri_b;
                OB_length = clampf(OB_length, -500.0, 500.0);
                for (int iter = 0; iter < 200; iter++) {
                    float ol_m = OB_length, ol_l = 0.999 * ol_m, ol_u = 1.001 * ol_m;
                    float fL = Ri_b - (ziF / ol_m) * Phi_h(ol_m, ziF, z0h) / powf(Phi_m(ol_m, ziF, z0), 2);
                    float dfL = ((-(ziF / ol_u) * Phi_h(ol_u, ziF, z0h) / (Phi_m(ol_u, ziF, z0) * Phi_m(ol_u, ziF, z0))) -
                                 (-(ziF / ol_l) * Phi_h(ol_l, ziF, z0h) / (Phi_m(ol_l, ziF, z0) * Phi_m(ol_l, ziF, z0)))) / (ol_u - ol_l);
                    OB_length -= 1.0f * fL / dfL;
                    if (fabsf(OB_length) > 1e-6) {
                        if (fabsf((OB_length - ol_m) / OB_length) < 1e-5) break;
                        else if (fabsf(OB_length - ol_m) < 1e-5) break;
                    }
                }
                u_star = 0.4 * ws / Phi_m(OB_length, ziF, z0);
                theta_star = 0.4 * (tempiF - theta_surface) / Phi_h(OB_length, ziF, z0h);
            } else {
                OB_length = 1e6;
                u_star = 0.4 * ws / logf(ziF / z0);
                theta_star = 0.4 * (tempiF - theta_surface) / logf(ziF / z0h);
            }
            float momentum_x = -rhoi * u_star * (uxi * u_star / ws);
            float momentum_y = -rhoi * u_star * (uyi * u_star / ws);
            Real shf = -rhoi * 1005 * u_star * theta_star * 100.0;   // Air_cp, Parameters.cuh:119
            // ghost node 5 m above: neighbours within ghost_tol receive heat flux
            float xg = (float)xi, yg = (float)yi, zg = (float)(zi + prm.most_ghost_dz);
            int ic, jc, kc;
            search_cell(xg, yg, zg, ic, jc, kc);
            cell_loop(ic, jc, kc, 1, [&](int j) {
                Real tdist = std::sqrt((xg - A.x[j]) * (xg - A.x[j]) + (yg - A.y[j]) * (yg - A.y[j]) + (zg - A.z[j]) * (zg - A.z[j])) - 1e-20;
                if (tdist < prm.ghost_tol) {
                    S3.dtemp[j] += 0.5 * shf / (space * rhoi * 1005);
                    A.hmz[j] = 0.5 * shf / (space * rhoi * 1005);
                }
            });
            A.fmx[i] = 1.0 * momentum_x * space * space / mi;
            A.fmy[i] = 1.0 * momentum_y * space * space / mi;
            S3.dtemp[i] += 0.5 * shf / (space * rhoi * 1005);
            A.hmz[i] = 0.5 * shf / (space * rhoi * 1005);
            A.f1[i] = u_star; A.f2[i] = theta_star; A.f3[i] = OB_length;
            // functions_MOST.cuh:316 (probe 600, 0 there)
            const double dxp = (double)xf[i] - prm.recycle_probe_x;
            const float dyp = yf[i] - (float)prm.recycle_probe_y;
            if (dxp * dxp + dyp * dyp < 1e-3) us_update = u_star;
        }
    }

    // KERNEL_Neumann_boundary3D, functions_BC.cuh:290-446 (snapshot semantics)
    void neumann(State<Real> &A) {
        const P Q = q();
        State<Real> O = A;     // pre-launch state
        for (int i = 0; i < n(); ++i) {
            if (O.p_type[i] == 1) continue;
            if (O.i_type[i] >= 3) continue;
            float search_coeff = (float)prm.neumann_coeff;
            Real hi = search_coeff * O.h[i];
            Real tmp_A = calc_tmpA(Q, hi);
            float srange = Q.skappa() * (float)(search_coeff * hf[i]);
            Real xi = O.x[i], yi = O.y[i], zi = O.z[i];
            bool mirror = (O.buffer_type[i] == 1 || O.buffer_type[i] == -1);
            Real xg = mirror ? (Real)(2.0 * prm.l2 - xi) : xi, yg = yi, zg = zi;
            float xgf = mirror ? (float)(2.0 * prm.l2 - xf[i]) : xf[i], ygf = yf[i], zgf = zf[i];
            int ic, jc, kc;
            search_cell(xgf, ygf, zgf, ic, jc, kc);
            Real pres_g = 0;
            cell_loop(ic, jc, kc, 1, [&](int j) {
                Real dist = std::sqrt((xg - O.x[j]) * (xg - O.x[j]) + (yg - O.y[j]) * (yg - O.y[j]) + (zg - O.z[j]) * (zg - O.z[j])) - 1e-20;
                if (dist < prm.ghost_tol) pres_g = O.pres[j];
            });
            Real tpres = 0, tux = 0, tuy = 0, tuz = 0, tflt = 0, gpx = 0, gpy = 0, gpz = 0;
            cell_loop(ic, jc, kc, O.ncell[i], [&](int j) {
                if (O.p_type[j] >= 1000) return;
                float tdf = std::sqrt(d2f(xgf, ygf, zgf, xf[j], yf[j], zf[j]));
                if (!(tdf < srange)) return;
                Real xj = O.x[j], yj = O.y[j], zj = O.z[j];
                Real tdist = std::sqrt((xg - xj) * (xg - xj) + (yg - yj) * (yg - yj) + (zg - zj) * (zg - zj)) - 1e-20;
                Real twij = calc_wij(Q, tmp_A, hi, tdist);
                Real tdwij = calc_dwij(Q, tmp_A, hi, tdist);
                Real tdwx = (xg - xj) / tdist * tdwij, tdwy = (yg - yj) / tdist * tdwij, tdwz = (zg - zj) / tdist * tdwij;
                if (Q.kgc_solve() == 1) { tdwx = 0; tdwy = 0; tdwz = 0; }   // Cm is never filled (all zero)
                Real mj = O.m[j], rhoj = O.rho[j], presj = O.pres[j];
                Real neighbor = (O.p_type[j] == 1) * (O.buffer_type[j] == 0);
                tpres += mj / rhoj * presj * twij * neighbor;
                tux += mj / rhoj * O.ux[j] * twij * neighbor;
                tuy += mj / rhoj * O.uy[j] * twij * neighbor;
                tuz += mj / rhoj * O.uz[j] * twij * neighbor;
                tflt += mj / rhoj * twij * neighbor;
                gpx += mj / rhoj * (presj - pres_g) * tdwx * neighbor;
                gpy += mj / rhoj * (presj - pres_g) * tdwy * neighbor;
                gpz += mj / rhoj * (presj - pres_g) * tdwz * neighbor;
            });
            if (tflt < 1e-6) {
                A.pres[i] = 0.0;
            } else {
                A.pres[i] = tpres / tflt;
                if (O.p_type[i] == -1) { A.ux[i] = tux / tflt; A.uy[i] = tuy / tflt; A.uz[i] = tuz / tflt; }
                if (mirror) A.pres[i] = pres_g + (xi - xg) * gpx + (yi - yg) * gpy + (zi - zg) * gpz;
            }
        }
    }

    // KERNEL_advection_force3D, functions_PPE.cuh:191-480, with the
    // conduction / Eulerian temperature term (con_solve), concentration
    // advection-diffusion (concn_solve) and Boussinesq buoyancy; the literal
    // types of the reference's expressions are kept (double constants promote
    // a float expression to double before it is stored).
    void advection(State<Real> &A) {
        const P Q = q();
        const bool con = Q.con_solve() != 0, cnc = Q.concn_solve() != 0, bsq = Q.boussinesq() != 0;
        for (int i = 0; i < n(); ++i) {
            if (A.i_type[i] > 2 || A.p_type[i] == 1000 || A.p_type[i] <= 0) continue;
            int ptypei = A.p_type[i];
            Real xi = A.x[i], yi = A.y[i], zi = A.z[i], uxi = A.ux[i], uyi = A.uy[i], uzi = A.uz[i];
            Real hi = A.h[i], mi = A.m[i], rhoi = A.rho[i], tempi = A.temp[i];
            Real tmp_A = calc_tmpA(Q, hi);
            Real kci = 0, cpi = 0, concni = 0, diffi = 0;
            if (con) {
                kci = SOLID_K * (ptypei == 0 || ptypei == 1000) + AIR_K * (ptypei == 1 || ptypei == -1);
                cpi = SOLID_CP * (ptypei == 0 || ptypei == 1000) + AIR_CP * (ptypei == 1 || ptypei == -1);
            }
            if (cnc) { concni = A.concn[i]; diffi = 2.0; }
            Real visi = viscosity2<Real>(prm, ptypei) + A.vis_t[i] * rhoi;
            Real betai = 1.0 / prm.t_ini;    // thermal_expansion, functions_PROP.cuh:203-212
            Real tx = 0, ty = 0, tz = 0, ex = 0, ey = 0, ez = 0;
            Real eulert = 0, tmp_Rc = 0, tmp_Rd = 0, tmp_temp = 0, tmp_flt = 0;
            const Real Alpha = (float)prm.av_alpha, Beta = (float)prm.av_beta, c0 = (float)prm.av_c0;
            for (int64_t e = nb_off[i]; e < nb_off[i + 1]; ++e) {
                int j = nb[e];
                if (A.p_type[j] >= 1000) continue;
                Real xj = A.x[j], yj = A.y[j], zj = A.z[j], hj = A.h[j];
                Real tdist = std::sqrt((xi - xj) * (xi - xj) + (yi - yj) * (yi - yj) + (zi - zj) * (zi - zj)) + 1e-20;
                Real twij = calc_wij(Q, tmp_A, hi, tdist);
                Real tdwij = calc_dwij(Q, tmp_A, hi, tdist);
                Real tdwx = tdwij * (xi - xj) / tdist, tdwy = tdwij * (yi - yj) / tdist, tdwz = tdwij * (zi - zj) / tdist;
                if (Q.kgc_solve() == 1) { tdwx = 0; tdwy = 0; tdwz = 0; }
                int ptypej = A.p_type[j];
                Real uxj = A.ux[j], uyj = A.uy[j], uzj = A.uz[j], mj = A.m[j], rhoj = A.rho[j], tempj = A.temp[j];
                if (Q.fv_solve() == 1) {
                    Real visj = viscosity2<Real>(prm, ptypej) + A.vis_t[j] * rhoj;
                    Real C_v = (xi - xj) * tdwx + (yi - yj) * tdwy + (zi - zj) * tdwz;
                    C_v *= (visi * visj) / (visi + visj);
                    C_v *= 4 * (mj / (rhoi * rhoj));
                    C_v /= tdist;
                    C_v /= tdist;
                    tx += C_v * (uxi - uxj); ty += C_v * (uyi - uyj); tz += C_v * (uzi - uzj);
                } else if (Q.fv_solve() == 2) {
                    Real uij_xij = (uxi - uxj) * (xi - xj) + (uyi - uyj) * (yi - yj) + (uzi - uzj) * (zi - zj);
                    Real visj = viscosity2<Real>(prm, ptypej) + A.vis_t[j] * rhoj;
                    Real phi_ij = uij_xij;
                    phi_ij /= (tdist * tdist + 0.01 * hi * hi);
                    Real P_ij = -2.0 * (3 + 2.0) * phi_ij * mj / rhoj;
                    Real C_v = 2.0 * (visi * visj) / (visi + visj - 1e-20);
                    Real nui = C_v / rhoi;
                    P_ij *= nui;
                    if (ptypei <= 0 || ptypei >= 1000) P_ij = 0.0;
                    if (ptypej <= 0 || ptypei >= 1000) P_ij = 0.0;
                    tx += -(P_ij)*tdwx; ty += -(P_ij)*tdwy; tz += -(P_ij)*tdwz;
                }
                if (A.eli[i] < 1.0) {
                    ex += (uxi * (uxj - uxi) * tdwx + uyi * (uxj - uxi) * tdwy + uzi * (uxj - uxi) * tdwz) * mj / rhoj * (1 - A.eli[i]);
                    ey += (uxi * (uyj - uyi) * tdwx + uyi * (uyj - uyi) * tdwy + uzi * (uyj - uyi) * tdwz) * mj / rhoj * (1 - A.eli[i]);
                    ez += (uxi * (uzj - uzi) * tdwx + uyi * (uzj - uzi) * tdwy + uzi * (uzj - uzi) * tdwz) * mj / rhoj * (1 - A.eli[i]);
                    if (con)
                        eulert -= 2.0 * mj / (rhoi + rhoj) * (tempj - tempi) *
                                  ((uxi - uxj) * tdwx + (uyi - uyj) * tdwy + (uzi - uzj) * tdwz) * (1 - A.eli[i]);
                    if (cnc) {
                        Real concnj = A.concn[j];
                        tmp_Rd -= (uxi * (concnj - concni) * tdwx + uyi * (concnj - concni) * tdwy +
                                   uzi * (concnj - concni) * tdwz) * mj / rhoj * (1 - A.eli[i]);
                    }
                }
                if (con) {   // conduction with the uncorrected dW/dr
                    Real kcj = SOLID_K * (ptypej == 0 || ptypej == 1000) + AIR_K * (ptypej == 1 || ptypej == -1);
                    Real rhoj_temp = (ptypej == 1 || ptypej == -1) ? rhoj : (Real)SOLID_RHO;
                    Real mj_temp = mj * rhoj_temp / rhoj;
                    Real sum_con_H = 4.0 * mj_temp * kcj * kci * (tempi - tempj) * tdwij;
                    sum_con_H /= (tdist + 1e-10) * rhoi * rhoj_temp * (kci + kcj);
                    tmp_Rc += sum_con_H;
                }
                if (cnc) {
                    Real concnj = A.concn[j];
                    Real diffj = 2.0;
                    Real tmprd = mi * (diffi * rhoi + diffj * rhoj);
                    tmprd *= ((xi - xj) * tdwx + (yi - yj) * tdwy + (zi - zj) * tdwz);
                    tmprd /= (rhoi * rhoj * (tdist * tdist + 0.01 * hi * hi));
                    Real tmprd1 = tmprd * (concni - concnj) * (ptypei == ptypej);
                    tmp_Rd += tmprd1;
                }
                if (bsq) {
                    tmp_temp += (mj / rhoj) * tempj * twij;
                    tmp_flt += (mj / rhoj) * twij;
                }
                Real uij_xij = (uxi - uxj) * (xi - xj) + (uyi - uyj) * (yi - yj) + (uzi - uzj) * (zi - zj);
                if (uij_xij < 0) {
                    Real h_ij = (hi + hj) * 0.5;
                    Real phi_ij = h_ij * uij_xij;
                    phi_ij /= (tdist * tdist + 0.01 * h_ij * h_ij);
                    Real P_ij = mi * phi_ij * (-Alpha * c0 + Beta * phi_ij);
                    P_ij /= (rhoi + rhoj);
                    P_ij *= 0.5;
                    tx += -(P_ij)*tdwx; ty += -(P_ij)*tdwy; tz += -(P_ij)*tdwz;
                }
            }
            if (Q.fg_solve()) tz += -GRAV;
            if (bsq && ptypei > 0 && ptypei < 1000) tz = betai * GRAV * (tmp_temp / tmp_flt - TEMPB);
            S3.ftx[i] = tx - ex; S3.fty[i] = ty - ey; S3.ftz[i] = tz - ez;
            S3.ft[i] = std::sqrt(tx * tx + ty * ty + tz * tz);
            if (con) {   // functions_PPE.cuh:460-468
                if (Q.enthalpy_eqn()) S3.denthalpy[i] = tmp_Rc * (ptypei != -1);
                else S3.dtemp[i] += tmp_Rc / cpi - eulert;
            }
            if (cnc) S3.dconcn[i] = tmp_Rd;
        }
    }

    // KERNEL_clc_projection, functions_TIME_ISPH.cuh:2-112
    void projection(State<Real> &A, Real tdt, float ttime) {
        for (int i = 0; i < n(); ++i) {
            if (A.i_type[i] >= 3 || A.p_type[i] >= 1000) continue;
            int bt = A.buffer_type[i], mo = A.most[i], pt = A.p_type[i];
            if (pt == 9) {
                S2.x0[i] = A.x[i]; S2.y0[i] = A.y[i]; S2.z0[i] = A.z[i];
                A.ux[i] = (float)prm.boundary_velocity; A.uy[i] = 0; A.uz[i] = 0;
                S2.ux0[i] = (float)prm.boundary_velocity; S2.uy0[i] = 0; S2.uz0[i] = 0;
            } else {
                Real tux0 = A.ux[i], tuy0 = A.uy[i], tuz0 = A.uz[i], tuxp, tuyp, tuzp;
                if (pt > 0) {
                    Real ax = S3.ftx[i] * (bt == 0 || mo == 1) + A.fmx[i];
                    Real ay = S3.fty[i] * (bt == 0 || mo == 1) + A.fmy[i];
                    Real az = S3.ftz[i] * (bt == 0 || mo == 1);
                    tuxp = tux0 + ax * (tdt); tuyp = tuy0 + ay * (tdt); tuzp = tuz0 + az * (tdt);
                } else {
                    tuxp = A.ux[i]; tuyp = A.uy[i]; tuzp = A.uz[i];
                }
                A.ux[i] = tuxp; A.uy[i] = tuyp; A.uz[i] = tuzp;
                S2.x0[i] = A.x[i]; S2.y0[i] = A.y[i]; S2.z0[i] = A.z[i];
                S2.ux0[i] = tux0; S2.uy0[i] = tuy0; S2.uz0[i] = tuz0;
            }
            if (ttime == 0) S2.rho_ref[i] = A.rho[i];
            if (q().con_solve() == 1) {   // functions_TIME_ISPH.cuh:89-101
                if (q().enthalpy_eqn()) {
                    const Real th = A.enthalpy[i];
                    S2.enthalpy0[i] = th;
                    A.temp[i] = htoT<Real>(th, A.p_type[i], q().prop_table() == 1, tab, A.temp[i]);
                } else {
                    S2.temp0[i] = A.temp[i];
                }
            }
            if (q().concn_solve() == 1) {
                Real tconcn = A.concn[i];
                S2.concn0[i] = tconcn;
                A.concn[i] = tconcn + S3.dconcn[i] * (tdt);
            }
        }
    }

    // KERNEL_periodic_boundary3D, functions_BC.cuh:1015-1154
    void periodic(State<Real> &A) {
        State<Real> O = A;
        for (int i = 0; i < n(); ++i) {
            int bt = O.buffer_type[i];
            if (bt == 0 || O.p_type[i] >= 1000) continue;
            if (bt != 3 && bt != 4) continue;
            Real xi = O.x[i], yi = O.y[i], zi = O.z[i];
            Real xg = xi, zg = zi;
            Real yg = (bt == 3) ? (Real)(yi + prm.l_right - prm.l_left) : (Real)(yi - prm.l_right + prm.l_left);
            float ygf = (bt == 3) ? (float)(yf[i] + prm.l_right - prm.l_left) : (float)(yf[i] - prm.l_right + prm.l_left);
            int ic, jc, kc;
            search_cell(xf[i], ygf, zf[i], ic, jc, kc);
            const P Q = q();
            int nc = O.ncell[i];
            Real tux = 0, tuy = 0, tuz = 0, tp = 0, tt = 0;
            bool flag = false;
            for (int z = -nc; z <= nc; z++)
                for (int y = -nc; y <= nc; y++)
                    for (int x = -nc; x <= nc; x++) {
                        if (flag) continue;
                        int k = (ic + x) + Q.NI() * (jc + y) + Q.NI() * Q.NJ() * (kc + z);
                        if (ic + x < 0 || ic + x > Q.NI() - 1 || jc + y < 0 || jc + y > Q.NJ() - 1 || kc + z < 0 || kc + z > Q.NK() - 1) continue;
                        if (g_str[k] == -1) continue;
                        for (int j = g_str[k]; j < g_end[k]; j++) {
                            Real tdist = std::sqrt((xg - O.x[j]) * (xg - O.x[j]) + (yg - O.y[j]) * (yg - O.y[j]) + (zg - O.z[j]) * (zg - O.z[j])) - 1e-20;
                            if (tdist < prm.partner_tol) {
                                tux = O.ux[j]; tuy = O.uy[j]; tuz = O.uz[j]; tp = O.pres[j]; tt = O.temp[j];
                                flag = true;
                            }
                        }
                    }
            A.ux[i] = tux; A.uy[i] = tuy; A.uz[i] = tuz; A.pres[i] = tp; A.temp[i] = tt;
        }
        // ghosts of the periodic box (new work, no reference counterpart):
        // u, p and T of the record at the wrapped position, after the y copy
        const State<Real> O2 = A;
        for (int i = 0; i < n(); ++i) {
            if (O2.buffer_type[i] != SPH_BUFFER_PERIODIC_GHOST) continue;
            const int j = ghost_partner(O2, i);
            A.ux[i] = j >= 0 ? O2.ux[j] : 0; A.uy[i] = j >= 0 ? O2.uy[j] : 0; A.uz[i] = j >= 0 ? O2.uz[j] : 0;
            A.pres[i] = j >= 0 ? O2.pres[j] : 0; A.temp[i] = j >= 0 ? O2.temp[j] : 0;
        }
    }

    // partner of a periodic-box ghost: the record (not a ghost) within
    // partner_tol of the ghost's position wrapped into the box, x - L
    // floor((x - x0) / L) per axis with x1 > x0, in double; the last match
    // in cell order
    int ghost_partner(const State<Real> &A, int i) const {
        const float v[3] = {xf[i], yf[i], zf[i]};
        double w[3];
        for (int a = 0; a < 3; ++a) {
            const double lo = prm.periodic_box[2 * a], len = prm.periodic_box[2 * a + 1] - lo;
            w[a] = (len > 0) ? (double)v[a] - len * std::floor(((double)v[a] - lo) / len) : (double)v[a];
        }
        int ic, jc, kc, found = -1;
        search_cell((float)w[0], (float)w[1], (float)w[2], ic, jc, kc);
        cell_loop(ic, jc, kc, 1, [&](int j) {
            if (A.buffer_type[j] == SPH_BUFFER_PERIODIC_GHOST) return;
            const double dx = w[0] - (double)xf[j], dy = w[1] - (double)yf[j], dz = w[2] - (double)zf[j];
            if (std::sqrt(dx * dx + dy * dy + dz * dz) < prm.partner_tol) found = j;
        });
        return found;
    }

    // KERNEL_freeslip_boundary3D, functions_BC.cuh:1156-1271
    void freeslip(State<Real> &A) {
        const P Q = q();
        State<Real> O = A;
        for (int i = 0; i < n(); ++i) {
            if (O.p_type[i] != -1) continue;
            if (O.i_type[i] >= 3) continue;
            Real hi = O.h[i];
            Real tmp_A = calc_tmpA(Q, hi);
            Real xi = O.x[i], yi = O.y[i], zi = O.z[i];
            Real tux = 0, tuy = 0, tuz = 0, tp = 0, tt = 0, tf = 0;
            for (int64_t e = nb_off[i]; e < nb_off[i + 1]; ++e) {
                int j = nb[e];
                float tdf = std::sqrt(d2f(xf[i], yf[i], zf[i], xf[j], yf[j], zf[j]));
                if (!(tdf < Q.skappa() * hf[i])) continue;
                Real xj = O.x[j], yj = O.y[j], zj = O.z[j];
                Real tdist = std::sqrt((xi - xj) * (xi - xj) + (yi - yj) * (yi - yj) + (zi - zj) * (zi - zj)) - 1e-20;
                Real neighbor = (O.p_type[j] == 1);
                Real twij = calc_wij(Q, tmp_A, hi, tdist);
                Real mj = O.m[j], rhoj = O.rho[j];
                tux += O.ux[j] * (mj / rhoj) * twij * neighbor;
                tuy += O.uy[j] * (mj / rhoj) * twij * neighbor;
                tuz += O.uz[j] * (mj / rhoj) * twij * neighbor;
                tp += O.pres[j] * (mj / rhoj) * twij * neighbor;
                tt += O.temp[j] * (mj / rhoj) * twij * neighbor;
                tf += (mj / rhoj) * twij * neighbor;
            }
            if (tf > 1e-5) {
                A.ux[i] = tux / tf; A.uy[i] = tuy / tf; A.uz[i] = tuz / tf; A.pres[i] = tp / tf; A.temp[i] = tt / tf;
            }
        }
    }

    // KERNEL_donothing_buffer3D, functions_BC.cuh:673-761
    void donothing(State<Real> &A) {
        State<Real> O = A;
        for (int i = 0; i < n(); ++i) {
            if (O.buffer_type[i] != 2) continue;
            Real yi = O.y[i], zi = O.z[i];
            int ic, jc, kc;
            search_cell(xf[i], yf[i], zf[i], ic, jc, kc);
            Real tux = 0, tuy = 0, tuz = 0, tp = 0, tt = 0;
            Real xg = (Real)(prm.l3 - prm.outlet_probe_dx);
            cell_loop(ic, jc, kc, 2 * O.ncell[i], [&](int j) {
                Real tdist = std::sqrt((xg - O.x[j]) * (xg - O.x[j]) + (yi - O.y[j]) * (yi - O.y[j]) + (zi - O.z[j]) * (zi - O.z[j])) - 1e-20;
                if (O.p_type[j] < 1000 && tdist < prm.partner_tol) {
                    tux = O.ux[j]; tuy = O.uy[j]; tuz = O.uz[j]; tp = O.pres[j]; tt = O.temp[j];
                }
            });
            A.pres[i] = tp; A.ux[i] = tux; A.uy[i] = tuy; A.uz[i] = tuz; A.temp[i] = tt;
        }
    }

    // KERNEL_open_boundary_extrapolation_buffer3D, functions_BC.cuh:763-855
    // (dormant in the shipped step; outlet_bc = 1): an outlet record off the
    // MOST layer takes the Shepard average of the fluid around its mirror
    // node across L3 and zero pressure, when that average has weight.  Every
    // record reads the pre-pass state.
    void extrapolation(State<Real> &A) {
        const P Q = q();
        State<Real> O = A;
        for (int i = 0; i < n(); ++i) {
            if (O.buffer_type[i] != 2 || O.most[i] == 1) continue;
            Real hi = O.h[i];
            Real tmp_A = calc_tmpA(Q, hi);
            Real search_range = Q.skappa() * hi;
            Real xg = 2 * prm.l3 - O.x[i], yg = O.y[i], zg = O.z[i];
            const float xgf = (float)(2 * prm.l3 - (double)xf[i]);
            int ic = bin_axis(xgf, Q.xmin(), Q.xmax(), Q.NI());
            int jc = bin_axis(yf[i], Q.ymin(), Q.ymax(), Q.NJ());
            int kc = bin_axis(zf[i], Q.zmin(), Q.zmax(), Q.NK());
            Real tpres = 0, tux = 0, tuy = 0, tuz = 0, tflt = 0;
            cell_loop(ic, jc, kc, O.ncell[i], [&](int j) {
                Real tdist = std::sqrt((xg - O.x[j]) * (xg - O.x[j]) + (yg - O.y[j]) * (yg - O.y[j]) + (zg - O.z[j]) * (zg - O.z[j])) - 1e-20;
                if (O.p_type[j] < 1000 && tdist < search_range) {
                    Real twij = calc_wij(Q, tmp_A, hi, tdist);
                    int on = (O.p_type[j] == 1) * (O.most[j] != 1);
                    Real mj = O.m[j], rhoj = O.rho[j];
                    tpres += mj / rhoj * O.pres[j] * twij * on;
                    tux += mj / rhoj * O.ux[j] * twij * on;
                    tuy += mj / rhoj * O.uy[j] * twij * on;
                    tuz += mj / rhoj * O.uz[j] * twij * on;
                    tflt += mj / rhoj * twij * on;
                }
            });
            if (tflt < 1e-6) continue;
            A.pres[i] = 0.0;
            A.ux[i] = tux / tflt; A.uy[i] = tuy / tflt; A.uz[i] = tuz / tflt;
        }
    }

    // KERNEL_inout_boundary3D, functions_BC.cuh:1274-1433 (dormant;
    // outlet_bc = 2): side buffers (3, 4) copy u, p and T of the record at
    // their periodic image (zero when there is none); outlet records are set
    // so that the interface value at x = L3, a Shepard average of interior
    // fluid with the pair-averaged h, is the mean of the record and its
    // mirror: u = 2 u_if - u.  Inlet records are left as they are.  Every
    // record reads the pre-pass state.
    void inout(State<Real> &A) {
        const P Q = q();
        State<Real> O = A;
        for (int i = 0; i < n(); ++i) {
            const int bt = O.buffer_type[i];
            if (bt == 0 || O.p_type[i] >= 1000) continue;
            if (bt != 2 && bt != 3 && bt != 4) continue;
            Real hi = O.h[i];
            Real search_range = Q.skappa() * hi;
            const int nc = O.ncell[i];
            if (bt == 3 || bt == 4) {
                Real xg = O.x[i], zg = O.z[i];
                Real yg = (bt == 3) ? (Real)(O.y[i] + prm.l_right - prm.l_left) : (Real)(O.y[i] - prm.l_right + prm.l_left);
                float ygf = (bt == 3) ? (float)(yf[i] + prm.l_right - prm.l_left) : (float)(yf[i] - prm.l_right + prm.l_left);
                int ic, jc, kc;
                search_cell(xf[i], ygf, zf[i], ic, jc, kc);
                Real tux = 0, tuy = 0, tuz = 0, tp = 0, tt = 0;
                bool flag = false;
                for (int z = -nc; z <= nc; z++)
                    for (int y = -nc; y <= nc; y++)
                        for (int x = -nc; x <= nc; x++) {
                            if (flag) continue;
                            if (ic + x < 0 || ic + x > Q.NI() - 1 || jc + y < 0 || jc + y > Q.NJ() - 1 || kc + z < 0 || kc + z > Q.NK() - 1) continue;
                            int k = (ic + x) + Q.NI() * (jc + y) + Q.NI() * Q.NJ() * (kc + z);
                            if (g_str[k] == -1) continue;
                            for (int j = g_str[k]; j < g_end[k]; j++) {
                                Real tdist = std::sqrt((xg - O.x[j]) * (xg - O.x[j]) + (yg - O.y[j]) * (yg - O.y[j]) + (zg - O.z[j]) * (zg - O.z[j])) - 1e-20;
                                if (tdist < 0.001) {
                                    tux = O.ux[j]; tuy = O.uy[j]; tuz = O.uz[j]; tp = O.pres[j]; tt = O.temp[j];
                                    flag = true;
                                }
                            }
                        }
                A.ux[i] = tux; A.uy[i] = tuy; A.uz[i] = tuz; A.pres[i] = tp; A.temp[i] = tt;
            } else {
                Real yg = O.y[i], zg = O.z[i];
                int ic = (int)std::min(std::floor((prm.l3 - (double)Q.xmin()) / (double)Q.dcell()), (double)(Q.NI() - 1));
                int jc = search_axis(yf[i], Q.ymin(), Q.ymax(), Q.dcell(), Q.NJ());
                int kc = search_axis(zf[i], Q.zmin(), Q.zmax(), Q.dcell(), Q.NK());
                if (ic < 0) ic = 0;
                Real ux_if = 0, uy_if = 0, uz_if = 0, p_if = 0, tflt = 0;
                cell_loop(ic, jc, kc, nc, [&](int j) {
                    Real tdist = std::sqrt((prm.l3 - O.x[j]) * (prm.l3 - O.x[j]) + (yg - O.y[j]) * (yg - O.y[j]) + (zg - O.z[j]) * (zg - O.z[j])) - 1e-20;
                    if (tdist < search_range) {
                        Real hij = 0.5 * (hi + O.h[j]);
                        Real tmp_Aij = calc_tmpA(Q, hij);
                        Real twij = calc_wij(Q, tmp_Aij, hij, tdist);
                        int on = (O.buffer_type[j] == 0) * (O.p_type[j] == 1);
                        Real vj = O.m[j] / O.rho[j];
                        ux_if += O.ux[j] * vj * twij * on;
                        uy_if += O.uy[j] * vj * twij * on;
                        uz_if += O.uz[j] * vj * twij * on;
                        p_if += O.pres[j] * vj * twij * on;
                        tflt += vj * twij * on;
                    }
                });
                A.ux[i] = -O.ux[i] + 2.0 * ux_if / tflt;
                A.uy[i] = -O.uy[i] + 2.0 * uy_if / tflt;
                A.uz[i] = -O.uz[i] + 2.0 * uz_if / tflt;
                A.pres[i] = -O.pres[i] + 2.0 * p_if / tflt;
            }
        }
    }

    // the pass at the outlet-buffer call sites (ISPH_Calc.cuh:151, 208)
    void outlet_bc(State<Real> &A) {
        if (prm.outlet_bc == 1) extrapolation(A);
        else if (prm.outlet_bc == 2) inout(A);
        else donothing(A);
    }

    // KERNEL_Recycling3D, functions_BC.cuh:1857-1941 (dormant; inlet_recycling
    // = 1, after the last boundary pass, ISPH_Calc.cuh:215).  Its neighbour
    // search there finds a record whose velocity is then not used; the inlet
    // takes the log law of the probe's friction velocity.
    void recycling(State<Real> &A) {
        for (int i = 0; i < n(); ++i) {
            if (A.buffer_type[i] != 1 && A.buffer_type[i] != -1) continue;
            A.ux[i] = (us_update / 0.4) * std::log(A.z[i] / prm.most_z0);
        }
    }

    // ---- PPE ----------------------------------------------------------------
    // row of KERNEL_PPE3D, functions_PPE.cuh:2-175: returns b_i, A_i and the
    // off-diagonal coefficients c_ij (p_i = (b_i + sum c_ij p_j) / A_i)
    void ppe_row(const State<Real> &A, int i, Real tdt, Real &bi, Real &Aij,
                 std::vector<std::pair<int, Real>> &cs) const {
        const P Q = q();
        cs.clear();
        Real hi = prm.pressure_length * A.h[i];
        Real tmp_A = calc_tmpA(Q, hi);
        Real xi = A.x[i], yi = A.y[i], zi = A.z[i], uxi = A.ux[i], uyi = A.uy[i], uzi = A.uz[i], rhoi = A.rho[i];
        Real gc11 = S3.gxx[i], gc12 = S3.gxy[i], gc22 = S3.gyy[i], gc23 = S3.gyz[i], gc31 = S3.gzx[i], gc33 = S3.gzz[i];
        Real bix = 0, biy = 0, biz = 0, divFb = 0.0;
        Aij = 0;
        for (int64_t e = nb_off[i]; e < nb_off[i + 1]; ++e) {
            int j = nb[e];
            if (A.p_type[j] >= 1000 || A.i_type[j] == 4) continue;
            Real xj = A.x[j], yj = A.y[j], zj = A.z[j], uxj = A.ux[j], uyj = A.uy[j], uzj = A.uz[j];
            Real rhoj = A.rho[j], mj = A.m[j];
            Real tdist = std::sqrt((xi - xj) * (xi - xj) + (yi - yj) * (yi - yj) + (zi - zj) * (zi - zj)) + 1e-20;
            Real tdwij;
            if (prm.ppe_pair_h == 1) {   // functions_PPE.cuh:113-116 (commented out there)
                Real hij = 0.5 * (hi + prm.pressure_length * A.h[j]);
                tdwij = calc_dwij_pressure(Q, calc_tmpA(Q, hij), hij, tdist);
            } else {
                tdwij = calc_dwij_pressure(Q, tmp_A, hi, tdist);
            }
            Real tdwx = tdwij * (xi - xj) / tdist, tdwy = tdwij * (yi - yj) / tdist, tdwz = tdwij * (zi - zj) / tdist;
            Real tdwxc = gc11 * tdwx + gc12 * tdwy + gc31 * tdwz;
            Real tdwyc = gc12 * tdwx + gc22 * tdwy + gc23 * tdwz;
            Real tdwzc = gc31 * tdwx + gc23 * tdwy + gc33 * tdwz;
            bix += mj / rhoj * (uxj - uxi) * tdwxc * (2.0 * rhoi * rhoj / (rhoi + rhoj));
            biy += mj / rhoj * (uyj - uyi) * tdwyc * (2.0 * rhoi * rhoj / (rhoi + rhoj));
            biz += mj / rhoj * (uzj - uzi) * tdwzc * (2.0 * rhoi * rhoj / (rhoi + rhoj));
            Real c = 2.0 * mj / rhoj * ((xi - xj) * tdwxc + (yi - yj) * tdwyc + (zi - zj) * tdwzc) / tdist / tdist;
            Aij += c;
            cs.push_back({j, c});
        }
        Real weight = 1.0;
        bi = weight * (bix + biy + biz + divFb) / tdt;
    }

    static bool is_fluid_row(const State<Real> &A, int i) {
        return !(A.i_type[i] > 2 || A.p_type[i] >= 1000 || A.p_type[i] <= 0);
    }

    // one snapshot sweep: p_i = p0_i + (b_i + sum c_ij (p_j - p0_j)) / A_i
    void ppe_sweep(State<Real> &A, Real tdt) {
        std::vector<Real> pnew = A.pres;
        std::vector<std::pair<int, Real>> cs;
        for (int i = 0; i < n(); ++i) {
            if (!is_fluid_row(A, i)) continue;
            Real bi, Aij;
            ppe_row(A, i, tdt, bi, Aij, cs);
            Real AijPij = 0;
            for (auto &c : cs) AijPij += c.second * (A.pres[c.first] - A.pres0[c.first]);
            pnew[i] = A.pres0[i] + (bi + AijPij) / Aij;
        }
        A.pres = pnew;
    }

    // Row classes of the converged system (see DESIGN: precedence of the
    // reference's overwrites): 0 identity, 1 fluid, 2 Neumann, 3 outlet copy.
    int row_class(const State<Real> &A, int i) const {
        if (A.i_type[i] >= 3) return 0;
        if (A.buffer_type[i] == 2 || A.buffer_type[i] == SPH_BUFFER_PERIODIC_GHOST) return 3;
        if (A.p_type[i] != 1) return 2;
        return 1;
    }

    // Assembles the converged PPE system M p = rhs in double.  Fluid rows:
    // A_i p_i - sum c_ij p_j = b_i; Neumann rows: p_w - (Shepard / mirror
    // weights) p = 0; outlet rows: p_o - p_partner = 0; identity rows: p = p_old.
    void assemble(const State<Real> &A, Real tdt, std::vector<int64_t> &ro, std::vector<int> &ci,
                  std::vector<double> &va, std::vector<double> &rhs) {
        const int N = n();
        ro.assign(N + 1, 0); ci.clear(); va.clear(); rhs.assign(N, 0.0);
        std::vector<std::pair<int, Real>> cs;
        std::vector<int> kind(N);
        for (int i = 0; i < N; ++i) {
            ro[i] = (int64_t)ci.size();
            const int rc = row_class(A, i);
            kind[i] = rc;
            if (rc == 0) { ci.push_back(i); va.push_back(1.0); rhs[i] = A.pres[i]; continue; }
            if (rc == 1) {
                Real bi, Aij;
                ppe_row(A, i, tdt, bi, Aij, cs);
                ci.push_back(i); va.push_back((double)Aij);
                for (auto &c : cs) if (c.first != i) { ci.push_back(c.first); va.push_back(-(double)c.second); }
                rhs[i] = (double)bi;
                continue;
            }
            if (rc == 3) {
                int partner = A.buffer_type[i] == SPH_BUFFER_PERIODIC_GHOST ? ghost_partner(A, i) : outlet_partner(A, i);
                ci.push_back(i); va.push_back(1.0);
                if (partner >= 0) { ci.push_back(partner); va.push_back(-1.0); }
                continue;
            }
            // Neumann row with its Shepard weights; the inlet mirror
            // extrapolation is applied after the solve by the Neumann pass
            std::vector<std::pair<int, double>> w;
            neumann_weights(A, i, w, /*operator_row=*/true);
            ci.push_back(i); va.push_back(1.0);
            for (auto &c : w) { ci.push_back(c.first); va.push_back(-c.second); }
        }
        ro[N] = (int64_t)ci.size();
        pins.clear();
        comp_of.assign(N, -1);
        comp_size.clear();
        if (prm.ppe_pin) {
            // Connected components of the operator's graph; a component with no
            // anchor row (a row that is only its diagonal: identity rows,
            // Neumann rows without fluid in range, outlet rows without
            // partner) is singular (its rows sum to zero, M 1 = 0).
            //  ppe_pin == 1: rank-one regularisation M' = M + D u w^T per such
            //    component, u = its fluid rows, w = u/|u|, D = the rows'
            //    diagonals (A_i < 0): the constant mode gets the eigenvalue 1
            //    of the Jacobi-scaled operator, beside the rest of its
            //    spectrum, and the compatibility defect of b becomes the
            //    source A_i lambda with lambda = w^T p;
            //  ppe_pin == 2: one row pinned to p = 0, the highest-index fluid
            //    row with buffer_type 0 (else the highest-index fluid row).
            std::vector<int> par(N);
            std::iota(par.begin(), par.end(), 0);
            std::function<int(int)> find = [&](int x) { while (par[x] != x) { par[x] = par[par[x]]; x = par[x]; } return x; };
            for (int i = 0; i < N; ++i)
                for (int64_t e = ro[i]; e < ro[i + 1]; ++e) {
                    int a = find(i), b = find(ci[e]);
                    if (a != b) par[std::max(a, b)] = std::min(a, b);
                }
            std::vector<char> anchored(N, 0);
            std::vector<int> cand(N, -1), cand_any(N, -1), cid(N, -1);
            for (int i = 0; i < N; ++i) {
                const int r = find(i);
                if (ro[i + 1] - ro[i] == 1 && kind[i] != 1) anchored[r] = 1;
                if (kind[i] == 1) {
                    cand_any[r] = std::max(cand_any[r], i);
                    if (A.buffer_type[i] == 0) cand[r] = std::max(cand[r], i);
                }
            }
            for (int r = 0; r < N; ++r) {
                if (find(r) != r || anchored[r] || cand_any[r] < 0) continue;
                if (prm.ppe_pin == 2 || (int)comp_size.size() >= 8) {
                    pins.push_back(cand[r] >= 0 ? cand[r] : cand_any[r]);
                } else {
                    cid[r] = (int)comp_size.size();
                    comp_size.push_back(0);
                }
            }
            for (int i = 0; i < N; ++i)
                if (kind[i] == 1 && cid[find(i)] >= 0) { comp_of[i] = cid[find(i)]; comp_size[comp_of[i]]++; }
            std::sort(pins.begin(), pins.end());
            if (!pins.empty()) {
                // rebuild with the pinned rows replaced by p = 0
                std::vector<int64_t> r2(N + 1, 0); std::vector<int> c2; std::vector<double> v2;
                size_t q = 0;
                for (int i = 0; i < N; ++i) {
                    r2[i] = (int64_t)c2.size();
                    if (q < pins.size() && pins[q] == i) { c2.push_back(i); v2.push_back(1.0); rhs[i] = 0.0; ++q; continue; }
                    for (int64_t e = ro[i]; e < ro[i + 1]; ++e) { c2.push_back(ci[e]); v2.push_back(va[e]); }
                }
                r2[N] = (int64_t)c2.size();
                ro.swap(r2); ci.swap(c2); va.swap(v2);
            }
        }
        pin_row = pins.empty() ? -1 : pins.back();
    }

    int outlet_partner(const State<Real> &A, int i) const {
        int ic, jc, kc, found = -1;
        search_cell(xf[i], yf[i], zf[i], ic, jc, kc);
        Real xg = (Real)(prm.l3 - prm.outlet_probe_dx), yi = A.y[i], zi = A.z[i];
        cell_loop(ic, jc, kc, 2 * A.ncell[i], [&](int j) {
            Real tdist = std::sqrt((xg - A.x[j]) * (xg - A.x[j]) + (yi - A.y[j]) * (yi - A.y[j]) + (zi - A.z[j]) * (zi - A.z[j])) - 1e-20;
            if (A.p_type[j] < 1000 && tdist < prm.partner_tol) found = j;
        });
        return found;
    }

    // linear weights of a Neumann row: p_w = sum_k w_k p_k
    // linear weights of a Neumann row: p_w = sum_k w_k p_k.  operator_row
    // selects the weights the converged operator uses: the Shepard weights
    // also for inlet mirror rows, and for a row whose Shepard set (fluid with
    // buffer_type 0, functions_BC.cuh:414) is empty -- p = 0 in the reference
    // -- the Shepard average over all fluid in range, buffers included, so
    // that such corner rows do not act as point Dirichlet anchors.
    void neumann_weights(const State<Real> &A, int i, std::vector<std::pair<int, double>> &w,
                         bool operator_row = false) const {
        const P Q = q();
        w.clear();
        float search_coeff = (float)prm.neumann_coeff;
        Real hi = search_coeff * A.h[i];
        Real tmp_A = calc_tmpA(Q, hi);
        float srange = Q.skappa() * (float)(search_coeff * hf[i]);
        Real xi = A.x[i], yi = A.y[i], zi = A.z[i];
        bool mirror = (A.buffer_type[i] == 1 || A.buffer_type[i] == -1);
        Real xg = mirror ? (Real)(2.0 * prm.l2 - xi) : xi, yg = yi, zg = zi;
        float xgf = mirror ? (float)(2.0 * prm.l2 - xf[i]) : xf[i];
        int ic, jc, kc;
        search_cell(xgf, yf[i], zf[i], ic, jc, kc);
        int g = -1;
        cell_loop(ic, jc, kc, 1, [&](int j) {
            Real dist = std::sqrt((xg - A.x[j]) * (xg - A.x[j]) + (yg - A.y[j]) * (yg - A.y[j]) + (zg - A.z[j]) * (zg - A.z[j])) - 1e-20;
            if (dist < prm.ghost_tol) g = j;
        });
        for (int pass = 0; pass < 2; ++pass) {
            // pass 0: the reference's set; pass 1 (operator rows only, when
            // pass 0 is empty): all fluid in range
            const bool all_fluid = pass == 1;
            std::vector<std::pair<int, double>> ws, gs;
            double tflt = 0, gsum = 0;
            cell_loop(ic, jc, kc, A.ncell[i], [&](int j) {
                if (A.p_type[j] >= 1000) return;
                float tdf = std::sqrt(d2f(xgf, yf[i], zf[i], xf[j], yf[j], zf[j]));
                if (!(tdf < srange)) return;
                if (!(A.p_type[j] == 1 && (all_fluid || A.buffer_type[j] == 0))) return;
                Real xj = A.x[j], yj = A.y[j], zj = A.z[j];
                Real tdist = std::sqrt((xg - xj) * (xg - xj) + (yg - yj) * (yg - yj) + (zg - zj) * (zg - zj)) - 1e-20;
                double vw = (double)(A.m[j] / A.rho[j]);
                double twij = calc_wij(Q, tmp_A, hi, tdist);
                double tdwij = calc_dwij(Q, tmp_A, hi, tdist);
                if (Q.kgc_solve() == 1) tdwij = 0;
                double proj = ((xi - xg) * (xg - xj) + (yi - yg) * (yg - yj) + (zi - zg) * (zg - zj)) / (double)tdist * tdwij;
                ws.push_back({j, vw * twij});
                gs.push_back({j, vw * proj});
                tflt += vw * twij;
                gsum += vw * proj;
            });
            if (tflt < 1e-6) {
                if (operator_row && pass == 0) continue;
                return;   // p_w = 0
            }
            if (!mirror || operator_row) {
                for (auto &c : ws) w.push_back({c.first, c.second / tflt});
            } else {
                // p_w = p_g + sum_j g_j (p_j - p_g)
                for (auto &c : gs) w.push_back({c.first, c.second});
                if (g >= 0) w.push_back({g, 1.0 - gsum});
            }
            return;
        }
    }

    // Jacobi-preconditioned BiCGSTAB in double
    int bicgstab(const std::vector<int64_t> &ro, const std::vector<int> &ci, const std::vector<double> &va,
                 const std::vector<double> &b, std::vector<double> &x, double tol, int maxit,
                 double &relres, int &iters) {
        const int N = (int)b.size();
        std::vector<double> dinv(N, 1.0);
        for (int i = 0; i < N; ++i)
            for (int64_t e = ro[i]; e < ro[i + 1]; ++e)
                if (ci[e] == i && va[e] != 0) dinv[i] = 1.0 / va[e];
        const int NC = (int)comp_size.size();
        auto spmv = [&](const std::vector<double> &v, std::vector<double> &y) {
            std::vector<double> mean(NC, 0.0);
            if (NC) {
                for (int i = 0; i < N; ++i) if (comp_of[i] >= 0) mean[comp_of[i]] += v[i];
                for (int k = 0; k < NC; ++k) mean[k] /= comp_size[k];
            }
            for (int i = 0; i < N; ++i) {
                double s = 0, diag_i = 0;
                for (int64_t e = ro[i]; e < ro[i + 1]; ++e) {
                    s += va[e] * v[ci[e]];
                    if (ci[e] == i) diag_i = va[e];
                }
                // rank-one term scaled by the row's own diagonal (A_i < 0), so
                // the constant mode lands beside the rest of the spectrum
                if (NC && comp_of[i] >= 0) s += diag_i * mean[comp_of[i]];
                y[i] = s;
            }
        };
        auto dot = [&](const std::vector<double> &a, const std::vector<double> &c) {
            double s = 0; for (int i = 0; i < N; ++i) s += a[i] * c[i]; return s;
        };
        std::vector<double> r(N), rh(N), pv(N, 0), v(N, 0), s(N), t(N), ph(N), sh(N);
        spmv(x, r);
        for (int i = 0; i < N; ++i) r[i] = b[i] - r[i];
        double bn = std::sqrt(dot(b, b));
        if (bn == 0) bn = 1;
        rh = r;
        double rho = 1, alpha = 1, omega = 1;
        iters = 0;
        relres = std::sqrt(dot(r, r)) / bn;
        while (relres > tol && iters < maxit) {
            double rho1 = dot(rh, r);
            if (rho1 == 0) { rh = r; rho = 1; alpha = 1; omega = 1; std::fill(pv.begin(), pv.end(), 0); std::fill(v.begin(), v.end(), 0); rho1 = dot(rh, r); }
            double beta = (rho1 / rho) * (alpha / omega);
            for (int i = 0; i < N; ++i) pv[i] = r[i] + beta * (pv[i] - omega * v[i]);
            for (int i = 0; i < N; ++i) ph[i] = dinv[i] * pv[i];
            spmv(ph, v);
            alpha = rho1 / dot(rh, v);
            for (int i = 0; i < N; ++i) s[i] = r[i] - alpha * v[i];
            for (int i = 0; i < N; ++i) sh[i] = dinv[i] * s[i];
            spmv(sh, t);
            double tt = dot(t, t);
            omega = tt > 0 ? dot(t, s) / tt : 0;
            for (int i = 0; i < N; ++i) x[i] += alpha * ph[i] + omega * sh[i];
            for (int i = 0; i < N; ++i) r[i] = s[i] - omega * t[i];
            rho = rho1;
            ++iters;
            relres = std::sqrt(dot(r, r)) / bn;
            if (omega == 0) break;
        }
        // true residual
        spmv(x, r);
        for (int i = 0; i < N; ++i) r[i] = b[i] - r[i];
        relres = std::sqrt(dot(r, r)) / bn;
        return relres <= tol ? SPH_OK : SPH_NOT_CONVERGED;
    }

    int ppe_converged(State<Real> &A, Real tdt, double tol, int maxit, double &relres, int &iters) {
        std::vector<int64_t> ro; std::vector<int> ci; std::vector<double> va, rhs;
        assemble(A, tdt, ro, ci, va, rhs);
        std::vector<double> x(n());
        for (int i = 0; i < n(); ++i) x[i] = (double)A.pres[i];
        for (int pr : pins) x[pr] = 0;
        int st = bicgstab(ro, ci, va, rhs, x, tol, maxit, relres, iters);
        for (int i = 0; i < n(); ++i) A.pres[i] = (Real)x[i];
        return st;
    }

    // IBM_force_interpolation3D, functions_IBM.cuh:342-490
    void ibm_force(State<Real> &A, Real t_dt) {
        const P Q = q();
        for (int i = 0; i < n(); ++i) {
            if (A.p_type[i] < 1000) continue;
            Real xi = A.x[i], yi = A.y[i], zi = A.z[i];
            Real tmp_h = prm.ibm_length * A.h[i];
            Real tmp_A = calc_tmpA(Q, tmp_h);
            float sr = Q.skappa() * (float)(prm.ibm_length * hf[i]);
            int ic = bin_axis(xf[i], Q.xmin(), Q.xmax(), Q.NI());
            int jc = bin_axis(yf[i], Q.ymin(), Q.ymax(), Q.NJ());
            int kc = bin_axis(zf[i], Q.zmin(), Q.zmax(), Q.NK());
            Real tux = 0, tuy = 0, tuz = 0, filt = 0;
            cell_loop(ic, jc, kc, A.ncell[i], [&](int j) {
                if (A.i_type[j] == 4 || A.p_type[j] != 1) return;
                float tdf = std::sqrt(d2f(xf[i], yf[i], zf[i], xf[j], yf[j], zf[j]));
                if (!(tdf < sr)) return;
                Real xj = A.x[j], yj = A.y[j], zj = A.z[j];
                Real tdist = std::sqrt((xi - xj) * (xi - xj) + (yi - yj) * (yi - yj) + (zi - zj) * (zi - zj)) + 1e-20;
                Real twij = calc_wij(Q, tmp_A, tmp_h, tdist);
                Real tmprho = A.m[j] / A.rho[j];
                tux += (A.ux[j]) * tmprho * twij; tuy += (A.uy[j]) * tmprho * twij; tuz += (A.uz[j]) * tmprho * twij;
                filt += tmprho * twij;
            });
            A.concentration[i] = filt;
            Real ufx = tux / (filt + 1e-10), ufy = tuy / (filt + 1e-10), ufz = tuz / (filt + 1e-10);
            Real nx = S3.nx[i], ny = S3.ny[i], nz = S3.nz[i];
            Real nmag = std::sqrt(nx * nx + ny * ny + nz * nz) + 1e-20;
            nx = nx / nmag; ny = ny / nmag; nz = nz / nmag;
            Real un = ufx * nx + ufy * ny + ufz * nz;
            Real utx = ufx - un * nx, uty = ufy - un * ny, utz = ufz - un * nz;
            Real Ubtx = prm.ibm_target_coeff * profile((double)A.z[i]);
            Real Ubty = 0.0f, Ubtz = 0.0f;
            Real beta_t = 1.0f;
            Real cx = (-un) * nx + beta_t * (Ubtx - utx);
            Real cy = (-un) * ny + beta_t * (Ubty - uty);
            Real cz = (-un) * nz + beta_t * (Ubtz - utz);
            A.fbx[i] = prm.rho_air * cx / t_dt;
            A.fby[i] = prm.rho_air * cy / t_dt;
            A.fbz[i] = prm.rho_air * cz / t_dt;
        }
    }

    // Device_Interpolate_ux_caseH, functions_IBM.cuh:308-338 (table from params)
    double profile(double z_inp) const {
        const int NP = prm.n_profile;
        const double *Z = prm.profile_z, *U = prm.profile_u;
        const double z = 1.0 * z_inp;
        if (z <= Z[0]) return U[0] + (z - Z[0]) * ((U[1] - U[0]) / ((Z[1] - Z[0]) + 1e-300));
        if (z >= Z[NP - 1]) return U[NP - 2] + (z - Z[NP - 2]) * ((U[NP - 1] - U[NP - 2]) / ((Z[NP - 1] - Z[NP - 2]) + 1e-300));
        int lo = 0, hi = NP - 1;
        while (hi - lo > 1) { int mid = (lo + hi) >> 1; if (z < Z[mid]) hi = mid; else lo = mid; }
        double t = (z - Z[lo]) / (Z[hi] - Z[lo] + 1e-300);
        return U[lo] + t * (U[hi] - U[lo]);
    }

    // IBM_spreading_interpolation3D, functions_IBM.cuh:492-613
    void ibm_spread(State<Real> &A) {
        const P Q = q();
        State<Real> O = A;
        for (int i = 0; i < n(); ++i) {
            if (O.p_type[i] != 1 || O.buffer_type[i] == 2) continue;
            Real xi = O.x[i], yi = O.y[i], zi = O.z[i];
            Real tmp_h = prm.ibm_length * O.h[i];
            Real tmp_A = calc_tmpA(Q, tmp_h);
            float sr = Q.skappa() * (float)(prm.ibm_length * hf[i]);
            int ic = bin_axis(xf[i], Q.xmin(), Q.xmax(), Q.NI());
            int jc = bin_axis(yf[i], Q.ymin(), Q.ymax(), Q.NJ());
            int kc = bin_axis(zf[i], Q.zmin(), Q.zmax(), Q.NK());
            Real fx = 0, fy = 0, fz = 0, filt = 0;
            cell_loop(ic, jc, kc, O.ncell[i], [&](int j) {
                if (O.i_type[j] == 4 || O.p_type[j] != 1000) return;
                float tdf = std::sqrt(d2f(xf[i], yf[i], zf[i], xf[j], yf[j], zf[j]));
                if (!(tdf < sr)) return;
                Real xj = O.x[j], yj = O.y[j], zj = O.z[j];
                Real tdist = std::sqrt((xi - xj) * (xi - xj) + (yi - yj) * (yi - yj) + (zi - zj) * (zi - zj)) + 1e-20;
                Real twij = calc_wij(Q, tmp_A, tmp_h, tdist);
                Real tmprho = O.m[j] / O.rho[j];
                fx += O.fbx[j] * twij * tmprho; fy += O.fby[j] * twij * tmprho; fz += O.fbz[j] * twij * tmprho;
                filt += tmprho * twij;
            });
            if (filt < 1e-12) { A.fbx[i] = 0.0f; A.fby[i] = 0.0f; A.fbz[i] = 0.0f; A.concentration[i] = 0.0f; continue; }
            A.fbx[i] = fx / (filt + 1e-10); A.fby[i] = fy / (filt + 1e-10); A.fbz[i] = fz / (filt + 1e-10);
            A.concentration[i] = filt;
        }
    }

    // KERNEL_pressureforce3D, functions_PPE.cuh:482-647
    void pressure_force(State<Real> &A) {
        const P Q = q();
        for (int i = 0; i < n(); ++i) {
            if (A.i_type[i] > 2 || A.p_type[i] >= 1000 || A.p_type[i] <= 0 || A.buffer_type[i] != 0) continue;
            Real xi = A.x[i], yi = A.y[i], zi = A.z[i], hi = A.h[i], pi = A.pres[i] - A.pres0[i], rhoi = A.rho[i];
            Real tx = 0, ty = 0, tz = 0;
            for (int64_t e = nb_off[i]; e < nb_off[i + 1]; ++e) {
                int j = nb[e];
                if (A.p_type[j] >= 1000) continue;
                Real xj = A.x[j], yj = A.y[j], zj = A.z[j], hj = A.h[j];
                Real tdist = std::sqrt((xi - xj) * (xi - xj) + (yi - yj) * (yi - yj) + (zi - zj) * (zi - zj)) - 1e-20;
                Real hij = 0.5 * (hi + hj);
                Real tmp_Aij = calc_tmpA(Q, hij);
                Real tdwij = calc_dwij(Q, tmp_Aij, hij, tdist);
                Real tdwx = tdwij * (xi - xj) / tdist, tdwy = tdwij * (yi - yj) / tdist, tdwz = tdwij * (zi - zj) / tdist;
                if (Q.kgc_solve() == 1) { tdwx = 0; tdwy = 0; tdwz = 0; }
                Real mj = A.m[j], rhoj = A.rho[j], pj = A.pres[j] - A.pres0[j];
                if (Q.fp_solve()) {
                    // pressure_force_form 1: the commented-out difference form
                    // of functions_PPE.cuh:626 with its stabilisation term zero
                    Real C_p = prm.pressure_force_form == 1
                                   ? -mj * (pj - pi) / (rhoi * rhoj)
                                   : -2.0 * mj / (rhoi * rhoj) * ((pi + 0.0) * rhoj + (pj + 0.0) * rhoi) / (rhoi + rhoj);
                    tx += C_p * tdwx; ty += C_p * tdwy; tz += C_p * tdwz;
                }
            }
            S3.fpx[i] = tx; S3.fpy[i] = ty; S3.fpz[i] = tz;
        }
    }

    // KERNEL_time_update_projection, functions_TIME_ISPH.cuh:115-296: SP1 -> P1
    void time_update(State<Real> &S, State<Real> &T, Real tdt, int tcount) {
        for (int i = 0; i < n(); ++i) {
            if (S.i_type[i] >= 3 || S.p_type[i] >= 1000) continue;
            int bt = S.buffer_type[i], pt = S.p_type[i];
            if (pt == 9) {
                T.ux[i] = S.ux[i]; T.uy[i] = S.uy[i]; T.uz[i] = S.uz[i];
            } else {
                Real tux0, tuy0, tuz0, dux, duy, duz;
                if (pt > 0) {
                    tux0 = S.ux[i]; tuy0 = S.uy[i]; tuz0 = S.uz[i];
                    if (bt == 1 || bt == -1) { tux0 = S2.ux0[i]; tuy0 = S2.uy0[i]; tuz0 = S2.uz0[i]; }
                    dux = S3.fpx[i] * (bt == 0) + S.fbx[i] / S.rho[i] + S.fmx[i];
                    duy = S3.fpy[i] * (bt == 0) + S.fby[i] / S.rho[i] + S.fmy[i];
                    duz = S3.fpz[i] * (bt == 0) + S.fbz[i] / S.rho[i];
                } else {
                    tux0 = S2.ux0[i]; tuy0 = S2.uy0[i]; tuz0 = S2.uz0[i];
                    dux = duy = duz = 0.0;
                }
                Real uxc = tux0 + dux * (tdt), uyc = tuy0 + duy * (tdt), uzc = tuz0 + duz * (tdt);
                float ul = q().u_limit();
                if ((uxc * uxc + uyc * uyc + uzc * uzc) >= ul * ul) { uxc = tux0; uyc = tuy0; uzc = tuz0; }
                T.ux[i] = uxc; T.uy[i] = uyc; T.uz[i] = uzc;
            }
            if (q().con_solve() == 1) {   // functions_TIME_ISPH.cuh:203-215
                if (q().enthalpy_eqn()) {
                    T.enthalpy[i] = S2.enthalpy0[i] + S3.denthalpy[i] * tdt;
                    T.temp[i] = S.temp[i];
                } else {
                    T.temp[i] = S2.temp0[i] + S3.dtemp[i] * tdt * (bt == 0);
                }
            } else {
                T.enthalpy[i] = S.enthalpy[i];
                T.temp[i] = S.temp[i];
            }
            if (q().concn_solve() == 1) {
                T.concn[i] = S2.concn0[i] + S3.dconcn[i] * tdt;
                if (T.concn[i] < 0.0) T.concn[i] = 0.0;
            } else {
                T.concn[i] = S.concn[i];
            }
            T.pres[i] = S.pres[i]; T.flt_s[i] = S.flt_s[i]; T.m[i] = S.m[i]; T.ncell[i] = S.ncell[i];
            T.h[i] = S.h[i]; T.k_turb[i] = S.k_turb[i]; T.e_turb[i] = S.e_turb[i]; T.eli[i] = S.eli[i];
            T.vol[i] = S.vol[i]; p2_rho_ref[i] = S2.rho_ref[i]; T.vis_t[i] = S.vis_t[i];
            T.fbx[i] = S.fbx[i]; T.fby[i] = S.fby[i]; T.fbz[i] = S.fbz[i];
            T.fmx[i] = S.fmx[i]; T.fmy[i] = S.fmy[i]; T.hmz[i] = S.hmz[i];
            T.f1[i] = S.f1[i]; T.f2[i] = S.f2[i]; T.f3[i] = S.f3[i];
            T.concentration[i] = S.concentration[i];
            if (T.source[i] == 1) T.concn[i] += 0.5 * tdt;
            if (T.p_type[i] == 0) {
                if (tdt * tcount >= prm.t_start && tdt * tcount < prm.t_con_t) T.temp[i] = prm.t_ini + tdt * tcount * (prm.t_con - prm.t_ini) / (prm.t_con_t - prm.t_start);
                else if (tdt * tcount < prm.t_start) T.temp[i] = prm.t_ini;
                else T.temp[i] = prm.t_con;
            }
        }
    }

    // IBM_corrector, functions_IBM.cuh:615-725
    void ibm_corrector(State<Real> &S, State<Real> &T) {
        for (int i = 0; i < n(); ++i) {
            if (S.p_type[i] < 1000) continue;
            T.fbx[i] = S.fbx[i]; T.fby[i] = S.fby[i]; T.fbz[i] = S.fbz[i];
            T.concentration[i] = S.concentration[i]; T.vol[i] = S.vol[i]; T.pres[i] = S.pres[i];
        }
    }

    // KERNEL_clc_IB_normal_vector3D, functions_PREP.cuh:923-1015
    void ib_normals(const State<Real> &A) {
        for (int i = 0; i < n(); ++i) {
            if (A.p_type[i] < 1000) continue;
            Real xi = A.x[i], yi = A.y[i], zi = A.z[i];
            Real nx = 0, ny = 0, nz = 0;
            const double *b = prm.ib_box;
            const double t = prm.ib_face_tol;
            if (std::abs(xi - b[0]) < t) nx = -1.0;
            if (std::abs(xi - b[1]) < t) nx = 1.0;
            if (std::abs(yi - b[2]) < t) ny = -1.0;
            if (std::abs(yi - b[3]) < t) ny = 1.0;
            if (std::abs(zi - b[4]) < t) nz = -1.0;
            if (std::abs(zi - b[5]) < t) nz = 1.0;
            Real mag = std::sqrt(nx * nx + ny * ny + nz * nz);
            if (mag > 1e-9) { S3.nx[i] = nx / mag; S3.ny[i] = ny / mag; S3.nz[i] = nz / mag; }
            else { S3.nx[i] = 0; S3.ny[i] = 0; S3.nz[i] = 0; }
        }
    }

    // ---- one step, SOPHIA_single_ISPH order -----------------------------------
    int step(int mode, double tol, int maxit, double &relres, int &iters) {
        const P Q = q();
        const Real tdt = Q.dt();
        int tc = count;
        float ttime = time;
        int st = SPH_OK;
        relres = 0; iters = 0;
        set_ncell(S1);
        if (tc == 0 || !built) {
            nnps();
            S3.reset(n());
            S = S1;
            S2.resize(n());
        } else {
            S = S1;
            // SP2 <- P2: only rho_ref carries over (P2's other fields are never
            // written back, ISPH_Calc.cuh:57 copies the initial zeros)
            S2.resize(n());
            S2.rho_ref = p2_rho_ref;
            S3.reset(n());
        }
#define PHASE(k) if (stop_after < (k)) return st
        PHASE(0);
        if (tc == 0) ib_normals(S1);
        PHASE(1);
        gradient_correction(S);
        PHASE(2);
        prep(S, tc, tdt);
        PHASE(3);
        if (Q.noslip() == 1) boundary(S);
        PHASE(4);
        most(S, tc, (float)tdt);
        PHASE(5);
        if (tc == 0) neumann(S);
        PHASE(6);
        advection(S);
        PHASE(7);
        if (Q.time_type() == 1) projection(S, tdt, ttime);
        PHASE(8);
        periodic(S);
        PHASE(9);
        freeslip(S);
        PHASE(10);
        if (mode == SPH_PPE_REF_SWEEP) ppe_sweep(S, tdt);
        else st = ppe_converged(S, tdt, tol, maxit, relres, iters);
        PHASE(11);
        neumann(S);
        PHASE(12);
        outlet_bc(S);
        PHASE(13);
        pressure_force(S);
        PHASE(14);
        ibm_force(S, tdt);
        PHASE(15);
        ibm_spread(S);
        PHASE(16);
        time_update(S, S1, tdt, tc);
        PHASE(17);
        ibm_corrector(S, S1);
        PHASE(18);
        neumann(S1);
        PHASE(19);
        outlet_bc(S1);
        PHASE(20);
        periodic(S1);
        PHASE(21);
        freeslip(S1);
        PHASE(22);
        if (prm.inlet_recycling == 1) recycling(S1);
#undef PHASE
        time = time + Q.dt();
        count = tc + 1;
        return st;
    }

    // KERNEL_clc_TemptoEnthalpy (functions_ENERGY.cuh:3-12): every record
    // but i_type 3 gets enthalpy = enthalpy0 = Ttoh(temp, p_type)
    void temp_to_enthalpy() {
        const bool pt = P{prm}.prop_table() == 1;
        for (int i = 0; i < n(); ++i) {
            if (S1.i_type[i] == 3) continue;
            const Real v = Ttoh<Real>(S1.temp[i], S1.p_type[i], pt, tab, S1.enthalpy[i]);
            S1.enthalpy[i] = v;
            S2.enthalpy0[i] = v;
        }
    }
    // KERNEL_clc_EnthalpytoTemp (functions_ENERGY.cuh:15-25): temp = htoT(enthalpy, p_type)
    void enthalpy_to_temp() {
        const bool pt = P{prm}.prop_table() == 1;
        for (int i = 0; i < n(); ++i) {
            if (S1.i_type[i] == 3) continue;
            S1.temp[i] = htoT<Real>(S1.enthalpy[i], S1.p_type[i], pt, tab, S1.temp[i]);
        }
    }

    void download(sph_part1 *A, sph_part2 *B, sph_part3 *C) const {
        for (int i = 0; i < n(); ++i) {
            if (A) {
                sph_part1 &r = A[i];
                std::memset(&r, 0, sizeof(r));
                r.i_type = S1.i_type[i]; r.buffer_type = S1.buffer_type[i]; r.MOST_buffer = S1.most[i];
                r.p_type = S1.p_type[i]; r.ncell = S1.ncell[i]; r.source = S1.source[i];
                r.x = S1.x[i]; r.y = S1.y[i]; r.z = S1.z[i]; r.ux = S1.ux[i]; r.uy = S1.uy[i]; r.uz = S1.uz[i];
                r.m = S1.m[i]; r.h = S1.h[i]; r.temp = S1.temp[i]; r.pres = S1.pres[i]; r.pres0 = S1.pres0[i];
                r.rho = S1.rho[i]; r.flt_s = S1.flt_s[i]; r.enthalpy = S1.enthalpy[i]; r.concn = S1.concn[i];
                r.concentration = S1.concentration[i]; r.k_turb = S1.k_turb[i]; r.e_turb = S1.e_turb[i];
                r.eli = S1.eli[i]; r.vol = S1.vol[i]; r.m_ref = S1.m_ref[i]; r.h_ref = S1.h_ref[i];
                r.vis_t = S1.vis_t[i]; r.fbx = S1.fbx[i]; r.fby = S1.fby[i]; r.fbz = S1.fbz[i];
                r.fmx = S1.fmx[i]; r.fmy = S1.fmy[i]; r.hmz = S1.hmz[i];
                r.float1 = S1.f1[i]; r.float2 = S1.f2[i]; r.float3 = S1.f3[i];
            }
            if (B) {
                sph_part2 &r = B[i];
                std::memset(&r, 0, sizeof(r));
                r.rho_ref = S2.rho_ref.empty() ? 0 : S2.rho_ref[i];
                r.SR = S2.SR.empty() ? 0 : S2.SR[i];
                r.x0 = S2.x0[i]; r.y0 = S2.y0[i]; r.z0 = S2.z0[i];
                r.ux0 = S2.ux0[i]; r.uy0 = S2.uy0[i]; r.uz0 = S2.uz0[i];
                r.temp0 = S2.temp0[i]; r.concn0 = S2.concn0[i]; r.enthalpy0 = S2.enthalpy0[i];
            }
            if (C) {
                sph_part3 &r = C[i];
                std::memset(&r, 0, sizeof(r));
                r.ftotalx = S3.ftx[i]; r.ftotaly = S3.fty[i]; r.ftotalz = S3.ftz[i]; r.ftotal = S3.ft[i];
                r.fpx = S3.fpx[i]; r.fpy = S3.fpy[i]; r.fpz = S3.fpz[i]; r.dtemp = S3.dtemp[i];
                r.dconcn = S3.dconcn[i]; r.denthalpy = S3.denthalpy[i];
                r.nx = S3.nx[i]; r.ny = S3.ny[i]; r.nz = S3.nz[i];
                r.inv_cm_xx = S3.gxx[i]; r.inv_cm_yy = S3.gyy[i]; r.inv_cm_zz = S3.gzz[i];
                r.inv_cm_xy = S3.gxy[i]; r.inv_cm_yz = S3.gyz[i]; r.inv_cm_zx = S3.gzx[i];
            }
        }
    }
};

struct OracleHandle {
    int prec;
    Oracle<float> *f = nullptr;
    Oracle<double> *d = nullptr;
};

}  // namespace

extern "C" {

void *orc_create(const sph_params *p, int precision) {
    OracleHandle *h = new OracleHandle();
    h->prec = precision;
    if (precision == SPH_PREC_FP64) { h->d = new Oracle<double>(); h->d->prm = *p; h->d->prec = 1; }
    else { h->f = new Oracle<float>(); h->f->prm = *p; h->f->prec = 0; }
    return h;
}

// the property tables of the enthalpy form's htoT (the upload of
// ISPH_Calc.cuh:370-377): h and T columns, index and size per slot
int orc_set_tables(void *hh, const sph_prop_tables *t) {
    OracleHandle *h = (OracleHandle *)hh;
    auto go = [&](auto *o) {
        if (!o) return;
        typedef typename std::remove_reference<decltype(o->tab.h[0])>::type R;
        for (int k = 0; k < SPH_TABLE_SIZE; ++k) { o->tab.h[k] = (R)t->h[k]; o->tab.T[k] = (R)t->T[k]; }
        for (int k = 0; k < SPH_TABLE_SLOTS; ++k) { o->tab.index[k] = t->index[k]; o->tab.size[k] = t->size[k]; }
        o->tab.set = true;
    };
    go(h->f);
    go(h->d);
    return SPH_OK;
}

int orc_temp_to_enthalpy(void *hh, int inverse) {
    OracleHandle *h = (OracleHandle *)hh;
    auto go = [&](auto *o) {
        if (!o) return;
        if (inverse) o->enthalpy_to_temp();
        else o->temp_to_enthalpy();
    };
    go(h->f);
    go(h->d);
    return SPH_OK;
}

void orc_destroy(void *hh) {
    OracleHandle *h = (OracleHandle *)hh;
    delete h->f; delete h->d; delete h;
}

int orc_set_params(void *hh, const sph_params *p) {
    OracleHandle *h = (OracleHandle *)hh;
    if (h->f) { int c = h->f->count; float t = h->f->time; h->f->prm = *p; h->f->count = c; h->f->time = t; }
    if (h->d) { int c = h->d->count; float t = h->d->time; h->d->prm = *p; h->d->count = c; h->d->time = t; }
    return SPH_OK;
}

int orc_upload(void *hh, const sph_part1 *P1, int n) {
    OracleHandle *h = (OracleHandle *)hh;
    if (h->f) h->f->upload(P1, n); else h->d->upload(P1, n);
    return SPH_OK;
}

int orc_nnps(void *hh) {
    OracleHandle *h = (OracleHandle *)hh;
    if (h->f) h->f->nnps(); else h->d->nnps();
    return SPH_OK;
}

int orc_export_nnps(void *hh, int32_t *g_idx, int32_t *p_idx, int32_t *g_str, int32_t *g_end) {
    OracleHandle *h = (OracleHandle *)hh;
    auto go = [&](auto *o) {
        const int N = o->n();
        const int NC = o->prm.vii[28] + 1;
        if (g_idx) std::memcpy(g_idx, o->g_idx.data(), 4 * N);
        if (p_idx) std::memcpy(p_idx, o->p_idx.data(), 4 * N);
        if (g_str) std::memcpy(g_str, o->g_str.data(), 4 * NC);
        if (g_end) std::memcpy(g_end, o->g_end.data(), 4 * NC);
    };
    if (h->f) go(h->f); else go(h->d);
    return SPH_OK;
}

int64_t orc_nnz(void *hh) {
    OracleHandle *h = (OracleHandle *)hh;
    return h->f ? (int64_t)h->f->nb.size() : (int64_t)h->d->nb.size();
}

int orc_export_neighbors(void *hh, int64_t *off, int32_t *list) {
    OracleHandle *h = (OracleHandle *)hh;
    auto go = [&](auto *o) {
        if (off) std::memcpy(off, o->nb_off.data(), 8 * (o->n() + 1));
        if (list) std::memcpy(list, o->nb.data(), 4 * o->nb.size());
    };
    if (h->f) go(h->f); else go(h->d);
    return SPH_OK;
}

int orc_step(void *hh, int mode, double tol, int maxit, double *relres, int *iters) {
    OracleHandle *h = (OracleHandle *)hh;
    double rr = 0; int it = 0;
    int st = h->f ? h->f->step(mode, tol, maxit, rr, it) : h->d->step(mode, tol, maxit, rr, it);
    if (relres) *relres = rr;
    if (iters) *iters = it;
    return st;
}

void orc_set_stop_after(void *hh, int k) {
    OracleHandle *h = (OracleHandle *)hh;
    if (h->f) h->f->stop_after = k; else h->d->stop_after = k;
}

// exports the working state (dev_SP1 of the reference) in P1 layout
int orc_download_work(void *hh, sph_part1 *P1) {
    OracleHandle *h = (OracleHandle *)hh;
    auto go = [&](auto *o) { auto keep = o->S1; o->S1 = o->S; o->download(P1, nullptr, nullptr); o->S1 = keep; };
    if (h->f) go(h->f); else go(h->d);
    return SPH_OK;
}

// assembles the converged-PPE system of the current working state (call
// after a step stopped at phase 10 with orc_set_stop_after); returns nnz
int64_t orc_assemble(void *hh, int64_t *ro, int32_t *ci, double *va, double *rhs) {
    OracleHandle *h = (OracleHandle *)hh;
    int64_t nnz = 0;
    auto go = [&](auto *o) {
        std::vector<int64_t> r; std::vector<int> c; std::vector<double> v, b;
        o->assemble(o->S, o->q().dt(), r, c, v, b);
        nnz = (int64_t)c.size();
        if (ro) std::memcpy(ro, r.data(), 8 * r.size());
        if (ci) std::memcpy(ci, c.data(), 4 * c.size());
        if (va) std::memcpy(va, v.data(), 8 * v.size());
        if (rhs) std::memcpy(rhs, b.data(), 8 * b.size());
    };
    if (h->f) go(h->f); else go(h->d);
    return nnz;
}

int orc_pin_row(void *hh) {
    OracleHandle *h = (OracleHandle *)hh;
    return h->f ? h->f->pin_row : h->d->pin_row;
}

int orc_ncomp(void *hh) {
    OracleHandle *h = (OracleHandle *)hh;
    return h->f ? (int)h->f->comp_size.size() : (int)h->d->comp_size.size();
}

int orc_pins(void *hh, int32_t *out) {
    OracleHandle *h = (OracleHandle *)hh;
    const std::vector<int> &v = h->f ? h->f->pins : h->d->pins;
    if (out) std::memcpy(out, v.data(), 4 * v.size());
    return (int)v.size();
}

int orc_download(void *hh, sph_part1 *P1, sph_part2 *P2, sph_part3 *P3) {
    OracleHandle *h = (OracleHandle *)hh;
    if (h->f) h->f->download(P1, P2, P3); else h->d->download(P1, P2, P3);
    return SPH_OK;
}

}  // extern "C"
