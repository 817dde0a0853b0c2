// Shared device definitions of the B200 ISPH step (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>

#include "sph_isph.h"

namespace sph {

// ---- status handling --------------------------------------------------------
#define SPH_CUDA_TRY(expr)                                                   \
    do {                                                                     \
        cudaError_t e_ = (expr);                                             \
        if (e_ != cudaSuccess) {                                             \
            ::sph::set_cuda_error(e_, #expr, __FILE__, __LINE__);            \
            return SPH_ERR_CUDA;                                             \
        }                                                                    \
    } while (0)

#define SPH_TRY(expr)                                                        \
    do {                                                                     \
        int s_ = (expr);                                                     \
        if (s_ < 0) return s_;                                               \
    } while (0)

void set_cuda_error(cudaError_t e, const char *what, const char *file, int line);
void set_error(const char *msg);

// ---- device parameters (by value in every launch) ---------------------------
struct DevParams {
    int n, NI, NJ, NK, num_cells;
    int kernel_type, time_type, freq_filt, fp_solve, fv_solve, fg_solve, kgc_solve, turb, noslip;
    int con_solve, boussinesq, concn_solve;
    int outlet_bc, inlet_recycling;
    int ppe_pair_h;        // 1: pair-averaged h in the pressure system
    int pforce_form;       // pressure-force pair term: 0 the reference's active form, 1 difference form
    int enthalpy_eqn;      // 1: the energy equation in enthalpy (with con_solve)
    int prop_table;        // vii[2] = 1: htoT reads the property tables (k_table_index / k_table_size)
    int tab_index[SPH_TABLE_SLOTS], tab_size[SPH_TABLE_SLOTS];
    double rp_x, rp_y;     // recycling probe
    double periodic_box[6];   // x0,x1,y0,y1,z0,z1 of the periodic box (ghost partners)
    float kappa, skappa, dcell, xmin, xmax, ymin, ymax, zmin, zmax, dt, u_limit, dt_structure;
    double cs_sgs, l2, l3, l_left, l_right, outlet_probe_dx, partner_tol, ghost_tol;
    double ib_box[6], ib_face_tol, most_z0, most_z0h, most_ghost_dz, rho_air, ibm_target_coeff;
    double visc_fluid, visc_wall, visc_marker, av_alpha, av_beta, av_c0;
    double pressure_length, ibm_length, neumann_coeff;
    double t_ini, t_con, t_start, t_con_t, boundary_velocity;
    int n_profile;
    double profile_z[SPH_MAX_PROFILE], profile_u[SPH_MAX_PROFILE];
};

DevParams make_dev_params(const sph_params &p);

// ---- step counter and time, read on the device ----------------------------
// The kernels that depend on the step (the filter period, rho_ref at step 0,
// the thermal ramp) read them here instead of taking them as launch
// arguments, so that a captured step replays correctly at any later step;
// the last kernel of each step advances them.
struct StepClock {
    int count;      // vii[SPH_VII_COUNT] of the step being computed
    float time;     // vif[SPH_VIF_TIME] of that step
};

// ---- neighbour-class bits of a particle (read on the j side of pair loops) --
enum : int {
    JB_PT1 = 1,          // p_type == 1 (fluid)
    JB_LT1000 = 2,       // p_type < 1000 (not an IBM marker)
    JB_POSN9 = 4,        // p_type > 0 && p_type != 9 (no-slip source)
    JB_PT1000 = 8,       // p_type == 1000
    JB_IT4 = 16,         // i_type == 4
    JB_BUF0 = 32,        // buffer_type == 0
    JB_PT0 = 64,         // p_type == 0
    JB_MON0 = 128,       // p_type <= 0 || p_type >= 1000
};

__host__ __device__ inline int jclass_of(int i_type, int buffer_type, int p_type) {
    int c = 0;
    if (p_type == 1) c |= JB_PT1;
    if (p_type < 1000) c |= JB_LT1000;
    if (p_type > 0 && p_type != 9) c |= JB_POSN9;
    if (p_type == 1000) c |= JB_PT1000;
    if (i_type == 4) c |= JB_IT4;
    if (buffer_type == 0) c |= JB_BUF0;
    if (p_type == 0) c |= JB_PT0;
    if (p_type <= 0 || p_type >= 1000) c |= JB_MON0;
    return c;
}

// ---- vector types -------------------------------------------------------------
template <class T> struct V4;
template <> struct V4<float> { typedef float4 type; };
template <> struct V4<double> { typedef double4 type; };
template <class T> struct V2;
template <> struct V2<float> { typedef float2 type; };
template <> struct V2<double> { typedef double2 type; };

// streaming (evict-first) loads of a Real4 read once per pass
__device__ __forceinline__ float4 ld_stream(const float4 *p) { return __ldcs(p); }
__device__ __forceinline__ double4 ld_stream(const double4 *p) {
    const double2 a = __ldcs(reinterpret_cast<const double2 *>(p));
    const double2 b = __ldcs(reinterpret_cast<const double2 *>(p) + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}

template <class T> __host__ __device__ inline typename V4<T>::type mk4(T a, T b, T c, T d) {
    typename V4<T>::type v; v.x = a; v.y = b; v.z = c; v.w = d; return v;
}

// ---- exact FP32 arithmetic for the NNPS predicates ---------------------------
// The reference evaluates cell indices and distance tests in FP32 IEEE
// arithmetic; these helpers keep nvcc from fusing them into FMAs so the
// results are the correctly rounded ones the reference's host build gives.
__device__ __forceinline__ float d2_rn(float xi, float yi, float zi, float xj, float yj, float zj) {
    float dx = __fsub_rn(xi, xj), dy = __fsub_rn(yi, yj), dz = __fsub_rn(zi, zj);
    return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}
__device__ __forceinline__ float dist_rn(float xi, float yi, float zi, float xj, float yj, float zj) {
    return __fsqrt_rn(d2_rn(xi, yi, zi, xj, yj, zj));
}

// binning formula, functions_NNPS.cuh:890-898
__host__ __device__ inline int bin_axis(float v, float vmin, float vmax, int N) {
    if (vmax == vmin) return 0;
#ifdef __CUDA_ARCH__
    float t = floorf(__fmul_rn(__fdiv_rn(__fsub_rn(v, vmin), __fsub_rn(vmax, vmin)), (float)N));
#else
    float t = std::floor((v - vmin) / (vmax - vmin) * N);
#endif
    int c = (int)((t < (float)(N - 1)) ? t : (float)(N - 1));
    return c < 0 ? 0 : c;
}
// search formula, functions_PPE.cuh:52-59
__host__ __device__ inline int search_axis(float v, float vmin, float vmax, float dcell, int N) {
    if (vmax == vmin) return 0;
#ifdef __CUDA_ARCH__
    float t = floorf(__fdiv_rn(__fsub_rn(v, vmin), dcell));
#else
    float t = std::floor((v - vmin) / dcell);
#endif
    int c = (int)((t < (float)(N - 1)) ? t : (float)(N - 1));
    return c < 0 ? 0 : c;
}

// ---- kernel functions, functions_KNL.cuh:2-103 and :326-369 -------------------
template <class Real>
__device__ __forceinline__ Real calc_tmpA(const DevParams &P, Real tH) {
    const float kap = P.kappa;
    const double PI_REF = 3.141592653;
    switch (P.kernel_type) {
        case 0: return (Real)(1.0 / (pow(PI_REF, 1.5) * pow((double)tH, 3.0)));
        case 1: return (Real)(3.0 / (359.0 * PI_REF * pow((double)tH, 3.0)));
        case 2: return (Real)(315.0 / (208.0 * PI_REF * pow((double)tH, 3.0)));
        case 3: return (Real)(3.342253804929802 / (kap * tH) / (kap * tH) / (kap * tH));
        case 4: return (Real)(4.923856051905513 / (kap * tH) / (kap * tH) / (kap * tH));
        case 5: return (Real)(6.788953041263660 / (kap * tH) / (kap * tH) / (kap * tH));
    }
    return (Real)0;
}

template <class Real>
__device__ __forceinline__ Real pw(Real a, int k) {
    Real r = 1;
    for (int i = 0; i < k; ++i) r *= a;
    return r;
}

// tR = rr / (kappa tH) as a product with the reciprocal, which the pair loops
// hoist out (tH is the row's smoothing length); within FP rounding of the
// reference's rr / tH / kappa
template <class Real>
__device__ __forceinline__ Real calc_wij(const DevParams &P, Real tA, Real tH, Real rr) {
    const Real tR = rr * ((Real)1 / (tH * (Real)P.kappa));
    const Real o = (Real)1 - tR;
    switch (P.kernel_type) {
        case 0: return tA * (Real)exp(-(double)(2 * tR) * (double)(2 * tR));
        case 1:
            if (tR < (Real)0.5) return tA * (pw<Real>(3 - 2 * tR, 5) - 6 * pw<Real>(2 - 2 * tR, 5) + 15 * pw<Real>(1 - 2 * tR, 5));
            if (tR < (Real)1) return tA * (pw<Real>(3 - 2 * tR, 5) - 6 * pw<Real>(2 - 2 * tR, 5));
            if (tR < (Real)1.5) return tA * pw<Real>(3 - 2 * tR, 5);
            return 0;
        case 2:
            return (tR < 1) ? tA * (Real)(2.0 / 3.0 - 9.0 / 2.0 * tR * tR + 19.0 / 3.0 * tR * tR * tR - 5.0 / 2.0 * tR * tR * tR * tR) : (Real)0;
        case 3: return (tR < 1) ? tA * o * o * o * o * (1 + 4 * tR) : (Real)0;
        case 4: return (tR < 1) ? tA * o * o * o * o * o * o * (Real)(1 + 6 * tR + (Real)11.666666666666666 * tR * tR) : (Real)0;
        case 5: {
            const Real o2 = o * o, o4 = o2 * o2;
            return (tR < 1) ? tA * o4 * o4 * (1 + 8 * tR + 25 * tR * tR + 32 * tR * tR * tR) : (Real)0;
        }
    }
    return 0;
}

template <class Real>
__device__ __forceinline__ Real calc_dwij(const DevParams &P, Real tA, Real tH, Real rr) {
    const Real kap = (Real)P.kappa;
    const Real tR = rr * ((Real)1 / (tH * kap));
    const Real o = (Real)1 - tR;
    switch (P.kernel_type) {
        case 0: return (1 / tH) * tA * (-4 * tR) * (Real)exp(-(double)(2 * tR) * (double)(2 * tR));
        case 1:
            if (tR < (Real)0.5) return (1 / tH) * tA * (-5 * pw<Real>(3 - 2 * tR, 4) + 30 * pw<Real>(2 - 2 * tR, 4) - 75 * pw<Real>(1 - 2 * tR, 4));
            if (tR < (Real)1) return (1 / tH) * tA * (-5 * pw<Real>(3 - 2 * tR, 4) + 30 * pw<Real>(2 - 2 * tR, 4));
            if (tR < (Real)1.5) return (1 / tH) * tA * (-5 * pw<Real>(3 - 2 * tR, 4));
            return 0;
        case 2:
            return (tR < 1) ? (1 / tH) * tA * (Real)(-9.0 * tR + 19.0 * tR * tR - 10.0 * tR * tR * tR) : (Real)0;
        case 3: return (tR < 1) ? (1 / (kap * tH)) * tA * (-20 * tR * o * o * o) : (Real)0;
        case 4: return (tR < 1) ? (1 / (kap * tH)) * tA * ((Real)-18.666666666666668 * tR * o * o * o * o * o * (5 * tR + 1)) : (Real)0;
        case 5: {
            const Real o2 = o * o, o4 = o2 * o2;
            return (tR < 1) ? (1 / (kap * tH)) * tA * (-22 * tR * o4 * o2 * o * (16 * tR * tR + 7 * tR + 1)) : (Real)0;
        }
    }
    return 0;
}

// Wendland-6 shape with the kernel_type normalisation (functions_PPE.cuh:20,102-103)
template <class Real>
__device__ __forceinline__ Real calc_dwij_pressure(const DevParams &P, Real tA, Real tH, Real rr) {
    const Real kap = (Real)P.kappa;
    const Real tR = rr * ((Real)1 / (tH * kap));
    const Real o = (Real)1 - tR, o2 = o * o, o4 = o2 * o2;
    return (tR < 1) ? (1 / (kap * tH)) * tA * (-22 * tR * o4 * o2 * o * (16 * tR * tR + 7 * tR + 1)) : (Real)0;
}

// viscosity2, functions_PROP.cuh:121-131, from the neighbour-class bits
template <class Real>
__device__ __forceinline__ Real visc2(const DevParams &P, int jc) {
    if (jc & JB_PT1) return (Real)(float)P.visc_fluid;
    if (jc & JB_PT0) return (Real)(float)P.visc_wall;
    if (jc & JB_PT1000) return (Real)(float)P.visc_marker;
    return (Real)(float)P.visc_fluid;
}

#define SPH_MAX_COMP 8

__host__ __device__ inline int div_up(long long a, long long b) { return (int)((a + b - 1) / b); }

// 16-bit neighbour codes of the pressure operator.  A row searches cell
// planes dz in [-2, 2] around its own; the records of plane dz that it can
// reach lie in cell_start[plane_cell(rc, dz)] ... onwards, with rc the
// row's first x-run cell in its own y-row and plane (dy = dz = 0).  An entry
// j is (dz + 2) << 13 | (j - that start), offsets up to 8191.
//
// The pressure coefficients and these codes are stored four entries of a row
// together (a slice of 32 rows holds a multiple of four entries per row):
// entry k of lane l sits at sell4(slice start, l, k), so one 16-byte load
// brings four FP32 coefficients and one 8-byte load four codes.
__host__ __device__ inline long long sell4(long long slice_base, int lane, int k) {
    return slice_base + 128LL * (k >> 2) + 4 * lane + (k & 3);
}
constexpr int kCodeShift = 13;
constexpr unsigned kCodeMask = (1u << kCodeShift) - 1u;
__host__ __device__ inline int plane_cell(int rc, int dz, int NI, int NINJ, int cs_max) {
    const int k = rc - 2 * NI + dz * NINJ;
    return k < 0 ? 0 : (k > cs_max ? cs_max : k);
}

}  // namespace sph
