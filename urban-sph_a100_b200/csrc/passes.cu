// Interaction and time-update passes of the ISPH step, one thread per
// particle over the SELL-32 neighbour lists (or over precomputed side lists
// for the boundary subsets).  Each kernel cites the reference kernel whose
// formula it evaluates.  Semantics differ from the reference only where the
// reference races: every pass reads the state as it was before the pass.
#include <algorithm>
#include <cfloat>
#include <cstdio>

#include "ctx.cuh"

namespace sph {

#define SELL_LOOP_BEGIN(i)                                                \
    const long long sbase_ = slice_off[(i) >> 5] + ((i)&31);              \
    const int scnt_ = ncnt[(i)];                                          \
    for (int k_ = 0; k_ < scnt_; ++k_) {                                  \
        const int j = __ldg(&nbr[sbase_ + 32LL * k_]);
#define SELL_LOOP_END }

#define LIST_ARGS const long long *__restrict__ slice_off, const int *__restrict__ ncnt, const int *__restrict__ nbr

template <class Real>
struct SoA {
    typedef typename V4<Real>::type R4;
    typedef typename V2<Real>::type R2;
    const float4 *__restrict__ pf;
    const R4 *__restrict__ pr;
    const R2 *__restrict__ mr;
    const int4 *__restrict__ ty;
    const int *__restrict__ jc;
};

// FP32 radius test of the individual kernels against kappa*h_i, needed only
// when h_j > h_i (the canonical list already holds r < kappa*max(h_i, h_j)).
__device__ __forceinline__ bool within_hi(const DevParams &P, float4 a, float4 b) {
    if (b.w <= a.w) return true;
    return dist_rn(a.x, a.y, a.z, b.x, b.y, b.z) < __fmul_rn(P.skappa, a.w);
}

// the device clock: set from the host's copy, and advanced by one step
// (the same float addition as the host's, so the two stay equal)
__global__ void k_set_clock(StepClock *clk, int count, float time) {
    clk->count = count;
    clk->time = time;
}

__global__ void k_advance_clock(StepClock *clk, float dt) {
    clk->count += 1;
    clk->time = __fadd_rn(clk->time, dt);
}

// ---------------------------------------------------------------------------
// step start: SP1 <- P1, SP2 <- P2, memset(P3) (ISPH_Calc.cuh:42-61)
// ---------------------------------------------------------------------------
template <class Real>
__global__ void k_begin_step(Ctx<Real> c) {
    typedef typename V4<Real>::type R4;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    const VarSet<Real> &A = c.A;
    const VarSet<Real> &S = c.S;
    S.u[i] = A.u[i]; S.p[i] = A.p[i]; S.temp[i] = A.temp[i]; S.flt[i] = A.flt[i];
    S.kt[i] = A.kt[i]; S.et[i] = A.et[i]; S.fb[i] = A.fb[i]; S.fm[i] = A.fm[i]; S.fl[i] = A.fl[i];
    S.concn[i] = A.concn[i]; S.enth[i] = A.enth[i];
    c.rho_ref_S[i] = c.rho_ref_A[i];
    c.SR[i] = 0;
    const R4 z = mk4<Real>(0, 0, 0, 0);
    c.u0[i] = z; c.ft[i] = z; c.fp[i] = z; c.nrm[i] = z;
    c.dtemp[i] = 0;
    c.dconcn[i] = 0; c.temp0[i] = 0; c.concn0[i] = 0;
    c.enth0[i] = 0; c.denth[i] = 0;
}

// KERNEL_clc_IB_normal_vector3D, functions_PREP.cuh:923-1015 (step 0 only)
// With several obstacles (sph_set_ib_boxes) a marker takes the normal of the
// first box on whose surface it lies; the reference has one hard-wired box.
template <class Real>
__global__ void k_ib_normals(DevParams P, const typename V4<Real>::type *pr, const int4 *ty,
                             typename V4<Real>::type *nrm, const double *boxes, int nbox, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || ty[i].w < 1000) return;
    const auto x = pr[i];
    Real nx = 0, ny = 0, nz = 0;
    const double t = P.ib_face_tol;
    for (int q = 0; q < (boxes ? nbox : 1); ++q) {
        const double *bb = boxes ? boxes + 6 * q : P.ib_box;
        const bool on = (double)x.x > bb[0] - t && (double)x.x < bb[1] + t && (double)x.y > bb[2] - t &&
                        (double)x.y < bb[3] + t && (double)x.z > bb[4] - t && (double)x.z < bb[5] + t;
        if (boxes && !on) continue;
        if (fabs((double)x.x - bb[0]) < t) nx = -1;
        if (fabs((double)x.x - bb[1]) < t) nx = 1;
        if (fabs((double)x.y - bb[2]) < t) ny = -1;
        if (fabs((double)x.y - bb[3]) < t) ny = 1;
        if (fabs((double)x.z - bb[4]) < t) nz = -1;
        if (fabs((double)x.z - bb[5]) < t) nz = 1;
        break;
    }
    const Real mag = sqrt(nx * nx + ny * ny + nz * nz);
    if (mag > (Real)1e-9) nrm[i] = mk4<Real>(nx / mag, ny / mag, nz / mag, 0);
    else nrm[i] = mk4<Real>(0, 0, 0, 0);
}

// ---------------------------------------------------------------------------
// KERNEL_clc_gradient_correction_3D, functions_KNL.cuh:216-324
// ---------------------------------------------------------------------------
template <class Real>
__global__ void __launch_bounds__(128) k_grad_corr(DevParams P, SoA<Real> s, LIST_ARGS, Real *__restrict__ g6, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const size_t N = (size_t)n;
    const float4 fi = s.pf[i];
    const auto xi = s.pr[i];
    const int pti = s.ty[i].w;
    Real txx = 0, tyy = 0, tzz = 0, txy = 0, tyz = 0, tzx = 0;
    if (s.ty[i].x != 3) {
        const Real hi = xi.w;
        const Real tA = calc_tmpA<Real>(P, hi);
        SELL_LOOP_BEGIN(i)
            const float4 fj = s.pf[j];
            if (fj.x == fi.x && fj.y == fi.y && fj.z == fi.z) continue;   // tdist > 0
            if (!within_hi(P, fi, fj)) continue;
            if (!(s.jc[j] & JB_PT1)) continue;
            const auto xj = s.pr[j];
            const auto mj = s.mr[j];
            const Real dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
            const Real tdist = sqrt(dx * dx + dy * dy + dz * dz);
            const Real tdwij = calc_dwij<Real>(P, tA, hi, tdist);
            const Real mtd = mj.x * tdwij;
            const Real rtd = (Real)1 / (mj.y * tdist);
            txx += -mtd * dx * dx * rtd;
            txy += -mtd * dy * dx * rtd;
            tyy += -mtd * dy * dy * rtd;
            tzx += -mtd * dx * dz * rtd;
            tyz += -mtd * dy * dz * rtd;
            tzz += -mtd * dz * dz * rtd;
        SELL_LOOP_END
    }
    Real det = txx * (tyy * tzz - tyz * tyz);
    det -= txy * (txy * tzz - tyz * tzx);
    det += tzx * (txy * tyz - tyy * tzx);
    Real gxx = 1, gyy = 1, gzz = 1, gxy = 0, gyz = 0, gzx = 0;
    if (fabs((double)det) > DBL_EPSILON && pti == 1) {
        const Real r = (Real)1 / det;
        gxx = (tyy * tzz - tyz * tyz) * r;
        gxy = (tzx * tyz - txy * tzz) * r;
        gzx = (txy * tyz - tzx * tyy) * r;
        gyy = (txx * tzz - tzx * tzx) * r;
        gyz = (tzx * txy - txx * tyz) * r;
        gzz = (txx * tyy - txy * txy) * r;
    }
    g6[i] = gxx; g6[N + i] = gyy; g6[2 * N + i] = gzz; g6[3 * N + i] = gxy; g6[4 * N + i] = gyz; g6[5 * N + i] = gzx;
}

// ---------------------------------------------------------------------------
// KERNEL_clc_prep3D, functions_PREP.cuh:287-488 (Shepard filter, strain rate,
// SSM / DDF sub-grid viscosity, reference density), in two parts.
// Particles never move, so the filter sum sum V_j W_ij, the LES length sum
// sum r^2 W_ij V_j and the strain weights V_j G_i grad W_ij of every pair
// are the same at every step (G_i = g6 while it is not recomputed):
// k_prep_cache computes them once per neighbour build (the reference's
// radius test against kappa h_i, fluid neighbours for the strain), and
// k_prep_cached evaluates the step's part, the strain rate from the
// velocities: 12 bytes of stored weights and ~15 flops per pair instead of
// ~110 flops.  The sums are those of the reference up to the order of two
// FP multiplications per pair (V_j (u_ji . G grad W) as (u_ji . V_j G grad W)).
// ---------------------------------------------------------------------------
template <class Real>
__global__ void __launch_bounds__(128) k_prep_cache(DevParams P, SoA<Real> s, LIST_ARGS, const Real *__restrict__ g6,
                                                    Real *__restrict__ prow, Real *__restrict__ pw, long long nnzp,
                                                    int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int4 ti = s.ty[i];
    if (ti.x > 2 || ti.w >= 1000 || ti.w <= 0) return;
    const size_t N = (size_t)n;
    const float4 fi = s.pf[i];
    const auto xi = s.pr[i];
    const Real gc11 = g6[i], gc22 = g6[N + i], gc33 = g6[2 * N + i], gc12 = g6[3 * N + i], gc23 = g6[4 * N + i], gc31 = g6[5 * N + i];
    const Real hi = xi.w;
    const Real tA = calc_tmpA<Real>(P, hi);
    Real tmp_flt = 0, tmp_sigma = 0;
    SELL_LOOP_BEGIN(i)
        const long long e = sbase_ + 32LL * k_;
        Real wx = 0, wy = 0, wz = 0;
        const float4 fj = s.pf[j];
        if (within_hi(P, fi, fj)) {
            const auto xj = s.pr[j];
            const auto mj = s.mr[j];
            const Real dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
            const Real tdist = sqrt(dx * dx + dy * dy + dz * dz) + (Real)1e-20;
            const Real w = calc_wij<Real>(P, tA, hi, tdist);
            const Real vj = mj.x / mj.y;
            tmp_flt += vj * w;
            tmp_sigma += tdist * tdist * w * vj;
            if (s.jc[j] & JB_PT1) {
                const Real dwi = calc_dwij<Real>(P, tA, hi, tdist) / tdist;
                const Real tdwx = dwi * dx, tdwy = dwi * dy, tdwz = dwi * dz;
                wx = vj * (gc11 * tdwx + gc12 * tdwy + gc31 * tdwz);
                wy = vj * (gc12 * tdwx + gc22 * tdwy + gc23 * tdwz);
                wz = vj * (gc31 * tdwx + gc23 * tdwy + gc33 * tdwz);
            }
        }
        pw[e] = wx; pw[nnzp + e] = wy; pw[2 * nnzp + e] = wz;
    SELL_LOOP_END
    prow[i] = tmp_flt;
    prow[N + i] = tmp_sigma;
}

template <class Real>
__global__ void __launch_bounds__(128) k_prep_cached(DevParams P, const int4 *__restrict__ ty, LIST_ARGS,
                                                     const Real *__restrict__ prow, const Real *__restrict__ pw,
                                                     long long nnzp, const typename V4<Real>::type *__restrict__ u,
                                                     const typename V2<Real>::type *__restrict__ mr,
                                                     const typename V4<Real>::type *__restrict__ pr,
                                                     Real *__restrict__ flt, Real *__restrict__ vis_out,
                                                     Real *__restrict__ kt, Real *__restrict__ et, Real *__restrict__ SR,
                                                     Real *__restrict__ rho_ref, const StepClock *__restrict__ clk,
                                                     Real tdt, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int4 ti = ty[i];
    const int tcount = clk->count;
    if (ti.x > 2 || ti.w >= 1000 || ti.w <= 0) return;
    const size_t N = (size_t)n;
    const bool filt = (tcount % P.freq_filt) == 0;
    const bool les = P.fv_solve != 0 && P.turb != 0;
    if (les) {
        const auto ui = u[i];
        const Real hi = pr[i].w;
        Real st11 = 0, st12 = 0, st22 = 0, st23 = 0, st31 = 0, st33 = 0;
        SELL_LOOP_BEGIN(i)
            const long long e = sbase_ + 32LL * k_;
            const Real cx = __ldcs(&pw[e]), cy = __ldcs(&pw[nnzp + e]), cz = __ldcs(&pw[2 * nnzp + e]);
            const auto uj = u[j];
            const Real ux = uj.x - ui.x, uy = uj.y - ui.y, uz = uj.z - ui.z;
            st11 += ux * cx;
            st12 += (Real)0.5 * (ux * cy + uy * cx);
            st22 += uy * cy;
            st23 += (Real)0.5 * (uy * cz + uz * cy);
            st31 += (Real)0.5 * (ux * cz + uz * cx);
            st33 += uz * cz;
        SELL_LOOP_END
        Real tmp_SR = 2 * (st11 * st11 + st22 * st22 + st33 * st33 + 2 * st12 * st12 + 2 * st31 * st31 + 2 * st23 * st23);
        tmp_SR = sqrt(tmp_SR);
        SR[i] = tmp_SR;
        const Real tmp_sigma = sqrt((Real)0.3333 * prow[N + i]);
        const Real cl = (tmp_sigma > hi) ? tmp_sigma : hi;
        const int bt = ti.y;
        if (P.turb == 4) {
            const Real v = (Real)(P.cs_sgs * P.cs_sgs) * cl * cl * tmp_SR;
            if (bt != 1) vis_out[i] = v;
        } else if (P.turb == 5) {
            Real ki = kt[i] > 0 ? kt[i] : (Real)0;
            const Real nui = ui.w;
            const Real pp = nui * tmp_SR * tmp_SR;
            const Real eps = (Real)0.93 * ki * sqrt(ki) / cl;     // Ce_sgs, Parameters.cuh:133
            ki += (pp - eps) * tdt;
            ki = (ki > (Real)1e-4) ? ki : (Real)1e-4;
            const Real v = (Real)0.1 * cl * sqrt(ki);              // Ck_sgs, Parameters.cuh:132
            if (bt != 1) { vis_out[i] = v; kt[i] = ki; et[i] = eps; }
        }
    }
    if (tcount == 0) rho_ref[i] = mr[i].y;
    if (filt) flt[i] = prow[i];
}

// The prep pass evaluated in full every step: used when the device has no
// room for the cached weights.
template <class Real>
__global__ void __launch_bounds__(128) k_prep(DevParams P, SoA<Real> s, LIST_ARGS, const Real *__restrict__ g6,
                                              const typename V4<Real>::type *__restrict__ u, Real *__restrict__ flt,
                                              Real *__restrict__ vis_out, Real *__restrict__ kt, Real *__restrict__ et,
                                              Real *__restrict__ SR, Real *__restrict__ rho_ref,
                                              const StepClock *__restrict__ clk, Real tdt, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int4 ti = s.ty[i];
    const int tcount = clk->count;
    if (ti.x > 2 || ti.w >= 1000 || ti.w <= 0) return;
    const size_t N = (size_t)n;
    const float4 fi = s.pf[i];
    const auto xi = s.pr[i];
    const auto ui = u[i];
    const auto mri = s.mr[i];
    const Real gc11 = g6[i], gc22 = g6[N + i], gc33 = g6[2 * N + i], gc12 = g6[3 * N + i], gc23 = g6[4 * N + i], gc31 = g6[5 * N + i];
    const Real hi = xi.w;
    const Real tA = calc_tmpA<Real>(P, hi);
    const bool filt = (tcount % P.freq_filt) == 0;
    const bool les = P.fv_solve != 0 && P.turb != 0;
    Real tmp_flt = 0, tmp_sigma = 0;
    Real st11 = 0, st12 = 0, st22 = 0, st23 = 0, st31 = 0, st33 = 0;
    SELL_LOOP_BEGIN(i)
        const float4 fj = s.pf[j];
        if (!within_hi(P, fi, fj)) continue;
        const auto xj = s.pr[j];
        const auto mj = s.mr[j];
        const Real dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
        const Real tdist = sqrt(dx * dx + dy * dy + dz * dz) + (Real)1e-20;
        const Real w = calc_wij<Real>(P, tA, hi, tdist);
        const Real vj = mj.x / mj.y;
        if (filt) tmp_flt += vj * w;
        if (les) {
            tmp_sigma += tdist * tdist * w * vj;
            if (s.jc[j] & JB_PT1) {
                const Real dwi = calc_dwij<Real>(P, tA, hi, tdist) / tdist;
                const Real tdwx = dwi * dx, tdwy = dwi * dy, tdwz = dwi * dz;
                const Real cx = gc11 * tdwx + gc12 * tdwy + gc31 * tdwz;
                const Real cy = gc12 * tdwx + gc22 * tdwy + gc23 * tdwz;
                const Real cz = gc31 * tdwx + gc23 * tdwy + gc33 * tdwz;
                const auto uj = u[j];
                const Real ux = uj.x - ui.x, uy = uj.y - ui.y, uz = uj.z - ui.z;
                st11 += vj * ux * cx;
                st12 += (Real)0.5 * vj * (ux * cy + uy * cx);
                st22 += vj * uy * cy;
                st23 += (Real)0.5 * vj * (uy * cz + uz * cy);
                st31 += (Real)0.5 * vj * (ux * cz + uz * cx);
                st33 += vj * uz * cz;
            }
        }
    SELL_LOOP_END
    if (les) {
        Real tmp_SR = 2 * (st11 * st11 + st22 * st22 + st33 * st33 + 2 * st12 * st12 + 2 * st31 * st31 + 2 * st23 * st23);
        tmp_SR = sqrt(tmp_SR);
        SR[i] = tmp_SR;
        tmp_sigma = sqrt((Real)0.3333 * tmp_sigma);
        const Real cl = (tmp_sigma > hi) ? tmp_sigma : hi;
        const int bt = ti.y;
        if (P.turb == 4) {
            const Real v = (Real)(P.cs_sgs * P.cs_sgs) * cl * cl * tmp_SR;
            if (bt != 1) vis_out[i] = v;
        } else if (P.turb == 5) {
            Real ki = kt[i] > 0 ? kt[i] : (Real)0;
            const Real nui = u[i].w;
            const Real pp = nui * tmp_SR * tmp_SR;
            const Real eps = (Real)0.93 * ki * sqrt(ki) / cl;     // Ce_sgs, Parameters.cuh:133
            ki += (pp - eps) * tdt;
            ki = (ki > (Real)1e-4) ? ki : (Real)1e-4;
            const Real v = (Real)0.1 * cl * sqrt(ki);              // Ck_sgs, Parameters.cuh:132
            if (bt != 1) { vis_out[i] = v; kt[i] = ki; et[i] = eps; }
        }
    }
    if (tcount == 0) rho_ref[i] = mri.y;
    if (filt) flt[i] = tmp_flt;
}

// vis_t lives in u.w; the LES result is staged and merged so that neighbours
// read the step-start value (the reference reads nu_j only in the unused Tk term)
template <class Real>
__global__ void k_merge_vis(typename V4<Real>::type *u, const Real *vis, const int4 *ty, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int4 t = ty[i];
    if (t.x > 2 || t.w >= 1000 || t.w <= 0 || t.y == 1) return;
    u[i].w = vis[i];
}

// ---------------------------------------------------------------------------
// KERNEL_boundary3D, functions_BC.cuh:100-190: wall velocity from fluid
// ---------------------------------------------------------------------------
template <class Real>
__global__ void __launch_bounds__(128) k_boundary(DevParams P, SoA<Real> s, LIST_ARGS,
                                                  typename V4<Real>::type *__restrict__ u, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int4 ti = s.ty[i];
    if (ti.x > 2 || ti.w != 0) return;
    const float4 fi = s.pf[i];
    const auto xi = s.pr[i];
    const Real hi = xi.w;
    const Real tA = calc_tmpA<Real>(P, hi);
    Real tx = 0, ty_ = 0, tz = 0, flt = (Real)1.0e-10;
    SELL_LOOP_BEGIN(i)
        if (!(s.jc[j] & JB_POSN9)) continue;
        const float4 fj = s.pf[j];
        if (!within_hi(P, fi, fj)) continue;
        const auto xj = s.pr[j];
        const Real dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
        const Real tdist = sqrt(dx * dx + dy * dy + dz * dz) - (Real)1e-20;
        const Real w = calc_wij<Real>(P, tA, hi, tdist);
        const auto uj = u[j];
        tx += uj.x * w; ty_ += uj.y * w; tz += uj.z * w; flt += w;
    SELL_LOOP_END
    auto ui = u[i];
    ui.x = -tx / flt; ui.y = -ty_ / flt; ui.z = -tz / flt;
    u[i] = ui;
}

// ---------------------------------------------------------------------------
// KERNEL_MOST_boundary3D, functions_MOST.cuh:151-322 (FP32 as written there)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float most_clamp(float v, float lo, float hi) { return fmaxf(lo, fminf(v, hi)); }
__device__ __forceinline__ double most_psi_m(float zeta) {
    if (zeta < 0.0f) {
        const float x = sqrtf(sqrtf(1.0f - 16.0f * zeta));
        return 3.14159265358979323846 * 0.5f - 2.0f * atanf(x) + logf((1.0f + x) * (1.0f + x) * (1.0f + x * x) * 0.125f);
    }
    return -5.0f * zeta;
}
__device__ __forceinline__ double most_psi_h(float zeta) {
    if (zeta < 0.0f) return 2.0f * logf(0.5f * (1.0f + sqrtf(1.0f - 16.0f * zeta)));
    return -5.0f * zeta;
}
__device__ __forceinline__ double most_Phi_m(float L, float z, float z0) { return logf(z / z0) - most_psi_m(z / L) + most_psi_m(z0 / L); }
__device__ __forceinline__ double most_Phi_h(float L, float z, float z0h) { return logf(z / z0h) - most_psi_h(z / L) + most_psi_h(z0h / L); }

template <class Real>
__global__ void k_most(DevParams P, SoA<Real> s, const int *rows, const int *off, const int *tgt, int nrows,
                       const typename V4<Real>::type *u, const Real *temp, typename V4<Real>::type *fm,
                       typename V4<Real>::type *fl, Real *dtemp, float *us_update, const StepClock *clk, float tdt) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nrows) return;
    const int tcount = clk->count;
    const int i = rows[k];
    const auto xi = s.pr[i];
    const auto ui = u[i];
    const float zi = (float)xi.z, tempi = (float)temp[i], rhoi = (float)s.mr[i].y, mi = (float)s.mr[i].x;
    const float uxi = (float)ui.x, uyi = (float)ui.y;
    const Real space = xi.w / (Real)1.5;    // h_coeff, Parameters.cuh:68
    const float z0 = (float)P.most_z0, z0h = (float)P.most_z0h;
    float u_star, theta_star, OB;
    float ts;
    if (tdt * tcount >= P.t_start && tdt * tcount < P.t_con_t) ts = P.t_ini + tdt * tcount * (P.t_con - P.t_ini) / (P.t_con_t - P.t_start);
    else if (tdt * tcount < P.t_start) ts = P.t_ini;
    else ts = P.t_con;
    float ws = sqrtf(uxi * uxi + uyi * uyi);
    ws = most_clamp(ws, 0.001f, 100.0f);
    const float Ri_b = (9.810 / tempi) * (tempi - ts) * zi / (ws * ws + 1e-10);
    if ((double)fabsf(Ri_b) > 1e-3) {
        OB = most_clamp(zi / Ri_b, -500.0f, 500.0f);
        for (int it = 0; it < 200; it++) {   // MAX_ITER, Parameters.cuh:109
            const float om = OB, ol = 0.999 * om, ou = 1.001 * om;
            const float fL = Ri_b - (zi / om) * most_Phi_h(om, zi, z0h) / powf((float)most_Phi_m(om, zi, z0), 2);
            const double pu = most_Phi_m(ou, zi, z0), pl = most_Phi_m(ol, zi, z0);
            const float dfL = ((-(zi / ou) * most_Phi_h(ou, zi, z0h) / (pu * pu)) - (-(zi / ol) * most_Phi_h(ol, zi, z0h) / (pl * pl))) / (ou - ol);
            OB -= 1.0f * fL / dfL;
            if ((double)fabsf(OB) > 1e-6) {   // TOLERANCE, Parameters.cuh:110
                if ((double)fabsf((OB - om) / OB) < 1e-5) break;
                else if ((double)fabsf(OB - om) < 1e-5) break;
            }
        }
        u_star = 0.4 * ws / most_Phi_m(OB, zi, z0);
        theta_star = 0.4 * (tempi - ts) / most_Phi_h(OB, zi, z0h);
    } else {
        OB = 1e6f;
        u_star = 0.4 * ws / logf(zi / z0);
        theta_star = 0.4 * (tempi - ts) / logf(zi / z0h);
    }
    const float mx = -rhoi * u_star * (uxi * u_star / ws);
    const float my = -rhoi * u_star * (uyi * u_star / ws);
    const Real shf = (Real)(-rhoi * 1005 * u_star * theta_star * 100.0);   // Air_cp, Parameters.cuh:119
    const Real q = (Real)0.5 * shf / (space * (Real)rhoi * (Real)1005);
    for (int e = off[k]; e < off[k + 1]; ++e) {
        const int j = tgt[e];
        atomicAdd(&dtemp[j], q);
        fm[j].z = q;
    }
    auto f = fm[i];
    f.x = (Real)(1.0 * mx * space * space / mi);
    f.y = (Real)(1.0 * my * space * space / mi);
    f.z = q;
    fm[i] = f;
    atomicAdd(&dtemp[i], q);
    fl[i] = mk4<Real>(u_star, theta_star, OB, 0);
    // the friction velocity at the recycling probe, functions_MOST.cuh:316
    const double dxp = (double)(float)xi.x - P.rp_x;
    const float dyp = (float)xi.y - (float)P.rp_y;
    if (dxp * dxp + (double)(dyp * dyp) < 1e-3) *us_update = u_star;
}

// ---------------------------------------------------------------------------
// KERNEL_Neumann_boundary3D, functions_BC.cuh:290-446, from the precomputed
// weights: p_w = sum w p (or the mirror extrapolation), u of p_type -1 from
// the Shepard weights; rows without fluid in range get p = 0.
// ---------------------------------------------------------------------------
template <class Real>
__global__ void __launch_bounds__(128) k_neumann_gather(const int *rows, const int *off, const int *nb, const int *mirror,
                                                        const double *w, const double *gw, int nrows, const Real *p,
                                                        const typename V4<Real>::type *u, const int4 *ty, Real *out_p,
                                                        typename V4<Real>::type *out_u) {
    // one warp per row: the lanes load 32 consecutive entries at a time
    // (coalesced) and form their terms, and every lane adds the terms in
    // entry order from the shuffles, so the sums are those of a sequential
    // loop over the row
    const int k = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (k >= nrows) return;   // uniform over the warp
    const int i = rows[k];
    const int s = off[k], e = off[k + 1];
    auto ui = u[i];
    Real pv = 0;
    if (e > s && !(mirror[k] & 2)) {
        const bool mir = (mirror[k] & 1) != 0;
        const bool vel = ty[i].w == -1;
        Real sp = 0, sx = 0, sy = 0, sz = 0;
        for (int q0 = s; q0 < e; q0 += 32) {
            const int q = q0 + lane;
            Real tp = 0, tx = 0, ty_ = 0, tz = 0;
            if (q < e) {
                const int j = nb[q];
                const Real wj = (Real)w[q];
                tp = (mir ? (Real)gw[q] : wj) * p[j];
                if (vel) { const auto uj = u[j]; tx = wj * uj.x; ty_ = wj * uj.y; tz = wj * uj.z; }
            }
            const int cnt = min(32, e - q0);
            for (int l = 0; l < cnt; ++l) {
                sp += __shfl_sync(0xffffffffu, tp, l);
                if (vel) {
                    sx += __shfl_sync(0xffffffffu, tx, l);
                    sy += __shfl_sync(0xffffffffu, ty_, l);
                    sz += __shfl_sync(0xffffffffu, tz, l);
                }
            }
        }
        pv = sp;
        if (vel) { ui.x = sx; ui.y = sy; ui.z = sz; }
    }
    if (lane == 0) {
        out_p[k] = pv;
        out_u[k] = ui;
    }
}

template <class Real>
__global__ void k_neumann_scatter(const int *rows, int nrows, const Real *in_p, const typename V4<Real>::type *in_u,
                                  Real *p, typename V4<Real>::type *u) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nrows) return;
    const int i = rows[k];
    p[i] = in_p[k];
    u[i] = in_u[k];
}

// ---------------------------------------------------------------------------
// KERNEL_advection_force3D, functions_PPE.cuh:191-480: viscous (Cleary or
// Monaghan), Eulerian convective term, artificial viscosity, gravity (~113
// flops per pair for Cleary with the Eulerian term, the artificial
// viscosity on about half the pairs, counted as for k_prep); with
// TH the scalar terms of the same pass: conduction and the Eulerian
// temperature term (con_solve -> dtemp), concentration advection-diffusion
// (concn_solve -> dconcn) and Boussinesq buoyancy (replaces the z force).
// Material constants of Parameters.cuh:120-131 and functions_PROP.cuh:192-212.
// ---------------------------------------------------------------------------
struct Scalars {
    const void *temp, *concn;
    void *dtemp, *dconcn, *denth;
};

__device__ __forceinline__ float th_k(int pt) {      // Solid_k / Air_k
    return (pt == 0 || pt == 1000) ? 1.0f : ((pt == 1 || pt == -1) ? 0.025f : 0.0f);
}
__device__ __forceinline__ float th_cp(int pt) {     // Solid_cp / Air_cp
    return (pt == 0 || pt == 1000) ? 900.0f : ((pt == 1 || pt == -1) ? 1005.0f : 0.0f);
}

template <class Real, int FV, int TH>
__global__ void __launch_bounds__(128) k_advection(DevParams P, SoA<Real> s, LIST_ARGS,
                                                   const typename V4<Real>::type *__restrict__ u,
                                                   const Real *__restrict__ eli,
                                                   typename V4<Real>::type *__restrict__ ft, Scalars sc, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int4 ti = s.ty[i];
    if (ti.x > 2 || ti.w == 1000 || ti.w <= 0) return;
    const Real *__restrict__ temp = (const Real *)sc.temp;
    const Real *__restrict__ concn = (const Real *)sc.concn;
    const bool con = TH && P.con_solve != 0, cnc = TH && P.concn_solve != 0, bsq = TH && P.boussinesq != 0;
    const Real tempi = TH ? temp[i] : (Real)0;
    const Real concni = cnc ? concn[i] : (Real)0;
    const Real kci = con ? (Real)th_k(ti.w) : (Real)0;
    Real eulert = 0, Rc = 0, Rd = 0, btemp = 0, bflt = 0;
    const int jci = s.jc[i];
    const auto xi = s.pr[i];
    const auto ui = u[i];
    const auto mri = s.mr[i];
    const Real hi = xi.w, mi = mri.x, rhoi = mri.y;
    const Real tA = calc_tmpA<Real>(P, hi);
    const Real visi = visc2<Real>(P, jci) + ui.w * rhoi;
    const Real el = eli[i];
    const Real Alpha = (Real)(float)P.av_alpha, Beta = (Real)(float)P.av_beta, c0 = (Real)(float)P.av_c0;
    const bool kgc = P.kgc_solve == 1;
    Real tx = 0, ty_ = 0, tz = 0, ex = 0, ey = 0, ez = 0;
    SELL_LOOP_BEGIN(i)
        const int jcj = s.jc[j];
        if (!(jcj & JB_LT1000)) continue;
        const auto xj = s.pr[j];
        const Real dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
        const Real tdist = sqrt(dx * dx + dy * dy + dz * dz) + (Real)1e-20;
        const Real it = (Real)1 / tdist;
        const Real dw_raw = calc_dwij<Real>(P, tA, hi, tdist);
        const Real dw = kgc ? (Real)0 : dw_raw;   // Cm is never filled on this path (all zero)
        const Real dwi = dw * it;
        const Real tdwx = dwi * dx, tdwy = dwi * dy, tdwz = dwi * dz;
        const auto uj = u[j];
        const auto mj = s.mr[j];
        const Real ux = ui.x - uj.x, uy = ui.y - uj.y, uz = ui.z - uj.z;
        if (FV == 1) {
            const Real visj = visc2<Real>(P, jcj) + uj.w * mj.y;
            Real C = dx * tdwx + dy * tdwy + dz * tdwz;
            C *= (visi * visj) / (visi + visj);
            C *= 4 * mj.x / (rhoi * mj.y);
            C *= it;   // twice, not it * it: the self pair has it = 1e20, whose square overflows FP32
            C *= it;
            tx += C * ux; ty_ += C * uy; tz += C * uz;
        } else if (FV == 2) {
            const Real uij_xij = ux * dx + uy * dy + uz * dz;
            const Real visj = visc2<Real>(P, jcj) + uj.w * mj.y;
            Real phi = uij_xij / (tdist * tdist + (Real)0.01 * hi * hi);
            Real Pij = (Real)(-2.0 * (3 + 2.0)) * phi * mj.x / mj.y;
            const Real Cv = (Real)2 * (visi * visj) / (visi + visj - (Real)1e-20);
            Pij *= Cv / rhoi;
            if ((jci & JB_MON0) || (jcj & JB_MON0)) Pij = 0;
            tx += -Pij * tdwx; ty_ += -Pij * tdwy; tz += -Pij * tdwz;
        }
        Real tempj = 0, concnj = 0;
        if (TH) { tempj = temp[j]; if (cnc) concnj = concn[j]; }
        if (el < (Real)1) {
            const Real vj = mj.x / mj.y * ((Real)1 - el);
            ex += (ui.x * (-ux) * tdwx + ui.y * (-ux) * tdwy + ui.z * (-ux) * tdwz) * vj;
            ey += (ui.x * (-uy) * tdwx + ui.y * (-uy) * tdwy + ui.z * (-uy) * tdwz) * vj;
            ez += (ui.x * (-uz) * tdwx + ui.y * (-uz) * tdwy + ui.z * (-uz) * tdwz) * vj;
            if (con)
                eulert -= (Real)2 * mj.x / (rhoi + mj.y) * (tempj - tempi) * (ux * tdwx + uy * tdwy + uz * tdwz) *
                          ((Real)1 - el);
            if (cnc) {
                const Real dc = concnj - concni;
                Rd -= (ui.x * dc * tdwx + ui.y * dc * tdwy + ui.z * dc * tdwz) * vj;
            }
        }
        if (TH && (con || cnc)) {
            const int ptj = s.ty[j].w;
            if (con) {   // conduction with the uncorrected dW/dr
                const Real kcj = (Real)th_k(ptj);
                const Real rhoj_t = (ptj == 1 || ptj == -1) ? mj.y : (Real)2300;
                const Real mj_t = mj.x * rhoj_t / mj.y;
                Real q = (Real)4 * mj_t * kcj * kci * (tempi - tempj) * dw_raw;
                q /= (tdist + (Real)1e-10) * rhoi * rhoj_t * (kci + kcj);
                Rc += q;
            }
            if (cnc) {   // diffusion_coefficient = 2
                Real d = mi * ((Real)2 * rhoi + (Real)2 * mj.y);
                d *= (dx * tdwx + dy * tdwy + dz * tdwz);
                d /= (rhoi * mj.y * (tdist * tdist + (Real)0.01 * hi * hi));
                Rd += (ti.w == ptj) ? d * (concni - concnj) : (Real)0;
            }
        }
        if (bsq) {
            const Real vw = mj.x / mj.y * calc_wij<Real>(P, tA, hi, tdist);
            btemp += vw * tempj;
            bflt += vw;
        }
        const Real uij_xij = ux * dx + uy * dy + uz * dz;
        if (uij_xij < 0) {
            const Real hij = (hi + xj.w) * (Real)0.5;
            Real phi = hij * uij_xij / (tdist * tdist + (Real)0.01 * hij * hij);
            Real Pij = mi * phi * (-Alpha * c0 + Beta * phi);
            Pij /= (rhoi + mj.y);
            Pij *= (Real)0.5;
            tx += -Pij * tdwx; ty_ += -Pij * tdwy; tz += -Pij * tdwz;
        }
    SELL_LOOP_END
    if (P.fg_solve) tz += (Real)-9.810;
    if (bsq && ti.w < 1000) tz = (Real)(1.0 / P.t_ini) * (Real)9.810 * (btemp / bflt - (Real)300);   // tempb 300 K
    ft[i] = mk4<Real>(tx - ex, ty_ - ey, tz - ez, sqrt(tx * tx + ty_ * ty_ + tz * tz));
    if (con) {   // functions_PPE.cuh:460-468
        if (P.enthalpy_eqn) ((Real *)sc.denth)[i] = Rc * (Real)(ti.w != -1);
        else ((Real *)sc.dtemp)[i] += Rc / (Real)th_cp(ti.w) - eulert;
    }
    if (cnc) ((Real *)sc.dconcn)[i] = Rd;
}

// interp2 (functions_PROP.cuh:8-41) over n >= 2 points: linear inside the
// table, the end segments extended outside it, each step of the segment
// formula rounded as the reference's Real arithmetic rounds it.  The slope
// multiplies the distance from the segment's left point, except past the
// last point, where the reference measures from the last point and adds its
// value (:16-21; equal in exact arithmetic, not in rounding).  The
// reference's search also tests the pair one past the table, but only for
// an x it cannot bracket, which a table with increasing x does not leave.
template <class Real>
__device__ __forceinline__ Real seg_rn(Real y0, Real y1, Real x0, Real x1, Real xa, Real ya, Real x);
template <>
__device__ __forceinline__ float seg_rn<float>(float y0, float y1, float x0, float x1, float xa, float ya, float x) {
    return __fadd_rn(__fmul_rn(__fdiv_rn(__fsub_rn(y1, y0), __fsub_rn(x1, x0)), __fsub_rn(x, xa)), ya);
}
template <>
__device__ __forceinline__ double seg_rn<double>(double y0, double y1, double x0, double x1, double xa, double ya,
                                                 double x) {
    return __dadd_rn(__dmul_rn(__ddiv_rn(__dsub_rn(y1, y0), __dsub_rn(x1, x0)), __dsub_rn(x, xa)), ya);
}
template <class Real>
__device__ Real interp2_rn(const Real *xd, const Real *yd, int n, Real x) {
    const int e = n - 1;
    if (xd[e] < x) return seg_rn<Real>(yd[e - 1], yd[e], xd[e - 1], xd[e], xd[e], yd[e], x);
    int a = 0;
    if (!(x <= xd[0]))
        for (int q = 0; q < e; ++q)
            if (xd[q] < x && x <= xd[q + 1]) { a = q; break; }
    return seg_rn<Real>(yd[a], yd[a + 1], xd[a], xd[a + 1], xd[a], yd[a], x);
}

// htoT / Ttoh (functions_PROP.cuh:43-93).  prop_table = 0: the built-in
// corium pairs (:45-46, :72-73).  prop_table = 1: table |p_type| of the
// property tables, whose h and T entries start at tab[index] and
// tab[SPH_TABLE_SIZE + index]; a slot without a table of two entries
// leaves the value as it was (the step refuses to run when a record the
// projection reaches has none).
template <class Real>
__device__ Real prop_lookup(const DevParams &P, const Real *tab, int p_type, Real x, Real keep, bool to_h) {
    if (!P.prop_table) {
        const Real H[5] = {(Real)-554932, (Real)215789, (Real)757894, (Real)905263, (Real)1268421};
        const Real T[5] = {(Real)280, (Real)1537, (Real)2300, (Real)2450, (Real)2650};
        return to_h ? interp2_rn<Real>(T, H, 5, x) : interp2_rn<Real>(H, T, 5, x);
    }
    const int t = p_type < 0 ? -p_type : p_type;
    if (t >= SPH_TABLE_SLOTS) return keep;
    const int n = P.tab_size[t];
    if (n < 2) return keep;
    const Real *h = tab + P.tab_index[t];
    const Real *T = tab + SPH_TABLE_SIZE + P.tab_index[t];
    return to_h ? interp2_rn<Real>(T, h, n, x) : interp2_rn<Real>(h, T, n, x);
}

// KERNEL_clc_TemptoEnthalpy (functions_ENERGY.cuh:3-12; its launch before
// the time loop, ISPH_Calc.cuh:480-482, is commented out there) and
// KERNEL_clc_EnthalpytoTemp (:15-25): every record but i_type 3
template <class Real>
__global__ void k_energy_convert(DevParams P, const int4 *ty, Real *temp, Real *enth, Real *enth0, const Real *tab,
                                 int to_h, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int4 t = ty[i];
    if (t.x == 3) return;
    if (to_h) {
        const Real v = prop_lookup<Real>(P, tab, t.w, temp[i], enth[i], true);
        enth[i] = v;
        enth0[i] = v;
    } else {
        temp[i] = prop_lookup<Real>(P, tab, t.w, enth[i], temp[i], false);
    }
}

template <class Real>
int energy_convert(Ctx<Real> &c, int to_h) {
    const int n = c.n;
    k_energy_convert<Real><<<grid_for(n, 256), 256, 0, c.stream>>>(c.dp, c.ty, c.A.temp, c.A.enth, c.enth0, c.tab,
                                                                  to_h, n);
    ++c.launches;
    SPH_CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}

// ---------------------------------------------------------------------------
// KERNEL_clc_projection, functions_TIME_ISPH.cuh:2-112 (predictor)
// ---------------------------------------------------------------------------
template <class Real>
__global__ void k_projection(DevParams P, const int4 *ty, typename V4<Real>::type *u,
                             typename V4<Real>::type *u0, const typename V4<Real>::type *ft,
                             const typename V4<Real>::type *fm, Real *rho_ref, const typename V2<Real>::type *mr,
                             Real *temp, Real *temp0, Real *concn, Real *concn0, const Real *dconcn,
                             const Real *enth, Real *enth0, const Real *tab, Real tdt, const StepClock *clk,
                             int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float ttime = clk->time;
    const int4 t = ty[i];
    if (t.x >= 3 || t.w >= 1000) return;
    auto ui = u[i];
    if (t.w == 9) {
        const Real bv = (Real)(float)P.boundary_velocity;
        ui.x = bv; ui.y = 0; ui.z = 0;
        u0[i] = mk4<Real>(bv, 0, 0, 1);
    } else {
        u0[i] = mk4<Real>(ui.x, ui.y, ui.z, 1);
        if (t.w > 0) {
            const Real on = (t.y == 0 || t.z == 1) ? (Real)1 : (Real)0;
            const auto f = ft[i];
            const auto m = fm[i];
            ui.x = ui.x + (f.x * on + m.x) * tdt;
            ui.y = ui.y + (f.y * on + m.y) * tdt;
            ui.z = ui.z + (f.z * on) * tdt;
        }
    }
    u[i] = ui;
    if (ttime == 0) rho_ref[i] = mr[i].y;
    if (P.con_solve == 1) {   // functions_TIME_ISPH.cuh:89-101
        if (P.enthalpy_eqn) {
            const Real h = enth[i];
            enth0[i] = h;
            temp[i] = prop_lookup<Real>(P, tab, t.w, h, temp[i], false);
        } else {
            temp0[i] = temp[i];
        }
    }
    if (P.concn_solve == 1) {
        const Real cc = concn[i];
        concn0[i] = cc;
        concn[i] = cc + dconcn[i] * tdt;
    }
}

// ---------------------------------------------------------------------------
// KERNEL_periodic_boundary3D (functions_BC.cuh:1015-1154) and
// KERNEL_donothing_buffer3D (functions_BC.cuh:673-761): copy u, p, T from the
// precomputed partner (zero when the reference finds none).  Gather first,
// then scatter, so every buffer particle reads the pre-pass state.
// ---------------------------------------------------------------------------
template <class Real>
__global__ void k_partner_gather(const int *rows, const int *partner, int nrows,
                                 const typename V4<Real>::type *u, const Real *p, const Real *temp,
                                 typename V4<Real>::type *ou, Real *op, Real *ot) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nrows) return;
    const int i = rows[k], j = partner[k];
    auto ui = u[i];
    if (j >= 0) {
        const auto uj = u[j];
        ui.x = uj.x; ui.y = uj.y; ui.z = uj.z;
        op[k] = p[j]; ot[k] = temp[j];
    } else {
        ui.x = 0; ui.y = 0; ui.z = 0;
        op[k] = 0; ot[k] = 0;
    }
    ou[k] = ui;
}

template <class Real>
__global__ void k_partner_scatter(const int *rows, int nrows, const typename V4<Real>::type *ou, const Real *op,
                                  const Real *ot, typename V4<Real>::type *u, Real *p, Real *temp) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nrows) return;
    const int i = rows[k];
    u[i] = ou[k]; p[i] = op[k]; temp[i] = ot[k];
}

// ---------------------------------------------------------------------------
// Open-boundary passes the reference ships commented out (gather halves; the
// scatter is k_partner_scatter, so every row reads the pre-pass state).
// KERNEL_open_boundary_extrapolation_buffer3D, functions_BC.cuh:763-855:
// Shepard average of the fluid around the mirror node (2 L3 - x, y, z) and
// zero pressure, when the average has weight 1e-6 or more.
// ---------------------------------------------------------------------------
template <class Real>
__global__ void k_extrap_gather(DevParams P, SoA<Real> s, const int *rows, const int *off, const int *nbr, int nrows,
                                const typename V4<Real>::type *u, const Real *p, const Real *temp,
                                typename V4<Real>::type *ou, Real *op, Real *ot) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nrows) return;
    const int i = rows[k];
    const auto xi = s.pr[i];
    const Real hi = xi.w;
    const Real tA = calc_tmpA<Real>(P, hi);
    const Real xg = (Real)(2.0 * P.l3 - (double)xi.x);
    Real tp = 0, tx = 0, ty = 0, tz = 0, tf = 0;
    for (int e = off[k]; e < off[k + 1]; ++e) {
        const int j = nbr[e];
        const auto xj = s.pr[j];
        const Real dx = xg - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
        const Real tdist = sqrt(dx * dx + dy * dy + dz * dz) - (Real)1e-20;
        const auto mj = s.mr[j];
        const Real vw = mj.x / mj.y * calc_wij<Real>(P, tA, hi, tdist);
        const auto uj = u[j];
        tp += vw * p[j]; tx += vw * uj.x; ty += vw * uj.y; tz += vw * uj.z; tf += vw;
    }
    auto ui = u[i];
    Real pi = p[i];
    if (tf >= (Real)1e-6) {
        ui.x = tx / tf; ui.y = ty / tf; ui.z = tz / tf;
        pi = 0;
    }
    ou[k] = ui; op[k] = pi; ot[k] = temp[i];
}

// KERNEL_inout_boundary3D, functions_BC.cuh:1274-1433: rows [0, nside) copy
// their periodic partner (zero without one); the outlet rows after them take
// 2 (interface value) - (own value) for u and p, the interface value being
// the Shepard average at (L3, y, z) with the pair-averaged h.
template <class Real>
__global__ void k_inout_gather(DevParams P, SoA<Real> s, const int *rows, const int *aux, int nside, const int *off,
                               const int *nbr, int nrows, const typename V4<Real>::type *u, const Real *p,
                               const Real *temp, typename V4<Real>::type *ou, Real *op, Real *ot) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nrows) return;
    const int i = rows[k];
    auto ui = u[i];
    if (k < nside) {
        const int j = aux[k];
        if (j >= 0) {
            const auto uj = u[j];
            ui.x = uj.x; ui.y = uj.y; ui.z = uj.z;
            op[k] = p[j]; ot[k] = temp[j];
        } else {
            ui.x = 0; ui.y = 0; ui.z = 0;
            op[k] = 0; ot[k] = 0;
        }
        ou[k] = ui;
        return;
    }
    const int q = k - nside;
    const auto xi = s.pr[i];
    const Real hi = xi.w;
    Real ax = 0, ay = 0, az = 0, ap = 0, tf = 0;
    for (int e = off[q]; e < off[q + 1]; ++e) {
        const int j = nbr[e];
        const auto xj = s.pr[j];
        const Real dx = (Real)(P.l3 - (double)xj.x), dy = xi.y - xj.y, dz = xi.z - xj.z;
        const Real tdist = sqrt(dx * dx + dy * dy + dz * dz) - (Real)1e-20;
        const Real hij = (Real)0.5 * (hi + xj.w);
        const Real tA = calc_tmpA<Real>(P, hij);
        const auto mj = s.mr[j];
        const Real vw = mj.x / mj.y * calc_wij<Real>(P, tA, hij, tdist);
        const auto uj = u[j];
        ax += uj.x * vw; ay += uj.y * vw; az += uj.z * vw; ap += p[j] * vw; tf += vw;
    }
    ui.x = -ui.x + (Real)2 * ax / tf;
    ui.y = -ui.y + (Real)2 * ay / tf;
    ui.z = -ui.z + (Real)2 * az / tf;
    ou[k] = ui;
    op[k] = -p[i] + (Real)2 * ap / tf;
    ot[k] = temp[i];
}

// KERNEL_Recycling3D, functions_BC.cuh:1857-1941: inlet ux from the log law
// of the probe's friction velocity (its neighbour search there finds a value
// that it does not use)
template <class Real>
__global__ void k_recycle(DevParams P, SoA<Real> s, const int *rows, int nrows, const float *us_update,
                          typename V4<Real>::type *u) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nrows) return;
    const int i = rows[k];
    u[i].x = (Real)((double)*us_update / 0.4 * log((double)s.pr[i].z / P.most_z0));
}

// ---------------------------------------------------------------------------
// KERNEL_freeslip_boundary3D, functions_BC.cuh:1156-1271
// ---------------------------------------------------------------------------
template <class Real>
__global__ void __launch_bounds__(128) k_freeslip(DevParams P, SoA<Real> s, LIST_ARGS,
                                                  const typename V4<Real>::type *__restrict__ u,
                                                  const Real *__restrict__ p, const Real *__restrict__ temp,
                                                  typename V4<Real>::type *__restrict__ ou,
                                                  Real *__restrict__ op, Real *__restrict__ ot, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int4 ti = s.ty[i];
    if (ti.w != -1 || ti.x >= 3) return;
    const float4 fi = s.pf[i];
    const auto xi = s.pr[i];
    const Real hi = xi.w;
    const Real tA = calc_tmpA<Real>(P, hi);
    Real tux = 0, tuy = 0, tuz = 0, tp = 0, tt = 0, tf = 0;
    SELL_LOOP_BEGIN(i)
        if (!(s.jc[j] & JB_PT1)) continue;
        const float4 fj = s.pf[j];
        if (!within_hi(P, fi, fj)) continue;
        const auto xj = s.pr[j];
        const Real dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
        const Real tdist = sqrt(dx * dx + dy * dy + dz * dz) - (Real)1e-20;
        const auto mj = s.mr[j];
        const Real vw = mj.x / mj.y * calc_wij<Real>(P, tA, hi, tdist);
        const auto uj = u[j];
        tux += uj.x * vw; tuy += uj.y * vw; tuz += uj.z * vw; tp += p[j] * vw; tt += temp[j] * vw; tf += vw;
    SELL_LOOP_END
    auto uo = u[i];
    Real po = p[i], to = temp[i];
    if (tf > (Real)1e-5) { uo.x = tux / tf; uo.y = tuy / tf; uo.z = tuz / tf; po = tp / tf; to = tt / tf; }
    ou[i] = uo; op[i] = po; ot[i] = to;
}

template <class Real>
__global__ void k_copy_rows(const int *rows, int nrows, const typename V4<Real>::type *su, const Real *sp,
                            const Real *st, typename V4<Real>::type *u, Real *p, Real *temp) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nrows) return;
    const int i = rows[k];
    u[i] = su[i]; p[i] = sp[i]; temp[i] = st[i];
}

// ---------------------------------------------------------------------------
// KERNEL_pressureforce3D, functions_PPE.cuh:482-647 (h_ij = (h_i+h_j)/2), in
// two parts.  The pair term is -2 m_j (p_i rho_j + p_j rho_i) /
// ((rho_i rho_j)(rho_i + rho_j)) dW(r, h_ij) / r x_ij; everything but the
// pressures is fixed while particles do not move, so k_pforce_cache stores
// g_ij = -2 m_j / ((rho_i rho_j)(rho_i + rho_j)) dW / r x_ij and rho_j per
// pair (one Real4, zero for markers and with the gradient correction's
// dW = 0) once per neighbour build, and k_pressure_force_cached sums
// (p_i rho_j + p_j rho_i) g_ij: one Real4 and the p_j gathers per pair
// instead of ~50 flops.  Same sums up to the grouping of the products.
// With pressure_force_form 1 the pair term is the reference's commented-out
// difference form -m_j (p_j - p_i) / (rho_i rho_j) dW / r x_ij: the cache
// then holds g_ij = -m_j / (rho_i^2 rho_j) dW / r x_ij and -rho_i, so the same
// cached sum (p_i g.w + p_j rho_i) g_ij gives it.
// ---------------------------------------------------------------------------
template <class Real>
__global__ void __launch_bounds__(128) k_pforce_cache(DevParams P, SoA<Real> s, LIST_ARGS,
                                                      typename V4<Real>::type *__restrict__ pw, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int4 ti = s.ty[i];
    if (ti.x > 2 || ti.w >= 1000 || ti.w <= 0 || ti.y != 0) return;
    const auto xi = s.pr[i];
    const Real hi = xi.w, rhoi = s.mr[i].y;
    const bool kgc = P.kgc_solve == 1;
    const Real tA_ii = calc_tmpA<Real>(P, hi);
    SELL_LOOP_BEGIN(i)
        const long long e = sbase_ + 32LL * k_;
        const auto mj = s.mr[j];
        Real gx = 0, gy = 0, gz = 0;
        if (s.jc[j] & JB_LT1000) {
            const auto xj = s.pr[j];
            const Real dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
            const Real tdist = sqrt(dx * dx + dy * dy + dz * dz) - (Real)1e-20;
            const Real hij = (Real)0.5 * (hi + xj.w);
            const Real tA = (xj.w == hi) ? tA_ii : calc_tmpA<Real>(P, hij);
            Real dw = calc_dwij<Real>(P, tA, hij, tdist);
            if (kgc) dw = 0;
            // difference form: (p_i (-rho_i) + p_j rho_i) g with g = -m_j / (rho_i^2 rho_j) dW / r x_ij
            const Real c = P.pforce_form == 1 ? -mj.x / ((rhoi * mj.y) * rhoi) * dw / tdist
                                              : (Real)-2 * mj.x / ((rhoi * mj.y) * (rhoi + mj.y)) * dw / tdist;
            gx = c * dx; gy = c * dy; gz = c * dz;
        }
        pw[e] = mk4<Real>(gx, gy, gz, P.pforce_form == 1 ? -rhoi : mj.y);
    SELL_LOOP_END
}

template <class Real>
__global__ void __launch_bounds__(128) k_pressure_force_cached(DevParams P, const int4 *__restrict__ ty,
                                                               const typename V2<Real>::type *__restrict__ mr, LIST_ARGS,
                                                               const typename V4<Real>::type *__restrict__ pw,
                                                               const Real *__restrict__ p, const Real *__restrict__ pres0,
                                                               typename V4<Real>::type *__restrict__ fp, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int4 ti = ty[i];
    if (ti.x > 2 || ti.w >= 1000 || ti.w <= 0 || ti.y != 0) return;
    const Real rhoi = mr[i].y, pi = p[i] - pres0[i];
    Real tx = 0, ty_ = 0, tz = 0;
    if (P.fp_solve) {
        SELL_LOOP_BEGIN(i)
            const auto g = ld_stream(&pw[sbase_ + 32LL * k_]);
            const Real pj = p[j] - pres0[j];
            const Real c = pi * g.w + pj * rhoi;
            tx += c * g.x; ty_ += c * g.y; tz += c * g.z;
        SELL_LOOP_END
    }
    fp[i] = mk4<Real>(tx, ty_, tz, 0);
}

// The pressure force evaluated in full every step: used when the device has
// no room for the cached pair factors.
template <class Real>
__global__ void __launch_bounds__(128) k_pressure_force(DevParams P, SoA<Real> s, LIST_ARGS, const Real *__restrict__ p,
                                                        const Real *__restrict__ pres0,
                                                        typename V4<Real>::type *__restrict__ fp, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int4 ti = s.ty[i];
    if (ti.x > 2 || ti.w >= 1000 || ti.w <= 0 || ti.y != 0) return;
    const auto xi = s.pr[i];
    const auto mri = s.mr[i];
    const Real hi = xi.w, rhoi = mri.y, pi = p[i] - pres0[i];
    const bool kgc = P.kgc_solve == 1;
    const bool uniform_hint = true;
    Real tA_ii = calc_tmpA<Real>(P, hi);
    Real tx = 0, ty_ = 0, tz = 0;
    if (P.fp_solve) {
        SELL_LOOP_BEGIN(i)
            if (!(s.jc[j] & JB_LT1000)) continue;
            const auto xj = s.pr[j];
            const Real dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
            const Real tdist = sqrt(dx * dx + dy * dy + dz * dz) - (Real)1e-20;
            const Real hij = (Real)0.5 * (hi + xj.w);
            const Real tA = (uniform_hint && xj.w == hi) ? tA_ii : calc_tmpA<Real>(P, hij);
            Real dw = calc_dwij<Real>(P, tA, hij, tdist);
            if (kgc) dw = 0;
            const auto mj = s.mr[j];
            const Real pj = p[j] - pres0[j];
            const Real Cp = P.pforce_form == 1 ? -mj.x * (pj - pi) / (rhoi * mj.y)
                                               : (Real)-2 * mj.x * (pi * mj.y + pj * rhoi) / ((rhoi * mj.y) * (rhoi + mj.y));
            const Real f = Cp * dw / tdist;
            tx += f * dx; ty_ += f * dy; tz += f * dz;
        SELL_LOOP_END
    }
    fp[i] = mk4<Real>(tx, ty_, tz, 0);
}

// ---------------------------------------------------------------------------
// IBM_force_interpolation3D (functions_IBM.cuh:342-490) and
// IBM_spreading_interpolation3D (functions_IBM.cuh:492-613)
// ---------------------------------------------------------------------------
__device__ double wall_profile(const DevParams &P, double z) {
    const int NP = P.n_profile;
    const double *Z = P.profile_z, *U = P.profile_u;
    if (z <= Z[0]) return U[0] + (z - Z[0]) * ((U[1] - U[0]) / ((Z[1] - Z[0]) + 1e-300));
    if (z >= Z[NP - 1]) return U[NP - 2] + (z - Z[NP - 2]) * ((U[NP - 1] - U[NP - 2]) / ((Z[NP - 1] - Z[NP - 2]) + 1e-300));
    int lo = 0, hi = NP - 1;
    while (hi - lo > 1) { const int mid = (lo + hi) >> 1; if (z < Z[mid]) hi = mid; else lo = mid; }
    const double t = (z - Z[lo]) / (Z[hi] - Z[lo] + 1e-300);
    return U[lo] + t * (U[hi] - U[lo]);
}

template <class Real>
__global__ void k_ibm_force(DevParams P, SoA<Real> s, const int *rows, const int *off, const int *nb, int nrows,
                            const typename V4<Real>::type *u, const typename V4<Real>::type *nrm,
                            typename V4<Real>::type *fb, Real t_dt) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nrows) return;
    const int i = rows[k];
    const auto xi = s.pr[i];
    const Real th = (Real)(P.ibm_length * (double)xi.w);
    const Real tA = calc_tmpA<Real>(P, th);
    Real tux = 0, tuy = 0, tuz = 0, filt = 0;
    for (int e = off[k]; e < off[k + 1]; ++e) {
        const int j = nb[e];
        const auto xj = s.pr[j];
        const Real dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
        const Real tdist = sqrt(dx * dx + dy * dy + dz * dz) + (Real)1e-20;
        const auto mj = s.mr[j];
        const Real vw = mj.x / mj.y * calc_wij<Real>(P, tA, th, tdist);
        const auto uj = u[j];
        tux += uj.x * vw; tuy += uj.y * vw; tuz += uj.z * vw; filt += vw;
    }
    const Real ufx = tux / (filt + (Real)1e-10), ufy = tuy / (filt + (Real)1e-10), ufz = tuz / (filt + (Real)1e-10);
    const auto nv = nrm[i];
    Real nx = nv.x, ny = nv.y, nz = nv.z;
    const Real nmag = sqrt(nx * nx + ny * ny + nz * nz) + (Real)1e-20;
    nx /= nmag; ny /= nmag; nz /= nmag;
    const Real un = ufx * nx + ufy * ny + ufz * nz;
    const Real utx = ufx - un * nx, uty = ufy - un * ny, utz = ufz - un * nz;
    const Real Ubtx = (Real)(P.ibm_target_coeff * wall_profile(P, (double)xi.z));
    const Real cx = -un * nx + (Ubtx - utx), cy = -un * ny + (0 - uty), cz = -un * nz + (0 - utz);
    fb[i] = mk4<Real>((Real)(P.rho_air * (double)cx / (double)t_dt), (Real)(P.rho_air * (double)cy / (double)t_dt),
                      (Real)(P.rho_air * (double)cz / (double)t_dt), filt);
}

template <class Real>
__global__ void k_ibm_spread(DevParams P, SoA<Real> s, const int *rows, const int *off, const int *nb, int nrows,
                             const typename V4<Real>::type *fbm, typename V4<Real>::type *fb) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nrows) return;
    const int i = rows[k];
    const auto xi = s.pr[i];
    const Real th = (Real)(P.ibm_length * (double)xi.w);
    const Real tA = calc_tmpA<Real>(P, th);
    Real fx = 0, fy = 0, fz = 0, filt = 0;
    for (int e = off[k]; e < off[k + 1]; ++e) {
        const int j = nb[e];
        const auto xj = s.pr[j];
        const Real dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
        const Real tdist = sqrt(dx * dx + dy * dy + dz * dz) + (Real)1e-20;
        const auto mj = s.mr[j];
        const Real vw = mj.x / mj.y * calc_wij<Real>(P, tA, th, tdist);
        const auto f = fbm[j];
        fx += f.x * vw; fy += f.y * vw; fz += f.z * vw; filt += vw;
    }
    if (filt < (Real)1e-12) fb[i] = mk4<Real>(0, 0, 0, 0);
    else fb[i] = mk4<Real>(fx / (filt + (Real)1e-10), fy / (filt + (Real)1e-10), fz / (filt + (Real)1e-10), filt);
}

template <class Real>
__global__ void k_zero_rows4(const int *rows, int nrows, typename V4<Real>::type *a) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nrows) a[rows[k]] = mk4<Real>(0, 0, 0, 0);
}

// ---------------------------------------------------------------------------
// KERNEL_time_update_projection (functions_TIME_ISPH.cuh:115-296) and
// IBM_corrector (functions_IBM.cuh:615-725): SP1 -> P1
// ---------------------------------------------------------------------------
template <class Real>
__global__ void k_time_update(Ctx<Real> c, Real tdt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    const int tcount = c.clk->count;
    const int4 t = c.ty[i];
    const VarSet<Real> &S = c.S;
    const VarSet<Real> &A = c.A;
    const DevParams &P = c.dp;
    if (t.w >= 1000) {   // IBM_corrector
        A.fb[i] = S.fb[i];
        A.p[i] = S.p[i];
        return;
    }
    if (t.x >= 3) return;
    auto us = S.u[i];
    auto ua = A.u[i];
    if (t.w == 9) {
        ua.x = us.x; ua.y = us.y; ua.z = us.z;
    } else {
        Real ux0, uy0, uz0, ax = 0, ay = 0, az = 0;
        const auto u0 = c.u0[i];
        if (t.w > 0) {
            ux0 = us.x; uy0 = us.y; uz0 = us.z;
            if (t.y == 1 || t.y == -1) { ux0 = u0.x; uy0 = u0.y; uz0 = u0.z; }
            const Real on = (t.y == 0) ? (Real)1 : (Real)0;
            const auto fp = c.fp[i];
            const auto fb = S.fb[i];
            const auto fm = S.fm[i];
            const Real rho = c.mr[i].y;
            ax = fp.x * on + fb.x / rho + fm.x;
            ay = fp.y * on + fb.y / rho + fm.y;
            az = fp.z * on + fb.z / rho;
        } else {
            ux0 = u0.x; uy0 = u0.y; uz0 = u0.z;
        }
        Real uxc = ux0 + ax * tdt, uyc = uy0 + ay * tdt, uzc = uz0 + az * tdt;
        const Real ul = (Real)P.u_limit;
        if (uxc * uxc + uyc * uyc + uzc * uzc >= ul * ul) { uxc = ux0; uyc = uy0; uzc = uz0; }
        ua.x = uxc; ua.y = uyc; ua.z = uzc;
    }
    ua.w = us.w;   // vis_t
    A.u[i] = ua;
    Real temp = S.temp[i];
    if (P.con_solve == 1) {   // functions_TIME_ISPH.cuh:203-215
        if (P.enthalpy_eqn) A.enth[i] = c.enth0[i] + c.denth[i] * tdt;   // the temperature stays the projection's
        else temp = c.temp0[i] + c.dtemp[i] * tdt * (Real)(t.y == 0);
    }
    if (t.w == 0) {
        const double tt = (double)(tdt * (Real)tcount);
        if (tt >= P.t_start && tt < P.t_con_t) temp = (Real)(P.t_ini + tt * (P.t_con - P.t_ini) / (P.t_con_t - P.t_start));
        else if (tt < P.t_start) temp = (Real)P.t_ini;
        else temp = (Real)P.t_con;
    }
    A.temp[i] = temp;
    if (P.con_solve != 1) A.enth[i] = S.enth[i];
    Real concn = S.concn[i];
    if (P.concn_solve == 1) {
        concn = c.concn0[i] + c.dconcn[i] * tdt;
        if (concn < (Real)0) concn = 0;
    }
    if (c.source[i] == 1) concn += (Real)0.5 * tdt;
    A.concn[i] = concn;
    A.p[i] = S.p[i]; A.flt[i] = S.flt[i]; A.kt[i] = S.kt[i]; A.et[i] = S.et[i];
    A.fb[i] = S.fb[i]; A.fm[i] = S.fm[i]; A.fl[i] = S.fl[i];
    c.rho_ref_A[i] = c.rho_ref_S[i];
}

// ---------------------------------------------------------------------------
// diagnostics, kernel_copy_max (functions_OUTPUT.cuh:19-33) + max reduction
// ---------------------------------------------------------------------------
template <class Real>
__global__ void k_diag(Ctx<Real> c, unsigned int *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float mu = 0, mr = 0, mf = 0;
    if (i < c.n) {
        const int4 t = c.ty[i];
        if (!(t.w == 0 || t.x >= 2)) {
            const auto u = c.A.u[i];
            mu = (float)sqrt(u.x * u.x + u.y * u.y + u.z * u.z);
            const Real rr = c.rho_ref_S[i];
            mr = (float)((c.mr[i].y - rr) / rr * (Real)100.0);
            mf = (float)c.ft[i].w;
        }
    }
    // order-preserving float -> unsigned map for atomicMax
    auto key = [](float f) -> unsigned int {
        unsigned int b = __float_as_uint(f);
        return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
    };
    for (int o = 16; o > 0; o >>= 1) {
        mu = fmaxf(mu, __shfl_xor_sync(0xffffffffu, mu, o));
        mr = fmaxf(mr, __shfl_xor_sync(0xffffffffu, mr, o));
        mf = fmaxf(mf, __shfl_xor_sync(0xffffffffu, mf, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&out[0], key(mu));
        atomicMax(&out[1], key(mr));
        atomicMax(&out[2], key(mf));
    }
}

// ---------------------------------------------------------------------------
// host drivers
// ---------------------------------------------------------------------------
template <class Real>
static SoA<Real> soa(Ctx<Real> &c) {
    SoA<Real> s;
    s.pf = c.pf; s.pr = c.pr; s.mr = c.mr; s.ty = c.ty; s.jc = c.jc;
    return s;
}

#define LIST(c) (c).slice_off, (c).ncnt, (c).nbr

// whether `bytes` more of device memory leave a tenth of the device free
// (the per-pair caches of the prep pass and the pressure force are an
// optimisation: without room the passes evaluate their pair terms in full)
static bool cache_fits(size_t bytes) {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return bytes + tot / 10 <= fr;
}

template <class Real>
int gradient_correction(Ctx<Real> &c) {
    k_grad_corr<Real><<<grid_for(c.n, 128), 128, 0, c.stream>>>(c.dp, soa(c), LIST(c), c.g6, c.n);
    ++c.launches;
    SPH_CUDA_TRY(cudaGetLastError());
    c.gc_valid = true;
    c.prep_valid = false;   // the strain weights hold G_i
    return SPH_OK;
}

// scratch for the gather/scatter passes (n-long u, p and temp buffers)
template <class Real>
static int scratch_rows(Ctx<Real> &c, typename V4<Real>::type *&ou, Real *&op, Real *&ot) {
    if (!c.sc_u) {
        SPH_TRY(c.alloc(c.sc_u, (size_t)c.n));
        SPH_TRY(c.alloc(c.sc_p, (size_t)c.n));
        SPH_TRY(c.alloc(c.sc_t, (size_t)c.n));
    }
    ou = c.sc_u;
    op = c.sc_p;
    ot = c.sc_t;
    return SPH_OK;
}

template <class Real>
int neumann_pass(Ctx<Real> &c, VarSet<Real> &V) {
    const SideLists &L = c.L;
    if (L.n_nm == 0) return SPH_OK;
    typename V4<Real>::type *ou; Real *op, *ot;
    SPH_TRY(scratch_rows(c, ou, op, ot));
    k_neumann_gather<Real><<<grid_for(32LL * L.n_nm, 128), 128, 0, c.stream>>>(L.nm_rows, L.nm_off, L.nm_nbr, L.nm_ghost,
                                                                        c.nm_w, c.nm_gw, L.n_nm, V.p, V.u, c.ty, op, ou);
    k_neumann_scatter<Real><<<grid_for(L.n_nm, 128), 128, 0, c.stream>>>(L.nm_rows, L.n_nm, op, ou, V.p, V.u);
    c.launches += 2;
    SPH_CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}

template <class Real>
static int partner_pass(Ctx<Real> &c, VarSet<Real> &V, const int *rows, const int *partner, int nrows) {
    if (nrows == 0) return SPH_OK;
    typename V4<Real>::type *ou; Real *op, *ot;
    SPH_TRY(scratch_rows(c, ou, op, ot));
    k_partner_gather<Real><<<grid_for(nrows, 128), 128, 0, c.stream>>>(rows, partner, nrows, V.u, V.p, V.temp, ou, op, ot);
    k_partner_scatter<Real><<<grid_for(nrows, 128), 128, 0, c.stream>>>(rows, nrows, ou, op, ot, V.u, V.p, V.temp);
    c.launches += 2;
    SPH_CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}

// the pass at the outlet-buffer call sites (ISPH_Calc.cuh:151, 208)
template <class Real>
int outlet_pass(Ctx<Real> &c, VarSet<Real> &V) {
    const SideLists &L = c.L;
    if (c.dp.outlet_bc == 0) return partner_pass(c, V, L.out_rows, L.out_partner, L.n_out);
    const int nrows = c.dp.outlet_bc == 1 ? L.n_xo : L.n_io;
    if (nrows == 0) return SPH_OK;
    typename V4<Real>::type *ou; Real *op, *ot;
    SPH_TRY(scratch_rows(c, ou, op, ot));
    if (c.dp.outlet_bc == 1) {
        k_extrap_gather<Real><<<grid_for(nrows, 128), 128, 0, c.stream>>>(c.dp, soa(c), L.xo_rows, L.xo_off, L.xo_nbr, nrows,
                                                                           V.u, V.p, V.temp, ou, op, ot);
        k_partner_scatter<Real><<<grid_for(nrows, 128), 128, 0, c.stream>>>(L.xo_rows, nrows, ou, op, ot, V.u, V.p, V.temp);
    } else {
        k_inout_gather<Real><<<grid_for(nrows, 128), 128, 0, c.stream>>>(c.dp, soa(c), L.io_rows, L.io_aux, L.n_ios, L.io_off,
                                                                          L.io_nbr, nrows, V.u, V.p, V.temp, ou, op, ot);
        k_partner_scatter<Real><<<grid_for(nrows, 128), 128, 0, c.stream>>>(L.io_rows, nrows, ou, op, ot, V.u, V.p, V.temp);
    }
    c.launches += 2;
    SPH_CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}

// the periodic-y copy (functions_BC.cuh:1015-1154), then the ghosts of a
// periodic box, which copy the record at their wrapped position
template <class Real>
int periodic_pass(Ctx<Real> &c, VarSet<Real> &V) {
    SPH_TRY(partner_pass(c, V, c.L.per_rows, c.L.per_partner, c.L.n_per));
    return partner_pass(c, V, c.L.gh_rows, c.L.gh_partner, c.L.n_gh);
}

template <class Real>
int freeslip_pass(Ctx<Real> &c, VarSet<Real> &V) {
    if (c.L.n_fs == 0) return SPH_OK;
    typename V4<Real>::type *ou; Real *op, *ot;
    SPH_TRY(scratch_rows(c, ou, op, ot));
    k_freeslip<Real><<<grid_for(c.n, 128), 128, 0, c.stream>>>(c.dp, soa(c), LIST(c), V.u, V.p, V.temp, ou, op, ot, c.n);
    k_copy_rows<Real><<<grid_for(c.L.n_fs, 128), 128, 0, c.stream>>>(c.L.fs_rows, c.L.n_fs, ou, op, ot, V.u, V.p, V.temp);
    c.launches += 2;
    SPH_CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}

// a step whose projection reads the property tables (prop_table = 1 with
// the enthalpy form, time_type 1) needs a table of two entries for every
// |p_type| among the records it reaches
template <class Real>
static int check_tables(const Ctx<Real> &c) {
    if (!(c.dp.prop_table && c.dp.con_solve == 1 && c.dp.enthalpy_eqn && c.dp.time_type == 1)) return SPH_OK;
    if (!c.tab_set) {
        set_error("prop_table = 1 with the enthalpy form needs sph_set_prop_tables");
        return SPH_ERR_STATE;
    }
    if (c.ptype_wide) {
        set_error("prop_table = 1: a record has |p_type| >= SPH_TABLE_SLOTS, which no table serves");
        return SPH_ERR_BAD_ARG;
    }
    for (int t = 0; t < SPH_TABLE_SLOTS; ++t)
        if (((c.ptype_slots >> t) & 1u) && c.tab_size[t] < 2) {
            set_error("prop_table = 1: a record's |p_type| has no property table of at least two entries");
            return SPH_ERR_BAD_ARG;
        }
    return SPH_OK;
}

template <class Real>
int phase_interaction(Ctx<Real> &c) {
    SPH_TRY(check_tables(c));
    cudaStream_t st = c.stream;
    const int n = c.n;
    const int tc = c.count;
    const Real tdt = (Real)c.dp.dt;
    if (!c.clk) SPH_TRY(c.alloc(c.clk, 1));
    if (!c.clk_synced) {
        k_set_clock<<<1, 1, 0, st>>>(c.clk, c.count, c.time);
        ++c.launches;
        c.clk_synced = true;
    }
    k_begin_step<Real><<<grid_for(n, 256), 256, 0, st>>>(c);
    ++c.launches;
    if (tc == 0) {
        k_ib_normals<Real><<<grid_for(n, 256), 256, 0, st>>>(c.dp, c.pr, c.ty, c.nrm, c.ib_boxes, c.n_ib_boxes, n);
        ++c.launches;
    }
    if (!c.gc_valid || c.prm.recompute_gc) SPH_TRY(gradient_correction(c));
    // prep / LES
    if (!c.vis_stage) SPH_TRY(c.alloc(c.vis_stage, n));
    Real *vis_stage = c.vis_stage;   // LES viscosity staged until every row has read the old one
    if (!c.prep_valid) {
        const long long nnzp = c.nnz_padded;
        if (c.prep_cap < nnzp) {
            c.release(c.prep_w);
            c.prep_cap = 0;
        }
        c.release(c.prep_row);
        const size_t need = (c.prep_w ? 0 : sizeof(Real) * 3 * (size_t)nnzp) + sizeof(Real) * 2 * (size_t)n;
        if (!c.prm.recompute_pairs && cache_fits(need)) {
            if (!c.prep_w) {
                SPH_TRY(c.alloc(c.prep_w, (size_t)(3 * nnzp)));
                c.prep_cap = nnzp;
            }
            SPH_TRY(c.alloc(c.prep_row, 2 * (size_t)n));
            SPH_CUDA_TRY(cudaMemsetAsync(c.prep_row, 0, sizeof(Real) * 2 * (size_t)n, st));
            k_prep_cache<Real><<<grid_for(n, 128), 128, 0, st>>>(c.dp, soa(c), LIST(c), c.g6, c.prep_row, c.prep_w, nnzp, n);
            ++c.launches;
            c.prep_valid = true;
        }
    }
    if (c.prep_valid)
        k_prep_cached<Real><<<grid_for(n, c.pair_block), c.pair_block, 0, st>>>(c.dp, c.ty, LIST(c), c.prep_row, c.prep_w, c.nnz_padded,
                                                              c.S.u, c.mr, c.pr, c.S.flt, vis_stage, c.S.kt, c.S.et, c.SR,
                                                              c.rho_ref_S, c.clk, tdt, n);
    else
        k_prep<Real><<<grid_for(n, c.pair_block), c.pair_block, 0, st>>>(c.dp, soa(c), LIST(c), c.g6, c.S.u, c.S.flt, vis_stage, c.S.kt,
                                                       c.S.et, c.SR, c.rho_ref_S, c.clk, tdt, n);
    ++c.launches;
    if (c.dp.fv_solve != 0 && (c.dp.turb == 4 || c.dp.turb == 5)) {
        k_merge_vis<Real><<<grid_for(n, 256), 256, 0, st>>>(c.S.u, vis_stage, c.ty, n);
        ++c.launches;
    }
    if (c.dp.noslip == 1) {
        k_boundary<Real><<<grid_for(n, c.pair_block), c.pair_block, 0, st>>>(c.dp, soa(c), LIST(c), c.S.u, n);
        ++c.launches;
    }
    if (c.L.n_most > 0) {
        k_most<Real><<<grid_for(c.L.n_most, 128), 128, 0, st>>>(c.dp, soa(c), c.L.most_rows, c.L.most_off, c.L.most_tgt,
                                                               c.L.n_most, c.S.u, c.S.temp, c.S.fm, c.S.fl, c.dtemp, c.us_update, c.clk, (float)tdt);
        ++c.launches;
    }
    if (tc == 0) SPH_TRY(neumann_pass(c, c.S));
    const Scalars sc{c.S.temp, c.S.concn, c.dtemp, c.dconcn, c.denth};
    const bool th = c.dp.con_solve != 0 || c.dp.concn_solve != 0 || c.dp.boussinesq != 0;
    const dim3 ga = grid_for(n, c.pair_block);
    if (th) {
        if (c.dp.fv_solve == 2) k_advection<Real, 2, 1><<<ga, c.pair_block, 0, st>>>(c.dp, soa(c), LIST(c), c.S.u, c.eli, c.ft, sc, n);
        else if (c.dp.fv_solve == 1) k_advection<Real, 1, 1><<<ga, c.pair_block, 0, st>>>(c.dp, soa(c), LIST(c), c.S.u, c.eli, c.ft, sc, n);
        else k_advection<Real, 0, 1><<<ga, c.pair_block, 0, st>>>(c.dp, soa(c), LIST(c), c.S.u, c.eli, c.ft, sc, n);
    } else {
        if (c.dp.fv_solve == 2) k_advection<Real, 2, 0><<<ga, c.pair_block, 0, st>>>(c.dp, soa(c), LIST(c), c.S.u, c.eli, c.ft, sc, n);
        else if (c.dp.fv_solve == 1) k_advection<Real, 1, 0><<<ga, c.pair_block, 0, st>>>(c.dp, soa(c), LIST(c), c.S.u, c.eli, c.ft, sc, n);
        else k_advection<Real, 0, 0><<<ga, c.pair_block, 0, st>>>(c.dp, soa(c), LIST(c), c.S.u, c.eli, c.ft, sc, n);
    }
    ++c.launches;
    if (c.dp.time_type == 1) {
        k_projection<Real><<<grid_for(n, 256), 256, 0, st>>>(c.dp, c.ty, c.S.u, c.u0, c.ft, c.S.fm, c.rho_ref_S, c.mr,
                                                             c.S.temp, c.temp0, c.S.concn, c.concn0, c.dconcn,
                                                             c.S.enth, c.enth0, c.tab, tdt, c.clk, n);
        ++c.launches;
    }
    SPH_TRY(periodic_pass(c, c.S));
    SPH_TRY(freeslip_pass(c, c.S));
    SPH_CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}

template <class Real>
int phase_time_update(Ctx<Real> &c) {
    cudaStream_t st = c.stream;
    const int n = c.n;
    const Real tdt = (Real)c.dp.dt;
    if (!c.pforce_valid) {
        const long long nnzp = c.nnz_padded;
        if (c.pforce_cap < nnzp) {
            c.release(c.pforce_w);
            c.pforce_cap = 0;
        }
        if (!c.prm.recompute_pairs && (c.pforce_w || cache_fits(sizeof(typename V4<Real>::type) * (size_t)nnzp))) {
            if (!c.pforce_w) {
                SPH_TRY(c.alloc(c.pforce_w, (size_t)nnzp));
                c.pforce_cap = nnzp;
            }
            k_pforce_cache<Real><<<grid_for(n, 128), 128, 0, st>>>(c.dp, soa(c), LIST(c), c.pforce_w, n);
            ++c.launches;
            c.pforce_valid = true;
        }
    }
    if (c.pforce_valid)
        k_pressure_force_cached<Real><<<grid_for(n, c.pair_block), c.pair_block, 0, st>>>(c.dp, c.ty, c.mr, LIST(c), c.pforce_w, c.S.p,
                                                                        c.pres0, c.fp, n);
    else
        k_pressure_force<Real><<<grid_for(n, c.pair_block), c.pair_block, 0, st>>>(c.dp, soa(c), LIST(c), c.S.p, c.pres0, c.fp, n);
    ++c.launches;
    if (c.L.n_mk > 0) {
        k_ibm_force<Real><<<grid_for(c.L.n_mk, 128), 128, 0, st>>>(c.dp, soa(c), c.L.mk_rows, c.L.mk_off, c.L.mk_nbr,
                                                                  c.L.n_mk, c.S.u, c.nrm, c.S.fb, tdt);
        ++c.launches;
    }
    if (c.L.n_sp > 0) {
        k_ibm_spread<Real><<<grid_for(c.L.n_sp, 128), 128, 0, st>>>(c.dp, soa(c), c.L.sp_rows, c.L.sp_off, c.L.sp_nbr,
                                                                   c.L.n_sp, c.S.fb, c.S.fb);
        ++c.launches;
    }
    if (c.L.n_sp_zero > 0) {
        k_zero_rows4<Real><<<grid_for(c.L.n_sp_zero, 256), 256, 0, st>>>(c.L.sp_zero, c.L.n_sp_zero, c.S.fb);
        ++c.launches;
    }
    k_time_update<Real><<<grid_for(n, 256), 256, 0, st>>>(c, tdt);
    ++c.launches;
    SPH_TRY(neumann_pass(c, c.A));
    SPH_TRY(outlet_pass(c, c.A));
    SPH_TRY(periodic_pass(c, c.A));
    SPH_TRY(freeslip_pass(c, c.A));
    if (c.dp.inlet_recycling == 1 && c.L.n_rc > 0) {   // ISPH_Calc.cuh:215
        k_recycle<Real><<<grid_for(c.L.n_rc, 128), 128, 0, st>>>(c.dp, soa(c), c.L.rc_rows, c.L.n_rc, c.us_update, c.A.u);
        ++c.launches;
    }
    k_advance_clock<<<1, 1, 0, st>>>(c.clk, c.dp.dt);
    ++c.launches;
    SPH_CUDA_TRY(cudaGetLastError());
    if (c.capturing) return SPH_OK;   // a replayed step graph calls finish_step itself
    return finish_step(c);
}

// the host's side of the end of a step: its copy of the counter and time,
// then APR every freq_apr steps (vii[35] = 1: cell-based)
template <class Real>
int finish_step(Ctx<Real> &c) {
    c.time = c.time + c.dp.dt;
    c.count += 1;
    const int freq_apr = c.prm.vii[SPH_VII_FREQ_APR];
    if (c.prm.vii[SPH_VII_APR_SOLV] == 1 && freq_apr > 0 && c.count % freq_apr == 0)
        SPH_TRY(apr_pass(c, nullptr, nullptr, nullptr));
    return SPH_OK;
}

template <class Real>
int ctx_diagnostics(Ctx<Real> &c, float *umax, float *drho, float *fmax) {
    unsigned int *d = (unsigned int *)c.cell_fill;   // reused scratch
    SPH_CUDA_TRY(cudaMemsetAsync(d, 0, 3 * sizeof(unsigned int), c.stream));
    k_diag<Real><<<grid_for(c.n, 256), 256, 0, c.stream>>>(c, d);
    ++c.launches;
    unsigned int h[3];
    SPH_CUDA_TRY(cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, c.stream));
    SPH_CUDA_TRY(cudaStreamSynchronize(c.stream));
    auto val = [](unsigned int k) {
        unsigned int b = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
        float f;
        memcpy(&f, &b, 4);
        return f;
    };
    if (umax) *umax = val(h[0]);
    if (drho) *drho = val(h[1]);
    if (fmax) *fmax = val(h[2]);
    return SPH_OK;
}

#define INST(R)                                                          \
    template int gradient_correction<R>(Ctx<R> &);                       \
    template int neumann_pass<R>(Ctx<R> &, VarSet<R> &);                 \
    template int outlet_pass<R>(Ctx<R> &, VarSet<R> &);                  \
    template int finish_step<R>(Ctx<R> &);                               \
    template int periodic_pass<R>(Ctx<R> &, VarSet<R> &);                \
    template int freeslip_pass<R>(Ctx<R> &, VarSet<R> &);                \
    template int phase_interaction<R>(Ctx<R> &);                         \
    template int energy_convert<R>(Ctx<R> &, int);                       \
    template int phase_time_update<R>(Ctx<R> &);                         \
    template int ctx_diagnostics<R>(Ctx<R> &, float *, float *, float *);
INST(float)
INST(double)
#undef INST

}  // namespace sph
