// Pressure phase of the ISPH step (ISPH_Calc.cuh:137-154).
//
// The reference runs one in-place point-Jacobi sweep of KERNEL_PPE3D
// (functions_PPE.cuh:2-175) per step:
//     p_i = p0_i + (b_i + sum_j c_ij (p_j - p0_j)) / A_i,   A_i = sum_j c_ij
//     b_i = sum_j m_j/rho_j (u_j - u_i).G_i gradW_ij 2 rho_i rho_j/(rho_i+rho_j) / dt
//     c_ij = 2 m_j/rho_j (r_ij . G_i gradW_ij) / |r_ij|^2
// followed by the Neumann wall pressure and the outlet copy.  SPH_PPE_REF_SWEEP
// reproduces that sweep with Jacobi (race-free) semantics.  The converged
// modes solve the linear system whose fixed point that sweep iterates
// towards: fluid rows A_i p_i - sum c_ij p_j = b_i, Neumann rows
// p_w - sum w p = 0, outlet rows p_o - p_partner = 0, optionally one pinned
// fluid row p = 0 for domains without a Dirichlet row.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "ctx.cuh"

namespace sph {

// ---- device scalars of the Krylov solver -----------------------------------
enum {
    SC_RHO = 0, SC_ALPHA, SC_OMEGA, SC_BETA, SC_RR, SC_BB, SC_RV, SC_TS, SC_TT, SC_FLAG, SC_TOL2,
    SC_RHO_NEW, SC_ITN, SC_COUNT
};
enum { FLAG_RUN = 0, FLAG_CONVERGED = 1, FLAG_BREAKDOWN = 2 };

// block-sum of NV doubles; the last block to finish sums the per-block
// partials in block order (deterministic) and calls finish(sums) on thread 0
template <int NV, class F>
__device__ __forceinline__ void reduce_finish(double (&v)[NV], double *partials, unsigned int *counter, F finish) {
    __shared__ double sh[NV][32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        double x = v[q];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) sh[q][wid] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            double s = 0;
            for (int w = 0; w < nw; ++w) s += sh[q][w];
            partials[(size_t)q * gridDim.x + blockIdx.x] = s;
        }
        __threadfence();
        const unsigned int t = atomicAdd(counter, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double tot[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        double s = 0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) s += ((volatile double *)partials)[(size_t)q * gridDim.x + b];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) sh[q][wid] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            double s = 0;
            for (int w = 0; w < nw; ++w) s += sh[q][w];
            tot[q] = s;
        }
        finish(tot);
        *counter = 0;
    }
}

#define LIST_ARGS const long long *__restrict__ slice_off, const int *__restrict__ ncnt, const int *__restrict__ nbr

static inline int red_grid(int n) { return std::max(1, std::min((n + 255) / 256, 148 * 8)); }

struct PpeRows {
    const int4 *ty;
    const int *kind;      // 0 identity, 1 fluid, 2 Neumann, 3 outlet copy, 4 pinned
    const int *aux;       // outlet partner per row (kind 3)
};

// ---------------------------------------------------------------------------
// PPE row assembly: b_i, A_i and (optionally) the cached c_ij
// ---------------------------------------------------------------------------
template <class Real, class C>
__global__ void __launch_bounds__(128) k_ppe_rows(DevParams P, const float4 *__restrict__ pf,
                                                  const typename V4<Real>::type *__restrict__ pr,
                                                  const typename V2<Real>::type *__restrict__ mr,
                                                  const int4 *__restrict__ ty, const int *__restrict__ jc, LIST_ARGS,
                                                  const Real *__restrict__ g6, const typename V4<Real>::type *__restrict__ u,
                                                  Real tdt, Real *__restrict__ b, Real *__restrict__ diag,
                                                  C *__restrict__ coef, Real *__restrict__ gb, long long nnzp, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int4 ti = ty[i];
    if (ti.x > 2 || ti.w >= 1000 || ti.w <= 0) return;
    const size_t N = (size_t)n;
    const auto xi = pr[i];
    const auto ui = u[i];
    const Real rhoi = mr[i].y;
    const Real gc11 = g6[i], gc22 = g6[N + i], gc33 = g6[2 * N + i], gc12 = g6[3 * N + i], gc23 = g6[4 * N + i], gc31 = g6[5 * N + i];
    const Real hi = (Real)(P.pressure_length * (double)xi.w);
    const Real tA = calc_tmpA<Real>(P, hi);
    Real bx = 0, by = 0, bz = 0, Aij = 0;
    const long long base = slice_off[i >> 5] + (i & 31);
    const int cnt = ncnt[i];
    for (int k = 0; k < cnt; ++k) {
        const long long e = base + 32LL * k;
        const int j = __ldg(&nbr[e]);
        const int jcj = jc[j];
        Real c = 0;
        if ((jcj & JB_LT1000) && !(jcj & JB_IT4)) {
            const auto xj = pr[j];
            const auto mj = mr[j];
            const Real dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
            const Real tdist = sqrt(dx * dx + dy * dy + dz * dz) + (Real)1e-20;
            Real dw;
            if (P.ppe_pair_h == 1) {   // the multi-resolution form, functions_PPE.cuh:113-116
                const Real hij = (Real)0.5 * (hi + (Real)(P.pressure_length * (double)xj.w));
                dw = calc_dwij_pressure<Real>(P, calc_tmpA<Real>(P, hij), hij, tdist);
            } else {
                dw = calc_dwij_pressure<Real>(P, tA, hi, tdist);
            }
            const Real tdx = dw * dx / tdist, tdy = dw * dy / tdist, tdz = dw * dz / tdist;
            const Real cx = gc11 * tdx + gc12 * tdy + gc31 * tdz;
            const Real cy = gc12 * tdx + gc22 * tdy + gc23 * tdz;
            const Real cz = gc31 * tdx + gc23 * tdy + gc33 * tdz;
            const auto uj = u[j];
            const Real vj = mj.x / mj.y;
            const Real wr = (Real)2 * rhoi * mj.y / (rhoi + mj.y);
            bx += vj * (uj.x - ui.x) * cx * wr;
            by += vj * (uj.y - ui.y) * cy * wr;
            bz += vj * (uj.z - ui.z) * cz * wr;
            c = (Real)2 * vj * (dx * cx + dy * cy + dz * cz) / tdist / tdist;
            Aij += c;
            if (gb) { gb[e] = vj * cx * wr; gb[nnzp + e] = vj * cy * wr; gb[2 * nnzp + e] = vj * cz * wr; }
        } else if (gb) {
            gb[e] = 0; gb[nnzp + e] = 0; gb[2 * nnzp + e] = 0;
        }
        if (coef) coef[sell4(slice_off[i >> 5], i & 31, k)] = (C)c;
    }
    b[i] = (bx + by + bz) / tdt;
    diag[i] = Aij;
}

// the right-hand side of later steps from the cached pair vectors (9 flops
// and 16 bytes of stored entry per pair: bandwidth bound)
// g_ij = m_j/rho_j * 2 rho_i rho_j / (rho_i + rho_j) * G_i grad W_ij (the
// particles, masses and densities do not change between steps)
template <class Real>
__global__ void __launch_bounds__(128) k_ppe_rhs(const int4 *__restrict__ ty, LIST_ARGS,
                                                 const typename V4<Real>::type *__restrict__ u,
                                                 const Real *__restrict__ gb, long long nnzp, Real tdt,
                                                 Real *__restrict__ b, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int4 ti = ty[i];
    if (ti.x > 2 || ti.w >= 1000 || ti.w <= 0) return;
    const auto ui = u[i];
    Real bx = 0, by = 0, bz = 0;
    const long long base = slice_off[i >> 5] + (i & 31);
    const int cnt = ncnt[i];
    for (int k = 0; k < cnt; ++k) {
        const long long e = base + 32LL * k;
        const auto uj = u[__ldg(&nbr[e])];
        bx += (uj.x - ui.x) * __ldcs(&gb[e]);
        by += (uj.y - ui.y) * __ldcs(&gb[nnzp + e]);
        bz += (uj.z - ui.z) * __ldcs(&gb[2 * nnzp + e]);
    }
    b[i] = (bx + by + bz) / tdt;
}

// one Jacobi sweep of KERNEL_PPE3D with the cached row: p_new = p0 + (b + sum c (p_j - p0_j)) / A
template <class Real, class C>
__global__ void __launch_bounds__(128) k_ppe_sweep(const int4 *__restrict__ ty, LIST_ARGS, const C *__restrict__ coef,
                                                   const Real *__restrict__ b, const Real *__restrict__ diag,
                                                   const Real *__restrict__ p, const Real *__restrict__ p0,
                                                   Real *__restrict__ pout, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int4 ti = ty[i];
    if (ti.x > 2 || ti.w >= 1000 || ti.w <= 0) { pout[i] = p[i]; return; }
    const long long base = slice_off[i >> 5] + (i & 31);
    const int cnt = ncnt[i];
    Real s = 0;
    for (int k = 0; k < cnt; ++k) {
        const long long e = base + 32LL * k;
        const int j = __ldg(&nbr[e]);
        s += (Real)coef[sell4(slice_off[i >> 5], i & 31, k)] * (p[j] - p0[j]);
    }
    pout[i] = p0[i] + (b[i] + s) / diag[i];
}

// ---------------------------------------------------------------------------
// operator y = M x with the cached coefficients (vectors of type V)
// ---------------------------------------------------------------------------
// One launch for the whole operator: the Neumann rows (one warp per row over
// their CSR weights) and the SELL rows (one thread per row) are disjoint row
// sets, so their blocks are interleaved in one grid and the latency-bound
// Neumann gathers run beside the bandwidth-bound SELL sweep.  Blocks
// alternate Neumann / SELL while both kinds remain; the rest are of the
// larger kind.
//
// The coefficients are read four entries at a time (sell4 layout): one
// 16-byte load per four FP32 coefficients, then the four gathers, which
// halves the load requests of the stream against one entry per load.
// L16: the neighbours are 16-bit codes (cell plane dz of the entry, offset
// from that plane's first reachable record; plane_cell in common.cuh), four
// per 8-byte load, instead of 32-bit indices.  A row's five plane starts
// come from the cell-start array (cache resident) once per row, and a
// select chain picks one per entry.  Both forms visit the entries of the
// 32-bit list in its order, so their sums are identical.
template <class C>
__device__ __forceinline__ void load_coef4(const C *p, C (&a)[4]);
template <>
__device__ __forceinline__ void load_coef4<float>(const float *p, float (&a)[4]) {
    const float4 v = __ldcs(reinterpret_cast<const float4 *>(p));
    a[0] = v.x; a[1] = v.y; a[2] = v.z; a[3] = v.w;
}
template <>
__device__ __forceinline__ void load_coef4<double>(const double *p, double (&a)[4]) {
    const double2 v = __ldcs(reinterpret_cast<const double2 *>(p));
    const double2 w = __ldcs(reinterpret_cast<const double2 *>(p) + 1);
    a[0] = v.x; a[1] = v.y; a[2] = w.x; a[3] = w.y;
}
template <>
__device__ __forceinline__ void load_coef4<__half>(const __half *p, __half (&a)[4]) {
    const uint2 v = __ldcs(reinterpret_cast<const uint2 *>(p));
    a[0] = __ushort_as_half((unsigned short)(v.x & 0xffffu));
    a[1] = __ushort_as_half((unsigned short)(v.x >> 16));
    a[2] = __ushort_as_half((unsigned short)(v.y & 0xffffu));
    a[3] = __ushort_as_half((unsigned short)(v.y >> 16));
}
template <class V, class C>
__device__ __forceinline__ V coef_to(C a) { return (V)a; }
template <>
__device__ __forceinline__ float coef_to<float, __half>(__half a) { return __half2float(a); }
// Gathers of the operand x_j with an L2 evict-last policy: the launch
// streams its codes and coefficients once (loaded evict-first with __ldcs),
// while x is gathered once per stored entry, so x should stay in L2 while
// the stream passes through it
__device__ __forceinline__ unsigned long long l2_keep_policy() {
    unsigned long long pol;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
template <class V>
__device__ __forceinline__ V ld_keep(const V *p, unsigned long long pol);
template <>
__device__ __forceinline__ float ld_keep<float>(const float *p, unsigned long long pol) {
    float v;
    asm("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
    return v;
}
template <>
__device__ __forceinline__ double ld_keep<double>(const double *p, unsigned long long pol) {
    double v;
    asm("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
    return v;
}

struct List16 {
    const uint16_t *code;
    const int *row_cell, *cs;
    int NI, NINJ, cs_max;
};

// one group of four entries of a row: the coefficients in one load, the
// neighbours from four 16-bit codes (plane starts in the thread's column of
// the shared table) or from the 32-bit list; GUARD only for the row's last,
// partly filled group
template <bool L16, bool GUARD, class V, class C>
__device__ __forceinline__ void quad_step(int k, int cnt, long long sb, int lane, const C *__restrict__ coef,
                                          const uint16_t *__restrict__ code, const int *__restrict__ nbr,
                                          const int *plane_start, const V *__restrict__ x, V xi, V &s,
                                          unsigned long long pol) {
    const long long e4 = sell4(sb, lane, k);
    C a[4];
    load_coef4<C>(coef + e4, a);
    int j[4];
    if (L16) {
        const uint2 q = __ldcs(reinterpret_cast<const uint2 *>(code + e4));
        const unsigned cc[4] = {q.x & 0xffffu, q.x >> 16, q.y & 0xffffu, q.y >> 16};
        // the padding entries of a last group hold no code: not decoded
#pragma unroll
        for (int t = 0; t < 4; ++t)
            j[t] = (!GUARD || k + t < cnt) ? plane_start[128 * (cc[t] >> kCodeShift)] + (int)(cc[t] & kCodeMask) : 0;
    } else {
        const long long e = sb + lane + 32LL * k;
#pragma unroll
        for (int t = 0; t < 4; ++t) j[t] = (!GUARD || k + t < cnt) ? __ldg(&nbr[e + 32 * t]) : 0;
    }
    V xj[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) xj[t] = (!GUARD || k + t < cnt) ? ld_keep<V>(x + j[t], pol) : xi;
#pragma unroll
    for (int t = 0; t < 4; ++t)   // difference form, entries in list order
        if (!GUARD || k + t < cnt) s += coef_to<V, C>(a[t]) * (xi - xj[t]);
}

template <class V, class C, class D, class W, bool L16>
__global__ void __launch_bounds__(128) k_spmv_fused(int nb_nm, int nb_sell, const int *__restrict__ kind,
                                                    const int *__restrict__ aux, LIST_ARGS, List16 l16,
                                                    const C *__restrict__ coef, const float *__restrict__ rowscale,
                                                    const D *__restrict__ diag, const int *__restrict__ comp_id,
                                                    const double *__restrict__ cmean, const int *__restrict__ nm_rows,
                                                    const int *__restrict__ nm_off, const int *__restrict__ nm_nb,
                                                    const W *__restrict__ nm_w, int n_nm, const V *__restrict__ x,
                                                    V *__restrict__ y, int n) {
    const int b = blockIdx.x;
    const int m = min(nb_nm, nb_sell);
    bool neu;
    int idx;
    if (b < 2 * m) { neu = (b & 1) == 0; idx = b >> 1; }
    else { neu = nb_nm > nb_sell; idx = m + (b - 2 * m); }
    if (neu) {
        const int k = idx * 4 + (threadIdx.x >> 5);
        const int lane = threadIdx.x & 31;
        if (k >= n_nm) return;   // uniform over the warp
        const int i = nm_rows[k];
        if (kind[i] != 2) return;   // an outlet copy row written by the SELL blocks
        const V xi = x[i];
        const int q0 = nm_off[k], q1 = nm_off[k + 1];
        double s = 0;   // the weights sum to one: x_w - sum w x_k = sum w (x_w - x_k)
        for (int q = q0 + lane; q < q1; q += 32) s += (double)__ldcs(&nm_w[q]) * (double)(xi - x[__ldcs(&nm_nb[q])]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) y[i] = (q1 > q0) ? (V)s : xi;
        return;
    }
    const int i = idx * 128 + threadIdx.x;
    if (i >= n) return;
    const int kd = kind[i];
    if (kd == 2) return;   // written by the Neumann blocks
    const V xi = x[i];
    V yi = xi;   // identity / pinned
    if (kd == 1) {
        const long long sb = slice_off[i >> 5];
        const int lane = i & 31;
        const int cnt = ncnt[i];
        V s = 0;
        // the row's five plane starts, in this thread's column (no other
        // thread reads it, so no barrier)
        __shared__ int plane_tab[5 * 128];
        int *ps = plane_tab + threadIdx.x;
        if (L16) {
            const int rc = l16.row_cell[i];
#pragma unroll
            for (int q = 0; q < 5; ++q)
                ps[128 * q] = __ldg(&l16.cs[plane_cell(rc, q - 2, l16.NI, l16.NINJ, l16.cs_max)]);
        }
        const int full = cnt & ~3;
        const unsigned long long pol = l2_keep_policy();
        int k = 0;
        for (; k < full; k += 4) quad_step<L16, false, V, C>(k, cnt, sb, lane, coef, l16.code, nbr, ps, x, xi, s, pol);
        if (k < cnt) quad_step<L16, true, V, C>(k, cnt, sb, lane, coef, l16.code, nbr, ps, x, xi, s, pol);
        yi = rowscale ? s * (V)rowscale[i] : s;
        if (comp_id) {
            const int cc = comp_id[i];
            if (cc >= 0) yi += (V)diag[i] * (V)cmean[cc];
        }
    } else if (kd == 3) {
        const int j = aux[i];
        if (j >= 0) yi = xi - x[j];
    }
    y[i] = yi;
}

// FP16 copy of the cached FP32 coefficients of the fluid rows, each row
// divided by its largest |c_ij| (kept as an FP32 row scale, 1 for rows
// without entries); the padding of a row's last group of four is zeroed
__global__ void __launch_bounds__(128) k_coef_half(const int *__restrict__ kind, const long long *__restrict__ slice_off,
                                                   const int *__restrict__ ncnt, const float *__restrict__ coef,
                                                   __half *__restrict__ ch, float *__restrict__ rs, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (kind[i] != 1) { rs[i] = 1.f; return; }
    const long long sb = slice_off[i >> 5];
    const int lane = i & 31, cnt = ncnt[i], padded = (cnt + 3) & ~3;
    float mx = 0.f;
    for (int k = 0; k < cnt; ++k) mx = fmaxf(mx, fabsf(coef[sell4(sb, lane, k)]));
    const float scale = mx > 0.f ? mx : 1.f;
    const float inv = 1.f / scale;
    for (int k = 0; k < padded; ++k) {
        const long long e = sell4(sb, lane, k);
        ch[e] = __float2half_rn(k < cnt ? coef[e] * inv : 0.f);
    }
    rs[i] = scale;
}

// z += Z y_c (coarse correction) with the per-component mean of the result
// for the rank-one term of the next operator application (the sums of
// k_comp_mean, in the same grid and order)
template <class V, int NC>
__global__ void k_coarse_add_mean(const int *agg, const double *yc, V *z, const int *comp_id, int n, int ncomp,
                                  const double *inv, double *partials, unsigned int *counter, double *cmean) {
    double v[NC];
#pragma unroll
    for (int q = 0; q < NC; ++q) v[q] = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int a = agg[i];
        V zi = z[i];
        if (a >= 0) { zi += (V)yc[a]; z[i] = zi; }
        const int cc = comp_id[i];
#pragma unroll
        for (int q = 0; q < NC; ++q)
            if (cc == q) v[q] += (double)zi;
    }
    reduce_finish<NC>(v, partials, counter, [&](double *t) {
        for (int q = 0; q < ncomp; ++q) cmean[q] = t[q] * inv[q];
    });
}

// per-component mean of x over the fluid rows of the singular components:
// cmean[c] = (1/|u_c|) sum_{i in u_c} x_i, deterministic (block partials)
// (NC = 1 for the common single-component case, SPH_MAX_COMP otherwise)
template <class V, int NC>
__global__ void k_comp_mean(const int *comp_id, const V *x, int n, int ncomp, const double *inv, double *partials,
                            unsigned int *counter, double *cmean) {
    double v[NC];
#pragma unroll
    for (int q = 0; q < NC; ++q) v[q] = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int cc = comp_id[i];
#pragma unroll
        for (int q = 0; q < NC; ++q)
            if (cc == q) v[q] += (double)x[i];
    }
    reduce_finish<NC>(v, partials, counter, [&](double *t) {
        for (int q = 0; q < ncomp; ++q) cmean[q] = t[q] * inv[q];
    });
}

// matrix-free variant: c_ij recomputed from the positions at every application
template <class Real, class V>
__global__ void __launch_bounds__(128) k_spmv_mf(DevParams P, const int *__restrict__ kind, const int *__restrict__ aux,
                                                 const typename V4<Real>::type *__restrict__ pr,
                                                 const typename V2<Real>::type *__restrict__ mr,
                                                 const int *__restrict__ jc, LIST_ARGS, const Real *__restrict__ g6,
                                                 const Real *__restrict__ diag, const int *__restrict__ comp_id,
                                                 const double *__restrict__ cmean, const V *__restrict__ x,
                                                 V *__restrict__ y, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int kd = kind[i];
    const V xi = x[i];
    V yi = xi;
    if (kd == 1) {
        const size_t N = (size_t)n;
        const auto xp = pr[i];
        const Real gc11 = g6[i], gc22 = g6[N + i], gc33 = g6[2 * N + i], gc12 = g6[3 * N + i], gc23 = g6[4 * N + i], gc31 = g6[5 * N + i];
        const Real hi = (Real)(P.pressure_length * (double)xp.w);
        const Real tA = calc_tmpA<Real>(P, hi);
        const long long base = slice_off[i >> 5] + (i & 31);
        const int cnt = ncnt[i];
        V s = 0;
        for (int k = 0; k < cnt; ++k) {
            const int j = __ldg(&nbr[base + 32LL * k]);
            const int jcj = jc[j];
            if (!(jcj & JB_LT1000) || (jcj & JB_IT4)) continue;
            const auto xj = pr[j];
            const auto mj = mr[j];
            const Real dx = xp.x - xj.x, dy = xp.y - xj.y, dz = xp.z - xj.z;
            const Real tdist = sqrt(dx * dx + dy * dy + dz * dz) + (Real)1e-20;
            Real dw;
            if (P.ppe_pair_h == 1) {   // the multi-resolution form, functions_PPE.cuh:113-116
                const Real hij = (Real)0.5 * (hi + (Real)(P.pressure_length * (double)xj.w));
                dw = calc_dwij_pressure<Real>(P, calc_tmpA<Real>(P, hij), hij, tdist);
            } else {
                dw = calc_dwij_pressure<Real>(P, tA, hi, tdist);
            }
            const Real tdx = dw * dx / tdist, tdy = dw * dy / tdist, tdz = dw * dz / tdist;
            const Real cx = gc11 * tdx + gc12 * tdy + gc31 * tdz;
            const Real cy = gc12 * tdx + gc22 * tdy + gc23 * tdz;
            const Real cz = gc31 * tdx + gc23 * tdy + gc33 * tdz;
            const Real c = (Real)2 * (mj.x / mj.y) * (dx * cx + dy * cy + dz * cz) / tdist / tdist;
            s += (V)c * (xi - x[j]);   // difference form, as k_spmv
        }
        yi = s;
        if (comp_id) {
            const int cc = comp_id[i];
            if (cc >= 0) yi += (V)diag[i] * (V)cmean[cc];   // A_i * mean: beside the spectrum
        }
    } else if (kd == 3) {
        const int j = aux[i];
        if (j >= 0) yi = xi - x[j];
    }
    y[i] = yi;
}

// Neumann rows of the operator: y_w = x_w - sum_k w_k x_k with the Shepard
// weights.  Inlet mirror rows also enter with their Shepard weights: the
// extrapolation weights (functions_BC.cuh:444) do not form a stochastic row
// and make the implicit system indefinite; the extrapolated pressure is set
// after the solve by the Neumann pass, as the reference sets it after its
// sweep.  Rows whose reference Shepard set is empty (p = 0 in the reference)
// enter with the Shepard average over all fluid in range, so that corner
// rows do not act as point Dirichlet anchors; the pass still writes p = 0.
// One warp per row: the lanes read the row's CSR entries coalesced.
template <class V, class W>
__global__ void __launch_bounds__(256) k_spmv_neumann(const int *__restrict__ kind, const int *__restrict__ rows,
                                                      const int *__restrict__ off, const int *__restrict__ nb,
                                                      const W *__restrict__ w, int nrows, const V *__restrict__ x,
                                                      V *__restrict__ y) {
    const int k = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (k >= nrows) return;   // uniform over the warp
    const int i = rows[k];
    if (kind[i] != 2) return;   // an outlet copy row (the row operator wrote it)
    const V xi = x[i];
    const int q0 = off[k], q1 = off[k + 1];
    double s = 0;   // the weights sum to one: x_w - sum w x_k = sum w (x_w - x_k)
    for (int q = q0 + lane; q < q1; q += 32) s += (double)__ldcs(&w[q]) * (double)(xi - x[__ldcs(&nb[q])]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) y[i] = (q1 > q0) ? (V)s : xi;
}

// ---------------------------------------------------------------------------
// BiCGSTAB vector kernels (device-resident scalars, enum SC_*)
// ---------------------------------------------------------------------------
template <class V>
__global__ void k_norm2(const V *a, int n, double *partials, unsigned int *counter, double *scal, int slot) {
    double v[1] = {0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[0] += (double)a[i] * (double)a[i];
    reduce_finish<1>(v, partials, counter, [&](double *t) { scal[slot] = t[0]; });
}

// after v = M ph: alpha = rho / (rh, v)
template <class V>
__global__ void k_alpha(const V *rh, const V *v, int n, double *partials, unsigned int *counter, double *scal) {
    if (scal[SC_FLAG] != FLAG_RUN) return;
    double d[1] = {0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) d[0] += (double)rh[i] * (double)v[i];
    reduce_finish<1>(d, partials, counter, [&](double *t) {
        scal[SC_RV] = t[0];
        if (t[0] == 0.0 || !isfinite(t[0])) { scal[SC_FLAG] = FLAG_BREAKDOWN; return; }
        scal[SC_ALPHA] = scal[SC_RHO] / t[0];
    });
}

// s = r - alpha v ; sh = dinv s
template <class V>
__global__ void k_s_update(const V *r, const V *v, V *s, V *sh, const V *dinv, int n, const double *scal) {
    if (scal[SC_FLAG] != FLAG_RUN) return;
    const V alpha = (V)scal[SC_ALPHA];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const V si = r[i] - alpha * v[i];
        s[i] = si;
        sh[i] = dinv[i] * si;
    }
}

// after t = M sh: omega = (t, s) / (t, t)
template <class V>
__global__ void k_omega(const V *t, const V *s, int n, double *partials, unsigned int *counter, double *scal) {
    if (scal[SC_FLAG] != FLAG_RUN) return;
    double d[2] = {0, 0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        d[0] += (double)t[i] * (double)s[i];
        d[1] += (double)t[i] * (double)t[i];
    }
    reduce_finish<2>(d, partials, counter, [&](double *tt) {
        scal[SC_TS] = tt[0];
        scal[SC_TT] = tt[1];
        scal[SC_OMEGA] = tt[1] > 0 ? tt[0] / tt[1] : 0.0;
    });
}

// x += alpha ph + omega sh ; r = s - omega t ; rho' = (rh, r), rr = (r, r)
template <class V>
__global__ void k_xr_update(V *x, V *r, const V *ph, const V *sh, const V *s, const V *t, const V *rh, int n,
                            double *partials, unsigned int *counter, double *scal) {
    if (scal[SC_FLAG] != FLAG_RUN) return;
    const V alpha = (V)scal[SC_ALPHA], omega = (V)scal[SC_OMEGA];
    double d[2] = {0, 0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        x[i] += alpha * ph[i] + omega * sh[i];
        const V ri = s[i] - omega * t[i];
        r[i] = ri;
        d[0] += (double)rh[i] * (double)ri;
        d[1] += (double)ri * (double)ri;
    }
    reduce_finish<2>(d, partials, counter, [&](double *tt) {
        const double rho_new = tt[0];
        scal[SC_RR] = tt[1];
        scal[SC_ITN] += 1.0;   // iterations that ran (the kernels idle once the flag is set)
        if (tt[1] <= scal[SC_TOL2]) scal[SC_FLAG] = FLAG_CONVERGED;
        else if (rho_new == 0.0 || scal[SC_OMEGA] == 0.0 || !isfinite(tt[1])) scal[SC_FLAG] = FLAG_BREAKDOWN;
        scal[SC_BETA] = (rho_new / scal[SC_RHO]) * (scal[SC_ALPHA] / scal[SC_OMEGA]);
        scal[SC_RHO] = rho_new;
    });
}

// p = r + beta (p - omega v) ; ph = dinv p
template <class V>
__global__ void k_p_update(V *p, V *ph, const V *r, const V *v, const V *dinv, int n, const double *scal) {
    if (scal[SC_FLAG] != FLAG_RUN) return;
    const V beta = (V)scal[SC_BETA], omega = (V)scal[SC_OMEGA];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const V pi = r[i] + beta * (p[i] - omega * v[i]);
        p[i] = pi;
        ph[i] = dinv[i] * pi;
    }
}

// r = b - y ; rh = r ; p = v = 0 (start / restart)
template <class V>
__global__ void k_residual_init(const V *b, const V *y, V *r, V *rh, V *p, V *v, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const V ri = b[i] - y[i];
        r[i] = ri; rh[i] = ri; p[i] = 0; v[i] = 0;
    }
}

// refinement residual: rd = bd - yd (FP64); rf = (float) rd; ef = 0
__global__ void k_ir_residual(const double *bd, const double *yd, double *rd, float *rf, float *ef, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double r = bd[i] - yd[i];
        rd[i] = r;
        rf[i] = (float)r;
        ef[i] = 0.f;
    }
}

template <class V, class D>
__global__ void k_dinv(const int *kind, const D *diag, V *dinv, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double a = 1.0;
    if (kind[i] == 1) {
        a = (double)diag[i];
        if (a == 0.0 || !isfinite(a)) a = 1.0;
    }
    dinv[i] = (V)(1.0 / a);
}

// right-hand side and initial guess (previous pressure) of the converged system
template <class Real>
__global__ void k_rhs(const int *kind, const Real *b, const Real *p_old, double *rhs, double *x0, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int kd = kind[i];
    double v = 0, x = (double)p_old[i];
    if (kd == 1) v = (double)b[i];
    else if (kd == 0) v = (double)p_old[i];
    else if (kd == 4) x = 0;
    rhs[i] = v;
    x0[i] = x;
}

template <class A, class B>
__global__ void k_cast(const A *a, B *b, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (B)a[i];
}
template <class A, class B>
__global__ void k_axpy_cast(const A *e, B *x, int n) {   // x += e
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] += (B)e[i];
}
__global__ void k_set_scal(double *scal, double rho, double tol2) {
    scal[SC_RHO] = rho; scal[SC_ALPHA] = 1; scal[SC_OMEGA] = 1; scal[SC_BETA] = 0;
    scal[SC_FLAG] = FLAG_RUN; scal[SC_TOL2] = tol2;
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

// y = M x, vectors of type V (V = Real for the Krylov iterations, V = double
// for the FP64 refinement residual of the mixed form)
// drains the pending operator timings into the running totals
template <class Real>
static void prof_drain(Ctx<Real> &c) {
    if (c.prof_pending == 0) return;
    cudaEventSynchronize(c.prof_ev[2 * c.prof_pending - 1]);
    for (int k = 0; k < c.prof_pending; ++k) {
        float ms = 0;
        cudaEventElapsedTime(&ms, c.prof_ev[2 * k], c.prof_ev[2 * k + 1]);
        c.prof_ms += ms;
        ++c.prof_launches;
    }
    c.prof_pending = 0;
}

template <class Real, class V>
static void apply_op(Ctx<Real> &c, const V *x, V *y, bool cached, bool mean_ready = false) {
    const int n = c.n;
    const bool timed = c.prof && sizeof(V) == sizeof(Real);
    // inside a graph capture the timing events become event-record nodes of
    // the graph (read after each replay)
    const bool cap_timed = timed && c.cap_ev && c.cap_n < c.cap_max;
    if (cap_timed) {
        cudaEventRecordWithFlags(c.cap_ev[2 * c.cap_n], c.stream, cudaEventRecordExternal);
    } else if (timed && !c.cap_ev) {
        if (c.prof_pending == 256) prof_drain(c);
        if (!c.prof_ev) {
            c.prof_ev = new cudaEvent_t[512];
            for (int k = 0; k < 512; ++k) cudaEventCreate(&c.prof_ev[k]);
        }
        cudaEventRecord(c.prof_ev[2 * c.prof_pending], c.stream);
    }
    const int *cid = nullptr;
    double *cmean = c.scal + 40;
    if (c.n_comp > 0) cid = c.comp_id;
    if (c.n_comp > 0 && !mean_ready) {
        if (c.n_comp == 1)
            k_comp_mean<V, 1><<<red_grid(n), 256, 0, c.stream>>>(c.comp_id, x, n, 1, c.comp_inv, c.red,
                                                                 (unsigned int *)(c.scal + 32), cmean);
        else
            k_comp_mean<V, SPH_MAX_COMP><<<red_grid(n), 256, 0, c.stream>>>(c.comp_id, x, n, c.n_comp, c.comp_inv, c.red,
                                                                            (unsigned int *)(c.scal + 32), cmean);
        ++c.launches;
    }
    if (cached) {
        // FP32 Neumann weights in the FP32 applications of the mixed form; the
        // FP64 applications (true residuals) keep the FP64 weights
        const int nb_nm = div_up((long long)c.L.n_nm, 4), nb_sell = div_up((long long)n, 128);
        const List16 l16{c.nbr16, c.row_cell, c.cell_start, c.dp.NI, c.dp.NI * c.dp.NJ, c.num_cells + 1};
#define SPMV_FUSED(C_, W_, COEF, RS, NMW)                                                                          \
    do {                                                                                                       \
        if (c.list16)                                                                                          \
            k_spmv_fused<V, C_, Real, W_, true><<<nb_nm + nb_sell, 128, 0, c.stream>>>(                        \
                nb_nm, nb_sell, c.row_kind, c.row_aux, c.slice_off, c.ncnt, c.nbr, l16, COEF, RS, c.diag, cid,   \
                cmean, c.L.nm_rows, c.L.nm_off, c.L.nm_nbr, NMW, c.L.n_nm, x, y, n);                            \
        else                                                                                                   \
            k_spmv_fused<V, C_, Real, W_, false><<<nb_nm + nb_sell, 128, 0, c.stream>>>(                       \
                nb_nm, nb_sell, c.row_kind, c.row_aux, c.slice_off, c.ncnt, c.nbr, l16, COEF, RS, c.diag, cid,   \
                cmean, c.L.nm_rows, c.L.nm_off, c.L.nm_nbr, NMW, c.L.n_nm, x, y, n);                            \
    } while (0)
        if (sizeof(Real) == 4 && sizeof(V) == 4 && c.prm.ppe_coef_half && c.coef_h_valid)
            SPMV_FUSED(__half, float, c.coef_h, c.coef_rs, c.nm_owf);
        else if (sizeof(Real) == 4 && sizeof(V) == 4)
            SPMV_FUSED(float, float, (const float *)c.coef, nullptr, c.nm_owf);
        else if (sizeof(Real) == 4)
            SPMV_FUSED(float, double, (const float *)c.coef, nullptr, c.nm_ow);
        else
            SPMV_FUSED(double, double, c.coef_d, nullptr, c.nm_ow);
#undef SPMV_FUSED
    } else {
        k_spmv_mf<Real, V><<<grid_for(n, 128), 128, 0, c.stream>>>(c.dp, c.row_kind, c.row_aux, c.pr, c.mr, c.jc, c.slice_off,
                                                                  c.ncnt, c.nbr, c.g6, c.diag, cid, cmean, x, y, n);
    }
    ++c.launches;
    if (cap_timed) {
        cudaEventRecordWithFlags(c.cap_ev[2 * c.cap_n + 1], c.stream, cudaEventRecordExternal);
        ++c.cap_n;
    } else if (timed && !c.cap_ev) {
        cudaEventRecord(c.prof_ev[2 * c.prof_pending + 1], c.stream);
        ++c.prof_pending;
    }
    if (!cached && c.L.n_nm > 0) {
        const int gnm = div_up((long long)c.L.n_nm * 32, 256);
        // FP32 weights in the FP32 applications of the mixed form; the FP64
        // applications (true residuals) keep the FP64 weights
        if (sizeof(Real) == 4 && sizeof(V) == 4)
            k_spmv_neumann<V, float><<<gnm, 256, 0, c.stream>>>(c.row_kind, c.L.nm_rows, c.L.nm_off, c.L.nm_nbr, c.nm_owf,
                                                                c.L.n_nm, x, y);
        else
            k_spmv_neumann<V, double><<<gnm, 256, 0, c.stream>>>(c.row_kind, c.L.nm_rows, c.L.nm_off, c.L.nm_nbr, c.nm_ow,
                                                                 c.L.n_nm, x, y);
        ++c.launches;
    }
}

// start vector a x with a = (b, y) / (y, y), y = M x: the multiple of x with
// the smallest residual (x unchanged when y = 0)
__global__ void k_start_factor(const double *b, const double *y, int n, double *partials, unsigned int *counter,
                               double *scal) {
    double d[2] = {0, 0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        d[0] += b[i] * y[i];
        d[1] += y[i] * y[i];
    }
    reduce_finish<2>(d, partials, counter, [&](double *t) { scal[SC_ALPHA] = t[1] > 0 ? t[0] / t[1] : 1.0; });
}

__global__ void k_scale_start(double *x, int n, const double *scal) {
    const double a = scal[SC_ALPHA];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] *= a;
}

// y = M x with FP64 vectors and the context's cached or matrix-free operator
template <class Real>
void ppe_apply_fp64(Ctx<Real> &c, const double *x, double *y) {
    apply_op<Real, double>(c, x, y, c.prm.ppe_matrix_free == 0);
}

template <class Real>
int operator_stats(Ctx<Real> &c, int64_t *launches, double *total_ms, double *bytes, int reset) {
    prof_drain(c);
    if (launches) *launches = c.prof_launches;
    if (total_ms) *total_ms = c.prof_ms;
    if (bytes) {
        // per row: kind and list length (4 + 4) + x_i + y_i (Real), with the
        // rank-one term also component id (4) + A_i (Real); per slice of 32
        // rows its offset (8); per stored entry of a fluid row (the only
        // rows whose entries the launch reads): index (4, or 2 for the
        // 16-bit codes, which add the row's cell (4) per row and the cell
        // starts once) + coefficient (float, or half with ppe_coef_half, in
        // the mixed form; double in the FP64 form; the FP16 coefficients add
        // a row scale (4) per row).  The Neumann rows of the same launch: row index
        // and offset (4 + 4) + x_i + y_i, per entry index (4) + weight
        // (Real).  The gathers x_j are not counted: an ideal kernel serves
        // them from L2.
        const double R = (double)sizeof(Real);
        const bool l16 = c.list16 && c.prm.ppe_matrix_free == 0;
        const bool half = sizeof(Real) == 4 && c.prm.ppe_coef_half && c.coef_h_valid && c.prm.ppe_matrix_free == 0;
        double row = 8.0 + 2.0 * R + (l16 ? 4.0 : 0.0) + (half ? 4.0 : 0.0);
        if (c.n_comp > 0) row += 4.0 + R;
        *bytes = (double)c.n * row + 8.0 * (double)((c.n + 31) / 32) +
                 (double)c.nnz_op * ((l16 ? 2.0 : 4.0) + (half ? 2.0 : R));
        if (l16) *bytes += 4.0 * ((double)c.num_cells + 2.0);
        if (c.prm.ppe_matrix_free == 0)
            *bytes += (double)c.L.n_nm * (8.0 + 2.0 * R) + (double)c.L.nm_nnz * (4.0 + R);
    }
    if (reset) { c.prof_launches = 0; c.prof_ms = 0; }
    return SPH_OK;
}

// Bytes of one operator launch in two accountings.  `stored`: what the
// launch's layout streams (the operator_stats figure).  `index_rule`: per row
// the fields read and written for it (kind, list length, x_i, y_i; component
// id and A_i with the rank-one term), per slice its offset, and 4 bytes per
// stored neighbour index, for the SELL rows and the Neumann rows alike --
// stored coefficients, the 16-bit code tables and the Neumann weights are
// not counted, since a kernel that recomputes them from the positions needs
// none of them.
template <class Real>
int operator_bytes(Ctx<Real> &c, double *stored, double *index_rule) {
    if (stored) SPH_TRY(operator_stats(c, nullptr, nullptr, stored, 0));
    if (index_rule) {
        const double R = (double)sizeof(Real);
        double row = 8.0 + 2.0 * R;
        if (c.n_comp > 0) row += 4.0 + R;
        *index_rule = (double)c.n * row + 8.0 * (double)((c.n + 31) / 32) + 4.0 * (double)c.nnz_op +
                      (double)c.L.n_nm * (8.0 + 2.0 * R) + 4.0 * (double)c.L.nm_nnz;
    }
    return SPH_OK;
}

// Two-level preconditioner on r, with z holding D^-1 r on entry: the
// additive form adds Z E^-1 Z^T r; the multiplicative form corrects the
// residual that the Jacobi step leaves, z += Z E^-1 Z^T (r - M z), at the
// cost of one more operator application (tmp receives M z).  With singular
// components the final add also forms the component means of z for the
// operator application that follows; returns whether it did.
template <class Real, class V>
static bool precond_coarse(Ctx<Real> &c, const V *r, V *z, V *tmp, bool cached) {
    if (c.cg_m <= 0) return false;
    const V *w = nullptr;
    if (c.prm.ppe_coarse_mode == 1) {
        apply_op<Real, V>(c, z, tmp, cached);
        w = tmp;
    }
    if (c.n_comp <= 0) {
        coarse_apply<Real, V>(c, r, z, w);
        return false;
    }
    coarse_restrict_solve<Real, V>(c, r, w);
    unsigned int *counter = (unsigned int *)(c.scal + 32);
    double *cmean = c.scal + 40;
    if (c.n_comp == 1)
        k_coarse_add_mean<V, 1><<<red_grid(c.n), 256, 0, c.stream>>>(c.cg_agg, c.cg_y, z, c.comp_id, c.n, 1, c.comp_inv,
                                                                    c.red, counter, cmean);
    else
        k_coarse_add_mean<V, SPH_MAX_COMP><<<red_grid(c.n), 256, 0, c.stream>>>(c.cg_agg, c.cg_y, z, c.comp_id, c.n,
                                                                               c.n_comp, c.comp_inv, c.red, counter, cmean);
    ++c.launches;
    return true;
}

// Jacobi-preconditioned BiCGSTAB on M x = b with vectors of type V (the
// workspace ws holds 9 of them) and FP64 dots; x holds the initial guess.
// Returns SPH_OK, SPH_NOT_CONVERGED or SPH_ERR_BREAKDOWN (> 20 restarts).
template <class Real, class V>
static int bicgstab_v(Ctx<Real> &c, V *const *ws, V *x, const V *b, double bnorm2, double tol, int maxit, bool cached,
                      int *iters, double *relres, int *restarts) {
    const int n = c.n;
    cudaStream_t st = c.stream;
    V *r = ws[0], *rh = ws[1], *p = ws[2], *v = ws[3], *s = ws[4];
    V *t = ws[5], *ph = ws[6], *sh = ws[7], *dinv = ws[8];
    const int G = red_grid(n);
    unsigned int *counter = (unsigned int *)(c.scal + 32);
    const double tol2 = tol * tol * bnorm2;
    k_dinv<V, Real><<<grid_for(n, 256), 256, 0, st>>>(c.row_kind, c.diag, dinv, n);
    SPH_CUDA_TRY(cudaMemsetAsync(c.scal + SC_ITN, 0, sizeof(double), st));
    ++c.launches;
    int it = 0;
    *restarts = 0;
    int status = SPH_NOT_CONVERGED;
    while (true) {
        apply_op<Real, V>(c, x, t, cached);
        k_residual_init<V><<<G, 256, 0, st>>>(b, t, r, rh, p, v, n);
        k_norm2<V><<<G, 256, 0, st>>>(r, n, c.red, counter, c.scal, SC_RR);
        c.launches += 2;
        SPH_CUDA_TRY(cudaMemcpyAsync(c.red_host, c.scal, sizeof(double) * SC_COUNT, cudaMemcpyDeviceToHost, st));
        SPH_CUDA_TRY(cudaStreamSynchronize(st));
        const double rr0 = c.red_host[SC_RR];
        *relres = std::sqrt(rr0 / bnorm2);
        if (c.init_relres < 0) c.init_relres = *relres;
        if (rr0 <= tol2) { status = SPH_OK; break; }
        if (it >= maxit) break;
        if (getenv("SPH_TRACE_PPE")) fprintf(stderr, "  bicgstab start it %d relres %.3e\n", it, *relres);
        k_set_scal<<<1, 1, 0, st>>>(c.scal, rr0, tol2);   // beta = 0: p = r on the first pass
        ++c.launches;
        bool restart = false;
        const int check = 4;
        while (it < maxit) {
            k_p_update<V><<<G, 256, 0, st>>>(p, ph, r, v, dinv, n, c.scal);
            bool mr = precond_coarse<Real, V>(c, p, ph, v, cached);   // v is free until M ph is written to it
            apply_op<Real, V>(c, ph, v, cached, mr);
            k_alpha<V><<<G, 256, 0, st>>>(rh, v, n, c.red, counter, c.scal);
            k_s_update<V><<<G, 256, 0, st>>>(r, v, s, sh, dinv, n, c.scal);
            mr = precond_coarse<Real, V>(c, s, sh, t, cached);        // t likewise
            apply_op<Real, V>(c, sh, t, cached, mr);
            k_omega<V><<<G, 256, 0, st>>>(t, s, n, c.red, counter, c.scal);
            k_xr_update<V><<<G, 256, 0, st>>>(x, r, ph, sh, s, t, rh, n, c.red, counter, c.scal);
            c.launches += 5;
            ++it;
            if (it % check == 0 || it >= maxit) {
                SPH_CUDA_TRY(cudaMemcpyAsync(c.red_host, c.scal, sizeof(double) * SC_COUNT, cudaMemcpyDeviceToHost, st));
                SPH_CUDA_TRY(cudaStreamSynchronize(st));
                const double flag = c.red_host[SC_FLAG];
                *relres = std::sqrt(c.red_host[SC_RR] / bnorm2);
                if (getenv("SPH_TRACE_PPE") && it % 20 == 0)
                    fprintf(stderr, "    it %d rr-rel %.3e alpha %.3e omega %.3e rho %.3e flag %g\n", it, *relres,
                            c.red_host[SC_ALPHA], c.red_host[SC_OMEGA], c.red_host[SC_RHO], flag);
                if (flag == FLAG_CONVERGED) { status = SPH_OK; break; }
                if (flag == FLAG_BREAKDOWN) { restart = true; break; }
            }
        }
        if (status == SPH_OK) break;
        if (restart) {
            if (++*restarts > 20) { status = SPH_ERR_BREAKDOWN; break; }
            continue;
        }
        break;   // iteration limit
    }
    SPH_CUDA_TRY(cudaGetLastError());
    *iters = it > 0 ? (int)c.red_host[SC_ITN] : 0;   // exact, not rounded up to the check interval
    return status;
}

template <class Real>
static int bicgstab(Ctx<Real> &c, Real *x, const Real *b, double bnorm2, double tol, int maxit, bool cached, int *iters,
                    double *relres, int *restarts) {
    return bicgstab_v<Real, Real>(c, c.kv, x, b, bnorm2, tol, maxit, cached, iters, relres, restarts);
}

// FP64 vectors on the context's operator (the mixed form's fallback)
template <class Real>
static int bicgstab_fp64(Ctx<Real> &c, double *x, const double *b, double bnorm2, double tol, int maxit, bool cached,
                         int *iters, double *relres, int *restarts) {
    return bicgstab_v<Real, double>(c, c.kd, x, b, bnorm2, tol, maxit, cached, iters, relres, restarts);
}

// ---------------------------------------------------------------------------
// mixed-precision BiCGSTAB with reliable updates (Sleijpen & van der Vorst,
// "Reliable updated residuals in hybrid Bi-CG methods", Computing 56, 1996;
// the FP32/FP64 use follows Clark et al., "Solving lattice QCD systems of
// equations using mixed precision solvers on GPUs", CPC 181, 2010).  The
// Krylov vectors, both operator applications of an iteration and the partial
// solution x_lo are FP32; the dot products are FP64.  When the recurrence
// residual has fallen by RELIABLE_DELTA since the last update, x_lo is added
// into the FP64 solution, the FP64 true residual b - M x replaces the
// recurrence residual and the search direction carries on: one FP64 operator
// application per update and no loss of the Krylov space, unlike a
// refinement loop that restarts the inner solver at every correction.
// ---------------------------------------------------------------------------
#define RELIABLE_DELTA 0.1

// The iterations between two host checks, captured once as a CUDA graph and
// replayed: one graph launch instead of about 60 kernel launches, which
// matters for the small cases of an ensemble, whose kernels last a few
// microseconds.  Only contexts on their own stream use it (the legacy
// default stream cannot be captured).  The key holds every pointer and size
// the captured launches use; a change (new lists, a rebuilt preconditioner,
// reallocated work space) recaptures.
struct KrylovGraph {
    cudaGraphExec_t exec = nullptr;
    std::vector<uintptr_t> key;
    long long nodes = 0;
    // with live operator timing on: a start / end event per operator
    // application, recorded by event nodes of the graph
    std::vector<cudaEvent_t> ev;
    int n_timed = 0;
    ~KrylovGraph() {
        for (cudaEvent_t e : ev) cudaEventDestroy(e);
    }
};

template <class Real>
static std::vector<uintptr_t> krylov_graph_key(Ctx<Real> &c, float *const *ws, const float *xlo) {
    std::vector<uintptr_t> k;
    for (int q = 0; q < 9; ++q) k.push_back((uintptr_t)ws[q]);
    const void *ptrs[] = {xlo, c.scal, c.red, c.row_kind, c.row_aux, c.slice_off, c.ncnt, c.nbr, c.coef, c.diag,
                          c.comp_id, c.comp_inv, c.L.nm_rows, c.L.nm_off, c.L.nm_nbr, c.nm_owf, c.cg_off, c.cg_rows,
                          c.cg_s, c.cg_y, c.cg_invf, c.cg_agg, c.nbr16, c.row_cell, c.cell_start, c.cg_piece,
                          c.cg_pfirst, c.cg_part, c.cg_cnt, c.coef_h, c.coef_rs};
    for (const void *q : ptrs) k.push_back((uintptr_t)q);
    const long long sizes[] = {c.n, c.n_comp, c.L.n_nm, c.cg_m, c.prm.ppe_coarse_mode, c.prof ? 1 : 0, c.list16 ? 1 : 0,
                               c.num_cells, c.cg_np};
    for (long long q : sizes) k.push_back((uintptr_t)q);
    return k;
}

// r = (float)(b - y); x_lo = 0; rho = (rh, r), rr = ||b - y||^2 (FP64);
// beta is rescaled to the replaced rho so the next direction stays conjugate
template <class V>
__global__ void k_reliable_replace(const double *bd, const double *yd, V *r, V *xlo, const V *rh, int n,
                                   double *partials, unsigned int *counter, double *scal) {
    double d[2] = {0, 0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double ri = bd[i] - yd[i];
        const V rf = (V)ri;
        r[i] = rf;
        xlo[i] = 0;
        d[0] += (double)rh[i] * (double)rf;
        d[1] += ri * ri;
    }
    reduce_finish<2>(d, partials, counter, [&](double *t) {
        const double rho_rec = scal[SC_RHO];
        if (rho_rec != 0.0 && isfinite(rho_rec)) scal[SC_BETA] *= t[0] / rho_rec;
        scal[SC_RHO] = t[0];
        scal[SC_RR] = t[1];
        scal[SC_FLAG] = (t[1] <= scal[SC_TOL2]) ? FLAG_CONVERGED : (t[0] == 0.0 ? FLAG_BREAKDOWN : FLAG_RUN);
    });
}

// restart: rh = r, p = v = 0
template <class V>
__global__ void k_restart_dirs(const V *r, V *rh, V *p, V *v, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        rh[i] = r[i]; p[i] = 0; v[i] = 0;
    }
}

// Solves M x = b for the FP64 x (initial guess in x) with FP32 Krylov
// vectors; yd is FP64 scratch.  *updates counts the reliable updates.
template <class Real>
static int bicgstab_reliable(Ctx<Real> &c, double *x, const double *b, double *yd, double bnorm2, double tol,
                             int maxit, bool cached, int *iters, double *relres, int *updates, int *restarts) {
    const int n = c.n;
    cudaStream_t st = c.stream;
    float *const *ws = (float *const *)c.kv;
    float *r = ws[0], *rh = ws[1], *p = ws[2], *v = ws[3], *s = ws[4];
    float *t = ws[5], *ph = ws[6], *sh = ws[7], *dinv = ws[8];
    float *xlo = c.xf;
    const int G = red_grid(n);
    unsigned int *counter = (unsigned int *)(c.scal + 32);
    const double tol2 = tol * tol * bnorm2;
    const bool trace = getenv("SPH_TRACE_PPE") != nullptr;
    k_dinv<float, Real><<<grid_for(n, 256), 256, 0, st>>>(c.row_kind, c.diag, dinv, n);
    SPH_CUDA_TRY(cudaMemsetAsync(xlo, 0, sizeof(float) * n, st));
    SPH_CUDA_TRY(cudaMemsetAsync(c.scal + SC_ITN, 0, sizeof(double), st));
    ++c.launches;
    *restarts = 0;
    *updates = 0;
    int it = 0;
    auto read_scal = [&]() -> int {
        SPH_CUDA_TRY(cudaMemcpyAsync(c.red_host, c.scal, sizeof(double) * SC_COUNT, cudaMemcpyDeviceToHost, st));
        SPH_CUDA_TRY(cudaStreamSynchronize(st));
        return SPH_OK;
    };
    // x += x_lo; r = b - M x (FP64), replacing the recurrence residual
    auto replace = [&]() {
        k_axpy_cast<float, double><<<grid_for(n, 256), 256, 0, st>>>(xlo, x, n);
        apply_op<Real, double>(c, x, yd, cached);
        k_reliable_replace<float><<<G, 256, 0, st>>>(b, yd, r, xlo, rh, n, c.red, counter, c.scal);
        c.launches += 2;
    };
    // fresh start from the true residual
    auto restart = [&]() -> int {
        replace();
        k_restart_dirs<float><<<G, 256, 0, st>>>(r, rh, p, v, n);
        k_norm2<float><<<G, 256, 0, st>>>(r, n, c.red, counter, c.scal, SC_RHO_NEW);
        c.launches += 2;
        SPH_TRY(read_scal());
        k_set_scal<<<1, 1, 0, st>>>(c.scal, c.red_host[SC_RHO_NEW], tol2);
        ++c.launches;
        return SPH_OK;
    };
    int status = SPH_NOT_CONVERGED;
    SPH_TRY(restart());
    double rr = c.red_host[SC_RR];
    double maxrr = rr;
    *relres = std::sqrt(rr / bnorm2);
    if (c.init_relres < 0) c.init_relres = *relres;
    if (trace) fprintf(stderr, "RU start relres %.3e\n", *relres);
    if (rr <= tol2) status = SPH_OK;
    const int check = 4;
    auto iteration = [&]() {
        k_p_update<float><<<G, 256, 0, st>>>(p, ph, r, v, dinv, n, c.scal);
        bool mr = precond_coarse<Real, float>(c, p, ph, v, cached);
        apply_op<Real, float>(c, ph, v, cached, mr);
        k_alpha<float><<<G, 256, 0, st>>>(rh, v, n, c.red, counter, c.scal);
        k_s_update<float><<<G, 256, 0, st>>>(r, v, s, sh, dinv, n, c.scal);
        mr = precond_coarse<Real, float>(c, s, sh, t, cached);
        apply_op<Real, float>(c, sh, t, cached, mr);
        k_omega<float><<<G, 256, 0, st>>>(t, s, n, c.red, counter, c.scal);
        k_xr_update<float><<<G, 256, 0, st>>>(xlo, r, ph, sh, s, t, rh, n, c.red, counter, c.scal);
        c.launches += 5;
    };
    // `check` iterations as one graph launch; false: run them one launch at a time
    auto graph_chunk = [&]() -> bool {
        if (c.kgraph_off || st == nullptr || !cached) return false;
        auto *g = (KrylovGraph *)c.kgraph;
        if (!g) { g = new KrylovGraph(); c.kgraph = g; }
        std::vector<uintptr_t> key = krylov_graph_key(c, ws, xlo);
        if (!g->exec || g->key != key) {
            if (g->exec) { cudaGraphExecDestroy(g->exec); g->exec = nullptr; }
            if (c.prof && g->ev.empty()) {
                g->ev.resize(4 * check);   // two applications per iteration
                for (auto &e : g->ev) cudaEventCreate(&e);
            }
            const long long l0 = c.launches;
            cudaGraph_t graph = nullptr;
            if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
                cudaGetLastError();
                c.kgraph_off = true;
                return false;
            }
            if (c.prof) { c.cap_ev = g->ev.data(); c.cap_n = 0; c.cap_max = 2 * check; }
            for (int q = 0; q < check; ++q) iteration();
            g->n_timed = c.prof ? c.cap_n : 0;
            c.cap_ev = nullptr;
            c.cap_n = c.cap_max = 0;
            const cudaError_t e1 = cudaStreamEndCapture(st, &graph);
            const cudaError_t e2 = e1 == cudaSuccess ? cudaGraphInstantiate(&g->exec, graph, 0) : e1;
            if (graph) cudaGraphDestroy(graph);
            g->nodes = c.launches - l0;
            c.launches = l0;
            if (e2 != cudaSuccess) {
                cudaGetLastError();
                g->exec = nullptr;
                c.kgraph_off = true;
                return false;
            }
            g->key = key;
        }
        if (cudaGraphLaunch(g->exec, st) != cudaSuccess) {
            cudaGetLastError();
            c.kgraph_off = true;
            return false;
        }
        c.launches += g->nodes;
        if (g->n_timed > 0) {
            // operator times of this replay (the host waits for the chunk's
            // scalars right after it anyway)
            prof_drain(c);
            cudaEventSynchronize(g->ev[2 * g->n_timed - 1]);
            for (int k = 0; k < g->n_timed; ++k) {
                float ms = 0;
                if (cudaEventElapsedTime(&ms, g->ev[2 * k], g->ev[2 * k + 1]) != cudaSuccess) {
                    cudaGetLastError();
                    continue;
                }
                c.prof_ms += ms;
                ++c.prof_launches;
            }
        }
        return true;
    };
    while (status != SPH_OK && it < maxit) {
        if (it % check == 0 && it + check <= maxit && graph_chunk()) {
            it += check;
        } else {
            iteration();
            ++it;
        }
        if (it % check != 0 && it < maxit) continue;
        SPH_TRY(read_scal());
        const double flag = c.red_host[SC_FLAG];
        rr = c.red_host[SC_RR];
        if (flag == FLAG_BREAKDOWN || !std::isfinite(rr)) {
            if (++*restarts > 20) { status = SPH_ERR_BREAKDOWN; break; }
            SPH_TRY(restart());
            ++*updates;
        } else if (flag == FLAG_CONVERGED || rr < RELIABLE_DELTA * RELIABLE_DELTA * maxrr || it >= maxit) {
            replace();
            SPH_TRY(read_scal());
            ++*updates;
            if (trace)
                fprintf(stderr, "  reliable update %d at it %d: recurrence %.3e true %.3e\n", *updates, it,
                        std::sqrt(rr / bnorm2), std::sqrt(c.red_host[SC_RR] / bnorm2));
            if (c.red_host[SC_FLAG] == FLAG_BREAKDOWN) {
                if (++*restarts > 20) { status = SPH_ERR_BREAKDOWN; break; }
                SPH_TRY(restart());
            }
        } else {
            maxrr = std::max(maxrr, rr);
            continue;
        }
        rr = c.red_host[SC_RR];
        maxrr = rr;
        *relres = std::sqrt(rr / bnorm2);
        if (rr <= tol2) status = SPH_OK;
    }
    if (status != SPH_OK && it > 0 && *updates == 0) *relres = std::sqrt(rr / bnorm2);
    SPH_CUDA_TRY(cudaGetLastError());
    *iters = it > 0 ? (int)c.red_host[SC_ITN] : 0;   // exact, not rounded up to the check interval
    return status;
}

// ---------------------------------------------------------------------------
// The same mixed BiCGSTAB with FP64 reliable updates, its control on the
// device (ppe_refinement = 4): one CUDA graph per solve, whose conditional
// WHILE node runs `check` iterations and then k_dev_decide, the host loop's
// decision as a kernel; conditional IF nodes run the reliable update
// (replace) and the restart.  The host launches the graph and reads nothing
// until the statistics are wanted, so steps follow one another on the stream
// without host round trips.  The kernels and their order are those of
// bicgstab_reliable, so the two give the same iterates.
// Termination: every trip of the loop counts SC_TRIPS, and the loop ends
// after maxit / check + 64 trips whatever the scalars say.
// ---------------------------------------------------------------------------
enum {
    SC_MAXRR = SC_COUNT, SC_MAXIT, SC_UPDATES, SC_RESTARTS, SC_TRIPS, SC_TRIPCAP, SC_STATUS, SC_RELRES, SC_BN2,
    SC_INITREL, SC_CONT, SC_DEV_END
};
static_assert(SC_DEV_END <= 32, "device scalars of the device-controlled solve overlap the reduction counter");

__global__ void k_dev_tol(double *scal, double tol, int maxit, int check) {
    double bb = scal[SC_BB];
    if (!(bb > 0)) bb = 1.0;
    scal[SC_BN2] = bb;
    scal[SC_TOL2] = tol * tol * bb;
    scal[SC_MAXIT] = maxit;
    scal[SC_ITN] = 0;
    scal[SC_UPDATES] = 0;
    scal[SC_RESTARTS] = 0;
    scal[SC_TRIPS] = 0;
    scal[SC_TRIPCAP] = maxit / check + 64;
    scal[SC_STATUS] = SPH_NOT_CONVERGED;
    scal[SC_CONT] = 0;
}

// k_set_scal with the rho of the restart's residual, read on the device
__global__ void k_dev_set_scal(double *scal) {
    scal[SC_RHO] = scal[SC_RHO_NEW]; scal[SC_ALPHA] = 1; scal[SC_OMEGA] = 1; scal[SC_BETA] = 0;
    scal[SC_FLAG] = FLAG_RUN;
}

// after a reliable update or a restart: the host loop's bookkeeping
__device__ void dev_finalize(double *scal) {
    const double rr = scal[SC_RR];
    scal[SC_MAXRR] = rr;
    scal[SC_RELRES] = sqrt(rr / scal[SC_BN2]);
    if (rr <= scal[SC_TOL2]) { scal[SC_STATUS] = SPH_OK; scal[SC_CONT] = 0; }
    else scal[SC_CONT] = scal[SC_ITN] < scal[SC_MAXIT] ? 1 : 0;
}

// after the first restart: start residual, and whether to iterate at all
__global__ void k_dev_start(double *scal, cudaGraphConditionalHandle h_loop) {
    dev_finalize(scal);
    scal[SC_INITREL] = scal[SC_RELRES];
    cudaGraphSetConditional(h_loop, scal[SC_CONT] != 0 ? 1u : 0u);
}

// after `check` iterations: restart on a breakdown, reliable update on
// convergence of the recurrence, on a 10x drop or at maxit, else go on
__global__ void k_dev_decide(double *scal, cudaGraphConditionalHandle h_rep, cudaGraphConditionalHandle h_res) {
    const double trips = scal[SC_TRIPS] + 1;
    scal[SC_TRIPS] = trips;
    unsigned rep = 0, res = 0;
    const double flag = scal[SC_FLAG], rr = scal[SC_RR];
    if (trips > scal[SC_TRIPCAP]) {
        scal[SC_CONT] = 0;
    } else if (flag == FLAG_BREAKDOWN || !isfinite(rr)) {
        scal[SC_RESTARTS] += 1;
        if (scal[SC_RESTARTS] > 20) { scal[SC_STATUS] = SPH_ERR_BREAKDOWN; scal[SC_CONT] = 0; }
        else { res = 1; scal[SC_UPDATES] += 1; }
    } else if (flag == FLAG_CONVERGED || rr < RELIABLE_DELTA * RELIABLE_DELTA * scal[SC_MAXRR] ||
               scal[SC_ITN] >= scal[SC_MAXIT]) {
        rep = 1;
        scal[SC_UPDATES] += 1;
    } else {
        scal[SC_MAXRR] = fmax(scal[SC_MAXRR], rr);
        scal[SC_CONT] = 1;
    }
    cudaGraphSetConditional(h_rep, rep);
    cudaGraphSetConditional(h_res, res);
}

// inside the reliable-update branch: a breakdown of the replaced residual
// asks for a restart, else the bookkeeping
__global__ void k_dev_after_replace(double *scal, cudaGraphConditionalHandle h_res) {
    if (scal[SC_FLAG] == FLAG_BREAKDOWN) {
        scal[SC_RESTARTS] += 1;
        if (scal[SC_RESTARTS] > 20) {
            scal[SC_STATUS] = SPH_ERR_BREAKDOWN;
            scal[SC_CONT] = 0;
            cudaGraphSetConditional(h_res, 0u);
        } else {
            cudaGraphSetConditional(h_res, 1u);
        }
        return;
    }
    dev_finalize(scal);
}

__global__ void k_dev_after_restart(double *scal) { dev_finalize(scal); }

__global__ void k_dev_tail(const double *scal, cudaGraphConditionalHandle h_loop) {
    cudaGraphSetConditional(h_loop, scal[SC_CONT] != 0 ? 1u : 0u);
}

struct DevLoopGraph {
    cudaGraphExec_t exec = nullptr;
    std::vector<uintptr_t> key;
    cudaStream_t s2 = nullptr, s3 = nullptr;   // capture streams of the loop body and its branches
    ~DevLoopGraph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (s2) cudaStreamDestroy(s2);
        if (s3) cudaStreamDestroy(s3);
    }
};

// adds a conditional node at the capture position of `st` and returns its body graph
static int add_conditional(cudaStream_t st, cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type,
                           cudaGraph_t *body) {
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    SPH_CUDA_TRY(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd));
    if (cs != cudaStreamCaptureStatusActive) { set_error("device-controlled solve: stream not capturing"); return SPH_ERR_CUDA; }
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = type;
    np.conditional.size = 1;
    cudaGraphNode_t node = nullptr;
    SPH_CUDA_TRY(cudaGraphAddNode(&node, g, deps, nd, &np));
    *body = np.conditional.phGraph_out[0];
    SPH_CUDA_TRY(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
    return SPH_OK;
}

// Appends the solve of M x = b, as bicgstab_reliable does it, for the FP64 x
// (initial guess in x, b_norm2 in scal[SC_BB]) with FP32 Krylov vectors and
// the cached operator, under device control, to the graph that `st` is
// capturing: its start, then the WHILE node, whose body and branches are
// captured on the loop graph's own streams.  The statistics stay in the
// device scalars (dev_solve_stats reads them).
template <class Real>
static int append_solve(Ctx<Real> &c, DevLoopGraph *g, cudaStream_t st, double *x, const double *b, double *yd,
                        double tol, int maxit) {
    const int n = c.n;
    float *const *ws = (float *const *)c.kv;
    float *r = ws[0], *rh = ws[1], *p = ws[2], *v = ws[3], *s = ws[4];
    float *t = ws[5], *ph = ws[6], *sh = ws[7], *dinv = ws[8];
    float *xlo = c.xf;
    const int G = red_grid(n);
    unsigned int *counter = (unsigned int *)(c.scal + 32);
    const int check = 4;
    auto replace = [&]() {
        k_axpy_cast<float, double><<<grid_for(n, 256), 256, 0, c.stream>>>(xlo, x, n);
        apply_op<Real, double>(c, x, yd, true);
        k_reliable_replace<float><<<G, 256, 0, c.stream>>>(b, yd, r, xlo, rh, n, c.red, counter, c.scal);
    };
    auto restart = [&]() {
        replace();
        k_restart_dirs<float><<<G, 256, 0, c.stream>>>(r, rh, p, v, n);
        k_norm2<float><<<G, 256, 0, c.stream>>>(r, n, c.red, counter, c.scal, SC_RHO_NEW);
        k_dev_set_scal<<<1, 1, 0, c.stream>>>(c.scal);
    };
    auto iteration = [&]() {
        k_p_update<float><<<G, 256, 0, c.stream>>>(p, ph, r, v, dinv, n, c.scal);
        bool mr = precond_coarse<Real, float>(c, p, ph, v, true);
        apply_op<Real, float>(c, ph, v, true, mr);
        k_alpha<float><<<G, 256, 0, c.stream>>>(rh, v, n, c.red, counter, c.scal);
        k_s_update<float><<<G, 256, 0, c.stream>>>(r, v, s, sh, dinv, n, c.scal);
        mr = precond_coarse<Real, float>(c, s, sh, t, true);
        apply_op<Real, float>(c, sh, t, true, mr);
        k_omega<float><<<G, 256, 0, c.stream>>>(t, s, n, c.red, counter, c.scal);
        k_xr_update<float><<<G, 256, 0, c.stream>>>(xlo, r, ph, sh, s, t, rh, n, c.red, counter, c.scal);
    };
    cudaStreamCaptureStatus cs;
    cudaGraph_t graph = nullptr;
    SPH_CUDA_TRY(cudaStreamGetCaptureInfo(st, &cs, nullptr, &graph, nullptr, nullptr));
    if (cs != cudaStreamCaptureStatusActive || !graph) { set_error("device-controlled solve: stream not capturing"); return SPH_ERR_CUDA; }
    cudaGraphConditionalHandle h_loop, h_rep, h_res;
    cudaGraph_t body = nullptr, body_rep = nullptr, body_res = nullptr;
    SPH_CUDA_TRY(cudaGraphConditionalHandleCreate(&h_loop, graph, 0, cudaGraphCondAssignDefault));
    const cudaStream_t outer = c.stream;
    c.stream = st;
    // the solve's start: the restart of bicgstab_reliable, then the loop
    k_dev_tol<<<1, 1, 0, st>>>(c.scal, tol, maxit, check);
    k_dinv<float, Real><<<grid_for(n, 256), 256, 0, st>>>(c.row_kind, c.diag, dinv, n);
    cudaMemsetAsync(xlo, 0, sizeof(float) * n, st);
    restart();
    k_dev_start<<<1, 1, 0, st>>>(c.scal, h_loop);
    int err = add_conditional(st, h_loop, cudaGraphCondTypeWhile, &body);
    // the loop body on s2, its two branches on s3
    if (err == SPH_OK && (cudaGraphConditionalHandleCreate(&h_rep, body, 0, cudaGraphCondAssignDefault) != cudaSuccess ||
                          cudaGraphConditionalHandleCreate(&h_res, body, 0, cudaGraphCondAssignDefault) != cudaSuccess))
        err = SPH_ERR_CUDA;
    if (err == SPH_OK) {
        c.stream = g->s2;
        if (cudaStreamBeginCaptureToGraph(g->s2, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            for (int q = 0; q < check; ++q) iteration();
            k_dev_decide<<<1, 1, 0, g->s2>>>(c.scal, h_rep, h_res);
            err = add_conditional(g->s2, h_rep, cudaGraphCondTypeIf, &body_rep);
            if (err == SPH_OK) err = add_conditional(g->s2, h_res, cudaGraphCondTypeIf, &body_res);
            if (err == SPH_OK) k_dev_tail<<<1, 1, 0, g->s2>>>(c.scal, h_loop);
            cudaGraph_t done = nullptr;
            if (cudaStreamEndCapture(g->s2, &done) != cudaSuccess && err == SPH_OK) err = SPH_ERR_CUDA;
        } else {
            err = SPH_ERR_CUDA;
        }
    }
    // the reliable update, then the restart branch
    if (err == SPH_OK) {
        c.stream = g->s3;
        bool ok = cudaStreamBeginCaptureToGraph(g->s3, body_rep, nullptr, nullptr, 0,
                                                cudaStreamCaptureModeThreadLocal) == cudaSuccess;
        if (ok) {
            replace();
            k_dev_after_replace<<<1, 1, 0, g->s3>>>(c.scal, h_res);
            cudaGraph_t done = nullptr;
            ok = cudaStreamEndCapture(g->s3, &done) == cudaSuccess;
        }
        if (ok) ok = cudaStreamBeginCaptureToGraph(g->s3, body_res, nullptr, nullptr, 0,
                                                   cudaStreamCaptureModeThreadLocal) == cudaSuccess;
        if (ok) {
            restart();
            k_dev_after_restart<<<1, 1, 0, g->s3>>>(c.scal);
            cudaGraph_t done = nullptr;
            ok = cudaStreamEndCapture(g->s3, &done) == cudaSuccess;
        }
        if (!ok) err = SPH_ERR_CUDA;
    }
    c.stream = outer;
    return err;
}

template <class Real>
static DevLoopGraph *devloop_graph(Ctx<Real> &c) {
    auto *g = (DevLoopGraph *)c.devloop;
    if (!g) {
        g = new DevLoopGraph();
        c.devloop = g;
        if (cudaStreamCreateWithFlags(&g->s2, cudaStreamNonBlocking) != cudaSuccess ||
            cudaStreamCreateWithFlags(&g->s3, cudaStreamNonBlocking) != cudaSuccess) {
            set_error("device-controlled solve: stream creation failed");
            return nullptr;
        }
    }
    return g;
}

// The solve as its own graph (launched on the context's stream), or, while a
// whole step is captured, appended to the step's graph.
template <class Real>
static int bicgstab_device(Ctx<Real> &c, double *x, const double *b, double *yd, double tol, int maxit) {
    cudaStream_t st = c.stream;
    DevLoopGraph *g = devloop_graph(c);
    if (!g) return SPH_ERR_CUDA;
    if (c.capturing) {
        const long long l0 = c.launches;
        SPH_TRY(append_solve(c, g, st, x, b, yd, tol, maxit));
        c.launches = l0 + 1;   // counted as one launch, as the solve's own graph is
        return SPH_OK;
    }
    std::vector<uintptr_t> key = krylov_graph_key(c, (float *const *)c.kv, c.xf);
    const uintptr_t extra[] = {(uintptr_t)x, (uintptr_t)b, (uintptr_t)yd, (uintptr_t)maxit, (uintptr_t)c.coef_h,
                               (uintptr_t)c.coef_rs, (uintptr_t)(c.prm.ppe_coef_half && c.coef_h_valid),
                               (uintptr_t)c.nm_ow, (uintptr_t)c.coef};
    for (uintptr_t q : extra) key.push_back(q);
    uint64_t tb;
    memcpy(&tb, &tol, sizeof tb);
    key.push_back((uintptr_t)tb);
    if (!g->exec || g->key != key) {
        if (g->exec) { cudaGraphExecDestroy(g->exec); g->exec = nullptr; }
        const long long l0 = c.launches;
        cudaGraph_t graph = nullptr;
        int err = SPH_OK;
        const bool prof = c.prof;
        c.prof = false;   // event-record nodes are not allowed in conditional bodies
        do {
            if (cudaGraphCreate(&graph, 0) != cudaSuccess) { err = SPH_ERR_CUDA; break; }
            if (cudaStreamBeginCaptureToGraph(st, graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) !=
                cudaSuccess) { err = SPH_ERR_CUDA; break; }
            err = append_solve(c, g, st, x, b, yd, tol, maxit);
            cudaGraph_t done = nullptr;
            const cudaError_t e1 = cudaStreamEndCapture(st, &done);
            if (err != SPH_OK || e1 != cudaSuccess) { if (err == SPH_OK) err = SPH_ERR_CUDA; break; }
            if (cudaGraphInstantiate(&g->exec, graph, 0) != cudaSuccess) { g->exec = nullptr; err = SPH_ERR_CUDA; break; }
            g->key = key;
        } while (0);
        c.prof = prof;
        c.stream = st;
        c.launches = l0;
        if (graph) cudaGraphDestroy(graph);
        if (err != SPH_OK || !g->exec) {
            const cudaError_t e = cudaGetLastError();
            static thread_local std::string msg;
            msg = std::string("device-controlled solve: graph construction failed: ") + cudaGetErrorString(e);
            set_error(msg.c_str());
            return SPH_ERR_CUDA;
        }
    }
    SPH_CUDA_TRY(cudaGraphLaunch(g->exec, st));
    ++c.launches;
    return SPH_OK;
}

// worst status of the device-controlled solves since the last reset
// (scal[48]: most negative error, scal[49]: 1 when a solve did not converge)
__global__ void k_dev_record(double *scal) {
    const double stt = scal[SC_STATUS];
    if (stt < 0) scal[48] = fmin(scal[48], stt);
    else if (stt > 0) scal[49] = 1;
}

// statistics of the last device-controlled solve (synchronises the stream)
template <class Real>
int dev_solve_stats(Ctx<Real> &c, sph_ppe_stats *S, int *worst) {
    double h[64];
    SPH_CUDA_TRY(cudaMemcpyAsync(h, c.scal, sizeof(double) * 64, cudaMemcpyDeviceToHost, c.stream));
    SPH_CUDA_TRY(cudaStreamSynchronize(c.stream));
    S->status = (int)h[SC_STATUS];
    S->iterations = (int)h[SC_ITN];
    S->refinements = (int)h[SC_UPDATES];
    S->restarts = (int)h[SC_RESTARTS];
    S->rel_residual = h[SC_RELRES];
    S->initial_residual = h[SC_INITREL];
    float ms = 0;
    cudaEventElapsedTime(&ms, c.ev[4], c.ev[5]);
    S->solve_ms = ms;
    c.last_ppe = *S;
    c.ppe_pending = false;
    if (worst) *worst = h[48] < 0 ? (int)h[48] : (h[49] > 0 ? SPH_NOT_CONVERGED : SPH_OK);
    return SPH_OK;
}

__global__ void k_dev_reset_worst(double *scal) { scal[48] = 0; scal[49] = 0; }

template <class Real>
int dev_reset_worst(Ctx<Real> &c) {
    if (!c.scal) return SPH_OK;
    k_dev_reset_worst<<<1, 1, 0, c.stream>>>(c.scal);
    ++c.launches;
    SPH_CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}

// ---------------------------------------------------------------------------
// IDR(s), the biorthogonal variant of van Gijzen & Sonneveld ("Algorithm
// 913: an elegant IDR(s) variant that efficiently exploits
// bi-orthogonality properties", ACM TOMS 38, 2011), right preconditioned
// with the Jacobi / two-level preconditioner, s = 4.  One operator
// application per step and s + 1 per cycle; the shadow space P is s
// orthonormalised seeded random vectors.  The small s x s lower-triangular
// system, the step scalars and the convergence flag live on the device
// (IdrWs::sc); the host reads the residual once per cycle.
// ---------------------------------------------------------------------------
#define IDR_S 4
enum { IS_M = 0, IS_F = IDR_S * IDR_S, IS_C = IS_F + IDR_S, IS_OM = IS_C + IDR_S, IS_RR, IS_FLAG, IS_TOL2, IS_COUNT };

template <class V>
struct IdrWs {
    V *P = nullptr, *G = nullptr, *U = nullptr;   // s columns of n each
    V *r = nullptr, *v = nullptr, *z = nullptr, *t = nullptr, *tmp = nullptr, *dinv = nullptr;
    double *sc = nullptr;
};

// c[k..s) from M[k..s, k..s) c = f[k..s) (lower triangular)
__global__ void k_idr_c(double *sc, int k) {
    if (threadIdx.x || blockIdx.x || sc[IS_FLAG] != 0) return;
    const double *M = sc + IS_M, *f = sc + IS_F;
    double *cc = sc + IS_C;
    for (int i = k; i < IDR_S; ++i) {
        double t = f[i];
        for (int j = k; j < i; ++j) t -= M[i * IDR_S + j] * cc[j];
        cc[i] = t / M[i * IDR_S + i];
    }
}

// v = r - sum_{j >= k} c_j G_j ; z = dinv v
template <class V>
__global__ void k_idr_v(const V *r, const V *G, const V *dinv, const double *sc, int k, V *v, V *z, int n) {
    if (sc[IS_FLAG] != 0) return;
    V cc[IDR_S];
#pragma unroll
    for (int j = 0; j < IDR_S; ++j) cc[j] = (V)sc[IS_C + j];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        V a = r[i];
#pragma unroll
        for (int j = 0; j < IDR_S; ++j)
            if (j >= k) a -= cc[j] * G[(size_t)j * n + i];
        v[i] = a;
        z[i] = dinv[i] * a;
    }
}

// U_k = sum_{j >= k} c_j U_j + om z
template <class V>
__global__ void k_idr_u(V *U, const V *z, const double *sc, int k, int n) {
    if (sc[IS_FLAG] != 0) return;
    V cc[IDR_S];
#pragma unroll
    for (int j = 0; j < IDR_S; ++j) cc[j] = (V)sc[IS_C + j];
    const V om = (V)sc[IS_OM];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        V a = om * z[i];
#pragma unroll
        for (int j = 0; j < IDR_S; ++j)
            if (j >= k) a += cc[j] * U[(size_t)j * n + i];
        U[(size_t)k * n + i] = a;
    }
}

// alpha = (P_i, G_k) / M_ii, then G_k -= alpha G_i, U_k -= alpha U_i (two kernels)
template <class V>
__global__ void k_idr_alpha(const V *Pi, const V *Gk, int i, int n, double *partials, unsigned int *counter,
                            double *sc, double *out) {
    if (sc[IS_FLAG] != 0) return;
    double d[1] = {0};
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) d[0] += (double)Pi[q] * (double)Gk[q];
    reduce_finish<1>(d, partials, counter, [&](double *t) { *out = t[0] / sc[IS_M + i * IDR_S + i]; });
}

template <class V>
__global__ void k_idr_axpy2(V *Gk, const V *Gi, V *Uk, const V *Ui, const double *sc, const double *alpha, int n) {
    if (sc[IS_FLAG] != 0) return;
    const V a = (V)*alpha;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        Gk[q] -= a * Gi[q];
        Uk[q] -= a * Ui[q];
    }
}

// M[j][k] = (P_j, G_k) for j >= k
template <class V>
__global__ void k_idr_mcol(const V *P, const V *Gk, int k, int n, double *partials, unsigned int *counter, double *sc) {
    if (sc[IS_FLAG] != 0) return;
    double d[IDR_S];
#pragma unroll
    for (int j = 0; j < IDR_S; ++j) d[j] = 0;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const double g = (double)Gk[q];
#pragma unroll
        for (int j = 0; j < IDR_S; ++j)
            if (j >= k) d[j] += (double)P[(size_t)j * n + q] * g;
    }
    reduce_finish<IDR_S>(d, partials, counter, [&](double *t) {
        for (int j = k; j < IDR_S; ++j) sc[IS_M + j * IDR_S + k] = t[j];
    });
}

// beta = f_k / M_kk ; r -= beta G_k ; x += beta U_k ; then f_j -= beta M_jk (j > k),
// rr = (r, r) and the convergence / breakdown flag
template <class V>
__global__ void k_idr_step(V *r, V *x, const V *Gk, const V *Uk, int k, int n, double *partials, unsigned int *counter,
                           double *sc) {
    if (sc[IS_FLAG] != 0) return;
    const double mkk = sc[IS_M + k * IDR_S + k];
    const double beta = mkk != 0 ? sc[IS_F + k] / mkk : 0.0;
    const V bv = (V)beta;
    double d[1] = {0};
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const V rq = r[q] - bv * Gk[q];
        r[q] = rq;
        x[q] += bv * Uk[q];
        d[0] += (double)rq * (double)rq;
    }
    reduce_finish<1>(d, partials, counter, [&](double *t) {
        for (int j = k + 1; j < IDR_S; ++j) sc[IS_F + j] -= beta * sc[IS_M + j * IDR_S + k];
        sc[IS_RR] = t[0];
        if (mkk == 0.0 || !isfinite(t[0])) sc[IS_FLAG] = 2;
        else if (t[0] <= sc[IS_TOL2]) sc[IS_FLAG] = 1;
    });
}

// om = (t, r) / (t, t), enlarged to keep |cos(t, r)| >= 0.7
template <class V>
__global__ void k_idr_om(const V *t, const V *r, int n, double *partials, unsigned int *counter, double *sc) {
    if (sc[IS_FLAG] != 0) return;
    double d[2] = {0, 0};
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        d[0] += (double)t[q] * (double)r[q];
        d[1] += (double)t[q] * (double)t[q];
    }
    reduce_finish<2>(d, partials, counter, [&](double *tt) {
        if (!(tt[1] > 0)) { sc[IS_FLAG] = 2; return; }
        double om = tt[0] / tt[1];
        const double rho = fabs(tt[0]) / (sqrt(tt[1]) * sqrt(sc[IS_RR]));
        if (rho < 0.7 && rho > 0) om *= 0.7 / rho;
        sc[IS_OM] = om;
    });
}

// x += om z ; r -= om t ; rr ; flag
template <class V>
__global__ void k_idr_xr(V *x, V *r, const V *z, const V *t, int n, double *partials, unsigned int *counter, double *sc) {
    if (sc[IS_FLAG] != 0) return;
    const V om = (V)sc[IS_OM];
    double d[1] = {0};
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        x[q] += om * z[q];
        const V rq = r[q] - om * t[q];
        r[q] = rq;
        d[0] += (double)rq * (double)rq;
    }
    reduce_finish<1>(d, partials, counter, [&](double *tt) {
        sc[IS_RR] = tt[0];
        if (!isfinite(tt[0])) sc[IS_FLAG] = 2;
        else if (tt[0] <= sc[IS_TOL2]) sc[IS_FLAG] = 1;
    });
}

// f = P^T r
template <class V>
__global__ void k_idr_f(const V *P, const V *r, int n, double *partials, unsigned int *counter, double *sc) {
    if (sc[IS_FLAG] != 0) return;
    double d[IDR_S];
#pragma unroll
    for (int j = 0; j < IDR_S; ++j) d[j] = 0;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const double rq = (double)r[q];
#pragma unroll
        for (int j = 0; j < IDR_S; ++j) d[j] += (double)P[(size_t)j * n + q] * rq;
    }
    reduce_finish<IDR_S>(d, partials, counter, [&](double *t) {
        for (int j = 0; j < IDR_S; ++j) sc[IS_F + j] = t[j];
    });
}

// z = d * r
template <class V>
__global__ void k_mul(const V *d, const V *r, V *z, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) z[i] = d[i] * r[i];
}

// r = b - y
template <class V>
__global__ void k_idr_res(const V *b, const V *y, V *r, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) r[i] = b[i] - y[i];
}

// sc: M = I, om = 1, flag 0, tol2
__global__ void k_idr_init(double *sc, double tol2) {
    if (threadIdx.x || blockIdx.x) return;
    for (int q = 0; q < IS_COUNT; ++q) sc[q] = 0;
    for (int j = 0; j < IDR_S; ++j) sc[IS_M + j * IDR_S + j] = 1;
    sc[IS_OM] = 1;
    sc[IS_TOL2] = tol2;
}

template <class Real, class V>
static int idr_ws(Ctx<Real> &c, IdrWs<V> &w) {
    const size_t n = (size_t)c.n;
    SPH_TRY(c.alloc(w.P, IDR_S * n)); SPH_TRY(c.alloc(w.G, IDR_S * n)); SPH_TRY(c.alloc(w.U, IDR_S * n));
    SPH_TRY(c.alloc(w.r, n)); SPH_TRY(c.alloc(w.v, n)); SPH_TRY(c.alloc(w.z, n)); SPH_TRY(c.alloc(w.t, n));
    SPH_TRY(c.alloc(w.tmp, n)); SPH_TRY(c.alloc(w.dinv, n)); SPH_TRY(c.alloc(w.sc, 64));
    // shadow space: s seeded random vectors, orthonormalised (modified
    // Gram-Schmidt in FP64 on the host)
    std::vector<double> Ph(IDR_S * n);
    unsigned long long st = 0x9E3779B97F4A7C15ULL;
    for (size_t q = 0; q < Ph.size(); ++q) {
        st ^= st << 13; st ^= st >> 7; st ^= st << 17;   // xorshift64
        Ph[q] = ((double)(st >> 11) * (1.0 / 9007199254740992.0)) - 0.5;
    }
    for (int j = 0; j < IDR_S; ++j) {
        double *pj = Ph.data() + (size_t)j * n;
        for (int i = 0; i < j; ++i) {
            const double *pi = Ph.data() + (size_t)i * n;
            double d = 0;
            for (size_t q = 0; q < n; ++q) d += pi[q] * pj[q];
            for (size_t q = 0; q < n; ++q) pj[q] -= d * pi[q];
        }
        double nn = 0;
        for (size_t q = 0; q < n; ++q) nn += pj[q] * pj[q];
        nn = 1.0 / std::sqrt(nn);
        for (size_t q = 0; q < n; ++q) pj[q] *= nn;
    }
    std::vector<V> Pv(Ph.begin(), Ph.end());
    SPH_CUDA_TRY(cudaMemcpyAsync(w.P, Pv.data(), sizeof(V) * Pv.size(), cudaMemcpyHostToDevice, c.stream));
    SPH_CUDA_TRY(cudaStreamSynchronize(c.stream));
    return SPH_OK;
}

// IDR(s) on M x = b; x holds the initial guess.  iters counts operator
// applications.  Returns SPH_OK, SPH_NOT_CONVERGED or SPH_ERR_BREAKDOWN.
template <class Real, class V>
static int idrs(Ctx<Real> &c, IdrWs<V> &w, V *x, const V *b, double bnorm2, double tol, int maxit, bool cached,
                int *iters, double *relres) {
    const int n = c.n;
    cudaStream_t st = c.stream;
    const int G = red_grid(n);
    unsigned int *counter = (unsigned int *)(c.scal + 32);
    const double tol2 = tol * tol * bnorm2;
    double *alpha = w.sc + IS_COUNT;
    k_dinv<V, Real><<<grid_for(n, 256), 256, 0, st>>>(c.row_kind, c.diag, w.dinv, n);
    ++c.launches;
    int mv = 0, restarts = 0, status = SPH_NOT_CONVERGED;
    *relres = 1;
    while (true) {
        // (re)start: r = b - M x, M = I, G = U = 0, om = 1, f = P^T r
        apply_op<Real, V>(c, x, w.t, cached);
        k_idr_res<V><<<G, 256, 0, st>>>(b, w.t, w.r, n);
        k_idr_init<<<1, 1, 0, st>>>(w.sc, tol2);
        k_norm2<V><<<G, 256, 0, st>>>(w.r, n, c.red, counter, w.sc, IS_RR);
        SPH_CUDA_TRY(cudaMemsetAsync(w.G, 0, sizeof(V) * IDR_S * (size_t)n, st));
        SPH_CUDA_TRY(cudaMemsetAsync(w.U, 0, sizeof(V) * IDR_S * (size_t)n, st));
        k_idr_f<V><<<G, 256, 0, st>>>(w.P, w.r, n, c.red, counter, w.sc);
        c.launches += 4;
        SPH_CUDA_TRY(cudaMemcpyAsync(c.red_host, w.sc, sizeof(double) * IS_COUNT, cudaMemcpyDeviceToHost, st));
        SPH_CUDA_TRY(cudaStreamSynchronize(st));
        double rr = c.red_host[IS_RR];
        *relres = std::sqrt(rr / bnorm2);
        if (c.init_relres < 0) c.init_relres = *relres;
        if (rr <= tol2) { status = SPH_OK; break; }
        if (mv >= maxit) break;
        bool restart = false;
        while (mv < maxit) {
            for (int k = 0; k < IDR_S; ++k) {
                V *Gk = w.G + (size_t)k * n, *Uk = w.U + (size_t)k * n;
                k_idr_c<<<1, 1, 0, st>>>(w.sc, k);
                k_idr_v<V><<<G, 256, 0, st>>>(w.r, w.G, w.dinv, w.sc, k, w.v, w.z, n);
                c.launches += 2;
                precond_coarse<Real, V>(c, w.v, w.z, w.tmp, cached);
                k_idr_u<V><<<G, 256, 0, st>>>(w.U, w.z, w.sc, k, n);
                ++c.launches;
                apply_op<Real, V>(c, Uk, Gk, cached);
                for (int i = 0; i < k; ++i) {
                    k_idr_alpha<V><<<G, 256, 0, st>>>(w.P + (size_t)i * n, Gk, i, n, c.red, counter, w.sc, alpha);
                    k_idr_axpy2<V><<<G, 256, 0, st>>>(Gk, w.G + (size_t)i * n, Uk, w.U + (size_t)i * n, w.sc, alpha, n);
                    c.launches += 2;
                }
                k_idr_mcol<V><<<G, 256, 0, st>>>(w.P, Gk, k, n, c.red, counter, w.sc);
                k_idr_step<V><<<G, 256, 0, st>>>(w.r, x, Gk, Uk, k, n, c.red, counter, w.sc);
                c.launches += 2;
                ++mv;
            }
            // the (s+1)-th step: z = M^-1 r, t = M z, om, x += om z, r -= om t
            k_mul<V><<<G, 256, 0, st>>>(w.dinv, w.r, w.z, n);
            ++c.launches;
            precond_coarse<Real, V>(c, w.r, w.z, w.tmp, cached);
            apply_op<Real, V>(c, w.z, w.t, cached);
            k_idr_om<V><<<G, 256, 0, st>>>(w.t, w.r, n, c.red, counter, w.sc);
            k_idr_xr<V><<<G, 256, 0, st>>>(x, w.r, w.z, w.t, n, c.red, counter, w.sc);
            k_idr_f<V><<<G, 256, 0, st>>>(w.P, w.r, n, c.red, counter, w.sc);
            c.launches += 3;
            ++mv;
            SPH_CUDA_TRY(cudaMemcpyAsync(c.red_host, w.sc, sizeof(double) * IS_COUNT, cudaMemcpyDeviceToHost, st));
            SPH_CUDA_TRY(cudaStreamSynchronize(st));
            const double flag = c.red_host[IS_FLAG];
            rr = c.red_host[IS_RR];
            *relres = std::sqrt(rr / bnorm2);
            if (flag == 1) { status = SPH_OK; break; }
            if (flag == 2) { restart = true; break; }
        }
        if (status == SPH_OK || !restart || mv >= maxit) break;
        if (++restarts > 20) { status = SPH_ERR_BREAKDOWN; break; }
    }
    SPH_CUDA_TRY(cudaGetLastError());
    *iters = mv;
    return status;
}

// ---------------------------------------------------------------------------
// restarted GMRES(m), right Jacobi preconditioning, classical Gram-Schmidt
// with a conditional second pass, FP64 dot products; the Hessenberg matrix,
// its Givens rotations and the small triangular solve live on the host
// ---------------------------------------------------------------------------
#define GM_MAXV 64

// h[k] = sum_i V_k[i] w[i], k < nv (runtime count up to GM_MAXV), last block
// writes the sums to out[0..nv)
template <class V>
__global__ void __launch_bounds__(256) k_multidot(V *const *basis, const V *w, int nv, int n, double *partials,
                                                  unsigned int *counter, double *out) {
    __shared__ double sh[GM_MAXV][8];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int k = 0; k < nv; ++k) {
        const V *vk = basis[k];
        double s = 0;
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += (double)vk[i] * (double)w[i];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) sh[k][wid] = s;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < nv; k += blockDim.x) {
        double s = 0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) s += sh[k][q];
        partials[(size_t)k * gridDim.x + blockIdx.x] = s;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(counter, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int k = wid; k < nv; k += (blockDim.x >> 5)) {
        double s = 0;
        for (int b = lane; b < (int)gridDim.x; b += 32) s += ((volatile double *)partials)[(size_t)k * gridDim.x + b];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) out[k] = s;
    }
    if (threadIdx.x == 0) *counter = 0;
}

// w -= sum_k h[k] V_k ; returns ||w||^2 (last block) into out[0]
template <class V>
__global__ void __launch_bounds__(256) k_orth_update(V *const *basis, V *w, const double *h, int nv, int n,
                                                     double *partials, unsigned int *counter, double *out) {
    double d[1] = {0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double wi = (double)w[i];
        for (int k = 0; k < nv; ++k) wi -= h[k] * (double)basis[k][i];
        const V wv = (V)wi;
        w[i] = wv;
        d[0] += (double)wv * (double)wv;
    }
    reduce_finish<1>(d, partials, counter, [&](double *t) { out[0] = t[0]; });
}

// v = w / nrm ; z = dinv * v (the next Arnoldi input)
template <class V>
__global__ void k_normalize(const V *w, V *v, V *z, const V *dinv, double nrm, int n) {
    const V s = (V)(1.0 / nrm);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const V vi = w[i] * s;
        v[i] = vi;
        z[i] = dinv[i] * vi;
    }
}

// x += dinv * sum_k y_k V_k
template <class V>
__global__ void k_gmres_update(V *const *basis, const double *y, int nv, const V *dinv, V *x, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double s = 0;
        for (int k = 0; k < nv; ++k) s += y[k] * (double)basis[k][i];
        x[i] += dinv[i] * (V)s;
    }
}

// u = sum_k y_k V_k
template <class V>
__global__ void k_gmres_combine(V *const *basis, const double *y, int nv, V *u, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double s = 0;
        for (int k = 0; k < nv; ++k) s += y[k] * (double)basis[k][i];
        u[i] = (V)s;
    }
}
// x += d * u
template <class V>
__global__ void k_mul_add(const V *d, const V *u, V *x, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] += d[i] * u[i];
}

template <class V>
__global__ void k_sub_norm(const V *b, V *w, int n, double *partials, unsigned int *counter, double *out) {
    double d[1] = {0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const V r = b[i] - w[i];
        w[i] = r;
        d[0] += (double)r * (double)r;
    }
    reduce_finish<1>(d, partials, counter, [&](double *t) { out[0] = t[0]; });
}

template <class Real, class V>
struct GmresWs {
    V **basis_dev = nullptr;   // device array of m+1 basis pointers
    V *basis[GM_MAXV + 1] = {};
    V *w = nullptr, *z = nullptr, *dinv = nullptr;
    int m = 0;
};

template <class Real, class V>
static int gmres_ws(Ctx<Real> &c, GmresWs<Real, V> &ws, int m) {
    ws.m = m;
    for (int k = 0; k <= m; ++k) SPH_TRY(c.alloc(ws.basis[k], (size_t)c.n));
    SPH_TRY(c.alloc(ws.w, (size_t)c.n));
    SPH_TRY(c.alloc(ws.z, (size_t)c.n));
    SPH_TRY(c.alloc(ws.dinv, (size_t)c.n));
    SPH_TRY(c.alloc(ws.basis_dev, (size_t)m + 1));
    SPH_CUDA_TRY(cudaMemcpyAsync(ws.basis_dev, ws.basis, sizeof(V *) * (m + 1), cudaMemcpyHostToDevice, c.stream));
    return SPH_OK;
}

// GMRES(m) on M x = b; x holds the initial guess.  bnorm2 = ||b||^2 of the
// target relative residual.  Returns SPH_OK or SPH_NOT_CONVERGED.
template <class Real, class V>
static int gmres(Ctx<Real> &c, GmresWs<Real, V> &ws, V *x, const V *b, double bnorm2, double tol, int maxit,
                 bool cached, int *iters, double *relres) {
    const int n = c.n, m = ws.m;
    cudaStream_t st = c.stream;
    const int G = red_grid(n);
    unsigned int *counter = (unsigned int *)(c.scal + 32);
    double *dres = c.scal + 48;              // 16 doubles: scalar results
    double *hdev = c.gm_h;                   // GM_MAXV + 1 doubles
    double *hh = c.red_host;                 // pinned, 64 doubles
    k_dinv<V, Real><<<grid_for(n, 256), 256, 0, st>>>(c.row_kind, c.diag, ws.dinv, n);
    ++c.launches;
    const double bn = std::sqrt(bnorm2);
    std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), g(m + 1), y(m);
    int it = 0;
    int status = SPH_NOT_CONVERGED;
    const bool trace = getenv("SPH_TRACE_PPE") != nullptr;
    while (true) {
        // r = b - M x ; beta = ||r||
        apply_op<Real, V>(c, x, ws.w, cached);
        k_sub_norm<V><<<G, 256, 0, st>>>(b, ws.w, n, c.red, counter, dres);
        c.launches += 1;
        SPH_CUDA_TRY(cudaMemcpyAsync(hh, dres, sizeof(double), cudaMemcpyDeviceToHost, st));
        SPH_CUDA_TRY(cudaStreamSynchronize(st));
        const double beta = std::sqrt(hh[0]);
        *relres = beta / bn;
        if (c.init_relres < 0) c.init_relres = *relres;
        if (trace) fprintf(stderr, "  gmres restart it %d relres %.3e\n", it, *relres);
        if (*relres <= tol) { status = SPH_OK; break; }
        if (it >= maxit || !(beta > 0) || !std::isfinite(beta)) break;
        k_normalize<V><<<G, 256, 0, st>>>(ws.w, ws.basis[0], ws.z, ws.dinv, beta, n);
        coarse_apply<Real, V>(c, ws.basis[0], ws.z);   // z = M^-1 v with the coarse correction
        ++c.launches;
        std::fill(g.begin(), g.end(), 0.0);
        g[0] = beta;
        int j = 0;
        bool done = false;
        for (; j < m && it < maxit; ++j, ++it) {
            apply_op<Real, V>(c, ws.z, ws.w, cached);
            // classical Gram-Schmidt, second pass when the first lost > 30 %
            k_multidot<V><<<G, 256, 0, st>>>(ws.basis_dev, ws.w, j + 1, n, c.red, counter, hdev);
            k_orth_update<V><<<G, 256, 0, st>>>(ws.basis_dev, ws.w, hdev, j + 1, n, c.red, counter, dres);
            c.launches += 2;
            SPH_CUDA_TRY(cudaMemcpyAsync(hh, hdev, sizeof(double) * (j + 1), cudaMemcpyDeviceToHost, st));
            SPH_CUDA_TRY(cudaMemcpyAsync(hh + GM_MAXV, dres, sizeof(double), cudaMemcpyDeviceToHost, st));
            SPH_CUDA_TRY(cudaStreamSynchronize(st));
            double hnorm2 = 0;
            for (int k = 0; k <= j; ++k) { H[(size_t)k * m + j] = hh[k]; hnorm2 += hh[k] * hh[k]; }
            double wn2 = hh[GM_MAXV];
            if (wn2 < 0.49 * (wn2 + hnorm2)) {
                k_multidot<V><<<G, 256, 0, st>>>(ws.basis_dev, ws.w, j + 1, n, c.red, counter, hdev);
                k_orth_update<V><<<G, 256, 0, st>>>(ws.basis_dev, ws.w, hdev, j + 1, n, c.red, counter, dres);
                c.launches += 2;
                SPH_CUDA_TRY(cudaMemcpyAsync(hh, hdev, sizeof(double) * (j + 1), cudaMemcpyDeviceToHost, st));
                SPH_CUDA_TRY(cudaMemcpyAsync(hh + GM_MAXV, dres, sizeof(double), cudaMemcpyDeviceToHost, st));
                SPH_CUDA_TRY(cudaStreamSynchronize(st));
                for (int k = 0; k <= j; ++k) H[(size_t)k * m + j] += hh[k];
                wn2 = hh[GM_MAXV];
            }
            const double hn = std::sqrt(std::max(wn2, 0.0));
            // apply the previous rotations to column j, then a new one
            for (int k = 0; k < j; ++k) {
                const double a = H[(size_t)k * m + j], bb = H[(size_t)(k + 1) * m + j];
                H[(size_t)k * m + j] = cs[k] * a + sn[k] * bb;
                H[(size_t)(k + 1) * m + j] = -sn[k] * a + cs[k] * bb;
            }
            const double a = H[(size_t)j * m + j];
            const double rr = std::hypot(a, hn);
            cs[j] = rr > 0 ? a / rr : 1.0;
            sn[j] = rr > 0 ? hn / rr : 0.0;
            H[(size_t)j * m + j] = rr;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            *relres = std::fabs(g[j + 1]) / bn;
            if (!(hn > 0) || *relres <= tol) { ++j; ++it; done = true; break; }
            k_normalize<V><<<G, 256, 0, st>>>(ws.w, ws.basis[j + 1], ws.z, ws.dinv, hn, n);
            coarse_apply<Real, V>(c, ws.basis[j + 1], ws.z);
            ++c.launches;
        }
        // y = H^-1 g (upper triangular j x j), x += dinv V y
        const int nv = j;
        for (int k = nv - 1; k >= 0; --k) {
            double s = g[k];
            for (int q = k + 1; q < nv; ++q) s -= H[(size_t)k * m + q] * y[q];
            y[k] = H[(size_t)k * m + k] != 0 ? s / H[(size_t)k * m + k] : 0.0;
        }
        if (nv > 0) {
            SPH_CUDA_TRY(cudaMemcpyAsync(hdev, y.data(), sizeof(double) * nv, cudaMemcpyHostToDevice, st));
            if (c.cg_m > 0) {
                // x += M^-1 (V y) = dinv (V y) + Z E^-1 Z^T (V y)
                k_gmres_combine<V><<<G, 256, 0, st>>>(ws.basis_dev, hdev, nv, ws.w, n);
                k_mul_add<V><<<G, 256, 0, st>>>(ws.dinv, ws.w, x, n);
                coarse_apply<Real, V>(c, ws.w, x);
                c.launches += 1;
            } else {
                k_gmres_update<V><<<G, 256, 0, st>>>(ws.basis_dev, hdev, nv, ws.dinv, x, n);
            }
            ++c.launches;
        }
        if (done && *relres <= tol) {
            // confirm with the true residual on the next pass of the loop
            continue;
        }
        if (it >= maxit) {
            apply_op<Real, V>(c, x, ws.w, cached);
            k_sub_norm<V><<<G, 256, 0, st>>>(b, ws.w, n, c.red, counter, dres);
            ++c.launches;
            SPH_CUDA_TRY(cudaMemcpyAsync(hh, dres, sizeof(double), cudaMemcpyDeviceToHost, st));
            SPH_CUDA_TRY(cudaStreamSynchronize(st));
            *relres = std::sqrt(hh[0]) / bn;
            status = *relres <= tol ? SPH_OK : SPH_NOT_CONVERGED;
            break;
        }
    }
    SPH_CUDA_TRY(cudaGetLastError());
    *iters = it;
    return status;
}

template <class Real>
static int ensure_ppe_ws(Ctx<Real> &c) {
    const int n = c.n;
    if (!c.kv[0]) for (int k = 0; k < 10; ++k) SPH_TRY(c.alloc(c.kv[k], (size_t)n));
    if (!c.xd) { SPH_TRY(c.alloc(c.xd, n)); SPH_TRY(c.alloc(c.rd, n)); SPH_TRY(c.alloc(c.bd, n)); }
    if (!c.xf) { SPH_TRY(c.alloc(c.xf, n)); SPH_TRY(c.alloc(c.bf, n)); }
    if (!c.red) {
        SPH_TRY(c.alloc(c.red, (size_t)(GM_MAXV + 1) * 2048));
        SPH_TRY(c.alloc(c.gm_h, GM_MAXV + 8));
        SPH_TRY(c.alloc(c.scal, 64));
        SPH_CUDA_TRY(cudaMemsetAsync(c.scal, 0, 64 * sizeof(double), c.stream));
        SPH_CUDA_TRY(cudaMallocHost(&c.red_host, 64 * sizeof(double)));
    }
    if (!c.coef_valid) {
        c.coef_h_valid = false;
        const size_t m = (size_t)std::max(c.nnz_padded, 1LL);
        if (sizeof(Real) == 4) { c.release(c.coef); SPH_TRY(c.alloc(c.coef, m)); }
        else { c.release(c.coef_d); SPH_TRY(c.alloc(c.coef_d, m)); }
        c.release(c.ppe_gb);
        SPH_TRY(c.alloc(c.ppe_gb, 3 * m));   // rhs pair vectors, three SELL arrays
    }
    return SPH_OK;
}

// ppe_refinement = 4 and what the device-controlled solve needs: the mixed
// form with the cached operator, a stream of its own, no live timing, no
// learned / extrapolated / scaled start and no sample collection
template <class Real>
bool solve_under_device_control(const Ctx<Real> &c) {
    return sizeof(Real) == 4 && c.prm.ppe_mode == SPH_PPE_MIXED_IR && c.prm.ppe_refinement == 4 &&
           c.prm.ppe_matrix_free == 0 && c.stream != nullptr && !c.prof && c.ml_every == 0 && c.prm.ppe_warm_start == 0;
}

template <class Real>
int phase_ppe(Ctx<Real> &c, sph_ppe_stats *stats) {
    cudaStream_t st = c.stream;
    const int n = c.n;
    const Real tdt = (Real)c.dp.dt;
    const int mode = c.prm.ppe_mode;
    const bool cached = c.prm.ppe_matrix_free == 0;
    sph_ppe_stats S{};
    SPH_TRY(ensure_ppe_ws(c));
    Real *b = c.kv[9];
    SPH_CUDA_TRY(record_event(c, c.ev[4]));
    // b_i, A_i every step; c_ij once per neighbour-list build (time-invariant
    // while the particles do not move)
    const long long nnzp = std::max(c.nnz_padded, 1LL);
    if (c.coef_valid && c.ppe_gb) {
        k_ppe_rhs<Real><<<grid_for(n, 128), 128, 0, st>>>(c.ty, c.slice_off, c.ncnt, c.nbr, c.S.u, c.ppe_gb, nnzp, tdt,
                                                         b, n);
    } else if (sizeof(Real) == 4) {
        k_ppe_rows<Real, float><<<grid_for(n, 128), 128, 0, st>>>(c.dp, c.pf, c.pr, c.mr, c.ty, c.jc, c.slice_off, c.ncnt,
                                                                 c.nbr, c.g6, c.S.u, tdt, b, c.diag,
                                                                 c.coef_valid ? nullptr : c.coef, c.ppe_gb, nnzp, n);
    } else {
        k_ppe_rows<Real, double><<<grid_for(n, 128), 128, 0, st>>>(c.dp, c.pf, c.pr, c.mr, c.ty, c.jc, c.slice_off, c.ncnt,
                                                                  c.nbr, c.g6, c.S.u, tdt, b, c.diag,
                                                                  c.coef_valid ? nullptr : c.coef_d, c.ppe_gb, nnzp, n);
    }
    ++c.launches;
    SPH_CUDA_TRY(cudaGetLastError());
    c.coef_valid = true;
    if (sizeof(Real) == 4 && c.prm.ppe_coef_half && !c.coef_h_valid && mode != SPH_PPE_REF_SWEEP) {
        c.release(c.coef_h);
        c.release(c.coef_rs);
        SPH_TRY(c.alloc(c.coef_h, (size_t)nnzp));
        SPH_TRY(c.alloc(c.coef_rs, (size_t)n));
        k_coef_half<<<grid_for(n, 128), 128, 0, st>>>(c.row_kind, c.slice_off, c.ncnt, (const float *)c.coef, c.coef_h,
                                                       c.coef_rs, n);
        ++c.launches;
        SPH_CUDA_TRY(cudaGetLastError());
        c.coef_h_valid = true;
    }
    if (mode != SPH_PPE_REF_SWEEP &&
        (!c.cg_valid || c.cg_block != c.prm.ppe_coarse_block || c.cg_max != c.prm.ppe_coarse_max))
        SPH_TRY(coarse_build(c));

    if (mode == SPH_PPE_REF_SWEEP) {
        Real *pout = c.kv[8];
        if (sizeof(Real) == 4)
            k_ppe_sweep<Real, float><<<grid_for(n, 128), 128, 0, st>>>(c.ty, c.slice_off, c.ncnt, c.nbr, c.coef, b, c.diag,
                                                                      c.S.p, c.pres0, pout, n);
        else
            k_ppe_sweep<Real, double><<<grid_for(n, 128), 128, 0, st>>>(c.ty, c.slice_off, c.ncnt, c.nbr, c.coef_d, b, c.diag,
                                                                       c.S.p, c.pres0, pout, n);
        ++c.launches;
        SPH_CUDA_TRY(cudaMemcpyAsync(c.S.p, pout, sizeof(Real) * n, cudaMemcpyDeviceToDevice, st));
        S.status = SPH_OK;
        S.iterations = 1;
    } else {
        double *xd = c.xd, *rd = c.rd, *bd = c.bd;
        k_rhs<Real><<<grid_for(n, 256), 256, 0, st>>>(c.row_kind, b, c.S.p, bd, xd, n);
        const int G = red_grid(n);
        unsigned int *counter = (unsigned int *)(c.scal + 32);
        k_norm2<double><<<G, 256, 0, st>>>(bd, n, c.red, counter, c.scal, SC_BB);
        c.launches += 2;
        // ppe_refinement = 4: the mixed form's solve under device control, the
        // host reading nothing until the statistics are wanted (only without
        // live timing, learned / extrapolated / scaled start vectors and
        // sample collection, which need the host; else the host-controlled loop)
        const bool devloop = solve_under_device_control(c);
        if (devloop) {
            const double tol = c.prm.ppe_tol > 0 ? c.prm.ppe_tol : 1e-6;
            const int maxit = c.prm.ppe_max_iter > 0 ? c.prm.ppe_max_iter : 2000;
            SPH_TRY(bicgstab_device(c, xd, bd, rd, tol, maxit));
            k_dev_record<<<1, 1, 0, st>>>(c.scal);
            k_cast<double, Real><<<grid_for(n, 256), 256, 0, st>>>(xd, c.S.p, n);
            c.launches += 2;
            SPH_CUDA_TRY(record_event(c, c.ev[5]));
            SPH_TRY(neumann_pass(c, c.S));
            SPH_TRY(outlet_pass(c, c.S));
            SPH_CUDA_TRY(cudaGetLastError());
            c.ppe_pending = true;
            if (!c.defer_stats) {
                sph_ppe_stats S2{};
                SPH_TRY(dev_solve_stats(c, &S2, nullptr));
                if (stats) *stats = S2;
                return S2.status < 0 ? S2.status : SPH_OK;
            }
            return SPH_OK;
        }
        SPH_CUDA_TRY(cudaMemcpyAsync(c.red_host, c.scal, sizeof(double) * SC_COUNT, cudaMemcpyDeviceToHost, st));
        SPH_CUDA_TRY(cudaStreamSynchronize(st));
        double bb = c.red_host[SC_BB];
        if (!(bb > 0)) bb = 1.0;
        // learned warm start: x0 = p_old + s_d * net(features); the features
        // are also what the sample collection stores
        c.init_relres = -1;
        const bool learned = mode == SPH_PPE_LEARNED && c.ml_ready;
        const bool extrap = c.prm.ppe_warm_start == 1;
        const bool subspace = c.prm.ppe_warm_start == 4 || c.prm.ppe_warm_start == 5;
        const bool history = learned || c.ml_every > 0 || extrap || subspace;
        if (history) SPH_TRY(ml_prepare(c, (const Real *)b, learned || c.ml_every > 0));
        if (extrap) SPH_TRY(ml_extrapolate(c, xd));
        if (subspace) SPH_TRY(ml_subspace_start(c, bd, xd, rd, learned, c.prm.ppe_warm_start == 4));
        else if (learned) SPH_TRY(ml_warm_start(c, bd, xd, rd));
        if (!learned && c.prm.ppe_warm_start == 3) {
            apply_op<Real, double>(c, xd, rd, cached);
            k_start_factor<<<G, 256, 0, st>>>(bd, rd, n, c.red, counter, c.scal);
            k_scale_start<<<G, 256, 0, st>>>(xd, n, c.scal);
            c.launches += 2;
        }
        const double tol = c.prm.ppe_tol > 0 ? c.prm.ppe_tol : 1e-6;
        const int maxit = c.prm.ppe_max_iter > 0 ? c.prm.ppe_max_iter : 2000;
        int status = SPH_OK, iters = 0, restarts = 0, refinements = 0;
        double relres = 0;
        const int m = std::max(4, std::min(GM_MAXV, c.prm.ppe_gmres_restart > 0 ? c.prm.ppe_gmres_restart : 40));
        auto ws_r = [&]() -> GmresWs<Real, Real> * {
            if (!c.gm_ws_r) {
                auto *w = new GmresWs<Real, Real>();
                if (gmres_ws(c, *w, m) < 0) { delete w; return nullptr; }
                c.gm_ws_r = w;
            }
            return (GmresWs<Real, Real> *)c.gm_ws_r;
        };
        auto ws_d = [&]() -> GmresWs<Real, double> * {
            if (!c.gm_ws_d) {
                auto *w = new GmresWs<Real, double>();
                if (gmres_ws(c, *w, m) < 0) { delete w; return nullptr; }
                c.gm_ws_d = w;
            }
            return (GmresWs<Real, double> *)c.gm_ws_d;
        };
        auto idr_r = [&]() -> IdrWs<Real> * {
            if (!c.idr_ws_r) {
                auto *w = new IdrWs<Real>();
                if (idr_ws(c, *w) < 0) { delete w; return nullptr; }
                c.idr_ws_r = w;
            }
            return (IdrWs<Real> *)c.idr_ws_r;
        };
        auto idr_f = [&]() -> IdrWs<float> * {
            if (!c.idr_ws_f) {
                auto *w = new IdrWs<float>();
                if (idr_ws(c, *w) < 0) { delete w; return nullptr; }
                c.idr_ws_f = w;
            }
            return (IdrWs<float> *)c.idr_ws_f;
        };
        const bool trace = getenv("SPH_TRACE_PPE") != nullptr;
        if (sizeof(Real) == 8 && mode == SPH_PPE_IDRS) {
            IdrWs<Real> *w = idr_r();
            if (!w) return SPH_ERR_OUT_OF_MEMORY;
            status = idrs<Real, Real>(c, *w, (Real *)xd, (const Real *)bd, bb, tol, maxit, cached, &iters, &relres);
        } else if (sizeof(Real) == 8) {
            // plain form: the whole solve in FP64
            if (mode != SPH_PPE_GMRES)
                status = bicgstab<Real>(c, (Real *)xd, (const Real *)bd, bb, tol, maxit, cached, &iters, &relres, &restarts);
            else {
                GmresWs<Real, Real> *w = ws_r();
                if (!w) return SPH_ERR_OUT_OF_MEMORY;
                status = gmres<Real, Real>(c, *w, (Real *)xd, (const Real *)bd, bb, tol, maxit, cached, &iters, &relres);
            }
        } else if (mode == SPH_PPE_BICGSTAB || mode == SPH_PPE_GMRES || mode == SPH_PPE_IDRS) {
            // FP32 vectors throughout, FP64 reductions
            k_cast<double, float><<<grid_for(n, 256), 256, 0, st>>>(xd, c.xf, n);
            k_cast<double, float><<<grid_for(n, 256), 256, 0, st>>>(bd, c.bf, n);
            c.launches += 2;
            if (mode == SPH_PPE_BICGSTAB) {
                status = bicgstab<Real>(c, (Real *)c.xf, (const Real *)c.bf, bb, tol, maxit, cached, &iters, &relres, &restarts);
            } else if (mode == SPH_PPE_IDRS) {
                IdrWs<float> *w = idr_f();
                if (!w) return SPH_ERR_OUT_OF_MEMORY;
                status = idrs<Real, float>(c, *w, c.xf, c.bf, bb, tol, maxit, cached, &iters, &relres);
            } else {
                GmresWs<Real, Real> *w = ws_r();
                if (!w) return SPH_ERR_OUT_OF_MEMORY;
                status = gmres<Real, Real>(c, *w, (Real *)c.xf, (const Real *)c.bf, bb, tol, maxit, cached, &iters, &relres);
            }
            if (trace) fprintf(stderr, "FP32 solve st %d it %d rel %.3e\n", status, iters, relres);
            k_cast<float, double><<<grid_for(n, 256), 256, 0, st>>>(c.xf, xd, n);
            ++c.launches;
        } else if (c.prm.ppe_refinement == 0 || c.prm.ppe_refinement == 4) {
            // FP32 BiCGSTAB with FP64 reliable updates; FP64 BiCGSTAB from
            // its last iterate if the FP32 recurrence breaks down
            status = bicgstab_reliable(c, xd, bd, rd, bb, tol, maxit, cached, &iters, &relres, &refinements, &restarts);
            if (trace) fprintf(stderr, "RU st %d it %d updates %d rel %.3e\n", status, iters, refinements, relres);
            if (status < 0 || (status != SPH_OK && iters < maxit)) {
                if (!c.kd[0]) for (int k = 0; k < 10; ++k) SPH_TRY(c.alloc(c.kd[k], (size_t)n));
                int it64 = 0, rs64 = 0;
                status = bicgstab_fp64(c, xd, bd, bb, tol, std::max(maxit - iters, 1), cached, &it64, &relres, &rs64);
                iters += it64;
                restarts += rs64 + 1000;   // marks the FP64 fallback in the statistics
            }
        } else {
            // FP32 Krylov corrections restarted at every refinement (BiCGSTAB
            // with ppe_refinement = 2, GMRES with ppe_refinement = 1) inside FP64
            // iterative refinement; the outer residual r = b - M x and the
            // update x += e are FP64
            float *ef = c.xf, *rf = c.bf;
            const double inner_tol = c.prm.ppe_inner_tol > 0 ? c.prm.ppe_inner_tol : 1e-3;
            GmresWs<Real, Real> *w = c.prm.ppe_refinement == 1 ? ws_r() : nullptr;
            if (c.prm.ppe_refinement == 1 && !w) return SPH_ERR_OUT_OF_MEMORY;
            IdrWs<float> *wi = c.prm.ppe_refinement == 3 ? idr_f() : nullptr;
            if (c.prm.ppe_refinement == 3 && !wi) return SPH_ERR_OUT_OF_MEMORY;
            status = SPH_NOT_CONVERGED;
            for (refinements = 0; refinements < 50; ++refinements) {
                apply_op<Real, double>(c, xd, rd, cached);
                k_ir_residual<<<G, 256, 0, st>>>(bd, rd, rd, rf, ef, n);
                k_norm2<double><<<G, 256, 0, st>>>(rd, n, c.red, counter, c.scal, SC_RR);
                c.launches += 2;
                SPH_CUDA_TRY(cudaMemcpyAsync(c.red_host, c.scal, sizeof(double) * SC_COUNT, cudaMemcpyDeviceToHost, st));
                SPH_CUDA_TRY(cudaStreamSynchronize(st));
                const double rr = c.red_host[SC_RR];
                relres = std::sqrt(rr / bb);
                if (relres <= tol) { status = SPH_OK; break; }
                if (iters >= maxit) break;
                int it_in = 0, rs_in = 0;
                double rel_in = 0;
                const int st_in = c.prm.ppe_refinement == 1
                                      ? gmres<Real, Real>(c, *w, (Real *)ef, (const Real *)rf, rr, inner_tol, maxit - iters,
                                                          cached, &it_in, &rel_in)
                                  : c.prm.ppe_refinement == 3
                                      ? idrs<Real, float>(c, *wi, ef, rf, rr, inner_tol, maxit - iters, cached, &it_in, &rel_in)
                                      : bicgstab<Real>(c, (Real *)ef, (const Real *)rf, rr, inner_tol, maxit - iters, cached,
                                                       &it_in, &rel_in, &rs_in);
                restarts += rs_in;
                if (trace)
                    fprintf(stderr, "IR %d outer relres %.3e inner st %d it %d rel %.3e\n", refinements, relres, st_in, it_in,
                            rel_in);
                iters += it_in;
                if (st_in != SPH_OK && !(rel_in < 1.0)) {
                    // the FP32 correction made no progress: finish in FP64
                    if (trace) fprintf(stderr, "IR fallback to FP64 BiCGSTAB at outer %.3e\n", relres);
                    if (!c.kd[0]) for (int k = 0; k < 10; ++k) SPH_TRY(c.alloc(c.kd[k], (size_t)n));
                    int it64 = 0, rs64 = 0;
                    status = bicgstab_fp64(c, xd, bd, bb, tol, std::max(maxit - iters, 1), cached, &it64, &relres, &rs64);
                    iters += it64;
                    restarts += rs64;
                    restarts += 1000;   // marks the FP64 fallback in the statistics
                    break;
                }
                k_axpy_cast<float, double><<<grid_for(n, 256), 256, 0, st>>>(ef, xd, n);
                ++c.launches;
            }
        }
        if (c.ml_every > 0 && status == SPH_OK) SPH_TRY(ml_collect(c, xd));
        if (history) SPH_TRY(ml_finish_step(c));
        k_cast<double, Real><<<grid_for(n, 256), 256, 0, st>>>(xd, c.S.p, n);
        ++c.launches;
        S.status = status;
        S.iterations = iters;
        S.refinements = refinements;
        S.restarts = restarts;
        S.rel_residual = relres;
        S.initial_residual = c.init_relres;
    }
    SPH_CUDA_TRY(cudaEventRecord(c.ev[5], st));
    SPH_TRY(neumann_pass(c, c.S));
    SPH_TRY(outlet_pass(c, c.S));
    SPH_CUDA_TRY(cudaGetLastError());
    SPH_CUDA_TRY(cudaEventSynchronize(c.ev[5]));
    float ms = 0;
    cudaEventElapsedTime(&ms, c.ev[4], c.ev[5]);
    S.solve_ms = ms;
    c.last_ppe = S;
    if (stats) *stats = S;
    return S.status < 0 ? S.status : SPH_OK;
}

template <class Real>
void release_solver_ws(Ctx<Real> &c) {
    delete (GmresWs<Real, Real> *)c.gm_ws_r;
    delete (GmresWs<Real, double> *)c.gm_ws_d;
    delete (IdrWs<Real> *)c.idr_ws_r;
    delete (IdrWs<float> *)c.idr_ws_f;
    if (c.kgraph) {
        auto *g = (KrylovGraph *)c.kgraph;
        if (g->exec) cudaGraphExecDestroy(g->exec);
        delete g;
        c.kgraph = nullptr;
    }
    delete (DevLoopGraph *)c.devloop;
    c.devloop = nullptr;
    ++c.mem_gen;   // a step graph captured over these workspaces is stale
    c.gm_ws_r = nullptr;
    c.gm_ws_d = nullptr;
    c.idr_ws_r = nullptr;
    c.idr_ws_f = nullptr;
}

#define INST(R) template int phase_ppe<R>(Ctx<R> &, sph_ppe_stats *); \
    template void release_solver_ws<R>(Ctx<R> &); \
    template int dev_solve_stats<R>(Ctx<R> &, sph_ppe_stats *, int *); \
    template int dev_reset_worst<R>(Ctx<R> &); \
    template bool solve_under_device_control<R>(const Ctx<R> &); \
    template int operator_stats<R>(Ctx<R> &, int64_t *, double *, double *, int); \
    template int operator_bytes<R>(Ctx<R> &, double *, double *); \
    template void ppe_apply_fp64<R>(Ctx<R> &, const double *, double *);
INST(float)
INST(double)
#undef INST

}  // namespace sph
