// Learned warm start of the converged pressure solve.
//
// A per-particle MLP predicts the pressure change of the step from local
// features of the previous pressure and the new right-hand side; the Krylov
// solve starts from p_old + prediction and still runs to the requested
// residual, so the network changes the iteration count, never the answer.
//
//   features (ML_F = 20 per fluid row, BF16, rows padded to 32 columns):
//     r_i = b_i - sum_j c_ij (p_i - p_j)   residual of the previous pressure
//     d_i = r_i / A_i                      its Jacobi update
//     g_i = p_old_i - p_oldold_i           the previous step's pressure change
//     0..4   d_i / s_d, r_i / s_r, b_i / s_b, (p_i - pbar) / s_p, g_i / s_d
//     5..12  for d and r: sum_j w_ij q_j, sum_j w_ij |q_j - q_i|, max_j, min_j
//     13..18 for b, p - pbar, g: sum_j w_ij q_j, sum_j w_ij |q_j - q_i|
//     19     sum of w_ij over non-fluid neighbours (wall proximity)
//            with w_ij = c_ij / A_i over the row's stored neighbours
//     s_* are root-mean-square values over the fluid rows of the step
//   network: 20 -> 64 (ReLU) -> 64 (ReLU) -> 1, target (p_new - p_old) / s_d
//   warm start: x0 = p_old + alpha z, z = s_d * net on the fluid rows and
//     alpha minimising ||b - M x0||_2 (two FP64 operator applications), so
//     the warm start never raises the initial residual
//   parameters (FP32, ML_NPARAM): W1[20][64], b1[64], W2[64][64], b2[64],
//     w3[64], b3; W[k][a] maps input k to unit a.
//
// Inference runs on the tensor cores: BF16 operands, FP32 accumulation,
// mma.sync m16n8k16, one warp per 16 rows, the layer-1 accumulators fed to
// layer 2 as A fragments without leaving registers.  Training (Adam, FP32
// master weights) runs its forward and backward passes on the CUDA cores in
// FP32 so that its gradients can be checked against a CPU restatement; both
// read the same BF16 features.  Samples come from the context's own
// converged solves (sph_ml_collect).
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "ctx.cuh"

namespace sph {

constexpr int ML_F = 20, ML_FP = 32, ML_H = 64;
constexpr int ML_OW1 = 0, ML_OB1 = ML_F * ML_H, ML_OW2 = ML_OB1 + ML_H, ML_OB2 = ML_OW2 + ML_H * ML_H,
              ML_OW3 = ML_OB2 + ML_H, ML_OB3 = ML_OW3 + ML_H, ML_NPARAM = ML_OB3 + 1;
static_assert(ML_NPARAM == SPH_ML_NPARAM, "parameter count of the header");
constexpr int ML_ROWS_TRAIN = 64;    // samples per block of the training kernel
constexpr long long ML_CAP_DEFAULT = 1LL << 21;

// ---- scales: deterministic block partials, last block finishes ------------------
struct MlScal { double sd, sr, sb, sp, pbar, cnt; };

template <int NV, class F>
__device__ __forceinline__ void ml_reduce(double (&v)[NV], double *partials, unsigned int *counter, F finish) {
    __shared__ double sh[NV][8];
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
        for (int q = 0; q < NV; ++q) {
            double s = 0;
            for (int w = 0; w < nw; ++w) s += sh[q][w];
            partials[(size_t)q * gridDim.x + blockIdx.x] = s;
        }
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    double t[NV];
    for (int q = 0; q < NV; ++q) {
        double s = 0;
        for (unsigned b = 0; b < gridDim.x; ++b) s += ((volatile double *)partials)[(size_t)q * gridDim.x + b];
        t[q] = s;
    }
    finish(t);
    *counter = 0;
}

// residual and Jacobi update of the previous pressure; p_old snapshot
template <class Real, class C>
__global__ void __launch_bounds__(256) k_ml_residual(const int *__restrict__ kind, const long long *__restrict__ slice_off,
                                                     const int *__restrict__ ncnt, const int *__restrict__ nbr,
                                                     const C *__restrict__ coef, const Real *__restrict__ diag,
                                                     const Real *__restrict__ b, const Real *__restrict__ p,
                                                     float *__restrict__ rr, float *__restrict__ dd,
                                                     float *__restrict__ pold, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float pi = (float)p[i];
    pold[i] = pi;
    float r = 0, d = 0;
    if (kind[i] == 1) {
        const long long base = slice_off[i >> 5] + (i & 31);
        const int cnt = ncnt[i];
        double s = 0;
        for (int k = 0; k < cnt; ++k) {
            const long long e = base + 32LL * k;
            s += (double)coef[sell4(base - (i & 31), i & 31, k)] * ((double)p[i] - (double)p[nbr[e]]);
        }
        r = (float)((double)b[i] - s);
        const double a = (double)diag[i];
        d = a != 0.0 ? (float)((double)r / a) : 0.f;
    }
    rr[i] = r;
    dd[i] = d;
}

template <class Real>
__global__ void __launch_bounds__(256) k_ml_scales(const int *kind, const float *rr, const float *dd, const Real *b,
                                                   const float *pold, int n, double *partials, unsigned int *counter,
                                                   MlScal *out) {
    double v[6] = {0, 0, 0, 0, 0, 0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (kind[i] != 1) continue;
        const double d = dd[i], r = rr[i], bb = (double)b[i], p = pold[i];
        v[0] += d * d; v[1] += r * r; v[2] += bb * bb; v[3] += p; v[4] += p * p; v[5] += 1;
    }
    ml_reduce<6>(v, partials, counter, [&](double *t) {
        const double c = t[5] > 0 ? t[5] : 1;
        auto rms = [](double x) { return x > 0 ? sqrt(x) : 1.0; };
        MlScal s;
        s.sd = rms(t[0] / c); s.sr = rms(t[1] / c); s.sb = rms(t[2] / c);
        s.pbar = t[3] / c;
        s.sp = rms(t[4] / c - s.pbar * s.pbar);
        s.cnt = t[5];
        *out = s;
    });
}

template <class Real, class C>
__global__ void __launch_bounds__(256) k_ml_features(const int *__restrict__ kind, const long long *__restrict__ slice_off,
                                                     const int *__restrict__ ncnt, const int *__restrict__ nbr,
                                                     const C *__restrict__ coef, const Real *__restrict__ diag,
                                                     const Real *__restrict__ b, const float *__restrict__ rr,
                                                     const float *__restrict__ dd, const float *__restrict__ pold,
                                                     const float *__restrict__ pprev, const MlScal *__restrict__ sc,
                                                     __nv_bfloat16 *__restrict__ X, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float f[ML_FP];
#pragma unroll
    for (int k = 0; k < ML_FP; ++k) f[k] = 0.f;
    if (kind[i] == 1) {
        const MlScal s = *sc;
        const float isd = (float)(1.0 / s.sd), isr = (float)(1.0 / s.sr), isb = (float)(1.0 / s.sb),
                    isp = (float)(1.0 / s.sp), pbar = (float)s.pbar;
        // q: Jacobi update, residual, rhs, pressure, previous pressure change
        const float qi[5] = {dd[i] * isd, rr[i] * isr, (float)b[i] * isb, (pold[i] - pbar) * isp,
                             pprev ? (pold[i] - pprev[i]) * isd : 0.f};
        float mean[5] = {0, 0, 0, 0, 0}, dev[5] = {0, 0, 0, 0, 0}, mx[2], mn[2], wall = 0.f;
#pragma unroll
        for (int q = 0; q < 2; ++q) { mx[q] = qi[q]; mn[q] = qi[q]; }
        const long long base = slice_off[i >> 5] + (i & 31);
        const int cnt = ncnt[i];
        const float ia = diag[i] != (Real)0 ? (float)(1.0 / (double)diag[i]) : 0.f;
        for (int k = 0; k < cnt; ++k) {
            const long long e = base + 32LL * k;
            const int j = nbr[e];
            const float w = (float)coef[sell4(base - (i & 31), i & 31, k)] * ia;
            const bool fl = kind[j] == 1;
            const float qj[5] = {fl ? dd[j] * isd : 0.f, fl ? rr[j] * isr : 0.f, fl ? (float)b[j] * isb : 0.f,
                                 (pold[j] - pbar) * isp, pprev ? (pold[j] - pprev[j]) * isd : 0.f};
            if (!fl) wall += w;
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                mean[q] += w * qj[q];
                dev[q] += w * fabsf(qj[q] - qi[q]);
            }
#pragma unroll
            for (int q = 0; q < 2; ++q) { mx[q] = fmaxf(mx[q], qj[q]); mn[q] = fminf(mn[q], qj[q]); }
        }
        // 0..4 own values; 5..8 / 9..12 mean, deviation, max, min of d / r;
        // 13..18 mean, deviation of b, p, previous change; 19 wall weight
#pragma unroll
        for (int q = 0; q < 5; ++q) f[q] = qi[q];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            f[5 + 4 * q] = mean[q]; f[6 + 4 * q] = dev[q]; f[7 + 4 * q] = mx[q]; f[8 + 4 * q] = mn[q];
        }
#pragma unroll
        for (int q = 2; q < 5; ++q) { f[13 + 2 * (q - 2)] = mean[q]; f[14 + 2 * (q - 2)] = dev[q]; }
        f[19] = wall;
    }
    __nv_bfloat162 *row = (__nv_bfloat162 *)(X + (size_t)i * ML_FP);
#pragma unroll
    for (int k = 0; k < ML_FP / 2; ++k) row[k] = __floats2bfloat162_rn(f[2 * k], f[2 * k + 1]);
}

// ---- tensor-core inference ----------------------------------------------------
__device__ __forceinline__ void mma_bf16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
    uint32_t u;
    memcpy(&u, &h, 4);
    return u;
}

// W1b[n][k] (64 x 32) and W2b[n][k] (64 x 64): B operands, k contiguous
__global__ void k_ml_pack(const float *w, __nv_bfloat16 *w1b, __nv_bfloat16 *w2b) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < ML_H * ML_FP) {
        const int nn = t / ML_FP, k = t % ML_FP;
        w1b[t] = __float2bfloat16_rn(k < ML_F ? w[ML_OW1 + k * ML_H + nn] : 0.f);
    }
    if (t < ML_H * ML_H) {
        const int nn = t / ML_H, k = t % ML_H;
        w2b[t] = __float2bfloat16_rn(w[ML_OW2 + k * ML_H + nn]);
    }
}

// y[r] for rows [0, rows) of X; 8 warps x 16 rows per block
__global__ void __launch_bounds__(256) k_ml_infer(const __nv_bfloat16 *__restrict__ X, const int *__restrict__ row_of,
                                                  const __nv_bfloat16 *__restrict__ w1b,
                                                  const __nv_bfloat16 *__restrict__ w2b, const float *__restrict__ w,
                                                  float *__restrict__ y, int rows) {
    __shared__ __align__(16) __nv_bfloat16 s1[ML_H * ML_FP];
    __shared__ __align__(16) __nv_bfloat16 s2[ML_H * ML_H];
    __shared__ float sb1[ML_H], sb2[ML_H], sw3[ML_H];
    for (int t = threadIdx.x; t < ML_H * ML_FP; t += blockDim.x) s1[t] = w1b[t];
    for (int t = threadIdx.x; t < ML_H * ML_H; t += blockDim.x) s2[t] = w2b[t];
    for (int t = threadIdx.x; t < ML_H; t += blockDim.x) {
        sb1[t] = w[ML_OB1 + t]; sb2[t] = w[ML_OB2 + t]; sw3[t] = w[ML_OW3 + t];
    }
    __syncthreads();
    const float b3 = w[ML_OB3];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, tg = lane & 3;
    const long long row0 = ((long long)blockIdx.x * 8 + warp) * 16;
    if (row0 >= rows) return;   // whole warp leaves together
    const long long ra = row0 + g, rb = row0 + g + 8;
    const bool va = ra < rows, vb = rb < rows;
    const long long xa = va ? (row_of ? row_of[ra] : ra) : 0, xb = vb ? (row_of ? row_of[rb] : rb) : 0;
    const uint32_t *Xa = (const uint32_t *)(X + xa * ML_FP), *Xb = (const uint32_t *)(X + xb * ML_FP);
    const uint32_t *W1 = (const uint32_t *)s1, *W2 = (const uint32_t *)s2;
    // layer 1: K = 32 (2 steps), N = 64 (8 tiles)
    float acc[8][4];
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        const int kw = (16 * s + 2 * tg) >> 1;   // 32-bit word of column 16s + 2tg
        const uint32_t a0 = va ? Xa[kw] : 0u, a1 = vb ? Xb[kw] : 0u;
        const uint32_t a2 = va ? Xa[kw + 4] : 0u, a3 = vb ? Xb[kw + 4] : 0u;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int nrow = (8 * j + g) * (ML_FP / 2);
            mma_bf16(acc[j], a0, a1, a2, a3, W1[nrow + kw], W1[nrow + kw + 4]);
        }
    }
    // bias + ReLU, repacked as the A fragments of layer 2
    uint32_t h[4][4];
#pragma unroll
    for (int s = 0; s < 4; ++s) {
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            const int j = 2 * s + half;
            const int col = 8 * j + 2 * tg;
            const float c0 = fmaxf(acc[j][0] + sb1[col], 0.f), c1 = fmaxf(acc[j][1] + sb1[col + 1], 0.f);
            const float c2 = fmaxf(acc[j][2] + sb1[col], 0.f), c3 = fmaxf(acc[j][3] + sb1[col + 1], 0.f);
            h[s][2 * half] = pack_bf16(c0, c1);       // rows g   : a0 / a2
            h[s][2 * half + 1] = pack_bf16(c2, c3);   // rows g+8 : a1 / a3
        }
    }
    // layer 2: K = 64 (4 steps), N = 64 (8 tiles)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        const int kw = (16 * s + 2 * tg) >> 1;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int nrow = (8 * j + g) * (ML_H / 2);
            mma_bf16(acc[j], h[s][0], h[s][1], h[s][2], h[s][3], W2[nrow + kw], W2[nrow + kw + 4]);
        }
    }
    // bias + ReLU, layer 3 in FP32
    float ya = 0.f, yb = 0.f;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int col = 8 * j + 2 * tg;
        ya += fmaxf(acc[j][0] + sb2[col], 0.f) * sw3[col] + fmaxf(acc[j][1] + sb2[col + 1], 0.f) * sw3[col + 1];
        yb += fmaxf(acc[j][2] + sb2[col], 0.f) * sw3[col] + fmaxf(acc[j][3] + sb2[col + 1], 0.f) * sw3[col + 1];
    }
    ya += __shfl_xor_sync(0xffffffffu, ya, 1);
    ya += __shfl_xor_sync(0xffffffffu, ya, 2);
    yb += __shfl_xor_sync(0xffffffffu, yb, 1);
    yb += __shfl_xor_sync(0xffffffffu, yb, 2);
    if (tg == 0) {
        if (va) y[ra] = ya + b3;
        if (vb) y[rb] = yb + b3;
    }
}

// predicted change z_i = s_d y_i on the fluid rows, 0 elsewhere
__global__ void k_ml_dir(const int *kind, const float *y, const MlScal *sc, double *z, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    z[i] = kind[i] == 1 ? sc->sd * (double)y[i] : 0.0;
}

// alpha = (r0, Mz) / (Mz, Mz) with r0 = b - M x0: the step along z that
// minimises the 2-norm of the new residual (0 when Mz vanishes)
__global__ void __launch_bounds__(256) k_ml_alpha(const double *b, const double *mx, const double *mz, int n,
                                                  double *partials, unsigned int *counter, double *alpha) {
    double v[2] = {0, 0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double r = b[i] - mx[i];
        v[0] += r * mz[i];
        v[1] += mz[i] * mz[i];
    }
    ml_reduce<2>(v, partials, counter, [&](double *t) { *alpha = t[1] > 0 ? t[0] / t[1] : 0.0; });
}

__global__ void k_ml_step(const double *z, const double *alpha, double *x, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] += *alpha * z[i];
}

// appends the selected rows' features and targets (p_new - p_old) / s_d
__global__ void k_ml_collect(const int *fluid, int off, int every, int take, const __nv_bfloat16 *X, const float *pold,
                             const double *xnew, const MlScal *sc, __nv_bfloat16 *SX, float *St, long long base) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= take) return;
    const int i = fluid[off + (long long)s * every];
    const uint4 *src = (const uint4 *)(X + (size_t)i * ML_FP);
    uint4 *dst = (uint4 *)(SX + (size_t)(base + s) * ML_FP);
#pragma unroll
    for (int k = 0; k < ML_FP * 2 / 16; ++k) dst[k] = src[k];
    St[base + s] = (float)((xnew[i] - (double)pold[i]) / sc->sd);
}

// ---- training: FP32 forward + backward of ML_ROWS_TRAIN samples per block ----
// partial gradients per block; loss partial = sum of squared errors
__global__ void __launch_bounds__(256) k_ml_fwd_bwd(const __nv_bfloat16 *__restrict__ SX, const float *__restrict__ St,
                                                    const int *__restrict__ idx, long long first, int rows,
                                                    const float *__restrict__ w, float gscale,
                                                    float *__restrict__ gpart, float *__restrict__ lpart) {
    extern __shared__ float smem[];
    const int R = ML_ROWS_TRAIN;
    float *x = smem;                    // R x 32
    float *h1 = x + R * ML_FP;          // R x 64
    float *h2 = h1 + R * ML_H;          // R x 64
    float *d2 = h2 + R * ML_H;          // R x 64
    float *d1 = d2 + R * ML_H;          // R x 64
    float *W1 = d1 + R * ML_H;          // 32 x 64 (rows >= 20 zero)
    float *W2 = W1 + ML_FP * ML_H;      // 64 x 64
    float *bb1 = W2 + ML_H * ML_H, *bb2 = bb1 + ML_H, *ww3 = bb2 + ML_H;
    float *dy = ww3 + ML_H;             // R
    float *red = dy + R;                // 8
    const int tid = threadIdx.x, nt = blockDim.x;
    const long long r0 = first + (long long)blockIdx.x * R;
    const long long left = first + rows - r0;
    const int nr = left <= 0 ? 0 : (left < R ? (int)left : R);
    for (int t = tid; t < ML_FP * ML_H; t += nt) W1[t] = (t / ML_H) < ML_F ? w[ML_OW1 + t] : 0.f;
    for (int t = tid; t < ML_H * ML_H; t += nt) W2[t] = w[ML_OW2 + t];
    for (int t = tid; t < ML_H; t += nt) { bb1[t] = w[ML_OB1 + t]; bb2[t] = w[ML_OB2 + t]; ww3[t] = w[ML_OW3 + t]; }
    for (int t = tid; t < R * ML_FP; t += nt) {
        const int r = t / ML_FP, k = t % ML_FP;
        float v = 0.f;
        if (r < nr) {
            const long long sidx = idx ? idx[r0 + r] : r0 + r;
            v = __bfloat162float(SX[(size_t)sidx * ML_FP + k]);
        }
        x[t] = v;
    }
    __syncthreads();
    for (int t = tid; t < R * ML_H; t += nt) {
        const int r = t / ML_H, a = t % ML_H;
        float s = bb1[a];
        for (int k = 0; k < ML_F; ++k) s += x[r * ML_FP + k] * W1[k * ML_H + a];
        h1[t] = fmaxf(s, 0.f);
    }
    __syncthreads();
    for (int t = tid; t < R * ML_H; t += nt) {
        const int r = t / ML_H, a = t % ML_H;
        float s = bb2[a];
        for (int k = 0; k < ML_H; ++k) s += h1[r * ML_H + k] * W2[k * ML_H + a];
        h2[t] = fmaxf(s, 0.f);
    }
    __syncthreads();
    const float b3 = w[ML_OB3];
    float lsum = 0.f;
    for (int r = tid; r < R; r += nt) {
        float e = 0.f;
        if (r < nr) {
            float s = b3;
            for (int a = 0; a < ML_H; ++a) s += h2[r * ML_H + a] * ww3[a];
            const long long sidx = idx ? idx[r0 + r] : r0 + r;
            e = s - St[sidx];
        }
        dy[r] = gscale * 2.f * e;   // d(loss)/dy with loss = gscale * sum e^2
        lsum += e * e;
    }
    __syncthreads();
    for (int t = tid; t < R * ML_H; t += nt) {
        const int r = t / ML_H, a = t % ML_H;
        d2[t] = h2[t] > 0.f ? dy[r] * ww3[a] : 0.f;
    }
    __syncthreads();
    for (int t = tid; t < R * ML_H; t += nt) {
        const int r = t / ML_H, k = t % ML_H;
        float s = 0.f;
        for (int a = 0; a < ML_H; ++a) s += W2[k * ML_H + a] * d2[r * ML_H + a];
        d1[t] = h1[t] > 0.f ? s : 0.f;
    }
    __syncthreads();
    float *gp = gpart + (size_t)blockIdx.x * ML_NPARAM;
    for (int t = tid; t < ML_F * ML_H; t += nt) {      // dW1[k][a] = sum_r x[r][k] d1[r][a]
        const int k = t / ML_H, a = t % ML_H;
        float s = 0.f;
        for (int r = 0; r < R; ++r) s += x[r * ML_FP + k] * d1[r * ML_H + a];
        gp[ML_OW1 + t] = s;
    }
    for (int t = tid; t < ML_H * ML_H; t += nt) {      // dW2[k][a] = sum_r h1[r][k] d2[r][a]
        const int k = t / ML_H, a = t % ML_H;
        float s = 0.f;
        for (int r = 0; r < R; ++r) s += h1[r * ML_H + k] * d2[r * ML_H + a];
        gp[ML_OW2 + t] = s;
    }
    for (int a = tid; a < ML_H; a += nt) {
        float s1 = 0.f, s2 = 0.f, s3 = 0.f;
        for (int r = 0; r < R; ++r) { s1 += d1[r * ML_H + a]; s2 += d2[r * ML_H + a]; s3 += dy[r] * h2[r * ML_H + a]; }
        gp[ML_OB1 + a] = s1; gp[ML_OB2 + a] = s2; gp[ML_OW3 + a] = s3;
    }
    if (tid == 0) {
        float s = 0.f;
        for (int r = 0; r < R; ++r) s += dy[r];
        gp[ML_OB3] = s;
    }
    // loss partial, fixed order
    for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
    if ((tid & 31) == 0) red[tid >> 5] = lsum;
    __syncthreads();
    if (tid == 0) {
        float s = 0.f;
        for (int q = 0; q < nt / 32; ++q) s += red[q];
        lpart[blockIdx.x] = s;
    }
}

static size_t ml_train_smem() {
    const int R = ML_ROWS_TRAIN;
    return sizeof(float) * ((size_t)R * ML_FP + 4 * (size_t)R * ML_H + ML_FP * ML_H + ML_H * ML_H + 3 * ML_H + R + 8);
}

// gradient = sum of the block partials in block order; optional Adam step
__global__ void k_ml_reduce(const float *gpart, int nparts, float *grad) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ML_NPARAM) return;
    float s = 0.f;
    for (int b = 0; b < nparts; ++b) s += gpart[(size_t)b * ML_NPARAM + p];
    grad[p] = s;
}

__global__ void k_ml_adam(float *w, float *m, float *v, const float *grad, float lr, float c1, float c2) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ML_NPARAM) return;
    const float g = grad[p];
    const float mm = 0.9f * m[p] + 0.1f * g, vv = 0.999f * v[p] + 0.001f * g * g;
    m[p] = mm; v[p] = vv;
    w[p] -= lr * (mm / c1) / (sqrtf(vv / c2) + 1e-8f);
}

// ---- host side ---------------------------------------------------------------

template <class Real>
static int ml_alloc(Ctx<Real> &c) {
    const int n = c.n;
    if (!c.ml_w) {
        SPH_TRY(c.alloc(c.ml_w, ML_NPARAM));
        SPH_TRY(c.alloc(c.ml_m, ML_NPARAM));
        SPH_TRY(c.alloc(c.ml_v, ML_NPARAM));
        SPH_TRY(c.alloc(c.ml_grad, ML_NPARAM));
        SPH_TRY(c.alloc(c.ml_w1b, ML_H * ML_FP));
        SPH_TRY(c.alloc(c.ml_w2b, ML_H * ML_H));
        SPH_TRY(c.alloc(c.ml_sc, 8));   // MlScal
        SPH_TRY(c.alloc(c.ml_red, 6 * 1184 + 8));
        SPH_TRY(c.alloc(c.ml_cnt, 1));
        SPH_CUDA_TRY(cudaMemsetAsync(c.ml_w, 0, sizeof(float) * ML_NPARAM, c.stream));
        SPH_CUDA_TRY(cudaMemsetAsync(c.ml_cnt, 0, sizeof(unsigned int), c.stream));
    }
    if (!c.ml_X) {
        SPH_TRY(c.alloc(c.ml_X, (size_t)n * ML_FP));
        SPH_TRY(c.alloc(c.ml_y, n));
        SPH_TRY(c.alloc(c.ml_pold, n));
        SPH_TRY(c.alloc(c.ml_rr, n));
        SPH_TRY(c.alloc(c.ml_dd, n));
        SPH_TRY(c.alloc(c.ml_pprev, n));
        c.ml_have_prev = false;
    }
    return SPH_OK;
}

template <class Real>
__global__ void k_ml_snapshot(const Real *p, float *pold, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) pold[i] = (float)p[i];
}

// x += p_old - p_oldold on the rows that are solved for (kinds 1, 2, 3)
__global__ void k_ml_extrapolate(const int *kind, const float *pold, const float *pprev, double *x, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int kd = kind[i];
    if (kd >= 1 && kd <= 3) x[i] += (double)pold[i] - (double)pprev[i];
}

template <class Real>
int ml_extrapolate(Ctx<Real> &c, double *x) {
    if (!c.ml_have_prev) return SPH_OK;
    k_ml_extrapolate<<<grid_for(c.n, 256), 256, 0, c.stream>>>(c.row_kind, c.ml_pold, c.ml_pprev, x, c.n);
    ++c.launches;
    SPH_CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}

// features of the current step from b, A, the cached c_ij and p_old (with
// `features` false only the p_old snapshot for the history)
template <class Real>
int ml_prepare(Ctx<Real> &c, const Real *b, bool features) {
    SPH_TRY(ml_alloc(c));
    const int n = c.n;
    cudaStream_t st = c.stream;
    if (!features) {
        k_ml_snapshot<Real><<<grid_for(n, 256), 256, 0, st>>>(c.S.p, c.ml_pold, n);
        ++c.launches;
        SPH_CUDA_TRY(cudaGetLastError());
        return SPH_OK;
    }
    const int G = std::max(1, std::min((n + 255) / 256, 1184));
    if (sizeof(Real) == 4) {
        k_ml_residual<Real, float><<<grid_for(n, 256), 256, 0, st>>>(c.row_kind, c.slice_off, c.ncnt, c.nbr, c.coef, c.diag,
                                                                    b, c.S.p, c.ml_rr, c.ml_dd, c.ml_pold, n);
    } else {
        k_ml_residual<Real, double><<<grid_for(n, 256), 256, 0, st>>>(c.row_kind, c.slice_off, c.ncnt, c.nbr, c.coef_d,
                                                                     c.diag, b, c.S.p, c.ml_rr, c.ml_dd, c.ml_pold, n);
    }
    k_ml_scales<Real><<<G, 256, 0, st>>>(c.row_kind, c.ml_rr, c.ml_dd, b, c.ml_pold, n, c.ml_red, c.ml_cnt,
                                         (MlScal *)c.ml_sc);
    if (sizeof(Real) == 4)
        k_ml_features<Real, float><<<grid_for(n, 256), 256, 0, st>>>(c.row_kind, c.slice_off, c.ncnt, c.nbr, c.coef, c.diag,
                                                                    b, c.ml_rr, c.ml_dd, c.ml_pold,
                                                                    c.ml_have_prev ? c.ml_pprev : nullptr,
                                                                    (MlScal *)c.ml_sc, c.ml_X, n);
    else
        k_ml_features<Real, double><<<grid_for(n, 256), 256, 0, st>>>(c.row_kind, c.slice_off, c.ncnt, c.nbr, c.coef_d,
                                                                     c.diag, b, c.ml_rr, c.ml_dd, c.ml_pold,
                                                                     c.ml_have_prev ? c.ml_pprev : nullptr,
                                                                     (MlScal *)c.ml_sc, c.ml_X, n);
    c.launches += 3;
    SPH_CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}

// x += s_d * net(features) on the fluid rows
template <class Real>
int ml_warm_start(Ctx<Real> &c, const double *b, double *x, double *tmp) {
    const int n = c.n;
    cudaStream_t st = c.stream;
    if (!c.ml_zd) { SPH_TRY(c.alloc(c.ml_zd, n)); SPH_TRY(c.alloc(c.ml_wd, n)); }
    k_ml_infer<<<div_up(n, 128), 256, 0, st>>>(c.ml_X, nullptr, c.ml_w1b, c.ml_w2b, c.ml_w, c.ml_y, n);
    k_ml_dir<<<grid_for(n, 256), 256, 0, st>>>(c.row_kind, c.ml_y, (MlScal *)c.ml_sc, c.ml_zd, n);
    c.launches += 2;
    ppe_apply_fp64(c, x, tmp);          // M x0
    ppe_apply_fp64(c, c.ml_zd, c.ml_wd);   // M z
    const int G = std::max(1, std::min((n + 255) / 256, 1184));
    k_ml_alpha<<<G, 256, 0, st>>>(b, tmp, c.ml_wd, n, c.ml_red, c.ml_cnt, c.ml_sc + 6);
    k_ml_step<<<grid_for(n, 256), 256, 0, st>>>(c.ml_zd, c.ml_sc + 6, x, n);
    c.launches += 2;
    SPH_CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}

// ---- subspace start ---------------------------------------------------------
// x0 = p_old + W y over up to three columns: the previous step's pressure
// change (p_old - p_old of the step before), the coarse correction of the
// start residual (Z E^-1 Z^T r0) and the network's predicted change; y solves
// the projected system, Galerkin (W^T M W) y = W^T r0 or least squares
// (MW)^T (MW) y = (MW)^T r0.
constexpr int ML_SUB = 3;

__global__ void k_ml_hist_dir(const int *kind, const float *pold, const float *pprev, double *w, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) w[i] = kind[i] == 1 ? (double)pold[i] - (double)pprev[i] : 0.0;
}

__global__ void k_ml_resid(const double *b, const double *mx, double *r, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) r[i] = b[i] - mx[i];
}

// the k x k projected matrix and right-hand side (12 sums at most)
__global__ void __launch_bounds__(256) k_ml_sub_dots(const double *W, const double *MW, const double *r, int k,
                                                     int galerkin, int n, double *partials, unsigned int *counter,
                                                     double *out) {
    double v[ML_SUB * ML_SUB + ML_SUB];
#pragma unroll
    for (int q = 0; q < ML_SUB * ML_SUB + ML_SUB; ++q) v[q] = 0;
    const size_t ns = (size_t)n;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double a[ML_SUB], m[ML_SUB];
#pragma unroll
        for (int q = 0; q < ML_SUB; ++q) {
            a[q] = q < k ? (galerkin ? W[q * ns + i] : MW[q * ns + i]) : 0.0;
            m[q] = q < k ? MW[q * ns + i] : 0.0;
        }
        const double ri = r[i];
#pragma unroll
        for (int p = 0; p < ML_SUB; ++p) {
#pragma unroll
            for (int q = 0; q < ML_SUB; ++q) v[p * ML_SUB + q] += a[p] * m[q];
            v[ML_SUB * ML_SUB + p] += a[p] * ri;
        }
    }
    ml_reduce<ML_SUB * ML_SUB + ML_SUB>(v, partials, counter, [&](double *t) {
        for (int q = 0; q < ML_SUB * ML_SUB + ML_SUB; ++q) out[q] = t[q];
    });
}

// y of the k x k system by Gaussian elimination with partial pivoting (one
// thread); a pivot below 1e-14 of the largest diagonal entry drops that
// column (y = 0 for it)
__global__ void k_ml_sub_solve(double *sys, int k) {
    if (threadIdx.x || blockIdx.x) return;
    double A[ML_SUB][ML_SUB], g[ML_SUB], y[ML_SUB];
    int col[ML_SUB];
    double dmax = 0;
    for (int p = 0; p < k; ++p) {
        for (int q = 0; q < k; ++q) A[p][q] = sys[p * ML_SUB + q];
        g[p] = sys[ML_SUB * ML_SUB + p];
        dmax = fmax(dmax, fabs(A[p][p]));
        col[p] = 1;
    }
    for (int p = 0; p < k; ++p) {
        int piv = p;
        for (int q = p + 1; q < k; ++q)
            if (fabs(A[q][p]) > fabs(A[piv][p])) piv = q;
        if (!(fabs(A[piv][p]) > 1e-14 * dmax)) { col[p] = 0; continue; }
        if (piv != p) {
            for (int q = 0; q < k; ++q) { const double t = A[p][q]; A[p][q] = A[piv][q]; A[piv][q] = t; }
            const double t = g[p]; g[p] = g[piv]; g[piv] = t;
        }
        for (int q = p + 1; q < k; ++q) {
            const double f = A[q][p] / A[p][p];
            for (int r = p; r < k; ++r) A[q][r] -= f * A[p][r];
            g[q] -= f * g[p];
        }
    }
    for (int p = k - 1; p >= 0; --p) {
        if (!col[p]) { y[p] = 0; continue; }
        double t = g[p];
        for (int q = p + 1; q < k; ++q) t -= A[p][q] * y[q];
        y[p] = t / A[p][p];
        if (!isfinite(y[p])) y[p] = 0;
    }
    for (int p = 0; p < ML_SUB; ++p) sys[ML_SUB * ML_SUB + ML_SUB + p] = p < k ? y[p] : 0.0;
}

__global__ void k_ml_sub_update(const double *W, const double *y, int k, double *x, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double t = x[i];
    for (int q = 0; q < k; ++q) t += y[q] * W[(size_t)q * n + i];
    x[i] = t;
}

template <class Real>
int ml_subspace_start(Ctx<Real> &c, const double *b, double *x, double *tmp, bool with_net, bool galerkin) {
    const int n = c.n;
    cudaStream_t st = c.stream;
    if (!c.ml_W) {
        SPH_TRY(c.alloc(c.ml_W, (size_t)ML_SUB * n));
        SPH_TRY(c.alloc(c.ml_MW, (size_t)ML_SUB * n));
        SPH_TRY(c.alloc(c.ml_r0, (size_t)n));
        SPH_TRY(c.alloc(c.ml_subred, (size_t)(ML_SUB * ML_SUB + ML_SUB) * 1184 + 32));
        SPH_TRY(c.alloc(c.ml_subcnt, 1));
        SPH_CUDA_TRY(cudaMemsetAsync(c.ml_subcnt, 0, sizeof(unsigned int), st));
    }
    ppe_apply_fp64(c, x, tmp);
    k_ml_resid<<<grid_for(n, 256), 256, 0, st>>>(b, tmp, c.ml_r0, n);
    ++c.launches;
    int k = 0;
    if (c.ml_have_prev) {
        k_ml_hist_dir<<<grid_for(n, 256), 256, 0, st>>>(c.row_kind, c.ml_pold, c.ml_pprev, c.ml_W + (size_t)k * n, n);
        ++c.launches;
        ++k;
    }
    if (c.cg_m > 0) {
        double *w = c.ml_W + (size_t)k * n;
        SPH_CUDA_TRY(cudaMemsetAsync(w, 0, sizeof(double) * n, st));
        coarse_apply<Real, double>(c, c.ml_r0, w);
        ++k;
    }
    if (with_net) {
        k_ml_infer<<<div_up(n, 128), 256, 0, st>>>(c.ml_X, nullptr, c.ml_w1b, c.ml_w2b, c.ml_w, c.ml_y, n);
        k_ml_dir<<<grid_for(n, 256), 256, 0, st>>>(c.row_kind, c.ml_y, (MlScal *)c.ml_sc, c.ml_W + (size_t)k * n, n);
        c.launches += 2;
        ++k;
    }
    if (k == 0) return SPH_OK;
    for (int q = 0; q < k; ++q) ppe_apply_fp64(c, c.ml_W + (size_t)q * n, c.ml_MW + (size_t)q * n);
    const int G = std::max(1, std::min((n + 255) / 256, 1184));
    double *sys = c.ml_subred + (size_t)(ML_SUB * ML_SUB + ML_SUB) * 1184;
    k_ml_sub_dots<<<G, 256, 0, st>>>(c.ml_W, c.ml_MW, c.ml_r0, k, galerkin ? 1 : 0, n, c.ml_subred, c.ml_subcnt, sys);
    k_ml_sub_solve<<<1, 32, 0, st>>>(sys, k);
    k_ml_sub_update<<<grid_for(n, 256), 256, 0, st>>>(c.ml_W, sys + ML_SUB * ML_SUB + ML_SUB, k, x, n);
    c.launches += 3;
    SPH_CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}

// samples of a converged solve: every k-th fluid row, offset rotating per step
template <class Real>
int ml_collect(Ctx<Real> &c, const double *xnew) {
    const int k = c.ml_every;
    if (k <= 0) return SPH_OK;
    if (!c.ml_SX) {
        c.ml_cap = ML_CAP_DEFAULT;
        SPH_TRY(c.alloc(c.ml_SX, (size_t)c.ml_cap * ML_FP));
        SPH_TRY(c.alloc(c.ml_St, (size_t)c.ml_cap));
        c.ml_count = 0;
    }
    if (!c.ml_fluid) {
        std::vector<int> kind(c.n), fl;
        SPH_CUDA_TRY(cudaMemcpyAsync(kind.data(), c.row_kind, sizeof(int) * c.n, cudaMemcpyDeviceToHost, c.stream));
        SPH_CUDA_TRY(cudaStreamSynchronize(c.stream));
        for (int i = 0; i < c.n; ++i)
            if (kind[i] == 1) fl.push_back(i);
        c.ml_nfluid = (int)fl.size();
        SPH_TRY(c.alloc(c.ml_fluid, std::max<size_t>(fl.size(), 1)));
        if (!fl.empty())
            SPH_CUDA_TRY(cudaMemcpyAsync(c.ml_fluid, fl.data(), sizeof(int) * fl.size(), cudaMemcpyHostToDevice, c.stream));
        SPH_CUDA_TRY(cudaStreamSynchronize(c.stream));
        c.ml_phase = 0;
    }
    const int nf = c.ml_nfluid;
    const int off = c.ml_phase % k;
    c.ml_phase++;
    const int nsel = nf > off ? (nf - off + k - 1) / k : 0;
    const long long room = c.ml_cap - c.ml_count;
    const int take = (int)std::min<long long>(nsel, room);
    if (take <= 0) return SPH_OK;
    k_ml_collect<<<grid_for(take, 256), 256, 0, c.stream>>>(c.ml_fluid, off, k, take, c.ml_X, c.ml_pold, xnew,
                                                          (MlScal *)c.ml_sc, c.ml_SX, c.ml_St, c.ml_count);
    ++c.launches;
    SPH_CUDA_TRY(cudaGetLastError());
    c.ml_count += take;
    return SPH_OK;
}

// after the solve: this step's p_old becomes the history of the next step
template <class Real>
int ml_finish_step(Ctx<Real> &c) {
    if (!c.ml_pold) return SPH_OK;
    SPH_CUDA_TRY(cudaMemcpyAsync(c.ml_pprev, c.ml_pold, sizeof(float) * c.n, cudaMemcpyDeviceToDevice, c.stream));
    c.ml_have_prev = true;
    return SPH_OK;
}

template <class Real>
int ml_pack(Ctx<Real> &c) {
    k_ml_pack<<<div_up(ML_H * ML_H, 256), 256, 0, c.stream>>>(c.ml_w, c.ml_w1b, c.ml_w2b);
    ++c.launches;
    SPH_CUDA_TRY(cudaGetLastError());
    c.ml_ready = true;
    return SPH_OK;
}

// loss and gradient over samples [first, first + rows) or the listed ones
template <class Real>
static int ml_grad_dev(Ctx<Real> &c, const int *idx, long long first, int rows, float *loss_out) {
    const int nb = div_up(rows, ML_ROWS_TRAIN);
    if (c.ml_part_cap < nb) {
        c.release(c.ml_part); c.release(c.ml_lpart);
        SPH_TRY(c.alloc(c.ml_part, (size_t)nb * ML_NPARAM));
        SPH_TRY(c.alloc(c.ml_lpart, nb));
        c.ml_part_cap = nb;
    }
    const size_t smem = ml_train_smem();
    SPH_CUDA_TRY(cudaFuncSetAttribute(k_ml_fwd_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_ml_fwd_bwd<<<nb, 256, smem, c.stream>>>(c.ml_SX, c.ml_St, idx, first, rows, c.ml_w, 1.0f / (float)rows, c.ml_part,
                                              c.ml_lpart);
    k_ml_reduce<<<div_up(ML_NPARAM, 256), 256, 0, c.stream>>>(c.ml_part, nb, c.ml_grad);
    c.launches += 2;
    SPH_CUDA_TRY(cudaGetLastError());
    if (loss_out) {
        std::vector<float> lp(nb);
        SPH_CUDA_TRY(cudaMemcpyAsync(lp.data(), c.ml_lpart, sizeof(float) * nb, cudaMemcpyDeviceToHost, c.stream));
        SPH_CUDA_TRY(cudaStreamSynchronize(c.stream));
        double s = 0;
        for (float v : lp) s += v;
        *loss_out = (float)(s / rows);
    }
    return SPH_OK;
}

template <class Real>
int ml_grad(Ctx<Real> &c, long long first, int rows, float *loss, float *grad) {
    if (!c.ml_SX || first < 0 || rows <= 0 || first + rows > c.ml_count) {
        set_error("sph_ml_grad: sample range outside the collected samples");
        return SPH_ERR_BAD_ARG;
    }
    SPH_TRY(ml_alloc(c));
    SPH_TRY(ml_grad_dev(c, nullptr, first, rows, loss));
    if (grad) {
        SPH_CUDA_TRY(cudaMemcpyAsync(grad, c.ml_grad, sizeof(float) * ML_NPARAM, cudaMemcpyDeviceToHost, c.stream));
        SPH_CUDA_TRY(cudaStreamSynchronize(c.stream));
    }
    return SPH_OK;
}

template <class Real>
int ml_train(Ctx<Real> &c, int epochs, int batch, float lr, unsigned long long seed, float *final_loss) {
    if (!c.ml_SX || c.ml_count < batch || batch <= 0 || epochs <= 0) {
        set_error("sph_ml_train: fewer collected samples than one batch");
        return SPH_ERR_STATE;
    }
    SPH_TRY(ml_alloc(c));
    const long long N = c.ml_count;
    // deterministic initialisation (He-uniform from the seed) unless weights were set
    if (!c.ml_init) {
        std::mt19937_64 g(seed);
        std::uniform_real_distribution<float> U(-1.f, 1.f);
        std::vector<float> w(ML_NPARAM, 0.f);
        for (int t = 0; t < ML_F * ML_H; ++t) w[ML_OW1 + t] = U(g) * std::sqrt(6.f / ML_F);
        for (int t = 0; t < ML_H * ML_H; ++t) w[ML_OW2 + t] = U(g) * std::sqrt(6.f / ML_H);
        for (int t = 0; t < ML_H; ++t) w[ML_OW3 + t] = U(g) * std::sqrt(1.f / ML_H);
        SPH_CUDA_TRY(cudaMemcpyAsync(c.ml_w, w.data(), sizeof(float) * ML_NPARAM, cudaMemcpyHostToDevice, c.stream));
        c.ml_init = true;
    }
    SPH_CUDA_TRY(cudaMemsetAsync(c.ml_m, 0, sizeof(float) * ML_NPARAM, c.stream));
    SPH_CUDA_TRY(cudaMemsetAsync(c.ml_v, 0, sizeof(float) * ML_NPARAM, c.stream));
    int *idx = nullptr;
    SPH_TRY(c.alloc(idx, (size_t)N));
    std::vector<int> perm(N);
    std::mt19937_64 g(seed ^ 0x9e3779b97f4a7c15ull);
    int t = 0;
    float loss = 0.f;
    for (int ep = 0; ep < epochs; ++ep) {
        for (long long q = 0; q < N; ++q) perm[q] = (int)q;
        std::shuffle(perm.begin(), perm.end(), g);
        SPH_CUDA_TRY(cudaMemcpyAsync(idx, perm.data(), sizeof(int) * N, cudaMemcpyHostToDevice, c.stream));
        for (long long q = 0; q + batch <= N; q += batch) {
            ++t;
            SPH_TRY(ml_grad_dev(c, idx, q, batch, nullptr));
            const float c1 = 1.f - std::pow(0.9f, (float)t), c2 = 1.f - std::pow(0.999f, (float)t);
            k_ml_adam<<<div_up(ML_NPARAM, 256), 256, 0, c.stream>>>(c.ml_w, c.ml_m, c.ml_v, c.ml_grad, lr, c1, c2);
            ++c.launches;
        }
        SPH_CUDA_TRY(cudaStreamSynchronize(c.stream));   // perm is rewritten next epoch
    }
    // loss over the first min(N, 65536) samples with the final weights
    SPH_TRY(ml_grad_dev(c, nullptr, 0, (int)std::min<long long>(N, 65536), &loss));
    c.release(idx);
    if (final_loss) *final_loss = loss;
    return ml_pack(c);
}

template <class Real>
int ml_set_weights(Ctx<Real> &c, const float *w) {
    SPH_TRY(ml_alloc(c));
    SPH_CUDA_TRY(cudaMemcpyAsync(c.ml_w, w, sizeof(float) * ML_NPARAM, cudaMemcpyHostToDevice, c.stream));
    c.ml_init = true;
    return ml_pack(c);
}

template <class Real>
int ml_get_weights(Ctx<Real> &c, float *w) {
    SPH_TRY(ml_alloc(c));
    SPH_CUDA_TRY(cudaMemcpyAsync(w, c.ml_w, sizeof(float) * ML_NPARAM, cudaMemcpyDeviceToHost, c.stream));
    SPH_CUDA_TRY(cudaStreamSynchronize(c.stream));
    return SPH_OK;
}

template <class Real>
int ml_samples(Ctx<Real> &c, long long first, long long rows, uint16_t *X, float *t, long long *count) {
    if (count) *count = c.ml_count;
    if (rows <= 0 || (!X && !t)) return SPH_OK;
    if (first < 0 || first + rows > c.ml_count) {
        set_error("sph_ml_samples: range outside the collected samples");
        return SPH_ERR_BAD_ARG;
    }
    if (X) SPH_CUDA_TRY(cudaMemcpyAsync(X, c.ml_SX + first * ML_FP, sizeof(uint16_t) * rows * ML_FP, cudaMemcpyDeviceToHost,
                                        c.stream));
    if (t) SPH_CUDA_TRY(cudaMemcpyAsync(t, c.ml_St + first, sizeof(float) * rows, cudaMemcpyDeviceToHost, c.stream));
    SPH_CUDA_TRY(cudaStreamSynchronize(c.stream));
    return SPH_OK;
}

// tensor-core inference on collected samples (checks the BF16 path)
template <class Real>
int ml_predict_samples(Ctx<Real> &c, long long first, int rows, float *y) {
    if (!c.ml_ready) { set_error("sph_ml_predict_samples: no weights"); return SPH_ERR_STATE; }
    if (first < 0 || rows <= 0 || first + rows > c.ml_count) {
        set_error("sph_ml_predict_samples: range outside the collected samples");
        return SPH_ERR_BAD_ARG;
    }
    float *dy = nullptr;
    SPH_TRY(c.alloc(dy, rows));
    k_ml_infer<<<div_up(rows, 128), 256, 0, c.stream>>>(c.ml_SX + first * ML_FP, nullptr, c.ml_w1b, c.ml_w2b, c.ml_w, dy,
                                                        rows);
    ++c.launches;
    SPH_CUDA_TRY(cudaGetLastError());
    SPH_CUDA_TRY(cudaMemcpyAsync(y, dy, sizeof(float) * rows, cudaMemcpyDeviceToHost, c.stream));
    SPH_CUDA_TRY(cudaStreamSynchronize(c.stream));
    c.release(dy);
    return SPH_OK;
}

#define INST(R)                                                                                          \
    template int ml_prepare<R>(Ctx<R> &, const R *, bool);                                               \
    template int ml_extrapolate<R>(Ctx<R> &, double *);                                                  \
    template int ml_warm_start<R>(Ctx<R> &, const double *, double *, double *);                         \
    template int ml_subspace_start<R>(Ctx<R> &, const double *, double *, double *, bool, bool);         \
    template int ml_finish_step<R>(Ctx<R> &);                                                            \
    template int ml_collect<R>(Ctx<R> &, const double *);                                                \
    template int ml_grad<R>(Ctx<R> &, long long, int, float *, float *);                                 \
    template int ml_train<R>(Ctx<R> &, int, int, float, unsigned long long, float *);                    \
    template int ml_set_weights<R>(Ctx<R> &, const float *);                                             \
    template int ml_get_weights<R>(Ctx<R> &, float *);                                                   \
    template int ml_samples<R>(Ctx<R> &, long long, long long, uint16_t *, float *, long long *);        \
    template int ml_predict_samples<R>(Ctx<R> &, long long, int, float *);
INST(float)
INST(double)
#undef INST

}  // namespace sph
