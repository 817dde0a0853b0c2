// Two-level preconditioner of the converged pressure solve: Jacobi plus an
// additive coarse correction on aggregates of B x B x B NNPS cells (or
// balanced octree boxes, ppe_coarse_block = -B),
//     M^-1 r = D^-1 r + Z E^-1 Z^T r,   E = Z^T M Z,
// with Z the indicator vectors of the aggregates (every row of the operator
// except identity / pinned rows belongs to exactly one) and M the converged
// operator of ppe.cu (difference-form fluid rows, Neumann rows with their
// operator weights, outlet copies, rank-one mean-pressure term).
//
// The particles never move, so the aggregates, E and its inverse are built
// once per neighbour-list build.  Jacobi alone needs O(L/h) BiCGSTAB
// iterations (the smooth modes); the coarse space removes the modes longer
// than the aggregate size, which also keeps FP32 Krylov vectors accurate
// enough for the mixed form.
//
// Determinism: E is accumulated in 64-bit fixed point (integer atomics are
// order-independent), every reduction has a fixed order, and the inverse is
// a blocked Gauss-Jordan with partial pivoting in a fixed sequence of
// launches (panel sweeps, then FP64 rank-64 updates with a fixed summation
// order), checked on four of its columns.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "ctx.cuh"
#include "octree.h"

namespace sph {

constexpr int kCoarseMaxAgg = 32768;      // the dense inverse holds m^2 entries
constexpr int kCoarseDefaultAgg = 4096;   // balanced aggregates without ppe_coarse_max
constexpr int kCoarsePiece = 1024;   // rows per block of the restriction

// deterministic block sum (fixed shuffle pattern, warps summed in order)
template <int NT>
__device__ __forceinline__ double block_sum(double v, double *sh) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double t = 0;
    if (threadIdx.x == 0)
        for (int w = 0; w < NT / 32; ++w) t += sh[w];
    __syncthreads();
    return t;   // valid on thread 0
}

// ---- set-up -------------------------------------------------------------------

// largest |c_ij| over the stored entries of the fluid rows (non-negative
// doubles order like their bit patterns, so an integer max is exact)
template <class C>
__global__ void k_coef_absmax(const int *kind, const long long *slice_off, const int *ncnt, const C *coef, int n,
                              unsigned long long *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double m = 0;
    if (i < n && kind[i] == 1) {
        const long long base = slice_off[i >> 5] + (i & 31);
        for (int k = 0; k < ncnt[i]; ++k) m = fmax(m, fabs((double)coef[sell4(base - (i & 31), i & 31, k)]));
    }
    if (m > 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// one block per aggregate I: row I of E = Z^T M Z in fixed point, and the
// sums of A_i of I's fluid rows per rank-one component
template <class C, class Real>
__global__ void __launch_bounds__(256) k_coarse_assemble(
    int m, const int *agg, const int *off, const int *rows, const int *kind, const int *aux,
    const long long *slice_off, const int *ncnt, const int *nbr, const C *coef, const int *nm_idx, const int *nm_off,
    const int *nm_nbr, const double *nm_ow, const int *comp_id, const Real *diag, int ncomp, double scale, double *E,
    double *a_comp, bool in_smem) {
    // row I of E accumulates in shared memory, or (m too large for it) in
    // its own row of E, read as 64-bit integers; only block I touches row I
    extern __shared__ unsigned long long acc_sh[];
    __shared__ double sh[8];
    const int I = blockIdx.x;
    unsigned long long *acc = in_smem ? acc_sh : reinterpret_cast<unsigned long long *>(E + (size_t)I * m);
    for (int J = threadIdx.x; J < m; J += blockDim.x) acc[J] = 0ull;
    __syncthreads();
    double asum[SPH_MAX_COMP];
#pragma unroll
    for (int q = 0; q < SPH_MAX_COMP; ++q) asum[q] = 0;
    auto add = [&](int J, double v) {
        atomicAdd(&acc[J], (unsigned long long)llrint(v * scale));
    };
    // (M z_J)_i for i in I: sum over the row's entries of w (z_i - z_j)
    auto couple = [&](int j, double w) {
        const int J = (j >= 0) ? agg[j] : -1;
        if (J == I) return;
        add(I, w);
        if (J >= 0) add(J, -w);
    };
    for (int q = off[I] + threadIdx.x; q < off[I + 1]; q += blockDim.x) {
        const int i = rows[q];
        const int kd = kind[i];
        if (kd == 1) {
            const long long base = slice_off[i >> 5] + (i & 31);
            const int cnt = ncnt[i];
            for (int k = 0; k < cnt; ++k) {
                const long long e = base + 32LL * k;
                couple(nbr[e], (double)coef[sell4(base - (i & 31), i & 31, k)]);
            }
            const int cc = comp_id ? comp_id[i] : -1;
#pragma unroll
            for (int t = 0; t < SPH_MAX_COMP; ++t)
                if (cc == t) asum[t] += (double)diag[i];
        } else if (kd == 2) {
            const int r = nm_idx[i];   // a row without a Neumann entry stays the identity
            const int q0 = r >= 0 ? nm_off[r] : 0, q1 = r >= 0 ? nm_off[r + 1] : 0;
            if (q1 == q0) add(I, 1.0);
            for (int qq = q0; qq < q1; ++qq) couple(nm_nbr[qq], nm_ow[qq]);
        } else if (kd == 3) {
            const int pj = aux[i];
            if (pj < 0) add(I, 1.0);
            else couple(pj, 1.0);
        }
    }
    __syncthreads();
    for (int J = threadIdx.x; J < m; J += blockDim.x) {
        const unsigned long long a = in_smem ? acc[J] : __ldcg(acc + J);
        E[(size_t)I * m + J] = (double)(long long)a / scale;
    }
    for (int t = 0; t < ncomp; ++t) {
        const double s = block_sum<256>(asum[t], sh);
        if (threadIdx.x == 0) a_comp[(size_t)I * ncomp + t] = s;
    }
}

// rank-one part: E_IJ += sum_c a_comp[I][c] * |J in c| / |c|
__global__ void k_coarse_rank_one(double *E, const double *a_comp, const int *cnt_comp, const double *comp_inv, int m,
                                  int ncomp) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)m * m) return;
    const int I = (int)(t / m), J = (int)(t % m);
    double v = 0;
    for (int c = 0; c < ncomp; ++c) v += a_comp[(size_t)I * ncomp + c] * (double)cnt_comp[(size_t)J * ncomp + c] * comp_inv[c];
    E[t] += v;
}

// pivot of column k: the row r >= k of largest |W[r,k]| (ties: the lowest
// row), its value, and the error flag when the column is zero from row k down
__global__ void k_gj_pivot(const double *W, int m, int k, int *piv, double *pval, int *err) {
    __shared__ double bv[32];
    __shared__ int bi[32];
    double best = -1;
    int idx = -1;
    for (int r = k + threadIdx.x; r < m; r += blockDim.x) {
        const double v = fabs(W[(size_t)r * m + k]);
        if (v > best) { best = v; idx = r; }
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, idx, o);
        if (ov > best || (ov == best && oi >= 0 && (idx < 0 || oi < idx))) { best = ov; idx = oi; }
    }
    if (lane == 0) { bv[wid] = best; bi[wid] = idx; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = -1;
        int p = -1;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
            if (bv[w] > b || (bv[w] == b && bi[w] >= 0 && (p < 0 || bi[w] < p))) { b = bv[w]; p = bi[w]; }
        if (!(b > 0) || p < 0) { *err = 1; p = k; }
        *piv = p;
        *pval = W[(size_t)p * m + k];
    }
}

// ---- blocked in-place Gauss-Jordan inverse ------------------------------------
// W (m x m, row-major, FP64) is inverted in place with partial pivoting, in
// panels of kGjPanel columns.  Within a panel each pivot column k is swept as
// the classical in-place Gauss-Jordan step restricted to the panel's columns
// (rows swapped and the pivot row scaled in the panel, every other row
// eliminated in the panel).  After the panel, with K its pivot rows, R the
// other rows and J the columns outside it, the block sweep
//     A_KJ <- A_KK^-1 A_KJ,   A_RJ <- A_RJ - A_RK A_KK^-1 A_KJ
// is W[:, J] <- (rows K zeroed) W[:, J] + N Bk, with N the panel's swept
// columns (A_KK^-1 in rows K, -A_RK A_KK^-1 in rows R) and Bk the pivot
// rows of the other columns before the sweep: one rank-kGjPanel update in
// FP64 (tiled, fixed summation order), after the panel's row swaps have
// been applied to the other columns.  The row interchanges leave the
// inverse's columns permuted; the FP32 copy gathers them back.
constexpr int kGjPanel = 64;

// panel step k: row k takes the pivot row's panel values (the pivot row
// takes row k's), scaled by 1 / pivot, with 1 / pivot in column k
__global__ void k_gj_pivot_row(double *W, int m, int k, int k0, int kb, const int *piv, const double *pval,
                               const int *err) {
    const int t = threadIdx.x;
    if (t >= kb || *err) return;
    const int p = *piv, c = k0 + t;
    const double a = W[(size_t)k * m + c], b = W[(size_t)p * m + c];
    if (p != k) W[(size_t)p * m + c] = a;
    const double inv = 1.0 / *pval;
    W[(size_t)k * m + c] = (c == k) ? inv : b * inv;
}

// panel step k, every row i != k (one warp per row): f = W[i,k];
// W[i,c] -= f W[k,c] in the panel, W[i,k] = -f / pivot
__global__ void k_gj_panel_elim(double *W, int m, int k, int k0, int kb, const int *err) {
    const int i = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= m || i == k || *err) return;   // uniform over the warp
    double *row = W + (size_t)i * m + k0;
    const double *rk = W + (size_t)k * m + k0;
    const double f = row[k - k0];
    __syncwarp();
    if (f == 0.0) return;
    for (int c = lane; c < kb; c += 32) {
        if (k0 + c == k) row[c] = -f * rk[c];
        else row[c] -= f * rk[c];
    }
}

// the panel's row interchanges, in order, in every column outside it
__global__ void k_gj_swap_rows(double *W, int m, int k0, int kb, const int *piv, const int *err) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m || (j >= k0 && j < k0 + kb) || *err) return;
    for (int t = 0; t < kb; ++t) {
        const int k = k0 + t, p = piv[k];
        if (p == k) continue;
        const double a = W[(size_t)k * m + j];
        W[(size_t)k * m + j] = W[(size_t)p * m + j];
        W[(size_t)p * m + j] = a;
    }
}

// Bk = the panel's pivot rows (kb x m)
__global__ void k_gj_copy_rows(const double *W, double *Bk, int m, int k0, int kb) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)kb * m) return;
    const int r = (int)(t / m), j = (int)(t % m);
    Bk[t] = W[(size_t)(k0 + r) * m + j];
}

// W[i,j] = (i a pivot row of the panel ? 0 : W[i,j]) + sum_t W[i,k0+t] Bk[t,j]
// for every column j outside the panel: 64 x 64 tiles, 4 x 4 per thread,
// t ascending in chunks of 32
__global__ void __launch_bounds__(256) k_gj_update(double *W, const double *__restrict__ Bk, int m, int k0, int kb,
                                                   const int *err) {
    __shared__ double Ns[64][33];
    __shared__ double Bs[32][64];
    const int j0 = blockIdx.x * 64, i0 = blockIdx.y * 64;
    if (j0 == k0 || *err) return;   // panels start at multiples of 64: this tile is the panel
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    double acc[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[r][q] = 0.0;
    for (int t0 = 0; t0 < kb; t0 += 32) {
        for (int e = threadIdx.x; e < 64 * 32; e += 256) {
            const int r = e >> 5, t = e & 31;
            const int i = i0 + r;
            Ns[r][t] = (i < m && t0 + t < kb) ? W[(size_t)i * m + k0 + t0 + t] : 0.0;
        }
        for (int e = threadIdx.x; e < 32 * 64; e += 256) {
            const int t = e >> 6, q = e & 63;
            const int j = j0 + q;
            Bs[t][q] = (j < m && t0 + t < kb) ? Bk[(size_t)(t0 + t) * m + j] : 0.0;
        }
        __syncthreads();
#pragma unroll 8
        for (int t = 0; t < 32; ++t) {
            double a[4], b[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) a[r] = Ns[ty * 4 + r][t];
#pragma unroll
            for (int q = 0; q < 4; ++q) b[q] = Bs[t][tx + 16 * q];
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[r][q] = fma(a[r], b[q], acc[r][q]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int i = i0 + ty * 4 + r;
        if (i >= m) continue;
        const bool pivot_row = i >= k0 && i < k0 + kb;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int j = j0 + tx + 16 * q;
            if (j >= m) continue;
            double *w = W + (size_t)i * m + j;
            *w = (pivot_row ? 0.0 : *w) + acc[r][q];
        }
    }
}

// FP32 copy of the inverse with its columns put back: column c of the
// inverse is column col[c] of W
__global__ void k_gj_to_float(const double *W, const int *col, float *out, int m) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)m * m) return;
    const int i = (int)(t / m), c = (int)(t % m);
    out[t] = (float)W[(size_t)i * m + col[c]];
}

// check of the inverse on a few of its columns: dev[q] = max_i |(E X)_ic - delta_ic|
// for c = cols[q] (one warp per row i, X[:, c] = W[:, col[c]])
__global__ void k_gj_check(const double *E, const double *W, const int *col, const int *cols, int ncheck, int m,
                           unsigned long long *dev) {
    const int i = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= m) return;
    for (int q = 0; q < ncheck; ++q) {
        const int c = cols[q], wc = col[c];
        double v = 0;
        for (int j = lane; j < m; j += 32) v += E[(size_t)i * m + j] * W[(size_t)j * m + wc];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) {
            const double d = fabs(v - (i == c ? 1.0 : 0.0));
            atomicMax(dev, (unsigned long long)__double_as_longlong(d == d ? d : 1e300));
        }
    }
}

// ---- application ----------------------------------------------------------

// s_I = sum over the rows of aggregate I of r (minus w when given).  The
// rows of every aggregate are cut into pieces of at most kCoarsePiece
// entries, one block per piece, so the launch has enough blocks to hide the
// gathers however few the aggregates; the last block of an aggregate to
// finish sums its pieces' partials in piece order, so the result does not
// depend on the order the blocks run in.
template <class V>
__global__ void __launch_bounds__(256) k_coarse_restrict(const int *__restrict__ piece, const int *__restrict__ pfirst,
                                                         const int *__restrict__ rows, const V *r, const V *w,
                                                         double *part, unsigned int *cnt, double *s) {
    __shared__ double sh[8];
    const int p = blockIdx.x;
    const int I = piece[3 * p], q0 = piece[3 * p + 1], q1 = piece[3 * p + 2];
    double v = 0;
    if (w)
        for (int q = q0 + threadIdx.x; q < q1; q += blockDim.x) { const int i = rows[q]; v += (double)(r[i] - w[i]); }
    else
        for (int q = q0 + threadIdx.x; q < q1; q += blockDim.x) v += (double)r[rows[q]];
    v = block_sum<256>(v, sh);
    if (threadIdx.x != 0) return;
    const int p0 = pfirst[I], np = pfirst[I + 1] - p0;
    if (np == 1) { s[I] = v; return; }
    part[p] = v;
    __threadfence();
    if (atomicAdd(&cnt[I], 1u) != (unsigned)(np - 1)) return;
    __threadfence();
    double t = 0;
    for (int k = 0; k < np; ++k) t += __ldcg(part + p0 + k);
    s[I] = t;
    cnt[I] = 0;
}

// y = E^-1 s, one warp per row; E^-1 is stored in FP32 (a preconditioner
// needs no more, and the m^2 matrix is the largest read of an application)
__global__ void __launch_bounds__(256) k_coarse_solve(const float *__restrict__ Inv, const double *__restrict__ s,
                                                      double *__restrict__ y, int m) {
    const int I = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (I >= m) return;
    const float *row = Inv + (size_t)I * m;
    double v = 0;
    for (int J = lane; J < m; J += 32) v += (double)row[J] * s[J];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) y[I] = v;
}

template <class V>
__global__ void k_coarse_add(const int *agg, const double *y, V *z, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int a = agg[i];
    if (a >= 0) z[i] += (V)y[a];
}

template <class Real, class V>
void coarse_restrict_solve(Ctx<Real> &c, const V *r, const V *w) {
    const int m = c.cg_m;
    k_coarse_restrict<V><<<c.cg_np, 256, 0, c.stream>>>(c.cg_piece, c.cg_pfirst, c.cg_rows, r, w, c.cg_part, c.cg_cnt,
                                                        c.cg_s);
    k_coarse_solve<<<div_up((long long)m * 32, 256), 256, 0, c.stream>>>(c.cg_invf, c.cg_s, c.cg_y, m);
    c.launches += 2;
}

template <class Real, class V>
void coarse_apply(Ctx<Real> &c, const V *r, V *z, const V *w) {
    if (c.cg_m <= 0) return;
    const int m = c.cg_m;
    k_coarse_restrict<V><<<c.cg_np, 256, 0, c.stream>>>(c.cg_piece, c.cg_pfirst, c.cg_rows, r, w, c.cg_part, c.cg_cnt,
                                                        c.cg_s);
    k_coarse_solve<<<div_up((long long)m * 32, 256), 256, 0, c.stream>>>(c.cg_invf, c.cg_s, c.cg_y, m);
    k_coarse_add<V><<<grid_for(c.n, 256), 256, 0, c.stream>>>(c.cg_agg, c.cg_y, z, c.n);
    c.launches += 3;
}

template <class Real>
int coarse_build(Ctx<Real> &c) {
    const int B = c.prm.ppe_coarse_block;
    c.cg_valid = true;
    c.cg_block = B;
    c.cg_max = c.prm.ppe_coarse_max;
    c.cg_m = 0;
    if (B == 0) return SPH_OK;
    const int n = c.n;
    cudaStream_t st = c.stream;
    // host copies of what the aggregation needs
    std::vector<int> kind(n), ncnt(n), comp(n, -1), aux(n);
    std::vector<float4> pos(n);
    SPH_CUDA_TRY(cudaMemcpyAsync(kind.data(), c.row_kind, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
    SPH_CUDA_TRY(cudaMemcpyAsync(aux.data(), c.row_aux, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
    SPH_CUDA_TRY(cudaMemcpyAsync(ncnt.data(), c.ncnt, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
    SPH_CUDA_TRY(cudaMemcpyAsync(pos.data(), c.pf, sizeof(float4) * n, cudaMemcpyDeviceToHost, st));
    if (c.n_comp > 0) SPH_CUDA_TRY(cudaMemcpyAsync(comp.data(), c.comp_id, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
    const int nnm = c.L.n_nm;
    std::vector<int> nm_rows(nnm);
    if (nnm > 0) SPH_CUDA_TRY(cudaMemcpyAsync(nm_rows.data(), c.L.nm_rows, sizeof(int) * nnm, cudaMemcpyDeviceToHost, st));
    SPH_CUDA_TRY(cudaStreamSynchronize(st));

    // aggregates: blocks of B^3 cells of the binning grid, numbered in order
    // of their first row (rows ascending), identity and pinned rows excluded.
    // A copy row (outlet partner, periodic ghost) joins its partner's block,
    // so that every coarse vector satisfies the copy rows exactly: a ghost
    // and the interior record it mirrors across the box share an aggregate.
    const DevParams &P = c.dp;
    const int Bb = B > 0 ? B : -B;
    auto member = [&](int k) { return kind[k] == 1 || kind[k] == 2 || kind[k] == 3; };
    std::vector<int> cell, mrow;   // cell coordinates and row of each member
    cell.reserve(3 * (size_t)n);
    for (int i = 0; i < n; ++i) {
        if (!member(i)) continue;
        int src = i;
        if (kind[i] == 3 && aux[i] >= 0 && aux[i] < n && member(aux[i])) src = aux[i];
        cell.push_back(bin_axis(pos[src].x, P.xmin, P.xmax, P.NI));
        cell.push_back(bin_axis(pos[src].y, P.ymin, P.ymax, P.NJ));
        cell.push_back(bin_axis(pos[src].z, P.zmin, P.zmax, P.NK));
        mrow.push_back(i);
    }
    const int nmem = (int)mrow.size();
    std::vector<int> box(nmem);   // block (B > 0) or balanced box (B < 0) of each member
    if (B > 0) {
        const int NBx = (P.NI + Bb - 1) / Bb, NBy = (P.NJ + Bb - 1) / Bb;
        for (int k = 0; k < nmem; ++k)
            box[k] = ((cell[3 * k + 2] / Bb) * NBy + cell[3 * k + 1] / Bb) * NBx + cell[3 * k] / Bb;
    } else {
        const int cap = c.prm.ppe_coarse_max > 0 ? std::min(c.prm.ppe_coarse_max, kCoarseMaxAgg) : kCoarseDefaultAgg;
        box = octree_aggregates(cell, nmem, Bb, P.NI, P.NJ, P.NK, cap);
    }
    // aggregates numbered in order of their first row (rows ascending)
    std::vector<int> agg(n, -1), size;
    std::unordered_map<int, int> number;
    int m = 0;
    for (int k = 0; k < nmem; ++k) {
        auto it = number.find(box[k]);
        int a;
        if (it == number.end()) { a = m++; number.emplace(box[k], a); size.push_back(0); }
        else a = it->second;
        agg[mrow[k]] = a;
        ++size[a];
    }
    if (m > kCoarseMaxAgg) {
        char msg[160];
        snprintf(msg, sizeof msg, "ppe_coarse_block %d gives %d aggregates (max %d): use a larger block", B, m, kCoarseMaxAgg);
        set_error(msg);
        return SPH_ERR_UNSUPPORTED;
    }
    if (m == 0) return SPH_OK;
    std::vector<int> off(m + 1, 0);
    for (int a = 0; a < m; ++a) off[a + 1] = off[a] + size[a];
    std::vector<int> rows(std::max(off[m], 1), 0), fill(off.begin(), off.end() - 1);
    for (int i = 0; i < n; ++i)
        if (agg[i] >= 0) rows[fill[agg[i]]++] = i;
    std::vector<int> nm_idx(n, -1);
    for (int k = 0; k < nnm; ++k) nm_idx[nm_rows[k]] = k;
    const int ncomp = c.n_comp;
    std::vector<int> cnt_comp((size_t)m * std::max(ncomp, 1), 0);
    for (int i = 0; i < n; ++i)
        if (agg[i] >= 0 && kind[i] == 1 && comp[i] >= 0 && comp[i] < ncomp) ++cnt_comp[(size_t)agg[i] * ncomp + comp[i]];
    int max_rows = 0, max_cnt = 0;
    for (int a = 0; a < m; ++a) max_rows = std::max(max_rows, size[a]);
    for (int i = 0; i < n; ++i) max_cnt = std::max(max_cnt, ncnt[i]);

    // device buffers (released with the context)
    auto up = [&](int *&dst, const std::vector<int> &v) -> int {
        c.release(dst);
        SPH_TRY(c.alloc(dst, v.size()));
        SPH_CUDA_TRY(cudaMemcpyAsync(dst, v.data(), sizeof(int) * v.size(), cudaMemcpyHostToDevice, st));
        return SPH_OK;
    };
    SPH_TRY(up(c.cg_agg, agg));
    SPH_TRY(up(c.cg_off, off));
    SPH_TRY(up(c.cg_rows, rows));
    // pieces of the restriction: every aggregate in ceil(rows / kCoarsePiece)
    // pieces of about equal length
    std::vector<int> piece, pfirst(m + 1, 0);
    for (int a = 0; a < m; ++a) {
        const int len = off[a + 1] - off[a];
        const int np = std::max(1, (len + kCoarsePiece - 1) / kCoarsePiece);
        for (int k = 0; k < np; ++k) {
            piece.push_back(a);
            piece.push_back(off[a] + (int)((long long)len * k / np));
            piece.push_back(off[a] + (int)((long long)len * (k + 1) / np));
        }
        pfirst[a + 1] = pfirst[a] + np;
    }
    c.cg_np = pfirst[m];
    SPH_TRY(up(c.cg_piece, piece));
    SPH_TRY(up(c.cg_pfirst, pfirst));
    c.release(c.cg_part);
    c.release(c.cg_cnt);
    SPH_TRY(c.alloc(c.cg_part, (size_t)c.cg_np));
    SPH_TRY(c.alloc(c.cg_cnt, (size_t)m));
    SPH_CUDA_TRY(cudaMemsetAsync(c.cg_cnt, 0, sizeof(unsigned int) * (size_t)m, st));
    int *d_nm_idx = nullptr, *d_cnt_comp = nullptr, *d_piv = nullptr, *d_err = nullptr;
    SPH_TRY(up(d_nm_idx, nm_idx));
    SPH_TRY(up(d_cnt_comp, cnt_comp));
    double *E = nullptr, *E0 = nullptr, *Bk = nullptr, *a_comp = nullptr, *pval = nullptr;
    unsigned long long *amax = nullptr, *d_dev = nullptr;
    int *d_col = nullptr, *d_cols = nullptr;
    c.release(c.cg_s); c.release(c.cg_y);
    SPH_TRY(c.alloc(c.cg_s, m));
    SPH_TRY(c.alloc(c.cg_y, m));
    SPH_TRY(c.alloc(E, (size_t)m * m));
    SPH_TRY(c.alloc(E0, (size_t)m * m));
    SPH_TRY(c.alloc(Bk, (size_t)kGjPanel * m));
    SPH_TRY(c.alloc(a_comp, (size_t)m * std::max(ncomp, 1)));
    SPH_TRY(c.alloc(pval, 1));
    SPH_TRY(c.alloc(amax, 1));
    SPH_TRY(c.alloc(d_dev, 1));
    SPH_TRY(c.alloc(d_piv, m));
    SPH_TRY(c.alloc(d_col, m));
    SPH_TRY(c.alloc(d_cols, 4));
    SPH_TRY(c.alloc(d_err, 1));

    // fixed-point scale: every term below 2^61 / (terms per entry)
    SPH_CUDA_TRY(cudaMemsetAsync(amax, 0, sizeof(unsigned long long), st));
    if (sizeof(Real) == 4)
        k_coef_absmax<float><<<grid_for(n, 256), 256, 0, st>>>(c.row_kind, c.slice_off, c.ncnt, c.coef, n, amax);
    else
        k_coef_absmax<double><<<grid_for(n, 256), 256, 0, st>>>(c.row_kind, c.slice_off, c.ncnt, c.coef_d, n, amax);
    unsigned long long hbits = 0;
    SPH_CUDA_TRY(cudaMemcpyAsync(&hbits, amax, sizeof hbits, cudaMemcpyDeviceToHost, st));
    SPH_CUDA_TRY(cudaStreamSynchronize(st));
    double cmax = 0;
    memcpy(&cmax, &hbits, sizeof cmax);
    cmax = std::max(cmax, 1.0);   // Neumann weights and copy rows contribute <= 1
    const double terms = (double)max_rows * (double)std::max(max_cnt, 64) + 1.0;
    const double scale = std::ldexp(1.0, (int)std::floor(61.0 - std::log2(cmax) - std::log2(terms)));

    const bool in_smem = m <= 24576;   // 192 KB of the 227 KB a block may use
    const size_t shmem = in_smem ? sizeof(unsigned long long) * (size_t)m : 0;
    if (sizeof(Real) == 4) {
        SPH_CUDA_TRY(cudaFuncSetAttribute(k_coarse_assemble<float, Real>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)shmem));
        k_coarse_assemble<float, Real><<<m, 256, shmem, st>>>(
            m, c.cg_agg, c.cg_off, c.cg_rows, c.row_kind, c.row_aux, c.slice_off, c.ncnt, c.nbr, c.coef, d_nm_idx,
            c.L.nm_off, c.L.nm_nbr, c.nm_ow, ncomp > 0 ? c.comp_id : nullptr, c.diag, ncomp, scale, E, a_comp,
            in_smem);
    } else {
        SPH_CUDA_TRY(cudaFuncSetAttribute(k_coarse_assemble<double, Real>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)shmem));
        k_coarse_assemble<double, Real><<<m, 256, shmem, st>>>(
            m, c.cg_agg, c.cg_off, c.cg_rows, c.row_kind, c.row_aux, c.slice_off, c.ncnt, c.nbr, c.coef_d, d_nm_idx,
            c.L.nm_off, c.L.nm_nbr, c.nm_ow, ncomp > 0 ? c.comp_id : nullptr, c.diag, ncomp, scale, E, a_comp,
            in_smem);
    }
    SPH_CUDA_TRY(cudaGetLastError());
    const long long mm = (long long)m * m;
    if (ncomp > 0) {
        k_coarse_rank_one<<<div_up(mm, 256), 256, 0, st>>>(E, a_comp, d_cnt_comp, c.comp_inv, m, ncomp);
        SPH_CUDA_TRY(cudaGetLastError());
    }
    // E^-1: blocked in-place Gauss-Jordan on E, E0 keeping E for the check
    SPH_CUDA_TRY(cudaMemcpyAsync(E0, E, sizeof(double) * (size_t)mm, cudaMemcpyDeviceToDevice, st));
    SPH_CUDA_TRY(cudaMemsetAsync(d_err, 0, sizeof(int), st));
    const dim3 tiles((unsigned)div_up(m, 64), (unsigned)div_up(m, 64));
    for (int k0 = 0; k0 < m; k0 += kGjPanel) {
        const int kb = std::min(kGjPanel, m - k0);
        for (int k = k0; k < k0 + kb; ++k) {
            k_gj_pivot<<<1, 1024, 0, st>>>(E, m, k, d_piv + k, pval, d_err);
            k_gj_pivot_row<<<1, kGjPanel, 0, st>>>(E, m, k, k0, kb, d_piv + k, pval, d_err);
            k_gj_panel_elim<<<div_up(32LL * m, 256), 256, 0, st>>>(E, m, k, k0, kb, d_err);
        }
        c.launches += 3LL * kb;
        if (kb < m) {
            k_gj_swap_rows<<<div_up(m, 256), 256, 0, st>>>(E, m, k0, kb, d_piv, d_err);
            k_gj_copy_rows<<<div_up((long long)kb * m, 256), 256, 0, st>>>(E, Bk, m, k0, kb);
            k_gj_update<<<tiles, 256, 0, st>>>(E, Bk, m, k0, kb, d_err);
            c.launches += 3;
        }
    }
    SPH_CUDA_TRY(cudaGetLastError());
    int herr = 0;
    std::vector<int> piv(m), col(m);
    SPH_CUDA_TRY(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    SPH_CUDA_TRY(cudaMemcpyAsync(piv.data(), d_piv, sizeof(int) * m, cudaMemcpyDeviceToHost, st));
    SPH_CUDA_TRY(cudaStreamSynchronize(st));
    // the row interchanges permuted the inverse's columns: undo them in
    // reverse order (column c of the inverse is column col[c] of E)
    for (int k = 0; k < m; ++k) col[k] = k;
    for (int k = m - 1; k >= 0; --k) {
        const int p = (piv[k] >= 0 && piv[k] < m) ? piv[k] : k;
        std::swap(col[k], col[p]);
    }
    const int cols[4] = {0, m / 3, (2 * m) / 3, m - 1};
    SPH_CUDA_TRY(cudaMemcpyAsync(d_col, col.data(), sizeof(int) * m, cudaMemcpyHostToDevice, st));
    SPH_CUDA_TRY(cudaMemcpyAsync(d_cols, cols, sizeof cols, cudaMemcpyHostToDevice, st));
    SPH_CUDA_TRY(cudaMemsetAsync(d_dev, 0, sizeof(unsigned long long), st));
    if (!herr) {
        k_gj_check<<<div_up(32LL * m, 256), 256, 0, st>>>(E0, E, d_col, d_cols, 4, m, d_dev);
        ++c.launches;
    }
    c.release(c.cg_invf);
    SPH_TRY(c.alloc(c.cg_invf, (size_t)m * m));
    k_gj_to_float<<<div_up(mm, 256), 256, 0, st>>>(E, d_col, c.cg_invf, m);
    ++c.launches;
    SPH_CUDA_TRY(cudaGetLastError());
    unsigned long long dbits = 0;
    SPH_CUDA_TRY(cudaMemcpyAsync(&dbits, d_dev, sizeof dbits, cudaMemcpyDeviceToHost, st));
    SPH_CUDA_TRY(cudaStreamSynchronize(st));
    double dev = 0;
    memcpy(&dev, &dbits, sizeof dev);
    c.release(E); c.release(E0); c.release(Bk); c.release(a_comp); c.release(pval); c.release(amax);
    c.release(d_dev); c.release(d_piv); c.release(d_col); c.release(d_cols); c.release(d_err);
    c.release(d_nm_idx); c.release(d_cnt_comp);
    if (herr) {
        set_error("coarse operator is singular");
        return SPH_ERR_BREAKDOWN;
    }
    if (!(dev <= 1e-6)) {   // E X - I on four columns of the inverse
        static thread_local char msg[128];
        snprintf(msg, sizeof msg, "coarse inverse check failed: max |E X - I| = %.3e on sampled columns", dev);
        set_error(msg);
        return SPH_ERR_BREAKDOWN;
    }
    c.cg_m = m;
    return SPH_OK;
}

template int coarse_build<float>(Ctx<float> &);
template int coarse_build<double>(Ctx<double> &);
template void coarse_apply<float, float>(Ctx<float> &, const float *, float *, const float *);
template void coarse_apply<float, double>(Ctx<float> &, const double *, double *, const double *);
template void coarse_apply<double, double>(Ctx<double> &, const double *, double *, const double *);
template void coarse_restrict_solve<float, float>(Ctx<float> &, const float *, const float *);
template void coarse_restrict_solve<float, double>(Ctx<float> &, const double *, const double *);
template void coarse_restrict_solve<double, double>(Ctx<double> &, const double *, const double *);

}  // namespace sph
