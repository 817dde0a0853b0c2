// Adaptive particle refinement: cell-based 3-D splitting and merging.
//
// Follows the reference's cell-based APR, which the shipped reference does
// not compile (SOPHIA_gpu.cu:113-114 keep functions_APR.cuh out):
//   * KERNEL_APR_condition3D_cell (functions_APR.cuh:270-403), per cell: a
//     particle's level is log(m_ref / m) / log(8); the first particle of the
//     cell (sorted order) whose target level M exceeds its level by >= 0.75
//     is marked to split (apr_cond = 1) and the cell asks to split; otherwise
//     the last particle whose level exceeds M by more than 0.3 is a merge
//     candidate: the particles of its family (blood_index) within
//     search_kappa * h of it are searched, the search gives up if one of them
//     has M == 1, and the family member of largest index is marked
//     (apr_cond = -1) and the cell asks to merge;
//   * Cell_index (functions_APR_etc.cuh:5-20): splitting cells are numbered
//     1, 2, ... and merging cells -1, -2, ... in cell order; the merging
//     cells here are those that hold a marked member (the reference numbers
//     every cell whose condition asked, and the merge slots of cells without
//     a marked member stay unused);
//   * KERNEL_cell_APR_3D (functions_APR.cuh:406-652), split: the marked
//     particle becomes eight children at k_num_part + num_buffer + 8 * number,
//     i.e. from 8 records past the first free record: copies of the parent at
//     x +- d, y +- d, z +- d with d = 0.25 cbrt(m / rho) (x sign slowest, the
//     reference's octant order), with m / 8, vol / 8, the parent's family and
//     h / 2 when h_change (vii[36]) is set; the parent becomes a dummy;
//   * merge: the reference's 3-D merge is commented out; this pass performs
//     its active 2-D merge (KERNEL_cell_APR_2D, functions_APR.cuh:119-186)
//     generalised to 3-D: in the cell holding the marked member, the family's
//     members (i_type 1, same family) in the cells around it are summed -- m
//     and vol, and 1/8 of each position, velocity and pressure -- and become
//     dummies; their merged record, a copy of the marked member with those
//     sums and h = h_ref cbrt(m / m_ref) (with h_change), goes to record
//     num_part2 + number (the tail of the array, counting down).  The 2-D
//     condition marks a family only when all 4 members are in range; the 3-D
//     merge here likewise acts only on a family of 8 members.
// Family and target level are the reference's part1 fields blood_index and
// M_num, which its shipped part1 keeps commented out: here they are
// per-record context arrays, sorted with the records.  The family of every
// record is set to its index + 1 at the first pass (KERNEL_remember_blood,
// functions_APR_etc.cuh:83-87); children and merged records inherit theirs.
// The target level is apr_max_level for fluid particles in NNPS cells within
// apr_zone of an IBM marker's cell, 0 elsewhere (the reference leaves M_num to
// the caller).
//
// The free records are the dummies the deck reserves: after NNPS they form
// the segment [cell_start[num_cells], n) of the sorted arrays.  A pass whose
// children and merged records do not fit splits the cells in cell order
// while their children fit, then merges the cells in cell order while their
// records at the tail stay past the children.  The particle set then changes, so the
// next step rebuilds NNPS, lists, side lists and the PPE operator.
#include <algorithm>
#include <cmath>
#include <vector>

#include "ctx.cuh"

namespace sph {

constexpr int kNcellInit = 2;   // ncell_init, Parameters.cuh:103

// marks every cell within `reach` cells of a cell holding an IBM marker
__global__ void k_apr_zone(const int4 *ty, const float4 *pf, DevParams P, int reach, unsigned char *zone, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int4 t = ty[i];
    if (t.w < 1000 || t.x >= 3) return;
    const float4 x = pf[i];
    const int ic = bin_axis(x.x, P.xmin, P.xmax, P.NI), jc = bin_axis(x.y, P.ymin, P.ymax, P.NJ),
              kc = bin_axis(x.z, P.zmin, P.zmax, P.NK);
    for (int dz = -reach; dz <= reach; ++dz)
        for (int dy = -reach; dy <= reach; ++dy)
            for (int dx = -reach; dx <= reach; ++dx) {
                const int a = ic + dx, b = jc + dy, c = kc + dz;
                if (a < 0 || b < 0 || c < 0 || a >= P.NI || b >= P.NJ || c >= P.NK) continue;
                zone[a + P.NI * (b + P.NJ * c)] = 1;
            }
}

// the target level of every record: apr_max_level for fluid in a zone cell
__global__ void k_apr_target(const int4 *ty, const int *key, const unsigned char *zone, int num_cells, int max_level,
                             float *target, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int4 t = ty[i];
    const int k = key[i];
    target[i] = (t.x < 3 && t.w == 1 && k >= 0 && k < num_cells && zone[k]) ? (float)max_level : 0.f;
}

__global__ void k_apr_family_init(int *family, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) family[i] = i + 1;
}

// mass_ratio = log(m_ref / m) / log(8.0) in the reference's types: the
// logarithm of a Real, divided by the double log(8.0), stored as a Real
template <class Real>
__device__ __forceinline__ Real apr_level(Real m_ref, Real m) {
    return (Real)((double)log(m_ref / m) / log(8.0));
}

// KERNEL_APR_condition3D_cell: per cell k, flag +1 (split), -1 (merge) or 0;
// apr_cond per record (cleared before the launch)
template <class Real>
__global__ void k_apr_condition(Ctx<Real> c, const float *target, const int *family, int *apr_cond, int *flag) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= c.num_cells) return;
    flag[k] = 0;
    const int s = c.cell_start[k], e = c.cell_start[k + 1];
    if (e <= s) return;
    int merge_index = 0, blood = 0;
    bool merge_flag = false;
    for (int j = s; j < e; ++j) {
        const Real level = apr_level<Real>(c.m_ref[j], c.mr[j].x);
        const Real M = (Real)target[j];
        if (M - level >= 0.75) {
            apr_cond[j] = 1;
            flag[k] = 1;
            return;
        } else if (M - level < -0.3) {
            merge_index = j;
            blood = family[j];
            merge_flag = true;
        }
    }
    if (!merge_flag) return;
    const DevParams &P = c.dp;
    const float4 xi = c.pf[merge_index];
    const int ic = bin_axis(xi.x, P.xmin, P.xmax, P.NI), jc = bin_axis(xi.y, P.ymin, P.ymax, P.NJ),
              kc = bin_axis(xi.z, P.zmin, P.zmax, P.NK);
    const int range = (int)ceilf(__fdiv_rn(__fmul_rn((float)kNcellInit, xi.w), (float)c.h_ref[merge_index]));
    const float search = __fmul_rn(P.skappa, xi.w);
    for (int dz = -range; dz <= range; ++dz)
        for (int dy = -range; dy <= range; ++dy)
            for (int dx = -range; dx <= range; ++dx) {
                const int a = ic + dx, b = jc + dy, cc = kc + dz;
                if (a < 0 || a > P.NI - 1 || b < 0 || b > P.NJ - 1 || cc < 0 || cc > P.NK - 1) continue;
                const int kk = a + P.NI * b + P.NI * P.NJ * cc;
                for (int j = c.cell_start[kk]; j < c.cell_start[kk + 1]; ++j) {
                    const float4 xj = c.pf[j];
                    const float r = (float)((double)dist_rn(xi.x, xi.y, xi.z, xj.x, xj.y, xj.z) + 1e-20);
                    if (!(r < search)) continue;
                    if (c.ty[j].x == 1 && family[j] == blood) {
                        if (target[j] == 1.f) return;
                        if (j > merge_index) merge_index = j;
                    }
                }
            }
    apr_cond[merge_index] = -1;   // the family member of largest index
    flag[k] = -1;
}

// calls f(i) for every active (i_type 1) member of family `blood` in the
// cells around record j (the reach of the condition's family search)
template <class Real, class F>
__device__ __forceinline__ void for_family(const Ctx<Real> &c, const int *family, int j, int blood, F &&f) {
    const DevParams &P = c.dp;
    const float4 xa = c.pf[j];
    const int ic = bin_axis(xa.x, P.xmin, P.xmax, P.NI), jc = bin_axis(xa.y, P.ymin, P.ymax, P.NJ),
              kc = bin_axis(xa.z, P.zmin, P.zmax, P.NK);
    const int range = (int)ceilf(__fdiv_rn(__fmul_rn((float)kNcellInit, xa.w), (float)c.h_ref[j]));
    for (int dz = -range; dz <= range; ++dz)
        for (int dy = -range; dy <= range; ++dy)
            for (int dx = -range; dx <= range; ++dx) {
                const int a = ic + dx, b = jc + dy, cc = kc + dz;
                if (a < 0 || a > P.NI - 1 || b < 0 || b > P.NJ - 1 || cc < 0 || cc > P.NK - 1) continue;
                const int kk = a + P.NI * b + P.NI * P.NJ * cc;
                for (int i = c.cell_start[kk]; i < c.cell_start[kk + 1]; ++i)
                    if (c.ty[i].x == 1 && family[i] == blood) f(i);
            }
}

// the record a merging cell merges: its first marked member, when that
// member's family is complete (eight active members around it) and it is the
// family's member of largest index; else -1
template <class Real>
__device__ int merge_record(const Ctx<Real> &c, const int *apr_cond, const int *family, int k) {
    int j = -1;
    for (int a = c.cell_start[k]; a < c.cell_start[k + 1]; ++a)
        if (apr_cond[a] == -1) { j = a; break; }
    if (j < 0) return -1;
    const int blood = family[j];
    if (blood == 0) return -1;
    int count = 0, last = -1;
    for_family(c, family, j, blood, [&](int i) { ++count; last = max(last, i); });
    return (count == 8 && last == j) ? j : -1;
}

// merging cells are the cells that hold a marked member (wherever the
// condition that marked it ran) whose family merges in this pass; only they
// get merge numbers, so the free records at the tail go to merges that
// happen
template <class Real>
__global__ void k_apr_merge_cells(Ctx<Real> c, const int *apr_cond, const int *family, int *flag) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= c.num_cells) return;
    if (flag[k] > 0) return;
    flag[k] = merge_record(c, apr_cond, family, k) >= 0 ? -1 : 0;
}

template <class T>
__device__ __forceinline__ void cp(T *a, int d, int s) { if (a) a[d] = a[s]; }

// copies every per-record array of record s into record d
template <class Real>
__device__ void copy_record(Ctx<Real> &c, const float *target, float *target_w, int *family, int d, int s) {
    cp(c.pf, d, s);
    if ((void *)c.pr != (void *)c.pf) cp(c.pr, d, s);
    cp(c.mr, d, s); cp(c.ty, d, s); cp(c.jc, d, s); cp(c.ncell, d, s);
    cp(c.vol, d, s); cp(c.m_ref, d, s); cp(c.h_ref, d, s); cp(c.eli, d, s); cp(c.pres0, d, s);
    cp(c.source, d, s);
    cp(c.A.u, d, s); cp(c.A.p, d, s); cp(c.A.temp, d, s); cp(c.A.flt, d, s); cp(c.A.kt, d, s);
    cp(c.A.et, d, s); cp(c.A.fb, d, s); cp(c.A.fm, d, s); cp(c.A.fl, d, s); cp(c.A.concn, d, s);
    cp(c.A.enth, d, s); cp(c.rho_ref_A, d, s);
    target_w[d] = target[s];
    family[d] = family[s];
}

// KERNEL_cell_APR_3D: the split of the marked particle of every splitting
// cell (number[k] > 0, at most max_split of them) and the merge of the
// marked family member of every merging cell (number[k] < 0) whose record
// n + number[k] lies at or past min_slot
template <class Real>
__global__ void k_apr_execute(Ctx<Real> c, const int *number, const int *apr_cond, float *target, int *family,
                              int first_free, int max_split, int min_slot, int h_change, int *merged) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= c.num_cells) return;
    const int q = number[k];
    const int s = c.cell_start[k], e = c.cell_start[k + 1];
    if (q == 0 || e <= s) return;
    typedef typename Ctx<Real>::R4 R4;
    if (q > 0) {
        if (q > max_split) return;
        int j = -1;
        for (int a = s; a < e; ++a) {
            if (c.ty[a].w != 1 && target[a] > 2.f) continue;
            if (apr_cond[a] == 1) { j = a; break; }
        }
        if (j < 0) return;
        const R4 xj = c.pr[j];
        const Real m = c.mr[j].x, rho = c.mr[j].y;
        const Real vm = m / rho;
        const Real d = (Real)cbrt(vm);
        for (int o = 0; o < 8; ++o) {
            const int dst = first_free + 8 * q + o;
            copy_record(c, target, target, family, dst, j);
            // octant o: x sign + for o < 4, y sign + for o in {0,1,4,5}, z sign + for even o
            const double sx = (o < 4) ? 0.25 : -0.25, sy = ((o & 2) == 0) ? 0.25 : -0.25,
                         sz = ((o & 1) == 0) ? 0.25 : -0.25;
            R4 x = xj;
            x.x = (Real)((double)xj.x + sx * (double)d);
            x.y = (Real)((double)xj.y + sy * (double)d);
            x.z = (Real)((double)xj.z + sz * (double)d);
            if (h_change) x.w = (Real)(0.5 * (double)xj.w);
            c.pr[dst] = x;
            float4 xf = c.pf[j];
            xf.x = (float)x.x; xf.y = (float)x.y; xf.z = (float)x.z; xf.w = (float)x.w;
            c.pf[dst] = xf;
            c.mr[dst].x = (Real)(0.125 * (double)m);
            c.vol[dst] = (Real)(0.125 * (double)c.vol[j]);
        }
        int4 t = c.ty[j];
        t.x = 3;   // the parent leaves the active set
        c.ty[j] = t;
        return;
    }
    if (c.n + q < min_slot) return;
    const int j = merge_record(c, apr_cond, family, k);
    if (j < 0) return;
    const int blood = family[j];
    auto for_members = [&](auto &&f) { for_family(c, family, j, blood, f); };
    Real m_sum = 0, vol_sum = 0, x_avg = 0, y_avg = 0, z_avg = 0, ux_avg = 0, uy_avg = 0, uz_avg = 0, p_avg = 0;
    for_members([&](int i) {
        const R4 xi = c.pr[i];
        const R4 ui = c.A.u[i];
        m_sum += c.mr[i].x;
        vol_sum += c.vol[i];
        x_avg = (Real)((double)x_avg + 0.125 * (double)xi.x);
        y_avg = (Real)((double)y_avg + 0.125 * (double)xi.y);
        z_avg = (Real)((double)z_avg + 0.125 * (double)xi.z);
        ux_avg = (Real)((double)ux_avg + 0.125 * (double)ui.x);
        uy_avg = (Real)((double)uy_avg + 0.125 * (double)ui.y);
        uz_avg = (Real)((double)uz_avg + 0.125 * (double)ui.z);
        p_avg = (Real)((double)p_avg + 0.125 * (double)c.A.p[i]);
    });
    const int dst = c.n + q;
    copy_record(c, target, target, family, dst, j);
    for_members([&](int i) {
        int4 t = c.ty[i];
        t.x = 3;
        c.ty[i] = t;
    });
    int4 t = c.ty[dst];
    t.x = 1;
    c.ty[dst] = t;
    R4 x = c.pr[dst];
    x.x = x_avg; x.y = y_avg; x.z = z_avg;
    if (h_change) x.w = c.h_ref[dst] * (Real)cbrt(m_sum / c.m_ref[dst]);
    c.pr[dst] = x;
    float4 xf = c.pf[dst];
    xf.x = (float)x.x; xf.y = (float)x.y; xf.z = (float)x.z; xf.w = (float)x.w;
    c.pf[dst] = xf;
    c.mr[dst].x = m_sum;
    c.vol[dst] = vol_sum;
    R4 u = c.A.u[dst];
    u.x = ux_avg; u.y = uy_avg; u.z = uz_avg;
    c.A.u[dst] = u;
    c.A.p[dst] = p_avg;
    atomicAdd(merged, 1);
}

template <class Real>
int apr_pass(Ctx<Real> &c, int *n_split, int *n_wanted, int *n_merged) {
    if (n_split) *n_split = 0;
    if (n_wanted) *n_wanted = 0;
    if (n_merged) *n_merged = 0;
    const int max_level = c.prm.apr_max_level;
    if (!c.built) return SPH_OK;
    if (max_level <= 0 && !c.apr_family) return SPH_OK;
    const int NC = c.num_cells, n = c.n;
    cudaStream_t st = c.stream;
    if (!c.apr_family) {
        SPH_TRY(c.alloc(c.apr_family, n));
        SPH_TRY(c.alloc(c.apr_target, n));
        k_apr_family_init<<<grid_for(n, 256), 256, 0, st>>>(c.apr_family, n);
        ++c.launches;
    }
    unsigned char *zone = nullptr;
    int *cond = nullptr, *flag = nullptr, *number = nullptr, *merged = nullptr;
    SPH_TRY(c.alloc(zone, NC));
    SPH_TRY(c.alloc(cond, n));
    SPH_TRY(c.alloc(flag, NC));
    SPH_TRY(c.alloc(number, NC));
    SPH_TRY(c.alloc(merged, 1));
    SPH_CUDA_TRY(cudaMemsetAsync(zone, 0, NC, st));
    SPH_CUDA_TRY(cudaMemsetAsync(cond, 0, sizeof(int) * (size_t)n, st));
    SPH_CUDA_TRY(cudaMemsetAsync(merged, 0, sizeof(int), st));
    const int reach = (int)std::ceil(c.prm.apr_zone / (double)c.dp.dcell);
    if (max_level > 0)
        k_apr_zone<<<grid_for(n, 256), 256, 0, st>>>(c.ty, c.pf, c.dp, reach, zone, n);
    k_apr_target<<<grid_for(n, 256), 256, 0, st>>>(c.ty, c.g_idx, zone, NC, std::max(max_level, 0), c.apr_target, n);
    k_apr_condition<Real><<<grid_for(NC, 256), 256, 0, st>>>(c, c.apr_target, c.apr_family, cond, flag);
    k_apr_merge_cells<Real><<<grid_for(NC, 256), 256, 0, st>>>(c, cond, c.apr_family, flag);
    c.launches += 4;
    SPH_CUDA_TRY(cudaGetLastError());
    // Cell_index in cell order, and the free records
    std::vector<int> hf(NC), cs(2);
    SPH_CUDA_TRY(cudaMemcpyAsync(hf.data(), flag, sizeof(int) * NC, cudaMemcpyDeviceToHost, st));
    SPH_CUDA_TRY(cudaMemcpyAsync(cs.data(), c.cell_start + NC, sizeof(int) * 2, cudaMemcpyDeviceToHost, st));
    SPH_CUDA_TRY(cudaStreamSynchronize(st));
    std::vector<int> num(NC, 0);
    int pos = 0, neg = 0;
    for (int k = 0; k < NC; ++k) {
        if (hf[k] > 0) num[k] = ++pos;
        else if (hf[k] < 0) num[k] = -(++neg);
    }
    const int first_free = cs[0], nfree = n - first_free;
    // children start 8 records past the first free one; merged records go to
    // the tail, counting down, while they stay past the children
    const int max_split = std::max(0, std::min(pos, (nfree - 8) / 8));
    const int min_slot = max_split > 0 ? first_free + 8 * (max_split + 1) : first_free;
    const int do_merge = (neg > 0 && n - 1 >= min_slot) ? 1 : 0;
    if (n_wanted) *n_wanted = pos;
    int hmerged = 0;
    if (max_split > 0 || do_merge) {
        SPH_CUDA_TRY(cudaMemcpyAsync(number, num.data(), sizeof(int) * NC, cudaMemcpyHostToDevice, st));
        k_apr_execute<Real><<<grid_for(NC, 256), 256, 0, st>>>(c, number, cond, c.apr_target, c.apr_family, first_free,
                                                               max_split, min_slot, c.prm.vii[SPH_VII_H_CHANGE], merged);
        ++c.launches;
        SPH_CUDA_TRY(cudaGetLastError());
        SPH_CUDA_TRY(cudaMemcpyAsync(&hmerged, merged, sizeof(int), cudaMemcpyDeviceToHost, st));
    }
    SPH_CUDA_TRY(cudaStreamSynchronize(st));
    if (max_split > 0 || hmerged > 0) {
        c.built = false;   // new particle set: NNPS and everything built on it again
        c.gc_valid = false;
        c.prep_valid = false;
        c.pforce_valid = false;
        c.coef_valid = false;
        c.cg_valid = false;
        c.ml_have_prev = false;
        c.release(c.ml_fluid);
    }
    c.release(zone); c.release(cond); c.release(flag); c.release(number); c.release(merged);
    c.apr_last_merged = hmerged;
    if (n_split) *n_split = max_split;
    if (n_merged) *n_merged = hmerged;
    return SPH_OK;
}

template <class Real>
int apr_state(Ctx<Real> &c, int32_t *family, float *target) {
    const int n = c.n;
    if (!c.apr_family) {
        if (family) for (int i = 0; i < n; ++i) family[i] = 0;
        if (target) for (int i = 0; i < n; ++i) target[i] = 0.f;
        return SPH_OK;
    }
    if (family) SPH_CUDA_TRY(cudaMemcpyAsync(family, c.apr_family, sizeof(int) * n, cudaMemcpyDeviceToHost, c.stream));
    if (target) SPH_CUDA_TRY(cudaMemcpyAsync(target, c.apr_target, sizeof(float) * n, cudaMemcpyDeviceToHost, c.stream));
    SPH_CUDA_TRY(cudaStreamSynchronize(c.stream));
    return SPH_OK;
}

template int apr_pass<float>(Ctx<float> &, int *, int *, int *);
template int apr_pass<double>(Ctx<double> &, int *, int *, int *);
template int apr_state<float>(Ctx<float> &, int32_t *, float *);
template int apr_state<double>(Ctx<double> &, int32_t *, float *);

}  // namespace sph
