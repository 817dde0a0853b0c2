// Adaptive particle refinement: 3-D splitting of one particle into eight.
//
// Follows the reference's cell-based APR (functions_APR.cuh:270-403,
// KERNEL_APR_condition3D_cell; functions_APR_etc.cuh:5-20, Cell_index;
// functions_APR.cuh:406-652, KERNEL_cell_APR_3D), which the shipped
// reference does not compile (SOPHIA_gpu.cu:113-114):
//   * a particle's level is log8(m_ref / m); a cell splits the first of its
//     particles (sorted order) whose target level exceeds its level by at
//     least 0.75, one particle per cell and pass;
//   * the split cells are numbered in cell order and each writes eight
//     children into free (dummy, i_type 3) records: copies of the parent at
//     x +- d, y +- d, z +- d with d = cbrt(m / rho) / 4, in the reference's
//     octant order (x sign slowest), with m / 8, vol / 8 and h / 2 when
//     h_change (vii[36]) is set; the parent becomes a dummy.
// The target level, a per-particle field the reference leaves to the caller
// (M_num), is here apr_max_level for fluid particles whose NNPS cell lies
// within apr_zone of an IBM marker cell, else 0.  The 3-D merge is commented
// out in the reference and is not performed here either.
//
// The free records are the dummies the deck reserves: after NNPS they form
// the segment [cell_start[num_cells], n) of the sorted arrays.  A pass that
// needs more children than there are free records splits the cells in cell
// order until the records run out.  The particle set then changes, so the
// next step rebuilds NNPS, lists, side lists and the PPE operator.
#include <algorithm>
#include <cmath>
#include <vector>

#include "ctx.cuh"

namespace sph {

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

// per cell: the first particle to split, or -1
template <class Real>
__global__ void k_apr_flag(Ctx<Real> c, const unsigned char *zone, int max_level, int *pick, int *flag) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= c.num_cells) return;
    int sel = -1;
    if (zone[k]) {
        for (int j = c.cell_start[k]; j < c.cell_start[k + 1]; ++j) {
            const int4 t = c.ty[j];
            if (t.w != 1 || t.x >= 3) continue;
            const double level = log((double)c.m_ref[j] / (double)c.mr[j].x) / log(8.0);
            if ((double)max_level - level >= 0.75) { sel = j; break; }
        }
    }
    pick[k] = sel;
    flag[k] = sel >= 0 ? 1 : 0;
}

template <class T>
__device__ __forceinline__ void cp(T *a, int d, int s) { if (a) a[d] = a[s]; }

// writes the eight children of the picked particle of every split cell
template <class Real>
__global__ void k_apr_split(Ctx<Real> c, const int *pick, const int *slot, int first_free, int max_cells, int h_change) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= c.num_cells) return;
    const int j = pick[k];
    if (j < 0) return;
    const int q = slot[k];
    if (q >= max_cells) return;
    typedef typename Ctx<Real>::R4 R4;
    const R4 xj = c.pr[j];
    const Real m = c.mr[j].x, rho = c.mr[j].y;
    const Real d = (Real)0.25 * cbrt(m / rho);
    for (int o = 0; o < 8; ++o) {
        const int dst = first_free + 8 * q + o;
        cp(c.pf, dst, j);
        if ((void *)c.pr != (void *)c.pf) cp(c.pr, dst, j);
        cp(c.mr, dst, j); cp(c.ty, dst, j); cp(c.jc, dst, j); cp(c.ncell, dst, j);
        cp(c.vol, dst, j); cp(c.m_ref, dst, j); cp(c.h_ref, dst, j); cp(c.eli, dst, j); cp(c.pres0, dst, j);
        cp(c.source, dst, j);
        cp(c.A.u, dst, j); cp(c.A.p, dst, j); cp(c.A.temp, dst, j); cp(c.A.flt, dst, j); cp(c.A.kt, dst, j);
        cp(c.A.et, dst, j); cp(c.A.fb, dst, j); cp(c.A.fm, dst, j); cp(c.A.fl, dst, j); cp(c.A.concn, dst, j);
        cp(c.A.enth, dst, j); cp(c.rho_ref_A, dst, j);
        // octant o: x sign + for o < 4, y sign + for o in {0,1,4,5}, z sign + for even o
        const Real sx = (o < 4) ? d : -d, sy = ((o & 2) == 0) ? d : -d, sz = ((o & 1) == 0) ? d : -d;
        R4 x = xj;
        x.x = xj.x + sx; x.y = xj.y + sy; x.z = xj.z + sz;
        if (h_change) x.w = (Real)0.5 * xj.w;
        c.pr[dst] = x;
        float4 xf = c.pf[j];
        xf.x = (float)x.x; xf.y = (float)x.y; xf.z = (float)x.z; xf.w = (float)x.w;
        c.pf[dst] = xf;
        c.mr[dst].x = (Real)0.125 * m;
        c.vol[dst] = (Real)0.125 * c.vol[j];
    }
    // the parent leaves the active set
    int4 t = c.ty[j];
    t.x = 3;
    c.ty[j] = t;
}

template <class Real>
int apr_split(Ctx<Real> &c, int *n_split, int *n_wanted) {
    if (n_split) *n_split = 0;
    if (n_wanted) *n_wanted = 0;
    const int max_level = c.prm.apr_max_level;
    if (max_level <= 0 || !c.built) return SPH_OK;
    const int NC = c.num_cells;
    cudaStream_t st = c.stream;
    unsigned char *zone = nullptr;
    int *pick = nullptr, *flag = nullptr, *slot = nullptr, *tmp = nullptr;
    SPH_TRY(c.alloc(zone, NC));
    SPH_TRY(c.alloc(pick, NC));
    SPH_TRY(c.alloc(flag, NC + 1));
    SPH_TRY(c.alloc(slot, NC + 1));
    SPH_CUDA_TRY(cudaMemsetAsync(zone, 0, NC, st));
    const int reach = (int)std::ceil(c.prm.apr_zone / (double)c.dp.dcell);
    k_apr_zone<<<grid_for(c.n, 256), 256, 0, st>>>(c.ty, c.pf, c.dp, reach, zone, c.n);
    k_apr_flag<Real><<<grid_for(NC, 256), 256, 0, st>>>(c, zone, max_level, pick, flag);
    c.launches += 2;
    SPH_CUDA_TRY(cudaGetLastError());
    // slots in cell order (Cell_index) and the free records
    std::vector<int> hf(NC), cs(2);
    SPH_CUDA_TRY(cudaMemcpyAsync(hf.data(), flag, sizeof(int) * NC, cudaMemcpyDeviceToHost, st));
    SPH_CUDA_TRY(cudaMemcpyAsync(cs.data(), c.cell_start + NC, sizeof(int) * 2, cudaMemcpyDeviceToHost, st));
    SPH_CUDA_TRY(cudaStreamSynchronize(st));
    std::vector<int> hs(NC);
    int q = 0;
    for (int k = 0; k < NC; ++k) { hs[k] = q; q += hf[k]; }
    const int first_free = cs[0], nfree = cs[1] - cs[0];
    const int cells = std::min(q, nfree / 8);
    if (n_wanted) *n_wanted = q;
    if (cells > 0) {
        SPH_CUDA_TRY(cudaMemcpyAsync(slot, hs.data(), sizeof(int) * NC, cudaMemcpyHostToDevice, st));
        k_apr_split<Real><<<grid_for(NC, 256), 256, 0, st>>>(c, pick, slot, first_free, cells,
                                                             c.prm.vii[SPH_VII_H_CHANGE]);
        ++c.launches;
        SPH_CUDA_TRY(cudaGetLastError());
        c.built = false;   // new particle set: NNPS and everything built on it again
        c.gc_valid = false;
        c.prep_valid = false;
        c.pforce_valid = false;
        c.coef_valid = false;
        c.cg_valid = false;
        c.ml_have_prev = false;
        c.release(c.ml_fluid);
    }
    SPH_CUDA_TRY(cudaStreamSynchronize(st));
    c.release(zone); c.release(pick); c.release(flag); c.release(slot);
    (void)tmp;
    if (n_split) *n_split = cells;
    return SPH_OK;
}

template int apr_split<float>(Ctx<float> &, int *, int *);
template int apr_split<double>(Ctx<double> &, int *, int *);

}  // namespace sph
