// NNPS of the ISPH step: cell hash, stable counting sort, cell ranges,
// reorder into sorted SoA, compacted neighbour lists (SELL-32) and the
// time-invariant side lists of the boundary passes.
//
// Reference: ISPH_Calc.cuh:20-45 (KERNEL_set_ncell, KERNEL_index_particle_to_cell,
// cub::DeviceRadixSort::SortPairs, KERNEL_reorder) and the per-kernel cell
// loops (e.g. functions_PPE.cuh:52-72) whose visit order the lists reproduce.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "ctx.cuh"

namespace sph {

// ---------------------------------------------------------------------------
// exclusive scan (int / long long), block-wise with warp shuffles
// ---------------------------------------------------------------------------
template <class T>
__global__ void k_scan_block(const T *in, T *out, T *bsum, long long n) {
    __shared__ T warp_tot[32];
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    T v = (i < n) ? in[i] : T(0);
    T x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[wid] = x;
    __syncthreads();
    if (wid == 0) {
        T w = (lane < (int)(blockDim.x >> 5)) ? warp_tot[lane] : T(0);
        T s = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            T y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        warp_tot[lane] = s - w;   // exclusive prefix of warp totals
        if (lane == 31 && bsum) bsum[blockIdx.x] = s;
    }
    __syncthreads();
    if (i < n) out[i] = x - v + warp_tot[wid];
}

template <class T>
__global__ void k_scan_add(T *out, const T *badd, long long n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += badd[blockIdx.x];
}

// exclusive scan of n entries of `in` into `out` (may alias); `tmp` must hold
// scan_tmp_size(n) elements.
template <class T>
static int exclusive_scan(const T *in, T *out, long long n, T *tmp, cudaStream_t st, long long &launches) {
    const int B = 1024;
    if (n <= 0) return SPH_OK;
    const long long nb = (n + B - 1) / B;
    T *bs = tmp;
    k_scan_block<T><<<(unsigned)nb, B, 0, st>>>(in, out, nb > 1 ? bs : nullptr, n);
    ++launches;
    if (nb > 1) {
        SPH_TRY(exclusive_scan<T>(bs, bs, nb, tmp + nb, st, launches));
        k_scan_add<T><<<(unsigned)nb, B, 0, st>>>(out, bs, n);
        ++launches;
    }
    SPH_CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}

static long long scan_tmp_size(long long n) {
    long long s = 0;
    while (n > 1) { n = (n + 1023) / 1024; s += n + 1; }
    return s + 8;
}

// ---------------------------------------------------------------------------
// AoS <-> SoA
// ---------------------------------------------------------------------------
template <class Real>
__global__ void k_unpack(Ctx<Real> c, const sph_part1 *P1, const sph_part2 *P2, int n) {
    typedef typename V4<Real>::type R4;
    typedef typename V2<Real>::type R2;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const sph_part1 r = P1[i];
    c.pf[i] = make_float4(r.x, r.y, r.z, r.h);
    if ((void *)c.pr != (void *)c.pf) c.pr[i] = mk4<Real>(r.x, r.y, r.z, r.h);
    R2 mr; mr.x = r.m; mr.y = r.rho;
    c.mr[i] = mr;
    c.ty[i] = make_int4(r.i_type, r.buffer_type, r.MOST_buffer, r.p_type);
    c.jc[i] = jclass_of(r.i_type, r.buffer_type, r.p_type);
    c.ncell[i] = r.ncell;
    c.vol[i] = r.vol; c.m_ref[i] = r.m_ref; c.h_ref[i] = r.h_ref; c.eli[i] = r.eli; c.pres0[i] = r.pres0;
    c.source[i] = r.source;
    VarSet<Real> &A = c.A;
    A.u[i] = mk4<Real>(r.ux, r.uy, r.uz, r.vis_t);
    A.p[i] = r.pres; A.temp[i] = r.temp; A.flt[i] = r.flt_s; A.kt[i] = r.k_turb; A.et[i] = r.e_turb;
    A.fb[i] = mk4<Real>(r.fbx, r.fby, r.fbz, r.concentration);
    A.fm[i] = mk4<Real>(r.fmx, r.fmy, r.hmz, 0);
    A.fl[i] = mk4<Real>(r.float1, r.float2, r.float3, 0);
    A.concn[i] = r.concn; A.enth[i] = r.enthalpy;
    c.rho_ref_A[i] = P2 ? (Real)P2[i].rho_ref : (Real)0;
}

// replaces the time-varying fields of an already sorted state
template <class Real>
__global__ void k_unpack_state(Ctx<Real> c, const sph_part1 *P1, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const sph_part1 r = P1[i];
    VarSet<Real> &A = c.A;
    A.u[i] = mk4<Real>(r.ux, r.uy, r.uz, r.vis_t);
    A.p[i] = r.pres; A.temp[i] = r.temp; A.flt[i] = r.flt_s; A.kt[i] = r.k_turb; A.et[i] = r.e_turb;
    A.fb[i] = mk4<Real>(r.fbx, r.fby, r.fbz, r.concentration);
    A.fm[i] = mk4<Real>(r.fmx, r.fmy, r.hmz, 0);
    A.fl[i] = mk4<Real>(r.float1, r.float2, r.float3, 0);
    A.concn[i] = r.concn; A.enth[i] = r.enthalpy;
}

template <class Real>
__global__ void k_pack(Ctx<Real> c, sph_part1 *P1, sph_part2 *P2, sph_part3 *P3, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const VarSet<Real> &A = c.A;
    if (P1) {
        sph_part1 r;
        const int4 t = c.ty[i];
        r.i_type = t.x; r.buffer_type = t.y; r.MOST_buffer = t.z; r.p_type = t.w;
        const auto x = c.pr[i];
        r.x = (float)x.x; r.y = (float)x.y; r.z = (float)x.z; r.h = (float)x.w;
        const auto u = A.u[i];
        r.ux = (float)u.x; r.uy = (float)u.y; r.uz = (float)u.z; r.vis_t = (float)u.w;
        r.m = (float)c.mr[i].x; r.rho = (float)c.mr[i].y;
        r.temp = (float)A.temp[i]; r.pres = (float)A.p[i]; r.pres0 = (float)c.pres0[i];
        r.flt_s = (float)A.flt[i]; r.enthalpy = (float)A.enth[i]; r.concn = (float)A.concn[i];
        const auto fb = A.fb[i];
        r.concentration = (float)fb.w;
        r.k_turb = (float)A.kt[i]; r.e_turb = (float)A.et[i];
        r.eli = (float)c.eli[i]; r.vol = (float)c.vol[i]; r.m_ref = (float)c.m_ref[i]; r.h_ref = (float)c.h_ref[i];
        r.fbx = (float)fb.x; r.fby = (float)fb.y; r.fbz = (float)fb.z;
        const auto fm = A.fm[i];
        r.fmx = (float)fm.x; r.fmy = (float)fm.y; r.hmz = (float)fm.z;
        const auto fl = A.fl[i];
        r.float1 = (float)fl.x; r.float2 = (float)fl.y; r.float3 = (float)fl.z;
        r.ncell = c.ncell[i]; r.source = c.source[i];
        P1[i] = r;
    }
    if (P2) {
        sph_part2 r;
        memset(&r, 0, sizeof(r));
        r.rho_ref = (float)c.rho_ref_S[i];
        r.SR = (float)c.SR[i];
        const auto u0 = c.u0[i];
        if (u0.w != 0) {
            const auto x = c.pr[i];
            r.x0 = (float)x.x; r.y0 = (float)x.y; r.z0 = (float)x.z;
        }
        r.ux0 = (float)u0.x; r.uy0 = (float)u0.y; r.uz0 = (float)u0.z;
        r.temp0 = (float)c.temp0[i]; r.concn0 = (float)c.concn0[i]; r.enthalpy0 = (float)c.enth0[i];
        P2[i] = r;
    }
    if (P3) {
        sph_part3 r;
        memset(&r, 0, sizeof(r));
        const auto ft = c.ft[i], fp = c.fp[i], nr = c.nrm[i];
        r.ftotalx = (float)ft.x; r.ftotaly = (float)ft.y; r.ftotalz = (float)ft.z; r.ftotal = (float)ft.w;
        r.fpx = (float)fp.x; r.fpy = (float)fp.y; r.fpz = (float)fp.z;
        r.dtemp = (float)c.dtemp[i];
        r.dconcn = (float)c.dconcn[i];
        r.denthalpy = (float)c.denth[i];
        r.nx = (float)nr.x; r.ny = (float)nr.y; r.nz = (float)nr.z;
        const size_t N = (size_t)c.n;
        r.inv_cm_xx = (float)c.g6[i]; r.inv_cm_yy = (float)c.g6[N + i]; r.inv_cm_zz = (float)c.g6[2 * N + i];
        r.inv_cm_xy = (float)c.g6[3 * N + i]; r.inv_cm_yz = (float)c.g6[4 * N + i]; r.inv_cm_zx = (float)c.g6[5 * N + i];
        P3[i] = r;
    }
}

template <class Real>
int ctx_allocate(Ctx<Real> &c) {
    const int n = c.n;
    SPH_TRY(c.alloc(c.pf, n));
    if (sizeof(Real) == sizeof(float)) c.pr = (typename Ctx<Real>::R4 *)c.pf;
    else SPH_TRY(c.alloc(c.pr, n));
    SPH_TRY(c.alloc(c.mr, n));
    SPH_TRY(c.alloc(c.ty, n));
    SPH_TRY(c.alloc(c.jc, n));
    SPH_TRY(c.alloc(c.ncell, n));
    SPH_TRY(c.alloc(c.vol, n)); SPH_TRY(c.alloc(c.m_ref, n)); SPH_TRY(c.alloc(c.h_ref, n));
    SPH_TRY(c.alloc(c.eli, n)); SPH_TRY(c.alloc(c.pres0, n)); SPH_TRY(c.alloc(c.source, n));
    for (VarSet<Real> *V : {&c.A, &c.S}) {
        SPH_TRY(c.alloc(V->u, n)); SPH_TRY(c.alloc(V->p, n)); SPH_TRY(c.alloc(V->temp, n));
        SPH_TRY(c.alloc(V->flt, n)); SPH_TRY(c.alloc(V->kt, n)); SPH_TRY(c.alloc(V->et, n));
        SPH_TRY(c.alloc(V->fb, n)); SPH_TRY(c.alloc(V->fm, n)); SPH_TRY(c.alloc(V->fl, n));
        SPH_TRY(c.alloc(V->concn, n)); SPH_TRY(c.alloc(V->enth, n));
    }
    SPH_TRY(c.alloc(c.rho_ref_A, n)); SPH_TRY(c.alloc(c.rho_ref_S, n)); SPH_TRY(c.alloc(c.SR, n));
    SPH_TRY(c.alloc(c.u0, n)); SPH_TRY(c.alloc(c.ft, n)); SPH_TRY(c.alloc(c.fp, n));
    SPH_TRY(c.alloc(c.dtemp, n)); SPH_TRY(c.alloc(c.nrm, n)); SPH_TRY(c.alloc(c.g6, 6 * (size_t)n));
    SPH_TRY(c.alloc(c.dconcn, n)); SPH_TRY(c.alloc(c.temp0, n)); SPH_TRY(c.alloc(c.concn0, n));
    SPH_TRY(c.alloc(c.enth0, n)); SPH_TRY(c.alloc(c.denth, n));
    SPH_TRY(c.alloc(c.tab, 2 * SPH_TABLE_SIZE));
    SPH_CUDA_TRY(cudaMemsetAsync(c.tab, 0, sizeof(Real) * 2 * SPH_TABLE_SIZE, c.stream));
    SPH_TRY(c.alloc(c.us_update, 1));
    SPH_CUDA_TRY(cudaMemsetAsync(c.us_update, 0, sizeof(float), c.stream));
    SPH_TRY(c.alloc(c.key, n)); SPH_TRY(c.alloc(c.perm, n)); SPH_TRY(c.alloc(c.g_idx, n));
    SPH_TRY(c.alloc(c.cell_start, (size_t)c.num_cells + 2));
    SPH_TRY(c.alloc(c.cell_fill, (size_t)c.num_cells + 2));
    SPH_TRY(c.alloc(c.scan_tmp, (size_t)scan_tmp_size(std::max((long long)n, (long long)c.num_cells + 2)) * 2));
    SPH_TRY(c.alloc(c.ncnt, n));
    SPH_TRY(c.alloc(c.slice_off, (size_t)(n + 31) / 32 + 2));
    SPH_TRY(c.alloc(c.diag, n));
    SPH_TRY(c.alloc(c.row_kind, n));
    SPH_TRY(c.alloc(c.row_aux, n));
    c.aos_bytes = sizeof(sph_part1) * (size_t)n + sizeof(sph_part2) * (size_t)n + sizeof(sph_part3) * (size_t)n;
    char *aos = nullptr;
    SPH_TRY(c.alloc(aos, c.aos_bytes));
    c.aos = aos;
    for (int k = 0; k < 8; ++k) SPH_CUDA_TRY(cudaEventCreate(&c.ev[k]));
    return SPH_OK;
}

// Records may sit in host memory (pageable or pinned) or in device memory:
// with unified addressing one cudaMemcpyDefault copy serves both.
static bool in_host_memory(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return true;
    }
    return a.type == cudaMemoryTypeUnregistered || a.type == cudaMemoryTypeHost;
}

// the |p_type| slots of the records the projection reaches (i_type < 3,
// p_type < 1000): bit t of out[0] for |p_type| = t < SPH_TABLE_SLOTS, out[1]
// set for any larger one
__global__ void k_ptype_slots(const sph_part1 *P1, int n, unsigned *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int it = P1[i].i_type, pt = P1[i].p_type;
    if (it >= 3 || pt >= 1000) return;
    const int t = pt < 0 ? -pt : pt;
    if (t < SPH_TABLE_SLOTS) atomicOr(&out[0], 1u << t);
    else atomicOr(&out[1], 1u);
}

template <class Real>
int ctx_upload(Ctx<Real> &c, const sph_part1 *P1, const sph_part2 *P2, int n) {
    if (n != c.n) { set_error("sph_upload: n differs from num_part2"); return SPH_ERR_BAD_ARG; }
    sph_part1 *d1 = (sph_part1 *)c.aos;
    sph_part2 *d2 = (sph_part2 *)((char *)c.aos + sizeof(sph_part1) * (size_t)n);
    SPH_CUDA_TRY(cudaMemcpyAsync(d1, P1, sizeof(sph_part1) * (size_t)n, cudaMemcpyDefault, c.stream));
    if (P2) SPH_CUDA_TRY(cudaMemcpyAsync(d2, P2, sizeof(sph_part2) * (size_t)n, cudaMemcpyDefault, c.stream));
    k_unpack<Real><<<grid_for(n, 256), 256, 0, c.stream>>>(c, d1, P2 ? d2 : nullptr, n);
    ++c.launches;
    SPH_CUDA_TRY(cudaGetLastError());
    // enthalpy0 of new records is 0 until a projection or sph_energy_convert sets it
    SPH_CUDA_TRY(cudaMemsetAsync(c.enth0, 0, sizeof(Real) * (size_t)n, c.stream));
    // the |p_type| slots htoT can read (records are only ever copied from
    // these: APR children and merged records keep their p_type)
    c.ptype_slots = 0;
    c.ptype_wide = false;
    if (in_host_memory(P1)) {
        for (int i = 0; i < n; ++i) {
            if (P1[i].i_type >= 3 || P1[i].p_type >= 1000) continue;
            const int t = P1[i].p_type < 0 ? -P1[i].p_type : P1[i].p_type;
            if (t < SPH_TABLE_SLOTS) c.ptype_slots |= 1u << t;
            else c.ptype_wide = true;
        }
    } else {
        if (!c.ptype_dev) SPH_TRY(c.alloc(c.ptype_dev, 2));
        SPH_CUDA_TRY(cudaMemsetAsync(c.ptype_dev, 0, 2 * sizeof(unsigned), c.stream));
        k_ptype_slots<<<grid_for(n, 256), 256, 0, c.stream>>>(d1, n, c.ptype_dev);
        ++c.launches;
        SPH_CUDA_TRY(cudaGetLastError());
        unsigned h[2] = {0, 0};
        SPH_CUDA_TRY(cudaMemcpyAsync(h, c.ptype_dev, sizeof(h), cudaMemcpyDeviceToHost, c.stream));
        SPH_CUDA_TRY(cudaStreamSynchronize(c.stream));
        c.ptype_slots = h[0];
        c.ptype_wide = h[1] != 0;
    }
    c.count = c.prm.vii[SPH_VII_COUNT];
    c.time = c.prm.vif[SPH_VIF_TIME];
    c.clk_synced = false;
    ++c.param_gen;
    c.release(c.apr_family);   // new records: APR families start again
    c.release(c.apr_target);
    c.uploaded = true;
    c.built = false;
    c.gc_valid = false;
    c.prep_valid = false;
    c.pforce_valid = false;
    c.coef_valid = false;
    return SPH_OK;
}

template <class Real>
int ctx_upload_state(Ctx<Real> &c, const sph_part1 *P1, int n) {
    if (n != c.n) { set_error("sph_upload_state: n differs from num_part2"); return SPH_ERR_BAD_ARG; }
    if (!c.built) { set_error("sph_upload_state: no sorted state yet (run a step first)"); return SPH_ERR_STATE; }
    sph_part1 *d1 = (sph_part1 *)c.aos;
    SPH_CUDA_TRY(cudaMemcpyAsync(d1, P1, sizeof(sph_part1) * (size_t)n, cudaMemcpyDefault, c.stream));
    k_unpack_state<Real><<<grid_for(n, 256), 256, 0, c.stream>>>(c, d1, n);
    ++c.launches;
    SPH_CUDA_TRY(cudaGetLastError());
    return SPH_OK;
}

template <class Real>
int ctx_download(Ctx<Real> &c, sph_part1 *P1, sph_part2 *P2, sph_part3 *P3) {
    const int n = c.n;
    sph_part1 *d1 = (sph_part1 *)c.aos;
    sph_part2 *d2 = (sph_part2 *)((char *)c.aos + sizeof(sph_part1) * (size_t)n);
    sph_part3 *d3 = (sph_part3 *)((char *)d2 + sizeof(sph_part2) * (size_t)n);
    k_pack<Real><<<grid_for(n, 128), 128, 0, c.stream>>>(c, P1 ? d1 : nullptr, P2 ? d2 : nullptr, P3 ? d3 : nullptr, n);
    ++c.launches;
    SPH_CUDA_TRY(cudaGetLastError());
    if (P1) SPH_CUDA_TRY(cudaMemcpyAsync(P1, d1, sizeof(sph_part1) * (size_t)n, cudaMemcpyDefault, c.stream));
    if (P2) SPH_CUDA_TRY(cudaMemcpyAsync(P2, d2, sizeof(sph_part2) * (size_t)n, cudaMemcpyDefault, c.stream));
    if (P3) SPH_CUDA_TRY(cudaMemcpyAsync(P3, d3, sizeof(sph_part3) * (size_t)n, cudaMemcpyDefault, c.stream));
    SPH_CUDA_TRY(cudaStreamSynchronize(c.stream));
    return SPH_OK;
}

// ---------------------------------------------------------------------------
// hash + counting sort
// ---------------------------------------------------------------------------
// KERNEL_set_ncell (functions_NNPS.cuh:943-955) fused with
// KERNEL_index_particle_to_cell (functions_NNPS.cuh:879-907) and the cell
// histogram of the counting sort.
__global__ void k_hash(DevParams P, const float4 *pf, const int4 *ty, const float *h_ref_f,
                       int *ncell, int *key, int *cell_cnt, int *dflag, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int4 t = ty[i];
    if (t.x == 3) {
        key[i] = P.num_cells;
        dflag[i] = 1;
        return;
    }
    dflag[i] = 0;
    const float4 x = pf[i];
    const float h0 = h_ref_f[i], h = x.w;
    ncell[i] = (int)(1.0 * (double)ceilf(__fdiv_rn(2.0f, __fdiv_rn(h0, h))));
    const int ic = bin_axis(x.x, P.xmin, P.xmax, P.NI);
    const int jc = bin_axis(x.y, P.ymin, P.ymax, P.NJ);
    const int kc = bin_axis(x.z, P.zmin, P.zmax, P.NK);
    const int k = ic + P.NI * jc + P.NI * P.NJ * kc;
    key[i] = k;
    atomicAdd(&cell_cnt[k], 1);
}

__global__ void k_scatter(const int *key, const int *cell_start, int *fill, const int *drank, int *perm,
                          int num_cells, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int k = key[i];
    int pos;
    if (k == num_cells) pos = cell_start[num_cells] + drank[i];
    else pos = cell_start[k] + atomicAdd(&fill[k], 1);
    perm[pos] = i;
}

// Orders every cell's segment of `perm` ascending: with the stable key order
// this reproduces the permutation of a stable radix sort of (key, index).
// Segments longer than 64 are left to k_sort_big.
__global__ void k_sort_small(const int *cell_start, int *perm, int *big, int *nbig, int num_cells) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= num_cells) return;
    const int s = cell_start[c], e = cell_start[c + 1], len = e - s;
    if (len <= 1) return;
    if (len > 64) { big[atomicAdd(nbig, 1)] = c; return; }
    int v[64];
    for (int a = 0; a < len; ++a) v[a] = perm[s + a];
    for (int a = 1; a < len; ++a) {
        int x = v[a], b = a - 1;
        while (b >= 0 && v[b] > x) { v[b + 1] = v[b]; --b; }
        v[b + 1] = x;
    }
    for (int a = 0; a < len; ++a) perm[s + a] = v[a];
}

// bitonic sort of up to 4096 indices in shared memory, one long segment per
// block at a time; the blocks stride over the list of long segments, so a
// small fixed grid (kSortBigGrid) serves any count
constexpr int kSortBigGrid = 296;
__global__ void k_sort_big(const int *cell_start, int *perm, const int *big, const int *nbig, int *err) {
    __shared__ int sv[4096];
    const int nb = *nbig;
    for (int q = blockIdx.x; q < nb; q += gridDim.x) {
        const int c = big[q];
        const int s = cell_start[c], len = cell_start[c + 1] - s;
        if (len > 4096) { if (threadIdx.x == 0) atomicExch(err, 1); continue; }
        int m = 1;
        while (m < len) m <<= 1;
        for (int a = threadIdx.x; a < m; a += blockDim.x) sv[a] = (a < len) ? perm[s + a] : 0x7fffffff;
        __syncthreads();
        for (int k = 2; k <= m; k <<= 1)
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int a = threadIdx.x; a < m; a += blockDim.x) {
                    const int b = a ^ j;
                    if (b > a) {
                        const bool up = (a & k) == 0;
                        const int x = sv[a], y = sv[b];
                        if ((x > y) == up) { sv[a] = y; sv[b] = x; }
                    }
                }
                __syncthreads();
            }
        for (int a = threadIdx.x; a < len; a += blockDim.x) perm[s + a] = sv[a];
        __syncthreads();   // sv is refilled by the next segment
    }
}

__global__ void k_sorted_keys(const int *key, const int *perm, int *g_idx, int n) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) g_idx[s] = key[perm[s]];
}

template <class T>
__global__ void k_gather(const T *src, T *dst, const int *perm, int n) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) dst[s] = src[perm[s]];
}

template <class Real>
__global__ void k_href_to_float(const Real *h_ref, float *out, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (float)h_ref[i];
}

// gathers one device array by `perm` through a scratch buffer
template <class Real, class T>
static int regather(Ctx<Real> &c, T *arr, void *scratch) {
    if (!arr) return SPH_OK;
    T *tmp = (T *)scratch;
    k_gather<T><<<grid_for(c.n, 256), 256, 0, c.stream>>>(arr, tmp, c.perm, c.n);
    ++c.launches;
    SPH_CUDA_TRY(cudaGetLastError());
    SPH_CUDA_TRY(cudaMemcpyAsync(arr, tmp, sizeof(T) * (size_t)c.n, cudaMemcpyDeviceToDevice, c.stream));
    return SPH_OK;
}

// ---------------------------------------------------------------------------
// canonical neighbour list in SELL-32 layout
// ---------------------------------------------------------------------------
// The reference visits, for particle i, the cells (z, y, x) in
// [-ncell, ncell]^3 around floor((x-xmin)/dcell) (functions_PPE.cuh:52-72)
// and particles j ascending inside each cell.  Cells of one (z, y) row are
// consecutive in the sorted array, so each row is one contiguous range and
// the row-by-row scan visits j in exactly the reference's order.  A pair is
// kept when sqrt(r2) < search_kappa * fmax(h_i, h_j) in FP32
// (functions_PPE.cuh:96-100; the +-1e-20 of the individual kernels does not
// change an FP32 comparison with a positive radius).
// The fill pass also writes the 16-bit codes of the pressure operator
// (nbr16, row_cell; flag16 set when a row cannot be coded: a search radius
// beyond two cells, or an offset beyond 8191 in its cell plane).
// One warp per row: the lanes test 32 consecutive candidates of a cell run
// at a time (coalesced loads of pf), __ballot_sync collects the kept ones
// and each kept lane writes its entry at the row's count plus the kept
// lanes below it (__popc), so the list keeps the visit order.  The count
// pass (FILL false) sizes the SELL slices, the fill pass writes them.
template <bool FILL>
__global__ void __launch_bounds__(128) k_list(DevParams P, const float4 *__restrict__ pf,
                                              const int4 *__restrict__ ty, const int *__restrict__ ncell,
                                              const int *__restrict__ cs, int *__restrict__ ncnt,
                                              const long long *__restrict__ slice_off, int *__restrict__ nbr,
                                              uint16_t *__restrict__ nbr16, int *__restrict__ row_cell,
                                              int *__restrict__ flag16, int n) {
    const int i = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= n) return;   // uniform over the warp
    int cnt = 0;
    if (FILL && nbr16 && lane == 0) row_cell[i] = 0;
    if (ty[i].x != 3) {
        const float4 xi = pf[i];
        const int ic = search_axis(xi.x, P.xmin, P.xmax, P.dcell, P.NI);
        const int jc = search_axis(xi.y, P.ymin, P.ymax, P.dcell, P.NJ);
        const int kc = search_axis(xi.z, P.zmin, P.zmax, P.dcell, P.NK);
        const int nc = ncell[i];
        const int x0 = max(ic - nc, 0), x1 = min(ic + nc, P.NI - 1);
        long long sb = 0, base = 0;
        if (FILL) { sb = slice_off[i >> 5]; base = sb + (i & 31); }
        const int rc = P.NI * jc + P.NI * P.NJ * kc + x0;
        if (FILL && nbr16 && lane == 0) {
            row_cell[i] = rc;
            if (nc > 2) atomicOr(flag16, 1);
        }
        const float reach_i = xi.w;
        for (int dz = -nc; dz <= nc; ++dz) {
            const int zz = kc + dz;
            if (zz < 0 || zz > P.NK - 1) continue;
            for (int dy = -nc; dy <= nc; ++dy) {
                const int yy = jc + dy;
                if (yy < 0 || yy > P.NJ - 1) continue;
                if (x0 > x1) continue;
                const int kb = P.NI * yy + P.NI * P.NJ * zz;
                const int s = cs[kb + x0], e = cs[kb + x1 + 1];
                const int s16 = (FILL && nbr16) ? cs[plane_cell(rc, dz, P.NI, P.NI * P.NJ, P.num_cells + 1)] : 0;
                for (int b0 = s; b0 < e; b0 += 32) {
                    const int j = b0 + lane;
                    bool keep = false;
                    if (j < e) {
                        const float4 xj = pf[j];
                        const float r = dist_rn(xi.x, xi.y, xi.z, xj.x, xj.y, xj.z);
                        keep = r < __fmul_rn(P.skappa, fmaxf(reach_i, xj.w));
                    }
                    const unsigned m = __ballot_sync(0xffffffffu, keep);
                    if (FILL && keep) {
                        const int pos = cnt + __popc(m & ((1u << lane) - 1u));
                        nbr[base + (long long)pos * 32] = j;
                        if (nbr16) {
                            const int off = j - s16;
                            if (off < 0 || off > (int)kCodeMask) atomicOr(flag16, 2);
                            nbr16[sell4(sb, i & 31, pos)] =
                                (uint16_t)(((unsigned)(dz + 2) << kCodeShift) | ((unsigned)off & kCodeMask));
                        }
                    }
                    cnt += __popc(m);
                }
            }
        }
    }
    if (!FILL && lane == 0) ncnt[i] = cnt;
}

// slice width (max count of the 32 particles of a slice, rounded up to a
// multiple of four) * 32
__global__ void k_slice_width(const int *ncnt, long long *w, int n, int nslices) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslices) return;
    int m = 0;
    for (int l = 0; l < 32; ++l) {
        const int i = s * 32 + l;
        if (i < n) m = max(m, ncnt[i]);
    }
    w[s] = (long long)((m + 3) & ~3) * 32;   // a multiple of four entries per row (sell4)
}

// ---------------------------------------------------------------------------
// side lists (CSR, built on the host from device copies; they touch small
// subsets: markers, walls, buffers, wall-layer particles)
// ---------------------------------------------------------------------------
struct HostGrid {
    DevParams P;
    std::vector<float4> pf;
    std::vector<int4> ty;
    std::vector<int> ncell, cs, jc;
    template <class F>
    void cell_loop(int ic, int jc_, int kc, int nc, F f) const {
        for (int z = -nc; z <= nc; z++)
            for (int y = -nc; y <= nc; y++)
                for (int x = -nc; x <= nc; x++) {
                    if (ic + x < 0 || ic + x > P.NI - 1 || jc_ + y < 0 || jc_ + y > P.NJ - 1 || kc + z < 0 || kc + z > P.NK - 1) continue;
                    const int k = (ic + x) + P.NI * (jc_ + y) + P.NI * P.NJ * (kc + z);
                    for (int j = cs[k]; j < cs[k + 1]; j++) f(j);
                }
    }
    void search_cell(float x, float y, float z, int &ic, int &jc_, int &kc) const {
        ic = search_axis(x, P.xmin, P.xmax, P.dcell, P.NI);
        jc_ = search_axis(y, P.ymin, P.ymax, P.dcell, P.NJ);
        kc = search_axis(z, P.zmin, P.zmax, P.dcell, P.NK);
    }
    void bin_cell(float x, float y, float z, int &ic, int &jc_, int &kc) const {
        ic = bin_axis(x, P.xmin, P.xmax, P.NI);
        jc_ = bin_axis(y, P.ymin, P.ymax, P.NJ);
        kc = bin_axis(z, P.zmin, P.zmax, P.NK);
    }
};

// a position wrapped into the periodic box (axes with x1 > x0), in double:
// v - L floor((v - x0) / L)
static inline void periodic_wrap(const double *box, float x, float y, float z, double *w) {
    const float v[3] = {x, y, z};
    for (int a = 0; a < 3; ++a) {
        const double lo = box[2 * a], len = box[2 * a + 1] - box[2 * a];
        w[a] = (len > 0) ? (double)v[a] - len * std::floor(((double)v[a] - lo) / len) : (double)v[a];
    }
}

static inline float hdist(float xi, float yi, float zi, float xj, float yj, float zj) {
    volatile float dx = xi - xj, dy = yi - yj, dz = zi - zj;
    volatile float a = dx * dx, b = dy * dy, cc = dz * dz;
    volatile float s = a + b;
    volatile float t = s + cc;
    return std::sqrt((float)t);
}

template <class Real, class T>
static int upload_vec(Ctx<Real> &c, T *&dst, const std::vector<T> &v) {
    c.release(dst);   // a rebuild replaces the previous list
    SPH_TRY(c.alloc(dst, v.size()));
    if (!v.empty()) SPH_CUDA_TRY(cudaMemcpyAsync(dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, c.stream));
    return SPH_OK;
}

// ---------------------------------------------------------------------------
// connected components of the pressure operator's graph (min-label
// propagation with pointer jumping) and one pinned row per component that has
// no anchor row; the oracle applies the same rule (sph_oracle.cpp, assemble)
// ---------------------------------------------------------------------------
__global__ void k_cc_init(int *label, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) label[i] = i;
}

__device__ __forceinline__ void cc_link(int *label, int a, int b, int *changed) {
    const int la = label[a], lb = label[b];
    if (la == lb) return;
    if (la < lb) { if (atomicMin(&label[b], la) > la) *changed = 1; }
    else { if (atomicMin(&label[a], lb) > lb) *changed = 1; }
}

__global__ void k_cc_fluid(const int *kind, const int *jc, const long long *slice_off, const int *ncnt, const int *nbr,
                           int *label, int *changed, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || kind[i] != 1) return;
    const long long base = slice_off[i >> 5] + (i & 31);
    const int cnt = ncnt[i];
    for (int k = 0; k < cnt; ++k) {
        const int j = nbr[base + 32LL * k];
        const int c = jc[j];
        if (j == i || !(c & JB_LT1000) || (c & JB_IT4)) continue;
        cc_link(label, i, j, changed);
    }
}

__global__ void k_cc_csr(const int *rows, const int *off, const int *nb, int nrows, int *label, int *changed) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nrows) return;
    for (int q = off[k]; q < off[k + 1]; ++q) cc_link(label, rows[k], nb[q], changed);
}

__global__ void k_cc_pairs(const int *rows, const int *partner, int nrows, int *label, int *changed) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nrows || partner[k] < 0) return;
    cc_link(label, rows[k], partner[k], changed);
}

__global__ void k_cc_jump(int *label, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int l = label[i];
    while (label[l] != l) l = label[l];
    label[i] = l;
}

// Singular components of the pressure operator (no anchor row: no identity
// row, no Neumann row without fluid in range, no outlet row without partner)
// get either the rank-one mean-pressure term (ppe_pin == 1, up to
// SPH_MAX_COMP components) or one row pinned to p = 0 (ppe_pin == 2, and any
// component beyond SPH_MAX_COMP).  Same rule as the oracle (sph_oracle.cpp,
// assemble).
template <class Real>
static int null_components(Ctx<Real> &c, std::vector<int> &kind, const std::vector<int> &nm_rows,
                           const std::vector<int> &nm_flags, const std::vector<int> &aux, const std::vector<int4> &ty) {
    const int n = c.n;
    cudaStream_t st = c.stream;
    int *label = nullptr, *flag = nullptr;
    SPH_TRY(c.alloc(label, n));
    SPH_TRY(c.alloc(flag, 2));
    SPH_CUDA_TRY(cudaMemcpyAsync(c.row_kind, kind.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
    k_cc_init<<<grid_for(n, 256), 256, 0, st>>>(label, n);
    ++c.launches;
    int changed = 1, rounds = 0;
    while (changed && rounds < 100000) {
        SPH_CUDA_TRY(cudaMemsetAsync(flag, 0, sizeof(int), st));
        k_cc_fluid<<<grid_for(n, 128), 128, 0, st>>>(c.row_kind, c.jc, c.slice_off, c.ncnt, c.nbr, label, flag, n);
        if (c.L.n_nm) k_cc_csr<<<grid_for(c.L.n_nm, 128), 128, 0, st>>>(c.L.nm_rows, c.L.nm_off, c.L.nm_nbr, c.L.n_nm, label, flag);
        if (c.L.n_out) k_cc_pairs<<<grid_for(c.L.n_out, 128), 128, 0, st>>>(c.L.out_rows, c.L.out_partner, c.L.n_out, label, flag);
        if (c.L.n_gh) k_cc_pairs<<<grid_for(c.L.n_gh, 128), 128, 0, st>>>(c.L.gh_rows, c.L.gh_partner, c.L.n_gh, label, flag);
        k_cc_jump<<<grid_for(n, 256), 256, 0, st>>>(label, n);
        c.launches += 4 + (c.L.n_gh ? 1 : 0);
        SPH_CUDA_TRY(cudaMemcpyAsync(&changed, flag, sizeof(int), cudaMemcpyDeviceToHost, st));
        SPH_CUDA_TRY(cudaStreamSynchronize(st));
        ++rounds;
    }
    SPH_CUDA_TRY(cudaGetLastError());
    std::vector<int> lab(n);
    SPH_CUDA_TRY(cudaMemcpyAsync(lab.data(), label, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
    SPH_CUDA_TRY(cudaStreamSynchronize(st));
    c.release(label);
    c.release(flag);
    std::vector<char> anchored(n, 0);
    std::vector<int> cand(n, -1), cand_any(n, -1), cid(n, -1), comp(n, -1);
    for (int i = 0; i < n; ++i) {
        const int kd = kind[i];
        if (kd == 0 || (kd == 3 && aux[i] < 0)) anchored[lab[i]] = 1;
        if (kd == 1) {
            cand_any[lab[i]] = std::max(cand_any[lab[i]], i);
            if (ty[i].y == 0) cand[lab[i]] = std::max(cand[lab[i]], i);
        }
    }
    // a Neumann row without fluid in range is an identity row of the operator
    // (an anchor); a Neumann candidate that is a copy row anchors only
    // without partner (above), as in the oracle
    for (size_t k = 0; k < nm_rows.size(); ++k)
        if ((nm_flags[k] & 4) && kind[nm_rows[k]] == 2) anchored[lab[nm_rows[k]]] = 1;
    c.n_pins = 0;
    c.n_comp = 0;
    for (int r = 0; r < n; ++r) {
        if (lab[r] != r || anchored[r] || cand_any[r] < 0) continue;
        if (c.prm.ppe_pin == 2 || c.n_comp >= SPH_MAX_COMP) {
            kind[cand[r] >= 0 ? cand[r] : cand_any[r]] = 4;
            ++c.n_pins;
        } else {
            cid[r] = c.n_comp++;
        }
    }
    std::vector<double> inv(SPH_MAX_COMP, 0.0);
    std::vector<long long> cnt(SPH_MAX_COMP, 0);
    for (int i = 0; i < n; ++i)
        if (kind[i] == 1 && cid[lab[i]] >= 0) { comp[i] = cid[lab[i]]; cnt[comp[i]]++; }
    for (int k = 0; k < c.n_comp; ++k) inv[k] = cnt[k] ? 1.0 / (double)cnt[k] : 0.0;
    if (!c.comp_id) SPH_TRY(c.alloc(c.comp_id, n));
    if (!c.comp_inv) SPH_TRY(c.alloc(c.comp_inv, SPH_MAX_COMP));
    SPH_CUDA_TRY(cudaMemcpyAsync(c.comp_id, comp.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
    SPH_CUDA_TRY(cudaMemcpyAsync(c.comp_inv, inv.data(), sizeof(double) * SPH_MAX_COMP, cudaMemcpyHostToDevice, st));
    SPH_CUDA_TRY(cudaMemcpyAsync(c.row_kind, kind.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
    SPH_CUDA_TRY(cudaStreamSynchronize(st));
    return SPH_OK;
}

template <class Real>
int build_side_lists(Ctx<Real> &c) {
    const int n = c.n;
    HostGrid G;
    G.P = c.dp;
    G.pf.resize(n); G.ty.resize(n); G.ncell.resize(n); G.cs.resize((size_t)c.num_cells + 2); G.jc.resize(n);
    SPH_CUDA_TRY(cudaMemcpyAsync(G.pf.data(), c.pf, sizeof(float4) * n, cudaMemcpyDeviceToHost, c.stream));
    SPH_CUDA_TRY(cudaMemcpyAsync(G.ty.data(), c.ty, sizeof(int4) * n, cudaMemcpyDeviceToHost, c.stream));
    SPH_CUDA_TRY(cudaMemcpyAsync(G.ncell.data(), c.ncell, sizeof(int) * n, cudaMemcpyDeviceToHost, c.stream));
    SPH_CUDA_TRY(cudaMemcpyAsync(G.cs.data(), c.cell_start, sizeof(int) * ((size_t)c.num_cells + 2), cudaMemcpyDeviceToHost, c.stream));
    std::vector<typename Ctx<Real>::R4> pr(n);
    std::vector<typename Ctx<Real>::R2> mr(n);
    SPH_CUDA_TRY(cudaMemcpyAsync(pr.data(), c.pr, sizeof(pr[0]) * n, cudaMemcpyDeviceToHost, c.stream));
    SPH_CUDA_TRY(cudaMemcpyAsync(mr.data(), c.mr, sizeof(mr[0]) * n, cudaMemcpyDeviceToHost, c.stream));
    SPH_CUDA_TRY(cudaStreamSynchronize(c.stream));
    const DevParams &P = c.dp;
    SideLists &L = c.L;
    std::vector<int> rows, off, nb, zero;

    // IBM marker interpolation list, functions_IBM.cuh:369-436
    rows.clear(); off.assign(1, 0); nb.clear();
    for (int i = 0; i < n; ++i) {
        if (G.ty[i].w < 1000) continue;
        rows.push_back(i);
        const float4 xi = G.pf[i];
        const float sr = P.skappa * (float)(P.ibm_length * xi.w);
        int ic, jc, kc;
        G.bin_cell(xi.x, xi.y, xi.z, ic, jc, kc);
        G.cell_loop(ic, jc, kc, G.ncell[i], [&](int j) {
            if (G.ty[j].x == 4 || G.ty[j].w != 1) return;
            const float4 xj = G.pf[j];
            if (hdist(xi.x, xi.y, xi.z, xj.x, xj.y, xj.z) < sr) nb.push_back(j);
        });
        off.push_back((int)nb.size());
    }
    L.n_mk = (int)rows.size();
    SPH_TRY(upload_vec(c, L.mk_rows, rows)); SPH_TRY(upload_vec(c, L.mk_off, off)); SPH_TRY(upload_vec(c, L.mk_nbr, nb));

    // IBM spreading list, functions_IBM.cuh:523-592 (fluid rows with at least
    // one marker in range; the others get fb = 0 every step)
    rows.clear(); off.assign(1, 0); nb.clear(); zero.clear();
    bool any_marker = false;
    for (int i = 0; i < n; ++i) if (G.ty[i].w == 1000) { any_marker = true; break; }
    for (int i = 0; i < n; ++i) {
        if (G.ty[i].w != 1 || G.ty[i].y == 2) continue;
        size_t before = nb.size();
        if (any_marker) {
            const float4 xi = G.pf[i];
            const float sr = P.skappa * (float)(P.ibm_length * xi.w);
            int ic, jc, kc;
            G.bin_cell(xi.x, xi.y, xi.z, ic, jc, kc);
            G.cell_loop(ic, jc, kc, G.ncell[i], [&](int j) {
                if (G.ty[j].x == 4 || G.ty[j].w != 1000) return;
                const float4 xj = G.pf[j];
                if (hdist(xi.x, xi.y, xi.z, xj.x, xj.y, xj.z) < sr) nb.push_back(j);
            });
        }
        if (nb.size() == before) zero.push_back(i);
        else { rows.push_back(i); off.push_back((int)nb.size()); }
    }
    L.n_sp = (int)rows.size();
    L.n_sp_zero = (int)zero.size();
    SPH_TRY(upload_vec(c, L.sp_rows, rows)); SPH_TRY(upload_vec(c, L.sp_off, off)); SPH_TRY(upload_vec(c, L.sp_nbr, nb));
    SPH_TRY(upload_vec(c, L.sp_zero, zero));

    // Neumann rows, functions_BC.cuh:290-446: fluid (p_type 1, buffer 0)
    // neighbours within search_kappa*2h of the (possibly mirrored) node, the
    // ghost partner within ghost_tol, and the linear weights of the row
    rows.clear(); off.assign(1, 0); nb.clear();
    std::vector<int> ghost, mir, aux;
    std::vector<double> w, gw;
    auto calc_tmpA_h = [&](double tH) -> double {
        const double k = P.kappa;
        switch (P.kernel_type) {
            case 0: return 1.0 / (pow(3.141592653, 1.5) * pow(tH, 3));
            case 1: return 3.0 / (359.0 * 3.141592653 * pow(tH, 3));
            case 2: return 315.0 / (208.0 * 3.141592653 * pow(tH, 3));
            case 3: return 3.342253804929802 / (k * tH) / (k * tH) / (k * tH);
            case 4: return 4.923856051905513 / (k * tH) / (k * tH) / (k * tH);
            case 5: return 6.788953041263660 / (k * tH) / (k * tH) / (k * tH);
        }
        return 0;
    };
    auto w_h = [&](double tA, double tH, double rr) -> double {
        const double tR = rr / tH / P.kappa, o = 1 - tR;
        if (tR >= 1 && P.kernel_type >= 2) return 0;
        switch (P.kernel_type) {
            case 0: return tA * exp(-(2 * tR) * (2 * tR));
            case 1:
                if (tR < 0.5) return tA * (pow(3 - 2 * tR, 5) - 6 * pow(2 - 2 * tR, 5) + 15 * pow(1 - 2 * tR, 5));
                if (tR < 1) return tA * (pow(3 - 2 * tR, 5) - 6 * pow(2 - 2 * tR, 5));
                if (tR < 1.5) return tA * pow(3 - 2 * tR, 5);
                return 0;
            case 2: return tA * (2.0 / 3 - 4.5 * tR * tR + 19.0 / 3 * tR * tR * tR - 2.5 * tR * tR * tR * tR);
            case 3: return tA * pow(o, 4) * (1 + 4 * tR);
            case 4: return tA * pow(o, 6) * (1 + 6 * tR + 11.666666666666666 * tR * tR);
            case 5: return tA * pow(o, 8) * (1 + 8 * tR + 25 * tR * tR + 32 * tR * tR * tR);
        }
        return 0;
    };
    auto dw_h = [&](double tA, double tH, double rr) -> double {
        const double k = P.kappa, tR = rr / tH / k, o = 1 - tR;
        if (tR >= 1 && P.kernel_type >= 2) return 0;
        switch (P.kernel_type) {
            case 0: return (1.0 / tH) * tA * (-4 * tR) * exp(-(2 * tR) * (2 * tR));
            case 1:
                if (tR < 0.5) return (1 / tH) * tA * (-5 * pow(3 - 2 * tR, 4) + 30 * pow(2 - 2 * tR, 4) - 75 * pow(1 - 2 * tR, 4));
                if (tR < 1) return (1 / tH) * tA * (-5 * pow(3 - 2 * tR, 4) + 30 * pow(2 - 2 * tR, 4));
                if (tR < 1.5) return (1 / tH) * tA * (-5 * pow(3 - 2 * tR, 4));
                return 0;
            case 2: return (1 / tH) * tA * (-9 * tR + 19 * tR * tR - 10 * tR * tR * tR);
            case 3: return (1 / (k * tH)) * tA * (-20 * tR * pow(o, 3));
            case 4: return (1 / (k * tH)) * tA * (-18.666666666666668 * tR * pow(o, 5) * (5 * tR + 1));
            case 5: return (1 / (k * tH)) * tA * (-22 * tR * pow(o, 7) * (16 * tR * tR + 7 * tR + 1));
        }
        return 0;
    };
    std::vector<double> ow;
    for (int i = 0; i < n; ++i) {
        if (G.ty[i].w == 1 || G.ty[i].x >= 3) continue;
        rows.push_back(i);
        const float4 xi = G.pf[i];
        const bool mirror = (G.ty[i].y == 1 || G.ty[i].y == -1);
        const float sc = (float)P.neumann_coeff;
        const float srange = P.skappa * (float)(sc * xi.w);
        const double xid = (double)pr[i].x, yid = (double)pr[i].y, zid = (double)pr[i].z;
        const double xg = mirror ? (double)(Real)(2.0 * P.l2 - (double)pr[i].x) : xid;
        const float xgf = mirror ? (float)(2.0 * P.l2 - xi.x) : xi.x;
        int ic, jc, kc;
        G.search_cell(xgf, xi.y, xi.z, ic, jc, kc);
        int g = -1;
        G.cell_loop(ic, jc, kc, 1, [&](int j) {
            const double d = std::sqrt((xg - pr[j].x) * (xg - pr[j].x) + (yid - pr[j].y) * (yid - pr[j].y) + (zid - pr[j].z) * (zid - pr[j].z));
            if (d - 1e-20 < P.ghost_tol) g = j;
        });
        const double hi = (double)sc * (double)(Real)xi.w;
        const double tA = calc_tmpA_h(hi);
        // pass 0: the reference's Shepard set (fluid with buffer_type 0);
        // pass 1, only when pass 0 is empty: all fluid in range, for the
        // converged operator (the pass itself then writes p = 0)
        int flags = mirror ? 1 : 0;
        for (int pass = 0; pass < 2; ++pass) {
            std::vector<int> js;
            std::vector<double> ww, gg;
            double tflt = 0, gsum = 0;
            G.cell_loop(ic, jc, kc, G.ncell[i], [&](int j) {
                if (G.ty[j].w >= 1000) return;
                if (!(G.ty[j].w == 1 && (pass == 1 || G.ty[j].y == 0))) return;
                const float4 xj = G.pf[j];
                if (!(hdist(xgf, xi.y, xi.z, xj.x, xj.y, xj.z) < srange)) return;
                const double dx = xg - pr[j].x, dy = yid - pr[j].y, dz = zid - pr[j].z;
                const double r = std::sqrt(dx * dx + dy * dy + dz * dz);
                const double vw = (double)mr[j].x / (double)mr[j].y;
                const double wv = w_h(tA, hi, r);
                double dwv = (r > 0) ? dw_h(tA, hi, r) : 0.0;
                if (P.kgc_solve == 1) dwv = 0;
                const double proj = (r > 0) ? ((xid - xg) * dx) / r * dwv : 0.0;
                js.push_back(j); ww.push_back(vw * wv); gg.push_back(vw * proj);
                tflt += vw * wv; gsum += vw * proj;
            });
            if (tflt < 1e-6) {
                if (pass == 0) { flags |= 2; continue; }   // the pass writes p = 0
                flags |= 4;                                // no fluid at all: anchor (p = 0)
                break;
            }
            for (size_t k = 0; k < js.size(); ++k) {
                nb.push_back(js[k]);
                const double sh = ww[k] / tflt;
                ow.push_back(sh);
                w.push_back(pass == 0 ? sh : 0.0);
                gw.push_back(pass == 0 && mirror ? gg[k] : 0.0);
            }
            if (pass == 0 && mirror && g >= 0) { nb.push_back(g); w.push_back(0.0); gw.push_back(1.0 - gsum); ow.push_back(0.0); }
            break;
        }
        off.push_back((int)nb.size());
        mir.push_back(flags);
    }
    L.n_nm = (int)rows.size();
    L.nm_nnz = (long long)nb.size();
    const std::vector<int> nmr = rows, nmo = off;
    SPH_TRY(upload_vec(c, L.nm_rows, rows)); SPH_TRY(upload_vec(c, L.nm_off, off)); SPH_TRY(upload_vec(c, L.nm_nbr, nb));
    SPH_TRY(upload_vec(c, L.nm_ghost, mir));
    SPH_TRY(upload_vec(c, c.nm_w, w));
    SPH_TRY(upload_vec(c, c.nm_gw, gw));
    SPH_TRY(upload_vec(c, c.nm_ow, ow));
    if (sizeof(Real) == 4) {
        const std::vector<float> owf(ow.begin(), ow.end());
        SPH_TRY(upload_vec(c, c.nm_owf, owf));
    }
    const std::vector<int> nmflags = mir;

    // periodic partners, functions_BC.cuh:1041-1133
    rows.clear(); nb.clear();
    for (int i = 0; i < n; ++i) {
        const int bt = G.ty[i].y;
        if (bt == 0 || G.ty[i].w >= 1000) continue;
        if (bt != 3 && bt != 4) continue;
        rows.push_back(i);
        const Real yR = (bt == 3) ? (Real)((double)pr[i].y + P.l_right - P.l_left) : (Real)((double)pr[i].y - P.l_right + P.l_left);
        const float ygf = (bt == 3) ? (float)((double)G.pf[i].y + P.l_right - P.l_left) : (float)((double)G.pf[i].y - P.l_right + P.l_left);
        int ic, jc, kc;
        G.search_cell(G.pf[i].x, ygf, G.pf[i].z, ic, jc, kc);
        const int nc = G.ncell[i];
        int found = -1;
        bool flag = false;
        for (int z = -nc; z <= nc; z++)
            for (int y = -nc; y <= nc; y++)
                for (int x = -nc; x <= nc; x++) {
                    if (flag) continue;
                    if (ic + x < 0 || ic + x > P.NI - 1 || jc + y < 0 || jc + y > P.NJ - 1 || kc + z < 0 || kc + z > P.NK - 1) continue;
                    const int k = (ic + x) + P.NI * (jc + y) + P.NI * P.NJ * (kc + z);
                    for (int j = G.cs[k]; j < G.cs[k + 1]; j++) {
                        const Real dx = pr[i].x - pr[j].x, dy = yR - pr[j].y, dz = pr[i].z - pr[j].z;
                        const Real d = (Real)(std::sqrt(dx * dx + dy * dy + dz * dz) - 1e-20);
                        if (d < P.partner_tol) { found = j; flag = true; }
                    }
                }
        nb.push_back(found);
    }
    L.n_per = (int)rows.size();
    SPH_TRY(upload_vec(c, L.per_rows, rows)); SPH_TRY(upload_vec(c, L.per_partner, nb));

    // ghosts of the periodic box (buffer 7): the record at the ghost's
    // position wrapped into the box, |d| < partner_tol, ghosts excluded; the
    // last match in cell order wins, as in the outlet search below
    std::vector<int> gh_rows, gh_nb;
    for (int i = 0; i < n; ++i) {
        if (G.ty[i].y != SPH_BUFFER_PERIODIC_GHOST) continue;
        gh_rows.push_back(i);
        double w[3];
        periodic_wrap(P.periodic_box, G.pf[i].x, G.pf[i].y, G.pf[i].z, w);
        int ic, jc, kc;
        G.search_cell((float)w[0], (float)w[1], (float)w[2], ic, jc, kc);
        int found = -1;
        G.cell_loop(ic, jc, kc, 1, [&](int j) {
            if (G.ty[j].y == SPH_BUFFER_PERIODIC_GHOST) return;
            const double dx = w[0] - (double)G.pf[j].x, dy = w[1] - (double)G.pf[j].y, dz = w[2] - (double)G.pf[j].z;
            if (std::sqrt(dx * dx + dy * dy + dz * dz) < P.partner_tol) found = j;
        });
        gh_nb.push_back(found);
    }
    L.n_gh = (int)gh_rows.size();
    SPH_TRY(upload_vec(c, L.gh_rows, gh_rows)); SPH_TRY(upload_vec(c, L.gh_partner, gh_nb));

    // outlet partners, functions_BC.cuh:673-761
    rows.clear(); nb.clear();
    for (int i = 0; i < n; ++i) {
        if (G.ty[i].y != 2) continue;
        rows.push_back(i);
        int ic, jc, kc;
        G.search_cell(G.pf[i].x, G.pf[i].y, G.pf[i].z, ic, jc, kc);
        const Real xg = (Real)(P.l3 - P.outlet_probe_dx);
        int found = -1;
        G.cell_loop(ic, jc, kc, 2 * G.ncell[i], [&](int j) {
            const Real dx = xg - pr[j].x, dy = pr[i].y - pr[j].y, dz = pr[i].z - pr[j].z;
            const Real d = (Real)(std::sqrt(dx * dx + dy * dy + dz * dz) - 1e-20);
            if (G.ty[j].w < 1000 && d < P.partner_tol) found = j;
        });
        nb.push_back(found);
    }
    L.n_out = (int)rows.size();
    SPH_TRY(upload_vec(c, L.out_rows, rows)); SPH_TRY(upload_vec(c, L.out_partner, nb));
    aux.assign(n, -1);
    for (size_t k = 0; k < rows.size(); ++k) aux[rows[k]] = nb[k];
    for (size_t k = 0; k < gh_rows.size(); ++k) aux[gh_rows[k]] = gh_nb[k];
    SPH_CUDA_TRY(cudaMemcpyAsync(c.row_aux, aux.data(), sizeof(int) * n, cudaMemcpyHostToDevice, c.stream));
    SPH_CUDA_TRY(cudaStreamSynchronize(c.stream));

    // extrapolation rows, functions_BC.cuh:763-855: outlet records off the
    // MOST layer; fluid (p_type 1, off the MOST layer) within kappa h_i of the
    // mirror node (2 L3 - x, y, z), cells by the normalised binning there
    rows.clear(); off.assign(1, 0); nb.clear();
    for (int i = 0; i < n; ++i) {
        if (G.ty[i].y != 2 || G.ty[i].z == 1) continue;
        rows.push_back(i);
        const Real xg = (Real)(2 * P.l3 - (double)pr[i].x);
        const float xgf = (float)(2 * P.l3 - (double)G.pf[i].x);
        const Real range = (Real)P.skappa * pr[i].w;
        int ic, jc, kc;
        G.bin_cell(xgf, G.pf[i].y, G.pf[i].z, ic, jc, kc);
        G.cell_loop(ic, jc, kc, G.ncell[i], [&](int j) {
            if (G.ty[j].w != 1 || G.ty[j].z == 1) return;
            const Real dx = xg - pr[j].x, dy = pr[i].y - pr[j].y, dz = pr[i].z - pr[j].z;
            const Real d = (Real)(std::sqrt(dx * dx + dy * dy + dz * dz) - 1e-20);
            if (d < range) nb.push_back(j);
        });
        off.push_back((int)nb.size());
    }
    L.n_xo = (int)rows.size();
    SPH_TRY(upload_vec(c, L.xo_rows, rows)); SPH_TRY(upload_vec(c, L.xo_off, off)); SPH_TRY(upload_vec(c, L.xo_nbr, nb));

    // inout rows, functions_BC.cuh:1274-1433: side buffers take the record
    // at 0.001 of their periodic image (the last one in the first cell that
    // has one), outlet records the interior fluid (buffer 0, p_type 1)
    // within kappa h_i of (L3, y, z)
    {
        std::vector<int> io_rows, io_aux, io_off(1, 0), io_nb;
        for (int i = 0; i < n; ++i) {
            const int bt = G.ty[i].y;
            if ((bt != 3 && bt != 4) || G.ty[i].w >= 1000) continue;
            io_rows.push_back(i);
            const Real yR = (bt == 3) ? (Real)((double)pr[i].y + P.l_right - P.l_left) : (Real)((double)pr[i].y - P.l_right + P.l_left);
            const float ygf = (bt == 3) ? (float)((double)G.pf[i].y + P.l_right - P.l_left) : (float)((double)G.pf[i].y - P.l_right + P.l_left);
            int ic, jc, kc;
            G.search_cell(G.pf[i].x, ygf, G.pf[i].z, ic, jc, kc);
            const int nc = G.ncell[i];
            int found = -1;
            bool flag = false;
            for (int z = -nc; z <= nc; z++)
                for (int y = -nc; y <= nc; y++)
                    for (int x = -nc; x <= nc; x++) {
                        if (flag) continue;
                        if (ic + x < 0 || ic + x > P.NI - 1 || jc + y < 0 || jc + y > P.NJ - 1 || kc + z < 0 || kc + z > P.NK - 1) continue;
                        const int k = (ic + x) + P.NI * (jc + y) + P.NI * P.NJ * (kc + z);
                        for (int j = G.cs[k]; j < G.cs[k + 1]; j++) {
                            const Real dx = pr[i].x - pr[j].x, dy = yR - pr[j].y, dz = pr[i].z - pr[j].z;
                            const Real d = (Real)(std::sqrt(dx * dx + dy * dy + dz * dz) - 1e-20);
                            if (d < (Real)0.001) { found = j; flag = true; }
                        }
                    }
            io_aux.push_back(found);
        }
        L.n_ios = (int)io_rows.size();
        for (int i = 0; i < n; ++i) {
            if (G.ty[i].y != 2 || G.ty[i].w >= 1000) continue;
            io_rows.push_back(i);
            const Real range = (Real)P.skappa * pr[i].w;
            int ic = (int)std::min(std::floor((P.l3 - (double)P.xmin) / (double)P.dcell), (double)(P.NI - 1));
            if (ic < 0) ic = 0;
            int ic_unused, jc, kc;
            G.search_cell(G.pf[i].x, G.pf[i].y, G.pf[i].z, ic_unused, jc, kc);
            G.cell_loop(ic, jc, kc, G.ncell[i], [&](int j) {
                if (G.ty[j].y != 0 || G.ty[j].w != 1) return;
                const Real dx = (Real)(P.l3 - (double)pr[j].x), dy = pr[i].y - pr[j].y, dz = pr[i].z - pr[j].z;
                const Real d = (Real)(std::sqrt(dx * dx + dy * dy + dz * dz) - 1e-20);
                if (d < range) io_nb.push_back(j);
            });
            io_off.push_back((int)io_nb.size());
        }
        L.n_io = (int)io_rows.size();
        SPH_TRY(upload_vec(c, L.io_rows, io_rows)); SPH_TRY(upload_vec(c, L.io_aux, io_aux));
        SPH_TRY(upload_vec(c, L.io_off, io_off)); SPH_TRY(upload_vec(c, L.io_nbr, io_nb));
    }

    // recycling rows, functions_BC.cuh:1861: buffer type 1 or -1
    rows.clear();
    for (int i = 0; i < n; ++i)
        if (G.ty[i].y == 1 || G.ty[i].y == -1) rows.push_back(i);
    L.n_rc = (int)rows.size();
    SPH_TRY(upload_vec(c, L.rc_rows, rows));

    // MOST wall-layer particles and their ghost-node targets, functions_MOST.cuh:262-305
    rows.clear(); off.assign(1, 0); nb.clear();
    for (int i = 0; i < n; ++i) {
        if (G.ty[i].z != 1) continue;
        rows.push_back(i);
        const float xg = (float)pr[i].x, yg = (float)pr[i].y, zg = (float)((double)(float)pr[i].z + P.most_ghost_dz);
        int ic, jc, kc;
        G.search_cell(xg, yg, zg, ic, jc, kc);
        G.cell_loop(ic, jc, kc, 1, [&](int j) {
            const double dx = xg - (double)pr[j].x, dy = yg - (double)pr[j].y, dz = zg - (double)pr[j].z;
            if (std::sqrt(dx * dx + dy * dy + dz * dz) - 1e-20 < P.ghost_tol) nb.push_back(j);
        });
        off.push_back((int)nb.size());
    }
    L.n_most = (int)rows.size();
    SPH_TRY(upload_vec(c, L.most_rows, rows)); SPH_TRY(upload_vec(c, L.most_off, off)); SPH_TRY(upload_vec(c, L.most_tgt, nb));

    // row classes of the passes
    std::vector<int> fl, wl, fs, kind(n, 0);
    for (int i = 0; i < n; ++i) {
        const int4 t = G.ty[i];
        if (!(t.x > 2 || t.w >= 1000 || t.w <= 0)) fl.push_back(i);
        if (t.x <= 2 && t.w <= 0 && t.w == 0) wl.push_back(i);
        if (t.w == -1) fs.push_back(i);
        // converged-PPE row classes (precedence of the reference's overwrites:
        // outlet copy after Neumann after the PPE sweep).  A record that is
        // both an outlet buffer and a Neumann row (a free-slip record past L3)
        // is a copy row, as the outlet copy overwrites the Neumann value; a
        // periodic-box ghost is a copy row too
        if (t.x >= 3) kind[i] = 0;
        else if (t.y == 2 || t.y == SPH_BUFFER_PERIODIC_GHOST) kind[i] = 3;
        else if (t.w != 1) kind[i] = 2;
        else kind[i] = 1;
    }
    L.n_fluid = (int)fl.size(); L.n_wall = (int)wl.size(); L.n_fs = (int)fs.size();
    SPH_TRY(upload_vec(c, L.fluid_rows, fl)); SPH_TRY(upload_vec(c, L.wall_rows, wl)); SPH_TRY(upload_vec(c, L.fs_rows, fs));
    c.n_pins = 0;
    c.n_comp = 0;
    if (c.prm.ppe_pin) {
        SPH_TRY(null_components(c, kind, nmr, nmflags, aux, G.ty));
    } else {
        SPH_CUDA_TRY(cudaMemcpyAsync(c.row_kind, kind.data(), sizeof(int) * n, cudaMemcpyHostToDevice, c.stream));
        SPH_CUDA_TRY(cudaStreamSynchronize(c.stream));
    }
    {   // stored entries of the rows the pressure operator visits (fluid rows)
        std::vector<int> cnt(n), kd(n);
        SPH_CUDA_TRY(cudaMemcpyAsync(cnt.data(), c.ncnt, sizeof(int) * n, cudaMemcpyDeviceToHost, c.stream));
        SPH_CUDA_TRY(cudaMemcpyAsync(kd.data(), c.row_kind, sizeof(int) * n, cudaMemcpyDeviceToHost, c.stream));
        SPH_CUDA_TRY(cudaStreamSynchronize(c.stream));
        long long s = 0;
        for (int i = 0; i < n; ++i)
            if (kd[i] == 1) s += cnt[i];
        c.nnz_op = s;
    }
    c.cg_valid = false;   // the coarse preconditioner follows the row kinds
    return SPH_OK;
}

// ---------------------------------------------------------------------------
// NNPS driver
// ---------------------------------------------------------------------------
template <class Real>
int nnps_build(Ctx<Real> &c) {
    const int n = c.n, NC = c.num_cells;
    cudaStream_t st = c.stream;
    // scratch: h_ref as float, dummy flags / ranks
    float *href = nullptr;
    int *dflag = nullptr, *drank = nullptr, *big = nullptr, *nbig = nullptr, *err = nullptr;
    void *scratch = nullptr;
    SPH_TRY(c.alloc(href, n)); SPH_TRY(c.alloc(dflag, n)); SPH_TRY(c.alloc(drank, n));
    SPH_TRY(c.alloc(big, NC + 1)); SPH_TRY(c.alloc(nbig, 2)); SPH_TRY(c.alloc(err, 1));
    char *scr = nullptr;
    SPH_TRY(c.alloc(scr, sizeof(double) * 4 * (size_t)n));
    scratch = scr;

    k_href_to_float<Real><<<grid_for(n, 256), 256, 0, st>>>(c.h_ref, href, n);
    SPH_CUDA_TRY(cudaMemsetAsync(c.cell_fill, 0, sizeof(int) * ((size_t)NC + 2), st));
    SPH_CUDA_TRY(cudaMemsetAsync(nbig, 0, sizeof(int) * 2, st));
    SPH_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int), st));
    k_hash<<<grid_for(n, 256), 256, 0, st>>>(c.dp, c.pf, c.ty, href, c.ncell, c.key, c.cell_fill, dflag, n);
    c.launches += 2;
    SPH_CUDA_TRY(cudaGetLastError());
    SPH_TRY(exclusive_scan<int>(c.cell_fill, c.cell_start, (long long)NC + 1, c.scan_tmp, st, c.launches));
    // cell_start[NC] = start of the dummy key; cell_start[NC+1] = n
    SPH_CUDA_TRY(cudaMemcpyAsync(c.cell_start + NC + 1, &n, sizeof(int), cudaMemcpyHostToDevice, st));
    SPH_TRY(exclusive_scan<int>(dflag, drank, n, c.scan_tmp, st, c.launches));
    SPH_CUDA_TRY(cudaMemsetAsync(c.cell_fill, 0, sizeof(int) * ((size_t)NC + 2), st));
    k_scatter<<<grid_for(n, 256), 256, 0, st>>>(c.key, c.cell_start, c.cell_fill, drank, c.perm, NC, n);
    k_sort_small<<<grid_for(NC, 256), 256, 0, st>>>(c.cell_start, c.perm, big, nbig, NC);
    k_sort_big<<<kSortBigGrid, 256, 0, st>>>(c.cell_start, c.perm, big, nbig, err);
    k_sorted_keys<<<grid_for(n, 256), 256, 0, st>>>(c.key, c.perm, c.g_idx, n);
    c.launches += 4;
    SPH_CUDA_TRY(cudaGetLastError());
    int herr = 0;
    SPH_CUDA_TRY(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    SPH_CUDA_TRY(cudaStreamSynchronize(st));
    if (herr) { set_error("nnps: a cell holds more than 4096 particles"); return SPH_ERR_UNSUPPORTED; }

    // reorder every per-particle array (KERNEL_reorder, functions_NNPS.cuh:840-843)
    SPH_TRY(regather(c, c.pf, scratch));
    if ((void *)c.pr != (void *)c.pf) SPH_TRY(regather(c, c.pr, scratch));
    SPH_TRY(regather(c, c.mr, scratch)); SPH_TRY(regather(c, c.ty, scratch)); SPH_TRY(regather(c, c.jc, scratch));
    SPH_TRY(regather(c, c.ncell, scratch));
    SPH_TRY(regather(c, c.vol, scratch)); SPH_TRY(regather(c, c.m_ref, scratch)); SPH_TRY(regather(c, c.h_ref, scratch));
    SPH_TRY(regather(c, c.eli, scratch)); SPH_TRY(regather(c, c.pres0, scratch)); SPH_TRY(regather(c, c.source, scratch));
    VarSet<Real> &A = c.A;
    SPH_TRY(regather(c, A.u, scratch)); SPH_TRY(regather(c, A.p, scratch)); SPH_TRY(regather(c, A.temp, scratch));
    SPH_TRY(regather(c, A.flt, scratch)); SPH_TRY(regather(c, A.kt, scratch)); SPH_TRY(regather(c, A.et, scratch));
    SPH_TRY(regather(c, A.fb, scratch)); SPH_TRY(regather(c, A.fm, scratch)); SPH_TRY(regather(c, A.fl, scratch));
    SPH_TRY(regather(c, A.concn, scratch)); SPH_TRY(regather(c, A.enth, scratch));
    SPH_TRY(regather(c, c.rho_ref_A, scratch));
    SPH_TRY(regather(c, c.apr_family, scratch)); SPH_TRY(regather(c, c.apr_target, scratch));

    // neighbour lists: count, slice widths, offsets, fill
    k_list<false><<<grid_for(32LL * n, 128), 128, 0, st>>>(c.dp, c.pf, c.ty, c.ncell, c.cell_start, c.ncnt, nullptr,
                                                           nullptr, nullptr, nullptr, nullptr, n);
    const int nslices = (n + 31) / 32;
    long long *w = (long long *)scratch;
    k_slice_width<<<grid_for(nslices, 256), 256, 0, st>>>(c.ncnt, w, n, nslices);
    c.launches += 2;
    SPH_CUDA_TRY(cudaGetLastError());
    long long *ltmp = (long long *)((char *)scratch + sizeof(long long) * ((size_t)nslices + 64));
    SPH_TRY(exclusive_scan<long long>(w, c.slice_off, nslices + 1, ltmp, st, c.launches));
    long long total = 0;
    SPH_CUDA_TRY(cudaMemcpyAsync(&total, c.slice_off + nslices, sizeof(long long), cudaMemcpyDeviceToHost, st));
    SPH_CUDA_TRY(cudaStreamSynchronize(st));
    c.nnz_padded = total;
    if (c.nbr && c.nbr_cap < total) { c.release(c.nbr); c.release(c.nbr16); }
    const bool want16 = c.prm.ppe_wide_index == 0;
    if (!want16) c.release(c.nbr16);
    if (!c.nbr) { SPH_TRY(c.alloc(c.nbr, (size_t)std::max(total, 1LL))); c.nbr_cap = std::max(total, 1LL); }
    if (want16 && !c.nbr16) SPH_TRY(c.alloc(c.nbr16, (size_t)c.nbr_cap));
    if (want16 && c.row_cell_cap < n) {
        c.release(c.row_cell);
        SPH_TRY(c.alloc(c.row_cell, (size_t)std::max(n, 1)));
        c.row_cell_cap = std::max(n, 1);
    }
    SPH_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int), st));
    k_list<true><<<grid_for(32LL * n, 128), 128, 0, st>>>(c.dp, c.pf, c.ty, c.ncell, c.cell_start, c.ncnt,
                                                          c.slice_off, c.nbr, want16 ? c.nbr16 : nullptr, c.row_cell,
                                                          err, n);
    ++c.launches;
    SPH_CUDA_TRY(cudaGetLastError());
    {
        std::vector<int> hc(n);
        int flag16 = 0;
        SPH_CUDA_TRY(cudaMemcpyAsync(hc.data(), c.ncnt, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
        SPH_CUDA_TRY(cudaMemcpyAsync(&flag16, err, sizeof(int), cudaMemcpyDeviceToHost, st));
        SPH_CUDA_TRY(cudaStreamSynchronize(st));
        c.list16 = want16 && flag16 == 0;
        if (!c.list16) {   // codes that cannot be used: their memory goes back
            c.release(c.nbr16);
            c.release(c.row_cell);
            c.row_cell_cap = 0;
        }
        long long s = 0;
        for (int v : hc) s += v;
        c.nnz = s;
    }
    SPH_TRY(build_side_lists(c));
    c.release(href); c.release(dflag); c.release(drank); c.release(big); c.release(nbig); c.release(err);
    c.release(scr);
    c.built = true;
    c.gc_valid = false;
    c.prep_valid = false;
    c.pforce_valid = false;
    c.coef_valid = false;
    return SPH_OK;
}

template <class Real>
int nnps_export(Ctx<Real> &c, int32_t *g_idx, int32_t *p_idx, int32_t *g_str, int32_t *g_end) {
    if (!c.built) { set_error("nnps_export: NNPS has not run"); return SPH_ERR_STATE; }
    const int n = c.n, NC = c.num_cells;
    if (g_idx) SPH_CUDA_TRY(cudaMemcpyAsync(g_idx, c.g_idx, sizeof(int) * n, cudaMemcpyDeviceToHost, c.stream));
    if (p_idx) SPH_CUDA_TRY(cudaMemcpyAsync(p_idx, c.perm, sizeof(int) * n, cudaMemcpyDeviceToHost, c.stream));
    if (g_str || g_end) {
        std::vector<int> cs((size_t)NC + 2);
        SPH_CUDA_TRY(cudaMemcpyAsync(cs.data(), c.cell_start, sizeof(int) * ((size_t)NC + 2), cudaMemcpyDeviceToHost, c.stream));
        SPH_CUDA_TRY(cudaStreamSynchronize(c.stream));
        for (int k = 0; k <= NC; ++k) {
            const bool occ = cs[k + 1] > cs[k];
            if (g_str) g_str[k] = occ ? cs[k] : -1;
            if (g_end) g_end[k] = occ ? cs[k + 1] : 0;
        }
    }
    SPH_CUDA_TRY(cudaStreamSynchronize(c.stream));
    return SPH_OK;
}

template <class Real>
int neighbors_export(Ctx<Real> &c, int64_t *off, int32_t *list, int64_t *nnz) {
    if (!c.built) { set_error("neighbors_export: NNPS has not run"); return SPH_ERR_STATE; }
    const int n = c.n, nslices = (n + 31) / 32;
    std::vector<int> cnt(n);
    std::vector<long long> so((size_t)nslices + 1);
    SPH_CUDA_TRY(cudaMemcpyAsync(cnt.data(), c.ncnt, sizeof(int) * n, cudaMemcpyDeviceToHost, c.stream));
    SPH_CUDA_TRY(cudaMemcpyAsync(so.data(), c.slice_off, sizeof(long long) * (nslices + 1), cudaMemcpyDeviceToHost, c.stream));
    SPH_CUDA_TRY(cudaStreamSynchronize(c.stream));
    int64_t acc = 0;
    for (int i = 0; i < n; ++i) { if (off) off[i] = acc; acc += cnt[i]; }
    if (off) off[n] = acc;
    if (nnz) *nnz = acc;
    if (list) {
        std::vector<int> sell((size_t)std::max(c.nnz_padded, 1LL));
        SPH_CUDA_TRY(cudaMemcpyAsync(sell.data(), c.nbr, sizeof(int) * (size_t)c.nnz_padded, cudaMemcpyDeviceToHost, c.stream));
        SPH_CUDA_TRY(cudaStreamSynchronize(c.stream));
        int64_t o = 0;
        for (int i = 0; i < n; ++i) {
            const long long b = so[i >> 5] + (i & 31);
            for (int k = 0; k < cnt[i]; ++k) list[o++] = sell[(size_t)(b + 32LL * k)];
        }
    }
    return SPH_OK;
}

#define INST(R)                                                                                          \
    template int ctx_allocate<R>(Ctx<R> &);                                                              \
    template int ctx_upload<R>(Ctx<R> &, const sph_part1 *, const sph_part2 *, int);                      \
    template int ctx_upload_state<R>(Ctx<R> &, const sph_part1 *, int);                                  \
    template int ctx_download<R>(Ctx<R> &, sph_part1 *, sph_part2 *, sph_part3 *);                        \
    template int nnps_build<R>(Ctx<R> &);                                                                \
    template int nnps_export<R>(Ctx<R> &, int32_t *, int32_t *, int32_t *, int32_t *);                    \
    template int neighbors_export<R>(Ctx<R> &, int64_t *, int32_t *, int64_t *);                          \
    template int build_side_lists<R>(Ctx<R> &);
INST(float)
INST(double)
#undef INST

}  // namespace sph

// ---------------------------------------------------------------------------
// Cell sort without device allocation (sph_nnps_sort_noalloc)
//
// For callers that cannot call cudaMalloc: a host code that hands all of its
// device memory to its own pool or arena, or a solver that must not allocate
// once its time loop has started.  The hash, counting sort and cell ranges
// of nnps_build run here on a scratch area that is a file-scope device
// array, sized for at most SPH_NOALLOC_MAX_PARTICLES particles and
// SPH_NOALLOC_MAX_CELLS cells (about 9.5 MB, held by every GPU that loads
// this library until the process exits).
// ---------------------------------------------------------------------------
namespace sph {
namespace noalloc {

constexpr long long kMaxN = SPH_NOALLOC_MAX_PARTICLES;
constexpr long long kMaxC = SPH_NOALLOC_MAX_CELLS;    // num_cells + 2 entries of the cell arrays
constexpr long long kScanTmp = 1024;                  // >= scan_tmp_size(max(kMaxN, kMaxC))
// int slots: key, dummy flag, dummy rank (n each); cell counts, cell starts,
// long-cell list (kMaxC each); long-cell count, overflow flag; scan scratch
constexpr long long kKey = 0, kDflag = kMaxN, kDrank = 2 * kMaxN, kCnt = 3 * kMaxN, kStart = kCnt + kMaxC,
                    kBig = kStart + kMaxC, kNbig = kBig + kMaxC, kErr = kNbig + 2, kTmp = kErr + 2,
                    kTotal = kTmp + kScanTmp;

static __device__ __align__(256) int g_scratch[kTotal];

constexpr int kMaxDevices = 64;
static std::mutex g_mtx;
static int *g_ptr[kMaxDevices] = {};

// device address of g_scratch on the current device, looked up once per device
static int scratch_address(int **out) {
    int dev = 0;
    SPH_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) { set_error("sph_nnps_sort_noalloc: device ordinal out of range"); return SPH_ERR_BAD_ARG; }
    std::lock_guard<std::mutex> lock(g_mtx);
    if (!g_ptr[dev]) {
        int *p = nullptr;
        SPH_CUDA_TRY(cudaGetSymbolAddress((void **)&p, g_scratch));
        g_ptr[dev] = p;
    }
    *out = g_ptr[dev];
    return SPH_OK;
}

// KERNEL_index_particle_to_cell (functions_NNPS.cuh:879-907) on separate
// coordinate arrays, with the cell histogram of the counting sort
__global__ void k_hash_xyz(DevParams P, const float *x, const float *y, const float *z, const int *i_type, int *key,
                           int *cell_cnt, int *dflag, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (i_type[i] == 3) {
        key[i] = P.num_cells;
        dflag[i] = 1;
        return;
    }
    dflag[i] = 0;
    const int ic = bin_axis(x[i], P.xmin, P.xmax, P.NI);
    const int jc = bin_axis(y[i], P.ymin, P.ymax, P.NJ);
    const int kc = bin_axis(z[i], P.zmin, P.zmax, P.NK);
    const int k = ic + P.NI * jc + P.NI * P.NJ * kc;
    key[i] = k;
    atomicAdd(&cell_cnt[k], 1);
}

__global__ void k_set_tail(int *cell_start, int num_cells, int n) { cell_start[num_cells + 1] = n; }

// g_str / g_end of KERNEL_reorder (functions_NNPS.cuh:813-844): -1 / 0 for empty cells
__global__ void k_cell_ranges(const int *cs, int *g_str, int *g_end, int ncells1) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ncells1) return;
    const int s = cs[k], e = cs[k + 1];
    const bool occ = e > s;
    g_str[k] = occ ? s : -1;
    g_end[k] = occ ? e : 0;
}

}  // namespace noalloc
}  // namespace sph

extern "C" int sph_nnps_sort_noalloc(const sph_params *params, const float *d_x, const float *d_y, const float *d_z,
                                     const int32_t *d_i_type, int32_t n, int32_t *d_g_idx, int32_t *d_p_idx,
                                     int32_t *d_g_str, int32_t *d_g_end, void *stream) {
    using namespace sph;
    using namespace sph::noalloc;
    if (!params || n < 0) { set_error("sph_nnps_sort_noalloc: null params or negative n"); return SPH_ERR_BAD_ARG; }
    const int NC = params->vii[SPH_VII_NUM_CELLS];
    if (NC < 1) { set_error("sph_nnps_sort_noalloc: params hold no cell grid (run sph_domain_setup)"); return SPH_ERR_BAD_ARG; }
    if ((long long)n > kMaxN) {
        set_error("sph_nnps_sort_noalloc: more particles than SPH_NOALLOC_MAX_PARTICLES");
        return SPH_ERR_BAD_ARG;
    }
    if ((long long)NC + 2 > kMaxC) {
        set_error("sph_nnps_sort_noalloc: num_cells + 2 exceeds SPH_NOALLOC_MAX_CELLS");
        return SPH_ERR_BAD_ARG;
    }
    if (!d_g_str || !d_g_end || (n > 0 && (!d_x || !d_y || !d_z || !d_i_type || !d_g_idx || !d_p_idx))) {
        set_error("sph_nnps_sort_noalloc: null array");
        return SPH_ERR_BAD_ARG;
    }
    int *S = nullptr;
    SPH_TRY(scratch_address(&S));
    cudaStream_t st = (cudaStream_t)stream;
    const DevParams P = make_dev_params(*params);
    int *key = S + kKey, *dflag = S + kDflag, *drank = S + kDrank, *cnt = S + kCnt, *cs = S + kStart;
    int *big = S + kBig, *nbig = S + kNbig, *err = S + kErr, *tmp = S + kTmp;
    long long launches = 0;
    // the scratch keeps the previous call's contents: clear the counters
    SPH_CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof(int) * ((size_t)NC + 2), st));
    SPH_CUDA_TRY(cudaMemsetAsync(nbig, 0, sizeof(int) * 4, st));   // nbig, its pad, err, its pad
    if (n > 0) {
        k_hash_xyz<<<grid_for(n, 256), 256, 0, st>>>(P, d_x, d_y, d_z, d_i_type, key, cnt, dflag, n);
        SPH_CUDA_TRY(cudaGetLastError());
    }
    SPH_TRY(exclusive_scan<int>(cnt, cs, (long long)NC + 1, tmp, st, launches));
    k_set_tail<<<1, 1, 0, st>>>(cs, NC, n);
    SPH_CUDA_TRY(cudaGetLastError());
    if (n > 0) {
        SPH_TRY(exclusive_scan<int>(dflag, drank, n, tmp, st, launches));
        SPH_CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof(int) * ((size_t)NC + 2), st));
        k_scatter<<<grid_for(n, 256), 256, 0, st>>>(key, cs, cnt, drank, d_p_idx, NC, n);
        k_sort_small<<<grid_for(NC, 256), 256, 0, st>>>(cs, d_p_idx, big, nbig, NC);
        k_sort_big<<<kSortBigGrid, 256, 0, st>>>(cs, d_p_idx, big, nbig, err);
        k_sorted_keys<<<grid_for(n, 256), 256, 0, st>>>(key, d_p_idx, d_g_idx, n);
        SPH_CUDA_TRY(cudaGetLastError());
    }
    k_cell_ranges<<<grid_for(NC + 1, 256), 256, 0, st>>>(cs, d_g_str, d_g_end, NC + 1);
    SPH_CUDA_TRY(cudaGetLastError());
    int flags[3] = {0, 0, 0};   // nbig, pad, err
    SPH_CUDA_TRY(cudaMemcpyAsync(flags, nbig, sizeof(int) * 3, cudaMemcpyDeviceToHost, st));
    SPH_CUDA_TRY(cudaStreamSynchronize(st));
    if (flags[2]) {
        set_error("sph_nnps_sort_noalloc: a cell holds more than 4096 particles");
        return SPH_ERR_UNSUPPORTED;
    }
    return SPH_OK;
}
