// Host build of the reference's APR kernels (test infrastructure, never shipped).
//
// The reference does not compile its APR (SOPHIA_gpu.cu:113-114 keep
// functions_APR.cuh and functions_APR_etc.cuh commented out), and the three
// per-particle fields those kernels read -- apr_cond, M_num, blood_index --
// are commented out of part1 (class_Cuda_Particle_Array.cuh:38-43).
// oracle/Makefile therefore compiles this file against a temporary copy of
// the reference headers in which only those field declarations are
// uncommented; of functions_APR_etc.cuh only the numbering function
// Cell_index is taken, since its other host functions drive CUDA and CUB.
// The kernels themselves are the reference's, compiled where they lie.
//
// The entry points below take records in the shipped 152-byte layout
// (sph_part1) plus the APR fields as separate arrays, copy them into the
// augmented struct, run the reference's kernels one thread at a time in
// launch order, and copy the results back:
//   refapr_condition: KERNEL_APR_condition3D_cell (functions_APR.cuh:270-403)
//                     over every cell, then Cell_index (functions_APR_etc.cuh:5-20)
//   refapr_split:     KERNEL_cell_APR_3D (functions_APR.cuh:406-652)

#include <cmath>
#include <math.h>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cstdint>
#include <cfloat>
#include <algorithm>
#include <vector>
#include <string>
#include <time.h>

#define __global__
#define __device__
#define __host__
#define __constant__
#define __forceinline__ inline
#define __shared__ thread_local
static inline void __syncthreads() {}
struct shim_dim3 { unsigned x, y, z; };
static thread_local shim_dim3 threadIdx = {0, 0, 0};
static thread_local shim_dim3 blockIdx = {0, 0, 0};
static thread_local shim_dim3 blockDim = {128, 1, 1};
typedef int cudaStream_t;
struct dim3 { unsigned x = 1, y = 1, z = 1; };
static inline int cudaDeviceSynchronize() { return 0; }

#include "Variable_Type.cuh"
#include "Parameters.cuh"
#include "class_Cuda_Particle_Array.cuh"

int_t vii[vii_size];
Real vif[vif_size];
int_t k_vii[vii_size];
Real k_vif[vif_size];
Real k_Tab_T[table_size], k_Tab_h[table_size], k_Tab_k[table_size];
Real k_Tab_cp[table_size], k_Tab_vis[table_size];
int k_table_index[10], k_table_size[10];
part1 *HP1;
part1 *DHP1[Max_GPU];
part1 *send_P1[Max_GPU], *send_rSP1[Max_GPU], *send_lSP1[Max_GPU], *recv_P1[Max_GPU];
p2p_part3 *send_P3[Max_GPU], *send_rSP3[Max_GPU], *send_lSP3[Max_GPU], *recv_P3[Max_GPU];
Real host_Tab_T[table_size], host_Tab_h[table_size], host_Tab_k[table_size];
Real host_Tab_cp[table_size], host_Tab_vis[table_size];
int host_table_index[10], host_table_size[10];
cudaStream_t str1[Max_GPU], str2[Max_GPU];
Real space;
int Nsx = 0, Nsy = 0, Nsz = 0, buffer_size = 0;
int num_buffer[1];
int num_plot_data;
char plot_data[20][20];
float us_update;
thread_local int sharedHash[129];

#include "function_init.cuh"
#include "functions_NNPS.cuh"
#include "functions_KNL.cuh"

#include "functions_APR.cuh"
#include "functions_APR_etc.cuh"

namespace {

// the shipped record layout (include/sph_isph.h, sph_part1)
struct rec152 {
    int32_t i_type, buffer_type, MOST_buffer, p_type;
    float x, y, z, ux, uy, uz, m, h, temp, pres, pres0, rho, flt_s, enthalpy, concn, concentration;
    float k_turb, e_turb, eli, vol, m_ref, h_ref, vis_t, fbx, fby, fbz, fmx, fmy, hmz, float1, float2, float3;
    int32_t ncell, source;
};
static_assert(sizeof(rec152) == 152, "sph_part1 layout");

void to_ref(const rec152 &s, part1 &d) {
    std::memset(&d, 0, sizeof d);
    d.i_type = s.i_type; d.buffer_type = s.buffer_type; d.MOST_buffer = s.MOST_buffer; d.p_type = s.p_type;
    d.x = s.x; d.y = s.y; d.z = s.z; d.ux = s.ux; d.uy = s.uy; d.uz = s.uz; d.m = s.m; d.h = s.h;
    d.temp = s.temp; d.pres = s.pres; d.pres0 = s.pres0; d.rho = s.rho; d.flt_s = s.flt_s;
    d.enthalpy = s.enthalpy; d.concn = s.concn; d.concentration = s.concentration;
    d.k_turb = s.k_turb; d.e_turb = s.e_turb; d.eli = s.eli; d.vol = s.vol; d.m_ref = s.m_ref; d.h_ref = s.h_ref;
    d.vis_t = s.vis_t; d.fbx = s.fbx; d.fby = s.fby; d.fbz = s.fbz; d.fmx = s.fmx; d.fmy = s.fmy; d.hmz = s.hmz;
    d.float1 = s.float1; d.float2 = s.float2; d.float3 = s.float3; d.ncell = s.ncell; d.source = s.source;
}

void from_ref(const part1 &s, rec152 &d) {
    d.i_type = s.i_type; d.buffer_type = s.buffer_type; d.MOST_buffer = s.MOST_buffer; d.p_type = s.p_type;
    d.x = s.x; d.y = s.y; d.z = s.z; d.ux = s.ux; d.uy = s.uy; d.uz = s.uz; d.m = s.m; d.h = s.h;
    d.temp = s.temp; d.pres = s.pres; d.pres0 = s.pres0; d.rho = s.rho; d.flt_s = s.flt_s;
    d.enthalpy = s.enthalpy; d.concn = s.concn; d.concentration = s.concentration;
    d.k_turb = s.k_turb; d.e_turb = s.e_turb; d.eli = s.eli; d.vol = s.vol; d.m_ref = s.m_ref; d.h_ref = s.h_ref;
    d.vis_t = s.vis_t; d.fbx = s.fbx; d.fby = s.fby; d.fbz = s.fbz; d.fmx = s.fmx; d.fmy = s.fmy; d.hmz = s.hmz;
    d.float1 = s.float1; d.float2 = s.float2; d.float3 = s.float3; d.ncell = s.ncell; d.source = s.source;
}

std::vector<part1> g_P;      // augmented records between the two calls
std::vector<int> g_cell;     // apr_cell after Cell_index

template <class F>
void launch(int n, F body) {
    const int tpb = 128;
    if (n <= 0) return;
    const int nb = (n - 1) / tpb + 1;
    for (int b = 0; b < nb; ++b) {
        blockIdx.x = b;
        blockDim.x = tpb;
        for (int t = 0; t < tpb; ++t) {
            threadIdx.x = t;
            body();
        }
    }
}

}  // namespace

extern "C" {

int refapr_sizeof_part1(void) { return (int)sizeof(part1); }

// k_vii / k_vif as cudaMemcpyToSymbol sets them (ISPH_Calc.cuh:366-367)
void refapr_set_params(const int *ivals, const float *fvals) {
    std::memcpy(vii, ivals, sizeof(int_t) * vii_size);
    std::memcpy(vif, fvals, sizeof(Real) * vif_size);
    std::memcpy(k_vii, ivals, sizeof(int_t) * vii_size);
    std::memcpy(k_vif, fvals, sizeof(Real) * vif_size);
}

// KERNEL_APR_condition3D_cell over every cell of the sorted records P (n),
// with M_num and blood_index per record and apr_cell cleared first, then
// Cell_index.  Writes apr_cond per record and the numbered apr_cell per cell
// (num_cells entries).
void refapr_condition(const void *P, int n, const float *M_num, const int *blood, const int *g_str,
                      const int *g_end, int *apr_cond_out, int *apr_cell_out) {
    const rec152 *R = (const rec152 *)P;
    g_P.assign(n, part1());
    for (int i = 0; i < n; ++i) {
        to_ref(R[i], g_P[i]);
        g_P[i].M_num = M_num[i];
        g_P[i].blood_index = blood[i];
        g_P[i].apr_cond = 0;
    }
    const int NC = k_num_cells;
    g_cell.assign(NC + 1, 0);
    launch(NC, [&] {
        KERNEL_APR_condition3D_cell(g_P.data(), g_cell.data(), (int_t *)g_str, (int_t *)g_end, 0);
    });
    Cell_index(g_cell.data());
    for (int i = 0; i < n; ++i) apr_cond_out[i] = g_P[i].apr_cond;
    std::memcpy(apr_cell_out, g_cell.data(), sizeof(int) * NC);
}

// KERNEL_cell_APR_3D over every cell on the records of the last
// refapr_condition call, with *num_buffer = num_buffer; writes the records
// back (P, n) with M_num and blood_index per record.
void refapr_split(void *P, int n, int num_buffer_value, const int *g_str, const int *g_end, float *M_num_out,
                  int *blood_out) {
    num_buffer[0] = num_buffer_value;
    std::vector<part2> P2(n);
    std::memset(P2.data(), 0, sizeof(part2) * n);
    const int NC = k_num_cells;
    launch(NC, [&] {
        KERNEL_cell_APR_3D(g_P.data(), P2.data(), (int_t *)g_str, (int_t *)g_end, g_cell.data(), 0);
    });
    rec152 *R = (rec152 *)P;
    for (int i = 0; i < n; ++i) {
        from_ref(g_P[i], R[i]);
        M_num_out[i] = g_P[i].M_num;
        blood_out[i] = g_P[i].blood_index;
    }
}

}  // extern "C"
