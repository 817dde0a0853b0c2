// Host build of the reference's own device code (test infrastructure, never shipped).
//
// This translation unit compiles the reference's CUDA headers, as they lie in
// the reference tree, as plain host C++: every `__global__` kernel becomes a
// host function that is run once per (blockIdx, threadIdx) pair by the
// launcher below, with blockDim.x = 128 as in ISPH_Calc.cuh:12.  Nothing of the
// reference is copied here; the include path points at the reference tree
// (see oracle/Makefile).  Only the tests, bench.py's reference arm and
// __graft_entry__.smoke may load the resulting library.
//
// Semantics that differ from a CUDA run and why:
//   * CUB DeviceRadixSort::SortPairs (ISPH_Calc.cuh:33) is stable and is given
//     p_idx_in[i] = i (functions_NNPS.cuh:886,899); std::stable_sort on the key
//     gives the identical permutation.
//   * KERNEL_reorder (functions_NNPS.cuh:813-844) uses a block-shared window and
//     one __syncthreads; each thread only reads window slots written by itself
//     or by a lower-numbered thread of its block, so running the threads of a
//     block in ascending order reproduces the barrier semantics exactly.
//   * KERNEL_PPE3D (functions_PPE.cuh:2-175) writes P1[i].pres in place while
//     other threads read P1[j].pres, and KERNEL_Neumann_boundary3D reads its
//     ghost partner's pressure the same way.  ref_step(..., snapshot=1) runs
//     each thread of those launches against the pre-launch records (Jacobi
//     semantics); snapshot=0 runs them in place in thread order (what a
//     serial CPU run of the kernels gives).
//   * Floating point: host IEEE float/double, compiled with -ffp-contract=off,
//     so no fused multiply-add is formed (nvcc forms them by default).

#include <cmath>
#include <math.h>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cstdint>
#include <cfloat>
#include <algorithm>
#include <vector>
#include <numeric>
#include <string>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

// ---- CUDA keyword and built-in emulation -----------------------------------
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

// ---- globals that SOPHIA_gpu.cu:41-95 defines for the included headers -----
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
#include "functions_PROP.cuh"
#include "functions_PREP.cuh"
#include "functions_IBM.cuh"
#include "functions_INTERACTION.cuh"
#include "functions_TIME.cuh"
#include "functions_PPE.cuh"
#include "functions_BC.cuh"
#include "functions_MOST.cuh"
#include "functions_TIME_ISPH.cuh"
#include "functions_OUTPUT.cuh"
#include "functions_ENERGY.cuh"

// ---- launcher ---------------------------------------------------------------
// Runs `body` for every thread of a <<<ceil(n/128),128>>> launch.  Blocks run in
// parallel under OpenMP when `parallel` is set; threads of one block run in
// ascending order on one host thread.
template <class F>
static void launch(int n, bool parallel, F body) {
    const int tpb = 128;
    const int nb = (n - 1) / tpb + 1;
    if (n <= 0) return;
#pragma omp parallel for schedule(dynamic, 16) if (parallel)
    for (int b = 0; b < nb; ++b) {
        blockIdx.x = b;
        blockDim.x = tpb;
        for (int t = 0; t < tpb; ++t) {
            threadIdx.x = t;
            body();
        }
    }
}

// Runs a launch whose threads write only their own record P1[i], with every
// thread reading the pre-launch state (race-free semantics of an in-place
// kernel such as KERNEL_PPE3D or the ghost read of KERNEL_Neumann_boundary3D).
template <class F>
static void launch_snapshot(int n, part1 *P1, F body) {
    if (n <= 0) return;
    std::vector<part1> snap(P1, P1 + n), out(n);
    const int tpb = 128;
    const int nb = (n - 1) / tpb + 1;
    for (int b = 0; b < nb; ++b) {
        blockIdx.x = b;
        blockDim.x = tpb;
        for (int t = 0; t < tpb; ++t) {
            threadIdx.x = t;
            const int i = b * tpb + t;
            if (i >= n) continue;
            body();
            out[i] = P1[i];
            P1[i] = snap[i];
        }
    }
    std::memcpy(P1, out.data(), sizeof(part1) * n);
}

static int g_threads_parallel = 1;
static int g_outlet_bc = 0;       // 0 donothing, 1 extrapolation, 2 inout
static int g_inlet_recycling = 0;
static int g_stop_after = 1000;   // debugging: phases of ref_step to run

extern "C" {

int ref_sizeof_part1(void) { return (int)sizeof(part1); }
int ref_sizeof_part2(void) { return (int)sizeof(part2); }
int ref_sizeof_part3(void) { return (int)sizeof(part3); }

void ref_set_parallel(int on) { g_threads_parallel = on; }

// Selects the pass run at the outlet-buffer call sites (ISPH_Calc.cuh:151,
// 208: the shipped KERNEL_donothing_buffer3D or one of the commented-out
// alternatives) and the commented-out KERNEL_Recycling3D (ISPH_Calc.cuh:215);
// with reset_probe, clears the u* of the recycling probe (a device global
// that lives across steps there).
void ref_set_boundary_variant(int outlet_bc, int inlet_recycling, int reset_probe) {
    g_outlet_bc = outlet_bc;
    g_inlet_recycling = inlet_recycling;
    if (reset_probe) us_update = 0.f;
}
void ref_set_stop_after(int k) { g_stop_after = k; }

int ref_num_threads(void) {
#ifdef _OPENMP
    return g_threads_parallel ? omp_get_max_threads() : 1;
#else
    return 1;
#endif
}

// Loads the solver parameter tables (k_vii / k_vif, function_init.cuh:84-163),
// as cudaMemcpyToSymbol does at ISPH_Calc.cuh:366-367.
void ref_set_params(const int *ivals, const float *fvals) {
    std::memcpy(vii, ivals, sizeof(int_t) * vii_size);
    std::memcpy(vif, fvals, sizeof(Real) * vif_size);
    std::memcpy(k_vii, ivals, sizeof(int_t) * vii_size);
    std::memcpy(k_vif, fvals, sizeof(Real) * vif_size);
}

// Host-side domain set-up of ISPH.cuh:83-97 and clc_num_cells
// (functions_NNPS.cuh:533-546): min/max (function_init.cuh:678-708), dcell,
// NI/NJ/NK and num_cells.  Writes the results into the parameter tables.
void ref_domain_setup(part1 *P1, int n) {
    num_part = n;
    Real cell_reduction_factor = 1.1;
    search_incr_factor = 1.0;
    search_kappa = kappa;
    find_minmax(vii, vif, P1);
    Real h0 = P1[0].h_ref;
    dcell = cell_reduction_factor * kappa * h0 / float(ncell_init);
    NI = (int)((x_max - x_min) / dcell) + 1;
    NJ = (int)((y_max - y_min) / dcell) + 1;
    NK = (int)((z_max - z_min) / dcell) + 1;
    num_cells = clc_num_cells();
    std::memcpy(k_vii, vii, sizeof(int_t) * vii_size);
    std::memcpy(k_vif, vif, sizeof(Real) * vif_size);
}

void ref_get_params(int *ivals, float *fvals) {
    std::memcpy(ivals, k_vii, sizeof(int_t) * vii_size);
    std::memcpy(fvals, k_vif, sizeof(Real) * vif_size);
}

// NNPS of ISPH_Calc.cuh:20-45: set_ncell, hash, stable sort, reorder.
// g_str/g_end must hold num_cells+1 entries (KERNEL_reorder writes the dummy
// key num_cells, one past the reference's own allocation).
void ref_nnps(part1 *P1, part2 *P2, part1 *SP1, part2 *SP2, int *g_idx, int *p_idx,
              int *g_str, int *g_end) {
    const int n = k_num_part2;
    launch(n, g_threads_parallel, [&] { KERNEL_set_ncell(P1); });
    std::vector<int> g_idx_in(n), p_idx_in(n);
    for (int c = 0; c <= k_num_cells; ++c) g_str[c] = (int)cu_memset;
    launch(n, g_threads_parallel, [&] { KERNEL_index_particle_to_cell(g_idx_in.data(), p_idx_in.data(), P1); });
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return g_idx_in[a] < g_idx_in[b]; });
    for (int i = 0; i < n; ++i) {
        g_idx[i] = g_idx_in[order[i]];
        p_idx[i] = p_idx_in[order[i]];
    }
    launch(n, false, [&] { KERNEL_reorder(g_idx, p_idx, g_str, g_end, P1, P2, SP1, SP2); });
}

// One ISPH step, SOPHIA_single_ISPH (ISPH_Calc.cuh:4-214) without output.
// Arrays: P1/SP1/P2/SP2/P3 of num_part2 records; g_str/g_end of num_cells+1.
// `tcount` is the reference's step counter `count`, `ttime` its `time`.
// ppe_snapshot selects the race-free (Jacobi) execution of KERNEL_PPE3D.
void ref_step(part1 *P1, part1 *SP1, part2 *P2, part2 *SP2, part3 *P3, int *g_idx,
              int *p_idx, int *g_str, int *g_end, int tcount, float ttime, int ppe_snapshot) {
    const int n = k_num_part2;
    const bool par = g_threads_parallel != 0;
    k_vii[27] = tcount;  // count
    k_vif[3] = ttime;    // time
    vii[27] = tcount;
    vif[3] = ttime;
    const Real tdt = k_vif[2];
    // KERNEL_Neumann_boundary3D reads the pressure of its ghost-node partner
    // (functions_BC.cuh:358-364), which may be another Neumann particle being
    // rewritten by the same launch: run it with snapshot semantics when asked.
    // the extrapolation and inout passes read records the same launch
    // rewrites (outlet and side buffers): snapshot semantics
    auto outlet = [&](part1 *A, part2 *B) {
        if (g_outlet_bc == 1)
            launch_snapshot(n, A, [&] { KERNEL_open_boundary_extrapolation_buffer3D(g_str, g_end, A, B, P3); });
        else if (g_outlet_bc == 2)
            launch_snapshot(n, A, [&] { KERNEL_inout_boundary3D(g_str, g_end, A, B, P3); });
        else
            launch(n, par, [&] { KERNEL_donothing_buffer3D(g_str, g_end, A, B, P3); });
    };
    auto neumann = [&](part1 *A, part2 *B) {
        if (ppe_snapshot)
            launch_snapshot(n, A, [&] { KERNEL_Neumann_boundary3D(g_str, g_end, A, B, P3); });
        else
            launch(n, false, [&] { KERNEL_Neumann_boundary3D(g_str, g_end, A, B, P3); });
    };

    launch(n, par, [&] { KERNEL_set_ncell(P1); });
    if (tcount == 0) {
        ref_nnps(P1, P2, SP1, SP2, g_idx, p_idx, g_str, g_end);
        std::memset(P3, 0, sizeof(part3) * n);
        std::memcpy(P1, SP1, sizeof(part1) * n);
    } else {
        std::memcpy(SP1, P1, sizeof(part1) * n);
        std::memcpy(SP2, P2, sizeof(part2) * n);
        std::memset(P3, 0, sizeof(part3) * n);
    }
#define PHASE(k) if (g_stop_after < (k)) return
    PHASE(0);
    if (tcount == 0) launch(n, par, [&] { KERNEL_clc_IB_normal_vector3D(g_str, g_end, P1, P3); });
    PHASE(1);
    launch(n, par, [&] { KERNEL_clc_gradient_correction_3D(g_str, g_end, SP1, P3); });
    PHASE(2);
    launch(n, par, [&] { KERNEL_clc_prep3D(g_str, g_end, SP1, SP2, P3, tcount, tdt); });
    PHASE(3);
    if (k_noslip_bc == 1) launch(n, par, [&] { KERNEL_boundary3D(g_str, g_end, SP1); });
    PHASE(4);
    launch(n, false, [&] { KERNEL_MOST_boundary3D(g_str, g_end, SP1, P3, tcount, tdt); });
    PHASE(5);
    if (tcount == 0) neumann(SP1, SP2);
    PHASE(6);
    launch(n, par, [&] { KERNEL_advection_force3D(1, g_str, g_end, SP1, SP2, P3, tcount); });
    PHASE(7);
    if (k_time_type == Pre_Cor)
        launch(n, par, [&] { KERNEL_clc_projection(tcount, tdt, ttime, SP1, SP2, P3); });
    PHASE(8);
    launch(n, par, [&] { KERNEL_periodic_boundary3D(g_str, g_end, SP1, SP2, P3); });
    PHASE(9);
    launch(n, par, [&] { KERNEL_freeslip_boundary3D(g_str, g_end, SP1, SP2, P3); });
    PHASE(10);
    if (ppe_snapshot)
        launch_snapshot(n, SP1, [&] { KERNEL_PPE3D(tdt, g_str, g_end, SP1, SP2, P3); });
    else
        launch(n, false, [&] { KERNEL_PPE3D(tdt, g_str, g_end, SP1, SP2, P3); });
    PHASE(11);
    neumann(SP1, SP2);
    PHASE(12);
    outlet(SP1, SP2);
    PHASE(13);
    launch(n, par, [&] { KERNEL_pressureforce3D(1, g_str, g_end, SP1, SP2, P3); });
    PHASE(14);
    launch(n, par, [&] { IBM_force_interpolation3D(tdt, g_str, g_end, SP1, SP2, P3); });
    PHASE(15);
    launch(n, par, [&] { IBM_spreading_interpolation3D(g_str, g_end, SP1, SP2, P3); });
    PHASE(16);
    launch(n, par, [&] { KERNEL_time_update_projection(tdt, SP1, P1, SP2, P2, P3, tcount); });
    PHASE(17);
    launch(n, par, [&] { IBM_corrector(k_vif[20], ttime, SP1, P1, SP2, P3); });
    PHASE(18);
    neumann(P1, SP2);
    PHASE(19);
    outlet(P1, SP2);
    PHASE(20);
    launch(n, par, [&] { KERNEL_periodic_boundary3D(g_str, g_end, P1, SP2, P3); });
    PHASE(21);
    launch(n, par, [&] { KERNEL_freeslip_boundary3D(g_str, g_end, P1, SP2, P3); });
    PHASE(22);
    if (g_inlet_recycling == 1) launch(n, par, [&] { KERNEL_Recycling3D(g_str, g_end, P1, SP2, P3); });
#undef PHASE
}

// read_solv_input (function_init.cuh:166-463) on the given tables (in/out);
// copies the plot labels out and returns their count
int ref_read_solv(const char *path, int *vii_io, float *vif_io, char *labels_out) {
    std::memcpy(vii, vii_io, sizeof(int_t) * vii_size);
    std::memcpy(vif, vif_io, sizeof(Real) * vif_size);
    num_plot_data = 0;
    read_solv_input(vii, vif, path);
    std::memcpy(vii_io, vii, sizeof(int_t) * vii_size);
    std::memcpy(vif_io, vif, sizeof(Real) * vif_size);
    for (int k = 0; k < num_plot_data && k < 20; ++k) std::memcpy(labels_out + 20 * k, plot_data[k], 20);
    return num_plot_data;
}

// c_initial_inner_outer_particle_single (functions_NNPS.cuh:196-373) over n
// records in place, with the open-boundary switch and dimension given; the
// terrain switch of the host shadow table is set to the one case that
// prints nothing per record
int ref_initial_records(part1 *P, int n, int open, int dimension) {
    vii[5] = open;
    vii[1] = dimension;
    vii[23] = n;
    k_vii[46] = 3;
    std::vector<part1> D(n > 0 ? n : 1);
    c_initial_inner_outer_particle_single(P, D.data(), 0);
    std::memcpy(P, D.data(), sizeof(part1) * n);
    return 0;
}

// read_input (function_init.cuh:550-676) into P1 (capacity records, i_type
// cleared first); returns the number of records read
int ref_read_input(part1 *P1, int capacity, const char *path) {
    for (int i = 0; i < capacity; ++i) P1[i].i_type = 0;
    read_input(P1, (char *)path);
    int n = 0;
    while (n < capacity && P1[n].i_type == 1) ++n;
    return n;
}

// save_vtk_bin_single_flag (functions_OUTPUT.cuh:121-616) for n records and
// the space-separated labels; writes ./<its hard-wired directory>/fluid_<step>stp.vtk
// relative to the current directory
void ref_save_vtk(part1 *P1, part2 *P2, part3 *P3, int n, int step, const char *labels) {
    num_part2 = n;
    count = step;
    num_plot_data = 0;
    char tmp[512];
    strncpy(tmp, labels, sizeof tmp - 1);
    tmp[sizeof tmp - 1] = 0;
    for (char *t = strtok(tmp, " "); t && num_plot_data < 20; t = strtok(nullptr, " ")) {
        strncpy(plot_data[num_plot_data], t, 19);
        plot_data[num_plot_data][19] = 0;
        ++num_plot_data;
    }
    save_vtk_bin_single_flag(P1, P2, P3);
}

// read_table (function_init.cuh:724-905) on the given file, then the upload
// of ISPH_Calc.cuh:370-377 into the k_Tab_* arrays the device code reads.
// cols receives T, h, k, cp, mu (table_size entries each, as stored in Real).
// The arrays are cleared first, so entries past the file's stay 0.
void ref_read_table(const char *path, double *cols, int *index, int *size) {
    Real *tabs[5] = {host_Tab_T, host_Tab_h, host_Tab_k, host_Tab_cp, host_Tab_vis};
    for (Real *t : tabs) std::fill(t, t + table_size, Real(0));
    std::fill(host_table_index, host_table_index + 10, 0);
    std::fill(host_table_size, host_table_size + 10, 0);
    read_table(path);
    for (int c = 0; c < 5; ++c)
        for (int k = 0; k < table_size; ++k) cols[c * table_size + k] = (double)tabs[c][k];
    for (int k = 0; k < 10; ++k) { index[k] = host_table_index[k]; size[k] = host_table_size[k]; }
    std::copy(host_Tab_T, host_Tab_T + table_size, k_Tab_T);
    std::copy(host_Tab_h, host_Tab_h + table_size, k_Tab_h);
    std::copy(host_Tab_k, host_Tab_k + table_size, k_Tab_k);
    std::copy(host_Tab_cp, host_Tab_cp + table_size, k_Tab_cp);
    std::copy(host_Tab_vis, host_Tab_vis + table_size, k_Tab_vis);
    std::copy(host_table_index, host_table_index + 10, k_table_index);
    std::copy(host_table_size, host_table_size + 10, k_table_size);
}

// KERNEL_clc_TemptoEnthalpy (functions_ENERGY.cuh:3-12), the launch that
// ISPH_Calc.cuh:480-482 keeps commented out before the time loop, and
// KERNEL_clc_EnthalpytoTemp (:15-25), over the first k_num_part2 records
void ref_temp_to_enthalpy(part1 *P1, part2 *P2, int n) {
    launch(n, false, [&] { KERNEL_clc_TemptoEnthalpy(P1, P2); });
}
void ref_enthalpy_to_temp(part1 *P1, int n) {
    launch(n, false, [&] { KERNEL_clc_EnthalpytoTemp(P1); });
}

}  // extern "C"
