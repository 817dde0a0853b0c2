// Device-side context of one ISPH simulation: SoA particle state in HBM,
// NNPS structures, neighbour lists and PPE workspace.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "common.cuh"

namespace sph {

// Time-varying per-particle fields of one particle-array copy (the
// reference's dev_P1 or dev_SP1, class_Cuda_Particle_Array.cuh:11-67).
template <class Real>
struct VarSet {
    typedef typename V4<Real>::type R4;
    R4 *u = nullptr;        // ux, uy, uz, vis_t
    Real *p = nullptr;      // pres
    Real *temp = nullptr;
    Real *flt = nullptr;    // flt_s
    Real *kt = nullptr;     // k_turb
    Real *et = nullptr;     // e_turb
    R4 *fb = nullptr;       // fbx, fby, fbz, concentration
    R4 *fm = nullptr;       // fmx, fmy, hmz, -
    R4 *fl = nullptr;       // float1, float2, float3, -
    Real *concn = nullptr;
    Real *enth = nullptr;
};

// Precomputed, time-invariant lists of the boundary passes.
struct SideLists {
    // IBM marker interpolation (markers i, fluid j) and spreading (fluid i,
    // markers j): CSR over the rows in `rows`.
    int n_mk = 0, n_sp = 0;
    int *mk_rows = nullptr, *mk_off = nullptr, *mk_nbr = nullptr;
    int *sp_rows = nullptr, *sp_off = nullptr, *sp_nbr = nullptr;
    int *sp_zero = nullptr; int n_sp_zero = 0;   // fluid rows with no marker in range
    // Neumann rows (p_type != 1): CSR of fluid j (p_type 1, buffer 0) in range
    int n_nm = 0;
    long long nm_nnz = 0;
    int *nm_rows = nullptr, *nm_off = nullptr, *nm_nbr = nullptr;
    int *nm_ghost = nullptr;     // flags: 1 mirror (inlet) row, 2 the pass writes p = 0,
                                 // 4 no fluid in range at all (operator anchor)
    // partners of periodic (buffer 3/4), outlet (buffer 2) and periodic-box
    // ghost (buffer 7) particles
    int n_per = 0, n_out = 0, n_gh = 0;
    int *per_rows = nullptr, *per_partner = nullptr;
    int *out_rows = nullptr, *out_partner = nullptr;
    int *gh_rows = nullptr, *gh_partner = nullptr;
    // dormant open-boundary variants of the reference (outlet_bc 1 / 2,
    // inlet_recycling): extrapolation rows (outlet, off the MOST layer) with
    // the fluid around their mirror node; inout rows, the side buffers first
    // (partner in io_aux) and then the outlet rows (CSR of the interior fluid
    // around their interface point); recycling rows (inlet)
    int n_xo = 0;
    int *xo_rows = nullptr, *xo_off = nullptr, *xo_nbr = nullptr;
    int n_ios = 0, n_io = 0;
    int *io_rows = nullptr, *io_aux = nullptr, *io_off = nullptr, *io_nbr = nullptr;
    int n_rc = 0;
    int *rc_rows = nullptr;
    // MOST wall-layer particles and their ghost-node targets
    int n_most = 0;
    int *most_rows = nullptr, *most_off = nullptr, *most_tgt = nullptr;
    // row lists of the passes
    int n_fluid = 0, n_wall = 0, n_fs = 0, n_pf = 0;
    int *fluid_rows = nullptr;   // i_type<=2, 0<p_type<1000 (prep/PPE rows)
    int *wall_rows = nullptr;    // no-slip walls (p_type 0, i_type<=2)
    int *fs_rows = nullptr;      // free-slip (p_type -1)
};

struct Timer {
    cudaEvent_t a = nullptr, b = nullptr;
};

template <class Real>
struct Ctx {
    typedef typename V4<Real>::type R4;
    typedef typename V2<Real>::type R2;

    sph_params prm;
    DevParams dp;
    int device = 0;
    cudaStream_t stream = nullptr;
    int n = 0;
    int num_cells = 0;
    int pair_block = 128;         // threads per block of the per-step pair passes (32, 64 or 128)
    int count = 0;
    float time = 0.f;
    bool uploaded = false;
    bool built = false;
    bool gc_valid = false;
    long long launches = 0;
    float phase_ms[4] = {0, 0, 0, 0};
    cudaEvent_t ev[8] = {};

    // device allocations owned by the context (held through a pointer so Ctx
    // stays trivially copyable and bulk kernels can take it by value)
    std::vector<void *> *allocs = nullptr;

    // ---- constant per particle (sorted order after NNPS) ----
    float4 *pf = nullptr;   // FP32 x, y, z, h (NNPS precision)
    R4 *pr = nullptr;       // Real x, y, z, h
    R2 *mr = nullptr;       // m, rho
    int4 *ty = nullptr;     // i_type, buffer_type, MOST_buffer, p_type
    int *jc = nullptr;      // neighbour-class bits
    int *ncell = nullptr;
    Real *vol = nullptr, *m_ref = nullptr, *h_ref = nullptr, *eli = nullptr, *pres0 = nullptr;
    int *source = nullptr;
    // ---- time-varying ----
    VarSet<Real> A, S;
    Real *rho_ref_A = nullptr, *rho_ref_S = nullptr, *SR = nullptr;
    R4 *u0 = nullptr;       // SP2: ux0, uy0, uz0, (x0 written flag)
    R4 *ft = nullptr;       // P3: ftotalx, ftotaly, ftotalz, ftotal
    R4 *fp = nullptr;       // P3: fpx, fpy, fpz
    Real *dtemp = nullptr;
    Real *dconcn = nullptr; // P3: dconcn (concn_solve)
    Real *temp0 = nullptr;  // SP2: temp0 (con_solve), concn0 (concn_solve)
    Real *concn0 = nullptr;
    Real *enth0 = nullptr;  // SP2: enthalpy0 (con_solve with enthalpy_eqn)
    Real *denth = nullptr;  // P3: denthalpy
    R4 *nrm = nullptr;      // P3: nx, ny, nz
    // property tables of htoT (k_Tab_h then k_Tab_T, SPH_TABLE_SIZE each),
    // allocated with the context so that captured steps keep the pointer
    Real *tab = nullptr;
    bool tab_set = false;
    int tab_index[SPH_TABLE_SLOTS] = {}, tab_size[SPH_TABLE_SLOTS] = {};
    unsigned ptype_slots = 0;     // bit t: a record the projection reaches has |p_type| = t
    bool ptype_wide = false;      // such a record has |p_type| >= SPH_TABLE_SLOTS
    unsigned *ptype_dev = nullptr;   // the same two words, found on the device for device records
    float *us_update = nullptr;   // u* of the recycling probe, kept across steps
    Real *g6 = nullptr;     // inv_cm: 6 arrays of n (xx, yy, zz, xy, yz, zx)
    // ---- NNPS ----
    int *key = nullptr, *perm = nullptr, *cell_start = nullptr, *cell_fill = nullptr;
    int *g_idx = nullptr;   // sorted keys (reference g_idx)
    int *scan_tmp = nullptr;
    // ---- SELL-32 canonical neighbour list ----
    int *ncnt = nullptr;          // list length per particle
    long long *slice_off = nullptr;
    int *nbr = nullptr;
    long long nnz = 0, nnz_padded = 0;
    long long nnz_op = 0;         // entries of the fluid rows, the ones the pressure operator reads
    long long nbr_cap = 0;
    // the same list as 16-bit codes for the pressure operator (plane_cell in
    // common.cuh): valid when every row searches at most two cells around
    // its own and every offset fits in 13 bits
    uint16_t *nbr16 = nullptr;
    int *row_cell = nullptr;      // cell index of the row's first x-run cell (dy = dz = 0)
    int row_cell_cap = 0;
    bool list16 = false;
    SideLists L;
    // ---- PPE ----
    Real *diag = nullptr;         // A_i of fluid rows
    int *row_kind = nullptr;      // 0 identity, 1 fluid, 2 Neumann, 3 outlet copy, 4 pinned
    int *row_aux = nullptr;       // partner of kind-3 rows (outlet copy, periodic ghost), -1 otherwise
    int n_pins = 0;               // rows pinned to p = 0 (one per unanchored component)
    int n_comp = 0;               // components carrying the rank-one mean-pressure term
    int *comp_id = nullptr;       // component of each fluid row (-1: none)
    double *comp_inv = nullptr;   // 1 / fluid rows of each component
    double *nm_w = nullptr;       // Neumann row weights (CSR aligned with nm_nbr)
    double *nm_gw = nullptr;      // mirror-row gradient weights
    double *nm_ow = nullptr;      // weights of the Neumann rows in the converged operator
    float *nm_owf = nullptr;      // the same in FP32 (mixed form)
    float *coef = nullptr;        // cached c_ij (SELL layout), mixed form
    double *coef_d = nullptr;     // cached c_ij, FP64 form
    bool coef_valid = false;
    __half *coef_h = nullptr;     // c_ij / (row's max |c_ij|) in FP16 (ppe_coef_half), mixed form
    float *coef_rs = nullptr;     // the row scales
    bool coef_h_valid = false;
    Real *ppe_gb = nullptr;       // cached rhs pair vectors g_ij (3 x SELL arrays)
    Real *vis_stage = nullptr;    // staging of the LES viscosity in the prep pass
    // time-invariant parts of the prep pass (particles never move): per row
    // the filter sum and the LES length sum, per pair the strain weights
    // V_j G_i grad W_ij (three SELL arrays); rebuilt with the lists or g6
    Real *prep_row = nullptr, *prep_w = nullptr;
    long long prep_cap = 0;
    bool prep_valid = false;
    // time-invariant part of the pressure force per pair: g_ij (3) and rho_j
    typename V4<Real>::type *pforce_w = nullptr;
    long long pforce_cap = 0;
    bool pforce_valid = false;
    double *ib_boxes = nullptr;   // obstacle boxes for the IB normals (NULL: params.ib_box)
    int n_ib_boxes = 0;
    // Krylov workspace
    Real *kv[10] = {};            // r, rh, p, v, s, t, ph, sh, dinv, b
    double *kd[10] = {};          // FP64 Krylov vectors of the mixed form's fallback
    double *gm_h = nullptr;       // GMRES Hessenberg column / coefficients (device)
    void *gm_ws_r = nullptr;      // GMRES workspace in the context precision
    void *gm_ws_d = nullptr;      // GMRES workspace with FP64 vectors (FP32 context)
    void *idr_ws_r = nullptr;     // IDR(s) workspace in the context precision
    void *idr_ws_f = nullptr;     // IDR(s) workspace with FP32 vectors (inner solves of the refinement)
    void *kgraph = nullptr;       // CUDA graph of the mixed BiCGSTAB's iterations between host checks
    void *devloop = nullptr;      // CUDA graph of a whole device-controlled solve (ppe_refinement = 4)
    void *stepgraph = nullptr;    // CUDA graph of a whole step around that solve (capi.cu)
    bool capturing = false;       // the phases are being captured into the step graph
    long long graph_steps = 0;    // steps run as a replay of it
    StepClock *clk = nullptr;     // step counter and time on the device
    bool clk_synced = false;      // clk holds count / time
    unsigned long long mem_gen = 0;     // bumped by every allocation and release
    unsigned long long param_gen = 0;   // bumped by every change of the parameters
    bool ppe_pending = false;     // a device-controlled solve whose statistics the host has not read
    bool defer_stats = false;     // inside sph_step: leave those statistics until the last step
    bool kgraph_off = false;      // capture failed once: launch the kernels one by one
    double *xd = nullptr, *rd = nullptr, *bd = nullptr;   // FP64 solution / residual / rhs
    float *xf = nullptr, *bf = nullptr;                   // FP32 correction / residual
    sph_ppe_stats last_ppe = {};
    double init_relres = -1;      // residual of the start vector of the current solve
    // two-level preconditioner (coarse.cu), rebuilt with the lists
    bool cg_valid = false;
    int cg_block = 0, cg_m = 0;   // aggregate edge in cells, aggregates in use
    int cg_max = 0;               // ppe_coarse_max the coarse space was built with
    int *cg_agg = nullptr;        // aggregate of each row, -1 for identity / pinned rows
    int *cg_off = nullptr, *cg_rows = nullptr;   // rows of each aggregate, ascending
    float *cg_invf = nullptr;     // E^-1, m x m, FP32 copy the solve reads
    double *cg_s = nullptr, *cg_y = nullptr;     // restricted residual, coarse correction
    int cg_np = 0;                // pieces of the restriction (at most kCoarsePiece rows each)
    int *cg_piece = nullptr;      // per piece: aggregate, first and end entry of cg_rows
    int *cg_pfirst = nullptr;     // first piece of each aggregate (m + 1)
    double *cg_part = nullptr;    // partial sum of each piece
    unsigned int *cg_cnt = nullptr;   // pieces summed per aggregate (back to 0 after each restriction)
    // live operator timing (sph_profile)
    bool prof = false;
    cudaEvent_t *prof_ev = nullptr;   // 512 events, created on first use
    int prof_pending = 0;
    cudaEvent_t *cap_ev = nullptr;    // while a Krylov graph is captured: its timing events
    int cap_n = 0, cap_max = 0;       // timed applications captured, room for
    long long prof_launches = 0;
    double prof_ms = 0;
    double *red = nullptr;        // block partial sums
    double *red_host = nullptr;   // pinned
    int red_blocks = 0;
    double *scal = nullptr;       // device scalars
    // learned warm start (learned.cu)
    int ml_every = 0;             // sample every k-th fluid row of each converged solve (0: off)
    bool ml_ready = false, ml_init = false;
    float *ml_w = nullptr, *ml_m = nullptr, *ml_v = nullptr, *ml_grad = nullptr;   // FP32 parameters, Adam moments
    __nv_bfloat16 *ml_w1b = nullptr, *ml_w2b = nullptr;   // BF16 B operands of the tensor-core inference
    double *ml_sc = nullptr, *ml_red = nullptr;           // feature scales, reduction partials
    unsigned int *ml_cnt = nullptr;
    __nv_bfloat16 *ml_X = nullptr;                        // features of the step (n x 32)
    float *ml_y = nullptr, *ml_pold = nullptr, *ml_rr = nullptr, *ml_dd = nullptr;
    float *ml_pprev = nullptr;                            // p_old of the previous step
    bool ml_have_prev = false;
    double *ml_zd = nullptr, *ml_wd = nullptr;            // predicted change and its image
    double *ml_W = nullptr, *ml_MW = nullptr, *ml_r0 = nullptr;   // subspace start: columns, images, r0
    double *ml_subred = nullptr;                          // its reduction partials and small system
    unsigned int *ml_subcnt = nullptr;
    __nv_bfloat16 *ml_SX = nullptr;                       // collected samples
    float *ml_St = nullptr;
    long long ml_cap = 0, ml_count = 0;
    int *ml_fluid = nullptr;
    int ml_nfluid = 0, ml_phase = 0;
    float *ml_part = nullptr, *ml_lpart = nullptr;        // per-block gradient / loss partials
    int ml_part_cap = 0;
    // APR (apr.cu): family (the reference's blood_index) and target level
    // (its M_num) per record, sorted with the records; allocated at the
    // first pass
    int *apr_family = nullptr;
    float *apr_target = nullptr;
    int apr_last_merged = 0;
    R4 *sc_u = nullptr;           // pass scratch
    Real *sc_p = nullptr, *sc_t = nullptr;

    // staging for AoS upload/download
    void *aos = nullptr;
    size_t aos_bytes = 0;

    template <class T>
    int alloc(T *&ptr, size_t count) {
        if (capturing) {   // no allocation inside a captured step: the capture fails and the step runs launch by launch
            set_error("allocation while a step is captured");
            return SPH_ERR_STATE;
        }
        void *p = nullptr;
        size_t bytes = sizeof(T) * (count ? count : 1);
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) {
            set_cuda_error(e, "cudaMalloc", __FILE__, __LINE__);
            return e == cudaErrorMemoryAllocation ? SPH_ERR_OUT_OF_MEMORY : SPH_ERR_CUDA;
        }
        allocs->push_back(p);
        ptr = (T *)p;
        ++mem_gen;
        return SPH_OK;
    }
    template <class T>
    void release(T *&ptr) {
        if (!ptr || capturing) return;   // (see alloc)
        ++mem_gen;
        for (size_t k = 0; k < allocs->size(); ++k)
            if ((*allocs)[k] == (void *)ptr) {
                cudaFree(ptr);
                (*allocs)[k] = allocs->back();
                allocs->pop_back();
                break;
            }
        ptr = nullptr;
    }
    void free_all() {
        if (!allocs) return;
        for (void *p : *allocs) cudaFree(p);
        allocs->clear();
    }
};

// ---- phases (nnps.cu, passes.cu, ppe.cu) ------------------------------------
template <class Real> int ctx_allocate(Ctx<Real> &c);
template <class Real> int ctx_upload(Ctx<Real> &c, const sph_part1 *P1, const sph_part2 *P2, int n);
template <class Real> int ctx_upload_state(Ctx<Real> &c, const sph_part1 *P1, int n);
template <class Real> int ctx_download(Ctx<Real> &c, sph_part1 *P1, sph_part2 *P2, sph_part3 *P3);
template <class Real> int nnps_build(Ctx<Real> &c);
template <class Real> int nnps_export(Ctx<Real> &c, int32_t *g_idx, int32_t *p_idx, int32_t *g_str, int32_t *g_end);
template <class Real> int neighbors_export(Ctx<Real> &c, int64_t *off, int32_t *list, int64_t *nnz);
template <class Real> int phase_interaction(Ctx<Real> &c);
template <class Real> int phase_ppe(Ctx<Real> &c, sph_ppe_stats *st);
template <class Real> int coarse_build(Ctx<Real> &c);
template <class Real> int apr_pass(Ctx<Real> &c, int *n_split, int *n_wanted, int *n_merged);
template <class Real> int apr_state(Ctx<Real> &c, int32_t *family, float *target);
template <class Real> int ml_prepare(Ctx<Real> &c, const Real *b, bool features);
template <class Real> int ml_extrapolate(Ctx<Real> &c, double *x);
template <class Real> int ml_warm_start(Ctx<Real> &c, const double *b, double *x, double *tmp);
template <class Real> int ml_subspace_start(Ctx<Real> &c, const double *b, double *x, double *tmp, bool with_net,
                                            bool galerkin);
template <class Real> int ml_finish_step(Ctx<Real> &c);
template <class Real> void ppe_apply_fp64(Ctx<Real> &c, const double *x, double *y);
template <class Real> int ml_collect(Ctx<Real> &c, const double *xnew);
template <class Real> int ml_grad(Ctx<Real> &c, long long first, int rows, float *loss, float *grad);
template <class Real> int ml_train(Ctx<Real> &c, int epochs, int batch, float lr, unsigned long long seed, float *loss);
template <class Real> int ml_set_weights(Ctx<Real> &c, const float *w);
template <class Real> int ml_get_weights(Ctx<Real> &c, float *w);
template <class Real> int ml_samples(Ctx<Real> &c, long long first, long long rows, uint16_t *X, float *t, long long *count);
template <class Real> int ml_predict_samples(Ctx<Real> &c, long long first, int rows, float *y);
template <class Real, class V> void coarse_apply(Ctx<Real> &c, const V *r, V *z, const V *w = nullptr);
// the restriction and coarse solve of coarse_apply (c.cg_y = E^-1 Z^T (r - w));
// the caller adds Z c.cg_y
template <class Real, class V> void coarse_restrict_solve(Ctx<Real> &c, const V *r, const V *w);
template <class Real> int phase_time_update(Ctx<Real> &c);

// an event record on the context's stream; while a whole step is captured it
// is an event-record node of the step's graph, so the phase times stay live
template <class Real>
inline cudaError_t record_event(const Ctx<Real> &c, cudaEvent_t e) {
    return c.capturing ? cudaEventRecordWithFlags(e, c.stream, cudaEventRecordExternal) : cudaEventRecord(e, c.stream);
}
template <class Real> int finish_step(Ctx<Real> &c);
// enthalpy = enthalpy0 = Ttoh(temp) (to_h = 1) or temp = htoT(enthalpy)
// (to_h = 0) for every record but i_type 3, on the current records
template <class Real> int energy_convert(Ctx<Real> &c, int to_h);
template <class Real> int dev_solve_stats(Ctx<Real> &c, sph_ppe_stats *S, int *worst);
template <class Real> int dev_reset_worst(Ctx<Real> &c);
template <class Real> bool solve_under_device_control(const Ctx<Real> &c);
template <class Real> int ctx_diagnostics(Ctx<Real> &c, float *umax, float *drho, float *fmax);
template <class Real> int gradient_correction(Ctx<Real> &c);
template <class Real> int neumann_pass(Ctx<Real> &c, VarSet<Real> &V);
template <class Real> int outlet_pass(Ctx<Real> &c, VarSet<Real> &V);
template <class Real> int periodic_pass(Ctx<Real> &c, VarSet<Real> &V);
template <class Real> int freeslip_pass(Ctx<Real> &c, VarSet<Real> &V);
template <class Real> int build_side_lists(Ctx<Real> &c);
template <class Real> void release_solver_ws(Ctx<Real> &c);
template <class Real> int operator_stats(Ctx<Real> &c, int64_t *launches, double *total_ms, double *bytes, int reset);
template <class Real> int operator_bytes(Ctx<Real> &c, double *stored, double *index_rule);

// launch helper: grid for n threads
inline dim3 grid_for(long long n, int block) { return dim3((unsigned)((n + block - 1) / block)); }

}  // namespace sph
