// C ABI of the B200 ISPH step (include/sph_isph.h).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <type_traits>

#include "ctx.cuh"

namespace sph {

static thread_local std::string g_last_error;

void set_cuda_error(cudaError_t e, const char *what, const char *file, int line) {
    char buf[512];
    snprintf(buf, sizeof(buf), "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
    g_last_error = buf;
}
void set_error(const char *msg) { g_last_error = msg; }

DevParams make_dev_params(const sph_params &p) {
    DevParams d;
    memset(&d, 0, sizeof(d));
    d.n = p.vii[SPH_VII_NUM_PART2];
    d.NI = p.vii[SPH_VII_NI]; d.NJ = p.vii[SPH_VII_NJ]; d.NK = p.vii[SPH_VII_NK];
    d.num_cells = p.vii[SPH_VII_NUM_CELLS];
    d.kernel_type = p.vii[SPH_VII_KERNEL_TYPE];
    d.time_type = p.vii[SPH_VII_TIME_TYPE];
    d.freq_filt = p.vii[SPH_VII_FREQ_FILT] > 0 ? p.vii[SPH_VII_FREQ_FILT] : 1;
    d.fp_solve = p.vii[SPH_VII_FP_SOLVE];
    d.fv_solve = p.vii[SPH_VII_FV_SOLVE];
    d.fg_solve = p.vii[SPH_VII_FG_SOLVE];
    d.kgc_solve = p.vii[SPH_VII_KGC_SOLVE];
    d.con_solve = p.vii[SPH_VII_CON_SOLVE];
    d.boussinesq = p.vii[SPH_VII_BOUSSINESQ];
    d.concn_solve = p.vii[SPH_VII_CONCN_SOLVE];
    d.outlet_bc = p.outlet_bc;
    d.ppe_pair_h = p.ppe_pair_h;
    d.pforce_form = p.pressure_force_form;
    d.enthalpy_eqn = p.enthalpy_eqn;
    d.prop_table = p.vii[SPH_VII_PROP_TABLE] == 1;   // the table slots come from the context
    d.inlet_recycling = p.inlet_recycling;
    d.rp_x = p.recycle_probe_x; d.rp_y = p.recycle_probe_y;
    for (int a = 0; a < 6; ++a) d.periodic_box[a] = p.periodic_box[a];
    d.turb = p.vii[SPH_VII_TURBULENCE];
    d.noslip = p.vii[SPH_VII_NOSLIP_BC];
    d.kappa = p.vif[SPH_VIF_KAPPA];
    d.skappa = p.vif[SPH_VIF_SEARCH_KAPPA];
    d.dcell = p.vif[SPH_VIF_DCELL];
    d.xmin = p.vif[SPH_VIF_X_MIN]; d.xmax = p.vif[SPH_VIF_X_MAX];
    d.ymin = p.vif[SPH_VIF_Y_MIN]; d.ymax = p.vif[SPH_VIF_Y_MAX];
    d.zmin = p.vif[SPH_VIF_Z_MIN]; d.zmax = p.vif[SPH_VIF_Z_MAX];
    d.dt = p.vif[SPH_VIF_DT];
    d.u_limit = p.vif[SPH_VIF_U_LIMIT];
    d.dt_structure = p.vif[SPH_VIF_DT_STRUCTURE];
    d.cs_sgs = p.cs_sgs; d.l2 = p.l2; d.l3 = p.l3; d.l_left = p.l_left; d.l_right = p.l_right;
    d.outlet_probe_dx = p.outlet_probe_dx; d.partner_tol = p.partner_tol; d.ghost_tol = p.ghost_tol;
    for (int k = 0; k < 6; ++k) d.ib_box[k] = p.ib_box[k];
    d.ib_face_tol = p.ib_face_tol; d.most_z0 = p.most_z0; d.most_z0h = p.most_z0h;
    d.most_ghost_dz = p.most_ghost_dz; d.rho_air = p.rho_air; d.ibm_target_coeff = p.ibm_target_coeff;
    d.visc_fluid = p.visc_fluid; d.visc_wall = p.visc_wall; d.visc_marker = p.visc_marker;
    d.av_alpha = p.av_alpha; d.av_beta = p.av_beta; d.av_c0 = p.av_c0;
    d.pressure_length = p.pressure_length; d.ibm_length = p.ibm_length; d.neumann_coeff = p.neumann_coeff;
    d.t_ini = p.t_ini; d.t_con = p.t_con; d.t_start = p.t_start; d.t_con_t = p.t_con_t;
    d.boundary_velocity = p.boundary_velocity;
    d.n_profile = p.n_profile;
    for (int k = 0; k < SPH_MAX_PROFILE; ++k) { d.profile_z[k] = p.profile_z[k]; d.profile_u[k] = p.profile_u[k]; }
    return d;
}

static int check_params(const sph_params &p) {
    if (p.vii[SPH_VII_DIM] != 3) { set_error("only dim = 3 is supported (the reference step is 3-D)"); return SPH_ERR_UNSUPPORTED; }
    if (p.vii[SPH_VII_NUM_PART2] <= 0) { set_error("num_part2 must be positive (call sph_domain_setup)"); return SPH_ERR_BAD_ARG; }
    if (p.vii[SPH_VII_NI] <= 0 || p.vii[SPH_VII_NJ] <= 0 || p.vii[SPH_VII_NK] <= 0) { set_error("cell grid not set up"); return SPH_ERR_BAD_ARG; }
    if ((long long)p.vii[SPH_VII_NI] * p.vii[SPH_VII_NJ] * p.vii[SPH_VII_NK] + 1 != p.vii[SPH_VII_NUM_CELLS]) {
        set_error("num_cells != NI*NJ*NK+1"); return SPH_ERR_BAD_ARG;
    }
    if (p.pressure_length != 1.0) { set_error("pressure_length other than 1 is not supported"); return SPH_ERR_UNSUPPORTED; }
    if (p.n_profile < 2 || p.n_profile > SPH_MAX_PROFILE) { set_error("n_profile must be in [2, 32]"); return SPH_ERR_BAD_ARG; }
    if (!(p.vif[SPH_VIF_DT] > 0)) { set_error("dt must be positive"); return SPH_ERR_BAD_ARG; }
    if (p.outlet_bc < 0 || p.outlet_bc > 2) { set_error("outlet_bc must be 0, 1 or 2"); return SPH_ERR_BAD_ARG; }
    if (p.ppe_coarse_max < 0 || p.ppe_coarse_max > 32768) {
        set_error("ppe_coarse_max must be in [0, 32768]"); return SPH_ERR_BAD_ARG;
    }
    if (p.enthalpy_eqn < 0 || p.enthalpy_eqn > 1) { set_error("enthalpy_eqn must be 0 or 1"); return SPH_ERR_BAD_ARG; }
    if (p.vii[SPH_VII_PROP_TABLE] < 0 || p.vii[SPH_VII_PROP_TABLE] > 1) {
        set_error("vii[prop_table] must be 0 (NO) or 1 (YES)");
        return SPH_ERR_BAD_ARG;
    }
    if (p.pressure_force_form < 0 || p.pressure_force_form > 1) {
        set_error("pressure_force_form must be 0 or 1"); return SPH_ERR_BAD_ARG;
    }
    return SPH_OK;
}

}  // namespace sph

using namespace sph;

struct sph_ctx {
    int prec = 0;
    Ctx<float> *f = nullptr;
    Ctx<double> *d = nullptr;
    std::vector<void *> *allocs = nullptr;
};

#define DISPATCH(ctx, expr_f, expr_d) ((ctx)->prec == SPH_PREC_FP64 ? (expr_d) : (expr_f))

// Every entry point below is declared extern "C" in sph_isph.h.

const char *sph_status_string(int status) {
    switch (status) {
        case SPH_OK: return "ok";
        case SPH_NOT_CONVERGED: return "not converged";
        case SPH_ERR_BAD_ARG: return "bad argument";
        case SPH_ERR_CUDA: return "CUDA error";
        case SPH_ERR_BREAKDOWN: return "Krylov breakdown";
        case SPH_ERR_STATE: return "call out of order";
        case SPH_ERR_NO_DEVICE: return "no CUDA device";
        case SPH_ERR_OUT_OF_MEMORY: return "out of device memory";
        case SPH_ERR_UNSUPPORTED: return "unsupported configuration";
    }
    return "unknown status";
}

const char *sph_last_error(void) { return sph::g_last_error.c_str(); }

int sph_params_init(sph_params *p) {
    if (!p) return SPH_ERR_BAD_ARG;
    memset(p, 0, sizeof(*p));
    p->vii[SPH_VII_SOLVER_TYPE] = 1;
    p->vii[SPH_VII_DIM] = 3;
    p->vii[SPH_VII_KERNEL_TYPE] = 5;   // Wendland6
    p->vii[SPH_VII_TIME_TYPE] = 1;     // Predictor_Corrector
    p->vii[SPH_VII_OPEN_BOUNDARY] = 1;
    p->vii[SPH_VII_FREQ_FILT] = 1;
    p->vii[SPH_VII_FREQ_OUTPUT] = 100;
    p->vii[SPH_VII_FP_SOLVE] = 1;
    p->vii[SPH_VII_FV_SOLVE] = 1;      // Cleary
    p->vii[SPH_VII_TURBULENCE] = 4;    // SSM
    p->vii[SPH_VII_NOSLIP_BC] = 1;
    p->vii[SPH_VII_NGPU] = 1;
    p->vif[SPH_VIF_KAPPA] = 2.0f;
    p->vif[SPH_VIF_DT] = 1e-4f;
    p->vif[SPH_VIF_TIME_END] = 1.0f;
    p->vif[SPH_VIF_U_LIMIT] = 50.0f;
    p->vif[SPH_VIF_DT_STRUCTURE] = 1e-4f;
    p->cs_sgs = 0.15;
    p->l2 = 0.028; p->l3 = 13.304; p->l_left = -0.412; p->l_right = 0.412;
    p->outlet_probe_dx = 0.008; p->partner_tol = 0.001; p->ghost_tol = 0.1;
    const double box[6] = {0.764, 0.836, -0.036, 0.036, 0.0, 0.152};
    for (int k = 0; k < 6; ++k) p->ib_box[k] = box[k];
    p->ib_face_tol = 1e-5;
    p->most_z0 = 1.0; p->most_z0h = 0.1; p->most_ghost_dz = 5.0;
    p->rho_air = 1.225; p->ibm_target_coeff = 0.2;
    p->visc_fluid = 1.8e-5; p->visc_wall = 1.0e-2; p->visc_marker = 1.0e-2;
    p->av_alpha = 0.05; p->av_beta = 0.05; p->av_c0 = 30.0;
    p->pressure_length = 1.0; p->ibm_length = 0.5; p->neumann_coeff = 2.0;
    p->t_ini = 300.0; p->t_con = 300.0; p->t_start = 0.0; p->t_con_t = 10.0;
    p->boundary_velocity = 1.0;
    // AIJ Case-H wall-model target profile (functions_IBM.cuh:289-304)
    static const double Z[30] = {0.005, 0.01, 0.02, 0.04, 0.06, 0.08, 0.1, 0.12, 0.14, 0.16, 0.165, 0.17, 0.18, 0.19, 0.21,
                                 0.23, 0.25, 0.3, 0.35, 0.4, 0.45, 0.5, 0.55, 0.6, 0.6528736, 0.7724136, 0.8390808, 0.8689656,
                                 0.88046, 0.8919544};
    static const double U[30] = {2.745, 2.935, 3.175, 3.435, 3.627, 3.824, 4.021, 4.21, 4.362, 4.491, 4.502, 4.586, 4.606, 4.712, 4.854,
                                 4.993, 5.132, 5.449, 5.782, 6.077, 6.338, 6.588, 6.693, 6.751, 6.751, 6.751, 6.751, 6.751, 6.751, 6.751};
    p->n_profile = 30;
    for (int k = 0; k < 30; ++k) { p->profile_z[k] = Z[k]; p->profile_u[k] = U[k]; }
    p->ppe_mode = SPH_PPE_MIXED_IR;
    p->ppe_max_iter = 2000;
    p->ppe_tol = 1e-6;
    p->ppe_pin = 1;
    p->ppe_inner_tol = 1e-3;
    p->recycle_probe_x = 600.0;   // functions_MOST.cuh:316
    p->recycle_probe_y = 0.0;
    return SPH_OK;
}

int sph_domain_setup(sph_params *p, const sph_part1 *P1, int num_part) {
    if (!p || !P1 || num_part <= 0) return SPH_ERR_BAD_ARG;
    // find_minmax scans records 0..num_part-2 (function_init.cuh:680-698)
    float mnx = P1[0].x, mxx = P1[0].x, mny = P1[0].y, mxy = P1[0].y, mnz = P1[0].z, mxz = P1[0].z;
    for (int i = 0; i < num_part - 1; ++i) {
        const float x = P1[i].x, y = P1[i].y, z = P1[i].z;
        if (x < mnx) mnx = x; if (x > mxx) mxx = x;
        if (y < mny) mny = y; if (y > mxy) mxy = y;
        if (z < mnz) mnz = z; if (z > mxz) mxz = z;
    }
    p->vif[SPH_VIF_X_MIN] = mnx; p->vif[SPH_VIF_X_MAX] = mxx;
    p->vif[SPH_VIF_Y_MIN] = mny; p->vif[SPH_VIF_Y_MAX] = mxy;
    p->vif[SPH_VIF_Z_MIN] = mnz; p->vif[SPH_VIF_Z_MAX] = mxz;
    const float kappa = p->vif[SPH_VIF_KAPPA];
    p->vif[SPH_VIF_SEARCH_INCR] = 1.0f;
    p->vif[SPH_VIF_SEARCH_KAPPA] = kappa;
    const float h0 = P1[0].h_ref;
    volatile float crf = 1.1f;                       // cell_reduction_factor, ISPH.cuh:82
    volatile float t1 = crf * kappa;
    volatile float t2 = t1 * h0;
    const float dcell = t2 / 2.0f;                   // ISPH.cuh:90, ncell_init = 2
    p->vif[SPH_VIF_DCELL] = dcell;
    volatile float ex = (mxx - mnx) / dcell, ey = (mxy - mny) / dcell, ez = (mxz - mnz) / dcell;
    const int NI = (int)ex + 1, NJ = (int)ey + 1, NK = (int)ez + 1;
    p->vii[SPH_VII_NI] = NI; p->vii[SPH_VII_NJ] = NJ; p->vii[SPH_VII_NK] = NK;
    const long long nc = (long long)NI * NJ * NK + 1;
    if (nc > 0x7ffffff0LL) { set_error("cell grid exceeds 2^31 cells"); return SPH_ERR_UNSUPPORTED; }
    p->vii[SPH_VII_NUM_CELLS] = (int)nc;
    p->vii[SPH_VII_NUM_PART] = num_part;
    p->vii[SPH_VII_NUM_PART2] = num_part;
    return SPH_OK;
}

// the property-table slots of the context into its device parameters
template <class Real>
static void apply_tables(Ctx<Real> &c) {
    for (int t = 0; t < SPH_TABLE_SLOTS; ++t) { c.dp.tab_index[t] = c.tab_index[t]; c.dp.tab_size[t] = c.tab_size[t]; }
}

template <class Real>
static int create_impl(const sph_params *p, int device, void *stream, Ctx<Real> **out) {
    Ctx<Real> *c = new (std::nothrow) Ctx<Real>();
    if (!c) return SPH_ERR_OUT_OF_MEMORY;
    c->allocs = new std::vector<void *>();
    c->prm = *p;
    c->dp = make_dev_params(*p);
    apply_tables(*c);
    c->device = device;
    c->stream = (cudaStream_t)stream;
    c->n = p->vii[SPH_VII_NUM_PART2];
    c->num_cells = p->vii[SPH_VII_NUM_CELLS];
    int st = ctx_allocate(*c);
    if (st < 0) { c->free_all(); delete c->allocs; delete c; return st; }
    *out = c;
    return SPH_OK;
}

int sph_create(const sph_params *p, int precision, int device, void *stream, sph_ctx **out) {
    if (!p || !out) return SPH_ERR_BAD_ARG;
    *out = nullptr;
    int st = check_params(*p);
    if (st < 0) return st;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) { set_error("no CUDA device visible"); return SPH_ERR_NO_DEVICE; }
    if (device < 0 || device >= ndev) return SPH_ERR_BAD_ARG;
    SPH_CUDA_TRY(cudaSetDevice(device));
    sph_ctx *h = new (std::nothrow) sph_ctx();
    if (!h) return SPH_ERR_OUT_OF_MEMORY;
    h->prec = precision;
    if (precision == SPH_PREC_FP64) st = create_impl<double>(p, device, stream, &h->d);
    else if (precision == SPH_PREC_MIXED) st = create_impl<float>(p, device, stream, &h->f);
    else st = SPH_ERR_BAD_ARG;
    if (st < 0) { delete h; return st; }
    *out = h;
    return SPH_OK;
}

static void delete_step_graph(void *g);

void sph_destroy(sph_ctx *ctx) {
    if (!ctx) return;
    auto go = [](auto *c) {
        if (!c) return;
        cudaSetDevice(c->device);
        cudaStreamSynchronize(c->stream);
        for (int k = 0; k < 8; ++k) if (c->ev[k]) cudaEventDestroy(c->ev[k]);
        if (c->prof_ev) {
            for (int k = 0; k < 512; ++k) cudaEventDestroy(c->prof_ev[k]);
            delete[] c->prof_ev;
        }
        if (c->red_host) cudaFreeHost(c->red_host);
        release_solver_ws(*c);
        delete_step_graph(c->stepgraph);
        c->free_all();
        delete c->allocs;
        delete c;
    };
    go(ctx->f);
    go(ctx->d);
    delete ctx;
}

int sph_set_params(sph_ctx *ctx, const sph_params *p) {
    if (!ctx || !p) return SPH_ERR_BAD_ARG;
    int st = check_params(*p);
    if (st < 0) return st;
    auto go = [&](auto *c) -> int {
        if (p->vii[SPH_VII_NUM_PART2] != c->n || p->vii[SPH_VII_NUM_CELLS] != c->num_cells) {
            set_error("sph_set_params: particle count or cell grid changed");
            return SPH_ERR_BAD_ARG;
        }
        const int recompute = (p->ppe_pin != c->prm.ppe_pin);
        // the stored pair factors (correction matrix, pressure coefficients,
        // prep and pressure-force factors) follow the kernel function and
        // the pair forms
        const sph_params &o = c->prm;
        if (p->vii[SPH_VII_KERNEL_TYPE] != o.vii[SPH_VII_KERNEL_TYPE] || p->vif[SPH_VIF_KAPPA] != o.vif[SPH_VIF_KAPPA] ||
            p->vii[SPH_VII_KGC_SOLVE] != o.vii[SPH_VII_KGC_SOLVE] || p->pressure_length != o.pressure_length ||
            p->ppe_pair_h != o.ppe_pair_h || p->recompute_pairs != o.recompute_pairs ||
            p->pressure_force_form != o.pressure_force_form) {
            c->gc_valid = false;
            c->coef_valid = false;
            c->prep_valid = false;
            c->pforce_valid = false;
        }
        c->prm = *p;
        c->dp = make_dev_params(*p);
        apply_tables(*c);
        ++c->param_gen;
        if (recompute && c->built) return build_side_lists(*c);
        return SPH_OK;
    };
    return DISPATCH(ctx, go(ctx->f), go(ctx->d));
}

int sph_upload(sph_ctx *ctx, const sph_part1 *P1, const sph_part2 *P2, int n) {
    if (!ctx || !P1) return SPH_ERR_BAD_ARG;
    return DISPATCH(ctx, ctx_upload(*ctx->f, P1, P2, n), ctx_upload(*ctx->d, P1, P2, n));
}

int sph_upload_state(sph_ctx *ctx, const sph_part1 *P1, int n) {
    if (!ctx || !P1) return SPH_ERR_BAD_ARG;
    return DISPATCH(ctx, ctx_upload_state(*ctx->f, P1, n), ctx_upload_state(*ctx->d, P1, n));
}

int sph_download(sph_ctx *ctx, sph_part1 *P1, sph_part2 *P2, sph_part3 *P3) {
    if (!ctx) return SPH_ERR_BAD_ARG;
    return DISPATCH(ctx, ctx_download(*ctx->f, P1, P2, P3), ctx_download(*ctx->d, P1, P2, P3));
}

template <class Real>
static int nnps_impl(Ctx<Real> &c) {
    if (!c.uploaded) { set_error("sph_nnps: no particles uploaded"); return SPH_ERR_STATE; }
    SPH_CUDA_TRY(cudaEventRecord(c.ev[0], c.stream));
    int st = nnps_build(c);
    SPH_CUDA_TRY(cudaEventRecord(c.ev[1], c.stream));
    SPH_CUDA_TRY(cudaEventSynchronize(c.ev[1]));
    float ms = 0;
    cudaEventElapsedTime(&ms, c.ev[0], c.ev[1]);
    c.phase_ms[0] = ms;
    return st;
}

int sph_nnps(sph_ctx *ctx) {
    if (!ctx) return SPH_ERR_BAD_ARG;
    return DISPATCH(ctx, nnps_impl(*ctx->f), nnps_impl(*ctx->d));
}

int sph_nnps_export(sph_ctx *ctx, int32_t *g_idx, int32_t *p_idx, int32_t *g_str, int32_t *g_end) {
    if (!ctx) return SPH_ERR_BAD_ARG;
    return DISPATCH(ctx, nnps_export(*ctx->f, g_idx, p_idx, g_str, g_end), nnps_export(*ctx->d, g_idx, p_idx, g_str, g_end));
}

int sph_neighbors_export(sph_ctx *ctx, int64_t *offsets, int32_t *list, int64_t *nnz) {
    if (!ctx) return SPH_ERR_BAD_ARG;
    return DISPATCH(ctx, neighbors_export(*ctx->f, offsets, list, nnz), neighbors_export(*ctx->d, offsets, list, nnz));
}

template <class Real>
static int ensure_built(Ctx<Real> &c) {
    if (!c.uploaded) { set_error("no particles uploaded"); return SPH_ERR_STATE; }
    if (!c.built) return nnps_impl(c);   // NNPS of step 0 (ISPH_Calc.cuh:23-52)
    return SPH_OK;
}

template <class Real>
static int interaction_impl(Ctx<Real> &c) {
    SPH_TRY(ensure_built(c));
    return phase_interaction(c);
}
int sph_interaction(sph_ctx *ctx) {
    if (!ctx) return SPH_ERR_BAD_ARG;
    return DISPATCH(ctx, interaction_impl(*ctx->f), interaction_impl(*ctx->d));
}

template <class Real>
static int ppe_impl(Ctx<Real> &c, sph_ppe_stats *st) {
    if (!c.built) { set_error("sph_ppe before sph_interaction"); return SPH_ERR_STATE; }
    c.defer_stats = false;
    sph_ppe_stats ps{};
    SPH_TRY(phase_ppe(c, &ps));
    if (st) *st = ps;
    return ps.status < 0 ? ps.status : SPH_OK;
}
int sph_ppe(sph_ctx *ctx, sph_ppe_stats *stats) {
    if (!ctx) return SPH_ERR_BAD_ARG;
    return DISPATCH(ctx, ppe_impl(*ctx->f, stats), ppe_impl(*ctx->d, stats));
}

template <class Real>
static int tu_impl(Ctx<Real> &c) {
    if (!c.built) { set_error("sph_time_update before sph_interaction"); return SPH_ERR_STATE; }
    return phase_time_update(c);
}
int sph_time_update(sph_ctx *ctx) {
    if (!ctx) return SPH_ERR_BAD_ARG;
    return DISPATCH(ctx, tu_impl(*ctx->f), tu_impl(*ctx->d));
}

// ---------------------------------------------------------------------------
// A whole step as one CUDA graph, for contexts whose solve runs under device
// control (ppe_refinement = 4).  Once a step at count >= 1 has run launch by
// launch, the next one with the same buffers and parameters is captured:
// the interaction passes, the solve with its conditional nodes, the time
// update and the device clock's advance, with the phase events as
// event-record nodes; later steps replay it.  The kernels read the step
// counter and time from the device clock, so a replay computes exactly what
// the launches would.  Steps at count 0 (the markers' normals and the step-0
// Neumann pass run only there), the first step after any allocation, release
// or change of parameters, and host-controlled solves run launch by launch.
// ---------------------------------------------------------------------------
struct StepGraph {
    cudaGraphExec_t exec = nullptr;
    std::vector<unsigned long long> key;      // state the graph was captured in
    std::vector<unsigned long long> warm;     // state after the last step run launch by launch at count >= 1
    std::vector<unsigned long long> failed;   // state in which a capture failed
    long long launches = 0;                   // launches one replay stands for (the solve counted as one)
    ~StepGraph() {
        if (exec) cudaGraphExecDestroy(exec);
    }
};

static void delete_step_graph(void *g) { delete (StepGraph *)g; }

template <class Real>
static std::vector<unsigned long long> step_key(const Ctx<Real> &c) {
    return {c.mem_gen, c.param_gen, (unsigned long long)c.n, (unsigned long long)c.nnz_padded,
            (unsigned long long)(uintptr_t)c.stream, (unsigned long long)c.pair_block, (unsigned long long)c.cg_block,
            (unsigned long long)((c.built ? 1 : 0) | (c.gc_valid ? 2 : 0) | (c.prep_valid ? 4 : 0) |
                                 (c.pforce_valid ? 8 : 0) | (c.coef_valid ? 16 : 0) | (c.coef_h_valid ? 32 : 0) |
                                 (c.cg_valid ? 64 : 0) | (c.clk_synced ? 128 : 0))};
}

// captures one step into sg->exec; on failure nothing has run on the device
template <class Real>
static int capture_step(Ctx<Real> &c, StepGraph *sg) {
    if (sg->exec) { cudaGraphExecDestroy(sg->exec); sg->exec = nullptr; }
    cudaGraph_t graph = nullptr;
    SPH_CUDA_TRY(cudaGraphCreate(&graph, 0));
    if (cudaStreamBeginCaptureToGraph(c.stream, graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) !=
        cudaSuccess) {
        cudaGraphDestroy(graph);
        cudaGetLastError();
        return SPH_ERR_CUDA;
    }
    const long long l0 = c.launches;
    c.capturing = true;
    sph_ppe_stats ps{};
    int st = record_event(c, c.ev[1]) == cudaSuccess ? SPH_OK : SPH_ERR_CUDA;
    if (st == SPH_OK) st = phase_interaction(c);
    if (st == SPH_OK) st = record_event(c, c.ev[2]) == cudaSuccess ? SPH_OK : SPH_ERR_CUDA;
    if (st == SPH_OK) st = phase_ppe(c, &ps);
    if (st == SPH_OK) st = record_event(c, c.ev[3]) == cudaSuccess ? SPH_OK : SPH_ERR_CUDA;
    if (st == SPH_OK) st = phase_time_update(c);
    if (st == SPH_OK) st = record_event(c, c.ev[6]) == cudaSuccess ? SPH_OK : SPH_ERR_CUDA;
    c.capturing = false;
    cudaGraph_t done = nullptr;
    const cudaError_t e = cudaStreamEndCapture(c.stream, &done);
    if (st == SPH_OK && e == cudaSuccess && cudaGraphInstantiate(&sg->exec, graph, 0) != cudaSuccess) sg->exec = nullptr;
    cudaGraphDestroy(graph);
    sg->launches = c.launches - l0;
    c.launches = l0;
    if (!sg->exec) {
        cudaGetLastError();
        return st < 0 ? st : SPH_ERR_CUDA;
    }
    return SPH_OK;
}

// runs the step as the step graph when it can; *ran tells whether it did
template <class Real>
static int step_graph(Ctx<Real> &c, bool *ran) {
    *ran = false;
    if (c.count < 1 || !solve_under_device_control(c)) return SPH_OK;
    auto *sg = (StepGraph *)c.stepgraph;
    if (!sg) {
        sg = new (std::nothrow) StepGraph();
        if (!sg) return SPH_ERR_OUT_OF_MEMORY;
        c.stepgraph = sg;
    }
    const std::vector<unsigned long long> key = step_key(c);
    static const bool trace = getenv("SPH_TRACE_STEP") != nullptr;
    if (!sg->exec || sg->key != key) {
        if (sg->warm != key || sg->failed == key) {
            if (trace)
                fprintf(stderr, "step %d: launch by launch (%s; mem_gen %llu param_gen %llu flags %llu)\n", c.count,
                        sg->failed == key ? "capture failed in this state" : "state not yet steady", c.mem_gen,
                        c.param_gen, key.back());
            return SPH_OK;
        }
        if (capture_step(c, sg) < 0) {
            if (trace) fprintf(stderr, "step %d: capture failed: %s\n", c.count, sph_last_error());
            sg->failed = key;
            return SPH_OK;   // this state steps launch by launch
        }
        if (trace) fprintf(stderr, "step %d: captured (%lld launches)\n", c.count, sg->launches);
        sg->key = key;
    }
    if (trace) fprintf(stderr, "step %d: replay\n", c.count);
    SPH_CUDA_TRY(cudaGraphLaunch(sg->exec, c.stream));
    c.launches += sg->launches;
    ++c.graph_steps;
    c.ppe_pending = true;
    *ran = true;
    return finish_step(c);
}

template <class Real>
static int step_impl(Ctx<Real> &c, int nsteps, sph_ppe_stats *stats) {
    int last = SPH_OK;
    // device-controlled solves (ppe_refinement = 4) leave their statistics on
    // the device: the steps then follow one another without host waits, and
    // the host reads the last solve's statistics and the worst status of all
    // of them once, after the last step
    SPH_TRY(dev_reset_worst(c));
    c.defer_stats = true;
    bool pending = false;
    for (int s = 0; s < nsteps; ++s) {
        int st = ensure_built(c);
        bool replayed = false;
        if (st == SPH_OK) st = step_graph(c, &replayed);
        if (st < 0) { c.defer_stats = false; return st; }
        if (replayed) {
            pending = true;
            continue;
        }
        const int count0 = c.count;
        const unsigned long long gen0 = c.mem_gen;
        if (st == SPH_OK) st = cudaEventRecord(c.ev[1], c.stream) == cudaSuccess ? SPH_OK : SPH_ERR_CUDA;
        if (st == SPH_OK) st = phase_interaction(c);
        if (st == SPH_OK) st = cudaEventRecord(c.ev[2], c.stream) == cudaSuccess ? SPH_OK : SPH_ERR_CUDA;
        sph_ppe_stats ps{};
        if (st == SPH_OK) st = phase_ppe(c, &ps);
        if (st == SPH_OK) st = cudaEventRecord(c.ev[3], c.stream) == cudaSuccess ? SPH_OK : SPH_ERR_CUDA;
        if (st == SPH_OK) st = phase_time_update(c);
        if (st == SPH_OK) st = cudaEventRecord(c.ev[6], c.stream) == cudaSuccess ? SPH_OK : SPH_ERR_CUDA;
        if (st < 0) { c.defer_stats = false; return st; }
        // a step that allocated nothing leaves a state the next step can be
        // captured in (a context that allocates every step, e.g. with
        // recompute_gc, stays launch by launch)
        if (c.stepgraph) {
            auto *sg = (StepGraph *)c.stepgraph;
            if (count0 >= 1 && c.mem_gen == gen0) sg->warm = step_key(c);
            else sg->warm.clear();
            if (getenv("SPH_TRACE_STEP"))
                fprintf(stderr, "step %d ran launch by launch: mem_gen %llu -> %llu\n", count0, gen0, c.mem_gen);
        }
        pending = c.ppe_pending;
        if (!pending) {
            SPH_CUDA_TRY(cudaEventSynchronize(c.ev[6]));
            cudaEventElapsedTime(&c.phase_ms[1], c.ev[1], c.ev[2]);
            cudaEventElapsedTime(&c.phase_ms[2], c.ev[2], c.ev[3]);
            cudaEventElapsedTime(&c.phase_ms[3], c.ev[3], c.ev[6]);
            if (stats) *stats = ps;
            last = ps.status;
        }
    }
    c.defer_stats = false;
    if (pending) {
        sph_ppe_stats ps{};
        int worst = SPH_OK;
        SPH_TRY(dev_solve_stats(c, &ps, &worst));
        cudaEventElapsedTime(&c.phase_ms[1], c.ev[1], c.ev[2]);
        cudaEventElapsedTime(&c.phase_ms[2], c.ev[2], c.ev[3]);
        cudaEventElapsedTime(&c.phase_ms[3], c.ev[3], c.ev[6]);
        if (stats) *stats = ps;
        if (worst < 0) { set_error("a device-controlled pressure solve broke down"); return worst; }
        last = worst;
    }
    return last == SPH_NOT_CONVERGED ? SPH_NOT_CONVERGED : SPH_OK;
}
int sph_step(sph_ctx *ctx, int nsteps, sph_ppe_stats *stats) {
    if (!ctx || nsteps < 0) return SPH_ERR_BAD_ARG;
    return DISPATCH(ctx, step_impl(*ctx->f, nsteps, stats), step_impl(*ctx->d, nsteps, stats));
}

int sph_diagnostics(sph_ctx *ctx, float *max_umag, float *max_drho_pct, float *max_ftotal) {
    if (!ctx) return SPH_ERR_BAD_ARG;
    return DISPATCH(ctx, ctx_diagnostics(*ctx->f, max_umag, max_drho_pct, max_ftotal),
                    ctx_diagnostics(*ctx->d, max_umag, max_drho_pct, max_ftotal));
}

int sph_last_phase_ms(sph_ctx *ctx, float *ms4) {
    if (!ctx || !ms4) return SPH_ERR_BAD_ARG;
    auto go = [&](auto *c) { for (int k = 0; k < 4; ++k) ms4[k] = c->phase_ms[k]; return SPH_OK; };
    return DISPATCH(ctx, go(ctx->f), go(ctx->d));
}

int64_t sph_launch_count(sph_ctx *ctx) {
    if (!ctx) return -1;
    return DISPATCH(ctx, ctx->f->launches, ctx->d->launches);
}

int sph_operator_counts(sph_ctx *ctx, int64_t counts[6]) {
    if (!ctx || !counts) return SPH_ERR_BAD_ARG;
    auto go = [&](auto *c) {
        counts[0] = c->n;
        counts[1] = c->nnz_op;
        counts[2] = c->L.n_nm;
        counts[3] = c->L.nm_nnz;
        counts[4] = c->num_cells;
        counts[5] = (c->list16 && c->prm.ppe_matrix_free == 0) ? 1 : 0;
        return SPH_OK;
    };
    return DISPATCH(ctx, go(ctx->f), go(ctx->d));
}

int sph_set_prop_tables(sph_ctx *ctx, const sph_prop_tables *t) {
    if (!ctx || !t) return SPH_ERR_BAD_ARG;
    for (int k = 0; k < SPH_TABLE_SLOTS; ++k)
        if (t->size[k] < 0 || t->size[k] > SPH_TABLE_SIZE || t->index[k] < 0 ||
            t->index[k] + t->size[k] > SPH_TABLE_SIZE) {
            set_error("sph_set_prop_tables: a table lies outside the SPH_TABLE_SIZE entries");
            return SPH_ERR_BAD_ARG;
        }
    auto go = [&](auto *c) -> int {
        typedef typename std::remove_pointer<decltype(c->tab)>::type R;
        R host[2 * SPH_TABLE_SIZE];
        for (int k = 0; k < SPH_TABLE_SIZE; ++k) { host[k] = (R)t->h[k]; host[SPH_TABLE_SIZE + k] = (R)t->T[k]; }
        SPH_CUDA_TRY(cudaSetDevice(c->device));
        // from pageable memory: the copy has taken the values when it returns
        SPH_CUDA_TRY(cudaMemcpyAsync(c->tab, host, sizeof(host), cudaMemcpyHostToDevice, c->stream));
        for (int k = 0; k < SPH_TABLE_SLOTS; ++k) { c->tab_index[k] = t->index[k]; c->tab_size[k] = t->size[k]; }
        c->tab_set = true;
        apply_tables(*c);
        ++c->param_gen;
        return SPH_OK;
    };
    return DISPATCH(ctx, go(ctx->f), go(ctx->d));
}

int sph_energy_convert(sph_ctx *ctx, int to_enthalpy) {
    if (!ctx || (to_enthalpy != 0 && to_enthalpy != 1)) return SPH_ERR_BAD_ARG;
    auto go = [&](auto *c) -> int {
        if (!c->uploaded) { set_error("sph_energy_convert: no records uploaded"); return SPH_ERR_STATE; }
        if (c->dp.prop_table && !c->tab_set) {
            set_error("sph_energy_convert: prop_table = 1 needs sph_set_prop_tables");
            return SPH_ERR_STATE;
        }
        SPH_CUDA_TRY(cudaSetDevice(c->device));
        return energy_convert(*c, to_enthalpy);
    };
    return DISPATCH(ctx, go(ctx->f), go(ctx->d));
}

int64_t sph_step_graph_count(sph_ctx *ctx) {
    if (!ctx) return -1;
    return DISPATCH(ctx, ctx->f->graph_steps, ctx->d->graph_steps);
}

int sph_set_pair_block(sph_ctx *ctx, int threads) {
    if (!ctx || (threads != 32 && threads != 64 && threads != 128)) {
        set_error("sph_set_pair_block: threads must be 32, 64 or 128");
        return SPH_ERR_BAD_ARG;
    }
    auto go = [&](auto *c) { c->pair_block = threads; ++c->param_gen; return SPH_OK; };
    return DISPATCH(ctx, go(ctx->f), go(ctx->d));
}

int sph_profile(sph_ctx *ctx, int enable) {
    if (!ctx) return SPH_ERR_BAD_ARG;
    auto go = [&](auto *c) { c->prof = enable != 0; return SPH_OK; };
    return DISPATCH(ctx, go(ctx->f), go(ctx->d));
}

int sph_operator_stats(sph_ctx *ctx, int64_t *launches, double *total_ms, double *bytes_per_launch, int reset) {
    if (!ctx) return SPH_ERR_BAD_ARG;
    return DISPATCH(ctx, operator_stats(*ctx->f, launches, total_ms, bytes_per_launch, reset),
                    operator_stats(*ctx->d, launches, total_ms, bytes_per_launch, reset));
}

int sph_operator_bytes(sph_ctx *ctx, double *stored, double *index_rule) {
    if (!ctx) return SPH_ERR_BAD_ARG;
    return DISPATCH(ctx, operator_bytes(*ctx->f, stored, index_rule), operator_bytes(*ctx->d, stored, index_rule));
}

// ---- learned warm start (learned.cu) ------------------------------------------
int sph_ml_collect(sph_ctx *ctx, int every) {
    if (!ctx || every < 0) return SPH_ERR_BAD_ARG;
    auto go = [&](auto *c) { c->ml_every = every; return SPH_OK; };
    return DISPATCH(ctx, go(ctx->f), go(ctx->d));
}

int sph_ml_samples(sph_ctx *ctx, int64_t first, int64_t rows, uint16_t *X, float *target, int64_t *count) {
    if (!ctx) return SPH_ERR_BAD_ARG;
    long long cnt = 0;
    const int st = DISPATCH(ctx, ml_samples(*ctx->f, first, rows, X, target, &cnt),
                            ml_samples(*ctx->d, first, rows, X, target, &cnt));
    if (count) *count = cnt;
    return st;
}

int sph_ml_train(sph_ctx *ctx, int epochs, int batch, float lr, uint64_t seed, float *final_loss) {
    if (!ctx || !(lr > 0)) return SPH_ERR_BAD_ARG;
    return DISPATCH(ctx, ml_train(*ctx->f, epochs, batch, lr, (unsigned long long)seed, final_loss),
                    ml_train(*ctx->d, epochs, batch, lr, (unsigned long long)seed, final_loss));
}

int sph_ml_set_weights(sph_ctx *ctx, const float *w) {
    if (!ctx || !w) return SPH_ERR_BAD_ARG;
    return DISPATCH(ctx, ml_set_weights(*ctx->f, w), ml_set_weights(*ctx->d, w));
}

int sph_ml_get_weights(sph_ctx *ctx, float *w) {
    if (!ctx || !w) return SPH_ERR_BAD_ARG;
    return DISPATCH(ctx, ml_get_weights(*ctx->f, w), ml_get_weights(*ctx->d, w));
}

int sph_ml_grad(sph_ctx *ctx, int64_t first, int32_t rows, float *loss, float *grad) {
    if (!ctx) return SPH_ERR_BAD_ARG;
    return DISPATCH(ctx, ml_grad(*ctx->f, first, rows, loss, grad), ml_grad(*ctx->d, first, rows, loss, grad));
}

int sph_ml_predict_samples(sph_ctx *ctx, int64_t first, int32_t rows, float *y) {
    if (!ctx || !y) return SPH_ERR_BAD_ARG;
    return DISPATCH(ctx, ml_predict_samples(*ctx->f, first, rows, y), ml_predict_samples(*ctx->d, first, rows, y));
}

int sph_apr(sph_ctx *ctx, int32_t *n_split, int32_t *n_wanted) {
    if (!ctx) return SPH_ERR_BAD_ARG;
    int a = 0, b = 0, m = 0;
    auto go = [&](auto *c) -> int {
        SPH_TRY(ensure_built(*c));
        return apr_pass(*c, &a, &b, &m);
    };
    const int st = DISPATCH(ctx, go(ctx->f), go(ctx->d));
    if (n_split) *n_split = a;
    if (n_wanted) *n_wanted = b;
    return st;
}

int sph_apr_state(sph_ctx *ctx, int32_t *family, float *target, int32_t *n_merged) {
    if (!ctx) return SPH_ERR_BAD_ARG;
    auto go = [&](auto *c) -> int {
        if (n_merged) *n_merged = c->apr_last_merged;
        return apr_state(*c, family, target);
    };
    return DISPATCH(ctx, go(ctx->f), go(ctx->d));
}

int sph_set_ib_boxes(sph_ctx *ctx, const double *boxes, int nbox) {
    if (!ctx || nbox < 0 || (nbox > 0 && !boxes)) return SPH_ERR_BAD_ARG;
    auto go = [&](auto *c) -> int {
        c->release(c->ib_boxes);
        c->n_ib_boxes = nbox;
        if (nbox == 0) return SPH_OK;
        SPH_TRY(c->alloc(c->ib_boxes, 6 * (size_t)nbox));
        SPH_CUDA_TRY(cudaMemcpyAsync(c->ib_boxes, boxes, sizeof(double) * 6 * nbox, cudaMemcpyHostToDevice, c->stream));
        SPH_CUDA_TRY(cudaStreamSynchronize(c->stream));
        return SPH_OK;
    };
    return DISPATCH(ctx, go(ctx->f), go(ctx->d));
}
