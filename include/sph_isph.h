/*
 * sph_isph.h -- C ABI of the B200-native ISPH time step.
 *
 * Drop-in boundary for the step the reference drives from
 * SOPHIA_single_ISPH (ISPH_Calc.cuh:4-233).  The reference has no library or
 * ABI: its "operator surface" is a set of __global__ kernels that take raw
 * device pointers to the AoS particle arrays part1/part2/part3
 * (class_Cuda_Particle_Array.cuh:11-112) and read every parameter from the
 * __constant__ tables k_vii[64] / k_vif[32] (SOPHIA_gpu.cu:47-48, names in
 * function_init.cuh:84-163).  This header keeps both: the particle records
 * below have the reference's exact layout (Real = float), and sph_params
 * carries the same two tables plus the constants the reference hard-wires as
 * #defines or literals (each field names the line it replaces).
 *
 * Conventions:
 *   - every call returns an int status (SPH_OK = 0, > 0 warnings, < 0 errors);
 *     no exception or exit() crosses the boundary;
 *   - a context owns all of its device memory, is bound to one device and one
 *     CUDA stream, and is not thread-safe (one host thread at a time);
 *   - calls are stream-ordered; only the *_download / *_export calls,
 *     sph_ppe's statistics and sph_upload of records in device memory
 *     synchronise the stream;
 *   - particle indices in exported arrays are in the reference's sorted
 *     order (the order KERNEL_reorder produces, functions_NNPS.cuh:840-843).
 */
#ifndef SPH_ISPH_H
#define SPH_ISPH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define SPH_OK                 0
#define SPH_NOT_CONVERGED      1   /* PPE stopped at max_iter above tol      */
#define SPH_ERR_BAD_ARG       -1
#define SPH_ERR_CUDA          -2
#define SPH_ERR_BREAKDOWN     -3   /* Krylov breakdown that restart could not cure */
#define SPH_ERR_STATE         -4   /* call made in the wrong order           */
#define SPH_ERR_NO_DEVICE     -5
#define SPH_ERR_OUT_OF_MEMORY -6
#define SPH_ERR_UNSUPPORTED   -7

/* ---- precision forms --------------------------------------------------- */
#define SPH_PREC_MIXED 0   /* FP32 state and neighbour sums, FP64 Krylov scalars */
#define SPH_PREC_FP64  1   /* whole step in FP64 (the plain form)              */

/* ---- pressure solve modes ---------------------------------------------- */
#define SPH_PPE_REF_SWEEP  0  /* one point-Jacobi sweep, KERNEL_PPE3D semantics
                                 (functions_PPE.cuh:2-175) without its race   */
#define SPH_PPE_BICGSTAB   1  /* Jacobi-preconditioned BiCGSTAB in the context's
                                 precision, FP64 reductions                   */
#define SPH_PPE_MIXED_IR   2  /* FP32 BiCGSTAB with FP64 reliable updates (FP64
                                 solution, FP64 true residual replacing the
                                 recurrence residual at every 10x drop);
                                 FP64 BiCGSTAB in an FP64 context             */
#define SPH_PPE_LEARNED    3  /* MIXED_IR warm-started by the per-particle net   */
#define SPH_PPE_GMRES      4  /* restarted GMRES(m) in the context's precision,
                                 FP64 reductions                              */
#define SPH_PPE_IDRS       5  /* IDR(4) (biorthogonal variant, right
                                 preconditioned) in the context's precision,
                                 FP64 reductions; iterations count operator
                                 applications (a BiCGSTAB iteration is two)  */

/* ---- particle records: class_Cuda_Particle_Array.cuh:11-112, Real=float --- */
typedef struct sph_part1 {
    int32_t i_type, buffer_type, MOST_buffer, p_type;
    float x, y, z;
    float ux, uy, uz;
    float m, h, temp, pres, pres0, rho, flt_s, enthalpy, concn, concentration;
    float k_turb, e_turb;
    float eli, vol;
    float m_ref, h_ref;
    float vis_t;
    float fbx, fby, fbz;
    float fmx, fmy, hmz;
    float float1, float2, float3;
    int32_t ncell, source;
} sph_part1;                                      /* 152 bytes */

typedef struct sph_part2 {
    float rho_ref, SR;
    float x0, y0, z0;
    float ux0, uy0, uz0;
    float rho0, drho0, temp0, concn0, enthalpy0;
} sph_part2;                                      /* 52 bytes */

typedef struct sph_part3 {
    float drho, dconcn, denthalpy;
    float ftotalx, ftotaly, ftotalz, ftotal;
    float fpx, fpy, fpz, fbody;
    float dtemp;
    float dk_turb, de_trub;
    float cc;
    float nx, ny, nz;
    float Cm[3][3];
    float inv_cm_xx, inv_cm_yy, inv_cm_zz;
    float inv_cm_xy, inv_cm_yz, inv_cm_zx;
    float Gxx, Gxy, Gyx, Gyy;
    float L11, L12, L21, L22;
} sph_part3;                                      /* 164 bytes */

/* ---- k_vii / k_vif slots (function_init.cuh:84-163) ------------------- */
enum sph_vii_slot {
    SPH_VII_SOLVER_TYPE = 0, SPH_VII_DIM = 1, SPH_VII_PROP_TABLE = 2, SPH_VII_KERNEL_TYPE = 3,
    SPH_VII_TIME_TYPE = 4, SPH_VII_OPEN_BOUNDARY = 5, SPH_VII_FREQ_FILT = 8,
    SPH_VII_FREQ_OUTPUT = 11, SPH_VII_FP_SOLVE = 12, SPH_VII_FV_SOLVE = 13, SPH_VII_FG_SOLVE = 14,
    SPH_VII_CON_SOLVE = 15, SPH_VII_BOUSSINESQ = 16, SPH_VII_KGC_SOLVE = 17,
    SPH_VII_TURBULENCE = 18, SPH_VII_CONCN_SOLVE = 19, SPH_VII_MIN_ITER = 20, SPH_VII_MAX_ITER = 21,
    SPH_VII_NUM_PART = 23, SPH_VII_NI = 24, SPH_VII_NJ = 25, SPH_VII_NK = 26, SPH_VII_COUNT = 27,
    SPH_VII_NUM_CELLS = 28, SPH_VII_NGPU = 29, SPH_VII_NUM_PART2 = 32, SPH_VII_NOSLIP_BC = 34,
    SPH_VII_APR_SOLV = 35, SPH_VII_H_CHANGE = 36, SPH_VII_FREQ_APR = 37
};
enum sph_vif_slot {
    SPH_VIF_KAPPA = 0, SPH_VIF_P_REF = 1, SPH_VIF_DT = 2, SPH_VIF_TIME = 3, SPH_VIF_TIME_END = 4,
    SPH_VIF_U_LIMIT = 5, SPH_VIF_DP_TH = 7, SPH_VIF_X_MIN = 9, SPH_VIF_X_MAX = 10,
    SPH_VIF_Y_MIN = 11, SPH_VIF_Y_MAX = 12, SPH_VIF_Z_MIN = 13, SPH_VIF_Z_MAX = 14,
    SPH_VIF_SEARCH_INCR = 16, SPH_VIF_SEARCH_KAPPA = 17, SPH_VIF_DCELL = 18,
    SPH_VIF_BUFFERSIZE = 19, SPH_VIF_DT_STRUCTURE = 20
};

#define SPH_MAX_PROFILE 32

/* ---- parameters --------------------------------------------------------- */
typedef struct sph_params {
    int32_t vii[64];      /* k_vii, same slots as the reference            */
    float   vif[32];      /* k_vif, same slots as the reference            */

    /* constants the reference hard-wires; defaults are the reference values.
       Stored as double: kernels convert each one to the type the reference
       evaluates it in at that use site (a double literal or a Real). */
    double cs_sgs;            /* Cs_sgs 0.15                 Parameters.cuh:135  */
    double l2, l3;            /* L2, L3 buffer planes         functions_NNPS.cuh:5-6 */
    double l_left, l_right;   /* periodic-y planes            functions_NNPS.cuh:9-10 */
    double outlet_probe_dx;   /* xg = L3 - 0.008              functions_BC.cuh:732 */
    double partner_tol;       /* exact-position match 1e-3    functions_BC.cuh:737,1122 */
    double ghost_tol;         /* ghost-node match 0.1         functions_BC.cuh:361, functions_MOST.cuh:294 */
    double ib_box[6];         /* IB face planes x0,x1,y0,y1,z0,z1  functions_PREP.cuh:958-963 */
    double ib_face_tol;       /* 1e-5                         functions_PREP.cuh:958 */
    double most_z0, most_z0h; /* MOST_z0 1.0, MOST_z0h 0.1    Parameters.cuh:114-115 */
    double most_ghost_dz;     /* ghost 5 m above              functions_MOST.cuh:266 */
    double rho_air;           /* Rho_air 1.225                Parameters.cuh:143 */
    double ibm_target_coeff;  /* Ubtx = 0.2*profile(z)        functions_IBM.cuh:470 */
    double visc_fluid, visc_wall, visc_marker; /* viscosity2  functions_PROP.cuh:121-131 */
    double av_alpha, av_beta, av_c0;  /* artificial viscosity functions_PPE.cuh:268-271 */
    double pressure_length, ibm_length, neumann_coeff; /* Parameters.cuh:105-106, functions_BC.cuh:308 */
    double t_ini, t_con, t_start, t_con_t;    /* wall temperature ramp Parameters.cuh:121-124 */
    double boundary_velocity; /* MOVING wall speed            Parameters.cuh:76 */
    int32_t n_profile;        /* wall-model target table      functions_IBM.cuh:289-304 */
    int32_t pad0;
    double profile_z[SPH_MAX_PROFILE];
    double profile_u[SPH_MAX_PROFILE];

    /* pressure solve (new work: the reference runs one sweep per step) */
    int32_t ppe_mode;        /* SPH_PPE_*                                      */
    int32_t ppe_max_iter;
    double  ppe_tol;         /* relative residual ||b-Ap||/||b||               */
    int32_t ppe_pin;         /* singular (pure-Neumann) pressure problems: 0 none,
                                1 rank-one mean-pressure term per singular
                                component (default), 2 one row pinned to p=0 */
    int32_t recompute_gc;    /* 1: recompute the correction matrix every step  */
    int32_t ppe_matrix_free; /* 1: PPE operator recomputes c_ij at every
                                application instead of reading the cache      */
    int32_t ppe_gmres_restart;   /* GMRES restart length (0: 40, max 64)       */
    int32_t ppe_refinement;  /* MIXED_IR: 0 reliable updates (default); 1 / 2 / 3
                                iterative refinement restarting FP32 GMRES /
                                BiCGSTAB / IDR(4) at every correction; 4 the
                                reliable updates under device control: the
                                whole solve is one CUDA graph whose conditional
                                nodes take the host loop's decisions, and
                                sph_step reads the statistics once, after its
                                last step; from the third step of a context
                                on (count >= 2, buffers and parameters
                                unchanged since the step before), sph_step
                                captures a whole step around the solve as one
                                graph and replays it (same iterates as 0; used
                                when the context has its own stream and no
                                live profiling, learned start or sample
                                collection, else 0 runs)                       */
    int32_t ppe_coarse_block;    /* BiCGSTAB preconditioner: 0 Jacobi; B > 0
                                adds a coarse correction on aggregates of
                                B x B x B NNPS cells (additive two-level); -B
                                aggregates balanced by row count: blocks of
                                B x B x B cells, the block with the most rows
                                split into octants again and again while at
                                most ppe_coarse_max aggregates result         */
    int32_t ppe_warm_start;  /* start vector of the converged solves: 0 previous
                                pressure; 1 linear extrapolation in time,
                                2 p_n - p_(n-1), once two solutions exist;
                                3 the previous pressure times the factor that
                                minimises the FP64 residual (so the start
                                residual never exceeds that of a zero start) */
    int32_t apr_max_level;   /* APR (vii[35] = 1, every vii[37] steps): target
                                level log8(m_ref/m) of fluid near IBM markers */
    int32_t outlet_bc;       /* pass at the outlet-buffer call sites of the step
                                (ISPH_Calc.cuh:151, 208): 0 the reference's
                                KERNEL_donothing_buffer3D; 1 its dormant
                                KERNEL_open_boundary_extrapolation_buffer3D
                                (functions_BC.cuh:763-855); 2 its dormant
                                KERNEL_inout_boundary3D (functions_BC.cuh:1274-1433) */
    int32_t inlet_recycling; /* 1: the dormant KERNEL_Recycling3D at the end of
                                the step (ISPH_Calc.cuh:215; functions_BC.cuh:
                                1857-1941): inlet ux = u* / kappa_vK log(z / z0)
                                with u* from the MOST particle at the probe    */
    int32_t ppe_coarse_mode; /* with ppe_coarse_block > 0 in the BiCGSTAB forms:
                                0 additive (D^-1 r + Z E^-1 Z^T r); 1
                                multiplicative (z = D^-1 r, then z += Z E^-1
                                Z^T (r - M z): one more operator application
                                per preconditioner call)                      */
    int32_t ppe_pair_h;      /* smoothing length of a pair in the pressure
                                system (rows, right-hand side, operator): 0 h_i
                                as KERNEL_PPE3D uses it; 1 (h_i + h_j) / 2, the
                                multi-resolution form that KERNEL_PPE3D keeps
                                commented out (functions_PPE.cuh:113-116) and
                                KERNEL_pressureforce3D uses (:598-602)         */
    int32_t ppe_wide_index;  /* 1: the pressure operator reads the 32-bit
                                neighbour indices; 0 (default): 16-bit codes
                                (cell plane of the entry, offset from the
                                plane's first reachable record) wherever every
                                row searches at most two cells around its own
                                and every offset is below 8192 -- same
                                entries, same order, same results, fewer
                                bytes; otherwise the 32-bit indices
                                (sph_operator_counts tells which)             */
    int32_t recompute_pairs; /* 1: the prep pass and the pressure force evaluate
                                their pair terms every step, as the reference
                                does; 0 (default): their time-invariant pair
                                factors are stored at the neighbour build (the
                                particles never move) when they fit with a
                                tenth of the device memory to spare          */
    int32_t pressure_force_form; /* pair term of the pressure force
                                (KERNEL_pressureforce3D, functions_PPE.cuh:
                                620-627): 0 (default) the reference's active
                                "Monaghan variation" -2 m_j ((p_i + Pb) rho_j +
                                (p_j + Pb) rho_i) / ((rho_i rho_j)(rho_i +
                                rho_j)), Pb = 0; 1 its commented-out difference
                                form -m_j (p_j - p_i) / (rho_i rho_j) (the
                                "pressure stabilization (KDH)" line with its
                                stabilisation term zero), which exerts no force
                                for a constant pressure                       */
    int32_t ppe_coef_half;   /* 1: the FP32 operator applications of the mixed
                                form read the cached coefficients as FP16,
                                each row's c_ij divided by the row's largest
                                |c_ij| (one FP32 scale per row): 2 bytes per
                                stored entry instead of 4.  The FP64
                                applications (true residuals, the solution
                                the tolerance is checked on) keep the FP32
                                coefficients                                  */
    int32_t ppe_coarse_max;  /* most aggregates of the balanced coarse space
                                (ppe_coarse_block < 0): 0 means 4096; at most
                                32768 (the dense coarse inverse holds m^2
                                entries: 4.3 GB in FP32 at 32768)             */
    int32_t enthalpy_eqn;    /* with vii con_solve = 1: 1 the energy equation
                                in enthalpy (the reference's enthalpy_eqn,
                                Parameters.cuh:96, compiled out there): the
                                conduction sum is the enthalpy rate, the
                                projection sets enthalpy0 and the temperature
                                htoT(enthalpy) from the built-in corium table
                                (functions_PROP.cuh:43-67), or with
                                vii[prop_table] = 1 from the tables of
                                sph_set_prop_tables, the time update
                                advances the enthalpy; 0 (default) the
                                temperature form                              */
    double  ppe_inner_tol;   /* inner FP32 tolerance of the restarted
                                refinement forms of SPH_PPE_MIXED_IR (0: 1e-3) */
    double  apr_zone;        /* APR: distance from an IBM marker's cell within
                                which fluid targets apr_max_level [m]          */
    double  recycle_probe_x, recycle_probe_y;   /* the MOST particle whose u*
                                feeds inlet recycling: (x - px)^2 + (y - py)^2
                                < 1e-3 (functions_MOST.cuh:316: 600, 0)        */
    double  periodic_box[6]; /* x0,x1,y0,y1,z0,z1 of a periodic box (new work:
                                the reference's only periodicity is the y copy
                                of functions_BC.cuh:1015-1154).  A record with
                                buffer_type SPH_BUFFER_PERIODIC_GHOST copies u,
                                p and T from the record at its position
                                wrapped into the box (|d| < partner_tol), after
                                the periodic-y copy at each of its call sites;
                                in the pressure system it is a copy row.      */
} sph_params;

#define SPH_BUFFER_PERIODIC_GHOST 7

typedef struct sph_ppe_stats {
    int32_t status;          /* SPH_OK / SPH_NOT_CONVERGED / error             */
    int32_t iterations;      /* Krylov iterations (all refinement sweeps)      */
    int32_t refinements;     /* FP64 residual replacements / refinement sweeps
                                (MIXED_IR)                                     */
    int32_t restarts;        /* breakdown restarts                             */
    double  rel_residual;    /* final ||b-Ap||_2/||b||_2, FP64                 */
    double  solve_ms;        /* device time from rhs ready to convergence      */
    double  initial_residual;    /* ||b-Ap0||_2/||b||_2 of the start vector p0 */
} sph_ppe_stats;

typedef struct sph_ctx sph_ctx;

/* Fills the reference defaults (read_solv_input zeroes, then the values a
 * Case-H solv.txt sets) and the promoted constants. */
int sph_params_init(sph_params *p);

/* Host-side domain set-up of ISPH.cuh:83-97 and clc_num_cells
 * (functions_NNPS.cuh:533-546): x/y/z min-max over records 0..n-2 exactly as
 * find_minmax (function_init.cuh:678-708) does, dcell = 1.1*kappa*h_ref[0]/2,
 * NI/NJ/NK and num_cells = NI*NJ*NK+1.  Also sets num_part and num_part2. */
int sph_domain_setup(sph_params *p, const sph_part1 *P1, int num_part);

/* Creates a context for num_part2 records on `device`, in `precision`
 * (SPH_PREC_*), ordered on `stream` (a cudaStream_t, NULL = default). */
int sph_create(const sph_params *p, int precision, int device, void *stream, sph_ctx **out);
void sph_destroy(sph_ctx *ctx);

/* Replaces the parameters (dt, time, flags); grid fields must not change. */
int sph_set_params(sph_ctx *ctx, const sph_params *p);

/* Uploads AoS records (the reference's DHP1 after
 * c_initial_inner_outer_particle_single, ISPH_Calc.cuh:386-387, or its
 * dev_P1 / dev_P2 copies): P1 and P2 may point to host memory (pageable or
 * pinned) or to device memory of the context's device.  P2 may be NULL
 * (zeroed as at ISPH_Calc.cuh:357).  Resets the step counter to vii[count].
 * With device records the call waits for its stream once (to learn the
 * records' p_type classes). */
int sph_upload(sph_ctx *ctx, const sph_part1 *P1, const sph_part2 *P2, int n);

/* Same as sph_upload for state that is already sorted by an earlier
 * sph_nnps of this context: only the time-varying fields are replaced and the
 * neighbour structures are kept. */
int sph_upload_state(sph_ctx *ctx, const sph_part1 *P1, int n);

/* Downloads the state in the reference layout: P1 (= dev_P1 after the step),
 * P2 (= dev_SP2), P3 (= dev_P3), to host memory or to device memory of the
 * context's device.  Any pointer may be NULL.  Synchronises. */
int sph_download(sph_ctx *ctx, sph_part1 *P1, sph_part2 *P2, sph_part3 *P3);

/* NNPS, ISPH_Calc.cuh:20-45: set_ncell, cell hash, stable sort, cell
 * start/end, reorder, plus the compacted neighbour lists every later pass
 * reads.  Runs automatically at the first step. */
int sph_nnps(sph_ctx *ctx);

/* Copies the NNPS arrays to host buffers: g_idx/p_idx [num_part2],
 * g_str/g_end [num_cells+1] in the reference's conventions (g_str = -1 for an
 * empty cell; g_end of an empty cell is left 0).  Any pointer may be NULL. */
int sph_nnps_export(sph_ctx *ctx, int32_t *g_idx, int32_t *p_idx, int32_t *g_str, int32_t *g_end);

/* Canonical neighbour list of every particle i (sorted index): all j, in the
 * reference's visit order (z, y, x cells ascending around the cell
 * floor((x-xmin)/dcell), j ascending within a cell, functions_PPE.cuh:52-72),
 * with sqrt(r2) < search_kappa*max(h_i,h_j) in FP32 (functions_PPE.cuh:96-100).
 * If `list` is NULL only *nnz and `offsets` are written. */
int sph_neighbors_export(sph_ctx *ctx, int64_t *offsets, int32_t *list, int64_t *nnz);

/* Interaction phase, ISPH_Calc.cuh:65-127: correction matrix, prep/LES,
 * no-slip walls, MOST, (step 0) Neumann, advection forces, predictor,
 * periodic and free-slip buffers. */
int sph_interaction(sph_ctx *ctx);

/* Pressure phase, ISPH_Calc.cuh:137-154: PPE in p->ppe_mode, then Neumann
 * wall pressure and the outlet copy.  `stats` may be NULL. */
int sph_ppe(sph_ctx *ctx, sph_ppe_stats *stats);

/* Time-update phase, ISPH_Calc.cuh:160-214: pressure force, IBM force and
 * spreading, corrector, IBM corrector, boundary passes on the new state;
 * advances count and time. */
int sph_time_update(sph_ctx *ctx);

/* nsteps full steps (interaction + ppe + time update).  `stats` receives the
 * last step's PPE statistics. */
int sph_step(sph_ctx *ctx, int nsteps, sph_ppe_stats *stats);

/* Diagnostics of ISPH_Calc.cuh:500-514 (kernel_copy_max + CUB Max):
 * max |u|, max |rho-rho_ref|/rho_ref*100 and max |ftotal|. */
int sph_diagnostics(sph_ctx *ctx, float *max_umag, float *max_drho_pct, float *max_ftotal);

/* Device-time breakdown of the last step in milliseconds, one entry per
 * phase: [0] nnps, [1] interaction, [2] ppe, [3] time update. */
int sph_last_phase_ms(sph_ctx *ctx, float *ms4);

/* Kernel launches issued by this context since creation (a replay of the
 * whole-step graph counts the launches it stands for, its solve as one). */
int64_t sph_launch_count(sph_ctx *ctx);

/* Sizes of the pressure operator of the current neighbour lists:
 * counts[0] rows (records), [1] stored entries of the fluid rows, [2]
 * Neumann rows, [3] their weight entries, [4] NNPS cells, [5] 1 when the
 * operator reads 16-bit neighbour codes, 0 when 32-bit indices. */
int sph_operator_counts(sph_ctx *ctx, int64_t counts[6]);

/* Steps this context ran as a replay of its whole-step graph
 * (ppe_refinement = 4). */
int64_t sph_step_graph_count(sph_ctx *ctx);

/* Live timing of the PPE operator kernel (the dominant kernel of a step):
 * with `enable` set, every operator launch is bracketed by CUDA events on the
 * context's stream.  sph_operator_stats returns the launches timed since the
 * last reset, their summed device time, and the algorithmic bytes of one
 * launch (per row: kind, list length, x_i, y_i, and component id and A_i
 * when the rank-one term is on; per 32 rows the slice offset; per stored
 * neighbour: index and coefficient; the gathered x_j are not counted).
 * `reset` clears the counters after reading. */
int sph_profile(sph_ctx *ctx, int enable);
/* Threads per block of the per-step pair passes (prep, no-slip walls,
 * advection, pressure force): 32, 64 or 128 (default).  No counterpart in
 * the reference (128 threads per block everywhere, ISPH_Calc.cuh:12).  The
 * results do not depend on it. */
int sph_set_pair_block(sph_ctx *ctx, int threads);
int sph_operator_stats(sph_ctx *ctx, int64_t *launches, double *total_ms, double *bytes_per_launch, int reset);
/* Algorithmic bytes of one operator launch in two accountings: `stored` is
 * the figure of sph_operator_stats (what the launch's layout streams,
 * including the cached coefficients and code tables); `index_rule` counts
 * per row the fields read and written for it, per slice its offset and 4
 * bytes per stored neighbour index (SELL and Neumann rows), and no stored
 * coefficient.  Either pointer may be NULL. */
int sph_operator_bytes(sph_ctx *ctx, double *stored, double *index_rule);

/* ---- files in the reference's formats (host code) -------------------------
 * sph_read_deck reads a particle deck in the format of read_input
 * (function_init.cuh:550-676): a line of tab-separated variable codes, then
 * one value per code and record; records get i_type 1.  With out = NULL and
 * capacity 0 it only counts.  sph_write_vtk writes the legacy binary VTK of
 * save_vtk_bin_single_flag (functions_OUTPUT.cuh:121-616) for the records
 * with i_type 1 or 2, one FIELD array per label (the reference's labels and
 * prefix matching); P2 / P3 may be NULL unless a label needs them. */
int sph_read_deck(const char *path, sph_part1 *out, int capacity, int *n);
/* The solver input of read_solv_input (function_init.cuh:166-463) into
 * p->vii / p->vif: the slots it sets and the switches it clears, the other
 * slots as the caller left them.  atmospheric-stability, terrain-type and
 * BAPR_frequency are read but, as in the reference (whose parser writes them
 * to the host shadow of the constant table, overwritten at
 * ISPH_Calc.cuh:366), change nothing.  plot-variables labels go to
 * plot_labels (20 x 20 chars, may be NULL), their count to *n_labels. */
int sph_read_solv(const char *path, sph_params *p, char *plot_labels, int *n_labels);

/* ---- property tables: host_Tab_* / host_table_index / host_table_size ----
 * (SOPHIA_gpu.cu:51-78, table_size 50 of Parameters.cuh:66).  Table t holds
 * entries index[t] .. index[t] + size[t] - 1 of each column and belongs to
 * the records with |p_type| = t. */
#define SPH_TABLE_SIZE  50
#define SPH_TABLE_SLOTS 10
typedef struct sph_prop_tables {
    int32_t n_tables;                 /* number_of_tables                     */
    int32_t n_data;                   /* data_numbers: entries in use          */
    int32_t index[SPH_TABLE_SLOTS];   /* host_table_index (0 past n_tables)    */
    int32_t size[SPH_TABLE_SLOTS];    /* host_table_size (0 past n_tables)     */
    double T[SPH_TABLE_SIZE], h[SPH_TABLE_SIZE], k[SPH_TABLE_SIZE];
    double cp[SPH_TABLE_SIZE], mu[SPH_TABLE_SIZE];   /* unset entries 0      */
} sph_prop_tables;                    /* 2088 bytes */

/* read_table (function_init.cuh:724-905), the file the reference reads as
 * input/data.txt (SOPHIA_gpu.cu:127-132): lines of at most 999 characters;
 * a line whose first space-separated token begins with `#p_type` opens table
 * number atoi(next token); inside it, a line whose first token begins with
 * `//T`, `//h`, `//k`, `//c` or `//m` (the reference compares three
 * characters of //T, //h, //k, //cp, //mu) is followed by one line of
 * comma-separated values (atof of every token, so a trailing comma adds a
 * 0), and a line beginning `#end` closes the table; other lines are skipped.
 * Every table's size is the value count of its last column line and the
 * tables are laid end to end in file order.  Where the reference's arrays or
 * arithmetic would be undefined the call returns SPH_ERR_BAD_ARG: a table
 * number other than 0, 1, 2, ... in file order (index and size come from the
 * cumulative counts of tables 0 .. n-1), more than SPH_TABLE_SLOTS tables, a
 * table with no column line or with column lines of different lengths, more
 * than SPH_TABLE_SIZE entries in all, a table left open at the end of the
 * file, or `#p_type` with no number. */
int sph_read_table(const char *path, sph_prop_tables *out);

/* The upload of the tables (ISPH_Calc.cuh:370-377) to the context, rounded
 * to its precision.  With vii[prop_table] = 1 (and con_solve = 1,
 * enthalpy_eqn = 1) the projection's htoT interpolates table |p_type| (h to
 * T, functions_PROP.cuh:43-67 with interp2 of :8-41) instead of the built-in
 * corium table; a step then needs tables set, and every record the
 * projection reaches (i_type < 3, p_type < 1000) needs |p_type| below
 * SPH_TABLE_SLOTS with a table of at least two entries (SPH_ERR_BAD_ARG
 * otherwise).  Rejected: sizes outside 0..SPH_TABLE_SIZE, an index + size
 * past SPH_TABLE_SIZE. */
int sph_set_prop_tables(sph_ctx *ctx, const sph_prop_tables *t);

/* The energy conversions of functions_ENERGY.cuh on the context's current
 * records, every record but i_type 3: to_enthalpy = 1 is
 * KERNEL_clc_TemptoEnthalpy (:3-12), enthalpy = enthalpy0 = Ttoh(temp,
 * p_type), the start-up pass the reference keeps commented out before its
 * time loop (ISPH_Calc.cuh:480-482); to_enthalpy = 0 is
 * KERNEL_clc_EnthalpytoTemp (:15-25), temp = htoT(enthalpy, p_type).  Ttoh
 * and htoT (functions_PROP.cuh:43-93) read the built-in corium table, or
 * with vii[prop_table] = 1 table |p_type| of sph_set_prop_tables (needed
 * then); a record whose |p_type| has no table of two entries keeps its value
 * (the reference reads past its arrays there).  Call after sph_upload;
 * asynchronous on the context's stream. */
int sph_energy_convert(sph_ctx *ctx, int to_enthalpy);
/* The host pass the reference runs on deck records before upload
 * (c_initial_inner_outer_particle_single, functions_NNPS.cuh:196-373), in
 * place: i_type 1, buffer_type 0, m_ref = m, uy = uz = 0, temp 300,
 * ux = p->profile_z/u table at z, k_turb = the k table at z (k_table = n_k
 * heights then n_k values; NULL = the reference's Case-H table,
 * functions_NNPS.cuh:156-171), p_type 3 -> 1, rho 1.225 for p_type 0 and
 * 1000, and with vii[open_boundary] > 0 the buffer classes of p_type +-1
 * against p->l2, p->l3, l4, p->l_left, p->l_right and l_ceiling
 * (functions_NNPS.cuh:5-11: 2210 and 1.910).  In 3-D ux is zeroed below
 * z = 0 and for p_type other than +-1. */
int sph_initial_records(const sph_params *p, sph_part1 *P1, int n, const double *k_table, int n_k,
                        double l4, double l_ceiling);
int sph_write_vtk(const char *path, const sph_part1 *P1, const sph_part2 *P2, const sph_part3 *P3, int n,
                  const char *const *labels, int nlabels);

/* ---- several IBM obstacles ------------------------------------------------
 * The reference hard-wires one IB box (functions_PREP.cuh:958-963, here
 * params.ib_box).  For decks with several obstacles, nbox boxes
 * (x0, x1, y0, y1, z0, z1 each) replace it in the marker normals, which are
 * computed at step 0 (set the boxes before the first step); nbox = 0 goes
 * back to params.ib_box. */
int sph_set_ib_boxes(sph_ctx *ctx, const double *boxes, int nbox);

/* ---- adaptive particle refinement ----------------------------------------
 * One pass of the reference's cell-based 3-D APR, which the shipped reference
 * does not compile (KERNEL_APR_condition3D_cell, functions_APR.cuh:270-403;
 * Cell_index, functions_APR_etc.cuh:5-20; KERNEL_cell_APR_3D,
 * functions_APR.cuh:406-652).  Per cell, the first particle whose target
 * level M exceeds its level log(m_ref/m)/log(8) by >= 0.75 splits into eight
 * children (m/8, vol/8, h/2 with vii[36], its family) written from 8 records
 * past the first free dummy record (i_type 3) the deck reserves; the parent
 * becomes a dummy.  Otherwise a complete family of eight whose members
 * exceed M by more than 0.3 merges into one record (sums of m and vol, means
 * of position, velocity and pressure, h = h_ref cbrt(m/m_ref) with vii[36];
 * the reference's 2-D merge, KERNEL_cell_APR_2D, functions_APR.cuh:119-186,
 * in 3-D) written to the tail records.  M is apr_max_level for fluid in NNPS
 * cells within apr_zone of an IBM marker's cell, 0 elsewhere; families (the
 * reference's blood_index) start as record index + 1 at the first pass.
 * Runs by itself every vii[37] steps when vii[35] = 1.  *n_split: cells
 * split; *n_wanted: cells that asked (more than the free records allow when
 * larger).  The next step rebuilds NNPS and the operators. */
int sph_apr(sph_ctx *ctx, int32_t *n_split, int32_t *n_wanted);
/* The APR state per record in the current (sorted) order: family (the
 * reference's blood_index; 0 before the first pass) and target level (its
 * M_num), and the families merged by the last pass.  Any pointer may be
 * NULL.  Synchronises. */
int sph_apr_state(sph_ctx *ctx, int32_t *family, float *target, int32_t *n_merged);

/* ---- learned warm start of the pressure solve -----------------------------
 * No counterpart in the reference (it runs one pressure sweep per step).  A
 * per-particle MLP, 20 features -> 64 -> 64 -> 1 with ReLU, predicts the
 * pressure change of the step; in SPH_PPE_LEARNED the Krylov solve starts
 * from p_old + prediction and still runs to ppe_tol.  Features per fluid
 * row (BF16, stored 32 per row, columns 20..31 zero): with r = b - M p_old
 * on the fluid rows and d = r / A_i, the scaled d_i, r_i, b_i, p_i - mean p,
 * then for each of those four: the c_ij/A_i-weighted neighbour mean, the
 * weighted mean absolute deviation, the neighbour max and min.  Scales are
 * the RMS values over the fluid rows; the target is (p_new - p_old) / RMS(d).
 * Parameters (SPH_ML_NPARAM floats): W1[20][64], b1[64], W2[64][64], b2[64],
 * w3[64], b3.  Inference: tensor cores (BF16 operands, FP32 accumulation);
 * training: FP32 forward/backward and Adam on the GPU. */
#define SPH_ML_NFEAT   20
#define SPH_ML_NPARAM  5569
/* Collect training samples from every later converged solve: every `every`-th
 * fluid row (offset rotating per step), features and target; 0 stops.  At
 * most 2^21 samples are kept. */
int sph_ml_collect(sph_ctx *ctx, int every);
/* Copies samples [first, first+rows) to host (X: rows x 32 BF16 bit
 * patterns, target: rows floats; either may be NULL) and the count. */
int sph_ml_samples(sph_ctx *ctx, int64_t first, int64_t rows, uint16_t *X, float *target, int64_t *count);
/* Adam on the collected samples (mini-batches of `batch`, `epochs` passes,
 * learning rate `lr`, shuffling and initial weights from `seed` unless
 * weights were set); *final_loss = mean squared error on up to 65536 samples. */
int sph_ml_train(sph_ctx *ctx, int epochs, int batch, float lr, uint64_t seed, float *final_loss);
int sph_ml_set_weights(sph_ctx *ctx, const float *w);
int sph_ml_get_weights(sph_ctx *ctx, float *w);
/* Mean squared error and its gradient (FP32, SPH_ML_NPARAM floats) over
 * samples [first, first+rows), with the current weights. */
int sph_ml_grad(sph_ctx *ctx, int64_t first, int32_t rows, float *loss, float *grad);
/* Tensor-core predictions for samples [first, first+rows). */
int sph_ml_predict_samples(sph_ctx *ctx, int64_t first, int32_t rows, float *y);

/* ---- ensembles of independent cases ---------------------------------------
 * No counterpart in the reference (one case per run there).  A batch holds
 * one context per case, each on its own non-blocking stream of `device`;
 * sph_batch_step advances every case by nsteps with a pool of host workers
 * that take cases largest first, so the kernels of many small cases run on
 * the GPU side by side.  Results are those of stepping each case alone. */
typedef struct sph_batch sph_batch;
/* P1[k] holds n[k] records of case k, params[k] its parameters (after
 * sph_domain_setup). */
int sph_batch_create(int ncase, const sph_params *params, const sph_part1 *const *P1, const int32_t *n, int precision,
                     int device, sph_batch **out);
void sph_batch_destroy(sph_batch *b);
/* nsteps steps of every case; stats[k] (may be NULL) gets case k's last PPE
 * statistics.  Returns the most severe status over the cases. */
int sph_batch_step(sph_batch *b, int nsteps, sph_ppe_stats *stats);
/* Cases in flight at once (0: all).  sph_batch_autotune times probe_steps
 * steps of every case at 1, 2, 4, ... and all workers, keeps the fastest and
 * reports it (the probe steps advance the cases). */
int sph_batch_set_workers(sph_batch *b, int workers);
int sph_batch_autotune(sph_batch *b, int probe_steps, int *workers, double *ms_per_step);
/* sph_batch_autotune, then the thread-block size of the per-step pair passes
 * (128, 64 or 32 threads, the same for every case) from probe steps at the
 * chosen worker count; keeps and reports the fastest of both. */
int sph_batch_autotune_shapes(sph_batch *b, int probe_steps, int *workers, int *pair_block, double *ms_per_step);
/* The context of case k (owned by the batch), e.g. for sph_download. */
int sph_batch_case(sph_batch *b, int k, sph_ctx **ctx);
int64_t sph_batch_particles(sph_batch *b);

/* ---- cell sort without device allocation --------------------------------
 * No counterpart in the reference: an addition for callers that cannot call
 * cudaMalloc, such as a host code that gives all of its device memory to its
 * own pool or arena, or one whose time loop must not allocate once it runs.
 * It does what sph_nnps + sph_nnps_export do for the cell hash and sort
 * (KERNEL_index_particle_to_cell and the stable sort by cell), for n
 * particles given as device arrays in their original order, and writes
 * g_idx, p_idx (n each) and g_str, g_end (num_cells + 1 each) to device
 * arrays the caller owns.  `params` needs the cell grid of
 * sph_domain_setup; i_type 3 marks dummies (key num_cells).  `stream` is a
 * cudaStream_t (NULL: the legacy default stream).
 *
 * The working memory is one static device array per GPU, about 9.5 MB,
 * which every GPU that loads this library holds until the process exits.
 * Limits: n <= SPH_NOALLOC_MAX_PARTICLES and num_cells + 2 <=
 * SPH_NOALLOC_MAX_CELLS; larger inputs return SPH_ERR_BAD_ARG.  The first
 * call on a device looks up that array's device address.  All calls on a
 * device share the array: calls that overlap on the GPU (other streams,
 * other host threads) race.  Every call ends by copying two flags to host
 * memory and waiting for its stream, to report a cell of more than 4096
 * particles (SPH_ERR_UNSUPPORTED); so do not make it while any stream of the
 * device is being captured into a CUDA graph.  It calls no cudaMalloc or
 * cudaFree. */
#define SPH_NOALLOC_MAX_PARTICLES 262144
#define SPH_NOALLOC_MAX_CELLS     524288
int sph_nnps_sort_noalloc(const sph_params *params, const float *d_x, const float *d_y, const float *d_z,
                          const int32_t *d_i_type, int32_t n, int32_t *d_g_idx, int32_t *d_p_idx,
                          int32_t *d_g_str, int32_t *d_g_end, void *stream);

const char *sph_status_string(int status);

/* Text of the last error raised on the calling host thread. */
const char *sph_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* SPH_ISPH_H */
