// sophia_b200 -- the reference's program (SOPHIA_gpu.cu main, ISPH, ISPH_Calc)
// as a thin native driver of the C ABI in include/sph_isph.h.
//
//   sophia_b200 solv.txt deck.txt out_dir [--steps N] [--fp64] [--table data.txt]
//               [--enthalpy] [--setup-only] [solver options]
//
// Solver options (settings the solver input cannot carry):
//   --ppe sweep|bicgstab|mixed|gmres|idrs   pressure solve (default mixed)
//   --tol X                                  its relative residual (default 1e-6)
//   --coarse B                               two-level preconditioner on B^3-cell
//                                            blocks; -B balanced by row count
//   --coarse-max M                           most balanced aggregates
//   --coef-half                              FP16 row-scaled coefficients
//   --device-control                         each solve one graph under device control
//   --pair-h                                 pair-averaged h in the pressure rows
//   --pforce-difference                      difference form of the pressure force
//
// What the reference does, and where:
//   * main (SOPHIA_gpu.cu:120-141): read_solv_input on the solver input, then
//     read_table on ./input/data.txt.  Here the tables are read when the
//     solver input sets property_table YES (the only case in which the step
//     reads them): from --table, else data.txt beside the solver input.
//   * ISPH (ISPH.cuh:53-125): read the particle deck (read_input), find the
//     domain and the cell grid, reserve buffersize * num_part extra records
//     (i_type 3) when APR is on (ISPH.cuh:116).
//   * ISPH_Calc (ISPH_Calc.cuh:239-528): the host record pass
//     (c_initial_inner_outer_particle_single, :386), the step counter from
//     floor(time / dt + 0.5) (:256), then steps until time >= time_end,
//     writing the binary VTK fluid_<count>stp.vtk after every step whose
//     counter (before its increment) is a multiple of freq_output, and the
//     max |u| / max |ftotal| lines every freq_output steps.
//   * --enthalpy: the energy equation in enthalpy (the reference's
//     compile-time enthalpy_eqn); the records' enthalpy is then set from their
//     temperature after the upload (KERNEL_clc_TemptoEnthalpy, the start-up
//     pass ISPH_Calc.cuh:480-482 keeps commented out), since decks carry
//     temperatures only.
//   * --setup-only: everything up to the device context, then one line
//     describing the case (for checks without a GPU).
// Settings the solver input does not carry (the PPE solver form, the
// wall-model constants, the inflow profile) are sph_params_init's.
#include <sys/stat.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "sph_isph.h"

namespace {

// the Case-H buffer planes the host record pass reads (functions_NNPS.cuh:7,11)
const double kCaseHL4 = 2210.0;
const double kCaseHLCeiling = 1.910;

struct Args {
    std::string solv, deck, out, table;
    long long steps = -1;
    bool fp64 = false, enthalpy = false, setup_only = false;
    int ppe = -1, coarse = 0, coarse_max = 0;
    double tol = 0;
    bool coef_half = false, device_control = false, pair_h = false, pforce_difference = false;
};

int ppe_mode_of(const std::string &s) {
    if (s == "sweep") return SPH_PPE_REF_SWEEP;
    if (s == "bicgstab") return SPH_PPE_BICGSTAB;
    if (s == "mixed") return SPH_PPE_MIXED_IR;
    if (s == "gmres") return SPH_PPE_GMRES;
    if (s == "idrs") return SPH_PPE_IDRS;
    return -1;
}

int usage() {
    fprintf(stderr,
            "usage: sophia_b200 solv.txt deck.txt out_dir [--steps N] [--fp64] [--table data.txt] [--enthalpy] "
            "[--setup-only]\n"
            "       [--ppe sweep|bicgstab|mixed|gmres|idrs] [--tol X] [--coarse B] [--coarse-max M] [--coef-half]\n"
            "       [--device-control] [--pair-h] [--pforce-difference]\n");
    return 2;
}

bool parse(int argc, char **argv, Args &a) {
    std::vector<std::string> pos;
    for (int k = 1; k < argc; ++k) {
        const std::string s = argv[k];
        if (s == "--steps" && k + 1 < argc) a.steps = atoll(argv[++k]);
        else if (s == "--table" && k + 1 < argc) a.table = argv[++k];
        else if (s == "--fp64") a.fp64 = true;
        else if (s == "--enthalpy") a.enthalpy = true;
        else if (s == "--setup-only") a.setup_only = true;
        else if (s == "--ppe" && k + 1 < argc) {
            a.ppe = ppe_mode_of(argv[++k]);
            if (a.ppe < 0) return false;
        }
        else if (s == "--tol" && k + 1 < argc) a.tol = atof(argv[++k]);
        else if (s == "--coarse" && k + 1 < argc) a.coarse = atoi(argv[++k]);
        else if (s == "--coarse-max" && k + 1 < argc) a.coarse_max = atoi(argv[++k]);
        else if (s == "--coef-half") a.coef_half = true;
        else if (s == "--device-control") a.device_control = true;
        else if (s == "--pair-h") a.pair_h = true;
        else if (s == "--pforce-difference") a.pforce_difference = true;
        else if (!s.empty() && s[0] == '-') return false;
        else pos.push_back(s);
    }
    if (pos.size() != 3) return false;
    a.solv = pos[0];
    a.deck = pos[1];
    a.out = pos[2];
    return true;
}

int fail(const char *what, int st) {
    fprintf(stderr, "sophia_b200: %s: %s (%s)\n", what, sph_status_string(st), sph_last_error());
    return 1;
}

std::string dir_of(const std::string &path) {
    const size_t k = path.find_last_of('/');
    return k == std::string::npos ? std::string(".") : path.substr(0, k);
}

bool exists(const std::string &path) {
    struct stat sb;
    return stat(path.c_str(), &sb) == 0;
}

}  // namespace

int main(int argc, char **argv) {
    Args a;
    if (!parse(argc, argv, a)) return usage();

    // ---- solver input (main) -------------------------------------------------
    sph_params p;
    sph_params_init(&p);
    if (a.enthalpy) p.enthalpy_eqn = 1;
    if (a.ppe >= 0) p.ppe_mode = a.ppe;
    if (a.tol > 0) p.ppe_tol = a.tol;
    p.ppe_coarse_block = a.coarse;
    p.ppe_coarse_max = a.coarse_max;
    if (a.coef_half) p.ppe_coef_half = 1;
    if (a.device_control) p.ppe_refinement = 4;
    if (a.pair_h) p.ppe_pair_h = 1;
    if (a.pforce_difference) p.pressure_force_form = 1;
    char labels_buf[20 * 20] = {0};
    int nlab = 0;
    int st = sph_read_solv(a.solv.c_str(), &p, labels_buf, &nlab);
    if (st < 0) return fail("solver input", st);
    if (nlab > 20) nlab = 20;
    std::vector<const char *> labels;
    for (int k = 0; k < nlab; ++k) labels.push_back(labels_buf + 20 * k);

    sph_prop_tables tables;
    const bool use_tables = p.vii[SPH_VII_PROP_TABLE] == 1;
    if (use_tables) {
        const std::string path = a.table.empty() ? dir_of(a.solv) + "/data.txt" : a.table;
        if (!exists(path)) {
            fprintf(stderr, "sophia_b200: property_table YES needs the table file %s\n", path.c_str());
            return 1;
        }
        st = sph_read_table(path.c_str(), &tables);
        if (st < 0) return fail("property tables", st);
    }

    // ---- particle deck, domain, host record pass, APR headroom (ISPH) -----------
    int n = 0;
    st = sph_read_deck(a.deck.c_str(), nullptr, 0, &n);
    if (st < 0) return fail("particle deck", st);
    if (n <= 0) { fprintf(stderr, "sophia_b200: the deck holds no records\n"); return 1; }
    std::vector<sph_part1> P(n);
    st = sph_read_deck(a.deck.c_str(), P.data(), n, &n);
    if (st < 0) return fail("particle deck", st);
    st = sph_domain_setup(&p, P.data(), n);
    if (st < 0) return fail("domain set-up", st);
    st = sph_initial_records(&p, P.data(), n, nullptr, 0, kCaseHL4, kCaseHLCeiling);
    if (st < 0) return fail("host record pass", st);
    const int extra = p.vii[SPH_VII_APR_SOLV] ? (int)((double)p.vif[SPH_VIF_BUFFERSIZE] * n) : 0;
    if (extra > 0) {
        sph_part1 d;
        memset(&d, 0, sizeof(d));
        d.i_type = 3;
        d.x = P[0].x; d.y = P[0].y; d.z = P[0].z;
        d.h = P[0].h; d.h_ref = P[0].h_ref; d.m = P[0].m; d.m_ref = P[0].m_ref;
        d.rho = P[0].rho; d.vol = P[0].vol;
        P.resize((size_t)n + extra, d);
    }
    p.vii[SPH_VII_NUM_PART] = n;
    p.vii[SPH_VII_NUM_PART2] = (int)P.size();
    const float dt = p.vif[SPH_VIF_DT];
    float t = p.vif[SPH_VIF_TIME];
    const float t_end = p.vif[SPH_VIF_TIME_END];
    long long count = (long long)std::floor((double)(t / dt) + 0.5);   // ISPH_Calc.cuh:256
    p.vii[SPH_VII_COUNT] = (int)count;

    if (a.setup_only) {
        printf("{\"num_part\": %d, \"num_part2\": %d, \"count\": %lld, \"NI\": %d, \"NJ\": %d, \"NK\": %d, "
               "\"num_cells\": %d, \"dcell\": %.9g, \"labels\": %d, \"tables\": %d, \"prop_table\": %d, "
               "\"ppe_mode\": %d, \"ppe_tol\": %.17g, \"ppe_coarse_block\": %d, \"ppe_coarse_max\": %d, "
               "\"ppe_coef_half\": %d, \"ppe_refinement\": %d, \"ppe_pair_h\": %d, \"pressure_force_form\": %d, "
               "\"enthalpy_eqn\": %d}\n",
               n, p.vii[SPH_VII_NUM_PART2], count, p.vii[SPH_VII_NI], p.vii[SPH_VII_NJ], p.vii[SPH_VII_NK],
               p.vii[SPH_VII_NUM_CELLS], (double)p.vif[SPH_VIF_DCELL], nlab, use_tables ? tables.n_tables : 0,
               p.vii[SPH_VII_PROP_TABLE], p.ppe_mode, p.ppe_tol, p.ppe_coarse_block, p.ppe_coarse_max,
               p.ppe_coef_half, p.ppe_refinement, p.ppe_pair_h, p.pressure_force_form, p.enthalpy_eqn);
        return 0;
    }

    // ---- device context and the time loop (ISPH_Calc) ---------------------------
    mkdir(a.out.c_str(), 0755);
    sph_ctx *ctx = nullptr;
    st = sph_create(&p, a.fp64 ? SPH_PREC_FP64 : SPH_PREC_MIXED, 0, nullptr, &ctx);
    if (st < 0) return fail("context", st);
    int rc = 0;
    const int freq = p.vii[SPH_VII_FREQ_OUTPUT] > 0 ? p.vii[SPH_VII_FREQ_OUTPUT] : 1;
    const int N2 = (int)P.size();
    std::vector<sph_part1> Q1(N2);
    std::vector<sph_part2> Q2(N2);
    std::vector<sph_part3> Q3(N2);
    const auto wall0 = std::chrono::steady_clock::now();
    long long steps = 0;
    do {
        if (use_tables && (st = sph_set_prop_tables(ctx, &tables)) < 0) { rc = fail("property tables", st); break; }
        if ((st = sph_upload(ctx, P.data(), nullptr, N2)) < 0) { rc = fail("upload", st); break; }
        if (p.enthalpy_eqn && p.vii[SPH_VII_CON_SOLVE] == 1 && (st = sph_energy_convert(ctx, 1)) < 0) {
            rc = fail("enthalpy from temperature", st);
            break;
        }
        for (;;) {
            sph_ppe_stats ps;
            st = sph_step(ctx, 1, &ps);
            if (st < 0) { rc = fail("step", st); break; }
            if (count % freq == 0) {
                if ((st = sph_download(ctx, Q1.data(), Q2.data(), Q3.data())) < 0) { rc = fail("download", st); break; }
                const std::string vtk = a.out + "/fluid_" + std::to_string(count) + "stp.vtk";
                st = sph_write_vtk(vtk.c_str(), Q1.data(), Q2.data(), Q3.data(), N2, labels.data(), (int)labels.size());
                if (st < 0) { rc = fail("VTK output", st); break; }
            }
            t = t + dt;
            ++count;
            ++steps;
            if (count % freq == 0) {
                float umax = 0, drho = 0, fmax = 0;
                if ((st = sph_diagnostics(ctx, &umax, &drho, &fmax)) < 0) { rc = fail("diagnostics", st); break; }
                const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - wall0).count();
                printf("Simulation time: %5.2f sec\n", (double)t);
                printf("Computing time: %5.2f sec\n", wall);
                printf("%lld\t tu_max=%5.2f\tftotal_max=%5.5f\n", count, (double)umax, (double)fmax);
                fflush(stdout);
            }
            if (t >= t_end || (a.steps >= 0 && steps >= a.steps)) break;
        }
    } while (false);
    sph_destroy(ctx);
    return rc;
}
