// Particle-deck reader and VTK writer in the reference's file formats, so
// the B200 step reads the authors' decks and writes the files their
// post-processing reads (host code; no device work).
//
//   deck (read_input, function_init.cuh:550-676): a first line of
//     tab-separated variable codes (1 x, 2 y, 3 z, 4-6 ux..uz, 7 m, 8 p_type,
//     9 h, 10 temp, 11 pres, 12 rho, 15 concn, 26 h0, 27 m0; the other codes
//     are read and ignored), then one whitespace-separated value per code
//     and record; every record gets i_type 1.
//   VTK (save_vtk_bin_single_flag, functions_OUTPUT.cuh:121-616): legacy
//     binary POLYDATA, big-endian, the records with i_type 1 or 2 as POINTS
//     and one FIELD array per requested label, each label selecting the
//     reference's arrays by the same prefix comparisons in the same order
//     (a label can select more than one array, as "rho_ref" selects rho and
//     rho_ref there; the FIELD count is the number of labels, as there).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"

namespace {

float be_float(float f) {
    unsigned char b[4], o[4];
    memcpy(b, &f, 4);
    o[0] = b[3]; o[1] = b[2]; o[2] = b[1]; o[3] = b[0];
    float r;
    memcpy(&r, o, 4);
    return r;
}

int be_int(int d) {
    unsigned char b[4], o[4];
    memcpy(b, &d, 4);
    o[0] = b[3]; o[1] = b[2]; o[2] = b[1]; o[3] = b[0];
    int r;
    memcpy(&r, o, 4);
    return r;
}

}  // namespace

extern "C" int sph_read_deck(const char *path, sph_part1 *out, int capacity, int *n) {
    using namespace sph;
    if (!path || !n || (out == nullptr && capacity != 0)) return SPH_ERR_BAD_ARG;
    FILE *f = fopen(path, "r");
    if (!f) { set_error("sph_read_deck: cannot open the deck"); return SPH_ERR_BAD_ARG; }
    char line[4096];
    if (!fgets(line, sizeof line, f)) { fclose(f); set_error("sph_read_deck: empty deck"); return SPH_ERR_BAD_ARG; }
    std::vector<int> codes;
    for (char *tok = strtok(line, "\t"); tok; tok = strtok(nullptr, "\t")) codes.push_back(atoi(tok));
    if (codes.empty()) { fclose(f); set_error("sph_read_deck: no variable codes"); return SPH_ERR_BAD_ARG; }
    char buf[1024];
    int nop = 0, st = SPH_OK;
    for (;;) {
        sph_part1 rec;
        memset(&rec, 0, sizeof rec);
        bool complete = true;
        for (size_t v = 0; v < codes.size(); ++v) {
            if (fscanf(f, "%1023s", buf) != 1) { complete = false; break; }
            const float fv = (float)atof(buf);
            switch (codes[v]) {
                case 1: rec.x = fv; break;
                case 2: rec.y = fv; break;
                case 3: rec.z = fv; break;
                case 4: rec.ux = fv; break;
                case 5: rec.uy = fv; break;
                case 6: rec.uz = fv; break;
                case 7: rec.m = fv; break;
                case 8: rec.p_type = atoi(buf); break;
                case 9: rec.h = fv; break;
                case 10: rec.temp = fv; break;
                case 11: rec.pres = fv; break;
                case 12: rec.rho = fv; break;
                case 15: rec.concn = fv; break;
                case 26: rec.h_ref = fv; break;
                case 27: rec.m_ref = fv; break;
                default: break;   // read and ignored, as the reference does
            }
        }
        if (!complete) break;
        rec.i_type = 1;
        if (out) {
            if (nop >= capacity) { st = SPH_ERR_BAD_ARG; set_error("sph_read_deck: more records than capacity"); break; }
            out[nop] = rec;
        }
        ++nop;
    }
    fclose(f);
    *n = nop;
    return st;
}

extern "C" int sph_write_vtk(const char *path, const sph_part1 *P1, const sph_part2 *P2, const sph_part3 *P3, int n,
                             const char *const *labels, int nlabels) {
    using namespace sph;
    if (!path || (!P1 && n > 0) || n < 0 || nlabels < 0 || (nlabels > 0 && !labels)) return SPH_ERR_BAD_ARG;
    FILE *f = fopen(path, "wb");
    if (!f) { set_error("sph_write_vtk: cannot open the output file"); return SPH_ERR_BAD_ARG; }
    std::vector<int> sel;
    for (int i = 0; i < n; ++i)
        if (P1[i].i_type == 1 || P1[i].i_type == 2) sel.push_back(i);
    const int np = (int)sel.size();
    fprintf(f, "# vtk DataFile Version 3.0\n");
    fprintf(f, "Print out results in vtk format\n");
    fprintf(f, "BINARY\n");
    fprintf(f, "DATASET POLYDATA\n");
    fprintf(f, "POINTS\t%d\tfloat\n", np);
    auto wf = [&](float v) { const float b = be_float(v); fwrite(&b, 4, 1, f); };
    auto wi = [&](int v) { const int b = be_int(v); fwrite(&b, 4, 1, f); };
    for (int i : sel) { wf(P1[i].x); wf(P1[i].y); wf(P1[i].z); }
    fprintf(f, "POINT_DATA\t%d\n", np);
    fprintf(f, "FIELD FieldData\t%d\n", nlabels);
    auto is = [](const char *label, const char *key, int k) { return strncmp(label, key, k) == 0; };
    int need = 0;   // arrays that need P2 / P3
    for (int q = 0; q < nlabels; ++q) {
        const char *L = labels[q];
        if (!L) continue;
        auto arr_i = [&](const char *name, auto get) {
            fprintf(f, "%s\t1\t%d\tint\n", name, np);
            for (int i : sel) wi(get(i));
        };
        auto arr_f = [&](const char *name, int nc, auto get) {
            fprintf(f, "%s\t%d\t%d\tfloat\n", name, nc, np);
            for (int i : sel) get(i);
        };
        if (is(L, "buffer_type", 3)) arr_i("buffer_type", [&](int i) { return P1[i].buffer_type; });
        if (is(L, "i_type", 3)) arr_i("i_type", [&](int i) { return P1[i].i_type; });
        if (is(L, "p_type", 3)) arr_i("p_type", [&](int i) { return P1[i].p_type; });
        if (is(L, "source", 5)) arr_i("source", [&](int i) { return P1[i].source; });
        if (is(L, "rho", 3)) arr_f("rho", 1, [&](int i) { wf(P1[i].rho); });
        if (is(L, "vol", 3)) arr_f("vol", 1, [&](int i) { wf(P1[i].vol); });
        if (is(L, "velocity", 4)) arr_f("velocity", 3, [&](int i) { wf(P1[i].ux); wf(P1[i].uy); wf(P1[i].uz); });
        if (is(L, "normal", 5)) {
            if (!P3) { ++need; continue; }
            arr_f("normal", 3, [&](int i) { wf(P3[i].nx); wf(P3[i].ny); wf(P3[i].nz); });
        }
        if (is(L, "b_force", 5)) arr_f("fb", 3, [&](int i) { wf(P1[i].fbx); wf(P1[i].fby); wf(P1[i].fbz); });
        if (is(L, "MOST_force", 7)) arr_f("fm", 2, [&](int i) { wf(P1[i].fmx); wf(P1[i].fmy); });
        if (is(L, "MOST_heat", 7)) arr_f("hm", 1, [&](int i) { wf(P1[i].hmz); });
        if (is(L, "pressure", 3)) arr_f("pressure", 1, [&](int i) { wf(P1[i].pres); });
        if (is(L, "vis_t", 5)) arr_f("vis_t", 1, [&](int i) { wf(P1[i].vis_t); });
        if (is(L, "temp", 3)) arr_f("temp", 1, [&](int i) { wf(P1[i].temp); });
        if (is(L, "flt_s", 3)) arr_f("flt_s", 1, [&](int i) { wf(P1[i].flt_s); });
        if (is(L, "concn", 5)) arr_f("concn", 1, [&](int i) { wf(P1[i].concn); });
        if (is(L, "concentration", 6)) arr_f("concentration", 1, [&](int i) { wf(P1[i].concentration); });
        if (is(L, "enthalpy", 4)) arr_f("enthalpy", 1, [&](int i) { wf(P1[i].enthalpy); });
        if (is(L, "mass", 4)) arr_f("mass", 1, [&](int i) { wf(P1[i].m); });
        if (is(L, "eli", 3)) arr_f("eli", 1, [&](int i) { wf(P1[i].eli); });
        if (is(L, "smoothing", 5)) arr_f("h", 1, [&](int i) { wf(P1[i].h); });
        if (is(L, "monitor", 5)) arr_f("monitor", 3, [&](int i) { wf(P1[i].float1); wf(P1[i].float2); wf(P1[i].float3); });
        if (is(L, "ncell", 5)) arr_i("ncell", [&](int i) { return P1[i].ncell; });
        if (is(L, "rho_ref", 5)) {
            if (!P2) { ++need; continue; }
            arr_f("rho_ref", 1, [&](int i) { wf(P2[i].rho_ref); });
        }
        if (is(L, "k_turb", 4)) arr_f("k_turb", 1, [&](int i) { wf(P1[i].k_turb); });
        if (is(L, "e_turb", 4)) arr_f("e_turb", 1, [&](int i) { wf(P1[i].e_turb); });
        if (is(L, "dtemp", 5)) {
            if (!P3) { ++need; continue; }
            arr_f("dtemp", 1, [&](int i) { wf(P3[i].dtemp); });
        }
    }
    fclose(f);
    if (need) { set_error("sph_write_vtk: a label needs the part2 / part3 records"); return SPH_ERR_BAD_ARG; }
    return SPH_OK;
}

// ---- solver input file -----------------------------------------------------------
// read_solv_input (function_init.cuh:166-463).  The file is a stream of
// whitespace-separated tokens.  For every token read, the keywords are tried
// in a fixed order against the CURRENT token; a keyword that matches reads
// its fixed number of tokens (the last one the value) and the later keywords
// are then tried against that value, exactly as the reference's chain of
// plain `if`s does.  A read past the end of the file leaves the token as it
// was, and the pass for the failed read still runs once before the loop
// ends, as the reference's does.
//
// Three keywords never reach the tables the step reads: function_init.cuh
// redefines atmos_stab, terrain_type (lines 133-134) and freq_bapr (line 128)
// to k_vii slots before the parser, so the parser clears and sets the host
// shadow of the __constant__ table, which the upload at ISPH_Calc.cuh:366
// then overwrites with vii.  Their tokens are read here as there (slot -1)
// and vii[40], vii[45] and vii[46] keep the caller's values.
namespace {

enum SolvKind { SOLV_INT, SOLV_FLOAT, SOLV_ENUM, SOLV_BLOCK, SOLV_LABELS };

struct SolvRule {
    const char *key;
    int tokens;          // tokens read after the keyword (the last one is the value)
    SolvKind kind;
    int slot;            // k_vii slot (INT, ENUM, BLOCK) or k_vif slot (FLOAT); -1 reads only
    const char *names;   // ENUM: "name=value" pairs, space separated
};

// Keyword order, token counts and slots of function_init.cuh:194-459.
const SolvRule kSolvRules[] = {
    {"solver_type", 2, SOLV_ENUM, 0, "WCSPH=0 ISPH=1"},
    {"dimension(1/2/3):", 1, SOLV_INT, 1, nullptr},
    {"property_table(YES/NO):", 1, SOLV_ENUM, 2, "YES=1 NO=0"},
    {"atmospheric-stability", 2, SOLV_ENUM, -1, "Unstable=0 Neutral=1 Stable=2"},
    {"terrain-type", 2, SOLV_ENUM, -1, "Flat=0 Grass=1 Forest=2 City=3 Ocean=4"},
    {"kernel", 3, SOLV_ENUM, 3, "Quartic=2 Gaussian=0 Quintic=1 Wendland2=3 Wendland4=4 Wendland6=5"},
    {"time", 3, SOLV_ENUM, 4, "Euler=0 Predictor_Corrector=1"},
    {"structure", 2, SOLV_ENUM, 44, "YES=1 NO=0"},
    {"open", 3, SOLV_ENUM, 5, "OPEN=1 PERIODIC=2 NO=0"},
    {"pressure-force", 2, SOLV_ENUM, 12, "YES=1 NO=0"},
    {"viscous-force", 2, SOLV_ENUM, 13, "NO=0 Cleary=1 Monaghan=2 Violeau=3"},
    {"turbulence-model", 2, SOLV_ENUM, 18, "Laminar=0 k-lm=1 k-e=2 HB=3 SSM=4 DDF=5"},
    {"gravitational-force", 2, SOLV_ENUM, 14, "YES=1 NO=0"},
    {"Conduction(YES/NO):", 1, SOLV_ENUM, 15, "YES=1 NO=0"},
    {"Boussinesq-natural-convection", 2, SOLV_ENUM, 16, "YES=1 NO=0"},
    {"Concentration-diffusion(YES/NO):", 1, SOLV_ENUM, 19, "YES=1 NO=0"},
    {"kernel-gradient-correction", 2, SOLV_ENUM, 17, "NO=0 KGC=1 FPM=2 DFPM=3 KGF=4"},
    {"switch_ptype", 2, SOLV_ENUM, 33, "YES=1 NO=0"},
    {"noslip_boundary", 2, SOLV_ENUM, 34, "YES=1 NO=0"},
    {"APR_solve", 2, SOLV_ENUM, 35, "Cell=1 Switch=2 Block=3 NO=0"},
    {"Block_configuration", 2, SOLV_BLOCK, 41, nullptr},
    {"Variable", 2, SOLV_ENUM, 36, "Abrupt=1 Smooth=2 NO=0"},
    {"Buffersize:", 1, SOLV_FLOAT, 19, nullptr},
    {"reference-pressure", 2, SOLV_FLOAT, 1, nullptr},
    {"kappa:", 1, SOLV_FLOAT, 0, nullptr},
    {"minimum-iteration:", 1, SOLV_INT, 20, nullptr},
    {"maximum-iteration:", 1, SOLV_INT, 21, nullptr},
    {"pressure-convergence", 2, SOLV_FLOAT, 7, nullptr},
    {"density-convergence", 2, SOLV_FLOAT, 6, nullptr},
    {"pressure-relaxation", 2, SOLV_FLOAT, 8, nullptr},
    {"time-step", 2, SOLV_FLOAT, 2, nullptr},
    {"start-time", 2, SOLV_FLOAT, 3, nullptr},
    {"end-time", 2, SOLV_FLOAT, 4, nullptr},
    {"neighbor", 4, SOLV_ENUM, 7, "3X3=0 5X5=1"},
    {"timestep", 3, SOLV_ENUM, 6, "YES=1 NO=0"},
    {"structure-timestep", 2, SOLV_FLOAT, 20, nullptr},
    {"filtering", 2, SOLV_INT, 8, nullptr},
    {"temperature-filtering", 2, SOLV_INT, 10, nullptr},
    {"plot-output", 2, SOLV_INT, 11, nullptr},
    {"APR_frequency:", 1, SOLV_INT, 37, nullptr},
    {"h-reset", 2, SOLV_INT, 38, nullptr},
    {"BAPR_frequency:", 1, SOLV_INT, -1, nullptr},
    {"plot-variables:", 1, SOLV_LABELS, 0, nullptr},
    {"velocity-limit", 2, SOLV_FLOAT, 5, nullptr},
};

// The value of `tok` in a "name=value" list, or false when it is not there.
bool solv_enum(const char *names, const char *tok, int *value) {
    const size_t n = strlen(tok);
    for (const char *q = names; *q;) {
        const char *eqs = strchr(q, '=');
        if ((size_t)(eqs - q) == n && strncmp(q, tok, n) == 0) {
            *value = atoi(eqs + 1);
            return true;
        }
        q = strchr(eqs, ' ');
        if (!q) break;
        ++q;
    }
    return false;
}

}  // namespace

extern "C" int sph_read_solv(const char *path, sph_params *p, char *plot_labels, int *n_labels) {
    using namespace sph;
    if (!path || !p) return SPH_ERR_BAD_ARG;
    FILE *f = fopen(path, "r");
    if (!f) { set_error("sph_read_solv: cannot open the solver input"); return SPH_ERR_BAD_ARG; }
    int *vii = p->vii;
    float *vif = p->vif;
    // the switches function_init.cuh:168-179 clears before reading
    vii[0] = 0;
    for (int s : {12, 13, 14, 15, 16, 17, 18, 19, 35, 44}) vii[s] = 0;
    char tok[1000];
    tok[0] = 0;
    auto next = [&]() { return fscanf(f, "%999s", tok) == 1; };
    int nlab = 0;
    for (;;) {
        const bool got = next();
        for (const SolvRule &r : kSolvRules) {
            if (strcmp(tok, r.key) != 0) continue;
            switch (r.kind) {
            case SOLV_INT:
                for (int q = 0; q < r.tokens; ++q) next();
                if (r.slot >= 0) vii[r.slot] = atoi(tok);
                break;
            case SOLV_FLOAT:
                for (int q = 0; q < r.tokens; ++q) next();
                vif[r.slot] = (float)atof(tok);
                break;
            case SOLV_ENUM: {
                for (int q = 0; q < r.tokens; ++q) next();
                int v;
                if (solv_enum(r.names, tok, &v) && r.slot >= 0) vii[r.slot] = v;
                break;
            }
            case SOLV_BLOCK:   // NBI, NBJ, NBK, each after one skipped token
                for (int d = 0; d < 3; ++d) {
                    next();
                    next();
                    vii[r.slot + d] = atoi(tok);
                }
                break;
            case SOLV_LABELS: {
                next();
                const int k = atoi(tok);
                nlab = k;
                for (int q = 0; q < k; ++q) {
                    char lab[1000];
                    if (fscanf(f, "%999s", lab) != 1) continue;
                    if (plot_labels && q < 20) {
                        strncpy(plot_labels + 20 * q, lab, 19);
                        plot_labels[20 * q + 19] = 0;
                    }
                }
                break;
            }
            }
        }
        if (!got) break;
    }
    fclose(f);
    if (n_labels) *n_labels = nlab;
    return SPH_OK;
}

// ---- property tables ------------------------------------------------------------
// read_table (function_init.cuh:724-905): fgets lines of at most 999
// characters, space-separated first tokens compared by prefix, values split
// at commas and read by atof, each table as long as its last column line, the
// tables laid end to end.  The cases the reference leaves undefined (an
// unnumbered table slot, an uninitialised count, a read past the arrays or
// past the end of the file) are errors here.
extern "C" int sph_read_table(const char *path, sph_prop_tables *out) {
    using namespace sph;
    if (!path || !out) return SPH_ERR_BAD_ARG;
    FILE *f = fopen(path, "r");
    if (!f) { set_error("sph_read_table: cannot open the property table file"); return SPH_ERR_BAD_ARG; }
    sph_prop_tables t;
    memset(&t, 0, sizeof(t));
    double *cols[5] = {t.T, t.h, t.k, t.cp, t.mu};
    const char *keys[5] = {"//T", "//h", "//k", "//c", "//m"};
    char line[1000];
    int data_numbers = 0, ntab = 0;
    int cum[SPH_TABLE_SLOTS] = {0};
    const char *err = nullptr;
    while (!err && fgets(line, sizeof(line), f)) {
        char *save = nullptr;
        char *tok = strtok_r(line, " ", &save);
        if (!tok || strncmp(tok, "#p_type", 7) != 0) continue;
        tok = strtok_r(nullptr, " ", &save);
        if (!tok) { err = "#p_type without a table number"; break; }
        const int number = atoi(tok);
        if (number != ntab) { err = "tables must be numbered 0, 1, 2, ... in file order"; break; }
        if (++ntab > SPH_TABLE_SLOTS) { err = "more than SPH_TABLE_SLOTS tables"; break; }
        int len = -1;   // values per column line of this table
        for (;;) {
            if (!fgets(line, sizeof(line), f)) { err = "table left open (no #end)"; break; }
            if (strncmp(line, "#end", 4) == 0) break;
            tok = strtok_r(line, " ", &save);
            if (!tok) continue;
            int col = -1;
            for (int c = 0; c < 5; ++c)
                if (strncmp(tok, keys[c], 3) == 0) { col = c; break; }
            if (col < 0) continue;
            if (!fgets(line, sizeof(line), f)) { err = "column line without a value line"; break; }
            int count = 0;
            for (tok = strtok_r(line, ",", &save); tok; tok = strtok_r(nullptr, ",", &save)) {
                if (data_numbers + count >= SPH_TABLE_SIZE) { err = "more than SPH_TABLE_SIZE entries"; break; }
                cols[col][data_numbers + count] = atof(tok);
                ++count;
            }
            if (err) break;
            if (count == 0) { err = "empty value line"; break; }
            if (len >= 0 && count != len) { err = "column lines of one table differ in length"; break; }
            len = count;
        }
        if (err) break;
        if (len < 0) { err = "table without a column line"; break; }
        data_numbers += len;
        cum[number] = data_numbers;
    }
    fclose(f);
    if (err) {
        set_error((std::string("sph_read_table: ") + err).c_str());
        return SPH_ERR_BAD_ARG;
    }
    t.n_tables = ntab;
    t.n_data = data_numbers;
    for (int i = 0; i < ntab; ++i) {
        t.index[i] = i == 0 ? 0 : cum[i - 1];
        t.size[i] = cum[i] - t.index[i];
    }
    *out = t;
    return SPH_OK;
}

// ---- record initialisation -------------------------------------------------------
// c_initial_inner_outer_particle_single (functions_NNPS.cuh:196-373): the
// host pass that turns deck records into the records the step starts from.
namespace {

// Case-H turbulent kinetic energy profile of Interpolate_k_caseH
// (functions_NNPS.cuh:156-171), z then k.
const double kCaseHK[2][22] = {
    {0.00393, 0.01178, 0.02356, 0.04123, 0.06086, 0.08245, 0.10209, 0.11975, 0.14135, 0.16294, 0.21202,
     0.23166, 0.25325, 0.30233, 0.35141, 0.40442, 0.4535, 0.50061, 0.55362, 0.60466, 0.70282, 0.74209},
    {0.3687, 0.39304, 0.4313, 0.49043, 0.53913, 0.56696, 0.58087, 0.62261, 0.62957, 0.64696, 0.66087,
     0.64696, 0.62261, 0.5913, 0.51826, 0.4313, 0.3513, 0.25043, 0.17043, 0.10087, 0.0, 0.0},
};

// Piecewise-linear table lookup of functions_NNPS.cuh:130-150: linear inside
// the table, extended past either end along its first or last segment.
double table_lerp(const double *zt, const double *vt, int n, double z) {
    if (z <= zt[0]) {
        const double dz = zt[1] - zt[0], dv = vt[1] - vt[0];
        return vt[0] + (dz == 0.0 ? 0.0 : (z - zt[0]) * (dv / dz));
    }
    if (z >= zt[n - 1]) {
        const double dz = zt[n - 1] - zt[n - 2], dv = vt[n - 1] - vt[n - 2];
        return vt[n - 2] + (dz == 0.0 ? 0.0 : (z - zt[n - 2]) * (dv / dz));
    }
    int lo = 0, hi = n;              // first entry with zt >= z
    while (lo < hi) {
        const int mid = (lo + hi) / 2;
        if (zt[mid] < z) lo = mid + 1; else hi = mid;
    }
    const int i = lo > 0 ? lo : 1;
    const double t = (z - zt[i - 1]) / (zt[i] - zt[i - 1]);
    return (1.0 - t) * vt[i - 1] + t * vt[i];
}

}  // namespace

extern "C" int sph_initial_records(const sph_params *p, sph_part1 *P1, int n, const double *k_table, int n_k,
                                   double l4, double l_ceiling) {
    using namespace sph;
    if (!p || (!P1 && n > 0) || n < 0) return SPH_ERR_BAD_ARG;
    if (p->n_profile < 2 || p->n_profile > SPH_MAX_PROFILE) {
        set_error("sph_initial_records: the velocity profile needs 2..SPH_MAX_PROFILE points");
        return SPH_ERR_BAD_ARG;
    }
    if (k_table && n_k < 2) { set_error("sph_initial_records: k table needs >= 2 points"); return SPH_ERR_BAD_ARG; }
    const double *kz = k_table ? k_table : kCaseHK[0];
    const double *kv = k_table ? k_table + n_k : kCaseHK[1];
    const int nk = k_table ? n_k : 22;
    const bool open = p->vii[SPH_VII_OPEN_BOUNDARY] > 0;
    const bool dim3 = p->vii[SPH_VII_DIM] == 3;
    const float scale = 0.16f / 0.16f;   // building height 0.16 m, as the reference hard-wires it
    for (int i = 0; i < n; ++i) {
        sph_part1 &r = P1[i];
        r.i_type = 1;
        r.buffer_type = 0;
        r.m_ref = r.m;
        r.uy = 0.0f;
        r.uz = 0.0f;
        r.temp = 300.0f;
        const float zs = scale * r.z;
        r.ux = (float)table_lerp(p->profile_z, p->profile_u, p->n_profile, zs);
        r.k_turb = (float)table_lerp(kz, kv, nk, zs);
        if (r.p_type == 3) r.p_type = 1;
        if (r.p_type == 0 || r.p_type == 1000) r.rho = 1.225f;
        const bool moving = r.p_type == 1 || r.p_type == -1;
        if (open && moving) {
            // buffer classes; the comparisons are in the record's float
            // promoted to double, as there
            if (r.y < p->l_left) { r.buffer_type = 3; r.i_type = 2; }
            else if (r.y > p->l_right) { r.buffer_type = 4; r.i_type = 2; }
            else if (r.x >= p->l3 - 1e-6 && r.x < l4 - 1e-6) { r.buffer_type = 2; r.i_type = 2; }
            else if (r.x < p->l2 - 1e-6) { r.buffer_type = 1; r.i_type = 2; }
            if (r.z >= l_ceiling && r.y < p->l_left && r.y > p->l_right) r.buffer_type = 5;
        }
        if (dim3) {
            if (moving) {
                if (r.z < 0) r.ux = 0.0f;
            } else {
                r.ux = 0.0f;
            }
        }
    }
    return SPH_OK;
}
