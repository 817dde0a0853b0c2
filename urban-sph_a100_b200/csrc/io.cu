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
