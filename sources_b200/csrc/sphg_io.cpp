// sphg_io.cpp — host-side input and output of libsphg: the case (steering)
// file reader of the reference (read_cas / treat_cmd / usr_def_parameter,
// declarations_sph.f90:61-335) and its Tecplot ASCII writer (output,
// declarations_sph.f90:1703-1810).  Plain C++, no device code: both work
// without a GPU.
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/sphg.h"

namespace {

std::string trim(const std::string& s) {
    size_t b = 0, e = s.size();
    while (b < e && std::isspace((unsigned char)s[b])) ++b;
    while (e > b && std::isspace((unsigned char)s[e - 1])) --e;
    return s.substr(b, e - b);
}

std::string upper(std::string s) {
    for (auto& c : s) c = (char)std::toupper((unsigned char)c);
    return s;
}

// Fortran list-directed items: separated by commas and/or blanks, strings
// optionally quoted with ' or ".
std::vector<std::string> items(const std::string& v) {
    std::vector<std::string> out;
    size_t i = 0, n = v.size();
    while (i < n) {
        while (i < n && (std::isspace((unsigned char)v[i]) || v[i] == ',')) ++i;
        if (i >= n) break;
        if (v[i] == '\'' || v[i] == '"') {
            char q = v[i++];
            size_t b = i;
            while (i < n && v[i] != q) ++i;
            out.push_back(v.substr(b, i - b));
            if (i < n) ++i;
        } else {
            size_t b = i;
            while (i < n && !std::isspace((unsigned char)v[i]) && v[i] != ',') ++i;
            out.push_back(v.substr(b, i - b));
        }
    }
    return out;
}

bool to_double(const std::string& s, double* out) {
    std::string t = s;
    for (auto& c : t) if (c == 'd' || c == 'D') c = 'e';   // Fortran double exponent
    char* end = nullptr;
    double v = std::strtod(t.c_str(), &end);
    if (end == t.c_str() || *end) return false;
    *out = v;
    return true;
}

bool to_int(const std::string& s, int32_t* out) {
    char* end = nullptr;
    long v = std::strtol(s.c_str(), &end, 10);
    if (end == s.c_str() || *end) return false;
    *out = (int32_t)v;
    return true;
}

// Fortran logical: .true./.false./T/F (leading dot optional)
bool to_logical(const std::string& s, int32_t* out) {
    std::string t = upper(s);
    size_t i = 0;
    if (i < t.size() && t[i] == '.') ++i;
    if (i >= t.size()) return false;
    if (t[i] == 'T') { *out = 1; return true; }
    if (t[i] == 'F') { *out = 0; return true; }
    return false;
}

void copy_str(char* dst, size_t cap, const std::string& s) {
    std::snprintf(dst, cap, "%s", s.c_str());
}

// usr_def_parameter: one "NAME = value" command
int treat_cmd(std::string cmd, sphg_params* p, sphg_case* c) {
    cmd = trim(cmd);
    if (cmd.empty()) return 0;
    if (cmd.back() == ',') cmd.pop_back();              // remove the last ","
    const size_t eq = cmd.find('=');
    if (eq == std::string::npos) return 0;
    const std::string name = upper(trim(cmd.substr(0, eq)));
    const std::string val = trim(cmd.substr(eq + 1));
    if (name.empty() || val.empty()) return 0;
    const std::vector<std::string> v = items(val);
    bool ok = !v.empty();
    auto d = [&](size_t i, double* o) { ok = ok && i < v.size() && to_double(v[i], o); };
    if (name == "PRINT STEP") ok = ok && to_int(v[0], &c->print_step);
    else if (name == "SAVE STEP") ok = ok && to_int(v[0], &c->save_step);
    else if (name == "PARTICLE PAIRS FIND METHOD") ok = ok && to_int(v[0], &c->nnps);
    else if (name == "RESULTS FILE") {
        for (size_t i = 0; i < 3 && i < v.size(); ++i) copy_str(c->results[i], sizeof(c->results[i]), v[i]);
        ok = v.size() >= 3;
    } else if (name == "INLET VELOCITY") d(0, &c->inlet_velocity);
    else if (name == "SINGLE PHASE") { ok = ok && to_logical(v[0], &c->single_phase); p->single_phase = c->single_phase; }
    else if (name == "FIRST PHASE" || name == "SECOND PHASE") {
        const std::string m = trim(v[0]);
        const int mat = m == "water" ? SPHG_WATER : (m == "soil" ? SPHG_SOIL : 0);
        ok = ok && mat != 0;
        if (name == "FIRST PHASE") { c->first_material = mat; p->first_material = mat; }
        else c->second_material = mat;
    } else if (name == "DRY SOIL") ok = ok && to_logical(v[0], &c->dry_soil);
    else if (name == "PARTICLE SIZE") copy_str(c->particle_size, sizeof(c->particle_size), v[0]);
    else if (name == "OPERATING MODE") copy_str(c->operating_mode, sizeof(c->operating_mode), v[0]);
    else if (name == "IMMERSE DEPTH") { /* read and ignored by the reference (declarations_sph.f90:277-281) */ }
    else if (name == "WITH NOZZLE") ok = ok && to_logical(v[0], &c->with_nozzle);
    else if (name == "WATER PROPERTY") {
        d(0, &p->water.rho0); d(1, &p->water.b); d(2, &p->water.gamma); d(3, &p->water.c); d(4, &p->water.viscosity);
    } else if (name == "SOIL PROPERTY") {
        d(0, &p->soil.rho0); d(1, &p->soil.k); d(2, &p->soil.E); d(3, &p->soil.niu); d(4, &p->soil.c);
    } else if (name == "DARCY PARAMETER") {
        d(0, &p->soil.porosity); d(1, &p->soil.permeability);
    } else if (name == "INTEGRATION SCHEME") ok = ok && to_int(v[0], &p->integrate_scheme);
    else if (name == "SOIL FAILURE CRITERIA") { d(0, &p->soil.cohesion); d(1, &p->soil.phi); }
    else if (name == "TIME STEP SIZE") { d(0, &p->dt); c->dt = p->dt; }
    else if (name == "MAXIMUM TIME STEP") { /* read and ignored by the reference (:321-325) */ }
    else {
        // the reference prints "Error: No such keyword" and carries on
        ++c->unknown_keywords;
        return 0;
    }
    if (!ok) ++c->bad_values;
    return 0;
}

}  // namespace

extern "C" int sphg_read_case(const char* path, sphg_params* p, sphg_case* c) {
    if (!path || !p || !c) return SPHG_ERR_BAD_ARG;
    FILE* f = std::fopen(path, "r");
    if (!f) return SPHG_ERR_BAD_ARG;   // the reference stops: "Steering file ... doesn't exist."
    std::memset(c, 0, sizeof(*c));
    std::string cmd;
    char buf[4096];
    bool eof = false;
    while (true) {
        std::string rec;
        if (!std::fgets(buf, sizeof(buf), f)) eof = true;
        else {
            rec = buf;
            while (!rec.empty() && (rec.back() == '\n' || rec.back() == '\r')) rec.pop_back();
        }
        rec = trim(rec);
        // end of file or '&': treat the unfinished command and stop (read_cas, :96-99)
        if (eof || (!rec.empty() && rec[0] == '&')) { treat_cmd(cmd, p, c); break; }
        if (rec.empty() || rec[0] == '#') continue;   // blank line, comment
        cmd += rec;
        if (rec.back() == ',') continue;              // command continues on the next line
        treat_cmd(cmd, p, c);
        cmd.clear();
    }
    std::fclose(f);
    return c->bad_values ? SPHG_ERR_BAD_ARG : SPHG_OK;
}

namespace {

void write_block(FILE* f, const double* a, int n, int stride, int comp) {
    for (int i = 0; i < n; ++i) std::fprintf(f, (i % 5 == 4 || i == n - 1) ? " %.15E\n" : " %.15E", a[(size_t)i * stride + comp]);
    if (n == 0) std::fprintf(f, "\n");
}
void write_iblock(FILE* f, const int32_t* a, int n) {
    for (int i = 0; i < n; ++i) std::fprintf(f, (i % 10 == 9 || i == n - 1) ? " %d\n" : " %d", a ? a[i] : 0);
    if (n == 0) std::fprintf(f, "\n");
}

}  // namespace

// output, declarations_sph.f90:1703-1810: one Tecplot ASCII zone in BLOCK
// format with the reference's variable list for the phase's material.
extern "C" int sphg_write_tecplot_phase(const char* path, int append, const sphg_phase_host* v, const int32_t* zone) {
    if (!path || !v || !v->x || !v->vx || !v->p || !v->rho || !v->mass) return SPHG_ERR_BAD_ARG;
    FILE* f = std::fopen(path, append ? "a" : "w");
    if (!f) return SPHG_ERR_BAD_ARG;
    const int n = v->ntotal + v->nvirt;
    if (v->material == SPHG_WATER) {
        if (!v->vof || !v->vof2) { std::fclose(f); return SPHG_ERR_BAD_ARG; }
        std::fprintf(f, " VARIABLES=\"X\",\"Y\",\"Pressure\",\"VoF\",\n");
        std::fprintf(f, " \"vx\",\"vy\",\"rho\",\"zone\",\"VoF2\",\"mass\" \n");
        std::fprintf(f, " ZONE I= %d  F=BLOCK\n", n);
        write_block(f, v->x, n, 2, 0); write_block(f, v->x, n, 2, 1);
        write_block(f, v->p, n, 1, 0); write_block(f, v->vof, n, 1, 0);
        write_block(f, v->vx, n, 2, 0); write_block(f, v->vx, n, 2, 1);
        write_block(f, v->rho, n, 1, 0); write_iblock(f, zone, n);
        write_block(f, v->vof2, n, 1, 0); write_block(f, v->mass, n, 1, 0);
    } else {
        if (!v->vof || !v->epsilon_p || !v->sxx || !v->sxy || !v->syy) { std::fclose(f); return SPHG_ERR_BAD_ARG; }
        std::fprintf(f, " VARIABLES=\"X\",\"Y\",\"Pressure\", \"VoF\", \"ep\",\n");
        std::fprintf(f, " \"sxy\", \"sxx\",\"syy\",\"vx\",\"vy\", \"rho\", \"mass\", \n");
        std::fprintf(f, " \"sigma_yy\", \"zone\" \n");
        std::fprintf(f, " ZONE I= %d  F=BLOCK\n", n);
        write_block(f, v->x, n, 2, 0); write_block(f, v->x, n, 2, 1);
        write_block(f, v->p, n, 1, 0); write_block(f, v->vof, n, 1, 0);
        write_block(f, v->epsilon_p, n, 1, 0); write_block(f, v->sxy, n, 1, 0);
        write_block(f, v->sxx, n, 1, 0); write_block(f, v->syy, n, 1, 0);
        write_block(f, v->vx, n, 2, 0); write_block(f, v->vx, n, 2, 1);
        write_block(f, v->rho, n, 1, 0); write_block(f, v->mass, n, 1, 0);
        std::vector<double> sig((size_t)n);
        for (int i = 0; i < n; ++i) sig[(size_t)i] = -v->p[i] + v->syy[i];   // sigma_yy = -p + syy
        write_block(f, sig.data(), n, 1, 0);
        write_iblock(f, zone, n);
    }
    std::fclose(f);
    return SPHG_OK;
}
