// sphg_scenes.cpp — the scene generators of libsphg, so that a Fortran or C
// host builds its particle arrays without a Python layer: the role of the
// reference's input_*.f90 routines (input_tank.f90, input_soilfail.f90,
// input_mix_Savage.f90), which lay particles on the cell centres of a
// lattice (block%cell_center, m_particles.f90:460-479: x outer loop, y inner
// loop, centres at (i-1)*dx + dx/2), tag them real or virtual by zone, and
// number real particles before virtual ones (take_real / take_virtual,
// m_particles.f90:808-893).  Plain C++, no device code.
//
// The choices the reference leaves to its case file are stated here:
//   * water b = rho0*c0^2/gamma with c0 = 10*sqrt(2*9.81*H) (H the depth of
//     the water), viscosity 1.0e-3 Pa s;
//   * soil K = E/(3(1-2nu)), G = E/(2(1+nu)), c = sqrt((K + 4G/3)/rho0);
//   * geostatic soil stress from K0 = 1 - sin(phi): with P the vertical
//     overburden, p = (1+2K0)/3 P, sxx = (1-K0)/3 P, syy = -2(1-K0)/3 P;
//   * hsml = dx*1.2 with 1.2 a single-precision literal
//     (input_mix_Savage.f90:60);
//   * two layers of virtual particles under the floor and outside both walls.
// The arithmetic follows sources_b200/scenes.py operation for operation, and
// a test holds the two equal bit for bit.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/sphg.h"

namespace {

const double kHFactor = (double)1.2f;

struct Lattice {
    std::vector<double> x, y;
    std::vector<char> virt;
};

// cell centres of a width x height box plus `layers` virtual rows under the
// floor and columns outside both walls (x outer, y inner)
Lattice box(double width, double height, double dx, int layers = 2) {
    const long m = (long)std::nearbyint(width / dx) + 2 * layers;
    const long n = (long)std::nearbyint(height / dx) + layers;
    const double x0 = -layers * dx, y0 = -layers * dx;
    Lattice L;
    L.x.resize((size_t)(m * n));
    L.y.resize((size_t)(m * n));
    L.virt.resize((size_t)(m * n));
    size_t k = 0;
    for (long i = 0; i < m; ++i)
        for (long j = 0; j < n; ++j, ++k) {
            L.x[k] = (double)i * dx + dx / 2.0 + x0;
            L.y[k] = (double)j * dx + dx / 2.0 + y0;
            L.virt[k] = (L.x[k] < 0.0) || (L.x[k] > width) || (L.y[k] < 0.0);
        }
    return L;
}

// indices of the real particles (in lattice order) then the virtual ones
template <class F>
void select(const Lattice& L, F real, std::vector<long>& idx, int32_t* ntotal, int32_t* nvirt) {
    idx.clear();
    for (size_t k = 0; k < L.x.size(); ++k)
        if (!L.virt[k] && real(L.x[k], L.y[k])) idx.push_back((long)k);
    *ntotal = (int32_t)idx.size();
    for (size_t k = 0; k < L.x.size(); ++k)
        if (L.virt[k]) idx.push_back((long)k);
    *nvirt = (int32_t)idx.size() - *ntotal;
}

struct Water { double rho0, gamma, c, b, mu; };
Water water_material(double depth) {
    Water w;
    w.rho0 = 1000.0; w.gamma = 7.0; w.mu = 1.0e-3;
    w.c = 10.0 * std::sqrt(2.0 * 9.81 * depth);
    w.b = w.rho0 * w.c * w.c / w.gamma;
    return w;
}
void set_water(sphg_material& m, const Water& w) {
    m.rho0 = w.rho0; m.gamma = w.gamma; m.c = w.c; m.b = w.b; m.viscosity = w.mu;
}

struct Soil { double rho0, E, nu, K, G, c, phi, cohesion, porosity, permeability; };
Soil soil_material(double phi_deg, double porosity, double permeability) {
    Soil s;
    s.rho0 = 1850.0; s.E = 0.84e6; s.nu = 0.3; s.cohesion = 0.0;
    s.porosity = porosity; s.permeability = permeability;
    s.K = s.E / (3.0 * (1.0 - 2.0 * s.nu));
    s.G = s.E / (2.0 * (1.0 + s.nu));
    s.c = std::sqrt((s.K + 4.0 * s.G / 3.0) / s.rho0);
    s.phi = phi_deg * (M_PI / 180.0);
    return s;
}
void set_soil(sphg_material& m, const Soil& s) {
    m.rho0 = s.rho0; m.E = s.E; m.niu = s.nu; m.k = s.K; m.G = s.G; m.c = s.c; m.phi = s.phi;
    m.cohesion = s.cohesion; m.porosity = s.porosity; m.permeability = s.permeability;
}

// every non-null array of the host view to zero
void zero_phase(sphg_phase_host* v, long n) {
    double* const vec[] = {v->x, v->vx, v->dvx, v->av, v->v_min};
    for (double* a : vec) if (a) std::memset(a, 0, sizeof(double) * 2 * (size_t)n);
    double* const sc[] = {v->rho, v->rho_min, v->drho, v->p, v->c, v->mass, v->hsml, v->vof, v->vof_min, v->dvof,
                          v->vof2, v->sxx, v->sxy, v->syy, v->dsxx, v->dsxy, v->dsyy, v->dp, v->sxx_min, v->sxy_min,
                          v->syy_min, v->p_min, v->epsilon_p, v->vcc, v->txx, v->tyy, v->txy};
    for (double* a : sc) if (a) std::memset(a, 0, sizeof(double) * (size_t)n);
    if (v->itype) std::memset(v->itype, 0, sizeof(int32_t) * (size_t)n);
    if (v->fail) std::memset(v->fail, 0, sizeof(int32_t) * (size_t)n);
}

// positions, h and particle types of a phase (setup_itype m_particles.f90:896-913:
// +-2 water, +-3 soil, negative for virtual particles)
void fill_phase(sphg_phase_host* v, const Lattice& L, const std::vector<long>& idx, int material, double dx) {
    const long n = (long)idx.size();
    zero_phase(v, n);
    v->material = material;
    v->dspp = dx;
    const int sign = material == SPHG_WATER ? 2 : 3;
    for (long a = 0; a < n; ++a) {
        v->x[2 * a] = L.x[(size_t)idx[(size_t)a]];
        v->x[2 * a + 1] = L.y[(size_t)idx[(size_t)a]];
        v->hsml[a] = dx * kHFactor;
        v->itype[a] = a < v->ntotal ? sign : -sign;
    }
}

void k0_stress(sphg_phase_host* v, const std::vector<double>& over, double phi) {
    const double k0 = 1.0 - std::sin(phi);
    const double fp = (1.0 + 2.0 * k0) / 3.0, fx = (1.0 - k0) / 3.0, fy = -2.0 * (1.0 - k0) / 3.0;
    const long n = (long)over.size();
    for (long a = 0; a < n; ++a) {
        v->p[a] = fp * over[(size_t)a];
        v->sxx[a] = fx * over[(size_t)a];
        v->syy[a] = fy * over[(size_t)a];
        v->sxy[a] = 0.0;
    }
}

// initial_density, m_particles.f90:2105-2130 (inverse Tait)
void initial_density(sphg_phase_host* v, long n, const Water& w) {
    for (long a = 0; a < n; ++a) v->rho[a] = w.rho0 * std::pow(v->p[a] / w.b + 1.0, 1.0 / w.gamma);
}

void finish(sphg_params* p, long nmax, double width, double height, double dx, int skf, int precision) {
    p->skf = skf;
    p->precision = precision;
    const double margin = 8 * dx;
    p->x_min = -2 * dx - margin; p->x_max = width + 2 * dx + margin;
    p->y_min = -2 * dx - margin; p->y_max = 2.0 * height + margin;
    const int sk = (skf == 2 || skf == 3) ? 3 : 2;
    p->max_interaction = (int64_t)(3 * sk * sk * nmax) + 4096;
}

bool valid(const sphg_scene_spec* s) {
    if (!s || !(s->dx > 0.0) || !(s->box_w > 0.0) || !(s->box_h > 0.0)) return false;
    if (!(s->col_w > 0.0) || !(s->col_h > 0.0) || s->skf < 1 || s->skf > 4) return false;
    if (s->precision != SPHG_FP64 && s->precision != SPHG_FP32) return false;
    if (s->box_w / s->dx > 1e6 || s->box_h / s->dx > 1e6) return false;
    if (s->kind == SPHG_SCENE_TWO_PHASE && (!(s->water_h > 0.0) || !(s->porosity > 0.0 && s->porosity < 1.0) ||
                                            !(s->permeability > 0.0) || !(s->forchheimer_b >= 0.0)))
        return false;
    return s->kind == SPHG_SCENE_DAM_BREAK || s->kind == SPHG_SCENE_GRANULAR_COLUMN || s->kind == SPHG_SCENE_TWO_PHASE;
}

// the real particles of each phase of a scene, with the lattice they come from
struct Layout {
    Lattice L;
    std::vector<long> idx[2];
    int32_t ntotal[2] = {0, 0}, nvirt[2] = {0, 0};
    int nphase = 1;
};

Layout layout(const sphg_scene_spec* s) {
    Layout o;
    o.L = box(s->box_w, s->box_h, s->dx);
    const double cw = s->col_w, ch = s->col_h;
    if (s->kind == SPHG_SCENE_TWO_PHASE) {
        const double wh = s->water_h;
        select(o.L, [&](double, double y) { return y < wh; }, o.idx[0], &o.ntotal[0], &o.nvirt[0]);
        select(o.L, [&](double x, double y) { return x < cw && y < ch; }, o.idx[1], &o.ntotal[1], &o.nvirt[1]);
        o.nphase = 2;
    } else {
        select(o.L, [&](double x, double y) { return x < cw && y < ch; }, o.idx[0], &o.ntotal[0], &o.nvirt[0]);
    }
    return o;
}

}  // namespace

extern "C" void sphg_scene_default(int kind, sphg_scene_spec* s) {
    if (!s) return;
    std::memset(s, 0, sizeof(*s));
    s->kind = kind;
    s->skf = 1;
    s->phi_deg = 19.8;
    s->porosity = 0.4;
    s->permeability = 1.0e-3;
    if (kind == SPHG_SCENE_DAM_BREAK) {
        s->precision = SPHG_FP64;
        s->dx = 0.005; s->box_w = 0.8; s->box_h = 0.6; s->col_w = 0.2; s->col_h = 0.4;
    } else if (kind == SPHG_SCENE_GRANULAR_COLUMN) {
        s->precision = SPHG_FP32;
        s->dx = 0.002; s->box_w = 1.0; s->box_h = 0.3; s->col_w = 0.2; s->col_h = 0.1;
    } else {
        s->precision = SPHG_FP32;
        s->dx = 0.002; s->box_w = 4.0; s->box_h = 1.0; s->col_w = 1.0; s->col_h = 0.4; s->water_h = 0.8;
    }
}

extern "C" int sphg_scene_size(const sphg_scene_spec* s, int32_t* n_phase, int32_t* ntotal, int32_t* nvirt) {
    if (!valid(s) || !n_phase || !ntotal || !nvirt) return SPHG_ERR_BAD_ARG;
    const Layout o = layout(s);
    *n_phase = o.nphase;
    for (int k = 0; k < o.nphase; ++k) { ntotal[k] = o.ntotal[k]; nvirt[k] = o.nvirt[k]; }
    return SPHG_OK;
}

extern "C" int sphg_make_scene(const sphg_scene_spec* s, sphg_params* p, sphg_phase_host* first,
                               sphg_phase_host* second) {
    if (!valid(s) || !p || !first) return SPHG_ERR_BAD_ARG;
    const Layout o = layout(s);
    sphg_phase_host* ph[2] = {first, second};
    for (int k = 0; k < o.nphase; ++k) {
        sphg_phase_host* v = ph[k];
        if (!v || v->ntotal != o.ntotal[k] || v->nvirt != o.nvirt[k]) return SPHG_ERR_BAD_ARG;
        if (!v->x || !v->hsml || !v->itype || !v->p || !v->c || !v->vof || !v->rho || !v->mass) return SPHG_ERR_BAD_ARG;
        if (s->kind != SPHG_SCENE_DAM_BREAK && (k == 1 || s->kind == SPHG_SCENE_GRANULAR_COLUMN) &&
            (!v->sxx || !v->sxy || !v->syy))
            return SPHG_ERR_BAD_ARG;
    }
    sphg_default_params(p);
    const double dx = s->dx, g = p->gravity;
    const double cw = s->col_w, ch = s->col_h;
    if (s->kind == SPHG_SCENE_DAM_BREAK) {
        sphg_phase_host* P = first;
        fill_phase(P, o.L, o.idx[0], SPHG_WATER, dx);
        const long n = (long)o.idx[0].size();
        const Water w = water_material(ch);
        set_water(p->water, w);
        for (long a = 0; a < n; ++a) {
            const double xx = P->x[2 * a], yy = P->x[2 * a + 1];
            P->p[a] = w.rho0 * g * (yy - ch);
            if (a >= P->ntotal && (xx >= cw || yy > ch)) P->p[a] = 0.0;
            P->c[a] = w.c;
            P->vof[a] = 1.0;
        }
        initial_density(P, n, w);
        for (long a = 0; a < n; ++a) P->mass[a] = dx * dx * P->rho[a];
        p->single_phase = 1;
        p->first_material = SPHG_WATER;
        p->alpha = 0.1; p->beta = 0.0; p->delta = 0.1;
        p->dt = 0.25 * P->hsml[0] / w.c;
        finish(p, n, s->box_w, s->box_h, dx, s->skf, s->precision);
    } else if (s->kind == SPHG_SCENE_GRANULAR_COLUMN) {
        sphg_phase_host* P = first;
        fill_phase(P, o.L, o.idx[0], SPHG_SOIL, dx);
        const long n = (long)o.idx[0].size();
        const Soil m = soil_material(s->phi_deg, s->porosity, s->permeability);
        set_soil(p->soil, m);
        std::vector<double> over((size_t)n);
        for (long a = 0; a < n; ++a) {
            const double xx = P->x[2 * a], yy = P->x[2 * a + 1];
            over[(size_t)a] = std::max(m.rho0 * g * (yy - ch), 0.0);
            if (a >= P->ntotal && xx >= cw) over[(size_t)a] = 0.0;
        }
        k0_stress(P, over, m.phi);
        for (long a = 0; a < n; ++a) {
            P->c[a] = m.c;
            P->rho[a] = m.rho0;
            P->mass[a] = dx * dx * P->rho[a];
        }
        p->single_phase = 1;
        p->first_material = SPHG_SOIL;
        p->alpha = 0.1;
        p->dt = 0.1 * P->hsml[0] / m.c;
        finish(p, n, s->box_w, s->box_h, dx, s->skf, s->precision);
    } else {
        sphg_phase_host* W = first;
        sphg_phase_host* S = second;
        fill_phase(W, o.L, o.idx[0], SPHG_WATER, dx);
        fill_phase(S, o.L, o.idx[1], SPHG_SOIL, dx);
        const long nw = (long)o.idx[0].size(), ns = (long)o.idx[1].size();
        const Water w = water_material(s->water_h);
        const Soil m = soil_material(s->phi_deg, s->porosity, s->permeability);
        set_water(p->water, w);
        set_soil(p->soil, m);
        // water: hydrostatic pressure, the porosity inside the soil block
        for (long a = 0; a < nw; ++a) {
            const double wx = W->x[2 * a], wy = W->x[2 * a + 1];
            W->p[a] = std::max(w.rho0 * g * (wy - s->water_h), 0.0);
            W->c[a] = w.c;
            W->vof[a] = (wx < cw && wy < ch) ? s->porosity : 1.0;
        }
        initial_density(W, nw, w);
        for (long a = 0; a < nw; ++a) {
            W->rho[a] = W->rho[a] * W->vof[a];
            W->mass[a] = dx * dx * W->rho[a];
        }
        // soil: buoyant overburden, K0 stress, solid fraction 1 - porosity
        std::vector<double> over((size_t)ns);
        for (long a = 0; a < ns; ++a) {
            const double sx = S->x[2 * a], sy = S->x[2 * a + 1];
            over[(size_t)a] = std::max((m.rho0 - w.rho0) * g * (sy - ch), 0.0);
            if (a >= S->ntotal && (sx >= cw || sy >= ch)) over[(size_t)a] = 0.0;
        }
        k0_stress(S, over, m.phi);
        for (long a = 0; a < ns; ++a) {
            S->c[a] = m.c;
            S->vof[a] = 1.0 - s->porosity;
            S->rho[a] = m.rho0 * S->vof[a];
            S->mass[a] = dx * dx * S->rho[a];
        }
        p->single_phase = 0;
        p->alpha = 0.1;
        p->forchheimer_b = s->forchheimer_b;
        const double h = W->hsml[0];
        p->dt = std::min(0.25 * h / w.c, 0.1 * h / m.c);
        finish(p, std::max(nw, ns), s->box_w, s->box_h, dx, s->skf, s->precision);
    }
    return SPHG_OK;
}
