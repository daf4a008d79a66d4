// sphg_kernels.cuh — the sm_100a kernels of libsphg.
//
// Per step (two-phase, declarations_sph.f90:525-791 with single_step :1131):
//   k_first_half      leapfrog predictor (+ Drucker-Prager on soil)      elementwise
//   k_cell_count      cell key per particle, rank inside its cell         elementwise
//   k_cell_scatter    counting-sort scatter into cell order              elementwise
//   k_cell_sort       order each cell by state index (determinism)       per cell
//   k_gather          sorted copies: x, h, (v, m, rho); soil: DP + stress pair pass inputs
//   k_water_sum       summation density (water-only step)                pair pass
//   k_water_pass_a    continuity / df2, delta-SPH(rho), strain rate, EOS  pair pass
//   k_water_pass_b    momentum, art. viscosity, delta-SPH(vof), wall force, XSPH  pair pass
//   k_soil_pass       every same-phase soil term + flow rule + Jaumann   pair pass
//   cross_soil_sums   Darcy drag + pore pressure on soil (in k_soil_pass) pair sums
//   cross_water_sums  Darcy drag, dvof, vof2 on water (in k_water_pass_b) pair sums
//   k_update          leapfrog corrector / first step (+ DP on soil)     elementwise
// Every pair pass is a gather: one thread per particle in cell order visits
// the 3 x 3 neighbouring cells (three contiguous row segments of the sorted
// list), evaluates the reference's pair test bit-exactly in FP64 and sums the
// particle's own side of each pair term.  The reference scatters each pair
// to both ends (e.g. m_particles.f90:2427-2428); the gather evaluates the pair
// once from each end, with the algebraically identical term, so the sums
// match the reference to rounding, and the pair set matches exactly.
#pragma once
#include "sphg_device.cuh"

struct SimConst {
    int skf, single_phase, summation_density, average_velocity, visc_artificial;
    int artificial_density, soil_artificial_stress, volume_fraction, water_artificial_volume;
    int volume_fraction_renorm, stress_integration, plasticity, yield_dp;
    int renorm_now;        // this step renormalises vof (itimestep % interval == 0)
    double gravity, numeric_gravity, alpha, beta, etq, dd, p1, p2, delta, epsilon, dt;
    double w_rho0, w_b, w_gamma, w_c, w_mu;
    double s_rho0, s_k, s_E, s_niu, s_c, s_perm, s_G, s_alpha1;
    double s_kb;           // permeability x Forchheimer b (0: linear Darcy)
    const SceneTab* tab;   // per-scene dt, water b and c, soil alpha1 (indexed by PhaseDev::sid)
};

#ifndef SPHG_TPB
#define SPHG_TPB 128
#endif
// Default x cells per neighbour cell (GridGeom::kx; sphg_tuning.x_split
// overrides it per context).  Step time on a B200 at 912,016 particles:
// 1: 0.596-0.603 ms, 2: 0.558-0.565, 3: 0.567, 4: 0.548 (the candidate
// strip narrows from 3 to 2.25 support radii; the pair set is the same).
#ifndef SPHG_X_SPLIT
#define SPHG_X_SPLIT 4
#endif
// minimum resident blocks per SM of each FP32 pair pass (register cap for
// the compiler: 65,536 / (SPHG_TPB * min blocks) registers per thread); the
// FP64 passes are left uncapped.  Timed on a B200 at 912,016 particles:
// water_pass_a (staged, recording the hit masks) 131 us at 8 blocks, 134 at
// 7, 138 at 10 (48 registers).  water_pass_b (replaying the masks, with the
// cross pairs) 176 us at 6 blocks, 164 at 7, 181 at 8 (spills).  soil_pass
// with the cross pairs: 86 us uncapped (128 registers), 91 at 5, 86 at 6.
#ifndef SPHG_MINB_A
#define SPHG_MINB_A 8
#endif
#ifndef SPHG_MINB_B
#define SPHG_MINB_B 7
#endif
// neighbours of one block of the two-phase water_pass_a staged in shared
// memory (records; the sizes of 128 consecutive particles' candidate runs at
// dx = 0.002 m: mean 414, largest 544).  Each lane tests its candidates
// from there one at a time and runs the pair body on each hit at once
// (scan_direct): 123.5 us per launch at 912,016 particles, against 130.7 us
// with the hit buffer that batches the bodies across the warp, and 130.4 us
// for the direct scan reading through L1.
#ifndef SPHG_STAGE_A
#define SPHG_STAGE_A 576
#endif
#ifndef SPHG_MINB_SOIL
#define SPHG_MINB_SOIL 1
#endif

// launch the step's kernels with programmatic stream serialization (0: plain launches)
#ifndef SPHG_PDL
#define SPHG_PDL 1
#endif

__device__ __forceinline__ int gtid() { return blockIdx.x * blockDim.x + threadIdx.x; }

// Programmatic dependent launch: the step's kernels are launched so that the
// next one may start while this one finishes (Engine::launch_pdl).  A kernel
// lets its successor launch as soon as all of its own blocks have started,
// and waits for its predecessor's results before touching any memory.
// Launched without the attribute, both are no-ops.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

// ----------------------------------------------------------------- cell list
// Cell key (row-major) of a particle at p and its rank inside its cell; the
// clamped and non-finite positions are counted into the step's counters, or
// into the next step's (next != 0).
__device__ __forceinline__ void cell_key(const GridGeom& g, double2 p, int a, int* __restrict__ cell_id,
                                         int* __restrict__ rank, int* __restrict__ counts, DevCounters* cnt, int next) {
    int cx, cy; bool clamped;
    cell_coords(g, p.x, p.y, cx, cy, clamped);
    if (clamped) atomicAdd(next ? &cnt->n_out_next : &cnt->n_out, 1);
    if (!(isfinite(p.x) && isfinite(p.y))) atomicAdd(next ? &cnt->nonfinite_next : &cnt->nonfinite, 1);
    const int c = cy * g.ncx + cx;
    cell_id[a] = c;
    rank[a] = atomicAdd(counts + c, 1);
}

static __global__ void __launch_bounds__(256) k_cell_count(const double2* __restrict__ x, int n, GridGeom g,
                                                    int* __restrict__ cell_id, int* __restrict__ rank,
                                                    int* __restrict__ counts, DevCounters* cnt, int next) {
    pdl_enter();
    int a = gtid();
    if (a >= n) return;
    cell_key(g, x[a], a, cell_id, rank, counts, cnt, next);
}

static __global__ void __launch_bounds__(256) k_cell_scatter(int n, const int* __restrict__ cell_id, const int* __restrict__ rank,
                                                      const int* __restrict__ cell_start, int* __restrict__ perm) {
    pdl_enter();
    int a = gtid();
    if (a >= n) return;
    perm[cell_start[cell_id[a]] + rank[a]] = a;
}

// Insertion sort of each cell's (few) entries by original particle index, so
// the visiting order, and with it every sum, depends neither on atomic timing
// nor on the current state order (a download/upload restart is bit-identical).
// The cell's count, consumed by the scan, is reset to zero for the corrector,
// which counts the next step's cells.
static __global__ void __launch_bounds__(256) k_cell_sort(int ncell, const int* __restrict__ cell_start,
                                                   const int* __restrict__ orig, int* __restrict__ perm,
                                                   int* __restrict__ counts) {
    pdl_enter();
    int c = gtid();
    if (c >= ncell) return;
    counts[c] = 0;
    int b = cell_start[c], e = cell_start[c + 1];
    for (int i = b + 1; i < e; ++i) {
        int v = perm[i], ov = orig[v], j = i - 1;
        while (j >= b && orig[perm[j]] > ov) { perm[j + 1] = perm[j]; --j; }
        perm[j + 1] = v;
    }
}

// ------------------------------------------------------------- integrators
// What the last pass of a phase does after its sums: nothing (right-hand side
// only, sphg_single_step) or the leapfrog corrector of this step.
struct StepCtl {
    int update;      // run the corrector (first_step or second_half)
    int first;       // itimestep == 1: first_step
    int with_vof;    // integrate the water volume fraction (two-phase)
    int do_dp;       // Drucker-Prager after the corrector (soil)
    int* ncount;     // non-null: after the corrector, the cell key and rank of the new position, counted
                     // into this phase's per-cell counts for the next step's cell list
};

// first_half, declarations_sph.f90:643-684 (and :812-825, :998-1025), plus the
// Drucker-Prager call that follows it on soil (:559, :1027).  Returns the
// particle's fail flag of that DP call.
template <typename T>
__device__ __forceinline__ int first_half_one(const PhaseDev<T>& P, int a, const SimConst& c, int with_vof, int do_dp) {
    const SceneTab& st = c.tab[P.sid[a]];
    const double dt = st.dt;
    if (!c.summation_density) { double r = P.rho[a]; P.rho_min[a] = r; P.rho[a] = r + (dt / 2.0) * (double)P.drho[a]; }
    if (with_vof && P.material == 1 && c.volume_fraction) {
        double f = P.vof[a]; P.vof_min[a] = f; P.vof[a] = f + (dt / 2.0) * (double)P.dvof[a];
    }
    int fail = 0;
    const bool soil = P.material == 2;
    double p = 0, sxx = 0, sxy = 0, syy = 0;
    if (soil) {
        p = P.p[a]; sxx = P.sxx[a]; sxy = P.sxy[a]; syy = P.syy[a];
        if (c.stress_integration == 2) {
            P.sxx_min[a] = sxx; P.sxy_min[a] = sxy; P.syy_min[a] = syy; P.p_min[a] = p;
            sxx = sxx + (dt / 2.0) * (double)P.dsxx[a];
            sxy = sxy + (dt / 2.0) * (double)P.dsxy[a];
            syy = syy + (dt / 2.0) * (double)P.dsyy[a];
            p = p + (dt / 2.0) * (double)P.dp[a];
        }
    }
    if (P.itype[a] >= 0) {
        double2 v = P.v[a];
        P.v_min[a] = v;
        const typename V2<T>::t d = P.dv[a];
        v.x = v.x + (dt / 2.0) * (double)d.x;
        v.y = v.y + (dt / 2.0) * (double)d.y;
        P.v[a] = v;
    }
    if (soil) {
        if (do_dp) { fail = dp_return(p, sxx, sxy, syy, st.s_alpha1); P.fail[a] = fail; }
        P.p[a] = p; P.sxx[a] = sxx; P.sxy[a] = sxy; P.syy[a] = syy;
    }
    return fail;
}

// first_step (:686-723) when first != 0, else second_half (:725-762), plus the
// Drucker-Prager call after it on soil (:583, :601, :1069, :1107).
template <typename T>
__device__ __forceinline__ int update_one(const PhaseDev<T>& P, int a, const SimConst& c, int first, int with_vof, int do_dp) {
    const SceneTab& st = c.tab[P.sid[a]];
    const double dt = st.dt;
    int fail = 0;
    if (!c.summation_density)
        P.rho[a] = first ? P.rho[a] + (dt / 2.0) * (double)P.drho[a] : P.rho_min[a] + dt * (double)P.drho[a];
    if (with_vof && P.material == 1 && c.volume_fraction)
        P.vof[a] = first ? P.vof[a] + (dt / 2.0) * (double)P.dvof[a] : P.vof_min[a] + dt * (double)P.dvof[a];
    if (P.material == 2) {
        double p = P.p[a], sxx = P.sxx[a], sxy = P.sxy[a], syy = P.syy[a];
        const double d0 = P.dsxx[a], d1 = P.dsxy[a], d2 = P.dsyy[a], d3 = P.dp[a];
        if (c.stress_integration == 1) {
            sxx = sxx + dt * d0; sxy = sxy + dt * d1; syy = syy + dt * d2; p = p + dt * d3;
        } else if (c.stress_integration == 2) {
            if (first) {
                sxx = sxx + (dt / 2.0) * d0; sxy = sxy + (dt / 2.0) * d1;
                syy = syy + (dt / 2.0) * d2; p = p + (dt / 2.0) * d3;
            } else {
                sxx = P.sxx_min[a] + dt * d0; sxy = P.sxy_min[a] + dt * d1;
                syy = P.syy_min[a] + dt * d2; p = P.p_min[a] + dt * d3;
            }
        }
        if (do_dp) { fail = dp_return(p, sxx, sxy, syy, st.s_alpha1); P.fail[a] = fail; }
        P.p[a] = p; P.sxx[a] = sxx; P.sxy[a] = sxy; P.syy[a] = syy;
    }
    if (P.itype[a] >= 0) {
        double2 v = first ? P.v[a] : P.v_min[a];
        const typename V2<T>::t d = P.dv[a];
        const typename V2<T>::t av = P.av[a];
        double2 x = P.x[a];
        const double h = first ? dt / 2.0 : dt;
        v.x = v.x + h * (double)d.x + (double)av.x;
        x.x = x.x + dt * v.x;
        v.y = v.y + h * (double)d.y + (double)av.y;
        x.y = x.y + dt * v.y;
        P.v[a] = v;
        P.x[a] = x;
    }
    return fail;
}

__device__ __forceinline__ void count_fail(DevCounters* cnt, int slot, int fail) {
    int s = __syncthreads_count(fail);
    if (threadIdx.x == 0 && s) atomicAdd(&cnt->nfail[slot], s);
}

// ------------------------------------------------------------------ gathers
// Sorted copies of position, h and (v, vol, rho).  With fh != 0 the particle's
// leapfrog predictor (first_half, + DP on soil) runs first, so the records
// carry the half-step state.  For soil also the in-step Drucker-Prager return
// (declarations_sph.f90:1242-1247) on the state and the stress/pressure
// record of the soil pass.
template <typename T>
__global__ void __launch_bounds__(256) k_gather(PhaseDev<T> P, SimConst c, int soil, int do_dp, int fh, int with_vof,
                                                int fh_dp, DevCounters* cnt) {
    pdl_enter();
    int k = gtid();
    int fail0 = 0, fail = 0;
    if (k < P.n) {
        int a = P.perm[k];
        if (fh) fail0 = first_half_one(P, a, c, with_vof, fh_dp);
        P.xs[k] = P.x[a];
        P.hs[k] = P.hsml[a];
        double2 v = P.v[a];
        RecA<T> ra;
        const double rho = P.rho[a];
        ra.vx = (T)v.x; ra.vy = (T)v.y; ra.vol = (T)(P.mass[a] / rho); ra.rho = (T)rho;
        P.recA[k] = ra;
        if (soil) {
            double p = P.p[a], sxx = P.sxx[a], sxy = P.sxy[a], syy = P.syy[a];
            if (do_dp) {
                fail = dp_return(p, sxx, sxy, syy, c.tab[P.sid[a]].s_alpha1);
                P.p[a] = p; P.sxx[a] = sxx; P.sxy[a] = sxy; P.syy[a] = syy;
                P.fail[a] = fail;
            }
            RecB<T> rb;
            rb.p = (T)p; rb.c = (T)P.c[a]; rb.vof = (T)P.vof[a];
            rb.sxx = (T)sxx; rb.sxy = (T)sxy; rb.syy = (T)syy;
            rb.itype = (T)P.itype[a]; rb.aux = T(0);
            P.recB[k] = rb;
        }
    }
    if (fh && fh_dp) count_fail(cnt, 0, fail0);
    if (soil && do_dp) count_fail(cnt, 1, fail);
}

// Per-particle interaction statistics (interaction_statistics,
// m_particles.f90:555-597) and the pair count of the list.
__device__ __forceinline__ void count_stats(DevCounters* cnt, int list, int phase_slot, int hits, bool valid) {
    unsigned long long h = valid ? (unsigned long long)hits : 0ull;
    int hmax = valid ? hits : 0, hmin = valid ? hits : 0x7fffffff, hz = (valid && hits == 0) ? 1 : 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        h += __shfl_xor_sync(0xffffffffu, h, o);
        hmax = max(hmax, __shfl_xor_sync(0xffffffffu, hmax, o));
        hmin = min(hmin, __shfl_xor_sync(0xffffffffu, hmin, o));
        hz += __shfl_xor_sync(0xffffffffu, hz, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&cnt->pairs[list], h);
        if (phase_slot >= 0) {
            atomicMax(&cnt->maxiac[phase_slot], hmax);
            atomicMin(&cnt->miniac[phase_slot], hmin);
            if (hz) atomicAdd(&cnt->noiac[phase_slot], hz);
        }
    }
}

// hit-buffer depth per thread: 24 covers the ~20 neighbours of a particle at
// support 2h = 2.4 dx in one drain (FP32); FP64 entries are larger.
template <typename T> struct Chunk { static const int value = sizeof(T) == 4 ? 24 : 16; };
#define SPHG_HITBUF(T) __shared__ HitBuf<T, SPHG_TPB, Chunk<T>::value> hb

// Kernel constants for particle a: per particle when every h is equal, else
// per pair (mhsml = (h_a + h_b)/2).
template <typename T, int SKF>
__device__ __forceinline__ void pair_kernel(const KernelConst<T, SKF>& ka, const SearchConst& sc, double ha,
                                            const double* __restrict__ hs, int m, T dx, T dy, T& w, T& s, T& r2,
                                            T& mh) {
    r2 = sqsum<T>(dx, dy);
    if (sc.uniform) {
        ka.eval(r2, w, s);
        mh = ka.h;
    } else {
        KernelConst<T, SKF> kb;
        const double mhd = (ha + hs[m]) / 2.0;
        kb.init((T)mhd);
        kb.eval(r2, w, s);
        mh = (T)mhd;
    }
}

// ------------------------------------------------------ water: summation rho
// sum_density (m_particles.f90:2243-2298) and the df2 divergence of the
// water-only step, drho = -rho*(df2(vx,'x') + df2(vy,'y'))
// (declarations_sph.f90:1465-1466, df2 m_particles.f90:1802-1831).
template <typename T, int SKF>
__global__ void __launch_bounds__(SPHG_TPB) k_water_sum(PhaseDev<T> P, GridGeom g, SearchConst sc, SimConst c, DevCounters* cnt) {
    pdl_enter();
    SPHG_HITBUF(T);
    const int k = gtid();
    const bool valid = k < P.n;
    const int kk = valid ? k : 0;
    const double2 xa = P.xs[kk];
    const double ha = P.hs[kk];
    const RecA<T> ra = P.recA[kk];
    KernelConst<T, SKF> ka;
    ka.init((T)ha);
    T w0, s0;
    ka.eval(T(0), w0, s0);
    const T ma = ra.vol * ra.rho;
    T wi = w0 * ma / ra.rho;
    T num = w0 * ma;
    T sx = T(0), sy = T(0);
    const RecA<T>* __restrict__ rec = P.recA;
    uint4 mask;
    const int hits = visit_batched_rec(hb, g, sc, P.cell_start, P.xs, P.hs, xa, ha, k, valid, mask, [&](int m, T dx, T dy) {
        const RecA<T> rb = rec[m];
        T w, sr, r2, mh;
        pair_kernel<T, SKF>(ka, sc, ha, P.hs, m, dx, dy, w, sr, r2, mh);
        const T mb = rb.vol * rb.rho;
        wi += rb.vol * w;
        num += mb * w;
        sx += mb * ((rb.vx - ra.vx) * (sr * dx));
        sy += mb * ((rb.vy - ra.vy) * (sr * dy));
    });
    if (valid) {
        const int a = P.perm[k];
        const T rho = num / wi;
        P.rho[a] = (double)rho;
        P.drho[a] = -rho * (sx / rho + sy / rho);
        RecA<T> r2;
        r2.vx = ra.vx; r2.vy = ra.vy; r2.vol = (T)(P.mass[a] / (double)rho); r2.rho = rho;
        P.recA2[k] = r2;
        P.countiac[a] = hits;
        if (P.hmask) P.hmask[k] = mask;
    }
    count_stats(cnt, 0, 0, hits, valid);
}

// ----------------------------------------------------------- water: pass A
// Two-phase (SINGLE = false), declarations_sph.f90:1195-1233:
//   con_density :2402, delta_sph(rho) :2658, shear_strain_rate :2855,
//   pressure :2133 (Tait with vof, c ~ (rho/rho0 vof)^3), newtonian_fluid :2484.
// Water-only (SINGLE = true), declarations_sph.f90:1471-1490:
//   delta_sph on the summation density, Tait without vof, t = df(v) form.
// delta_sph's (dx . grad W) 2 (f_a - f_b) / r^2 is evaluated as 2 s (f_a - f_b)
// since grad W = s dx.
template <typename T, int SKF, bool SINGLE>
__global__ void __launch_bounds__(SPHG_TPB, sizeof(T) == 4 ? SPHG_MINB_A : 1) k_water_pass_a(PhaseDev<T> P, GridGeom g, SearchConst sc, SimConst c, DevCounters* cnt) {
    pdl_enter();
    const int k = gtid();
    const bool valid = k < P.n;
    const int kk = valid ? k : 0;
    const int a = P.perm[kk];
    const double2 xa = P.xs[kk];
    const double ha = P.hs[kk];
    const RecA<T>* __restrict__ rec = SINGLE ? P.recA2 : P.recA;
    const RecA<T> ra = rec[kk];
    const T pref = (T)(c.delta * ha * P.c[a]);   // delta*hsml(i)*c(i), c of the previous EOS call
    const T c23 = (T)SPHG_F32LIT(2.0f / 3.0f);
    const bool dens = c.artificial_density;
    KernelConst<T, SKF> ka;
    ka.init((T)ha);
    T con = 0, dl = 0, t0 = 0, t1 = 0, t2 = 0, t3 = 0;
    uint4 mask = make_uint4(0u, 0u, 0u, 0u);
    if (SINGLE && valid) mask = P.hmask[k];   // recorded by k_water_sum
    auto body = [&](const RecA<T>* R, int m, T dx, T dy) {
        const RecA<T> rb = R[m];
        T w, sr, r2, mh;
        pair_kernel<T, SKF>(ka, sc, ha, P.hs, m, dx, dy, w, sr, r2, mh);
        const T gx = sr * dx, gy = sr * dy;
        if (!SINGLE) con += (rb.vol * rb.rho) * ((ra.vx - rb.vx) * gx + (ra.vy - rb.vy) * gy);
        if (dens) dl += pref * rb.vol * ((ra.rho - rb.rho) * (T(2) * sr));
        if (SINGLE) {   // df(vx,'x'), df(vy,'y'), df(vx,'y'), df(vy,'x')
            const T su = ra.vx + rb.vx, sv = ra.vy + rb.vy;
            t0 += rb.vol * (su * gx);
            t1 += rb.vol * (sv * gy);
            t2 += rb.vol * (su * gy);
            t3 += rb.vol * (sv * gx);
        } else {        // shear_strain_rate, dv = v_b - v_a
            const T du = rb.vx - ra.vx, dv = rb.vy - ra.vy;
            t0 += rb.vol * (c23 * (T(2) * du * gx - dv * gy));
            t1 += rb.vol * (du * gy + dv * gx);
            t2 += rb.vol * (c23 * (T(2) * dv * gy - du * gx));
        }
    };
    int hits;
    if constexpr (SINGLE) {
        hits = visit_masked<T>(g, sc, P.cell_start, P.xs, P.hs, xa, ha, k, valid, mask,
                               [&](int m, T dx, T dy) { body(rec, m, dx, dy); });
    } else {
        // neighbours staged in shared memory when they fit (positions and records)
        extern __shared__ __align__(128) unsigned char stage_mem[];
        __shared__ StageHdr H;
        const int cap = stage_capacity(16 + (int)sizeof(RecA<T>));
        int cx, cy;
        bool cl;
        cell_coords(g, xa.x, xa.y, cx, cy, cl);
        const CandRuns cr = candidate_runs(g, P.cell_start, xa, valid);
        StageArrays<2> A;
        A.src[0] = P.xs; A.dst[0] = stage_mem; A.esize[0] = 16;
        A.src[1] = rec; A.dst[1] = stage_mem + (size_t)cap * 16; A.esize[1] = (int)sizeof(RecA<T>);
        if (cap > 0 && stage_block<SPHG_TPB, 2>(H, A, g, P.cell_start, P.xs, P.n, cap, sc.uniform, cx, cy, valid,
                                                 &cnt->timeout)) {
            int self_s;
            const CandRuns sr = staged_runs(H, cr, cy, k, self_s);
            const double2* sxs = (const double2*)stage_mem;
            const RecA<T>* sA = (const RecA<T>*)(stage_mem + (size_t)cap * 16);
            hits = scan_direct<true, T>(sc, sr, sxs, P.hs, xa, ha, self_s, mask,
                                        [&](int m, T dx, T dy) { body(sA, m, dx, dy); });
        } else {   // rare: the block's runs do not fit
            hits = scan_direct<true, T>(sc, cr, P.xs, P.hs, xa, ha, k, mask,
                                        [&](int m, T dx, T dy) { body(rec, m, dx, dy); });
        }
    }
    if (valid) {
        T txx, txy, tyy, drho;
        double p, cnew, vof;
        const double rho = P.rho[a];
        if (SINGLE) {
            drho = P.drho[a] + dl;
            txx = c23 * (T(2) * t0 - t1);
            txy = t2 + t3;
            tyy = c23 * (T(2) * t1 - t0);
            p = P.p[a];
            if (rho > 0.0) p = c.tab[P.sid[a]].w_b * (pow(rho / c.w_rho0, c.w_gamma) - 1);
            cnew = P.c[a];
            vof = 1.0;
        } else {
            drho = con + dl;
            txx = t0; txy = t1; tyy = t2;
            vof = P.vof[a];
            const double ratio = rho / (c.w_rho0 * vof);
            const SceneTab& st = c.tab[P.sid[a]];
            p = st.w_b * (pow(ratio, c.w_gamma) - 1);
            cnew = st.w_c * pow(ratio, 3.0);
            P.c[a] = cnew;
        }
        P.drho[a] = drho;
        P.p[a] = p;
        // newtonian_fluid: sxx = mu*txx in place (sxx and txx are one array)
        const double sxx = c.w_mu * (double)txx, sxy = c.w_mu * (double)txy, syy = c.w_mu * (double)tyy;
        P.sxx[a] = sxx; P.sxy[a] = sxy; P.syy[a] = syy;
        RecB<T> rb;
        rb.p = (T)p; rb.c = (T)cnew; rb.vof = (T)vof;
        rb.sxx = (T)sxx; rb.sxy = (T)sxy; rb.syy = (T)syy;
        rb.itype = (T)P.itype[a]; rb.aux = T(0);
        P.recB[k] = rb;
        P.countiac[a] = hits;
        if (!SINGLE) P.hmask[k] = mask;
    }
    if (!SINGLE) count_stats(cnt, 0, 0, hits, valid);
}

// ------------------------------------------------------------- cross phase
// Neighbour sums over the water x soil pairs (direct_find_2
// m_particles.f90:1004), run inside the last same-phase pass of each phase.
// Neighbours come from the other phase's records of this step.  FCH: the
// Forchheimer drag, each pair's Darcy term scaled by (1 + k b |v_w - v_s|).
//
// Soil side: darcy_law :3832 and pore_water_pressure :3877; the gradient is
// taken, as the reference does, with dx = x_water - x_soil.  With m =
// vol*rho, Darcy's m_w*cf*(v_w - v_s)*W/(rho_w rho_s) becomes
// vol_w*rho_w*vof_w*vof_s*(-g/k)*(v_w - v_s)*W/rho_s; the sums here are the
// pair parts, the particle factors are applied by the caller.  The pore
// pressure m_w p_w/(rho_w rho_s) becomes vol_w p_w / rho_s.
template <typename T, int SKF, bool FCH, class HB>
__device__ __forceinline__ void cross_soil_sums(HB& hb, const PhaseDev<T>& W, const GridGeom& g, const SearchConst& sc,
                                                const SimConst& c, const KernelConst<T, SKF>& ka, double2 xa, double ha,
                                                const RecA<T>& ra, bool valid, T& ddx, T& ddy, T& dpx, T& dpy) {
    visit_batched(hb, g, sc, W.cell_start, W.xs, W.hs, xa, ha, -1, valid, [&](int m, T dx, T dy) {
        const RecA<T> rb = W.recA[m];
        const RecB<T> qb = W.recB[m];
        T w, sr, rr, mh;
        pair_kernel<T, SKF>(ka, sc, ha, W.hs, m, dx, dy, w, sr, rr, mh);
        // x_water - x_soil = -(x_a - x_b)
        const T gx = -sr * dx, gy = -sr * dy;
        T q = rb.vol * rb.rho * qb.vof * w;
        const T ux = rb.vx - ra.vx, uy = rb.vy - ra.vy;
        if constexpr (FCH) q *= T(1) + (T)c.s_kb * sqrt(ux * ux + uy * uy);
        ddx += q * ux;
        ddy += q * uy;
        const T mp = rb.vol * qb.p;
        dpx += mp * gx;
        dpy += mp * gy;
    });
}

// Water side: darcy_law :3832, volume_fraction_water2 :3940 (dvof) and
// volume_fraction_water :3912 (vof2).  Returns the number of pairs.
template <typename T, int SKF, bool FCH, class HB>
__device__ __forceinline__ int cross_water_sums(HB& hb, const PhaseDev<T>& S, const GridGeom& g, const SearchConst& sc,
                                                const SimConst& c, const KernelConst<T, SKF>& ka, double2 xa, double ha,
                                                const RecA<T>& ra, bool valid, T& ddx, T& ddy, T& dvof, T& v2) {
    return visit_batched(hb, g, sc, S.cell_start, S.xs, S.hs, xa, ha, -1, valid, [&](int m, T dx, T dy) {
        const RecA<T> rb = S.recA[m];
        const T phis = S.recB[m].vof;
        T w, sr, rr, mh;
        pair_kernel<T, SKF>(ka, sc, ha, S.hs, m, dx, dy, w, sr, rr, mh);
        const T mb = rb.vol * rb.rho;
        const T ux = ra.vx - rb.vx, uy = ra.vy - rb.vy;
        T q = rb.vol * phis * w;
        if constexpr (FCH) q *= T(1) + (T)c.s_kb * sqrt(ux * ux + uy * uy);
        ddx -= q * ux;
        ddy -= q * uy;
        dvof -= mb * (sr * (ux * dx + uy * dy));
        v2 += mb * w;
    });
}

// ----------------------------------------------------------- water: pass B
// Momentum dv = (-vof*df(p) + df(vof*sxx) + df(vof*sxy)) / rho
// (declarations_sph.f90:1257-1265; df m_particles.f90:1711), art_visc :2504,
// delta_sph(vof) :2658, repulsive_force :1605, gravity, av_vel :2761.
// The water-only step (declarations_sph.f90:1494-1518) is the same with
// vof = 1 and neither wall force nor delta-SPH on vof.  The wall force takes
// dx = x_real - x_virtual, as the reference does with real particles
// numbered before virtual ones.
//
// Two-phase (SINGLE = false): the water side of the cross pairs follows in
// the same kernel (cross_water_sums), then the renormalisation rho <-
// rho/vof*vof2, vof <- vof2 every renorm_interval steps
// (declarations_sph.f90:1414-1421), then, as the last pass of the water
// phase, the leapfrog corrector.  FCH as in cross_water_sums.
template <typename T, int SKF, bool SINGLE, bool FCH>
__global__ void __launch_bounds__(SPHG_TPB, sizeof(T) == 4 ? SPHG_MINB_B : 1) k_water_pass_b(PhaseDev<T> P, PhaseDev<T> S, GridGeom g, SearchConst sc,
                                                          SearchConst scx, SimConst c, StepCtl u, DevCounters* cnt) {
    pdl_enter();
    typedef typename V2<T>::t T2;
    SPHG_HITBUF(T);
    const int k = gtid();
    const bool valid = k < P.n;
    const int kk = valid ? k : 0;
    const int a = P.perm[kk];
    const double2 xa = P.xs[kk];
    const double ha = P.hs[kk];
    const RecA<T>* __restrict__ rec = SINGLE ? P.recA2 : P.recA;
    const RecA<T> ra = rec[kk];
    const RecB<T> qa = P.recB[kk];
    const bool real_a = P.itype[a] > 0;
    const T phia = qa.vof;
    const T fa_xx = phia * qa.sxx, fa_xy = phia * qa.sxy, fa_yy = phia * qa.syy;
    const T pref = (T)(c.delta * ha) * qa.c;
    const T alpha = (T)c.alpha, beta = (T)c.beta, etq2 = (T)(c.etq * c.etq);
    const T r0 = (T)P.dspp, dd = (T)c.dd, p1 = (T)c.p1, p2 = (T)c.p2;
    const bool do_rep = !SINGLE && real_a;
    const bool do_dvof = !SINGLE && c.water_artificial_volume;
    const bool visc = c.visc_artificial, xsph = c.average_velocity;
    KernelConst<T, SKF> ka;
    ka.init((T)ha);
    // x/y pairs: d1 = sum vb (pa+pb) gradW; d2 = sum vb (sxx, sxy) dW/dx;
    // d3 = sum vb (sxy, syy) dW/dy; av, rp, xv as art_visc, repulsive_force, av_vel
    T2 d1 = splat2(T(0)), d2 = splat2(T(0)), d3 = splat2(T(0)), av = splat2(T(0)), rp = splat2(T(0)), xv = splat2(T(0));
    T dvf = 0;
    T2 fa_a, fa_b, va;
    fa_a.x = fa_xx; fa_a.y = fa_xy; fa_b.x = fa_xy; fa_b.y = fa_yy;
    va.x = ra.vx; va.y = ra.vy;
    const uint4 mask = valid ? P.hmask[k] : make_uint4(0u, 0u, 0u, 0u);   // recorded by the step's first water pass
    auto body = [&](const RecA<T>* RA, const RecB<T>* RB, int m, T dx, T dy) {
        const RecA<T> rb = RA[m];
        const RecB<T> qb = RB[m];
        T w, sr, rr, mh;
        pair_kernel<T, SKF>(ka, sc, ha, P.hs, m, dx, dy, w, sr, rr, mh);
        T2 d, vb2;
        d.x = dx; d.y = dy;
        vb2.x = rb.vx; vb2.y = rb.vy;
        const T2 gr = mul2(splat2(sr), d);                       // (gx, gy)
        const T vb = rb.vol;
        const T pp = qa.p + qb.p;
        d1 = fma2(splat2(vb), mul2(splat2(pp), gr), d1);
        T2 sb_a, sb_b;                                           // (sxx, sxy), (sxy, syy) of the neighbour
        sb_a.x = qb.sxx; sb_a.y = qb.sxy; sb_b.x = qb.sxy; sb_b.y = qb.syy;
        const T2 s_a = fma2(splat2(qb.vof), sb_a, fa_a);          // phi_a s_a + phi_b s_b
        const T2 s_b = fma2(splat2(qb.vof), sb_b, fa_b);
        d2 = fma2(splat2(vb), mul2(s_a, splat2(gr.x)), d2);
        d3 = fma2(splat2(vb), mul2(s_b, splat2(gr.y)), d3);
        const T2 dv = sub2(va, vb2);                              // v_a - v_b
        const T mb = vb * rb.rho;
        const T irho = rcp_<T>(T(0.5) * (ra.rho + rb.rho));       // 1 / mean density (art_visc and av_vel)
        if (visc) {
            const T vr = dv.x * dx + dv.y * dy;
            if (vr < T(0)) {
                const T muv = div_<T>(mh * vr, rr + mh * mh * etq2);
                const T mc = T(0.5) * (qa.c + qb.c);
                const T piv = ((beta * muv - alpha * mc) * muv) * irho;
                av = fma2(splat2(-mb), mul2(splat2(piv), gr), av);
            }
        }
        if (do_dvof) dvf += pref * vb * ((phia - qb.vof) * (T(2) * sr));
        if (do_rep && qb.itype < T(0)) {
            const T r = sqrt(rr);
            if (!(r > r0)) {
                const T f = (powr_<T>(r0 / r, p1) - powr_<T>(r0 / r, p2)) / (r * r);
                rp = fma2(mul2(splat2(dd), d), splat2(f), rp);
            }
        }
        if (xsph) {
            const T q = (mb * w) * irho;
            xv = fma2(splat2(-q), dv, xv);
        }
    };
    // Neighbours read through L1, not staged in shared memory: staging them
    // (positions and both records, up to 560 per block) cut the resident
    // blocks to 6 per SM and measured 179 us per launch at 912,016 particles
    // against 164 us for this form at 7 blocks.  Loading each lane's next
    // hit's records during the current one (16 more registers) measured 210
    // us at 6 blocks.
    visit_masked<T>(g, sc, P.cell_start, P.xs, P.hs, xa, ha, k, valid, mask,
                    [&](int m, T dx, T dy) { body(rec, P.recB, m, dx, dy); });
    const T d1x = d1.x, d1y = d1.y, d2x = d2.x, d2y = d2.y, d3x = d3.x, d3y = d3.y;
    const T avx = av.x, avy = av.y, rpx = rp.x, rpy = rp.y, xsx = xv.x, xsy = xv.y;
    T dvx = -(phia * d1x) + d2x + d3x;
    T dvy = -(phia * d1y) + d2y + d3y;
    if (ra.rho > T(0)) { dvx = dvx / ra.rho; dvy = dvy / ra.rho; }
    dvx = dvx + avx + rpx;
    dvy = dvy + avy + rpy + (T)c.gravity;
    if (valid && xsph) {
        const T eps = (T)c.epsilon;
        T2 av; av.x = real_a ? eps * xsx : xsx; av.y = real_a ? eps * xsy : xsy;
        P.av[a] = av;
    }
    if constexpr (SINGLE) {
        if (valid) {
            T2 o; o.x = dvx; o.y = dvy;
            P.dv[a] = o;
            if (u.update) update_one(P, a, c, u.first, 0, 0);   // last pass of the water-only step
            if (u.ncount) cell_key(g, P.x[a], a, P.cell_id, P.cell_fill, u.ncount, cnt, 1);
        }
    } else {
        T cdx = 0, cdy = 0, cdvof = 0, cv2 = 0;
        const int chits = cross_water_sums<T, SKF, FCH>(hb, S, g, scx, c, ka, xa, ha, ra, valid, cdx, cdy, cdvof, cv2);
        if (valid) {
            const T fd = phia * (T)(-c.numeric_gravity / c.s_perm);
            T2 o; o.x = dvx + fd * cdx; o.y = dvy + fd * cdy;
            P.dv[a] = o;
            if (c.volume_fraction) {
                const T irho0 = (T)(1.0 / c.s_rho0);
                P.dvof[a] = dvf + cdvof * irho0;
                const T vof2 = T(1) - cv2 * irho0;
                P.vof2[a] = vof2;
                if (c.renorm_now) {
                    double rho = P.rho[a] / P.vof[a];
                    P.vof[a] = (double)vof2;
                    P.rho[a] = rho * (double)vof2;
                }
            } else {
                P.dvof[a] = dvf;
            }
            P.countiac[a] = chits;
            if (u.update) update_one(P, a, c, u.first, u.with_vof, 0);   // last pass of the water phase
            if (u.ncount) cell_key(g, P.x[a], a, P.cell_id, P.cell_fill, u.ncount, cnt, 1);
        }
        count_stats(cnt, 2, -1, chits, valid);
    }
}

// ------------------------------------------------------------------ soil
// Same-phase soil terms in one pass (declarations_sph.f90:1195-1373 for the
// two-phase step, :1546-1645 for the soil-only step): con_density,
// delta_sph(rho), shear_strain_rate, velocity_divergence, momentum (df3 of
// vof-weighted p and s two-phase, df soil-only), art_visc, delta_sph on p and
// s, repulsive_force (two-phase only), gravity, av_vel; then per particle
// plastic_or_not :3447, plastic_flow_rule3 :3700 and Jaumann_rate :3047,
// whose spin sum wxy comes from the same pass.
//
// Two-phase (SINGLE = false): the soil side of the cross pairs follows in the
// same kernel (cross_soil_sums), then volume_fraction_soil :3970 and, as the
// last pass of the soil phase, the leapfrog corrector.  FCH as in
// cross_soil_sums.
template <typename T, int SKF, bool SINGLE, bool FCH>
__global__ void __launch_bounds__(SPHG_TPB, sizeof(T) == 4 ? SPHG_MINB_SOIL : 1) k_soil_pass(PhaseDev<T> P, PhaseDev<T> W, GridGeom g, SearchConst sc,
                                                       SearchConst scx, SimConst c, DevCounters* cnt, int slot, StepCtl u) {
    pdl_enter();
    typedef typename V2<T>::t T2;
    SPHG_HITBUF(T);
    const int k = gtid();
    const bool valid = k < P.n;
    const int kk = valid ? k : 0;
    const int a = P.perm[kk];
    const double2 xa = P.xs[kk];
    const double ha = P.hs[kk];
    const RecA<T> ra = P.recA[kk];
    const RecB<T> qa = P.recB[kk];
    const bool real_a = P.itype[a] > 0;
    const T cs = (T)c.s_c;                          // pressure(): c = soil%c
    const T pref_old = (T)(c.delta * ha) * qa.c;    // delta_sph(rho) runs before pressure()
    const T pref = (T)(c.delta * ha) * cs;
    const T c23 = (T)SPHG_F32LIT(2.0f / 3.0f);
    const T alpha = (T)c.alpha, beta = (T)c.beta, etq2 = (T)(c.etq * c.etq);
    const T r0 = (T)P.dspp, dd = (T)c.dd, p1 = (T)c.p1, p2 = (T)c.p2;
    const T phia = SINGLE ? T(1) : qa.vof;
    const T fap = phia * qa.p, faxx = phia * qa.sxx, faxy = phia * qa.sxy, fayy = phia * qa.syy;
    const T ira2 = T(1) / (ra.rho * ra.rho);
    const bool dens = c.artificial_density, visc = c.visc_artificial, xsph = c.average_velocity;
    const bool dstress = c.soil_artificial_stress, do_rep = !SINGLE && real_a;
    KernelConst<T, SKF> ka;
    ka.init((T)ha);
    T con = 0, dl = 0, txx = 0, txy = 0, tyy = 0, vcc = 0, wxy = 0;
    T s1x = 0, s1y = 0, s2x = 0, s3x = 0, s2y = 0, s3y = 0;
    T avx = 0, avy = 0, rpx = 0, rpy = 0, xsx = 0, xsy = 0;
    T dpp = 0, dsx = 0, dsxy = 0, dsy = 0;
    const int hits = visit_batched(hb, g, sc, P.cell_start, P.xs, P.hs, xa, ha, k, valid, [&](int m, T dx, T dy) {
        const RecA<T> rb = P.recA[m];
        const RecB<T> qb = P.recB[m];
        T w, sr, rr, mh;
        pair_kernel<T, SKF>(ka, sc, ha, P.hs, m, dx, dy, w, sr, rr, mh);
        const T gx = sr * dx, gy = sr * dy;
        const T du = rb.vx - ra.vx, dv = rb.vy - ra.vy;   // v_b - v_a
        const T vb = rb.vol, mb = vb * rb.rho;
        const T e = T(2) * sr;                            // 2 (dx . grad W) / r^2
        con -= mb * (du * gx + dv * gy);
        if (dens) dl += pref_old * vb * ((ra.rho - rb.rho) * e);
        txx += vb * (c23 * (T(2) * du * gx - dv * gy));
        txy += vb * (du * gy + dv * gx);
        tyy += vb * (c23 * (T(2) * dv * gy - du * gx));
        vcc += vb * (du * gx + dv * gy);
        wxy += vb * (T(0.5) * (du * gy - dv * gx));
        if (SINGLE) {       // df: m_b/rho_b (f_a + f_b) gradW
            const T pp = fap + qb.p;
            s1x += vb * (pp * gx); s1y += vb * (pp * gy);
            s2x += vb * ((faxx + qb.sxx) * gx);
            s3x += vb * ((faxy + qb.sxy) * gy);
            s2y += vb * ((faxy + qb.sxy) * gx);
            s3y += vb * ((fayy + qb.syy) * gy);
        } else {            // df3: m_b (f_a/rho_a^2 + f_b/rho_b^2) gradW
            const T irb = rcp_<T>(rb.rho);
            const T ib = qb.vof * irb * irb;
            const T pp = fap * ira2 + qb.p * ib;
            s1x += mb * (pp * gx); s1y += mb * (pp * gy);
            const T xx = faxx * ira2 + qb.sxx * ib;
            const T xy = faxy * ira2 + qb.sxy * ib;
            const T yy = fayy * ira2 + qb.syy * ib;
            s2x += mb * (xx * gx);
            s3x += mb * (xy * gy);
            s2y += mb * (xy * gx);
            s3y += mb * (yy * gy);
        }
        if (visc) {
            const T vr = -(du * dx + dv * dy);
            if (vr < T(0)) {
                const T muv = div_<T>(mh * vr, rr + mh * mh * etq2);
                const T mrho = T(0.5) * (ra.rho + rb.rho);
                const T piv = div_<T>((beta * muv - alpha * cs) * muv, mrho);
                avx -= mb * (piv * gx);
                avy -= mb * (piv * gy);
            }
        }
        if (dstress) {
            const T q = pref * vb * e;
            dpp += q * (qa.p - qb.p);
            dsx += q * (qa.sxx - qb.sxx);
            dsxy += q * (qa.sxy - qb.sxy);
            dsy += q * (qa.syy - qb.syy);
        }
        if (do_rep && qb.itype < T(0)) {
            const T r = sqrt(rr);
            if (!(r > r0)) {
                const T f = (powr_<T>(r0 / r, p1) - powr_<T>(r0 / r, p2)) / (r * r);
                rpx += dd * dx * f;
                rpy += dd * dy * f;
            }
        }
        if (xsph) {
            const T q = div_<T>(mb * w, (ra.rho + rb.rho) / T(2));
            xsx += q * du;
            xsy += q * dv;
        }
    });
    int fail = 0, fail3 = 0;
    T dvx, dvy;
    if (SINGLE) { dvx = -s1x + s2x + s3x; dvy = -s1y + s2y + s3y; }
    else {
        dvx = -(s1x * ra.rho) + s2x * ra.rho + s3x * ra.rho;
        dvy = -(s1y * ra.rho) + s2y * ra.rho + s3y * ra.rho;
    }
    if (ra.rho > T(0)) { dvx = dvx / ra.rho; dvy = dvy / ra.rho; }
    dvx = dvx + avx + rpx;
    dvy = dvy + avy + rpy + (T)c.gravity;
    if (valid) {
        if (SINGLE) { T2 o; o.x = dvx; o.y = dvy; P.dv[a] = o; }
        if (xsph) {
            const T eps = (T)c.epsilon;
            T2 av; av.x = real_a ? eps * xsx : xsx; av.y = real_a ? eps * xsy : xsy;
            P.av[a] = av;
        }
        P.drho[a] = con + dl;
        // plastic_or_not + plastic_flow_rule3 + Jaumann_rate on the post-DP state
        const double p = P.p[a], sxx = P.sxx[a], sxy = P.sxy[a], syy = P.syy[a];
        const double dtxx = (double)txx, dtxy = (double)txy, dtyy = (double)tyy, dvcc = (double)vcc;
        const double G = c.s_E / (2.0 * (1 + c.s_niu));
        double ds0 = 0.0, ds1 = 0.0, ds2 = 0.0, dp = 0.0;
        if (c.plasticity == 3) {
            const double J2a = sqrt((sxx * sxx + 2.0 * (sxy * sxy) + syy * syy + (sxx + syy) * (sxx + syy)) / 2.0) + 1.0e-6;
            const double alpha1 = c.tab[P.sid[a]].s_alpha1;
            if (fabs(J2a - alpha1 * (3.0 * p)) < SPHG_F32LIT(1.0e-5f)) fail = 1;
            P.fail[a] = fail;
            if (fail) {
                const double exx = dtxx / 2.0 + dvcc / 3.0, exy = dtxy / 2.0, eyy = dtyy / 2.0 + dvcc / 3.0;
                const double sde = sxx * exx + 2.0 * sxy * exy + syy * eyy;
                double J2 = (sxx * sxx + 2.0 * (sxy * sxy) + syy * syy + (sxx + syy) * (sxx + syy)) / 2.0;
                J2 = J2 + 1.0e-10;
                const double al = alpha1, K = c.s_k;
                const double dlambda = (3.0 * al * K * dvcc + G / sqrt(J2) * sde) / (9.0 * (al * al) * K + G);
                if (!(dlambda < 0)) {
                    ds0 = ds0 - dlambda * (G / sqrt(J2) * sxx);
                    ds1 = ds1 - dlambda * (G / sqrt(J2) * sxy);
                    ds2 = ds2 - dlambda * (G / sqrt(J2) * syy);
                    dp = dp + 3.0 * K * al * dlambda;
                    P.eps_p[a] = P.eps_p[a] + dlambda * sxy / (2 * sqrt(J2)) * SPHG_F32LIT(0.000005f);
                }
            }
        }
        const double dwxy = (double)wxy;
        ds0 = ds0 + G * dtxx; ds1 = ds1 + G * dtxy; ds2 = ds2 + G * dtyy;
        dp = dp - c.s_k * dvcc;
        ds0 = ds0 + 2.0 * sxy * dwxy;
        ds1 = ds1 - (sxx - syy) * dwxy;
        ds2 = ds2 - 2.0 * sxy * dwxy;
        P.dsxx[a] = (T)(ds0 + (double)dsx);
        P.dsxy[a] = (T)(ds1 + (double)dsxy);
        P.dsyy[a] = (T)(ds2 + (double)dsy);
        P.dp[a] = (T)(dp + (double)dpp);
        P.c[a] = c.s_c;
        P.txx[a] = txx; P.tyy[a] = tyy; P.txy[a] = wxy;   // wxy is txy (alias)
        P.vcc[a] = vcc;
        P.countiac[a] = hits;
        if (SINGLE && u.update) fail3 = update_one(P, a, c, u.first, 0, u.do_dp);   // last pass of the soil-only step
        if (SINGLE && u.ncount) cell_key(g, P.x[a], a, P.cell_id, P.cell_fill, u.ncount, cnt, 1);
    }
    if constexpr (!SINGLE) {
        T cdx = 0, cdy = 0, cpx = 0, cpy = 0;
        cross_soil_sums<T, SKF, FCH>(hb, W, g, scx, c, ka, xa, ha, ra, valid, cdx, cdy, cpx, cpy);
        if (valid) {
            const T phis = qa.vof;
            const T irs = T(1) / ra.rho;
            const T fd = phis * (T)(-c.numeric_gravity / c.s_perm) * irs, fp = irs * phis;
            T2 o; o.x = dvx + (fd * cdx + fp * cpx); o.y = dvy + (fd * cdy + fp * cpy);
            P.dv[a] = o;
            if (c.volume_fraction) P.vof[a] = P.rho[a] / c.s_rho0;
            if (u.update) fail3 = update_one(P, a, c, u.first, u.with_vof, u.do_dp);   // last pass of the soil phase
            if (u.ncount) cell_key(g, P.x[a], a, P.cell_id, P.cell_fill, u.ncount, cnt, 1);
        }
    }
    count_stats(cnt, slot, slot, hits, valid);
    if (c.plasticity == 3) count_fail(cnt, 2, fail);
    if (u.update && u.do_dp) count_fail(cnt, 3, fail3);
}

// The step's counters and the batch's sticky flags as the host reads them.
struct CounterMirror { DevCounters c; int sticky[4]; };

// Sticky per-batch flags: a pair list above max_interaction (the reference
// stops there, m_particles.f90:992-993) and non-finite positions.  With a
// mirror (mapped pinned host memory) the step's counters and the flags are
// also written there, so the host reads them after its synchronisation with
// no copy of its own.
static __global__ void k_check(const DevCounters* __restrict__ c, int* __restrict__ sticky, unsigned long long cap,
                               CounterMirror* __restrict__ mirror) {
    pdl_enter();
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        const int f[3] = {c->pairs[0] / 2 > cap || c->pairs[1] / 2 > cap || c->pairs[2] > cap, c->nonfinite != 0,
                          c->timeout != 0};
        for (int i = 0; i < 3; ++i)
            if (f[i]) sticky[i] = 1;
        if (mirror) {
            mirror->c = *c;
            for (int i = 0; i < 3; ++i)
                if (f[i]) mirror->sticky[i] = 1;
            __threadfence_system();
        }
    }
}

// ------------------------------------------------------- layout transforms
// Every persistent field of a phase permuted into the current cell order in
// one launch: dst_i[k] = src_i[perm[k]].
struct PermField { const void* src; void* dst; int bytes; int pad; };
struct PermList { int count; int pad; PermField f[44]; };
// Per-step counters to their initial values (a kernel, so that it can live in a graph).
// take_next: the step's cell keys were counted by the previous step's
// corrector, with its clamped and non-finite positions.
static __global__ void k_reset_counters(DevCounters* c, int take_next) {
    pdl_enter();
    int i = threadIdx.x;
    if (i < 3) c->pairs[i] = 0ull;
    if (i < 2) { c->maxiac[i] = 0; c->miniac[i] = 0x7fffffff; c->noiac[i] = 0; }
    if (i < 4) c->nfail[i] = 0;
    if (i == 0) {
        c->n_out = take_next ? c->n_out_next : 0;
        c->nonfinite = take_next ? c->nonfinite_next : 0;
        c->n_out_next = 0; c->nonfinite_next = 0;
        c->overflow = 0; c->timeout = 0;
    }
}

static __global__ void __launch_bounds__(256) k_permute_all(int n, const int* __restrict__ perm, PermList L) {
    pdl_enter();
    int k = gtid();
    if (k >= n) return;
    const int a = perm[k];
    for (int i = 0; i < L.count; ++i) {
        const PermField& f = L.f[i];
        if (f.bytes == 4) ((int*)f.dst)[k] = ((const int*)f.src)[a];
        else if (f.bytes == 8) ((long long*)f.dst)[k] = ((const long long*)f.src)[a];
        else ((int4*)f.dst)[k] = ((const int4*)f.src)[a];
    }
}

// Morton (Z-order) state order: the key of the particle in sorted slot k is
// the interleaved bits of its support-radius cell (x cell / kx, row); the
// stable sort of the slots by key keeps the cell list's order inside a cell.
__device__ __forceinline__ unsigned spread_bits16(unsigned v) {
    v &= 0xffffu;
    v = (v | (v << 8)) & 0x00ff00ffu;
    v = (v | (v << 4)) & 0x0f0f0f0fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}
static __global__ void __launch_bounds__(256) k_morton_keys(int n, const int* __restrict__ perm,
                                                            const int* __restrict__ cell_id, GridGeom g,
                                                            unsigned* __restrict__ key, int* __restrict__ val) {
    pdl_enter();
    const int k = gtid();
    if (k >= n) return;
    const int a = perm[k];
    const int c = cell_id[a];
    key[k] = spread_bits16((unsigned)((c % g.ncx) / g.kx)) | (spread_bits16((unsigned)(c / g.ncx)) << 1);
    val[k] = a;
}
// new state index of each old one (inv[order[j]] = j), then the cell list's
// slots renumbered to the new state indices
static __global__ void __launch_bounds__(256) k_invert(int n, const int* __restrict__ order, int* __restrict__ inv) {
    pdl_enter();
    const int j = gtid();
    if (j < n) inv[order[j]] = j;
}
static __global__ void __launch_bounds__(256) k_renumber(int n, const int* __restrict__ inv, int* __restrict__ perm) {
    pdl_enter();
    const int k = gtid();
    if (k < n) perm[k] = inv[perm[k]];
}

template <typename S>
__global__ void __launch_bounds__(256) k_permute(int n, const int* __restrict__ perm, const S* __restrict__ src, S* __restrict__ dst) {
    int k = gtid();
    if (k < n) dst[k] = src[perm[k]];
}
static __global__ void __launch_bounds__(256) k_iota(int n, int* __restrict__ v) {
    pdl_enter();
    int k = gtid();
    if (k < n) v[k] = k;
}
// state order -> original (Fortran) order, widening to double
template <typename S>
__global__ void __launch_bounds__(256) k_to_original(int n, const int* __restrict__ orig, const S* __restrict__ src,
                                                     double* __restrict__ dst, int comps) {
    int a = gtid();
    if (a >= n) return;
    const S* s = src + (size_t)a * comps;
    double* d = dst + (size_t)orig[a] * comps;
    for (int t = 0; t < comps; ++t) d[t] = (double)s[t];
}
// original order -> state order, narrowing from double
template <typename S>
__global__ void __launch_bounds__(256) k_from_original(int n, const int* __restrict__ orig, const double* __restrict__ src,
                                                       S* __restrict__ dst, int comps) {
    int a = gtid();
    if (a >= n) return;
    const double* s = src + (size_t)orig[a] * comps;
    S* d = dst + (size_t)a * comps;
    for (int t = 0; t < comps; ++t) d[t] = (S)s[t];
}
static __global__ void __launch_bounds__(256) k_to_original_i(int n, const int* __restrict__ orig, const int* __restrict__ src,
                                                       int* __restrict__ dst) {
    int a = gtid();
    if (a < n) dst[orig[a]] = src[a];
}
static __global__ void __launch_bounds__(256) k_from_original_i(int n, const int* __restrict__ orig, const int* __restrict__ src,
                                                         int* __restrict__ dst) {
    int a = gtid();
    if (a < n) dst[a] = src[orig[a]];
}

// Several fields of a phase at once between the state order and the caller's
// original order, through one staging area in which field i occupies
// stage[off, off + n*comps) in original order.  wide: the device field is
// FP64, else of the precision's type S.  One launch per group of fields lets
// the host copies of the group run back to back on the copy engine; each
// field has its own row of blocks (blockIdx.y), so that the fields' loads do
// not wait on one another.
struct XferField { void* dev; long long off; int comps; int wide; };
struct XferList { int count; int pad; XferField f[40]; };
template <typename S>
__global__ void __launch_bounds__(256) k_to_original_all(int n, const int* __restrict__ orig, const __grid_constant__ XferList L,
                                                         double* __restrict__ stage) {
    const int a = gtid();
    if (a >= n || (int)blockIdx.y >= L.count) return;
    const XferField& f = L.f[blockIdx.y];
    double* d = stage + f.off + (size_t)orig[a] * f.comps;
    if (f.wide) {
        const double* s = (const double*)f.dev + (size_t)a * f.comps;
        for (int t = 0; t < f.comps; ++t) d[t] = s[t];
    } else {
        const S* s = (const S*)f.dev + (size_t)a * f.comps;
        for (int t = 0; t < f.comps; ++t) d[t] = (double)s[t];
    }
}
// The water's shared working arrays after a two-phase step (sxx => txx,
// syy => tyy, sxy => txy; declarations_sph.f90:371-377, 414-415): the soil
// pass has written the first n_soil entries with soil values, indexed by the
// soil's original order, and txy holds zero beyond them (Jaumann_rate,
// m_particles.f90:3077).  stage: the water field staged in the water's
// original order (nw entries).
template <typename S>
__global__ void __launch_bounds__(256) k_alias_soil(int ns, int nw, const int* __restrict__ sorig, const S* __restrict__ src,
                                                    double* __restrict__ stage, int zero_tail) {
    const int i = gtid();
    if (i < ns) {
        const int o = sorig[i];
        if (o < nw) stage[o] = (double)src[i];
    } else if (zero_tail && i < nw) {
        stage[i] = 0.0;
    }
}
template <typename S>
__global__ void __launch_bounds__(256) k_from_original_all(int n, const int* __restrict__ orig, const __grid_constant__ XferList L,
                                                           const double* __restrict__ stage) {
    const int a = gtid();
    if (a >= n || (int)blockIdx.y >= L.count) return;
    const XferField& f = L.f[blockIdx.y];
    const double* s = stage + f.off + (size_t)orig[a] * f.comps;
    if (f.wide) {
        double* d = (double*)f.dev + (size_t)a * f.comps;
        for (int t = 0; t < f.comps; ++t) d[t] = s[t];
    } else {
        S* d = (S*)f.dev + (size_t)a * f.comps;
        for (int t = 0; t < f.comps; ++t) d[t] = (S)s[t];
    }
}

// Pair export: per particle (original index i), the neighbours j > i (or, for
// the cross list, every neighbour), sorted, written at offset[i].
static __global__ void __launch_bounds__(SPHG_TPB) k_pairs_count(int n, const int* __restrict__ perm, const int* __restrict__ orig,
                                                          const double2* __restrict__ xs, const double* __restrict__ hs,
                                                          GridGeom g, SearchConst sc, const int* __restrict__ cstart_o,
                                                          const double2* __restrict__ xs_o, const double* __restrict__ hs_o,
                                                          const int* __restrict__ perm_o, const int* __restrict__ orig_o,
                                                          int cross, int* __restrict__ count, int pass, const long long* __restrict__ offset,
                                                          int* __restrict__ out_i, int* __restrict__ out_j, long long cap) {
    int k = gtid();
    if (k >= n) return;
    const int oi = orig[perm[k]];
    const double2 xa = xs[k];
    const double ha = hs[k];
    int cnt = 0;
    long long base = pass ? offset[oi] : 0;
    visit_neighbours(g, sc, cstart_o, xs_o, hs_o, xa, ha, cross ? -1 : k,
        [&](int m, double, double, double, double) {
            const int oj = orig_o[perm_o[m]];
            if (!cross && oj <= oi) return;
            if (pass) {
                long long pos = base + cnt;
                if (pos < cap) { out_i[pos] = oi + 1; out_j[pos] = oj + 1; }
            }
            ++cnt;
        });
    if (!pass) { count[oi] = cnt; return; }
    // sort this particle's j's (few) in place
    long long b = base, e = base + cnt;
    if (e > cap) e = cap;
    for (long long i = b + 1; i < e; ++i) {
        int v = out_j[i];
        long long j = i - 1;
        while (j >= b && out_j[j] > v) { out_j[j + 1] = out_j[j]; --j; }
        out_j[j + 1] = v;
    }
}
