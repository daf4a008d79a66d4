// sphg_device.cuh — device data layout and inline device helpers of libsphg.
//
// Layout in HBM (one `PhaseDev` per phase):
//   * state order: the integrated state (x, v, rho, vof, p, stress, ...) in
//     FP64, one array per field (SoA).  State order is a spatial cell order:
//     the state is permuted into cell order at upload and every
//     `reorder_interval` steps, so elementwise kernels stay coalesced and the
//     per-step permutation stays close to the identity.
//   * rates and per-step sums (drho, dv, av, ds, dp, dvof, txx, ...) in T
//     (double in FP64 mode, float in FP32 mode), state order.
//   * sorted order (rebuilt every step by a counting sort over cells): the
//     positions/h of each particle and the per-neighbour records `recA`
//     (vx, vy, m, rho) and `recB` (p, c, vof, sxx, sxy, syy, itype, -) the pair
//     passes gather.  A pass reads neighbours only from these sorted copies,
//     so it may overwrite the state of its own particle while other threads
//     still read that particle's previous values.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define SPHG_F32LIT(v) ((double)(float)(v))

// pi of m_particles.f90:1483 (a double parameter set from a default-real literal)
#define SPHG_PI_REF 3.1415927410125732

template <typename T> struct V2;
template <> struct V2<double> { typedef double2 t; };
template <> struct V2<float> { typedef float2 t; };
template <typename T> struct V4;
template <> struct V4<double> { typedef double4 t; };
template <> struct V4<float> { typedef float4 t; };

// Sorted-order neighbour records.  Fields are named for what the pair passes
// read: vol = m/rho, so the particle mass is vol*rho; `itype` is stored in T
// (values +-2, +-3 are exact).
template <typename T> struct __align__(4 * sizeof(T)) RecA { T vx, vy, vol, rho; };
template <typename T> struct __align__(4 * sizeof(T)) RecB { T p, c, vof, sxx, sxy, syy, itype, aux; };

// Cell grid.  Rows are one support-radius-sized cell high; along x each such
// cell is split into kx cells, so a particle's neighbours lie in 3 rows of
// 2*kx+1 cells, each row one contiguous run of the cell-sorted list.
struct GridGeom {
    int ncx, ncy;         // cells along x (kx per row cell) and rows
    int kx;               // x cells per support-radius cell (stencil half-width)
    double x0, y0;        // origin
    double inv;           // 1 / row height
    double invx;          // 1 / x cell width (= kx * inv)
};

// Neighbour-search constants of one pair list.
struct SearchConst {
    double scale_k;       // get_scale_k (m_particles.f90:916)
    double r2_uniform;    // exact squared-radius threshold when every h is equal
    int uniform;          // all particles of both lists share one h
};

// The parameters that differ between the scenes of a batched context
// (several independent scenes side by side in one set of arrays); every
// particle carries the index of its scene.  A single scene is entry 0.
struct SceneTab {
    double dt;        // time step
    double w_b;       // water Tait b
    double w_c;       // water reference sound speed
    double s_alpha1;  // Drucker-Prager alpha1 = tan(phi)/sqrt(9+12 tan^2(phi))
};

// Counters the host reads after a batch of steps.
struct DevCounters {
    unsigned long long pairs[3];     // phase 1, phase 2, cross (last step)
    int maxiac[2], miniac[2], noiac[2];
    int nfail[4];                    // soil points flagged by: DP after the predictor,
                                     // in-step DP, plastic_or_not, DP after the corrector
    int n_out;                       // particles clamped into edge cells
    int nonfinite;                   // NaN/Inf positions met
    int overflow;                    // a pair list exceeded max_interaction
    int timeout;                     // blocks whose bounded staging wait ran out
    int n_out_next, nonfinite_next;  // the same, of the positions the corrector wrote for the next step
};

template <typename T>
struct PhaseDev {
    typedef typename V2<T>::t T2;
    int n, ntotal, material;
    double dspp;
    // state order, FP64
    double2 *x, *v, *v_min;
    double *rho, *rho_min, *vof, *vof_min, *p, *c, *mass, *hsml;
    double *sxx, *sxy, *syy, *sxx_min, *sxy_min, *syy_min, *p_min, *eps_p;
    int *itype, *orig, *fail, *sid;
    // state order, T
    T *drho, *dvof, *dsxx, *dsxy, *dsyy, *dp, *txx, *txy, *tyy, *vcc, *wxy, *vof2;
    T2 *dv, *av;
    int *countiac;
    // cell list and sorted copies
    int *cell_id, *cell_fill, *cell_start, *perm;
    double2 *xs;
    double *hs;
    RecA<T> *recA, *recA2;
    RecB<T> *recB;
    // sorted order: which of the particle's candidates passed the pair test in
    // the first same-phase pass of the step (bit t = candidate t of the three
    // row runs; bit 127 alone = more than 127 candidates, not recorded).  The
    // later same-phase passes of the step replay it instead of testing again.
    uint4* hmask;
};

// ---------------------------------------------------------------------------
__device__ __forceinline__ void cell_coords(const GridGeom& g, double x, double y, int& cx, int& cy, bool& clamped) {
    double fx = floor((x - g.x0) * g.invx), fy = floor((y - g.y0) * g.inv);
    clamped = false;
    if (!(fx >= 0.0)) { fx = 0.0; clamped = true; }       // also catches NaN
    if (fx > g.ncx - 1) { fx = g.ncx - 1; clamped = true; }
    if (!(fy >= 0.0)) { fy = 0.0; clamped = true; }
    if (fy > g.ncy - 1) { fy = g.ncy - 1; clamped = true; }
    cx = (int)fx; cy = (int)fy;
}

// kernel, m_particles.f90:1469-1602, dim = 2, gradient with respect to the
// first particle of dx = x_a - x_b.  Evaluated in T in the reference's
// operation order.
template <typename T>
__device__ __forceinline__ void sph_kernel(int skf, T r, T dx, T dy, T h, T& w, T& gx, T& gy) {
    const T pi = (T)SPHG_PI_REF;
    T q = r / h;
    w = T(0); gx = T(0); gy = T(0);
    if (skf == 1) {
        T factor = T(15) / (T(7) * pi * h * h);
        if (q >= T(0) && q <= T(1)) {
            w = factor * ((T)SPHG_F32LIT(2.0f / 3.0f) - q * q + q * q * q / T(2));
            T s = factor * (T(-2) + T(1.5) * q) / (h * h);
            gx = s * dx; gy = s * dy;
        } else if (q > T(1) && q <= T(2)) {
            T u = T(2) - q;
            w = factor * T(1) / T(6) * (u * u * u);
            T s = -(factor * T(1) / T(6) * T(3) * (u * u) / h);
            gx = s * (dx / r); gy = s * (dy / r);
        }
    } else if (skf == 2) {
        T factor = T(1) / ((h * h) * pi);
        if (q >= T(0) && q <= T(3)) {
            w = factor * exp(-q * q);
            gx = w * (T(-2) * dx / h / h); gy = w * (T(-2) * dy / h / h);
        }
    } else if (skf == 3) {
        T factor = T(7) / (T(478) * pi * h * h);
        T a = T(3) - q, b = T(2) - q, c = T(1) - q;
        T a4 = a * a * a * a, b4 = b * b * b * b, c4 = c * c * c * c;
        if (q >= T(0) && q <= T(1)) {
            w = factor * (a4 * a - T(6) * (b4 * b) + T(15) * (c4 * c));
            T s = factor * ((T(-120) + T(120) * q - T(50) * (q * q)) / (h * h));
            gx = s * dx; gy = s * dy;
        } else if (q > T(1) && q <= T(2)) {
            w = factor * (a4 * a - T(6) * (b4 * b));
            T s = factor * (T(-5) * a4 + T(30) * b4) / h;
            gx = s * (dx / r); gy = s * (dy / r);
        } else if (q > T(2) && q <= T(3)) {
            w = factor * (a4 * a);
            T s = factor * (T(-5) * a4) / h;
            gx = s * (dx / r); gy = s * (dy / r);
        }
    } else if (skf == 4) {
        T factor = T(7) / (T(4) * pi * h * h);
        if (q >= T(0) && q <= T(2)) {
            T u = T(1) - q / T(2);
            w = factor * ((u * u * u * u) * (T(1) + T(2) * q));
            T s = factor * (T(-5) + T(15) * q / T(2) - T(15) * (q * q) / T(4) + T(5) * (q * q * q) / T(8)) / (h * h);
            gx = s * dx; gy = s * dy;
        }
    }
}

// Visit every particle of a sorted list whose distance to (xa, ha) passes
// the reference's pair test sqrt(dx^2 + dy^2) < scale_k * (ha + hb)/2
// (m_particles.f90:966-973, 1027-1034) evaluated bit-exactly: unfused
// double products and sum, IEEE sqrt (or its exact squared threshold when
// every h is equal).  `self` (a sorted index) is skipped.
// f(m, dx, dy, r2, mhsml) gets dx = xa - xb.
template <class F>
__device__ __forceinline__ int visit_neighbours(const GridGeom& g, const SearchConst& sc,
                                                const int* __restrict__ cstart,
                                                const double2* __restrict__ xs,
                                                const double* __restrict__ hs,
                                                double2 xa, double ha, int self, F&& f) {
    int cx, cy; bool clamped;
    cell_coords(g, xa.x, xa.y, cx, cy, clamped);
    const int x0 = cx > g.kx ? cx - g.kx : 0;
    const int x1 = cx < g.ncx - 1 - g.kx ? cx + g.kx : g.ncx - 1;
    const int y0 = cy > 0 ? cy - 1 : 0;
    const int y1 = cy < g.ncy - 1 ? cy + 1 : g.ncy - 1;
    int hits = 0;
#pragma unroll 1
    for (int yy = y0; yy <= y1; ++yy) {
        const int beg = __ldg(cstart + yy * g.ncx + x0);
        const int end = __ldg(cstart + yy * g.ncx + x1 + 1);
#pragma unroll 1
        for (int m = beg; m < end; ++m) {
            if (m == self) continue;
            const double2 xb = xs[m];
            const double dx = xa.x - xb.x;
            const double dy = xa.y - xb.y;
            const double r2 = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
            double mh;
            bool hit;
            if (sc.uniform) {
                mh = ha;
                hit = r2 < sc.r2_uniform;
            } else {
                mh = (ha + hs[m]) / 2.0;
                hit = __dsqrt_rn(r2) < sc.scale_k * mh;
            }
            if (hit) { ++hits; f(m, dx, dy, r2, mh); }
        }
    }
    return hits;
}

// Drucker-Prager return, drucker_prager_failure_criterion
// (m_particles.f90:3323-3381).  Returns the fail flag.
__device__ __forceinline__ int dp_return(double& p, double& sxx, double& sxy, double& syy, double alpha1) {
    if (p < 0.0) p = 0.0;
    const double I1 = 3.0 * p;
    double J2 = sxx * sxx + 2.0 * (sxy * sxy) + syy * syy + (sxx + syy) * (sxx + syy);
    J2 = sqrt(J2 / 2.0) + 1.0e-6;
    if (J2 > alpha1 * I1) {
        const double skale = alpha1 * I1 / J2;
        sxx = skale * sxx; sxy = skale * sxy; syy = skale * syy;
        return 1;
    }
    return 0;
}

// x/y pairs of the pair terms.  In FP32 they use Blackwell's packed pair
// arithmetic (fma/mul/add.rn.f32x2: one instruction for both components,
// each rounded as the scalar operation); in FP64 they are two scalar
// operations.  fma2(a, b, c) = a*b + c with one rounding, as the compiler
// contracts the scalar `c += a*b`.
__device__ __forceinline__ float2 splat2(float v) { return make_float2(v, v); }
__device__ __forceinline__ double2 splat2(double v) { return make_double2(v, v); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ double2 mul2(double2 a, double2 b) { return make_double2(a.x * b.x, a.y * b.y); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ double2 add2(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(make_float2(-1.0f, -1.0f), b, a); }
__device__ __forceinline__ double2 sub2(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ double2 fma2(double2 a, double2 b, double2 c) {
    return make_double2(fma(a.x, b.x, c.x), fma(a.y, b.y, c.y));
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ int warp_max(int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ int warp_min(int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}


// ---------------------------------------------------------------------------
// Smoothing kernel with the per-particle constants hoisted out of the pair
// loop (every pair of a particle shares one h when all h are equal).
// eval() returns W and the radial factor s with grad W = s * dx, so that
// dx . grad W = s * r^2.  T = double keeps the IEEE sqrt and divisions of
// the reference's expression; T = float uses rsqrt/reciprocal.
template <typename T> __device__ __forceinline__ T rcp_(T x) { return T(1) / x; }
template <> __device__ __forceinline__ float rcp_<float>(float x) { return __frcp_rn(x); }
template <typename T> __device__ __forceinline__ T div_(T a, T b) { return a / b; }
template <> __device__ __forceinline__ float div_<float>(float a, float b) { return __fdividef(a, b); }

// x^p of the wall force: pow in FP64; in FP32 the fast exp2(p log2 x) (a few
// ulp at the exponents and ranges of the wall force, p = 12 and 4, x >= 1)
template <typename T> __device__ __forceinline__ T powr_(T x, T p) { return pow(x, p); }
template <> __device__ __forceinline__ float powr_<float>(float x, float p) { return __powf(x, p); }

template <typename T> __device__ __forceinline__ T sqsum(T dx, T dy) { return dx * dx + dy * dy; }
template <> __device__ __forceinline__ double sqsum<double>(double dx, double dy) {
    return __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
}

template <typename T, int SKF>
struct KernelConst {
    T h, inv_h, inv_h2, fac;
    __device__ __forceinline__ void init(T hh) {
        const T pi = (T)SPHG_PI_REF;
        h = hh;
        inv_h = T(1) / hh;
        inv_h2 = inv_h * inv_h;
        if (SKF == 1) fac = T(15) / (T(7) * pi * hh * hh);
        else if (SKF == 2) fac = T(1) / ((hh * hh) * pi);
        else if (SKF == 3) fac = T(7) / (T(478) * pi * hh * hh);
        else fac = T(7) / (T(4) * pi * hh * hh);
    }
    // r2 = dx^2 + dy^2 of the pair
    __device__ __forceinline__ void eval(T r2, T& w, T& s) const {
        T r, rinv;
        if (sizeof(T) == 8) { r = sqrt(r2); rinv = T(1) / r; }
        else {
            rinv = (T)rsqrtf((float)fmaxf((float)r2, 1e-30f));
            r = r2 * rinv;
        }
        const T q = sizeof(T) == 8 ? r / h : r * inv_h;
        w = T(0); s = T(0);
        if (SKF == 1) {
            if (q <= T(1)) {
                w = fac * ((T)SPHG_F32LIT(2.0f / 3.0f) - q * q + q * q * q / T(2));
                s = fac * (T(-2) + T(1.5) * q) * inv_h2;
            } else if (q <= T(2)) {
                const T u = T(2) - q;
                w = fac / T(6) * (u * u * u);
                s = -(fac / T(6) * T(3) * (u * u) * inv_h) * rinv;
            }
        } else if (SKF == 2) {
            if (q <= T(3)) {
                w = fac * exp(-q * q);
                s = w * T(-2) * inv_h2;
            }
        } else if (SKF == 3) {
            const T a = T(3) - q, b = T(2) - q, c = T(1) - q;
            const T a4 = a * a * a * a, b4 = b * b * b * b, c4 = c * c * c * c;
            if (q <= T(1)) {
                w = fac * (a4 * a - T(6) * (b4 * b) + T(15) * (c4 * c));
                s = fac * (T(-120) + T(120) * q - T(50) * (q * q)) * inv_h2;   // as m_particles.f90:1554
            } else if (q <= T(2)) {
                w = fac * (a4 * a - T(6) * (b4 * b));
                s = fac * (T(-5) * a4 + T(30) * b4) * inv_h * rinv;
            } else if (q <= T(3)) {
                w = fac * (a4 * a);
                s = fac * (T(-5) * a4) * inv_h * rinv;
            }
        } else {
            if (q <= T(2)) {
                const T u = T(1) - q / T(2);
                w = fac * ((u * u * u * u) * (T(1) + T(2) * q));
                s = fac * (T(-5) + T(15) * q / T(2) - T(15) * (q * q) / T(4) + T(5) * (q * q * q) / T(8)) * inv_h2;
            }
        }
    }
};

// Per-thread hit buffer in shared memory: entry i of thread t at [i*TPB + t],
// so a warp's accesses are conflict-free.  Only the neighbour index is kept;
// dx, dy are recomputed from the sorted positions when the buffer drains,
// which leaves more of the unified L1/shared memory to L1, where the
// neighbour records live.  Measured on a B200 at 912,016 particles and
// dropped: an FP32 prefilter of the candidate test (0.595 -> 0.735 ms per
// step), two neighbours per drain iteration (within 1 %), dx and dy kept in
// the buffer (slower) and an L1 prefetch of the buffered records (no gain).
#ifndef SPHG_SCAN_U
#define SPHG_SCAN_U 4
#endif

template <typename T, int TPB, int CH, typename I = int>
struct HitBuf {
    I m[CH * TPB];
};

// A particle's candidates: the three row runs of the cell-sorted list around
// its cell (rows cy-1, cy, cy+1; cells cx-kx .. cx+kx), numbered 0 .. tot-1
// in that order.
struct CandRuns {
    int b0, b1, b2, L0, L1, L2;
    __device__ __forceinline__ int total() const { return L0 + L1 + L2; }
    // sorted index of candidate t
    __device__ __forceinline__ int at(int t) const {
        return t < L0 ? b0 + t : (t < L0 + L1 ? b1 + (t - L0) : b2 + (t - L0 - L1));
    }
};

__device__ __forceinline__ CandRuns candidate_runs(const GridGeom& g, const int* __restrict__ cstart, double2 xa,
                                                   bool active) {
    CandRuns r{0, 0, 0, 0, 0, 0};
    if (active) {
        int cx, cy; bool clamped;
        cell_coords(g, xa.x, xa.y, cx, cy, clamped);
        const int x0 = cx > g.kx ? cx - g.kx : 0;
        const int x1 = cx < g.ncx - 1 - g.kx ? cx + g.kx : g.ncx - 1;
        if (cy - 1 >= 0) { r.b0 = __ldg(cstart + (cy - 1) * g.ncx + x0); r.L0 = __ldg(cstart + (cy - 1) * g.ncx + x1 + 1) - r.b0; }
        r.b1 = __ldg(cstart + cy * g.ncx + x0); r.L1 = __ldg(cstart + cy * g.ncx + x1 + 1) - r.b1;
        if (cy + 1 < g.ncy) { r.b2 = __ldg(cstart + (cy + 1) * g.ncx + x0); r.L2 = __ldg(cstart + (cy + 1) * g.ncx + x1 + 1) - r.b2; }
    }
    return r;
}

// Hit mask of the candidates (CandRuns numbering) that passed the pair test;
// bit 127 alone marks a particle with more than 127 candidates.
constexpr int SPHG_MASK_BITS = 127;
__device__ __forceinline__ bool mask_overflow(uint4 m) { return m.w == 0x80000000u && !(m.x | m.y | m.z); }

// Every particle of a sorted list that passes the reference's pair test
// against (xa, ha) (m_particles.f90:966-973, 1027-1034), evaluated
// bit-exactly: unfused double products and sum, IEEE sqrt (or its exact
// squared threshold when every h is equal).  `self` (a sorted index) is
// skipped.  Each lane tests its own candidates, U at a time, and keeps the
// hits in its column of `buf`; whenever a lane's column is full, or every
// lane is done, the warp drains its columns through `body(m, dx, dy)` (dx =
// xa - x_m) together, so the pair body runs at full SIMT width.  The visiting
// order is candidate order.  With REC the hits are also returned as a mask.
template <bool REC, int U = SPHG_SCAN_U, typename T, int TPB, int CH, typename I, class F>
__device__ __forceinline__ int scan_runs(HitBuf<T, TPB, CH, I>& buf, const SearchConst& sc, const CandRuns& cr,
                                         const double2* __restrict__ xs, const double* __restrict__ hs, double2 xa,
                                         double ha, int self, uint4& mask, F&& body) {
    const unsigned FULL = 0xffffffffu;
    const int tid = threadIdx.x;
    const int b0 = cr.b0, b1 = cr.b1, b2 = cr.b2, L0 = cr.L0, L1 = cr.L1;
    const int tot = cr.total();
    unsigned long long mlo = 0ull, mhi = 0ull;
    // U: candidates per lane per iteration (independent loads and FP64 chains in flight)
    int t = 0, cnt = 0, hits = 0;
    bool more = true;
    while (more) {
        while (true) {
            more = __any_sync(FULL, t < tot);
            if (!more || __any_sync(FULL, cnt > CH - U)) break;
            int mm[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int tt = t + u;
                mm[u] = tt < L0 ? b0 + tt : (tt < L0 + L1 ? b1 + (tt - L0) : b2 + (tt - L0 - L1));
            }
            double2 xb[U];
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (t + u < tot) xb[u] = xs[mm[u]];
            // exact FP64 test (the reference's operations, m_particles.f90:972-973)
            bool hitu[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                hitu[u] = false;
                if (t + u < tot && mm[u] != self) {
                    const double dx = xa.x - xb[u].x;
                    const double dy = xa.y - xb[u].y;
                    const double r2 = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
                    hitu[u] = sc.uniform ? (r2 < sc.r2_uniform)
                                         : (__dsqrt_rn(r2) < sc.scale_k * ((ha + hs[mm[u]]) / 2.0));
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (hitu[u]) {
                    buf.m[cnt * TPB + tid] = (I)mm[u];
                    ++cnt;
                    ++hits;
                    if (REC) {
                        const int tt = t + u;
                        if (tt < 64) mlo |= 1ull << tt;
                        else mhi |= 1ull << (tt & 63);
                    }
                }
            }
            t = t + U < tot ? t + U : tot;
        }
        for (int i = 0; __any_sync(FULL, i < cnt); ++i) {
            if (i < cnt) {
                const int m = buf.m[i * TPB + tid];
                const double2 xb = xs[m];
                body(m, (T)(xa.x - xb.x), (T)(xa.y - xb.y));
            }
        }
        cnt = 0;
    }
    if (REC) {
        if (tot > SPHG_MASK_BITS) { mlo = 0ull; mhi = 1ull << 63; }
        mask = make_uint4((unsigned)mlo, (unsigned)(mlo >> 32), (unsigned)mhi, (unsigned)(mhi >> 32));
    }
    return hits;
}

template <typename T, int TPB, int CH, class F>
__device__ __forceinline__ int visit_batched(HitBuf<T, TPB, CH>& buf, const GridGeom& g, const SearchConst& sc,
                                             const int* __restrict__ cstart, const double2* __restrict__ xs,
                                             const double* __restrict__ hs, double2 xa, double ha, int self,
                                             bool active, F&& body) {
    uint4 unused;
    return scan_runs<false>(buf, sc, candidate_runs(g, cstart, xa, active), xs, hs, xa, ha, self, unused, body);
}

// visit_batched that also returns the hit mask (CandRuns numbering).
template <typename T, int TPB, int CH, class F>
__device__ __forceinline__ int visit_batched_rec(HitBuf<T, TPB, CH>& buf, const GridGeom& g, const SearchConst& sc,
                                                 const int* __restrict__ cstart, const double2* __restrict__ xs,
                                                 const double* __restrict__ hs, double2 xa, double ha, int self,
                                                 bool active, uint4& mask, F&& body) {
    return scan_runs<true>(buf, sc, candidate_runs(g, cstart, xa, active), xs, hs, xa, ha, self, mask, body);
}

// The same visit without the hit buffer: each lane tests its candidates one
// at a time and runs the body on each hit at once (lanes diverge).  For the
// rare particles and blocks the batched forms do not cover.
template <bool REC, typename T, class F>
__device__ __forceinline__ int scan_direct(const SearchConst& sc, const CandRuns& cr, const double2* __restrict__ xs,
                                           const double* __restrict__ hs, double2 xa, double ha, int self,
                                           uint4& mask, F&& body) {
    unsigned long long mlo = 0ull, mhi = 0ull;
    int hits = 0;
    const int tot = cr.total();
    for (int t = 0; t < tot; ++t) {
        const int m = cr.at(t);
        if (m == self) continue;
        const double2 xb = xs[m];
        const double dx = xa.x - xb.x, dy = xa.y - xb.y;
        const double r2 = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
        const bool hit = sc.uniform ? (r2 < sc.r2_uniform) : (__dsqrt_rn(r2) < sc.scale_k * ((ha + hs[m]) / 2.0));
        if (hit) {
            ++hits;
            if (REC) {
                if (t < 64) mlo |= 1ull << t;
                else mhi |= 1ull << (t & 63);
            }
            body(m, (T)dx, (T)dy);
        }
    }
    if (REC) {
        if (tot > SPHG_MASK_BITS) { mlo = 0ull; mhi = 1ull << 63; }
        mask = make_uint4((unsigned)mlo, (unsigned)(mlo >> 32), (unsigned)mhi, (unsigned)(mhi >> 32));
    }
    return hits;
}

// The same visit replayed from the hit mask an earlier pass of this step
// recorded over the same sorted positions: the same neighbours in the same
// order, so every sum is bit-identical, without testing any candidate again.
// Each lane walks its own set bits.  A lane whose candidates did not fit the
// mask (more than 127, three times the count of an uncompressed lattice)
// tests them again, one at a time, in the same order.
template <typename T, class F>
__device__ __forceinline__ int replay_runs(const SearchConst& sc, const CandRuns& cr, const double2* __restrict__ xs,
                                           const double* __restrict__ hs, double2 xa, double ha, int self,
                                           bool active, uint4 mask, F&& body) {
    const unsigned FULL = 0xffffffffu;
    if (active && mask_overflow(mask)) {
        uint4 unused;
        return scan_direct<false, T>(sc, cr, xs, hs, xa, ha, self, unused, body);
    }
    unsigned long long lo = active ? ((unsigned long long)mask.y << 32 | mask.x) : 0ull;
    unsigned long long hi = active ? ((unsigned long long)mask.w << 32 | mask.z) : 0ull;
    const int hits = __popcll(lo) + __popcll(hi);
    while (__any_sync(FULL, (lo | hi) != 0ull)) {
        if (lo | hi) {
            int t;
            if (lo) { t = __ffsll((long long)lo) - 1; lo &= lo - 1; }
            else { t = 63 + __ffsll((long long)hi); hi &= hi - 1; }
            const int m = cr.at(t);
            const double2 xb = xs[m];
            body(m, (T)(xa.x - xb.x), (T)(xa.y - xb.y));
        }
    }
    return hits;
}

template <typename T, class F>
__device__ __forceinline__ int visit_masked(const GridGeom& g, const SearchConst& sc,
                                            const int* __restrict__ cstart, const double2* __restrict__ xs,
                                            const double* __restrict__ hs, double2 xa, double ha, int self,
                                            bool active, uint4 mask, F&& body) {
    return replay_runs<T>(sc, candidate_runs(g, cstart, xa, active), xs, hs, xa, ha, self, active, mask, body);
}

// ---------------------------------------------------------------------------
// Shared-memory staging of a block's neighbour candidates.
//
// A block's particles are consecutive in the cell-sorted list: they lie in
// one row of cells, or at the end of one row and the start of a later one.
// For each such row part p (row row[p], cells xlo[p] .. xhi[p]) the
// candidates of all its particles lie in three runs of the sorted list: rows
// row[p]-1 .. row[p]+1, cells xlo[p]-kx .. xhi[p]+kx.  Those (at most six)
// runs of each per-neighbour array are copied into shared memory by the
// bulk-copy engine (cp.async.bulk, every copy completing on one mbarrier),
// and the pass reads its neighbours from there.  A block whose runs exceed
// the staging space, whose particles span three non-empty rows, or whose h
// are not all equal reads from global memory instead.
struct StageHdr {
    unsigned long long bar;
    int staged, total, bad;
    int row[2], xlo[2], xhi[2];
    int gbeg[6], len[6], soff[6];
};

template <int NB>
struct StageArrays {
    const void* src[NB];   // global, sorted order
    void* dst[NB];         // shared, room for `cap` elements each
    int esize[NB];         // bytes per element, a multiple of 16
};

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait_parity(unsigned long long* bar, unsigned parity) {
    unsigned done;
    asm volatile("{\n\t.reg .pred P1;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                 "selp.b32 %0, 1, 0, P1;\n\t}"
                 : "=r"(done) : "r"(smem_addr(bar)), "r"(parity) : "memory");
    return done != 0;
}

// Bounded wait on the staging barrier: on running out the block sets the
// timeout counter and waits once more (bounded) for its copies in flight.
constexpr long long SPHG_STAGE_WAIT = 1LL << 22;
__device__ __forceinline__ void stage_wait(StageHdr& H, int* timeout) {
    long long i = 0;
    while (!mbar_try_wait_parity(&H.bar, 0)) {
        if (++i == SPHG_STAGE_WAIT) {
            if (threadIdx.x == 0) atomicAdd(timeout, 1);
            for (long long j = 0; j < SPHG_STAGE_WAIT && !mbar_try_wait_parity(&H.bar, 0); ++j) {}
            return;
        }
    }
}

// Whole block.  (cx, cy): the thread's particle's cell (valid particles).
// Returns true (block-uniform) when the candidates are in shared memory.
template <int TPB, int NB>
__device__ __forceinline__ bool stage_block(StageHdr& H, const StageArrays<NB>& A, const GridGeom& g,
                                            const int* __restrict__ cstart, const double2* __restrict__ xs, int n,
                                            int cap, bool uniform, int cx, int cy, bool valid, int* timeout) {
    const int tid = threadIdx.x;
    if (tid == 0) {
        const int k0 = blockIdx.x * TPB;
        const int k1 = (k0 + TPB < n ? k0 + TPB : n) - 1;
        const double2 p0 = xs[k0], p1 = xs[k1];
        int c0x, c0y, c1x, c1y;
        bool cl;
        cell_coords(g, p0.x, p0.y, c0x, c0y, cl);
        cell_coords(g, p1.x, p1.y, c1x, c1y, cl);
        H.row[0] = c0y; H.row[1] = c1y;
        H.xlo[0] = c0x; H.xhi[0] = c0x; H.xlo[1] = c1x; H.xhi[1] = c1x;
        H.bad = uniform ? 0 : 1;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&H.bar)) : "memory");
    }
    __syncthreads();
    if (valid) {
        if (cy == H.row[0]) atomicMax(&H.xhi[0], cx);
        else if (cy == H.row[1]) atomicMin(&H.xlo[1], cx);
        else H.bad = 1;
    }
    __syncthreads();
    if (tid < 6) {
        const int p = tid / 3, y = H.row[p] + tid % 3 - 1;
        int gb = 0, len = 0;
        if ((p == 0 || H.row[1] != H.row[0]) && y >= 0 && y < g.ncy) {
            const int xl = H.xlo[p] - g.kx > 0 ? H.xlo[p] - g.kx : 0;
            const int xh = H.xhi[p] + g.kx < g.ncx - 1 ? H.xhi[p] + g.kx : g.ncx - 1;
            gb = cstart[y * g.ncx + xl];
            len = cstart[y * g.ncx + xh + 1] - gb;
        }
        H.gbeg[tid] = gb;
        H.len[tid] = len;
    }
    __syncthreads();
    if (tid == 0) {
        int off = 0;
        for (int j = 0; j < 6; ++j) { H.soff[j] = off; off += H.len[j]; }
        H.total = off;
        const int st = !H.bad && off <= cap;
        H.staged = st;
        if (st) {
            unsigned bytes = 0;
            for (int i = 0; i < NB; ++i) bytes += (unsigned)off * (unsigned)A.esize[i];
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(&H.bar)), "r"(bytes)
                         : "memory");
            for (int j = 0; j < 6; ++j) {
                if (H.len[j] <= 0) continue;
                for (int i = 0; i < NB; ++i)
                    bulk_copy_g2s((char*)A.dst[i] + (size_t)H.soff[j] * A.esize[i],
                                  (const char*)A.src[i] + (size_t)H.gbeg[j] * A.esize[i],
                                  (unsigned)H.len[j] * (unsigned)A.esize[i], &H.bar);
            }
        }
    }
    __syncthreads();
    if (!H.staged) return false;
    stage_wait(H, timeout);
    return true;
}

// Room for staged records: the launch's dynamic shared memory over the bytes
// one staged neighbour takes (0 when launched without dynamic shared memory).
__device__ __forceinline__ int stage_capacity(int bytes_per_record) {
    unsigned dyn;
    asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
    return (int)(dyn / (unsigned)bytes_per_record);
}

// A particle's candidate runs as indices into the staged arrays, and its own
// staged index.  cy: the particle's row.
__device__ __forceinline__ CandRuns staged_runs(const StageHdr& H, CandRuns r, int cy, int k, int& self_s) {
    const int j = cy == H.row[0] ? 0 : 3;
    r.b0 = H.soff[j] + (r.b0 - H.gbeg[j]);
    r.b1 = H.soff[j + 1] + (r.b1 - H.gbeg[j + 1]);
    r.b2 = H.soff[j + 2] + (r.b2 - H.gbeg[j + 2]);
    self_s = H.soff[j + 1] + (k - H.gbeg[j + 1]);
    return r;
}
