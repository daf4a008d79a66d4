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

template <typename T, int TPB, int CH>
struct HitBuf {
    int m[CH * TPB];
};

template <typename T, int TPB, int CH, class F>
__device__ __forceinline__ int visit_batched(HitBuf<T, TPB, CH>& buf, const GridGeom& g, const SearchConst& sc,
                                             const int* __restrict__ cstart, const double2* __restrict__ xs,
                                             const double* __restrict__ hs, double2 xa, double ha, int self,
                                             bool active, F&& body) {
    const unsigned FULL = 0xffffffffu;
    const int tid = threadIdx.x;
    int b0 = 0, b1 = 0, b2 = 0, L0 = 0, L1 = 0, L2 = 0;
    if (active) {
        int cx, cy; bool clamped;
        cell_coords(g, xa.x, xa.y, cx, cy, clamped);
        const int x0 = cx > g.kx ? cx - g.kx : 0;
        const int x1 = cx < g.ncx - 1 - g.kx ? cx + g.kx : g.ncx - 1;
        if (cy - 1 >= 0) { b0 = __ldg(cstart + (cy - 1) * g.ncx + x0); L0 = __ldg(cstart + (cy - 1) * g.ncx + x1 + 1) - b0; }
        b1 = __ldg(cstart + cy * g.ncx + x0); L1 = __ldg(cstart + cy * g.ncx + x1 + 1) - b1;
        if (cy + 1 < g.ncy) { b2 = __ldg(cstart + (cy + 1) * g.ncx + x0); L2 = __ldg(cstart + (cy + 1) * g.ncx + x1 + 1) - b2; }
    }
    const int tot = L0 + L1 + L2;
    constexpr int U = SPHG_SCAN_U;   // candidates per lane per iteration: independent loads and FP64 chains in flight
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
                    buf.m[cnt * TPB + tid] = mm[u];
                    ++cnt;
                    ++hits;
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
    return hits;
}
