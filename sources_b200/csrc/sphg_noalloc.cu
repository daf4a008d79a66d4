// sphg_noalloc.cu — summation density (the kernel sum of the water-only step)
// for callers that cannot allocate device memory.
//
// Some hosts cannot call cudaMalloc when they call into this library: a
// Fortran or C program whose device memory is owned by another runtime's
// pool allocator (which may already hold nearly all of the GPU), or a solver
// loop that runs on a fixed, pre-planned memory budget and may not allocate
// or free during its time steps.  sphg_sum_density_noalloc serves them: its
// working memory (cell list, sorted copies, counters) is one file-scope
// __device__ array of fixed size, loaded with the library, so a call
// allocates nothing.  The caller passes device pointers for every input and
// output.
//
// Limits: at most SPHG_NOALLOC_MAX_PARTICLES particles and a neighbour grid
// of at most SPHG_NOALLOC_MAX_CELLS cells; larger requests return
// SPHG_ERR_BAD_ARG without touching the GPU.  Every GPU that loads the
// library holds the array until the process exits.
//
// Sharing: every call, from any context or thread, uses the same array and
// finds the previous call's data in it; the call clears what must start at
// zero.  Calls whose GPU work overlaps (two streams, or two host threads)
// race on the array and must be serialised by the caller.
//
// Set-up: every call looks up the array's device address
// (cudaGetSymbolAddress) with the caller's device current, so the address is
// right even after the caller has reset the device and the module was loaded
// anew.  The first call on a device loads the library's device module, and
// with it the array; that first call should come before any stream capture.
// Every call also waits once on its stream, for the smoothing-length range
// it needs to size the grid and for the finiteness check of the positions.
//
// Errors: NaN or infinite positions return SPHG_ERR_NONFINITE and
// non-positive or non-finite h return SPHG_ERR_BAD_ARG, both before any
// density kernel runs.  Particles outside [x_min, x_max] x [y_min, y_max]
// are clamped into the edge cells of the grid; every x cell is at least one
// support radius wide, so their pairs are still all found.
#include <cuda_runtime.h>

#include <cmath>

#include "../../include/sphg.h"
#include "sphg_kernels.cuh"

namespace {

constexpr int kMaxN = SPHG_NOALLOC_MAX_PARTICLES;
constexpr int kMaxC = SPHG_NOALLOC_MAX_CELLS;

constexpr size_t pad256(size_t b) { return (b + 255) / 256 * 256; }

// byte offsets of each region inside the scratch array
constexpr size_t kOffCnt = 0;
constexpr size_t kOffH = kOffCnt + pad256(sizeof(DevCounters));
constexpr size_t kOffCounts = kOffH + pad256(4 * sizeof(double));
constexpr size_t kOffStart = kOffCounts + pad256(sizeof(int) * (kMaxC + 1));
constexpr size_t kOffCellId = kOffStart + pad256(sizeof(int) * (kMaxC + 1));
constexpr size_t kOffRank = kOffCellId + pad256(sizeof(int) * kMaxN);
constexpr size_t kOffPerm = kOffRank + pad256(sizeof(int) * kMaxN);
constexpr size_t kOffIdent = kOffPerm + pad256(sizeof(int) * kMaxN);
constexpr size_t kOffCount = kOffIdent + pad256(sizeof(int) * kMaxN);
constexpr size_t kOffXs = kOffCount + pad256(sizeof(int) * kMaxN);
constexpr size_t kOffHs = kOffXs + pad256(sizeof(double2) * kMaxN);
constexpr size_t kOffRecA = kOffHs + pad256(sizeof(double) * kMaxN);
constexpr size_t kOffRecA2 = kOffRecA + pad256(sizeof(RecA<double>) * kMaxN);
constexpr size_t kOffDrho = kOffRecA2 + pad256(sizeof(RecA<double>) * kMaxN);
constexpr size_t kBytes = kOffDrho + pad256(sizeof(double) * kMaxN);

}  // namespace

// The working memory of sphg_sum_density_noalloc (about 4.3 MB).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kBytes];

namespace {

// Device address of the scratch array on the current device.
int scratch_base(void** out) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) return SPHG_ERR_CUDA;
    *out = p;
    return SPHG_OK;
}

// smoothing-length range [min, max], a flag for non-positive/non-finite h
// and a flag for non-finite positions: out = {hmin, hmax, bad h, bad x}
__global__ void __launch_bounds__(1024) k_na_hrange(int n, const double* __restrict__ h, const double2* __restrict__ x,
                                                    double* __restrict__ out) {
    __shared__ double smin[32], smax[32];
    __shared__ int sbad[32], sbadx[32];
    double lo = INFINITY, hi = 0.0;
    int bad = 0, badx = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double v = h[i];
        if (!(v > 0.0) || !isfinite(v)) bad = 1;
        lo = fmin(lo, v); hi = fmax(hi, v);
        const double2 p = x[i];
        if (!(isfinite(p.x) && isfinite(p.y))) badx = 1;
    }
    for (int o = 16; o > 0; o >>= 1) {
        lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        bad |= __shfl_xor_sync(0xffffffffu, bad, o);
        badx |= __shfl_xor_sync(0xffffffffu, badx, o);
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) { smin[w] = lo; smax[w] = hi; sbad[w] = bad; sbadx[w] = badx; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 1; i < (int)(blockDim.x >> 5); ++i) {
            lo = fmin(lo, smin[i]); hi = fmax(hi, smax[i]); bad |= sbad[i]; badx |= sbadx[i];
        }
        out[0] = lo; out[1] = hi; out[2] = bad ? 1.0 : 0.0; out[3] = badx ? 1.0 : 0.0;
    }
}

__global__ void __launch_bounds__(256) k_na_zero(int* __restrict__ p, int count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) p[i] = 0;
}

// Exclusive scan of counts[0..m) into start[0..m) by one block of 1024
// threads (m <= kMaxC + 1): each thread scans a contiguous chunk, then the
// chunk totals are scanned in shared memory.
__global__ void __launch_bounds__(1024) k_na_scan(const int* __restrict__ counts, int* __restrict__ start, int m) {
    __shared__ int tot[1024];
    const int t = threadIdx.x;
    const int per = (m + blockDim.x - 1) / blockDim.x;
    const int b = t * per, e = min(b + per, m);
    int s = 0;
    for (int i = b; i < e; ++i) s += counts[i];
    tot[t] = s;
    __syncthreads();
    for (int o = 1; o < (int)blockDim.x; o <<= 1) {
        const int v = t >= o ? tot[t - o] : 0;
        __syncthreads();
        tot[t] += v;
        __syncthreads();
    }
    int run = t > 0 ? tot[t - 1] : 0;
    for (int i = b; i < e; ++i) { start[i] = run; run += counts[i]; }
}

// sorted copies of position, h and (0, 0, vol, rho) for the density sum
__global__ void __launch_bounds__(256) k_na_gather(int n, const int* __restrict__ perm, const double2* __restrict__ x,
                                                   const double* __restrict__ hsml, const double* __restrict__ mass,
                                                   const double* __restrict__ rho, double2* __restrict__ xs,
                                                   double* __restrict__ hs, RecA<double>* __restrict__ rec) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int a = perm[k];
    xs[k] = x[a];
    hs[k] = hsml[a];
    RecA<double> r;
    r.vx = 0.0; r.vy = 0.0; r.vol = mass[a] / rho[a]; r.rho = rho[a];
    rec[k] = r;
}

template <int SKF>
void launch_sum(int n, PhaseDev<double> D, GridGeom g, SearchConst sc, SimConst c, DevCounters* cnt, cudaStream_t s) {
    k_water_sum<double, SKF><<<(n + SPHG_TPB - 1) / SPHG_TPB, SPHG_TPB, 0, s>>>(D, g, sc, c, cnt);
}

}  // namespace

extern "C" int sphg_sum_density_noalloc(const sphg_params* p, int32_t n, const double* x, const double* hsml,
                                        const double* mass, const double* rho, double* rho_out, void* cuda_stream) {
    if (!p || !x || !hsml || !mass || !rho || !rho_out) return SPHG_ERR_BAD_ARG;
    if (p->dim != 2) return SPHG_ERR_BAD_ARG;
    if (p->skf < 1 || p->skf > 4) return SPHG_ERR_BAD_KERNEL;
    if (n < 1 || n > kMaxN) return SPHG_ERR_BAD_ARG;
    if (!(p->x_max > p->x_min) || !(p->y_max > p->y_min)) return SPHG_ERR_BAD_ARG;
    void* base = nullptr;
    int rc = scratch_base(&base);
    if (rc) return rc;
    unsigned char* B = (unsigned char*)base;
    cudaStream_t s = (cudaStream_t)cuda_stream;
    DevCounters* cnt = (DevCounters*)(B + kOffCnt);
    double* hr = (double*)(B + kOffH);

    // smoothing-length range, to size the grid as the other entry points do,
    // and the finiteness of the positions (the step's own check,
    // SPHG_ERR_NONFINITE), before any density kernel runs
    k_na_hrange<<<1, 1024, 0, s>>>(n, hsml, (const double2*)x, hr);
    double hh[4] = {0, 0, 0, 0};
    if (cudaMemcpyAsync(hh, hr, sizeof(hh), cudaMemcpyDeviceToHost, s) != cudaSuccess) return SPHG_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return SPHG_ERR_CUDA;
    if (hh[2] != 0.0) return SPHG_ERR_BAD_ARG;
    if (hh[3] != 0.0) return SPHG_ERR_NONFINITE;
    const int sk = (p->skf == 2 || p->skf == 3) ? 3 : 2;
    const double cell = sk * hh[1] * (1.0 + 1e-6);
    const double ncx = std::ceil((p->x_max - p->x_min) / cell) + 1, ncy = std::ceil((p->y_max - p->y_min) / cell) + 1;
    if (!(ncx * ncy <= (double)kMaxC)) return SPHG_ERR_BAD_ARG;
    GridGeom g;
    g.ncx = (int)ncx; g.ncy = (int)ncy; g.x0 = p->x_min; g.y0 = p->y_min; g.inv = 1.0 / cell;
    g.kx = 1; g.invx = g.inv;
    const int ncell = g.ncx * g.ncy;
    SearchConst sc{};
    sc.scale_k = sk;
    sc.uniform = hh[0] == hh[1];
    sc.r2_uniform = 0.0;
    if (sc.uniform) {   // smallest t with sqrt(t) >= K: sqrt(r2) < K  <=>  r2 < t
        const double K = sk * hh[1];
        double t = K * K;
        while (t > 0 && std::sqrt(t) >= K) t = std::nextafter(t, 0.0);
        while (std::sqrt(t) < K) t = std::nextafter(t, INFINITY);
        sc.r2_uniform = t;
    }

    int* counts = (int*)(B + kOffCounts);
    PhaseDev<double> D;
    memset(&D, 0, sizeof(D));
    D.n = n;
    D.cell_start = (int*)(B + kOffStart);
    D.cell_id = (int*)(B + kOffCellId);
    D.cell_fill = (int*)(B + kOffRank);
    D.perm = (int*)(B + kOffPerm);
    D.orig = (int*)(B + kOffIdent);
    D.countiac = (int*)(B + kOffCount);
    D.xs = (double2*)(B + kOffXs);
    D.hs = (double*)(B + kOffHs);
    D.recA = (RecA<double>*)(B + kOffRecA);
    D.recA2 = (RecA<double>*)(B + kOffRecA2);
    D.drho = (double*)(B + kOffDrho);
    D.mass = const_cast<double*>(mass);
    D.rho = rho_out;

    // what must start at zero: the per-cell counts and the counters
    k_na_zero<<<(ncell + 1 + 255) / 256, 256, 0, s>>>(counts, ncell + 1);
    k_na_zero<<<1, 256, 0, s>>>((int*)cnt, (int)(sizeof(DevCounters) / sizeof(int)));
    k_iota<<<(n + 255) / 256, 256, 0, s>>>(n, D.orig);
    k_cell_count<<<(n + 255) / 256, 256, 0, s>>>((const double2*)x, n, g, D.cell_id, D.cell_fill, counts, cnt, 0);
    k_na_scan<<<1, 1024, 0, s>>>(counts, D.cell_start, ncell + 1);
    k_cell_scatter<<<(n + 255) / 256, 256, 0, s>>>(n, D.cell_id, D.cell_fill, D.cell_start, D.perm);
    k_cell_sort<<<(ncell + 255) / 256, 256, 0, s>>>(ncell, D.cell_start, D.orig, D.perm, counts);
    k_na_gather<<<(n + 255) / 256, 256, 0, s>>>(n, D.perm, (const double2*)x, hsml, mass, rho, D.xs, D.hs, D.recA);
    SimConst c;
    memset(&c, 0, sizeof(c));
    c.skf = p->skf;
    switch (p->skf) {
        case 1: launch_sum<1>(n, D, g, sc, c, cnt, s); break;
        case 2: launch_sum<2>(n, D, g, sc, c, cnt, s); break;
        case 3: launch_sum<3>(n, D, g, sc, c, cnt, s); break;
        default: launch_sum<4>(n, D, g, sc, c, cnt, s); break;
    }
    return cudaGetLastError() == cudaSuccess ? SPHG_OK : SPHG_ERR_CUDA;
}
