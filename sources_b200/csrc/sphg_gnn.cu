// sphg_gnn.cu — graph, feature and element-wise kernels of the learned
// particle stepper (a message-passing network over the particles).  The
// dense layers run on the tcgen05 GEMM of sphg_umma.cu; everything between
// them is here:
//   graph      cell list by counting sort (cell = radius), per-cell index
//              sort, per-receiver degree, CSR fill: edges grouped by
//              receiver, receivers in node order, senders in cell-scan order
//   features   node inputs (velocity history, type, wall distances, scene
//              constants, displacement since a reference state) and edge
//              inputs (offset / radius, distance, same type, change of the
//              offset since the reference state) as bf16 rows of 64
//   layers     segment sums, concatenations and their backward passes,
//              ReLU backward, transposes for the weight-gradient GEMMs,
//              column sums, loss, Adam (bias, activation and the edge
//              layer's gathers are fused into the GEMM epilogues)
//   rollout    stride update of velocity history and position, the
//              number-density and energy sums of the fallback gates
// Feature matrices are row-major (feature index contiguous) with the row
// count padded to a multiple of 128 for the GEMM; padded rows are kept
// finite and their gradients zero.
#include <cub/device/device_scan.cuh>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/sphg.h"
#include "../../include/sphg_learn.h"

namespace {

typedef __nv_bfloat16 bf16;

inline unsigned nb(long long n, int t) { return (unsigned)((n + t - 1) / t); }
__device__ __forceinline__ long long gid() { return (long long)blockIdx.x * blockDim.x + threadIdx.x; }
inline int ok_or_cuda() { return cudaGetLastError() == cudaSuccess ? SPHG_OK : SPHG_ERR_CUDA; }

// ------------------------------------------------------------------ graph

__device__ __forceinline__ int cell_of(double x, double y, double xmin, double ymin, double inv_r, int nx, int ny,
                                       int* cx, int* cy) {
    int ix = (int)floor((x - xmin) * inv_r), iy = (int)floor((y - ymin) * inv_r);
    // clamping keeps every pair closer than the radius in neighbouring cells
    ix = ix < 0 ? 0 : (ix >= nx ? nx - 1 : ix);
    iy = iy < 0 ? 0 : (iy >= ny ? ny - 1 : iy);
    *cx = ix;
    *cy = iy;
    return iy * nx + ix;
}

__global__ void k_graph_count(const double2* __restrict__ x, int n, double xmin, double ymin, double inv_r, int nx,
                              int ny, int* __restrict__ node_cell, int* __restrict__ count) {
    const int i = (int)gid();
    if (i >= n) return;
    int cx, cy;
    const double2 p = x[i];
    const int c = cell_of(p.x, p.y, xmin, ymin, inv_r, nx, ny, &cx, &cy);
    node_cell[i] = c;
    atomicAdd(count + c, 1);
}

__global__ void k_graph_scatter(int n, const int* __restrict__ node_cell, int* __restrict__ cursor,
                                int* __restrict__ order) {
    const int i = (int)gid();
    if (i >= n) return;
    order[atomicAdd(cursor + node_cell[i], 1)] = i;
}

__global__ void k_graph_cell_sort(int ncell, const int* __restrict__ start, int* __restrict__ order) {
    const int c = (int)gid();
    if (c >= ncell) return;
    const int b = start[c], e = start[c + 1];
    for (int i = b + 1; i < e; ++i) {
        const int v = order[i];
        int j = i - 1;
        while (j >= b && order[j] > v) { order[j + 1] = order[j]; --j; }
        order[j + 1] = v;
    }
}

// visits every j != i closer than the radius, in cell-scan order
template <typename F>
__device__ __forceinline__ void for_neighbours(int i, const double2* __restrict__ x, const int* __restrict__ start,
                                               const int* __restrict__ order, double xmin, double ymin, double inv_r,
                                               double r2, int nx, int ny, F f) {
    const double2 p = x[i];
    int cx, cy;
    cell_of(p.x, p.y, xmin, ymin, inv_r, nx, ny, &cx, &cy);
    for (int yy = max(cy - 1, 0); yy <= min(cy + 1, ny - 1); ++yy) {
        const int row = yy * nx;
        const int b = start[row + max(cx - 1, 0)], e = start[row + min(cx + 1, nx - 1) + 1];
        for (int s = b; s < e; ++s) {
            const int j = order[s];
            if (j == i) continue;
            const double2 q = x[j];
            const double dx = p.x - q.x, dy = p.y - q.y;
            if (dx * dx + dy * dy < r2) f(j);
        }
    }
}

__global__ void k_graph_degree(const double2* __restrict__ x, int n, const int* __restrict__ start,
                               const int* __restrict__ order, double xmin, double ymin, double inv_r, double r2,
                               int nx, int ny, int* __restrict__ deg) {
    const int i = (int)gid();
    if (i > n) return;
    int c = 0;   // deg[n] = 0 closes the exclusive scan
    if (i < n) for_neighbours(i, x, start, order, xmin, ymin, inv_r, r2, nx, ny, [&](int) { ++c; });
    deg[i] = c;
}

__global__ void k_graph_fill(const double2* __restrict__ x, int n, const int* __restrict__ start,
                             const int* __restrict__ order, double xmin, double ymin, double inv_r, double r2, int nx,
                             int ny, const int64_t* __restrict__ off, int* __restrict__ src, int* __restrict__ dst) {
    const int i = (int)gid();
    if (i >= n) return;
    long long k = off[i];
    for_neighbours(i, x, start, order, xmin, ymin, inv_r, r2, nx, ny, [&](int j) {
        src[k] = j;
        dst[k] = i;
        ++k;
    });
}

// --------------------------------------------------------------- features
//
// Row kernels: a row of C values is handled by C/4 (fp32, float4) or C/8
// (bf16, 16-byte) adjacent threads, so every access is a full-width
// vector and no index needs a division by a run-time width.

constexpr int LW = 128;              // latent width the layer kernels are compiled for
constexpr int FW = SPHG_GNN_FEATURES;

template <int TPR>
__device__ __forceinline__ void row_lane(long long& r, int& lane) {
    r = (long long)blockIdx.x * (256 / TPR) + threadIdx.x / TPR;
    lane = threadIdx.x % TPR;
}

__device__ __forceinline__ uint4 pack8(const float* v) {
    uint4 u;
    __nv_bfloat162 t;
    t = __floats2bfloat162_rn(v[0], v[1]); u.x = *reinterpret_cast<uint32_t*>(&t);
    t = __floats2bfloat162_rn(v[2], v[3]); u.y = *reinterpret_cast<uint32_t*>(&t);
    t = __floats2bfloat162_rn(v[4], v[5]); u.z = *reinterpret_cast<uint32_t*>(&t);
    t = __floats2bfloat162_rn(v[6], v[7]); u.w = *reinterpret_cast<uint32_t*>(&t);
    return u;
}

__device__ __forceinline__ uint2 pack4(float4 v) {
    uint2 u;
    __nv_bfloat162 t;
    t = __floats2bfloat162_rn(v.x, v.y); u.x = *reinterpret_cast<uint32_t*>(&t);
    t = __floats2bfloat162_rn(v.z, v.w); u.y = *reinterpret_cast<uint32_t*>(&t);
    return u;
}

__device__ __forceinline__ float4 add4(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
__device__ __forceinline__ float4 relu4(float4 a) {
    return make_float4(fmaxf(a.x, 0.f), fmaxf(a.y, 0.f), fmaxf(a.z, 0.f), fmaxf(a.w, 0.f));
}

// node rows of 64 bf16, 8 threads per row, 8 features each
__global__ void k_node_features(const double2* __restrict__ x, const double2* __restrict__ x0,
                                const float2* __restrict__ vhist, int head, const sphg_gnn_node* __restrict__ st, int n,
                                int n_pad, float inv2h, float inv_vscale, bf16* __restrict__ out) {
    long long i;
    int lane;
    row_lane<FW / 8>(i, lane);
    if (i >= n_pad) return;
    float v[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (i < n && lane < 3) {
        const sphg_gnn_node s = st[i];
        for (int k = 0; k < 8; ++k) {
            const int f = lane * 8 + k;
            if (f < 2 * SPHG_GNN_HISTORY) {
                const int slot = (head + (f >> 1)) % SPHG_GNN_HISTORY;
                const float2 u = vhist[(size_t)slot * n + i];
                v[k] = ((f & 1) ? u.y : u.x) * inv_vscale;
            } else if (f < 13) {
                v[k] = (f - 10) == s.type ? 1.f : 0.f;
            } else if (f < 16) {
                const double2 p = x[i];
                const double d = f == 13 ? p.x - s.xl : (f == 14 ? s.xr - p.x : p.y - s.yf);
                v[k] = fminf(fmaxf((float)d * inv2h, 0.f), 1.f);
            } else if (f == 16) v[k] = s.porosity;
            else if (f == 17) v[k] = s.phi;
            else if (f == 18) v[k] = s.dts * 1.0e3f;
            else if (f < 21 && x0) {     // displacement since the reference state / 2h
                const double d = f == 19 ? x[i].x - x0[i].x : x[i].y - x0[i].y;
                v[k] = fminf(fmaxf((float)d * inv2h, -16.f), 16.f);
            }
        }
    }
    reinterpret_cast<uint4*>(out)[i * (FW / 8) + lane] = pack8(v);
}

// The first 8 of the 64 bf16 columns of edge a <- b (receiver a, sender b); the
// other 56 are zero:
//   0, 1  (x_a - x_b) / 2h
//   2     |x_a - x_b| / 2h
//   3     1 when a and b have the same type
//   4, 5  the change of (x_a - x_b) / 2h since the reference positions x0,
//         clipped to [-4, 4] (zero without x0): the local strain
// The products and sums are rounded one by one (no contraction).
__device__ __forceinline__ uint4 sphg_edge_feature_chunk(const double2* __restrict__ x, const double2* __restrict__ x0,
                                                         const sphg_gnn_node* __restrict__ st, int a, int b,
                                                         double inv2h) {
    float v[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    const double2 p = x[a], q = x[b];
    const double dx = __dmul_rn(__dsub_rn(p.x, q.x), inv2h), dy = __dmul_rn(__dsub_rn(p.y, q.y), inv2h);
    v[0] = (float)dx;
    v[1] = (float)dy;
    v[2] = (float)__dsqrt_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)));
    v[3] = st[a].type == st[b].type ? 1.f : 0.f;
    if (x0) {
        const double2 p0 = x0[a], q0 = x0[b];
        v[4] = fminf(fmaxf((float)__dsub_rn(dx, __dmul_rn(__dsub_rn(p0.x, q0.x), inv2h)), -4.f), 4.f);
        v[5] = fminf(fmaxf((float)__dsub_rn(dy, __dmul_rn(__dsub_rn(p0.y, q0.y), inv2h)), -4.f), 4.f);
    }
    uint4 u;
    __nv_bfloat162 t;
    t = __floats2bfloat162_rn(v[0], v[1]); u.x = *reinterpret_cast<uint32_t*>(&t);
    t = __floats2bfloat162_rn(v[2], v[3]); u.y = *reinterpret_cast<uint32_t*>(&t);
    t = __floats2bfloat162_rn(v[4], v[5]); u.z = *reinterpret_cast<uint32_t*>(&t);
    t = __floats2bfloat162_rn(v[6], v[7]); u.w = *reinterpret_cast<uint32_t*>(&t);
    return u;
}

// edge rows of 64 bf16 (sphg_edge_feature_chunk): one thread per edge row writes its
// 8 16-byte chunks, so 32 rows' gathers are in flight per warp.  Computing the rows
// inside the encoder kernel's loader instead measured slower (0.66 ms against
// 0.21 + 0.41 ms per 5.12M rows): its loader warps could not hide the gathers.
__global__ void k_edge_features(const double2* __restrict__ x, const double2* __restrict__ x0,
                                const sphg_gnn_node* __restrict__ st, const int* __restrict__ src,
                                const int* __restrict__ dst, long long nedge, long long nedge_pad, double inv2h,
                                bf16* __restrict__ out) {
    const long long k = gid();
    if (k >= nedge_pad) return;
    const uint4 z = make_uint4(0u, 0u, 0u, 0u);
    const uint4 c0 = k < nedge ? sphg_edge_feature_chunk(x, x0, st, dst[k], src[k], inv2h) : z;
    uint4* row = reinterpret_cast<uint4*>(out) + k * (FW / 8);
    row[0] = c0;
#pragma unroll
    for (int c = 1; c < FW / 8; ++c) row[c] = z;
}

// ----------------------------------------------------------------- layers

// n % 4 == 0
__global__ void k_f32_to_bf16(const float4* __restrict__ x, uint2* __restrict__ y, long long n4) {
    const long long i = gid();
    if (i < n4) y[i] = pack4(x[i]);
}

// dz = dh * (z > 0), fp32 and bf16; n % 4 == 0
__global__ void k_relu_bwd(const float4* __restrict__ dh, const float4* __restrict__ z, float4* __restrict__ dz,
                           uint2* __restrict__ dzb, long long n4) {
    const long long i = gid();
    if (i >= n4) return;
    const float4 g = dh[i], m = z[i];
    const float4 v = make_float4(m.x > 0.f ? g.x : 0.f, m.y > 0.f ? g.y : 0.f, m.z > 0.f ? g.z : 0.f,
                                 m.w > 0.f ? g.w : 0.f);
    dz[i] = v;
    dzb[i] = pack4(v);
}

// out[c] += sum over rows of x[r, c]; 512 rows per block
__global__ void k_colsum(const float* __restrict__ x, long long rows, int cols, float* __restrict__ out) {
    const int c = blockIdx.y * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    const long long r0 = (long long)blockIdx.x * 512;
    const long long r1 = r0 + 512 < rows ? r0 + 512 : rows;
    float s = 0.f;
    for (long long r = r0; r < r1; ++r) s += x[r * cols + c];
    atomicAdd(out + c, s);
}

// out[c, r] = in[r, c] in bf16 (32 x 32 tiles through shared memory)
template <typename S>
__global__ void k_transpose(const S* __restrict__ in, bf16* __restrict__ out, long long rows, int cols) {
    __shared__ float tile[32][33];
    const long long by = (long long)blockIdx.x * 32;
    const int bx = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += 8) {
        const long long r = by + j;
        const int c = bx + threadIdx.x;
        if (r < rows && c < cols) tile[j][threadIdx.x] = (float)in[r * cols + c];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += 8) {
        const int c = bx + j;
        const long long r = by + threadIdx.x;
        if (r < rows && c < cols) out[(long long)c * rows + r] = __float2bfloat16_rn(tile[threadIdx.x][j]);
    }
}

// agg[n] = scale * sum of e over the edges received by n
__global__ void k_segsum(const float* __restrict__ e, const int64_t* __restrict__ off, float* __restrict__ agg,
                         int nnode, float scale) {
    long long n;
    int lane;
    row_lane<LW / 4>(n, lane);
    if (n >= nnode) return;
    float4 s = make_float4(0.f, 0.f, 0.f, 0.f);
    for (long long k = off[n]; k < off[n + 1]; ++k) s = add4(s, reinterpret_cast<const float4*>(e + k * LW)[lane]);
    reinterpret_cast<float4*>(agg + n * LW)[lane] = make_float4(s.x * scale, s.y * scale, s.z * scale, s.w * scale);
}

// the same over bf16 edge rows: each lane sums 4 columns of every received row
__global__ void k_segsum_bf16(const __nv_bfloat16* __restrict__ e, const int64_t* __restrict__ off,
                              float* __restrict__ agg, int nnode, float scale) {
    long long n;
    int lane;
    row_lane<LW / 4>(n, lane);
    if (n >= nnode) return;
    float4 s = make_float4(0.f, 0.f, 0.f, 0.f);
    for (long long k = off[n]; k < off[n + 1]; ++k) {
        const uint2 u = reinterpret_cast<const uint2*>(e + k * LW)[lane];
        const float2 lo = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u.x));
        const float2 hi = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u.y));
        s = add4(s, make_float4(lo.x, lo.y, hi.x, hi.y));
    }
    reinterpret_cast<float4*>(agg + n * LW)[lane] = make_float4(s.x * scale, s.y * scale, s.z * scale, s.w * scale);
}

// The receiver sums written straight into the node MLP's input rows (inference):
// out[n] = [h[n] | bf16(scale * sum of e over the edges n receives)], the same bits
// as k_segsum_bf16 followed by k_node_concat, without the fp32 agg rows; rows from
// nnode to npad get zero sums.  One warp per node: lane l copies 8 bytes of h and
// sums columns 4l .. 4l + 3 in edge order.
__global__ void k_segsum_cat(const __nv_bfloat16* __restrict__ e, const int64_t* __restrict__ off,
                             const bf16* __restrict__ h, bf16* __restrict__ out, int nnode, long long npad,
                             float scale) {
    long long n;
    int lane;
    row_lane<LW / 4>(n, lane);
    if (n >= npad) return;
    float4 s = make_float4(0.f, 0.f, 0.f, 0.f);
    if (n < nnode) {
        for (long long k = off[n]; k < off[n + 1]; ++k) {
            const uint2 u = reinterpret_cast<const uint2*>(e + k * LW)[lane];
            const float2 lo = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u.x));
            const float2 hi = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u.y));
            s = add4(s, make_float4(lo.x, lo.y, hi.x, hi.y));
        }
    }
    uint2* row = reinterpret_cast<uint2*>(out + n * 2 * LW);
    row[lane] = reinterpret_cast<const uint2*>(h + n * LW)[lane];
    __nv_bfloat162 t0 = __floats2bfloat162_rn(s.x * scale, s.y * scale), t1 = __floats2bfloat162_rn(s.z * scale, s.w * scale);
    uint2 a;
    a.x = *reinterpret_cast<uint32_t*>(&t0);
    a.y = *reinterpret_cast<uint32_t*>(&t1);
    row[LW / 4 + lane] = a;
}

// de[k] += scale * dagg[receiver of k]
__global__ void k_segsum_bwd(const float* __restrict__ dagg, const int* __restrict__ dst, float* __restrict__ de,
                             long long nedge, float scale) {
    long long k;
    int lane;
    row_lane<LW / 4>(k, lane);
    if (k >= nedge) return;
    const float4 g = reinterpret_cast<const float4*>(dagg + (long long)dst[k] * LW)[lane];
    float4* d = reinterpret_cast<float4*>(de + k * LW) + lane;
    *d = add4(*d, make_float4(g.x * scale, g.y * scale, g.z * scale, g.w * scale));
}

// backward of the gathered projections: dP[n][L + f] = sum of dz over the
// edges n receives; dP[n][f] += dz over the edges n sends (atomic; dP[n][f]
// must be zero before)
__global__ void k_gather_bwd_dst(const float* __restrict__ dz, const int64_t* __restrict__ off,
                                 float* __restrict__ dP, int nnode) {
    long long n;
    int lane;
    row_lane<LW / 4>(n, lane);
    if (n >= nnode) return;
    float4 s = make_float4(0.f, 0.f, 0.f, 0.f);
    for (long long k = off[n]; k < off[n + 1]; ++k) s = add4(s, reinterpret_cast<const float4*>(dz + k * LW)[lane]);
    reinterpret_cast<float4*>(dP + n * 2 * LW + LW)[lane] = s;
}

__global__ void k_gather_bwd_src(const float* __restrict__ dz, const int* __restrict__ src, float* __restrict__ dP,
                                 long long nedge) {
    long long k;
    int lane;
    row_lane<LW / 4>(k, lane);
    if (k >= nedge) return;
    const float4 g = reinterpret_cast<const float4*>(dz + k * LW)[lane];
    float* d = dP + (long long)src[k] * 2 * LW + lane * 4;
    atomicAdd(d, g.x);
    atomicAdd(d + 1, g.y);
    atomicAdd(d + 2, g.z);
    atomicAdd(d + 3, g.w);
}

// [h | agg] as bf16 rows of 2L: 16 bytes (8 values) per thread
__global__ void k_node_concat(const bf16* __restrict__ h, const float* __restrict__ agg, bf16* __restrict__ out,
                              long long nnode) {
    long long n;
    int lane;
    row_lane<2 * LW / 8>(n, lane);
    if (n >= nnode) return;
    uint4 v;
    if (lane < LW / 8) {
        v = reinterpret_cast<const uint4*>(h + n * LW)[lane];
    } else {
        const float4* a = reinterpret_cast<const float4*>(agg + n * LW) + 2 * (lane - LW / 8);
        const float4 p = a[0], q = a[1];
        const float t[8] = {p.x, p.y, p.z, p.w, q.x, q.y, q.z, q.w};
        v = pack8(t);
    }
    reinterpret_cast<uint4*>(out + n * 2 * LW)[lane] = v;
}

__global__ void k_node_concat_bwd(const float* __restrict__ d, float* __restrict__ dh, float* __restrict__ dagg,
                                  long long nnode) {
    long long n;
    int lane;
    row_lane<2 * LW / 4>(n, lane);
    if (n >= nnode) return;
    const float4 g = reinterpret_cast<const float4*>(d + n * 2 * LW)[lane];
    if (lane < LW / 4) {
        float4* t = reinterpret_cast<float4*>(dh + n * LW) + lane;
        *t = add4(*t, g);
    } else {
        reinterpret_cast<float4*>(dagg + n * LW)[lane - LW / 4] = g;
    }
}

// Huber loss (squared error up to |d| = delta, linear beyond; plain squared
// error for delta <= 0) over the rows with mask != 0, first nout columns of
// pred (row stride ld), scaled by inv_count; dpred = d loss / d pred (zero
// elsewhere)
__global__ void k_mse(const float* __restrict__ pred, int ld, const float* __restrict__ target, int nout,
                      const float* __restrict__ mask, long long rows, float inv_count, float delta,
                      float* __restrict__ dpred, float* __restrict__ loss) {
    const long long i = gid();
    if (i >= rows * ld) return;
    const long long r = i / ld;
    const int c = (int)(i % ld);
    float g = 0.f;
    if (c < nout && mask[r] != 0.f) {
        const float d = pred[i] - target[r * nout + c];
        const float a = fabsf(d);
        if (delta <= 0.f || a <= delta) {
            g = 2.f * d * inv_count;
            atomicAdd(loss, d * d * inv_count);
        } else {
            g = copysignf(2.f * delta, d) * inv_count;
            atomicAdd(loss, delta * (2.f * a - delta) * inv_count);
        }
    }
    dpred[i] = g;
}

// Adam (Kingma & Ba 2015) on fp32 master weights [rows x cols]; rows at or
// beyond row_limit stay zero (padded outputs); refreshes the bf16 copy and
// its transpose [cols x rows] when given
__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, bf16* __restrict__ wb, bf16* __restrict__ wt, int rows, int cols,
                       float lr, float b1, float b2, float eps, float c1, float c2, int row_limit) {
    const long long i = gid();
    if (i >= (long long)rows * cols) return;
    const int r = (int)(i / cols), c = (int)(i % cols);
    float wi = 0.f;
    if (r < row_limit) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16_rn(wi);
    if (wt) wt[(long long)c * rows + r] = __float2bfloat16_rn(wi);
}

// ---------------------------------------------------------------- rollout

// one learned stride of length dts (per node): a = pred * std + mean,
// v' = v + a dts, x' = x + v' dts (semi-implicit Euler: with v the stride
// velocity (x - x_prev) / dts and a the stride acceleration, exactly the
// next position), clamped inside the walls; v' goes to history slot
// head_new; boundary nodes stay put
__global__ void k_stride_update(const float* __restrict__ pred, int ld, const float* __restrict__ norm,
                                const sphg_gnn_node* __restrict__ st, double2* __restrict__ x,
                                float2* __restrict__ vhist, int head_old, int head_new, int n, double margin) {
    const int i = (int)gid();
    if (i >= n) return;
    const sphg_gnn_node s = st[i];
    float2 vn = make_float2(0.f, 0.f);
    if (s.type != SPHG_GNN_BOUNDARY) {
        const float2 vo = vhist[(size_t)head_old * n + i];
        const float ax = pred[(long long)i * ld] * norm[2] + norm[0];
        const float ay = pred[(long long)i * ld + 1] * norm[3] + norm[1];
        vn = make_float2(vo.x + ax * s.dts, vo.y + ay * s.dts);
        double2 p = x[i];
        p.x += (double)s.dts * (double)vn.x;
        p.y += (double)s.dts * (double)vn.y;
        p.x = fmin(fmax(p.x, (double)s.xl + margin), (double)s.xr - margin);
        p.y = fmax(p.y, (double)s.yf + margin);
        x[i] = p;
    }
    vhist[(size_t)head_new * n + i] = vn;
}

// cubic-spline shape (Monaghan 1992), unnormalised, q = r / h
__device__ __forceinline__ double w_cubic(double q) {
    if (q < 1.0) return 1.0 - 1.5 * q * q + 0.75 * q * q * q;
    if (q < 2.0) { const double t = 2.0 - q; return 0.25 * t * t * t; }
    return 0.0;
}

// number density sigma_i = W(0) + sum over received edges of W(r / h)
__global__ void k_number_density(const double2* __restrict__ x, const int64_t* __restrict__ off,
                                 const int* __restrict__ src, int n, double inv_h, double* __restrict__ sigma) {
    const int i = (int)gid();
    if (i >= n) return;
    const double2 p = x[i];
    double s = 1.0;
    for (long long k = off[i]; k < off[i + 1]; ++k) {
        const double2 q = x[src[k]];
        const double dx = p.x - q.x, dy = p.y - q.y;
        s += w_cubic(sqrt(dx * dx + dy * dy) * inv_h);
    }
    sigma[i] = s;
}

// gate sums over real nodes: [0] sum (sigma_new / sigma_old - 1)^2,
// [1] count, [2] kinetic energy, [3] potential energy above the floor
__global__ void k_gate_sums(const double* __restrict__ sig_new, const double* __restrict__ sig_old,
                            const double2* __restrict__ x, const float2* __restrict__ vnew,
                            const sphg_gnn_node* __restrict__ st, int n, double g, double* __restrict__ out) {
    const int i = (int)gid();
    double a = 0.0, c = 0.0, ke = 0.0, pe = 0.0;
    if (i < n) {
        const sphg_gnn_node s = st[i];
        if (s.type != SPHG_GNN_BOUNDARY) {
            const double r = sig_new[i] / sig_old[i] - 1.0;
            a = r * r;
            c = 1.0;
            const float2 v = vnew[i];
            ke = 0.5 * (double)s.mass * ((double)v.x * v.x + (double)v.y * v.y);
            pe = (double)s.mass * g * (x[i].y - (double)s.yf);
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        c += __shfl_down_sync(0xffffffffu, c, o);
        ke += __shfl_down_sync(0xffffffffu, ke, o);
        pe += __shfl_down_sync(0xffffffffu, pe, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(out, a);
        atomicAdd(out + 1, c);
        atomicAdd(out + 2, ke);
        atomicAdd(out + 3, pe);
    }
}

}  // namespace

extern "C" {

#define LAUNCH1(kern, n, ...)                                                                \
    do {                                                                                     \
        if ((n) > 0) kern<<<nb((n), 256), 256, 0, (cudaStream_t)stream>>>(__VA_ARGS__);      \
        return ok_or_cuda();                                                                 \
    } while (0)

int sphg_gnn_scan_bytes(int n, size_t* bytes) {
    if (!bytes || n < 0) return SPHG_ERR_BAD_ARG;
    size_t b = 0, b2 = 0;
    if (cub::DeviceScan::ExclusiveSum(nullptr, b, (const int*)nullptr, (long long*)nullptr, n + 1) != cudaSuccess)
        return SPHG_ERR_CUDA;
    if (cub::DeviceScan::ExclusiveSum(nullptr, b2, (const int*)nullptr, (int*)nullptr, n + 1) != cudaSuccess)
        return SPHG_ERR_CUDA;
    *bytes = b > b2 ? b : b2;
    return SPHG_OK;
}

int sphg_gnn_graph_count(const sphg_gnn_grid* g, const double* x, int n, int* order, int* cell_count,
                         int* cell_start, int* deg, int64_t* off, void* tmp, size_t tmp_bytes, void* stream) {
    if (!g || !x || n <= 0 || !order || !cell_count || !cell_start || !deg || !off || !tmp) return SPHG_ERR_BAD_ARG;
    if (g->nx <= 0 || g->ny <= 0 || !(g->radius > 0.0)) return SPHG_ERR_BAD_ARG;
    const long long ncell = (long long)g->nx * g->ny;
    if (ncell >= (1LL << 31) - 1) return SPHG_ERR_BAD_ARG;
    size_t need = 0;
    if (sphg_gnn_scan_bytes((int)(ncell > n ? ncell : n), &need) != SPHG_OK || need > tmp_bytes)
        return SPHG_ERR_BAD_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const double inv_r = 1.0 / g->radius, r2 = g->radius * g->radius;
    const double2* X = (const double2*)x;
    if (cudaMemsetAsync(cell_count, 0, (ncell + 1) * sizeof(int), s) != cudaSuccess) return SPHG_ERR_CUDA;
    // deg holds each node's cell until the degree pass
    k_graph_count<<<nb(n, 256), 256, 0, s>>>(X, n, g->xmin, g->ymin, inv_r, g->nx, g->ny, deg, cell_count);
    if (cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, cell_count, cell_start, (int)ncell + 1, s) != cudaSuccess)
        return SPHG_ERR_CUDA;
    // the scatter cursor reuses cell_count
    if (cudaMemcpyAsync(cell_count, cell_start, (ncell + 1) * sizeof(int), cudaMemcpyDeviceToDevice, s) != cudaSuccess)
        return SPHG_ERR_CUDA;
    k_graph_scatter<<<nb(n, 256), 256, 0, s>>>(n, deg, cell_count, order);
    k_graph_cell_sort<<<nb(ncell, 256), 256, 0, s>>>((int)ncell, cell_start, order);
    k_graph_degree<<<nb(n + 1, 128), 128, 0, s>>>(X, n, cell_start, order, g->xmin, g->ymin, inv_r, r2, g->nx,
                                                   g->ny, deg);
    if (cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, deg, off, n + 1, s) != cudaSuccess) return SPHG_ERR_CUDA;
    return ok_or_cuda();
}

int sphg_gnn_graph_fill(const sphg_gnn_grid* g, const double* x, int n, const int* order, const int* cell_start,
                        const int64_t* off, int* src, int* dst, void* stream) {
    if (!g || !x || n <= 0 || !order || !cell_start || !off || !src || !dst) return SPHG_ERR_BAD_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    k_graph_fill<<<nb(n, 128), 128, 0, s>>>((const double2*)x, n, cell_start, order, g->xmin, g->ymin,
                                             1.0 / g->radius, g->radius * g->radius, g->nx, g->ny, off, src, dst);
    return ok_or_cuda();
}

// blocks of 256 threads for `rows` rows of TPR threads each
inline unsigned row_blocks(long long rows, int tpr) { return nb(rows, 256 / tpr); }
#define ROWS(kern, rows, tpr, ...)                                                            \
    do {                                                                                      \
        if ((rows) > 0) kern<<<row_blocks((rows), (tpr)), 256, 0, (cudaStream_t)stream>>>(__VA_ARGS__); \
        return ok_or_cuda();                                                                  \
    } while (0)

int sphg_gnn_node_features(const double* x, const double* x0, const float* vhist, int head, const sphg_gnn_node* st,
                           int n, int n_pad, float inv2h, float inv_vscale, void* out, void* stream) {
    if (head < 0 || head >= SPHG_GNN_HISTORY || n_pad < n) return SPHG_ERR_BAD_ARG;
    ROWS(k_node_features, n_pad, FW / 8, (const double2*)x, (const double2*)x0, (const float2*)vhist, head, st, n,
         n_pad, inv2h, inv_vscale, (bf16*)out);
}

int sphg_gnn_edge_features(const double* x, const double* x0, const sphg_gnn_node* st, const int* src, const int* dst,
                           long long nedge, long long nedge_pad, double inv2h, void* out, void* stream) {
    if (nedge_pad < nedge) return SPHG_ERR_BAD_ARG;
    LAUNCH1(k_edge_features, nedge_pad, (const double2*)x, (const double2*)x0, st, src, dst, nedge, nedge_pad, inv2h,
            (bf16*)out);
}

int sphg_gnn_f32_to_bf16(const float* x, void* y, long long n, void* stream) {
    if (n % 4) return SPHG_ERR_BAD_ARG;
    LAUNCH1(k_f32_to_bf16, n / 4, (const float4*)x, (uint2*)y, n / 4);
}

int sphg_gnn_relu_bwd(const float* dh, const float* z, float* dz, void* dzb, long long n, void* stream) {
    if (n % 4) return SPHG_ERR_BAD_ARG;
    LAUNCH1(k_relu_bwd, n / 4, (const float4*)dh, (const float4*)z, (float4*)dz, (uint2*)dzb, n / 4);
}

int sphg_gnn_colsum(const float* x, long long rows, int cols, float* out, void* stream) {
    if (rows <= 0 || cols <= 0) return SPHG_OK;
    dim3 grid(nb(rows, 512), nb(cols, 128));
    k_colsum<<<grid, 128, 0, (cudaStream_t)stream>>>(x, rows, cols, out);
    return ok_or_cuda();
}

int sphg_gnn_transpose(const void* in, int in_is_f32, void* out, long long rows, int cols, void* stream) {
    if (rows <= 0 || cols <= 0) return SPHG_OK;
    dim3 grid(nb(rows, 32), nb(cols, 32)), block(32, 8);
    if (in_is_f32)
        k_transpose<float><<<grid, block, 0, (cudaStream_t)stream>>>((const float*)in, (bf16*)out, rows, cols);
    else
        k_transpose<bf16><<<grid, block, 0, (cudaStream_t)stream>>>((const bf16*)in, (bf16*)out, rows, cols);
    return ok_or_cuda();
}

int sphg_gnn_segsum(const float* e, const int64_t* off, float* agg, int nnode, int L, float scale, void* stream) {
    if (L != LW) return SPHG_ERR_BAD_ARG;
    ROWS(k_segsum, (long long)nnode, LW / 4, e, off, agg, nnode, scale);
}

int sphg_gnn_segsum_bf16(const void* e, const int64_t* off, float* agg, int nnode, int L, float scale, void* stream) {
    if (L != LW) return SPHG_ERR_BAD_ARG;
    ROWS(k_segsum_bf16, (long long)nnode, LW / 4, (const __nv_bfloat16*)e, off, agg, nnode, scale);
}

int sphg_gnn_segsum_cat(const void* e, const int64_t* off, const void* h, void* out, int nnode, long long npad, int L,
                        float scale, void* stream) {
    if (L != LW || npad < nnode) return SPHG_ERR_BAD_ARG;
    ROWS(k_segsum_cat, npad, LW / 4, (const __nv_bfloat16*)e, off, (const bf16*)h, (bf16*)out, nnode, npad, scale);
}

int sphg_gnn_segsum_bwd(const float* dagg, const int* dst, float* de, long long nedge, int L, float scale,
                        void* stream) {
    if (L != LW) return SPHG_ERR_BAD_ARG;
    ROWS(k_segsum_bwd, nedge, LW / 4, dagg, dst, de, nedge, scale);
}

int sphg_gnn_gather_bwd(const float* dz, const int* src, const int64_t* off, float* dP, int nnode,
                        long long nedge, int L, void* stream) {
    if (L != LW) return SPHG_ERR_BAD_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    if (nnode > 0) k_gather_bwd_dst<<<row_blocks(nnode, LW / 4), 256, 0, s>>>(dz, off, dP, nnode);
    if (nedge > 0) k_gather_bwd_src<<<row_blocks(nedge, LW / 4), 256, 0, s>>>(dz, src, dP, nedge);
    return ok_or_cuda();
}

int sphg_gnn_node_concat(const void* h, const float* agg, void* out, long long nnode, int L, void* stream) {
    if (L != LW) return SPHG_ERR_BAD_ARG;
    ROWS(k_node_concat, nnode, 2 * LW / 8, (const bf16*)h, agg, (bf16*)out, nnode);
}

int sphg_gnn_node_concat_bwd(const float* d, float* dh, float* dagg, long long nnode, int L, void* stream) {
    if (L != LW) return SPHG_ERR_BAD_ARG;
    ROWS(k_node_concat_bwd, nnode, 2 * LW / 4, d, dh, dagg, nnode);
}

int sphg_gnn_mse(const float* pred, int ld, const float* target, int nout, const float* mask, long long rows,
                 float inv_count, float delta, float* dpred, float* loss, void* stream) {
    LAUNCH1(k_mse, rows * ld, pred, ld, target, nout, mask, rows, inv_count, delta, dpred, loss);
}

int sphg_gnn_adam(float* w, const float* g, float* m, float* v, void* wb, void* wt, int rows, int cols, float lr,
                  float b1, float b2, float eps, int step, int row_limit, void* stream) {
    if (step < 1) return SPHG_ERR_BAD_ARG;
    const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
    LAUNCH1(k_adam, (long long)rows * cols, w, g, m, v, (bf16*)wb, (bf16*)wt, rows, cols, lr, b1, b2, eps, c1, c2,
            row_limit);
}

int sphg_gnn_stride_update(const float* pred, int ld, const float* norm, const sphg_gnn_node* st, double* x,
                           float* vhist, int head_old, int head_new, int n, double margin, void* stream) {
    if (head_old < 0 || head_old >= SPHG_GNN_HISTORY || head_new < 0 || head_new >= SPHG_GNN_HISTORY)
        return SPHG_ERR_BAD_ARG;
    LAUNCH1(k_stride_update, n, pred, ld, norm, st, (double2*)x, (float2*)vhist, head_old, head_new, n, margin);
}

int sphg_gnn_number_density(const double* x, const int64_t* off, const int* src, int n, double h, double* sigma,
                            void* stream) {
    if (!(h > 0.0)) return SPHG_ERR_BAD_ARG;
    LAUNCH1(k_number_density, n, (const double2*)x, off, src, n, 1.0 / h, sigma);
}

int sphg_gnn_gate_sums(const double* sig_new, const double* sig_old, const double* x, const float* vnew,
                       const sphg_gnn_node* st, int n, double g, double* out, void* stream) {
    if (cudaMemsetAsync(out, 0, 4 * sizeof(double), (cudaStream_t)stream) != cudaSuccess) return SPHG_ERR_CUDA;
    LAUNCH1(k_gate_sums, n, sig_new, sig_old, (const double2*)x, (const float2*)vnew, st, n, g, out);
}

}  // extern "C"
