// sphg_umma.cu — BF16 GEMM on the 5th-generation tensor cores (tcgen05) for
// the learned particle stepper: C[M x N] (+)= A[M x K] * B[N x K]^T, A and B
// row-major bf16 (K contiguous), C row-major fp32.
//
// One CTA of 128 threads computes a 128 x BN tile with UMMA M = 128:
//   * warp 0 allocates BN (>= 32) TMEM columns for the fp32 accumulator;
//   * every K block of 64 the CTA stages A (128 x 64) and B (BN x 64) in
//     shared memory in the canonical no-swizzle K-major layout (8-row x
//     16-byte core matrices; K halves LBO apart, 8-row groups SBO = 128 B
//     apart), fences the generic->async proxy, and one thread issues four
//     K = 16 tcgen05.mma instructions followed by tcgen05.commit to an
//     mbarrier;
//   * every wait on that mbarrier is bounded: on timeout the kernel sets
//     *err, waits (bounded again) for its MMAs, frees TMEM and returns;
//   * the epilogue reads the accumulator with tcgen05.ld (warp w owns TMEM
//     lanes 32w..32w+31 = tile rows) and stores, adds to, or atomically adds
//     into C (split-K over gridDim.z).
// Shapes: M % 128 == 0, N % BN == 0 with BN in {16, 32, 64, 128, 256},
// K % 64 == 0, 16-byte aligned rows.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/sphg.h"
#include "../../include/sphg_learn.h"

namespace {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor, no swizzle, K-major (version 1 = sm_100)
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;          // version
    // base offset 0, lbo mode 0, layout type 0 (SWIZZLE_NONE)
    return d;
}

// instruction descriptor: D fp32, A and B bf16, both K-major, M = 128, N = BN
__host__ __device__ constexpr uint32_t make_idesc(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t parity, long long limit) {
    for (long long i = 0; i < limit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

constexpr long long kWaitLimit = 1LL << 22;

template <int BN>
__global__ void __launch_bounds__(128, 1) k_gemm_bf16_tn(const __nv_bfloat16* __restrict__ A,
                                                         const __nv_bfloat16* __restrict__ B, float* __restrict__ C,
                                                         int M, int N, int K, int k_per_split, int accumulate,
                                                         int atomic_out, int* __restrict__ err,
                                                         long long probe_spins) {
    constexpr int TCOLS = BN < 32 ? 32 : BN;
    constexpr uint32_t A_KC = 128 * 16;     // bytes between K chunks of the A stage
    constexpr uint32_t B_KC = BN * 16;      // bytes between K chunks of the B stage
    extern __shared__ __align__(128) uint8_t smem[];
    uint8_t* sA = smem;
    uint8_t* sB = smem + 8 * A_KC;
    uint64_t* mbar = (uint64_t*)(sB + 8 * B_KC);
    uint32_t* tslot = (uint32_t*)(mbar + 1);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * 128, n0 = blockIdx.y * BN;
    const int kbeg = blockIdx.z * k_per_split;
    const int kend = min(K, kbeg + k_per_split);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(TCOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::);
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::);
    const uint32_t tmem = *tslot;
    const uint32_t mbar_a = smem_u32(mbar);
    const uint32_t idesc = make_idesc(BN);

    bool ok = true;
    uint32_t parity = 0;
    int issued = 0;
    // probe_spins > 0 (sphg_gemm_wait_probe): the first K block issues no MMA
    // and waits for it with that many polls, so the bounded wait runs out
    // while nothing is in flight and the kernel takes its error exit
    const bool probe = probe_spins > 0;
    for (int k0 = kbeg; k0 < kend && ok; k0 += 64) {
        // stage A and B in the canonical K-major layout
        for (int c = tid; c < 128 * 8; c += 128) {
            const int r = c >> 3, kc = c & 7;
            const uint4 v = *reinterpret_cast<const uint4*>(A + (size_t)(m0 + r) * K + k0 + kc * 8);
            *reinterpret_cast<uint4*>(sA + kc * A_KC + (r >> 3) * 128 + (r & 7) * 16) = v;
        }
        for (int c = tid; c < BN * 8; c += 128) {
            const int r = c >> 3, kc = c & 7;
            const uint4 v = *reinterpret_cast<const uint4*>(B + (size_t)(n0 + r) * K + k0 + kc * 8);
            *reinterpret_cast<uint4*>(sB + kc * B_KC + (r >> 3) * 128 + (r & 7) * 16) = v;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0 && !probe) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::);
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
                const uint64_t da = make_desc(smem_u32(sA + kk * 2 * A_KC), A_KC, 128);
                const uint64_t db = make_desc(smem_u32(sB + kk * 2 * B_KC), B_KC, 128);
                const uint32_t en = (k0 > kbeg || kk > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
                    ::"r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(en), "r"(0), "r"(0), "r"(0), "r"(0));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         ::"r"(mbar_a) : "memory");
        }
        if (!probe) ++issued;
        const bool done = mbar_wait(mbar_a, parity, probe ? probe_spins : kWaitLimit);
        parity ^= 1u;
        ok = __syncthreads_and(done ? 1 : 0) != 0;   // block-uniform: every thread leaves the loop together
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::);

    if (ok && issued > 0) {
        const int row = m0 + warp * 32 + lane;
        const uint32_t tbase = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
        for (int c = 0; c < BN; c += 8) {
            uint32_t r[8];
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                         : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                           "=r"(r[7])
                         : "r"(tbase + (uint32_t)c));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            float* out = C + (size_t)row * N + n0 + c;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const float v = __uint_as_float(r[j]);
                if (atomic_out) atomicAdd(out + j, v);
                else if (accumulate) out[j] += v;
                else out[j] = v;
            }
        }
    } else if (!ok) {
        if (tid == 0) atomicExch(err, 1);
        // a bounded second wait for MMAs that may still be in flight
        if (issued > 0) mbar_wait(mbar_a, parity ^ 1u, kWaitLimit);
    } else if (!accumulate && !atomic_out && !probe) {
        // empty K range: C = 0
        const int row = m0 + warp * 32 + lane;
        for (int c = 0; c < BN; ++c) C[(size_t)row * N + n0 + c] = 0.f;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::);
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TCOLS));
}

template <int BN>
int launch_gemm(const __nv_bfloat16* A, const __nv_bfloat16* B, float* C, int M, int N, int K, int accumulate,
                int split, int* err, cudaStream_t s, long long probe_spins = 0) {
    const size_t smem = 8 * (128 * 16) + 8 * (BN * 16) + 16 + 16;
    static bool configured = false;
    if (!configured) {
        if (cudaFuncSetAttribute(k_gemm_bf16_tn<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess)
            return SPHG_ERR_CUDA;
        configured = true;
    }
    const int kblocks = K / 64;
    const int per = (kblocks + split - 1) / split;
    dim3 grid(M / 128, N / BN, split);
    k_gemm_bf16_tn<BN><<<grid, 128, smem, s>>>(A, B, C, M, N, K, per * 64, accumulate, split > 1 ? 1 : 0, err,
                                               probe_spins);
    return cudaGetLastError() == cudaSuccess ? SPHG_OK : SPHG_ERR_CUDA;
}

// ------------------------------------------------------------------------
// Weight-stationary persistent GEMM for tall-skinny products: C[M x N] =
// A[M x K] * B[N x K]^T with B (the weights, N * K <= 32k elements) resident
// in shared memory for the whole launch.  Each CTA loops over 128-row tiles
// of A (tile = blockIdx.x + i * gridDim.x): the A tile of step i + 1 is
// copied (cp.async, 16 bytes per request, into the canonical no-swizzle
// K-major layout) while the MMAs of step i run on the tensor cores and the
// epilogue of step i - 1 drains the other TMEM accumulator, so load, MMA
// and epilogue overlap.  Every wait on an MMA is bounded; on timeout the
// kernel sets *err, waits (bounded) for its MMAs and copies, frees TMEM and
// returns.  Epilogues fuse what follows the product in the network:
//   STORE     z = acc
//   ACC       z += acc
//   BIAS_ACT  z = acc + bias (kept when z != null), h = bf16(act(z))
//   EDGE      z = acc + bias + P[src[row], :N] + P[dst[row], N:] (rows < nedge),
//             h = bf16(relu(z))
//   RESID     z = z + acc + bias, h = bf16(z) when h != null

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }


template <int N, int K>
struct WsShape {
    static constexpr uint32_t A_KC = 128 * 16;          // bytes between K chunks of an A tile
    static constexpr uint32_t B_KC = N * 16;            // ... of the resident B
    static constexpr uint32_t A_BYTES = (K / 8) * A_KC;
    static constexpr uint32_t B_BYTES = (K / 8) * B_KC;
    static constexpr uint32_t STAGE_OFF = B_BYTES + 2 * A_BYTES + 32;   // epilogue staging, 16-byte aligned
    static constexpr uint32_t STAGE_BYTES = 8 * 32 * 64;                  // 8 warps x 32 rows x 16 fp32
    static constexpr uint32_t SMEM = STAGE_OFF + STAGE_BYTES;
    static constexpr int TCOLS = 2 * N;                 // two accumulators
    // at most 2 CTAs per SM (TMEM: 2 x 256 columns), 1 when N = 256; the SM
    // holds 228 KB of shared memory, 1 KB of it reserved per CTA
    static constexpr uint32_t SMEM_REQ = N == 256 ? (SMEM > 120 * 1024 ? SMEM : 120 * 1024)
                                                  : (SMEM > 100 * 1024 ? SMEM : 100 * 1024);
    static constexpr int PER_SM = N == 256 || 2 * (SMEM_REQ + 1024) > 228 * 1024 ? 1 : 2;
};

constexpr int WS_THREADS = 256;   // 8 warps: warps w and w + 4 share TMEM lanes 32 (w % 4) ..

template <int N, int K, int NT = WS_THREADS>
__device__ __forceinline__ void ws_load_a(uint8_t* sA, const __nv_bfloat16* __restrict__ A, int m0, int tid) {
    constexpr int KC = K / 8;
#pragma unroll 4
    for (int c = tid; c < 128 * KC; c += NT) {
        const int r = c / KC, kc = c % KC;
        cp_async16(smem_u32(sA + kc * WsShape<N, K>::A_KC + (r >> 3) * 128 + (r & 7) * 16),
                   A + (size_t)(m0 + r) * K + kc * 8);
    }
}

__device__ __forceinline__ float4 add4f(float4 a, float4 b) {
    return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
}

// 16 accumulator columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

// The epilogue of a warp's 32 accumulator rows (one per lane, as TMEM
// delivers them) over its columns, through a per-warp staging tile in shared
// memory.  The warp's 32 accumulator rows (one per lane, as TMEM delivers them) are
// written to shared memory and read back so that 4 lanes cover the 64
// contiguous bytes of one row's 16-column chunk: every global load and store
// of the epilogue then touches 8 rows per instruction instead of 32.  In the
// staging tile row r holds 4 16-byte units, unit u at slot u ^ ((r >> 1) & 3),
// so that both the row-per-lane writes and the 4-lanes-per-row reads are free
// of bank conflicts.  Each chunk of 16 columns forms z = acc + (((residual) +
// (P[src] + P[dst])) + bias), the parts that apply to the mode, in that order.
template <int N, int K, int MODE = -1>   // MODE >= 0: the epilogue mode known at compile time
__device__ __forceinline__ void ws_epilogue_staged(const SphgGemmEpi& ep, uint32_t tacc, long long row0, int c0,
                                                   float4* __restrict__ stage, int lane, uint8_t* hs = nullptr,
                                                   int r0s = 0, int ncols = N / 2,
                                                   const __nv_bfloat16* zb = nullptr) {
    constexpr int CW = 16;
    const int q = lane & 3, rs = lane >> 2;   // this lane's 16-byte unit, and its row within each group of 8
    const int mode = MODE >= 0 ? MODE : ep.mode;
    const bool readz = mode == SPHG_EPI_ACC || mode == SPHG_EPI_RESID;
    const bool bias = mode != SPHG_EPI_STORE && mode != SPHG_EPI_ACC;
    const bool hout = mode != SPHG_EPI_STORE && mode != SPHG_EPI_ACC && (ep.h || hs);
    const bool act = mode == SPHG_EPI_EDGE || (mode == SPHG_EPI_BIAS_ACT && ep.relu);
    bool edge[4];
    const float4* ps[4];
    const float4* pd[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const long long r = row0 + 8 * i + rs;
        edge[i] = mode == SPHG_EPI_EDGE && r < ep.nedge;
        ps[i] = pd[i] = nullptr;
        if (edge[i]) {
            ps[i] = reinterpret_cast<const float4*>(ep.P + (long long)ep.src[r] * 2 * N);
            pd[i] = reinterpret_cast<const float4*>(ep.P + (long long)ep.dst[r] * 2 * N + N);
        }
    }
    const int wsw = (lane >> 1) & 3;   // swizzle of this lane's own staging row
    // A chunk's global inputs are loaded one chunk ahead: the loads of chunk
    // c + CW are in flight while chunk c is read from TMEM, staged and stored.
    float4 zf[4], pa[4], pb[4], bb = make_float4(0.f, 0.f, 0.f, 0.f);
    uint2 zh[4];
    auto load_chunk = [&](int cc) {
        const int col = cc + 4 * q;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            if (readz) {
                if (ep.z) zf[i] = reinterpret_cast<const float4*>(ep.z + (row0 + 8 * i + rs) * N)[col / 4];
                else zh[i] = reinterpret_cast<const uint2*>(zb + (row0 + 8 * i + rs) * N)[col / 4];
            }
            if (edge[i]) { pa[i] = ps[i][col / 4]; pb[i] = pd[i][col / 4]; }
        }
        if (bias) bb = reinterpret_cast<const float4*>(ep.bias)[col / 4];
    };
    load_chunk(c0);
#pragma unroll 1
    for (int c = c0; c < c0 + ncols; c += CW) {
        const int col = c + 4 * q;
        float4 add[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            add[i] = make_float4(0.f, 0.f, 0.f, 0.f);
            if (readz) {
                if (ep.z) {
                    add[i] = zf[i];
                } else {   // the residual as bf16 rows (zb); may be the rows this epilogue writes to h
                    const float2 lo = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&zh[i].x));
                    const float2 hi = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&zh[i].y));
                    add[i] = make_float4(lo.x, lo.y, hi.x, hi.y);
                }
            }
            if (edge[i]) add[i] = add4f(add[i], add4f(pa[i], pb[i]));
        }
        if (bias) {
#pragma unroll
            for (int i = 0; i < 4; ++i) add[i] = add4f(add[i], bb);
        }
        if (c + CW < c0 + ncols) load_chunk(c + CW);
        float v[CW];
        tmem_ld16(tacc + (uint32_t)c, v);
#pragma unroll
        for (int u = 0; u < 4; ++u)
            stage[lane * 4 + (u ^ wsw)] = make_float4(v[4 * u], v[4 * u + 1], v[4 * u + 2], v[4 * u + 3]);
        __syncwarp();
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int r = 8 * i + rs;
            const float4 a = stage[r * 4 + (q ^ ((r >> 1) & 3))];
            float o[4] = {a.x + add[i].x, a.y + add[i].y, a.z + add[i].z, a.w + add[i].w};
            const long long grow = row0 + r;
            if (ep.z) reinterpret_cast<float4*>(ep.z + grow * N)[col / 4] = make_float4(o[0], o[1], o[2], o[3]);
            if (hout) {
                if (act) {
#pragma unroll
                    for (int j = 0; j < 4; ++j) o[j] = fmaxf(o[j], 0.f);
                }
                __nv_bfloat162 t0 = __floats2bfloat162_rn(o[0], o[1]), t1 = __floats2bfloat162_rn(o[2], o[3]);
                uint2 hv;
                hv.x = *reinterpret_cast<uint32_t*>(&t0);
                hv.y = *reinterpret_cast<uint32_t*>(&t1);
                if (hs) {   // into shared memory as the A operand of a following MMA (tile row r0s + r)
                    const int tr = r0s + r;
                    *reinterpret_cast<uint2*>(hs + (col >> 3) * (128 * 16) + (tr >> 3) * 128 + (tr & 7) * 16 +
                                              (col & 7) * 2) = hv;
                } else {
                    reinterpret_cast<uint2*>(static_cast<__nv_bfloat16*>(ep.h) + grow * N)[col / 4] = hv;
                }
            }
        }
        __syncwarp();
    }
}

template <int N, int K, int MODE>
__global__ void __launch_bounds__(WS_THREADS, 2) k_gemm_ws(const __nv_bfloat16* __restrict__ A,
                                                    const __nv_bfloat16* __restrict__ B, int M, SphgGemmEpi ep,
                                                    int* __restrict__ err) {
    typedef WsShape<N, K> S;
    extern __shared__ __align__(128) uint8_t smem[];
    uint8_t* sB = smem;
    uint8_t* sA0 = smem + S::B_BYTES;    // A buffer s at sA0 + s * A_BYTES
    uint64_t* mbar = (uint64_t*)(smem + S::B_BYTES + 2 * S::A_BYTES);
    uint32_t* tslot = (uint32_t*)(mbar + 2);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    float4* stage = reinterpret_cast<float4*>(smem + S::STAGE_OFF) + warp * 128;
    const int ntiles = M / 128;
    const int my = blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    auto tile_m0 = [&](int i) { return ((int)blockIdx.x + i * (int)gridDim.x) * 128; };

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(S::TCOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(1));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar + 1)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::);
    }
    // resident B in the canonical K-major layout
    constexpr int KC = K / 8;
    for (int c = tid; c < N * KC; c += WS_THREADS) {
        const int r = c / KC, kc = c % KC;
        *reinterpret_cast<uint4*>(sB + kc * S::B_KC + (r >> 3) * 128 + (r & 7) * 16) =
            *reinterpret_cast<const uint4*>(B + (size_t)r * K + kc * 8);
    }
    if (my > 0) ws_load_a<N, K>(sA0, A, tile_m0(0), tid);
    cp_async_commit();
    cp_async_wait_all();
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::);
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::);
    const uint32_t tmem = *tslot;
    const uint32_t idesc = make_idesc(N);
    const uint32_t lane_off = (uint32_t)((warp & 3) * 32) << 16;
    const int col0 = (warp >> 2) * (N / 2);    // the column half of this warp
    uint32_t ph = 0u;    // bit s: parity of the next completion of mbar[s]
    bool ok = true;
    int issued = 0, waited = 0;   // MMA steps issued, and seen complete

    for (int i = 0; i < my && ok; ++i) {
        const int s = i & 1;
        if (i > 0) {
            cp_async_wait_all();
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
        }
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::);
#pragma unroll
            for (int kk = 0; kk < K / 16; ++kk) {
                const uint64_t da = make_desc(smem_u32(sA0 + s * S::A_BYTES + kk * 2 * S::A_KC), S::A_KC, 128);
                const uint64_t db = make_desc(smem_u32(sB + kk * 2 * S::B_KC), S::B_KC, 128);
                const uint32_t en = kk > 0 ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
                    ::"r"(tmem + (uint32_t)(s * N)), "l"(da), "l"(db), "r"(idesc), "r"(en), "r"(0), "r"(0), "r"(0),
                      "r"(0));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         ::"r"(smem_u32(mbar + s)) : "memory");
        }
        ++issued;
        if (i == 0) {
            if (my > 1) ws_load_a<N, K>(sA0 + S::A_BYTES, A, tile_m0(1), tid);
            cp_async_commit();
            continue;
        }
        // MMA(i - 1) done: its A buffer is free and its accumulator is ready
        const int p = s ^ 1;
        const bool done = mbar_wait(smem_u32(mbar + p), (ph >> p) & 1u, kWaitLimit);
        ok = __syncthreads_and(done ? 1 : 0) != 0;
        if (!ok) break;
        ph ^= 1u << p;
        ++waited;
        asm volatile("tcgen05.fence::after_thread_sync;" ::);
        if (i + 1 < my) ws_load_a<N, K>(sA0 + p * S::A_BYTES, A, tile_m0(i + 1), tid);
        cp_async_commit();
        ws_epilogue_staged<N, K, MODE>(ep, tmem + lane_off + (uint32_t)(p * N),
                                       (long long)tile_m0(i - 1) + (warp & 3) * 32, col0, stage, lane);
        asm volatile("tcgen05.fence::before_thread_sync;" ::);
        __syncthreads();
    }
    if (ok && my > 0) {
        const int s = (my - 1) & 1;
        const bool done = mbar_wait(smem_u32(mbar + s), (ph >> s) & 1u, kWaitLimit);
        ok = __syncthreads_and(done ? 1 : 0) != 0;
        if (ok) {
            ph ^= 1u << s;
            ++waited;
            asm volatile("tcgen05.fence::after_thread_sync;" ::);
            ws_epilogue_staged<N, K, MODE>(ep, tmem + lane_off + (uint32_t)(s * N),
                                           (long long)tile_m0(my - 1) + (warp & 3) * 32, col0, stage, lane);
        }
    }
    if (!ok) {
        if (tid == 0) atomicExch(err, 1);
        // bounded waits for the MMAs issued but not yet seen complete
        for (int j = waited; j < issued; ++j) {
            const int s = j & 1;
            mbar_wait(smem_u32(mbar + s), (ph >> s) & 1u, kWaitLimit);
            ph ^= 1u << s;
        }
    }
    cp_async_wait_all();
    asm volatile("tcgen05.fence::before_thread_sync;" ::);
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(S::TCOLS));
}

template <int N, int K, int MODE>
int launch_ws_mode(const __nv_bfloat16* A, const __nv_bfloat16* B, int M, const SphgGemmEpi& ep, int* err,
                   cudaStream_t s) {
    typedef WsShape<N, K> S;
    static bool configured = false;
    if (!configured) {
        if (cudaFuncSetAttribute(k_gemm_ws<N, K, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)S::SMEM_REQ) != cudaSuccess)
            return SPHG_ERR_CUDA;
        configured = true;
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int ntiles = M / 128;
    const int grid = ntiles < sms * S::PER_SM ? ntiles : sms * S::PER_SM;
    k_gemm_ws<N, K, MODE><<<grid, WS_THREADS, S::SMEM_REQ, s>>>(A, B, M, ep, err);
    return cudaGetLastError() == cudaSuccess ? SPHG_OK : SPHG_ERR_CUDA;
}

// one kernel per epilogue mode, so that each carries only its mode's registers
template <int N, int K>
int launch_ws(const __nv_bfloat16* A, const __nv_bfloat16* B, int M, const SphgGemmEpi& ep, int* err,
              cudaStream_t s) {
    switch (ep.mode) {
        case SPHG_EPI_STORE: return launch_ws_mode<N, K, SPHG_EPI_STORE>(A, B, M, ep, err, s);
        case SPHG_EPI_ACC: return launch_ws_mode<N, K, SPHG_EPI_ACC>(A, B, M, ep, err, s);
        case SPHG_EPI_BIAS_ACT: return launch_ws_mode<N, K, SPHG_EPI_BIAS_ACT>(A, B, M, ep, err, s);
        case SPHG_EPI_EDGE: return launch_ws_mode<N, K, SPHG_EPI_EDGE>(A, B, M, ep, err, s);
        default: return launch_ws_mode<N, K, SPHG_EPI_RESID>(A, B, M, ep, err, s);
    }
}

// ------------------------------------------------------------------------
// One message-passing edge layer in one kernel (inference):
//   a  = bf16(relu(E We^T + be + P[src, :128] + P[dst, 128:]))   (rows < nedge gather)
//   EF = EF + a W2^T + b2,   Eout = bf16(EF)
// or, without EF (a bf16 residual stream), Eout = bf16(E + a W2^T + b2) with
// E read back from the tile's copy in shared memory;
// which the network otherwise runs as two weight-stationary GEMMs (EDGE and
// RESID epilogues) with the 128-wide hidden rows `a` written to and read
// back from global memory.  Here a tile's hidden rows go from the first
// accumulator (TMEM columns 0..127) through the EDGE epilogue straight into
// shared memory, in the canonical K-major layout, as the A operand of the
// second MMA (columns 128..255).  Both weight matrices stay in shared memory
// for the whole launch.  Each CTA (one per SM, 16 warps: each TMEM lane
// quarter of the tile's rows is read by four warps of 32 columns each, so
// that enough epilogue loads are in flight) loops over 128-row tiles; the
// next tile's E rows are copied (cp.async) while the current tile's MMAs and
// epilogues run.  Sums are formed in the order of the two-GEMM path, so the
// results are bit-identical to it.  Every MMA wait is bounded; on timeout
// the kernel sets *err, waits (bounded) for its MMAs, frees TMEM and returns.
struct EdgeShape {
    static constexpr uint32_t T = 32 * 1024;                  // one 128 x 128 bf16 operand
    static constexpr int NBUF = 3;                            // tiles in flight: E rows, then the hidden rows
    static constexpr uint32_t B1 = 0, B2 = T, BUF = 2 * T;
    static constexpr uint32_t BAR = BUF + NBUF * T;           // mbarriers, TMEM slot, abort flag
    static constexpr int THREADS = 512;                       // two groups of 8 warps
    static constexpr uint32_t STAGE = BAR + 128;              // 16 warps x 2 KB staging
    static constexpr uint32_t SMEM = STAGE + (THREADS / 32) * 32 * 64;
};

template <int NT>
__device__ __forceinline__ void load_b128(uint8_t* sB, const __nv_bfloat16* __restrict__ B, int tid) {
    for (int c = tid; c < 128 * 16; c += NT) {
        const int r = c / 16, kc = c % 16;
        *reinterpret_cast<uint4*>(sB + kc * (128 * 16) + (r >> 3) * 128 + (r & 7) * 16) =
            *reinterpret_cast<const uint4*>(B + (size_t)r * 128 + kc * 8);
    }
}

__device__ __forceinline__ void mma_128x128(uint32_t tacc, const uint8_t* sA, const uint8_t* sB, uint64_t* bar) {
    const uint32_t idesc = make_idesc(128);
#pragma unroll
    for (int kk = 0; kk < 8; ++kk) {
        const uint64_t da = make_desc(smem_u32(sA + kk * 2 * 2048), 2048, 128);
        const uint64_t db = make_desc(smem_u32(sB + kk * 2 * 2048), 2048, 128);
        const uint32_t en = kk > 0 ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
            ::"r"(tacc), "l"(da), "l"(db), "r"(idesc), "r"(en), "r"(0), "r"(0), "r"(0), "r"(0));
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// barrier of one 256-thread group (named barrier id) that also ANDs `ok` over the group
__device__ __forceinline__ bool group_and(int id, bool ok) {
    uint32_t r;
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.and.pred p, %2, 256, p;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(r) : "r"(ok ? 1u : 0u), "r"(id) : "memory");
    return r != 0;
}

// The layer as a two-stage pipeline over the CTA's tiles.  Warps 0-7 (group
// 1) run the EDGE epilogue of tile i from the first accumulator into the
// tile's buffer (its E rows are no longer needed once the first MMA has read
// them); their thread 0 then issues the first MMA of tile i + 1.  Warps 8-15
// (group 2) issue the second MMA of tile i once its hidden rows are in
// place, run the RESID epilogue from the second accumulator, and load the E
// rows of tile i + NBUF into the buffer that tile i has freed (NBUF = 3).  So
// group 1 works on tile i + 1 while group 2 finishes tile i, and neither
// waits for the other's epilogue.  mbarriers: mma[0] / mma[1] each MMA
// group's completion (tcgen05.commit), z[b] the hidden rows of buffer b's
// tile written (group 1), buf[b] the E rows of buffer b's next tile loaded
// (the 256 threads of group 2); per buffer, so that no waiter can fall two
// phases behind its barrier.  Every wait is bounded; a group that gives up sets
// *err and the abort flag, and both groups leave their loops at the next wait.
__global__ void __launch_bounds__(EdgeShape::THREADS, 1) k_edge_layer(const __nv_bfloat16* __restrict__ E, int M,
                                                               const __nv_bfloat16* __restrict__ We,
                                                               const __nv_bfloat16* __restrict__ W2,
                                                               SphgGemmEpi e1, SphgGemmEpi e2,
                                                               int* __restrict__ err) {
    typedef EdgeShape S;
    extern __shared__ __align__(128) uint8_t smem[];
    uint64_t* bar_mma = (uint64_t*)(smem + S::BAR);      // [2]
    uint64_t* bar_z = bar_mma + 2;                       // [NBUF]
    uint64_t* bar_buf = bar_z + S::NBUF;                 // [NBUF]
    uint32_t* tslot = (uint32_t*)(bar_buf + S::NBUF);
    volatile int* abort_flag = (volatile int*)(tslot + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const bool g1 = warp < 8;
    float4* stage = reinterpret_cast<float4*>(smem + S::STAGE) + warp * 128;
    const int ntiles = M / 128;
    const int my = blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    auto tile_m0 = [&](int i) { return ((int)blockIdx.x + i * (int)gridDim.x) * 128; };
    auto buf = [&](int i) { return smem + S::BUF + (i % S::NBUF) * S::T; };

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(256));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar_mma)), "r"(1));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar_mma + 1)), "r"(1));
        for (int b = 0; b < S::NBUF; ++b) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar_z + b)), "r"(1));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar_buf + b)), "r"(256));
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::);
        *abort_flag = 0;
    }
    load_b128<S::THREADS>(smem + S::B1, We, tid);
    load_b128<S::THREADS>(smem + S::B2, W2, tid);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::);
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::);
    const uint32_t tmem = *tslot;
    const uint32_t lane_off = (uint32_t)((warp & 3) * 32) << 16;
    const int col0 = ((warp & 7) >> 2) * 64;    // this warp's half of the 128 columns
    const int gt = tid & 255;                    // thread index within the group
    int issued = 0;                              // MMA groups issued by this thread (thread 0 or 256)
    auto fail = [&]() { atomicExch(err, 1); *abort_flag = 1; };

    if (g1) {
        bool ok = true;
        for (int i = 0; i < my && ok; ++i) {
            if (tid == 0 && i == 0) {
                if (mbar_wait(smem_u32(bar_buf), 0u, kWaitLimit)) {
                    asm volatile("tcgen05.fence::after_thread_sync;" ::);
                    mma_128x128(tmem, buf(0), smem + S::B1, bar_mma);
                    ++issued;
                } else {
                    fail();
                }
            }
            const bool done = !*abort_flag && mbar_wait(smem_u32(bar_mma), (uint32_t)(i & 1), kWaitLimit);
            ok = group_and(1, done);
            if (!ok) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::);
            ws_epilogue_staged<128, 128, SPHG_EPI_EDGE>(e1, tmem + lane_off, (long long)tile_m0(i) + (warp & 3) * 32,
                                                        col0, stage, lane, buf(i), (warp & 3) * 32);
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;" ::);
            group_and(1, true);
            if (tid == 0) {
                mbar_arrive(bar_z + i % S::NBUF);   // tile i's hidden rows are in its buffer
                if (i + 1 < my) {
                    if (mbar_wait(smem_u32(bar_buf + (i + 1) % S::NBUF), (uint32_t)(((i + 1) / S::NBUF) & 1),
                                  kWaitLimit)) {
                        asm volatile("tcgen05.fence::after_thread_sync;" ::);
                        mma_128x128(tmem, buf(i + 1), smem + S::B1, bar_mma);
                        ++issued;
                    } else {
                        fail();   // the group leaves at its next wait
                    }
                }
            }
        }
        if (!ok && tid == 0) fail();
    } else {
        bool ok = true;
        // the first tiles' E rows
        for (int j = 0; j < S::NBUF && j < my; ++j) ws_load_a<128, 128, 256>(buf(j), E, tile_m0(j), gt);
        cp_async_commit();
        cp_async_wait_all();
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        for (int j = 0; j < S::NBUF && j < my; ++j) mbar_arrive(bar_buf + j);
        for (int i = 0; i < my && ok; ++i) {
            if (gt == 0) {   // the second MMA of tile i, once its hidden rows are in place
                if (!*abort_flag && mbar_wait(smem_u32(bar_z + i % S::NBUF), (uint32_t)((i / S::NBUF) & 1), kWaitLimit)) {
                    asm volatile("tcgen05.fence::after_thread_sync;" ::);
                    mma_128x128(tmem + 128u, buf(i), smem + S::B2, bar_mma + 1);
                    ++issued;
                } else {
                    fail();
                }
            }
            const bool done = !*abort_flag && mbar_wait(smem_u32(bar_mma + 1), (uint32_t)(i & 1), kWaitLimit);
            ok = group_and(2, done);
            if (!ok) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::);
            // both MMAs of tile i are done: its buffer takes the E rows of tile i + NBUF
            const bool more = i + S::NBUF < my;
            if (more) ws_load_a<128, 128, 256>(buf(i), E, tile_m0(i + S::NBUF), gt);
            cp_async_commit();
            // the residual is EF (e2.z) or, without it, tile i's bf16 E rows
            ws_epilogue_staged<128, 128, SPHG_EPI_RESID>(e2, tmem + lane_off + 128u,
                                                         (long long)tile_m0(i) + (warp & 3) * 32, col0, stage, lane,
                                                         nullptr, 0, 64, E);
            asm volatile("tcgen05.fence::before_thread_sync;" ::);
            group_and(2, true);   // the second accumulator is read out before the next MMA into it
            if (more) {
                cp_async_wait_all();
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                mbar_arrive(bar_buf + i % S::NBUF);
            }
        }
        cp_async_wait_all();
        if (!ok && gt == 0) fail();
    }
    if (*abort_flag && gt == 0 && issued > 0)   // bounded wait for this thread's last MMA group
        mbar_wait(smem_u32(bar_mma + (g1 ? 0 : 1)), (uint32_t)((issued - 1) & 1), kWaitLimit);
    asm volatile("tcgen05.fence::before_thread_sync;" ::);
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256));
}


// ------------------------------------------------------------------------
// Edge layer with the sender term inside the first GEMM (inference):
//   z  = [e | h[src]] . [We | Ws]^T + (Pd[dst] + be)      (K = 256)
//   e' = bf16(e + (relu(z) . W2^T + b2))
// h is the bf16 node latent, Ws the sender half of the node projection and
// Pd = h Wd^T its receiver half, computed once per node (fp32).  The sender
// rows are products of the same bf16 operands as the projection GEMM,
// accumulated in the same fp32 accumulator as the edge term; they are TMA
// gathers into shared memory that run ahead of the MMAs.  The receiver term
// is added in the epilogue: edges are sorted by receiver, so a tile's rows
// share a few Pd rows and their loads are L1 hits.  Warp roles:
//   warps 0-3, 13-16  hidden epilogue, two warps per TMEM lane quarter (64
//               columns each): acc1 -> + (Pd[dst] + be), relu, bf16 -> the
//               hidden rows, written back into acc1's columns 0-31 and 64-95
//   warps 4-7   output epilogue: acc2 -> + (e + b2) -> bf16 e' (global)
//   warp 8      one thread issues GEMM1 of every tile (as its K blocks arrive)
//   warp 9      one thread issues GEMM2 of every tile (as its hidden rows
//               arrive), with A (the hidden rows) read from TMEM
//   warp 10     loader: TMA copies of 16 KB K blocks into a ring of NSLOT
//               slots, in the 128-byte swizzle layout: an E block is one 2-D
//               tile, the first half of the sender rows 32 tile::gather4
//               copies of 4 rows; the slot's full barrier completes on the
//               copies' byte count
//   warps 11-12 row loaders: the second half of the sender rows by cp.async,
//               so that the TMA unit and the load/store path gather at once
// The encoder form (MODE 1) uses the same roles with one TMA feature block per
// tile and no row loaders; the node-MLP form (MODE 2) four TMA blocks of the
// [h | agg] rows and an output epilogue onto the fp32 residual stream.
// TMEM: two GEMM1 accumulators (each also holding its tile's hidden rows
// until GEMM2 has read them) and two GEMM2 accumulators, 512 columns; so
// GEMM1 of tile i + 1 overlaps the epilogues and GEMM2 of tile i, and neither
// GEMM's issue waits for the other's inputs.  Resident in shared memory:
// [We | Ws] (64 KB), W2 (32 KB), the ring (64 KB: one tile's K blocks), be
// and b2.  Every wait is bounded; a role that gives up sets *err and the
// abort flag, the others leave at their next wait, and each MMA thread drains
// its MMAs before TMEM is freed.
struct EdgeNodeShape {
    static constexpr uint32_t KC = 128 * 16;             // one 16-byte column of a 128-row operand
    static constexpr uint32_t B1 = 0;                    // [We | Ws]: 32 columns
    static constexpr uint32_t B2 = B1 + 32 * KC;         // W2: 16 columns
    // four slots (one tile's K blocks) measured faster than eight (0.893 against 0.927 ms
    // per 5.12M rows): the shared memory they leave to L1 holds the prefetched receiver rows
    static constexpr int NSLOT = 4;
    static constexpr uint32_t SLOT = 8 * KC;             // one K block of 64 (128 rows x 128 swizzled bytes)
    static constexpr uint32_t RING = B2 + 16 * KC;
    static constexpr uint32_t BIAS = RING + NSLOT * SLOT;  // be, b2 (fp32)
    static constexpr uint32_t BAR = BIAS + 2 * 128 * 4;
    static constexpr uint32_t SMEM = BAR + 256 + 1024;   // + alignment of the ring to 1024 bytes
    static constexpr int KBLK = 4;                       // K blocks of GEMM1 per tile: E, E, h[src], h[src]
    static constexpr int CPB = 3;                        // the K block copied by cp.async (slot 3)
    static constexpr int ROWLOADERS = 64;                // its copy threads (warps 11-12)
    static constexpr int THREADS = 17 * 32;              // + warps 13-16: the second half of the hidden epilogue
};
static_assert(EdgeNodeShape::SMEM <= 227 * 1024, "edge layer shared memory");
static_assert(EdgeNodeShape::NSLOT % EdgeNodeShape::KBLK == 0, "a slot always holds the same K block");


// 32 accumulator columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}

// 32 contiguous bytes per thread (256-bit global accesses, sm_100); the load is
// cached in L2 only
__device__ __forceinline__ void ld_global_32B(const void* p, uint32_t* r) {
    asm volatile("ld.global.cg.v8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "l"(p));
}
__device__ __forceinline__ void st_global_32B(void* p, const uint32_t* r) {
    asm volatile("st.global.v8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(p), "r"(r[0]), "r"(r[1]), "r"(r[2]),
                 "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
                 : "memory");
}

// shared-memory descriptor of a K-major operand in the 128-byte swizzle layout that
// TMA writes with CU_TENSOR_MAP_SWIZZLE_128B: row r of an 8-row, 1024-byte atom at
// r * 128 with its 16-byte chunks XOR-permuted by r; atoms SBO = 1024 bytes apart.
// The start address moves 32 bytes per K = 16 step inside the 128-byte rows.
__device__ __forceinline__ uint64_t make_desc_sw128(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;              // leading byte offset: unused for swizzled K-major (16 bytes)
    d |= (uint64_t)(1024 >> 4) << 32;    // stride byte offset: 8 rows x 128 bytes
    d |= (uint64_t)1 << 46;              // version
    d |= (uint64_t)2 << 61;              // SWIZZLE_128B
    return d;
}

__device__ __forceinline__ void umma_f16(uint32_t tacc, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        ::"r"(tacc), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}
// A from TMEM (tcgen05.mma ... [d], [a], b_desc, ...): the A tile is 128 lanes (rows)
// x 8 columns per K = 16 step, two bf16 of consecutive K in each 32-bit column
__device__ __forceinline__ void umma_f16_ta(uint32_t tacc, uint32_t ta, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        ::"r"(tacc), "r"(ta), "l"(db), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}
// 8 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t* r) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(taddr),
                 "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
                 : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// MODE 0: the edge layer.  MODE 1 (ENC): the edge encoder in the same pipeline,
// E_out = bf16(relu(E We^T + be) W2^T + b2) with E the [M x 64] bf16 edge features
// (one K block per tile, no node rows, no receiver term, no residual).  MODE 2
// (NODE): a node MLP, z = z + (relu(E We^T + be) W2^T + b2) with E the [M x 256]
// bf16 rows [h | agg] (four TMA K blocks per tile) and z the fp32 residual stream
// (Z, in place), E_out = bf16(z).  The encoder and node forms form the same sums, in
// the same order, as two weight-stationary GEMMs (BIAS_ACT, then BIAS_ACT or RESID).
template <int MODE>
__global__ void __launch_bounds__(EdgeNodeShape::THREADS, 1)
    k_edge_layer_nodes(const __grid_constant__ CUtensorMap tmE, const __grid_constant__ CUtensorMap tmH,
                       const __nv_bfloat16* E, __nv_bfloat16* E_out, const __nv_bfloat16* __restrict__ H,
                       const float* __restrict__ Pd, int nnode,
                       const int* __restrict__ src, const int* __restrict__ dst, long long nedge, int M,
                       const __nv_bfloat16* __restrict__ We, const __nv_bfloat16* __restrict__ Ws,
                       const float* __restrict__ be,
                       const __nv_bfloat16* __restrict__ W2, const float* __restrict__ b2, float* Z,
                       int* __restrict__ err) {
    typedef EdgeNodeShape S;
    constexpr bool ENC = MODE == 1, NODE = MODE == 2, GATHER = MODE == 0;
    constexpr int KBLK = ENC ? 1 : S::KBLK;              // K blocks of GEMM1 per tile
    constexpr int CPB = GATHER ? S::CPB : -1;            // the block the row loaders copy
    extern __shared__ __align__(128) uint8_t smem[];
    // the swizzled ring slots need 1024-byte alignment in the shared window
    uint8_t* sm = smem + ((1024u - (smem_u32(smem) & 1023u)) & 1023u);
    uint64_t* full = (uint64_t*)(sm + S::BAR);          // [NSLOT] loaders -> MMA
    uint64_t* empty = full + S::NSLOT;                    // [NSLOT] MMA (commit) -> loaders
    uint64_t* acc1_full = empty + S::NSLOT;               // [2]
    uint64_t* acc1_empty = acc1_full + 2;                 // [2]
    uint64_t* acc2_full = acc1_empty + 2;                 // [2]
    uint64_t* acc2_empty = acc2_full + 2;                 // [2]
    uint64_t* hid_full = acc2_empty + 2;                 // [2] per GEMM1 accumulator: no waiter can fall
                                                         // two phases behind (ep1 may run a tile ahead)
    uint64_t* drain = hid_full + 2;                      // [2] one per MMA thread
    uint32_t* tslot = (uint32_t*)(drain + 2);
    volatile int* abort_flag = (volatile int*)(tslot + 1);
    const float* sbe = (const float*)(sm + S::BIAS);
    const float* sb2 = sbe + 128;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ntiles = M / 128;
    const int my = blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    auto tile_m0 = [&](int i) { return ((long long)blockIdx.x + (long long)i * gridDim.x) * 128; };
    auto fail = [&]() { atomicOr(err, 1); *abort_flag = 1; };

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(512));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (tid == 0) {
        for (int s = 0; s < S::NSLOT; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(full + s)),
                         "r"(s % KBLK == CPB ? S::ROWLOADERS : 1));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(empty + s)), "r"(1));
        }
        for (int a = 0; a < 2; ++a) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(acc1_full + a)), "r"(1));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(acc1_empty + a)), "r"(1));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(acc2_full + a)), "r"(1));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(acc2_empty + a)), "r"(128));
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(hid_full)), "r"(256));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(hid_full + 1)), "r"(256));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(drain)), "r"(1));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(drain + 1)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::);
        *abort_flag = 0;
    }
    // resident operands: column kc of [We | Ws] (of We alone, K = 64, for ENC) holds K
    // elements 8 kc .. 8 kc + 7
    constexpr int B1COLS = ENC ? 8 : 32;
    for (int c = tid; c < 128 * B1COLS; c += S::THREADS) {
        const int n = c / B1COLS, kc = c % B1COLS;
        const __nv_bfloat16* from = ENC ? We + (size_t)n * 64 + kc * 8
                                  : NODE ? We + (size_t)n * 256 + kc * 8
                                  : kc < 16 ? We + (size_t)n * 128 + kc * 8 : Ws + (size_t)n * 128 + (kc - 16) * 8;
        *reinterpret_cast<uint4*>(sm + S::B1 + kc * S::KC + (n >> 3) * 128 + (n & 7) * 16) =
            *reinterpret_cast<const uint4*>(from);
    }
    load_b128<S::THREADS>(sm + S::B2, W2, tid);
    for (int c = tid; c < 256; c += S::THREADS)
        reinterpret_cast<float*>(sm + S::BIAS)[c] = c < 128 ? be[c] : b2[c - 128];
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::);
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::);
    const uint32_t tmem = *tslot;

    if (warp < 4 || warp >= 13) {
        // ---- hidden epilogue, two warps per TMEM lane quarter (warp % 4): warps 0-3 take
        // accumulator columns 0-63, warps 13-16 columns 64-127, 16 at a time.  The hidden
        // rows go back into columns the warp has itself read: K 0-63 to columns 0-31, K
        // 64-127 to columns 64-95 (two bf16 per column).  The receiver's row of Pd is
        // prefetched into L1 a tile ahead (its index loaded two tiles ahead); rows of a
        // tile share few receivers, so most of these loads hit the same lines.
        const int q4 = warp & 3, half = warp >= 13 ? 1 : 0;
        const uint32_t lane_off = (uint32_t)(q4 * 32) << 16;
        const int r = q4 * 32 + lane;
        auto receiver = [&](int i) {
            const long long e = tile_m0(i) + r;
            return GATHER && e < nedge ? dst[e] : -1;
        };
        auto checked = [&](int i, int d) {   // -1 for padding rows and (flagged) indices outside the node rows
            if (GATHER && tile_m0(i) + r < nedge && (d < 0 || d >= nnode)) {
                if (half == 0) atomicOr(err, 2);
                return -1;
            }
            return d;
        };
        auto prefetch_row = [&](int d) {
            if (d >= 0)
                for (int q = 0; q < 2; ++q)
                    asm volatile("prefetch.global.L1 [%0];" ::"l"(Pd + (size_t)d * 128 + 64 * half + 32 * q));
        };
        int d_cur = my > 0 ? checked(0, receiver(0)) : -1;
        int d_next = my > 1 ? receiver(1) : -1;
        prefetch_row(d_cur);
        for (int i = 0; i < my; ++i) {
            const int a = i & 1;
            if (i + 1 < my) { d_next = checked(i + 1, d_next); prefetch_row(d_next); }
            const int d_after = i + 2 < my ? receiver(i + 2) : -1;
            const float4* pd =
                d_cur >= 0 ? reinterpret_cast<const float4*>(Pd + (size_t)d_cur * 128 + 64 * half) : nullptr;
            float4 pa[4], pb[4];   // Pd chunks c and c + 1 (16 columns each)
#pragma unroll
            for (int q = 0; q < 4; ++q) pa[q] = pd ? pd[q] : make_float4(0.f, 0.f, 0.f, 0.f);
            bool ok = !*abort_flag && mbar_wait(smem_u32(acc1_full + a), (uint32_t)((i >> 1) & 1), kWaitLimit);
            ok = __all_sync(0xffffffffu, ok);   // the warp's tcgen05.ld / st are warp-collective
            if (!ok) { fail(); break; }
            asm volatile("tcgen05.fence::after_thread_sync;" ::);
            const uint32_t acc = tmem + lane_off + (uint32_t)(a * 128);
#pragma unroll
            for (int c = 0; c < 4; ++c) {   // 16 accumulator columns at a time
                float4* p = (c & 1) ? pb : pa;
                float4* pn = (c & 1) ? pa : pb;
                if (c < 3) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) pn[q] = pd ? pd[4 * (c + 1) + q] : make_float4(0.f, 0.f, 0.f, 0.f);
                }
                const int cg = 64 * half + 16 * c;   // the chunk's first accumulator column
                float v[16];
                tmem_ld16(acc + (uint32_t)cg, v);
                uint32_t h[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int col = cg + 2 * j;
                    const float4 t4 = p[j >> 1];
                    const float p0 = (j & 1) ? t4.z : t4.x, p1 = (j & 1) ? t4.w : t4.y;
                    const __nv_bfloat162 t = __floats2bfloat162_rn(fmaxf(v[2 * j] + (p0 + sbe[col]), 0.f),
                                                                   fmaxf(v[2 * j + 1] + (p1 + sbe[col + 1]), 0.f));
                    h[j] = *reinterpret_cast<const uint32_t*>(&t);
                }
                tmem_st8(acc + (uint32_t)(64 * half + 8 * c), h);
            }
            asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;" ::);
            mbar_arrive(hid_full + a);
            d_cur = d_next;
            d_next = d_after;
        }
    } else if (warp < 8) {
        // ---- output epilogue
        const int w = warp & 3, r = w * 32 + lane;
        const uint32_t lane_off = (uint32_t)(w * 32) << 16;
        for (int i = 0; i < my; ++i) {
            const int a = i & 1;
            const long long grow = tile_m0(i) + r;
            // the residual row, 32 columns (64 bytes) at a time, each chunk loaded one chunk
            // ahead; the first while the tile's GEMMs run (one lane per row, 32-byte accesses)
            const uint8_t* er = reinterpret_cast<const uint8_t*>(E + grow * 128);
            uint32_t ra_[16], rb_[16];
            if (GATHER) { ld_global_32B(er, ra_); ld_global_32B(er + 32, ra_ + 8); }
            bool ok = !*abort_flag && mbar_wait(smem_u32(acc2_full + a), (uint32_t)((i >> 1) & 1), kWaitLimit);
            ok = __all_sync(0xffffffffu, ok);
            if (!ok) { fail(); break; }
            asm volatile("tcgen05.fence::after_thread_sync;" ::);
            uint8_t* out = reinterpret_cast<uint8_t*>(E_out + grow * 128);
            if (NODE) {   // z = acc + (z + b2), in place; E_out = bf16(z)
                float4* zr = reinterpret_cast<float4*>(Z + grow * 128);
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    float4 zc[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) zc[q] = zr[8 * c + q];
                    float v[32];
                    tmem_ld32(tmem + lane_off + (uint32_t)(256 + a * 128 + 32 * c), v);
                    uint32_t o[16];
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        const int col = 32 * c + 4 * q;
                        const float4 zq = zc[q];
                        const float4 nz = make_float4(v[4 * q] + (zq.x + sb2[col]), v[4 * q + 1] + (zq.y + sb2[col + 1]),
                                                      v[4 * q + 2] + (zq.z + sb2[col + 2]),
                                                      v[4 * q + 3] + (zq.w + sb2[col + 3]));
                        zr[8 * c + q] = nz;
                        const __nv_bfloat162 t0 = __floats2bfloat162_rn(nz.x, nz.y), t1 = __floats2bfloat162_rn(nz.z, nz.w);
                        o[2 * q] = *reinterpret_cast<const uint32_t*>(&t0);
                        o[2 * q + 1] = *reinterpret_cast<const uint32_t*>(&t1);
                    }
                    st_global_32B(out + 64 * c, o);
                    st_global_32B(out + 64 * c + 32, o + 8);
                }
            }
#pragma unroll
            for (int c = 0; c < (NODE ? 0 : 4); ++c) {
                uint32_t* res = (c & 1) ? rb_ : ra_;
                uint32_t* rn = (c & 1) ? ra_ : rb_;
                if (GATHER && c < 3) { ld_global_32B(er + 64 * (c + 1), rn); ld_global_32B(er + 64 * (c + 1) + 32, rn + 8); }
                float v[32];
                tmem_ld32(tmem + lane_off + (uint32_t)(256 + a * 128 + 32 * c), v);
                uint32_t o[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int col = 32 * c + 2 * j;
                    __nv_bfloat162 t;
                    if (ENC) {
                        t = __floats2bfloat162_rn(v[2 * j] + sb2[col], v[2 * j + 1] + sb2[col + 1]);
                    } else {
                        const float2 e2 = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&res[j]));
                        t = __floats2bfloat162_rn(v[2 * j] + (e2.x + sb2[col]), v[2 * j + 1] + (e2.y + sb2[col + 1]));
                    }
                    o[j] = *reinterpret_cast<const uint32_t*>(&t);
                }
                st_global_32B(out + 64 * c, o);
                st_global_32B(out + 64 * c + 32, o + 8);
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::);
            mbar_arrive(acc2_empty + a);
        }
    } else if (warp < 10) {
        // ---- MMA issue: lane 0 of warp 8 issues GEMM1 of every tile, lane 0 of warp 9 GEMM2
        if (lane == 0) {
            const uint32_t idesc = make_idesc(128);
            bool ok = true;
            if (warp == 8) {
                for (int i = 0; i < my && ok; ++i) {
                    const int a = i & 1;
                    if (i >= 2 && !(ok = !*abort_flag && mbar_wait(smem_u32(acc1_empty + a),
                                                                   (uint32_t)(((i >> 1) & 1) ^ 1), kWaitLimit)))
                        break;
                    for (int kb = 0; kb < KBLK && ok; ++kb) {
                        const int j = i * KBLK + kb, s = j % S::NSLOT;
                        if (!(ok = !*abort_flag &&
                                   mbar_wait(smem_u32(full + s), (uint32_t)((j / S::NSLOT) & 1), kWaitLimit)))
                            break;
                        // the cp.async block was written through the generic proxy; the MMAs read the async proxy
                        if (kb == CPB) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                        asm volatile("tcgen05.fence::after_thread_sync;" ::);
#pragma unroll
                        for (int kk = 0; kk < 4; ++kk) {   // K = 16 is 32 bytes into the swizzled 128-byte rows
                            const uint64_t da = make_desc_sw128(smem_u32(sm + S::RING + s * S::SLOT + kk * 32));
                            const uint64_t db = make_desc(smem_u32(sm + S::B1 + (kb * 8 + kk * 2) * S::KC), S::KC, 128);
                            umma_f16(tmem + (uint32_t)(a * 128), da, db, idesc, (kb | kk) != 0 ? 1u : 0u);
                        }
                        umma_commit(empty + s);   // the slot is free once these MMAs have read it
                    }
                    if (ok) umma_commit(acc1_full + a);
                }
            } else {
                for (int i = 0; i < my && ok; ++i) {
                    const int a = i & 1;
                    if (!(ok = !*abort_flag &&
                               mbar_wait(smem_u32(hid_full + a), (uint32_t)((i >> 1) & 1), kWaitLimit)))
                        break;
                    if (i >= 2 && !(ok = !*abort_flag && mbar_wait(smem_u32(acc2_empty + a),
                                                                   (uint32_t)(((i >> 1) & 1) ^ 1), kWaitLimit)))
                        break;
                    asm volatile("tcgen05.fence::after_thread_sync;" ::);
#pragma unroll
                    for (int kk = 0; kk < 8; ++kk) {
                        const uint64_t db = make_desc(smem_u32(sm + S::B2 + kk * 2 * S::KC), S::KC, 128);
                        umma_f16_ta(tmem + (uint32_t)(256 + a * 128), tmem + (uint32_t)(a * 128 + (kk < 4 ? 8 * kk : 64 + 8 * (kk - 4))), db, idesc,
                                    kk != 0 ? 1u : 0u);
                    }
                    umma_commit(acc1_empty + a);   // the hidden rows (in GEMM1's accumulator) have been read
                    umma_commit(acc2_full + a);
                }
            }
            if (!ok) fail();
            // every MMA issued by this thread has completed before TMEM is freed
            umma_commit(drain + (warp - 8));
            mbar_wait(smem_u32(drain + (warp - 8)), 0u, kWaitLimit);
        }
    } else if (warp == 10) {
        // ---- loader warp: TMA copies into the ring.  An edge-row block is one 2-D tile
        // (64 columns x 128 rows); a node-row block is 32 tile::gather4 copies, lane l
        // bringing the rows of edges 4l .. 4l + 3.  An index outside [0, nnode) becomes
        // row nnode, which lies outside the tensor map and is filled with zeros.
        bool ok = true;
        int sr[4], nsr[4];
        auto fetch = [&](int i) {   // raw sender indices of the lane's 4 rows, loaded one tile ahead
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const long long e = tile_m0(i) + 4 * lane + q;
                nsr[q] = GATHER && e < nedge ? src[e] : 0;
            }
        };
        if (my > 0) fetch(0);
        for (int i = 0; i < my && ok; ++i) {
            const long long m0 = tile_m0(i);
#pragma unroll
            for (int q = 0; q < 4; ++q) sr[q] = nsr[q];
            if (i + 1 < my) fetch(i + 1);
            if (lane == 0) {   // the edge rows of the tile after next into L2 (one bulk prefetch)
                constexpr int ROWB = ENC ? 128 : NODE ? 512 : 256;   // bytes per row of E
                for (int t = i == 0 ? 1 : i + 2; t <= i + 2 && t < my; ++t)
                    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(
                                     reinterpret_cast<const uint8_t*>(E) + tile_m0(t) * ROWB),
                                 "r"(128 * ROWB)
                                 : "memory");
            }
            bool bad = false;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const bool real = m0 + 4 * lane + q < nedge;
                const bool sv = sr[q] >= 0 && sr[q] < nnode;
                bad |= real && !sv;
                if (!real || !sv) sr[q] = nnode;
            }
            if (GATHER && bad) atomicOr(err, 2);   // an index outside the node rows
            for (int kb = 0; kb < KBLK; ++kb) {
                if (kb == CPB) continue;   // the row loaders' block
                const int j = i * KBLK + kb, s = j % S::NSLOT;
                bool got = true;
                if (lane == 0 && j >= S::NSLOT)
                    got = !*abort_flag &&
                          mbar_wait(smem_u32(empty + s), (uint32_t)(((j / S::NSLOT) & 1) ^ 1), kWaitLimit);
                if (!(ok = __shfl_sync(0xffffffffu, got, 0))) break;
                const uint32_t slot = smem_u32(sm + S::RING + s * S::SLOT);
                const uint32_t fb = smem_u32(full + s);
                const int x = NODE ? kb * 64 : (kb & 1) * 64;   // first column of the block (128 bytes: the swizzle span)
                if (lane == 0)
                    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(fb), "r"(S::SLOT)
                                 : "memory");
                __syncwarp();
                if (kb < 2 || !GATHER) {
                    if (lane == 0)
                        asm volatile(
                            "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                            " [%0], [%1, {%2, %3}], [%4];" ::"r"(slot), "l"(&tmE), "r"(x), "r"((int)m0), "r"(fb)
                            : "memory");
                } else {
                    asm volatile(
                        "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes"
                        " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(slot + 4 * lane * 128), "l"(&tmH), "r"(x),
                        "r"(sr[0]), "r"(sr[1]), "r"(sr[2]), "r"(sr[3]), "r"(fb)
                        : "memory");
                }
            }
        }
        if (!ok && lane == 0) fail();
    } else if (GATHER) {
        // ---- row loaders (warps 11-12): the second half of the sender rows (K block CPB)
        // by cp.async, 16 bytes per request, into the same 128-byte swizzle layout
        // (16-byte chunk u of row r at r * 128 + (u ^ (r & 7)) * 16); each instruction
        // covers 8 rows x 64 contiguous bytes, and the 8 rows' chunks fall in distinct
        // banks.  The slot's full barrier counts each thread once its copies have landed.
        const int lt = tid - 11 * 32, lw = lt >> 5;
        const int rlo = lane & 7, uq = lane >> 3;
        bool ok = true;
        int sn[8], nsn[8];
        auto fetch = [&](int i) {
#pragma unroll
            for (int g = 0; g < 8; ++g) {
                const long long e = tile_m0(i) + 64 * lw + 8 * g + rlo;
                nsn[g] = e < nedge ? src[e] : -1;
            }
        };
        if (my > 0) fetch(0);
        for (int i = 0; i < my && ok; ++i) {
            const long long m0 = tile_m0(i);
#pragma unroll
            for (int g = 0; g < 8; ++g) sn[g] = nsn[g];
            if (i + 1 < my) fetch(i + 1);
            const int j = i * S::KBLK + S::CPB, s = j % S::NSLOT;
            if (j >= S::NSLOT &&
                !(ok = !*abort_flag &&
                       mbar_wait(smem_u32(empty + s), (uint32_t)(((j / S::NSLOT) & 1) ^ 1), kWaitLimit)))
                break;
            const uint32_t slot = smem_u32(sm + S::RING + s * S::SLOT);
#pragma unroll
            for (int g = 0; g < 8; ++g) {
                const int row = 64 * lw + 8 * g + rlo;
                const bool v = sn[g] >= 0 && sn[g] < nnode;   // out-of-range indices are flagged by the TMA loader
                const __nv_bfloat16* from = H + (size_t)(v ? sn[g] : 0) * 128 + 64;
#pragma unroll
                for (int t = 0; t < 2; ++t) {
                    const int u = 4 * t + uq;
                    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(slot + row * 128 +
                                                                                       ((u ^ rlo) << 4)),
                                 "l"(from + u * 8), "r"(v ? 16 : 0)
                                 : "memory");
                }
            }
            asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(full + s)) : "memory");
        }
        cp_async_wait_all();
        if (!ok) fail();
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::);
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
}

}  // namespace

// cuTensorMapEncodeTiled from the driver, through the runtime (no link to libcuda)
static CUresult encode_tiled(CUtensorMap* map, const void* base, uint64_t rows, uint32_t box_rows,
                             uint64_t cols = 128) {
    typedef CUresult (*Encode)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                               const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                               CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    static Encode encode = nullptr;
    if (!encode) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            return CUDA_ERROR_NOT_FOUND;
        encode = (Encode)fn;
    }
    // rows of `cols` bf16; boxes of 64 columns (128 bytes, the swizzle span)
    const cuuint64_t dims[2] = {cols, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {cols * 2};
    const cuuint32_t box[2] = {64, box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
}

extern "C" int sphg_gnn_edge_layer_nodes(const void* E, void* E_out, const void* H, const float* Pd, int nnode,
                                         const int* src, const int* dst, long long nedge, int M, const void* We,
                                         const void* Ws, const float* be, const void* W2, const float* b2,
                                         int* err_dev, void* stream) {
    if (!E || !E_out || !H || !Pd || !src || !dst || !We || !Ws || !be || !W2 || !b2 || !err_dev)
        return SPHG_ERR_BAD_ARG;
    if (M <= 0 || M % 128 || nedge < 0 || nedge > M || nnode <= 0 || nnode >= (1 << 30)) return SPHG_ERR_BAD_ARG;
    if (((((uintptr_t)E) | ((uintptr_t)E_out)) & 31) ||
        ((((uintptr_t)H) | ((uintptr_t)Pd) | ((uintptr_t)We) | ((uintptr_t)Ws) | ((uintptr_t)be) | ((uintptr_t)W2) |
          ((uintptr_t)b2)) &
         15))
        return SPHG_ERR_BAD_ARG;
    static bool configured = false;
    if (!configured) {
        if (cudaFuncSetAttribute(k_edge_layer_nodes<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)EdgeNodeShape::SMEM) != cudaSuccess)
            return SPHG_ERR_CUDA;
        configured = true;
    }
    CUtensorMap tmE, tmH;   // E: 128-row tiles; H: one row per gather4 row (the box is one row high)
    if (encode_tiled(&tmE, E, (uint64_t)M, 128) != CUDA_SUCCESS || encode_tiled(&tmH, H, (uint64_t)nnode, 1) != CUDA_SUCCESS)
        return SPHG_ERR_CUDA;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int ntiles = M / 128;
    const int grid = ntiles < sms ? ntiles : sms;
    k_edge_layer_nodes<0><<<grid, EdgeNodeShape::THREADS, EdgeNodeShape::SMEM, (cudaStream_t)stream>>>(
        tmE, tmH, (const __nv_bfloat16*)E, (__nv_bfloat16*)E_out, (const __nv_bfloat16*)H, Pd, nnode, src, dst, nedge, M,
        (const __nv_bfloat16*)We, (const __nv_bfloat16*)Ws, be, (const __nv_bfloat16*)W2, b2, nullptr, err_dev);
    return cudaGetLastError() == cudaSuccess ? SPHG_OK : SPHG_ERR_CUDA;
}

extern "C" int sphg_gnn_edge_encoder(const void* F, void* E_out, int M, const void* W1, const float* b1, const void* W2,
                                     const float* b2, int* err_dev, void* stream) {
    if (!F || !E_out || !W1 || !b1 || !W2 || !b2 || !err_dev) return SPHG_ERR_BAD_ARG;
    if (M <= 0 || M % 128) return SPHG_ERR_BAD_ARG;
    if ((((uintptr_t)E_out) & 31) ||
        ((((uintptr_t)F) | ((uintptr_t)W1) | ((uintptr_t)b1) | ((uintptr_t)W2) | ((uintptr_t)b2)) & 15))
        return SPHG_ERR_BAD_ARG;
    static bool configured = false;
    if (!configured) {
        if (cudaFuncSetAttribute(k_edge_layer_nodes<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)EdgeNodeShape::SMEM) != cudaSuccess)
            return SPHG_ERR_CUDA;
        configured = true;
    }
    CUtensorMap tmF;   // 128-row tiles of the 64 feature columns
    if (encode_tiled(&tmF, F, (uint64_t)M, 128, 64) != CUDA_SUCCESS) return SPHG_ERR_CUDA;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int ntiles = M / 128;
    const int grid = ntiles < sms ? ntiles : sms;
    // the node-row map is unused by the encoder form; pass the feature map in its place
    k_edge_layer_nodes<1><<<grid, EdgeNodeShape::THREADS, EdgeNodeShape::SMEM, (cudaStream_t)stream>>>(
        tmF, tmF, (const __nv_bfloat16*)F, (__nv_bfloat16*)E_out, nullptr, nullptr, 1, nullptr, nullptr, 0, M,
        (const __nv_bfloat16*)W1, nullptr, b1, (const __nv_bfloat16*)W2, b2, nullptr, err_dev);
    return cudaGetLastError() == cudaSuccess ? SPHG_OK : SPHG_ERR_CUDA;
}

extern "C" int sphg_gnn_node_mlp(const void* X, int M, const void* V1, const float* c1, const void* V2,
                                 const float* c2, float* Z, void* H_out, int* err_dev, void* stream) {
    if (!X || !V1 || !c1 || !V2 || !c2 || !Z || !H_out || !err_dev) return SPHG_ERR_BAD_ARG;
    if (M <= 0 || M % 128) return SPHG_ERR_BAD_ARG;
    if ((((uintptr_t)H_out) & 31) || ((((uintptr_t)X) | ((uintptr_t)V1) | ((uintptr_t)c1) | ((uintptr_t)V2) |
                                        ((uintptr_t)c2) | ((uintptr_t)Z)) & 15))
        return SPHG_ERR_BAD_ARG;
    static bool configured = false;
    if (!configured) {
        if (cudaFuncSetAttribute(k_edge_layer_nodes<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)EdgeNodeShape::SMEM) != cudaSuccess)
            return SPHG_ERR_CUDA;
        configured = true;
    }
    CUtensorMap tmX;   // 128-row tiles of the 256 columns [h | agg]
    if (encode_tiled(&tmX, X, (uint64_t)M, 128, 256) != CUDA_SUCCESS) return SPHG_ERR_CUDA;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int ntiles = M / 128;
    const int grid = ntiles < sms ? ntiles : sms;
    k_edge_layer_nodes<2><<<grid, EdgeNodeShape::THREADS, EdgeNodeShape::SMEM, (cudaStream_t)stream>>>(
        tmX, tmX, (const __nv_bfloat16*)X, (__nv_bfloat16*)H_out, nullptr, nullptr, 1, nullptr, nullptr, 0, M,
        (const __nv_bfloat16*)V1, nullptr, c1, (const __nv_bfloat16*)V2, c2, Z, err_dev);
    return cudaGetLastError() == cudaSuccess ? SPHG_OK : SPHG_ERR_CUDA;
}

extern "C" int sphg_gnn_edge_layer(const void* E, float* EF, void* E_out, const float* P, const int* src,
                                   const int* dst, long long nedge, int M, const void* We, const float* be,
                                   const void* W2, const float* b2, int* err_dev, void* stream) {
    if (!E || !E_out || !P || !src || !dst || !We || !be || !W2 || !b2 || !err_dev) return SPHG_ERR_BAD_ARG;
    if (M <= 0 || M % 128 || nedge < 0 || nedge > M) return SPHG_ERR_BAD_ARG;
    if ((((uintptr_t)E) | ((uintptr_t)EF) | ((uintptr_t)E_out) | ((uintptr_t)P) | ((uintptr_t)We) | ((uintptr_t)be) |
         ((uintptr_t)W2) | ((uintptr_t)b2)) & 15)
        return SPHG_ERR_BAD_ARG;
    static bool configured = false;
    if (!configured) {
        if (cudaFuncSetAttribute(k_edge_layer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)EdgeShape::SMEM) !=
            cudaSuccess)
            return SPHG_ERR_CUDA;
        configured = true;
    }
    SphgGemmEpi e1{};
    e1.mode = SPHG_EPI_EDGE; e1.relu = 1; e1.bias = be; e1.P = P; e1.src = src; e1.dst = dst; e1.nedge = nedge;
    SphgGemmEpi e2{};
    e2.mode = SPHG_EPI_RESID; e2.bias = b2; e2.z = EF; e2.h = E_out;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int ntiles = M / 128;
    const int grid = ntiles < sms ? ntiles : sms;
    k_edge_layer<<<grid, EdgeShape::THREADS, EdgeShape::SMEM, (cudaStream_t)stream>>>(
        (const __nv_bfloat16*)E, M, (const __nv_bfloat16*)We, (const __nv_bfloat16*)W2, e1, e2, err_dev);
    return cudaGetLastError() == cudaSuccess ? SPHG_OK : SPHG_ERR_CUDA;
}

extern "C" int sphg_gemm_bf16_ws(const void* A, const void* B, int M, int N, int K, const SphgGemmEpi* epi,
                                 int* err_dev, void* stream) {
    if (!A || !B || !epi || !err_dev || M <= 0 || M % 128) return SPHG_ERR_BAD_ARG;
    if ((((uintptr_t)A) | ((uintptr_t)B)) & 15) return SPHG_ERR_BAD_ARG;
    const SphgGemmEpi& e = *epi;
    if (e.mode < SPHG_EPI_STORE || e.mode > SPHG_EPI_RESID) return SPHG_ERR_BAD_ARG;
    const bool need_z = e.mode == SPHG_EPI_STORE || e.mode == SPHG_EPI_ACC || e.mode == SPHG_EPI_RESID;
    if ((need_z && !e.z) || (e.mode != SPHG_EPI_STORE && e.mode != SPHG_EPI_ACC && !e.bias)) return SPHG_ERR_BAD_ARG;
    if (e.mode == SPHG_EPI_EDGE && (!e.P || !e.src || !e.dst || !e.h || e.nedge < 0 || e.nedge > M))
        return SPHG_ERR_BAD_ARG;
    if ((((uintptr_t)e.z) | ((uintptr_t)e.h) | ((uintptr_t)e.bias) | ((uintptr_t)e.P)) & 15) return SPHG_ERR_BAD_ARG;
    const __nv_bfloat16* a = (const __nv_bfloat16*)A;
    const __nv_bfloat16* b = (const __nv_bfloat16*)B;
    cudaStream_t s = (cudaStream_t)stream;
    if (N == 128 && K == 64) return launch_ws<128, 64>(a, b, M, e, err_dev, s);
    if (N == 128 && K == 128) return launch_ws<128, 128>(a, b, M, e, err_dev, s);
    if (N == 256 && K == 128) return launch_ws<256, 128>(a, b, M, e, err_dev, s);
    if (N == 128 && K == 256) return launch_ws<128, 256>(a, b, M, e, err_dev, s);
    return SPHG_ERR_UNSUPPORTED;
}

extern "C" int sphg_gemm_bf16_tn(const void* A, const void* B, float* C, int M, int N, int K, int accumulate,
                                 int split_k, int* err_dev, void* stream) {
    if (!A || !B || !C || !err_dev) return SPHG_ERR_BAD_ARG;
    if (M <= 0 || N <= 0 || K <= 0 || M % 128 || N % 16 || K % 64) return SPHG_ERR_BAD_ARG;
    if ((((uintptr_t)A) | ((uintptr_t)B)) & 15) return SPHG_ERR_BAD_ARG;
    if (split_k < 1) split_k = 1;
    if (split_k > K / 64) split_k = K / 64;
    const __nv_bfloat16* a = (const __nv_bfloat16*)A;
    const __nv_bfloat16* b = (const __nv_bfloat16*)B;
    cudaStream_t s = (cudaStream_t)stream;
    if (N % 128 == 0) return launch_gemm<128>(a, b, C, M, N, K, accumulate, split_k, err_dev, s);
    if (N % 64 == 0) return launch_gemm<64>(a, b, C, M, N, K, accumulate, split_k, err_dev, s);
    if (N % 32 == 0) return launch_gemm<32>(a, b, C, M, N, K, accumulate, split_k, err_dev, s);
    return launch_gemm<16>(a, b, C, M, N, K, accumulate, split_k, err_dev, s);
}

extern "C" int sphg_gemm_wait_probe(const void* A, const void* B, int M, int N, int K, long long spins, int* err_dev,
                                    void* stream) {
    if (!A || !B || !err_dev || spins <= 0) return SPHG_ERR_BAD_ARG;
    if (M <= 0 || N <= 0 || K <= 0 || M % 128 || N % 128 || K % 64) return SPHG_ERR_BAD_ARG;
    if ((((uintptr_t)A) | ((uintptr_t)B)) & 15) return SPHG_ERR_BAD_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    int rc = launch_gemm<128>((const __nv_bfloat16*)A, (const __nv_bfloat16*)B, nullptr, M, N, K, 0, 1, err_dev, s,
                              spins);
    if (rc) return rc;
    int h = 0;
    if (cudaMemcpyAsync(&h, err_dev, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess) return SPHG_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return SPHG_ERR_CUDA;
    return h ? SPHG_ERR_TIMEOUT : SPHG_OK;
}
