/*
 * sphg_learn.h — the learned particle stepper of libsphg (no counterpart in
 * the reference, whose step is the SPH solver alone): tensor-core (tcgen05)
 * BF16 GEMM used by the message-passing network's forward and backward
 * passes.  Device pointers throughout; errors are sphg_status codes.
 */
#ifndef SPHG_LEARN_H
#define SPHG_LEARN_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* C[M x N] = A[M x K] * B[N x K]^T  (accumulate: C += ...).  A and B are
 * row-major bf16 with K contiguous, C row-major fp32; M % 128 == 0,
 * N % 16 == 0, K % 64 == 0, rows 16-byte aligned.  split_k > 1 splits K over
 * CTAs that add into C atomically (C must hold the value to add to).  A
 * device wait that gives up sets *err_dev to 1 (the call still returns). */
int sphg_gemm_bf16_tn(const void* A, const void* B, float* C, int M, int N, int K, int accumulate, int split_k,
                      int* err_dev, void* cuda_stream);

/* Epilogues of the weight-stationary GEMM (acc = the A B^T tile):
 *   STORE     z = acc                 ACC    z += acc
 *   BIAS_ACT  z = acc + bias (z kept when non-null), h = bf16(relu ? max(z, 0) : z)
 *   EDGE      z = acc + bias + P[src[r], :N] + P[dst[r], N:2N] for rows r < nedge
 *             (z kept when non-null), h = bf16(max(z, 0))
 *   RESID     z = z + acc + bias, h = bf16(z) when h is non-null */
enum { SPHG_EPI_STORE = 0, SPHG_EPI_ACC = 1, SPHG_EPI_BIAS_ACT = 2, SPHG_EPI_EDGE = 3, SPHG_EPI_RESID = 4 };

typedef struct SphgGemmEpi {
    int32_t mode, relu;
    const float* bias;   /* [N] */
    float* z;            /* [M x N] fp32 */
    void* h;             /* [M x N] bf16 */
    const float* P;      /* EDGE: [nodes x 2N] projections gathered per row */
    const int* src;
    const int* dst;
    long long nedge;
} SphgGemmEpi;

/* Weight-stationary persistent GEMM C[M x N] = A[M x K] * B[N x K]^T with
 * B resident in shared memory and a fused epilogue; (N, K) in {(128, 64),
 * (128, 128), (256, 128), (128, 256)} (SPHG_ERR_UNSUPPORTED otherwise),
 * M % 128 == 0, 16-byte aligned arrays.  A device wait that gives up sets
 * *err_dev to 1. */
int sphg_gemm_bf16_ws(const void* A, const void* B, int M, int N, int K, const SphgGemmEpi* epilogue, int* err_dev,
                      void* cuda_stream);

/* One message-passing edge layer in one kernel (inference; no counterpart in
 * the reference):
 *   a    = bf16(relu(E We^T + be + P[src[r], :128] + P[dst[r], 128:256]))   (gather for rows r < nedge)
 *   EF   = EF + a W2^T + b2         (fp32, in place)
 *   Eout = bf16(EF)
 * the same results, bit for bit, as sphg_gemm_bf16_ws with the EDGE epilogue
 * (h = a) followed by the RESID epilogue on a, without writing a.  With EF
 * NULL the residual stream is bf16 alone: Eout = bf16(E + a W2^T + b2), E
 * taken as its fp32 value (as the RESID epilogue with z = fp32(E)).  E and Eout
 * are [M x 128] bf16 and may be the same array (each 128-row tile of E is
 * read before the same tile of Eout is written), EF [M x 128] fp32,
 * P [nodes x 256] fp32,
 * We and W2 [128 x 128] bf16, be and b2 [128] fp32; M % 128 == 0, 0 <=
 * nedge <= M, 16-byte aligned arrays.  A device wait that gives up sets
 * *err_dev to 1. */
int sphg_gnn_edge_layer(const void* E, float* EF, void* E_out, const float* P, const int* src, const int* dst,
                        long long nedge, int M, const void* We, const float* be, const void* W2, const float* b2,
                        int* err_dev, void* cuda_stream);

/* The edge layer of the network in inference form with the sender term
 * inside the first GEMM (one kernel, K = 256):
 *   z    = [E | H[src]] . [We | Ws]^T + (Pd[dst] + be)
 *   Eout = bf16(E + (relu(z) . W2^T + b2))
 * where Ws is the sender half of the node projection (rows 0..127 of wsd) and
 * Pd = H Wd^T its receiver half per node (fp32, rows 128..255 of wsd, e.g.
 * from sphg_gemm_bf16_ws with the STORE epilogue).  This is the same layer as
 * sphg_gnn_edge_layer with EF NULL and P = [H Ws^T | Pd], except that the
 * sender term is summed in the accumulator with the edge term instead of
 * being rounded to an fp32 P row first (the results differ from it in the
 * last bits of the fp32 sums).  Rows of E and Eout beyond nedge use zero node
 * terms.  H [nnode x 128] bf16, Pd [nnode x 128] fp32, E and Eout [M x 128]
 * bf16 (may be the same array), src and dst per edge, We, Ws and W2
 * [128 x 128] bf16, be and b2 [128] fp32; M % 128 == 0, 0 <= nedge <= M,
 * E and Eout 32-byte aligned, the other arrays 16-byte aligned.  *err_dev:
 * bit 0 set when a device wait gave up, bit 1 when an index lies outside
 * [0, nnode) (that node term is taken as zero). */
int sphg_gnn_edge_layer_nodes(const void* E, void* E_out, const void* H, const float* Pd, int nnode, const int* src,
                              const int* dst, long long nedge, int M, const void* We, const void* Ws, const float* be,
                              const void* W2, const float* b2, int* err_dev, void* cuda_stream);

/* The edge encoder in one kernel (inference):
 *   E_out = bf16(bf16(relu(F W1^T + b1)) W2^T + b2)
 * with F the [M x 64] bf16 edge features, W1 [128 x 64] and W2 [128 x 128]
 * bf16, b1 and b2 [128] fp32; the hidden rows stay in TMEM.  The same bits
 * as sphg_gemm_bf16_ws with the BIAS_ACT epilogue twice (ReLU, then none),
 * without writing the hidden rows.  M % 128 == 0; E_out 32-byte aligned, the
 * other arrays 16-byte aligned.  A device wait that gives up sets *err_dev. */
int sphg_gnn_edge_encoder(const void* F, void* E_out, int M, const void* W1, const float* b1, const void* W2,
                          const float* b2, int* err_dev, void* cuda_stream);

/* A node MLP of the message-passing layer in one kernel (inference):
 *   Z     = Z + (bf16(relu(X V1^T + c1)) V2^T + c2)      (fp32, in place)
 *   H_out = bf16(Z)
 * with X the [M x 256] bf16 rows [h | agg], V1 [128 x 256] and V2 [128 x 128]
 * bf16, c1 and c2 [128] fp32; the hidden rows stay in TMEM.  The same bits as
 * sphg_gemm_bf16_ws with the BIAS_ACT epilogue (ReLU) followed by the RESID
 * epilogue on Z, without writing the hidden rows.  M % 128 == 0; H_out
 * 32-byte aligned, the other arrays 16-byte aligned.  A device wait that gives
 * up sets *err_dev. */
int sphg_gnn_node_mlp(const void* X, int M, const void* V1, const float* c1, const void* V2, const float* c2,
                      float* Z, void* H_out, int* err_dev, void* cuda_stream);

/* Test of the bounded device waits (no counterpart in the reference, whose
 * only failure path is `stop`): launches sphg_gemm_bf16_tn's kernel on
 * A (M x K) and B (N x K) so that its first K block issues no MMA and waits
 * for it with `spins` polls of the mbarrier.  The wait runs out while no MMA
 * or copy is in flight; the kernel sets *err_dev, frees its TMEM and returns
 * without writing any output.  The call waits for the stream and returns
 * SPHG_ERR_TIMEOUT when *err_dev was set.  M % 128 == 0, N % 128 == 0,
 * K % 64 == 0, spins > 0. */
int sphg_gemm_wait_probe(const void* A, const void* B, int M, int N, int K, long long spins, int* err_dev,
                         void* cuda_stream);

/* ---------------------------------------------------------------------
 * Message-passing network kernels.  Feature matrices are row-major bf16 or
 * fp32 with the row count padded to a multiple of 128; L is the latent
 * width, which must be 128 (the width the kernels are compiled for; other
 * values return SPHG_ERR_BAD_ARG); element counts n are multiples of 4.  Graphs are CSR by receiver: off[n + 1] (int64), src[e] and dst[e]
 * (int32), receivers in node order.
 * ------------------------------------------------------------------- */

#define SPHG_GNN_FEATURES 64 /* padded input width of node and edge rows */
#define SPHG_GNN_HISTORY 5   /* velocities kept per node */

enum { SPHG_GNN_WATER = 0, SPHG_GNN_SOIL = 1, SPHG_GNN_BOUNDARY = 2 };

/* per-node constants of the learned stepper (32 bytes) */
typedef struct {
    float xl, xr, yf;   /* left wall, right wall, floor of the node's scene */
    float dts;          /* stride length: k solver steps of the scene's dt  */
    float porosity;     /* scene porosity (0 without a soil-water mixture)  */
    float phi;          /* scene friction angle (rad), 0 for water scenes   */
    float mass;
    int32_t type;       /* SPHG_GNN_WATER / SOIL / BOUNDARY                 */
} sphg_gnn_node;

/* cell grid of the radius-graph search: cells of side `radius` from
 * (xmin, ymin), nx * ny of them; positions outside are clamped in */
typedef struct {
    double xmin, ymin, radius;
    int32_t nx, ny;
} sphg_gnn_grid;

/* scratch bytes of the scans for up to n items (cells or nodes) */
int sphg_gnn_scan_bytes(int n, size_t* bytes);
/* radius graph, pass 1: cell list (order[n]: nodes by cell, by index
 * within a cell; cell_count and cell_start hold nx * ny + 1), degrees
 * (deg[n + 1]) and off[n + 1] = exclusive scan of the degrees; off[n] is the
 * edge count, read by the caller to size src and dst */
int sphg_gnn_graph_count(const sphg_gnn_grid* grid, const double* x, int n, int* order, int* cell_count,
                         int* cell_start, int* deg, int64_t* off, void* scan_tmp, size_t scan_tmp_bytes,
                         void* cuda_stream);
/* radius graph, pass 2: every pair closer than the radius, both
 * directions, no self edges */
int sphg_gnn_graph_fill(const sphg_gnn_grid* grid, const double* x, int n, const int* order, const int* cell_start,
                        const int64_t* off, int* src, int* dst, void* cuda_stream);

/* node rows: 5 velocities (newest first, / vscale), type one-hot, wall
 * distances / 2h clipped to [0, 1], porosity, friction angle, stride (ms),
 * displacement (x - x0) / 2h clipped to [-16, 16] (zero when x0 is NULL) */
int sphg_gnn_node_features(const double* x, const double* x0, const float* vhist, int head,
                           const sphg_gnn_node* nodes, int n, int n_pad, float inv2h, float inv_vscale, void* out_bf16,
                           void* cuda_stream);
/* edge rows: (x_dst - x_src) / 2h, distance / 2h, same-type flag, change of
 * that offset since the reference positions x0 (clipped to [-4, 4]; zero
 * when x0 is NULL) */
int sphg_gnn_edge_features(const double* x, const double* x0, const sphg_gnn_node* nodes, const int* src,
                           const int* dst, long long nedge, long long nedge_pad, double inv2h, void* out_bf16,
                           void* cuda_stream);

int sphg_gnn_f32_to_bf16(const float* x, void* y_bf16, long long n, void* cuda_stream);
int sphg_gnn_relu_bwd(const float* dh, const float* z, float* dz, void* dz_bf16, long long n, void* cuda_stream);
/* out[c] += sum_r x[r, c] */
int sphg_gnn_colsum(const float* x, long long rows, int cols, float* out, void* cuda_stream);
/* out[c, r] = in[r, c] as bf16; in is fp32 (in_is_f32) or bf16 */
int sphg_gnn_transpose(const void* in, int in_is_f32, void* out_bf16, long long rows, int cols, void* cuda_stream);
/* agg[n] = scale * sum of e over the edges n receives */
int sphg_gnn_segsum(const float* e, const int64_t* off, float* agg, int nnode, int L, float scale, void* cuda_stream);
/* the same over bf16 edge rows */
int sphg_gnn_segsum_bf16(const void* e_bf16, const int64_t* off, float* agg, int nnode, int L, float scale,
                         void* cuda_stream);

/* The receiver sums written straight into the node MLP's input rows
 * (inference): out[n] = [h[n] | bf16(scale * sum of e over the edges n
 * receives)], out [npad x 2L] bf16, h [npad x L] bf16, e bf16 edge rows; the
 * same bits as sphg_gnn_segsum_bf16 followed by sphg_gnn_node_concat, without
 * the fp32 sums.  Rows from nnode to npad get zero sums; L must be 128. */
int sphg_gnn_segsum_cat(const void* e_bf16, const int64_t* off, const void* h_bf16, void* out_bf16, int nnode,
                        long long npad, int L, float scale, void* cuda_stream);
int sphg_gnn_segsum_bwd(const float* dagg, const int* dst, float* de, long long nedge, int L, float scale,
                        void* cuda_stream);
/* dP [nnode x 2L] (sender half zero on entry) from dz of the fused layer */
int sphg_gnn_gather_bwd(const float* dz, const int* src, const int64_t* off, float* dP, int nnode, long long nedge,
                        int L, void* cuda_stream);
/* [h | agg] as bf16 rows of 2L, and its backward (dh += ..., dagg = ...) */
int sphg_gnn_node_concat(const void* h_bf16, const float* agg, void* out_bf16, long long nnode, int L,
                         void* cuda_stream);
int sphg_gnn_node_concat_bwd(const float* d, float* dh, float* dagg, long long nnode, int L, void* cuda_stream);
/* squared error (Huber beyond |d| = delta when delta > 0) over masked rows
 * and the first nout columns, times inv_count; loss += ..., dpred = d/dpred */
int sphg_gnn_mse(const float* pred, int ld, const float* target, int nout, const float* mask, long long rows,
                 float inv_count, float delta, float* dpred, float* loss, void* cuda_stream);
/* Adam on w [rows x cols]; rows >= row_limit held at zero; refreshes the
 * bf16 copy w_bf16 and its transpose wt_bf16 [cols x rows] when non-null */
int sphg_gnn_adam(float* w, const float* g, float* m, float* v, void* w_bf16, void* wt_bf16, int rows, int cols,
                  float lr, float beta1, float beta2, float eps, int step, int row_limit, void* cuda_stream);

/* learned stride: a = pred[:, :2] * norm[2:4] + norm[0:2]; v' = v + a dts;
 * x += v' dts clamped to the walls (margin); v' -> slot head_new */
int sphg_gnn_stride_update(const float* pred, int ld, const float* norm, const sphg_gnn_node* nodes, double* x,
                           float* vhist, int head_old, int head_new, int n, double margin, void* cuda_stream);
/* sigma_i = 1 + sum over received edges of the cubic-spline shape W(r/h) */
int sphg_gnn_number_density(const double* x, const int64_t* off, const int* src, int n, double h, double* sigma,
                            void* cuda_stream);
/* out[4] = {sum (sigma_new/sigma_old - 1)^2, count, kinetic, potential
 * energy} over the non-boundary nodes */
int sphg_gnn_gate_sums(const double* sigma_new, const double* sigma_old, const double* x, const float* v_new,
                       const sphg_gnn_node* nodes, int n, double g, double* out, void* cuda_stream);

#ifdef __cplusplus
}
#endif
#endif /* SPHG_LEARN_H */
