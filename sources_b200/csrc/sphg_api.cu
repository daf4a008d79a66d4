// sphg_api.cu — context management, step orchestration and the C ABI of
// libsphg (include/sphg.h).
//
// The engine is templated on the pair arithmetic T (double for SPHG_FP64,
// float for SPHG_FP32).  One context owns one CUDA stream; every launch and
// copy goes to that stream (or to a stream the caller sets).
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/sphg.h"
#include "sphg_kernels.cuh"

namespace {

inline int blocks(long long n, int tpb) { return (int)((n + tpb - 1) / tpb); }

// Per-kernel CUDA-event timing on the launching stream.  Events come from a
// pool so that timing a long run adds no event creation to the step.
struct Profiler {
    bool on = false;
    long long launches = 0;   // kernels launched since the context was created
    struct Pending { const char* name; cudaEvent_t a, b; };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> pool;
    std::map<std::string, std::pair<long long, double>> acc;
    cudaEvent_t get() {
        if (pool.empty()) { cudaEvent_t e; cudaEventCreate(&e); return e; }
        cudaEvent_t e = pool.back(); pool.pop_back(); return e;
    }
    void resolve() {
        for (auto& p : pending) {
            float ms = 0.f;
            cudaEventSynchronize(p.b);
            cudaEventElapsedTime(&ms, p.a, p.b);
            auto& e = acc[p.name];
            e.first += 1;
            e.second += ms;
            pool.push_back(p.a);
            pool.push_back(p.b);
        }
        pending.clear();
    }
    ~Profiler() { for (auto e : pool) cudaEventDestroy(e); }
};

}  // namespace

struct EngineBase {
    virtual ~EngineBase() {}
    virtual int upload(int phase, const sphg_phase_host* v) = 0;
    virtual int download(int phase, sphg_phase_host* v) = 0;
    virtual int rhs(int itimestep) = 0;
    virtual int step(int itimestep) = 0;
    virtual int begin_batch() = 0;
    virtual int finish_batch() = 0;
    virtual int export_pairs(int which, int32_t* pi, int32_t* pj, int64_t cap, int64_t* n) = 0;
    virtual int stats(sphg_stats_t* out) = 0;
    virtual int set_scenes(int nscenes, const sphg_scene* sc) = 0;
    virtual int upload_scene_ids(int phase, const int32_t* ids) = 0;
    virtual int set_tuning(const sphg_tuning* t) = 0;
    virtual int xv_device(int phase, double* x, double* v, int to_caller) = 0;
    // Joint graphs of several contexts (sphg_group_*): the kind of graph a
    // regular step replays (-1: this step runs without a graph), the step's
    // launches on ctx->stream for capture, and the bookkeeping of a replay.
    virtual int graph_kind(int itimestep) = 0;
    virtual int prepare_graph_step() = 0;
    virtual int capture_step(int itimestep) = 0;
    virtual void after_graph_step(long long launches, int kind) = 0;
    virtual long long graph_epoch() const = 0;
};

struct sphg_ctx {
    sphg_params prm;
    int nphase = 1;
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    EngineBase* eng = nullptr;
    Profiler prof;
    int itimestep = 0;
    double time = 0.0;
    double last_step_ms = 0.0;
    cudaEvent_t ev_a = nullptr, ev_b = nullptr;   // timing of sphg_time_integration, made once
    // the soil pass runs beside water_pass_b on this stream, forked and joined by events
    cudaStream_t side_stream = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    // the soil's cell list and gather run on the side stream beside the water's
    cudaEvent_t ev_fork2 = nullptr, ev_join2 = nullptr;
};

#define CUDA_TRY(x)                                        \
    do {                                                   \
        cudaError_t e_ = (x);                              \
        if (e_ != cudaSuccess) {                           \
            fprintf(stderr, "libsphg: %s failed: %s\n", #x, cudaGetErrorString(e_)); \
            return SPHG_ERR_CUDA;                          \
        }                                                  \
    } while (0)

template <typename T>
struct Engine : EngineBase {
    typedef typename V2<T>::t T2;
    sphg_ctx* ctx;
    PhaseDev<T> P[2];
    bool have[2] = {false, false};
    bool prepared = false;
    bool aliased = false;        // a two-phase step overwrote the shared working arrays
    GridGeom grid{};
    SearchConst sc_same{}, sc_cross{};
    int ncell = 0;
    int* counts[2] = {nullptr, nullptr};
    int* cell_start_buf[2] = {nullptr, nullptr};
    void* cub_tmp = nullptr;
    void* cub_tmp1 = nullptr;        // the second phase's scan, which may run beside the first's
    size_t cub_bytes = 0;
    // The step's counters and the sticky flags side by side on the device.
    // Each step's check also writes them into mapped pinned host memory
    // (hblk), which the host reads after a batch with no copy; without it
    // (cudaHostAlloc failed) one copy into hblk_heap reads both.
    typedef CounterMirror CounterBlock;
    CounterBlock* cblk = nullptr;   // device
    CounterBlock* hblk = nullptr;   // mapped pinned host memory, or nullptr
    CounterBlock* hblk_dev = nullptr;   // its device address
    CounterBlock hblk_heap{};
    DevCounters* cnt = nullptr;     // device, &cblk->c
    DevCounters hcnt{};             // host copy
    int* sticky = nullptr;          // device, cblk->sticky: [overflow, nonfinite, staging timeout]
    double* stage = nullptr;        // transfer staging, 2*nmax doubles
    double* xstage = nullptr;       // staging of a group of fields (bulk transfers), xstage_cap doubles
    size_t xstage_cap = 0;
    int* stage_i = nullptr;
    long long* stage_l = nullptr;
    std::vector<void*> shadow[2];   // the second buffer of every persistent field
    int par[2] = {0, 0};            // per phase: flipped whenever fields and shadows swap
    int nmax = 0;
    double hrange[2][2] = {{0, 0}, {0, 0}};
    // per-scene parameters (entry 0 = the context's own parameters)
    std::vector<SceneTab> tab_host;
    SceneTab* tab_dev = nullptr;
    int tab_cap = 0;
    bool tab_custom = false;
    double cell_factor = 1.0;       // neighbour cell = factor * support radius (autotuned)
    int x_split = 0;                // x cells per neighbour cell (0: SPHG_X_SPLIT)
    int state_order = 0;            // order of the state after a reorder: 0 cell list, 1 Morton curve
    // Morton reorder scratch (state_order 1), one set per phase, since the two
    // phases' reorders run on two streams at once: keys and slots in and out,
    // the inverse order, the sort's space
    struct MortonScratch {
        unsigned* key[2] = {nullptr, nullptr};
        int* val[2] = {nullptr, nullptr};
        int* inv = nullptr;
        void* tmp = nullptr;
        size_t tmp_bytes = 0;
        int n = 0;
    } morton[2];
    std::vector<void*> allocs;
    SimConst sim{};
    int nfail_slot = 3;             // which DP site the reported nfail comes from

    explicit Engine(sphg_ctx* c) : ctx(c) { memset(P, 0, sizeof(P)); }
    ~Engine() override {
        drop_graphs();
        for (void* p : allocs) cudaFree(p);
        if (hblk) cudaFreeHost(hblk);
    }

    template <typename S>
    int alloc(S** p, size_t count) {
        void* q = nullptr;
        CUDA_TRY(cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(S)));
        CUDA_TRY(cudaMemsetAsync(q, 0, std::max<size_t>(count, 1) * sizeof(S), ctx->stream));
        allocs.push_back(q);
        *p = (S*)q;
        return 0;
    }
    void release(void* p) {
        if (!p) return;
        auto it = std::find(allocs.begin(), allocs.end(), p);
        if (it != allocs.end()) { cudaFree(p); allocs.erase(it); }
    }

    // ---------------------------------------------------------------- launch
    template <typename K, typename... A>
    int launch(const char* name, K kern, int grid_, int block, A... args) {
        return launch_ex(name, false, kern, grid_, block, 0, args...);
    }
    // gx blocks for each of gy fields (blockIdx.y)
    template <typename K, typename... A>
    int launch_fields(const char* name, K kern, int gx, int gy, int block, A... args) {
        if (gx <= 0 || gy <= 0) return 0;
        return launch_dim(name, false, kern, dim3((unsigned)gx, (unsigned)gy), block, 0, args...);
    }
    // with `smem` bytes of dynamic shared memory (the neighbour staging space)
    template <typename K, typename... A>
    int launch_smem(const char* name, K kern, int grid_, int block, size_t smem, A... args) {
        return launch_ex(name, false, kern, grid_, block, smem, args...);
    }
    // A kernel of the step chain (it begins with pdl_enter): launched with
    // programmatic stream serialization, so that it may launch while its
    // predecessor on the stream finishes.  Not while kernels are timed one by
    // one.
    template <typename K, typename... A>
    int launch_pdl(const char* name, K kern, int grid_, int block, size_t smem, A... args) {
        return launch_ex(name, true, kern, grid_, block, smem, args...);
    }
    bool use_pdl = SPHG_PDL != 0;
    template <typename K, typename... A>
    int launch_ex(const char* name, bool pdl, K kern, int grid_, int block, size_t smem, A... args) {
        if (grid_ <= 0) return 0;
        return launch_dim(name, pdl, kern, dim3((unsigned)grid_), block, smem, args...);
    }
    template <typename K, typename... A>
    int launch_dim(const char* name, bool pdl, K kern, dim3 grid_, int block, size_t smem, A... args) {
        cudaEvent_t a = nullptr, b = nullptr;
        if (ctx->prof.on) {
            a = ctx->prof.get(); b = ctx->prof.get();
            cudaEventRecord(a, ctx->stream);
        }
        if (pdl && use_pdl && !ctx->prof.on) {
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = grid_;
            cfg.blockDim = dim3((unsigned)block);
            cfg.dynamicSmemBytes = smem;
            cfg.stream = ctx->stream;
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
            at[0].val.programmaticStreamSerializationAllowed = 1;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            cudaLaunchKernelEx(&cfg, kern, args...);
        } else {
            kern<<<grid_, block, smem, ctx->stream>>>(args...);
        }
        ctx->prof.launches++;
        counters_fresh = false;
        cudaError_t e = cudaGetLastError();
        if (ctx->prof.on) {
            cudaEventRecord(b, ctx->stream);
            ctx->prof.pending.push_back({name, a, b});
        }
        if (e != cudaSuccess) {
            fprintf(stderr, "libsphg: launch %s failed: %s\n", name, cudaGetErrorString(e));
            return SPHG_ERR_CUDA;
        }
        return 0;
    }

    // ------------------------------------------------------------ constants
    void make_sim(int itimestep) {
        const sphg_params& p = ctx->prm;
        SimConst& s = sim;
        s.skf = p.skf; s.single_phase = p.single_phase; s.summation_density = p.summation_density;
        s.average_velocity = p.average_velocity; s.visc_artificial = p.visc_artificial;
        s.artificial_density = p.artificial_density; s.soil_artificial_stress = p.soil_artificial_stress;
        s.volume_fraction = p.volume_fraction; s.water_artificial_volume = p.water_artificial_volume;
        s.volume_fraction_renorm = p.volume_fraction_renorm; s.stress_integration = p.stress_integration;
        s.plasticity = p.plasticity; s.yield_dp = p.yield_criterion == 2;
        s.renorm_now = p.volume_fraction_renorm && p.renorm_interval > 0 && (itimestep % p.renorm_interval) == 0;
        s.gravity = p.gravity; s.numeric_gravity = p.numeric_gravity;
        s.alpha = p.alpha; s.beta = p.beta; s.etq = p.etq; s.dd = p.dd; s.p1 = p.p1; s.p2 = p.p2;
        s.delta = p.delta; s.epsilon = p.epsilon; s.dt = p.dt;
        s.w_rho0 = p.water.rho0; s.w_b = p.water.b; s.w_gamma = p.water.gamma; s.w_c = p.water.c; s.w_mu = p.water.viscosity;
        s.s_rho0 = p.soil.rho0; s.s_k = p.soil.k; s.s_E = p.soil.E; s.s_niu = p.soil.niu; s.s_c = p.soil.c;
        s.s_perm = p.soil.permeability; s.s_G = p.soil.G;
        s.s_kb = p.soil.permeability * p.forchheimer_b;
        s.s_alpha1 = alpha1_of(p.soil.phi);
        s.tab = tab_dev;
    }

    static double alpha1_of(double phi) {   // m_particles.f90:3338
        double t = tan(phi);
        return t / sqrt(9.0 + 12.0 * (t * t));
    }

    // Copy the scene table to the device; entry 0 follows the context's
    // parameters unless the host set its own table.
    int sync_table() {
        const sphg_params& p = ctx->prm;
        if (!tab_custom) {
            tab_host.assign(1, SceneTab{p.dt, p.water.b, p.water.c, alpha1_of(p.soil.phi)});
        }
        if ((int)tab_host.size() > tab_cap) {
            release(tab_dev);
            tab_dev = nullptr;
            tab_cap = (int)tab_host.size();
            if (alloc(&tab_dev, (size_t)tab_cap)) return SPHG_ERR_CUDA;
        }
        CUDA_TRY(cudaMemcpyAsync(tab_dev, tab_host.data(), sizeof(SceneTab) * tab_host.size(), cudaMemcpyHostToDevice,
                                 ctx->stream));
        CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        return 0;
    }

    int set_scenes(int nscenes, const sphg_scene* sc) override {
        if (nscenes < 1 || !sc) return SPHG_ERR_BAD_ARG;
        std::vector<SceneTab> t((size_t)nscenes);
        for (int i = 0; i < nscenes; ++i) {
            if (!(sc[i].dt > 0.0)) return SPHG_ERR_BAD_ARG;
            t[(size_t)i] = SceneTab{sc[i].dt, sc[i].water_b, sc[i].water_c, alpha1_of(sc[i].soil_phi)};
        }
        tab_host.swap(t);
        tab_custom = true;
        return sync_table();
    }

    int upload_scene_ids(int phase, const int32_t* ids) override {
        if (phase < 1 || phase > ctx->nphase || !ids) return SPHG_ERR_BAD_ARG;
        const int ph = phase - 1;
        if (!have[ph]) return SPHG_ERR_STATE;
        PhaseDev<T>& D = P[ph];
        for (int i = 0; i < D.n; ++i)
            if (ids[i] < 0 || ids[i] >= (int)std::max<size_t>(tab_host.size(), 1)) return SPHG_ERR_BAD_ARG;
        CUDA_TRY(cudaMemcpyAsync(stage_i, ids, sizeof(int) * (size_t)D.n, cudaMemcpyHostToDevice, ctx->stream));
        int rc = launch("upload", k_from_original_i, blocks(D.n, 256), 256, D.n, (const int*)D.orig,
                        (const int*)stage_i, D.sid);
        if (rc) return rc;
        CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        return 0;
    }

    int set_tuning(const sphg_tuning* t) override {
        cells_ready = false;
        if (!t || !(t->cell_factor >= 1.0) || t->cell_factor > 4.0 || t->reorder_interval < 0) return SPHG_ERR_BAD_ARG;
        if (t->x_split < 0 || t->x_split > 8) return SPHG_ERR_BAD_ARG;
        if (t->state_order < 0 || t->state_order > 1) return SPHG_ERR_BAD_ARG;
        cell_factor = t->cell_factor;
        x_split = t->x_split;
        state_order = t->state_order;
        ctx->prm.reorder_interval = t->reorder_interval;
        prepared = false;
        drop_graphs();
        return 0;
    }

    static int scale_k(int skf) {
        switch (skf) { case 1: return 2; case 2: return 3; case 3: return 3; case 4: return 2; }
        return -1;
    }

    // smallest double t with sqrt(t) >= K: then sqrt(r2) < K  <=>  r2 < t
    static double exact_threshold(double K) {
        double t = K * K;
        while (t > 0 && std::sqrt(t) >= K) t = std::nextafter(t, 0.0);
        while (std::sqrt(t) < K) t = std::nextafter(t, INFINITY);
        return t;
    }

    // ------------------------------------------------------------ allocation
    int alloc_phase(int ph, int n) {
        PhaseDev<T>& D = P[ph];
        if (have[ph] && D.n == n) return 0;   // same size: reuse every buffer
        // a re-upload replaces the arrays
        void* old[] = {D.x, D.v, D.v_min, D.rho, D.rho_min, D.vof, D.vof_min, D.p, D.c, D.mass, D.hsml, D.sxx, D.sxy,
                       D.syy, D.sxx_min, D.sxy_min, D.syy_min, D.p_min, D.eps_p, D.itype, D.orig, D.fail, D.sid, D.drho,
                       D.dvof, D.dsxx, D.dsxy, D.dsyy, D.dp, D.txx, D.txy, D.tyy, D.vcc, D.wxy, D.vof2, D.dv, D.av,
                       D.countiac, D.cell_id, D.cell_fill, D.perm, D.xs, D.hs, D.recA, D.recA2, D.recB, D.hmask};
        for (void* p : old) release(p);
        for (void* p : shadow[ph]) release(p);
        shadow[ph].clear();
        par[ph] = 0;
        memset(&D, 0, sizeof(D));
        D.n = n;
        size_t N = (size_t)n;
        int rc = 0;
        rc |= alloc(&D.x, N); rc |= alloc(&D.v, N); rc |= alloc(&D.v_min, N);
        rc |= alloc(&D.rho, N); rc |= alloc(&D.rho_min, N); rc |= alloc(&D.vof, N); rc |= alloc(&D.vof_min, N);
        rc |= alloc(&D.p, N); rc |= alloc(&D.c, N); rc |= alloc(&D.mass, N); rc |= alloc(&D.hsml, N);
        rc |= alloc(&D.sxx, N); rc |= alloc(&D.sxy, N); rc |= alloc(&D.syy, N);
        rc |= alloc(&D.sxx_min, N); rc |= alloc(&D.sxy_min, N); rc |= alloc(&D.syy_min, N); rc |= alloc(&D.p_min, N);
        rc |= alloc(&D.eps_p, N);
        rc |= alloc(&D.itype, N); rc |= alloc(&D.orig, N); rc |= alloc(&D.fail, N); rc |= alloc(&D.sid, N);
        rc |= alloc(&D.drho, N); rc |= alloc(&D.dvof, N); rc |= alloc(&D.dsxx, N); rc |= alloc(&D.dsxy, N);
        rc |= alloc(&D.dsyy, N); rc |= alloc(&D.dp, N); rc |= alloc(&D.txx, N); rc |= alloc(&D.txy, N);
        rc |= alloc(&D.tyy, N); rc |= alloc(&D.vcc, N); rc |= alloc(&D.wxy, N); rc |= alloc(&D.vof2, N);
        rc |= alloc(&D.dv, N); rc |= alloc(&D.av, N);
        rc |= alloc(&D.countiac, N); rc |= alloc(&D.cell_id, N); rc |= alloc(&D.cell_fill, N); rc |= alloc(&D.perm, N);
        rc |= alloc(&D.xs, N); rc |= alloc(&D.hs, N);
        rc |= alloc(&D.recA, N); rc |= alloc(&D.recA2, N); rc |= alloc(&D.recB, N); rc |= alloc(&D.hmask, N);
        if (rc) return SPHG_ERR_CUDA;
        for (auto& f : field_refs(ph)) {
            char* q = nullptr;
            if (alloc(&q, (size_t)f.second * N)) return SPHG_ERR_CUDA;
            shadow[ph].push_back(q);
        }
        if (n > nmax) {
            release(stage); release(stage_i); release(stage_l);
            nmax = n;
            if (alloc(&stage, 2 * (size_t)n) || alloc(&stage_i, (size_t)n) || alloc(&stage_l, (size_t)n + 1))
                return SPHG_ERR_CUDA;
        }
        if (!cnt) {
            if (alloc(&cblk, 1)) return SPHG_ERR_CUDA;
            cnt = &cblk->c;
            sticky = cblk->sticky;
            void* hp = nullptr;
            void* dp = nullptr;
            if (cudaHostAlloc(&hp, sizeof(CounterBlock), cudaHostAllocMapped) == cudaSuccess) {
                if (cudaHostGetDevicePointer(&dp, hp, 0) == cudaSuccess) {
                    hblk = (CounterBlock*)hp;
                    hblk_dev = (CounterBlock*)dp;
                    memset(hblk, 0, sizeof(CounterBlock));
                } else {
                    cudaGetLastError();
                    cudaFreeHost(hp);
                }
            } else {
                cudaGetLastError();
            }
        }
        return 0;
    }

    // A host array in original order and its device field in state order
    // (wide: FP64 on the device, else the precision's type T).
    struct HostField { const double* h; void* d; int comps; int wide; };
    // A device field and the host arrays it is copied to (h1: a second copy,
    // for the water's shared stress/strain-rate working arrays).
    struct DevField { const void* d; int comps; int wide; double* h0; double* h1; };
    // A staged water field whose first entries the soil's values replace
    // (k_alias_soil) before it is copied out.
    struct SoilAlias { const void* d; const T* src; int zero_tail; };

    // On an error after copies were queued, let them finish before returning:
    // the caller may release its host arrays once the call has returned.
    int upload(int phase, const sphg_phase_host* h) override {
        const int rc = upload_work(phase, h);
        if (rc && ctx) cudaStreamSynchronize(ctx->stream);
        return rc;
    }
    int download(int phase, sphg_phase_host* h) override {
        const int rc = download_work(phase, h);
        if (rc && ctx) cudaStreamSynchronize(ctx->stream);
        return rc;
    }

    int upload_work(int phase, const sphg_phase_host* h) {
        cells_ready = false;
        if (phase < 1 || phase > ctx->nphase || !h) return SPHG_ERR_BAD_ARG;
        if (!h->x || !h->vx || !h->rho || !h->p || !h->c || !h->mass || !h->hsml || !h->itype) return SPHG_ERR_BAD_ARG;
        int n = h->ntotal + h->nvirt;
        if (n <= 0 || h->ntotal < 0 || h->nvirt < 0) return SPHG_ERR_BAD_ARG;
        int ph = phase - 1;
        // Same particles again (size, material; the h range is checked below):
        // start the copies into the staging area now, so that the scan of h
        // below runs while they are in flight.
        const bool same = have[ph] && prepared && P[ph].n == n && P[ph].ntotal == h->ntotal &&
                          P[ph].material == h->material;
        int rc = alloc_phase(ph, n);   // keeps every buffer when the size is the same
        if (rc) return rc;
        PhaseDev<T>& D = P[ph];
        std::vector<HostField> f;
        XferList L;
        bool staged = false;
        if (same) {
            f = host_fields(h, D);
            if ((rc = stage_fields(n, f, L, staged))) return rc;
        }
        D.ntotal = h->ntotal; D.material = h->material; D.dspp = h->dspp;
        // every h positive and finite; their range (four independent lanes, no
        // branch per element: this scan is part of every upload)
        double lo4[4] = {INFINITY, INFINITY, INFINITY, INFINITY}, hi4[4] = {0.0, 0.0, 0.0, 0.0};
        int ok = 1;
        int i = 0;
        for (; i + 4 <= n; i += 4) {
            for (int j = 0; j < 4; ++j) {
                const double v = h->hsml[i + j];
                ok &= (v > 0.0) & (v < INFINITY);
                lo4[j] = v < lo4[j] ? v : lo4[j];
                hi4[j] = v > hi4[j] ? v : hi4[j];
            }
        }
        for (; i < n; ++i) {
            const double v = h->hsml[i];
            ok &= (v > 0.0) & (v < INFINITY);
            lo4[0] = v < lo4[0] ? v : lo4[0];
            hi4[0] = v > hi4[0] ? v : hi4[0];
        }
        const double lo = std::min(std::min(lo4[0], lo4[1]), std::min(lo4[2], lo4[3]));
        const double hi = std::max(std::max(hi4[0], hi4[1]), std::max(hi4[2], hi4[3]));
        // same particles and h range: refill the arrays in the current state
        // order and keep the grid, the cell order and the captured graphs
        if (ok && same && hrange[ph][0] == lo && hrange[ph][1] == hi)
            return refill(ph, h, staged ? &f : nullptr, staged ? &L : nullptr);
        // otherwise the staged copies go unused: let them finish before the
        // caller's arrays can be released
        if (staged) CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        if (!ok) return SPHG_ERR_BAD_ARG;
        hrange[ph][0] = lo; hrange[ph][1] = hi;
        // original order == state order until the first reorder
        if ((rc = launch("iota", k_iota, blocks(n, 256), 256, n, D.orig))) return rc;
        rc |= put_state(n, h->x, (double*)D.x, 2); rc |= put_state(n, h->vx, (double*)D.v, 2);
        rc |= put_state(n, h->v_min, (double*)D.v_min, 2);
        rc |= put_state(n, h->rho, D.rho, 1); rc |= put_state(n, h->rho_min, D.rho_min, 1);
        rc |= put_state(n, h->vof, D.vof, 1); rc |= put_state(n, h->vof_min, D.vof_min, 1);
        rc |= put_state(n, h->p, D.p, 1); rc |= put_state(n, h->c, D.c, 1); rc |= put_state(n, h->mass, D.mass, 1);
        rc |= put_state(n, h->hsml, D.hsml, 1);
        rc |= put_state(n, h->sxx, D.sxx, 1); rc |= put_state(n, h->sxy, D.sxy, 1); rc |= put_state(n, h->syy, D.syy, 1);
        rc |= put_state(n, h->sxx_min, D.sxx_min, 1); rc |= put_state(n, h->sxy_min, D.sxy_min, 1);
        rc |= put_state(n, h->syy_min, D.syy_min, 1); rc |= put_state(n, h->p_min, D.p_min, 1);
        rc |= put_state(n, h->epsilon_p, D.eps_p, 1);
        rc |= put_rate(n, h->drho, D.drho, 1); rc |= put_rate(n, h->dvof, D.dvof, 1);
        rc |= put_rate(n, h->dsxx, D.dsxx, 1); rc |= put_rate(n, h->dsxy, D.dsxy, 1); rc |= put_rate(n, h->dsyy, D.dsyy, 1);
        rc |= put_rate(n, h->dp, D.dp, 1); rc |= put_rate(n, h->dvx, (T*)D.dv, 2); rc |= put_rate(n, h->av, (T*)D.av, 2);
        rc |= put_rate(n, h->vof2, D.vof2, 1); rc |= put_rate(n, h->vcc, D.vcc, 1);
        rc |= put_rate(n, h->txx, D.txx, 1); rc |= put_rate(n, h->tyy, D.tyy, 1); rc |= put_rate(n, h->txy, D.txy, 1);
        if (rc) return SPHG_ERR_CUDA;
        CUDA_TRY(cudaMemcpyAsync(D.itype, h->itype, sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, ctx->stream));
        CUDA_TRY(cudaMemsetAsync(D.sid, 0, sizeof(int) * (size_t)n, ctx->stream));
        have[ph] = true;
        prepared = false;
        aliased = false;
        drop_graphs();
        CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        return 0;
    }

    // host (original order) -> state order through the current permutation
    int refill(int ph, const sphg_phase_host* h, const std::vector<HostField>* staged = nullptr,
               const XferList* L = nullptr) {
        PhaseDev<T>& D = P[ph];
        const int n = D.n;
        D.dspp = h->dspp;
        int rc = staged ? finish_fields(n, D.orig, *staged, *L) : put_fields(n, D.orig, host_fields(h, D));
        if (rc) return rc;
        CUDA_TRY(cudaMemcpyAsync(stage_i, h->itype, sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, ctx->stream));
        if (launch("refill", k_from_original_i, blocks(n, 256), 256, n, D.orig, (const int*)stage_i, D.itype))
            return SPHG_ERR_CUDA;
        aliased = false;
        CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        return 0;
    }

    // ------------------------------------------------------- bulk transfers
    // Staging for every transferred field of an n-particle phase (37 doubles
    // a particle), up to 2^26 doubles (512 MB) and at least one
    // two-component field.  Sized for all fields, whatever one call moves, so
    // that an upload after a download (or the reverse) never reallocates: a
    // cudaFree would synchronise the device.
    static constexpr size_t kXferDoubles = 37;
    int xstage_reserve(int n) {
        const size_t want = std::max<size_t>(2 * (size_t)n, std::min<size_t>(kXferDoubles * n, (size_t)1 << 26));
        if (xstage_cap >= want) return 0;
        release(xstage);
        xstage = nullptr;
        xstage_cap = 0;
        if (alloc(&xstage, want)) return SPHG_ERR_CUDA;
        xstage_cap = want;
        return 0;
    }

    // Every host array of a phase and its device field.
    std::vector<HostField> host_fields(const sphg_phase_host* h, PhaseDev<T>& D) {
        return {{h->x, D.x, 2, 1}, {h->vx, D.v, 2, 1}, {h->v_min, D.v_min, 2, 1},
                {h->rho, D.rho, 1, 1}, {h->rho_min, D.rho_min, 1, 1}, {h->vof, D.vof, 1, 1}, {h->vof_min, D.vof_min, 1, 1},
                {h->p, D.p, 1, 1}, {h->c, D.c, 1, 1}, {h->mass, D.mass, 1, 1}, {h->hsml, D.hsml, 1, 1},
                {h->sxx, D.sxx, 1, 1}, {h->sxy, D.sxy, 1, 1}, {h->syy, D.syy, 1, 1},
                {h->sxx_min, D.sxx_min, 1, 1}, {h->sxy_min, D.sxy_min, 1, 1}, {h->syy_min, D.syy_min, 1, 1},
                {h->p_min, D.p_min, 1, 1}, {h->epsilon_p, D.eps_p, 1, 1},
                {h->drho, D.drho, 1, 0}, {h->dvof, D.dvof, 1, 0}, {h->dsxx, D.dsxx, 1, 0}, {h->dsxy, D.dsxy, 1, 0},
                {h->dsyy, D.dsyy, 1, 0}, {h->dp, D.dp, 1, 0}, {h->dvx, D.dv, 2, 0}, {h->av, D.av, 2, 0},
                {h->vof2, D.vof2, 1, 0}, {h->vcc, D.vcc, 1, 0}, {h->txx, D.txx, 1, 0}, {h->tyy, D.tyy, 1, 0},
                {h->txy, D.txy, 1, 0}};
    }

    // The copies of every non-null host array into the staging area, when
    // they fit one group (staged; L the group).  The state is not touched, so
    // the caller may still decline the transfer (after a synchronisation).
    int stage_fields(int n, const std::vector<HostField>& f, XferList& L, bool& staged) {
        staged = false;
        int rc = xstage_reserve(n);
        if (rc) return rc;
        size_t need = 0;
        int nf = 0;
        for (const HostField& e : f)
            if (e.h) { need += (size_t)n * e.comps; ++nf; }
        if (need > xstage_cap || nf > (int)(sizeof(L.f) / sizeof(L.f[0]))) return 0;
        memset(&L, 0, sizeof(L));
        size_t off = 0;
        for (const HostField& e : f) {
            if (!e.h) continue;
            const size_t cnt_d = (size_t)n * e.comps;
            CUDA_TRY(cudaMemcpyAsync(xstage + off, e.h, cnt_d * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
            L.f[L.count++] = XferField{e.d, (long long)off, e.comps, e.wide};
            off += cnt_d;
        }
        staged = true;
        return 0;
    }
    // The rest of a staged transfer: zero the fields without a host array,
    // then permute and narrow the group into the state.
    int finish_fields(int n, const int* orig, const std::vector<HostField>& f, const XferList& L) {
        for (const HostField& e : f)
            if (!e.h)
                CUDA_TRY(cudaMemsetAsync(e.d, 0, (size_t)n * e.comps * (e.wide ? sizeof(double) : sizeof(T)), ctx->stream));
        return launch_fields("refill", k_from_original_all<T>, blocks(n, 256), L.count, 256, n, orig, L, (const double*)xstage);
    }

    // Host -> state order for a list of fields: the copies of a group of
    // fields go back to back into the staging area, then one launch permutes
    // and narrows the whole group.  A null host array zeroes its field.
    int put_fields(int n, const int* orig, const std::vector<HostField>& f) {
        XferList L;
        bool staged = false;
        int rc = stage_fields(n, f, L, staged);
        if (rc) return rc;
        if (staged) return finish_fields(n, orig, f, L);
        memset(&L, 0, sizeof(L));
        size_t off = 0;
        auto flush = [&]() -> int {
            if (L.count == 0) return 0;
            const int r = launch_fields("refill", k_from_original_all<T>, blocks(n, 256), L.count, 256, n, orig, L,
                                        (const double*)xstage);
            L.count = 0;
            off = 0;
            return r;
        };
        const int cap = (int)(sizeof(L.f) / sizeof(L.f[0]));
        for (const HostField& e : f) {
            const size_t cnt_d = (size_t)n * e.comps;
            if (!e.h) {
                CUDA_TRY(cudaMemsetAsync(e.d, 0, cnt_d * (e.wide ? sizeof(double) : sizeof(T)), ctx->stream));
                continue;
            }
            if (L.count == cap || off + cnt_d > xstage_cap)
                if ((rc = flush())) return rc;
            CUDA_TRY(cudaMemcpyAsync(xstage + off, e.h, cnt_d * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
            L.f[L.count++] = XferField{e.d, (long long)off, e.comps, e.wide};
            off += cnt_d;
        }
        return flush();
    }

    // State order -> host for a list of fields: one launch permutes and
    // widens a group of fields into the staging area, then their copies to
    // the host go back to back.
    int get_fields(int n, const int* orig, const std::vector<DevField>& f, const std::vector<SoilAlias>& alias = {}) {
        int rc = xstage_reserve(n);
        if (rc) return rc;
        XferList L;
        memset(&L, 0, sizeof(L));
        const DevField* grp[sizeof(L.f) / sizeof(L.f[0])];
        size_t off = 0;
        auto flush = [&]() -> int {
            if (L.count == 0) return 0;
            int r = launch_fields("download", k_to_original_all<T>, blocks(n, 256), L.count, 256, n, orig, L, xstage);
            if (r) return r;
            for (const SoilAlias& al : alias) {
                for (int i = 0; i < L.count; ++i) {
                    if (L.f[i].dev != al.d) continue;
                    const int ns = P[1].n;
                    if ((r = launch("download", k_alias_soil<T>, blocks(std::max(ns, n), 256), 256, ns, n,
                                    (const int*)P[1].orig, al.src, xstage + L.f[i].off, al.zero_tail)))
                        return r;
                }
            }
            for (int i = 0; i < L.count; ++i) {
                const size_t bytes = (size_t)n * grp[i]->comps * sizeof(double);
                double* const hd[2] = {grp[i]->h0, grp[i]->h1};
                for (int k = 0; k < 2; ++k) {
                    if (!hd[k]) continue;
                    CUDA_TRY(cudaMemcpyAsync(hd[k], xstage + L.f[i].off, bytes, cudaMemcpyDeviceToHost, ctx->stream));
                }
            }
            L.count = 0;
            off = 0;
            return 0;
        };
        const int cap = (int)(sizeof(L.f) / sizeof(L.f[0]));
        for (const DevField& e : f) {
            if (!e.h0 && !e.h1) continue;
            const size_t cnt_d = (size_t)n * e.comps;
            if (L.count == cap || off + cnt_d > xstage_cap)
                if ((rc = flush())) return rc;
            grp[L.count] = &e;
            L.f[L.count++] = XferField{const_cast<void*>(e.d), (long long)off, e.comps, e.wide};
            off += cnt_d;
        }
        return flush();
    }

    int put_state(int n, const double* src, double* dst, int comps) {
        if (!src) { CUDA_TRY(cudaMemsetAsync(dst, 0, sizeof(double) * (size_t)n * comps, ctx->stream)); return 0; }
        CUDA_TRY(cudaMemcpyAsync(dst, src, sizeof(double) * (size_t)n * comps, cudaMemcpyHostToDevice, ctx->stream));
        return 0;
    }
    int put_rate(int n, const double* src, T* dst, int comps) {
        if (!src) { CUDA_TRY(cudaMemsetAsync(dst, 0, sizeof(T) * (size_t)n * comps, ctx->stream)); return 0; }
        if (sizeof(T) == sizeof(double)) {
            CUDA_TRY(cudaMemcpyAsync(dst, src, sizeof(double) * (size_t)n * comps, cudaMemcpyHostToDevice, ctx->stream));
            return 0;
        }
        CUDA_TRY(cudaMemcpyAsync(stage, src, sizeof(double) * (size_t)n * comps, cudaMemcpyHostToDevice, ctx->stream));
        // identity order: the phase was just uploaded, orig == iota
        return launch("upload_convert", k_from_original<T>, blocks(n, 256), 256, n, (const int*)P_orig_identity(n),
                      (const double*)stage, dst, comps);
    }
    const int* P_orig_identity(int n) {
        // stage_i holds an identity map, rebuilt on demand
        launch("iota", k_iota, blocks(n, 256), 256, n, stage_i);
        return stage_i;
    }

    // -------------------------------------------------------------- prepare
    // Grid and search constants, once every phase is on the device.
    int prepare() {
        if (prepared) return 0;
        int rc0;
        for (int ph = 0; ph < ctx->nphase; ++ph) if (!have[ph]) return SPHG_ERR_STATE;
        const sphg_params& p = ctx->prm;
        int sk = scale_k(p.skf);
        if (sk < 0) return SPHG_ERR_BAD_KERNEL;
        // h range over all phases (from the uploaded host arrays)
        double hmin = INFINITY, hmax = 0.0;
        for (int ph = 0; ph < ctx->nphase; ++ph) {
            hmin = std::min(hmin, hrange[ph][0]);
            hmax = std::max(hmax, hrange[ph][1]);
        }
        if ((rc0 = sync_table())) return rc0;
        double cell = sk * hmax * cell_factor * (1.0 + 1e-6);
        if (!(p.x_max > p.x_min) || !(p.y_max > p.y_min)) return SPHG_ERR_BAD_ARG;
        // rows one cell high; kx cells per cell along x (each at least
        // support/kx wide, so the 2*kx+1 cells around a particle's own cover
        // its support, clamped edge cells included)
        const int kx = x_split > 0 ? x_split : SPHG_X_SPLIT;
        const double cellx = cell / kx;
        double ncx = std::ceil((p.x_max - p.x_min) / cellx) + 1, ncy = std::ceil((p.y_max - p.y_min) / cell) + 1;
        if (ncx * ncy > 2.0e8) return SPHG_ERR_BAD_ARG;
        grid.ncx = (int)ncx; grid.ncy = (int)ncy; grid.kx = kx; grid.x0 = p.x_min; grid.y0 = p.y_min;
        grid.inv = 1.0 / cell; grid.invx = 1.0 / cellx;
        int nc = grid.ncx * grid.ncy;
        if (nc != ncell) {
            for (int ph = 0; ph < 2; ++ph) {
                release(counts[ph]); counts[ph] = nullptr;
                release(cell_start_buf[ph]); cell_start_buf[ph] = nullptr;
            }
            release(cub_tmp); cub_tmp = nullptr;
            release(cub_tmp1); cub_tmp1 = nullptr;
            ncell = nc;
        }
        for (int ph = 0; ph < ctx->nphase; ++ph) {
            if (!counts[ph] && alloc(&counts[ph], (size_t)nc + 1)) return SPHG_ERR_CUDA;
            if (!cell_start_buf[ph] && alloc(&cell_start_buf[ph], (size_t)nc + 1)) return SPHG_ERR_CUDA;
            P[ph].cell_start = cell_start_buf[ph];
        }
        if (!cub_tmp) {
            size_t bytes = 0;
            cub::DeviceScan::ExclusiveSum(nullptr, bytes, counts[0], P[0].cell_start, nc + 1, ctx->stream);
            size_t b2 = 0;
            cub::DeviceScan::ExclusiveSum(nullptr, b2, (long long*)nullptr, (long long*)nullptr, nmax + 1, ctx->stream);
            cub_bytes = std::max(bytes, b2);
            if (alloc((char**)&cub_tmp, cub_bytes)) return SPHG_ERR_CUDA;
        }
        if (ctx->nphase == 2 && !cub_tmp1 && alloc((char**)&cub_tmp1, cub_bytes)) return SPHG_ERR_CUDA;
        for (int ph = 0; state_order == 1 && ph < ctx->nphase; ++ph) {   // outside any stream capture
            MortonScratch& M = morton[ph];
            const int n = P[ph].n;
            if (M.n >= n) continue;
            for (int i = 0; i < 2; ++i) { release(M.key[i]); release(M.val[i]); M.key[i] = nullptr; M.val[i] = nullptr; }
            release(M.inv); release(M.tmp);
            M.inv = nullptr; M.tmp = nullptr;
            size_t b = 0;
            cub::DeviceRadixSort::SortPairs(nullptr, b, (unsigned*)nullptr, (unsigned*)nullptr, (int*)nullptr,
                                            (int*)nullptr, n, 0, 32, ctx->stream);
            M.tmp_bytes = b;
            for (int i = 0; i < 2; ++i)
                if (alloc(&M.key[i], (size_t)n) || alloc(&M.val[i], (size_t)n)) return SPHG_ERR_CUDA;
            if (alloc(&M.inv, (size_t)n) || alloc((char**)&M.tmp, M.tmp_bytes)) return SPHG_ERR_CUDA;
            M.n = n;
        }
        bool uniform = hmin == hmax;
        double K = sk * hmax;
        sc_same.scale_k = sk; sc_same.uniform = uniform; sc_same.r2_uniform = uniform ? exact_threshold(K) : 0.0;
        sc_cross = sc_same;
        switch (p.skf) {
            case 1: rc0 = stage_attrs<1>(); break;
            case 2: rc0 = stage_attrs<2>(); break;
            case 3: rc0 = stage_attrs<3>(); break;
            default: rc0 = stage_attrs<4>(); break;
        }
        if (rc0) return rc0;
        prepared = true;
        // spatial order from the start
        cells_ready = false;
        for (int ph = 0; ph < ctx->nphase; ++ph) {
            int rc = build_cells(ph);
            if (rc) return rc;
            if ((rc = reorder(ph))) return rc;
        }
        return 0;
    }

    // The cell keys, ranks and per-cell counts of the current positions: made
    // by the previous step's corrector (cells_ready), else counted here.
    bool cells_ready = false;
    int count_cells(int ph, int next) {
        PhaseDev<T>& D = P[ph];
        CUDA_TRY(cudaMemsetAsync(counts[ph], 0, sizeof(int) * ((size_t)ncell + 1), ctx->stream));
        return launch_pdl("cell_count", k_cell_count, blocks(D.n, 256), 256, 0, (const double2*)D.x, D.n, grid,
                          D.cell_id, D.cell_fill, counts[ph], cnt, next);
    }
    // Count the current positions' cells as a corrector would have, so that a
    // captured step (which expects them) can run.
    int prime_cells() {
        if (cells_ready) return 0;
        for (int ph = 0; ph < ctx->nphase; ++ph) {
            int rc = count_cells(ph, 1);
            if (rc) return rc;
        }
        cells_ready = true;
        return 0;
    }
    int build_cells(int ph) {
        PhaseDev<T>& D = P[ph];
        int rc = 0;
        if (!cells_ready && (rc = count_cells(ph, 0))) return rc;
        size_t bytes = cub_bytes;
        CUDA_TRY(cub::DeviceScan::ExclusiveSum(ph == 1 && cub_tmp1 ? cub_tmp1 : cub_tmp, bytes, counts[ph], D.cell_start,
                                               ncell + 1, ctx->stream));
        if ((rc = launch_pdl("cell_scatter", k_cell_scatter, blocks(D.n, 256), 256, 0, D.n, (const int*)D.cell_id,
                             (const int*)D.cell_fill, (const int*)D.cell_start, D.perm)))
            return rc;
        return launch_pdl("cell_sort", k_cell_sort, blocks(ncell, 256), 256, 0, ncell, (const int*)D.cell_start,
                          (const int*)D.orig, D.perm, counts[ph]);
    }

    // The persistent per-particle fields of a phase and their element sizes.
    std::vector<std::pair<void**, int>> field_refs(int ph) {
        PhaseDev<T>& D = P[ph];
        std::vector<std::pair<void**, int>> f;
        auto add = [&](void** p, int b) { f.push_back({p, b}); };
        add((void**)&D.x, 16); add((void**)&D.v, 16); add((void**)&D.v_min, 16);
        for (double** q : {&D.rho, &D.rho_min, &D.vof, &D.vof_min, &D.p, &D.c, &D.mass, &D.hsml, &D.sxx, &D.sxy,
                           &D.syy, &D.sxx_min, &D.sxy_min, &D.syy_min, &D.p_min, &D.eps_p})
            add((void**)q, 8);
        for (int** q : {&D.itype, &D.orig, &D.fail, &D.countiac, &D.sid}) add((void**)q, 4);
        for (T** q : {&D.drho, &D.dvof, &D.dsxx, &D.dsxy, &D.dsyy, &D.dp, &D.txx, &D.txy, &D.tyy, &D.vcc, &D.wxy, &D.vof2})
            add((void**)q, (int)sizeof(T));
        add((void**)&D.dv, (int)sizeof(T2)); add((void**)&D.av, (int)sizeof(T2));
        return f;
    }

    // Swap every persistent field of a phase with its shadow buffer.
    void swap_buffers(int ph) {
        auto refs = field_refs(ph);
        for (size_t i = 0; i < refs.size() && i < shadow[ph].size(); ++i) std::swap(*refs[i].first, shadow[ph][i]);
        par[ph] ^= 1;
    }

    // Permute every persistent field into the current cell order in one launch
    // (each into its shadow buffer), then swap fields and shadows: the later
    // launches of the step read the new buffers.  Every field thus lives in
    // one of two fixed buffers, and a captured step graph is kept per
    // combination of the phases' buffer sets (graph_index).
    int reorder(int ph) {
        PhaseDev<T>& D = P[ph];
        auto refs = field_refs(ph);
        PermList L;
        memset(&L, 0, sizeof(L));
        if (refs.size() > sizeof(L.f) / sizeof(L.f[0]) || refs.size() != shadow[ph].size()) return SPHG_ERR_STATE;
        L.count = (int)refs.size();
        for (size_t i = 0; i < refs.size(); ++i) {
            L.f[i].src = *refs[i].first;
            L.f[i].dst = shadow[ph][i];
            L.f[i].bytes = refs[i].second;
        }
        if (state_order == 1) return reorder_morton(ph, L);
        int rc = launch_pdl("reorder", k_permute_all, blocks(D.n, 256), 256, 0, D.n, (const int*)D.perm, L);
        if (rc) return rc;
        swap_buffers(ph);
        return launch_pdl("iota", k_iota, blocks(D.n, 256), 256, 0, D.n, D.perm);
    }
    // The same into the Morton order of the support-radius cells: the cell
    // list's slots sorted (stably) by their cells' Morton keys give the new
    // state order; the cell list is then renumbered to the new state indices.
    int reorder_morton(int ph, const PermList& L) {
        PhaseDev<T>& D = P[ph];
        MortonScratch& M = morton[ph];
        const int n = D.n;
        if (M.n < n || !M.tmp) return SPHG_ERR_STATE;
        int rc = launch_pdl("reorder", k_morton_keys, blocks(n, 256), 256, 0, n, (const int*)D.perm,
                            (const int*)D.cell_id, grid, M.key[0], M.val[0]);
        if (rc) return rc;
        size_t b = M.tmp_bytes;
        CUDA_TRY(cub::DeviceRadixSort::SortPairs(M.tmp, b, M.key[0], M.key[1], M.val[0], M.val[1], n, 0, 32,
                                                 ctx->stream));
        if ((rc = launch_pdl("reorder", k_permute_all, blocks(n, 256), 256, 0, n, (const int*)M.val[1], L))) return rc;
        swap_buffers(ph);
        if ((rc = launch_pdl("reorder", k_invert, blocks(n, 256), 256, 0, n, (const int*)M.val[1], M.inv))) return rc;
        return launch_pdl("reorder", k_renumber, blocks(n, 256), 256, 0, n, (const int*)M.inv, D.perm);
    }

    // Launches above 48 KB of dynamic shared memory must be allowed per kernel
    // (outside any stream capture: prepare() runs before every capture).
    template <int SKF>
    int stage_attrs() {
        const int a = (int)((size_t)SPHG_STAGE_A * (16 + sizeof(RecA<T>)));
        if (a > 48 * 1024)
            CUDA_TRY(cudaFuncSetAttribute(k_water_pass_a<T, SKF, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, a));
        return 0;
    }

    // -------------------------------------------------------------- the step
    int reset_counters() { return launch_pdl("reset", k_reset_counters, 1, 32, 0, cnt, cells_ready ? 1 : 0); }

    // The pair passes of one step for kernel function SKF.  fh: run the
    // leapfrog predictor inside the gathers; u: what the last pass of each
    // phase does after its sums (nothing, or the corrector).
    template <int SKF>
    int passes(int fh, StepCtl u) {
        const sphg_params& p = ctx->prm;
        u.ncount = nullptr;   // set per phase: the corrector counts that phase's next cells
        const int tpb = SPHG_TPB;
        const int dp = sim.yield_dp;
        int rc;
        if (p.single_phase) {
            PhaseDev<T>& D = P[0];
            if (D.material == SPHG_WATER) {
                if ((rc = launch_pdl("gather", k_gather<T>, blocks(D.n, 256), 256, 0, D, sim, 0, 0, fh, 0, 0, cnt))) return rc;
                if ((rc = launch_pdl("water_sum", k_water_sum<T, SKF>, blocks(D.n, tpb), tpb, 0, D, grid, sc_same, sim, cnt))) return rc;
                if ((rc = launch_pdl("water_pass_a", k_water_pass_a<T, SKF, true>, blocks(D.n, tpb), tpb, 0, D, grid, sc_same, sim, cnt))) return rc;
                StepCtl uw = u;
                uw.ncount = u.update ? counts[0] : nullptr;
                if ((rc = launch_pdl("water_pass_b", k_water_pass_b<T, SKF, true, false>, blocks(D.n, tpb), tpb, 0, D, D, grid, sc_same,
                                 sc_same, sim, uw, cnt))) return rc;
            } else {
                if ((rc = launch_pdl("gather", k_gather<T>, blocks(D.n, 256), 256, 0, D, sim, 1, dp, fh, 0, dp, cnt))) return rc;
                StepCtl us = u; us.with_vof = 0; us.do_dp = dp;
                us.ncount = u.update ? counts[0] : nullptr;
                if ((rc = launch_pdl("soil_pass", k_soil_pass<T, SKF, true, false>, blocks(D.n, tpb), tpb, 0, D, D, grid, sc_same, sc_same,
                                 sim, cnt, 0, us))) return rc;
            }
        } else {
            PhaseDev<T>& W = P[0];
            PhaseDev<T>& S = P[1];
            StepCtl uw = u; uw.with_vof = 1; uw.do_dp = 0;
            StepCtl us = u; us.with_vof = 1; us.do_dp = dp;
            uw.ncount = u.update ? counts[0] : nullptr;
            us.ncount = u.update ? counts[1] : nullptr;
            // the soil's gather was launched by run() on the side stream
            if ((rc = launch_pdl("gather", k_gather<T>, blocks(W.n, 256), 256, 0, W, sim, 0, 0, fh, 1, 0, cnt))) return rc;
            if ((rc = launch_pdl("water_pass_a", k_water_pass_a<T, SKF, false>, blocks(W.n, tpb), tpb,
                                  (size_t)SPHG_STAGE_A * (16 + sizeof(RecA<T>)), W, grid, sc_same, sim, cnt)))
                return rc;
            // The cross pairs run inside the last pass of each phase; the soil
            // pass reads the water pressure that water_pass_a sets.  After
            // water_pass_a the two last passes share no data: each reads the
            // other phase's sorted records only, and writes its own phase's
            // state (the counters by atomics).  So the soil pass runs on a
            // side stream beside water_pass_b and fills the SMs its last
            // partial wave leaves idle.  While kernels are timed one by one
            // (sphg_kernel_profile) it runs on the main stream, so that each
            // pass's time is its own.
            const bool fch = p.forchheimer_b != 0.0;
            cudaStream_t main_stream = ctx->stream;
            cudaStream_t side = ctx->prof.on ? main_stream : ctx->side_stream;
            if (side != main_stream) {
                CUDA_TRY(cudaEventRecord(ctx->ev_fork, main_stream));
                CUDA_TRY(cudaStreamWaitEvent(side, ctx->ev_fork, 0));
            }
            ctx->stream = side;
            rc = fch ? launch_pdl("soil_pass", k_soil_pass<T, SKF, false, true>, blocks(S.n, tpb), tpb, 0, S, W, grid, sc_same,
                              sc_cross, sim, cnt, 1, us)
                     : launch_pdl("soil_pass", k_soil_pass<T, SKF, false, false>, blocks(S.n, tpb), tpb, 0, S, W, grid, sc_same,
                              sc_cross, sim, cnt, 1, us);
            cudaError_t ej = side != main_stream ? cudaEventRecord(ctx->ev_join, side) : cudaSuccess;
            ctx->stream = main_stream;
            // water_pass_b reads the soil's records: wait for the soil's gather
            if (side != main_stream) {
                cudaError_t e2 = cudaStreamWaitEvent(main_stream, ctx->ev_join2, 0);
                if (e2 != cudaSuccess && rc == 0) rc = SPHG_ERR_CUDA;
            }
            if (rc == 0)
                rc = fch ? launch_pdl("water_pass_b", k_water_pass_b<T, SKF, false, true>, blocks(W.n, tpb), tpb, 0, W, S, grid,
                                  sc_same, sc_cross, sim, uw, cnt)
                         : launch_pdl("water_pass_b", k_water_pass_b<T, SKF, false, false>, blocks(W.n, tpb), tpb, 0, W, S, grid,
                                  sc_same, sc_cross, sim, uw, cnt);
            // join in every case, so that a capture in progress ends joined
            cudaError_t ew = ej != cudaSuccess ? ej
                             : side != main_stream ? cudaStreamWaitEvent(main_stream, ctx->ev_join, 0) : cudaSuccess;
            if (rc) return rc;
            if (ew != cudaSuccess) {
                fprintf(stderr, "libsphg: joining the soil pass failed: %s\n", cudaGetErrorString(ew));
                return SPHG_ERR_CUDA;
            }
            aliased = true;
        }
        return 0;
    }

    // One captured CUDA graph per kind of regular step (itimestep >= 2) and
    // buffer set: bit 0 = reorder step, bit 1 = renormalisation step, bits 2
    // and 3 = each phase's buffer set (par).  Buffers are allocated once per
    // phase, so a graph stays valid until the next upload of another size.
    static constexpr int NGRAPH = 16;
    cudaGraphExec_t graphs[NGRAPH] = {};
    bool use_graphs = true;

    long long epoch = 0;    // counts drop_graphs(): joint graphs of older epochs are stale
    void drop_graphs() {
        for (auto& g : graphs) if (g) { cudaGraphExecDestroy(g); g = nullptr; }
        ++epoch;
    }

    int graph_index(int itimestep) const { return step_kind(itimestep) | par[0] << 2 | par[1] << 3; }
    int graph_kind(int itimestep) override {
        if (itimestep < 2 || !use_graphs || ctx->prof.on) return -1;
        return graph_index(itimestep);
    }
    int prepare_graph_step() override {
        int rc = prepare();
        return rc ? rc : prime_cells();
    }
    // Record the step into the stream being captured.  The host's buffer
    // sets are left as before the step: they change when the graph is
    // launched (after_graph_step).
    int capture_step(int itimestep) override {
        StepCtl u{};
        u.update = 1;
        const int p0 = par[0], p1 = par[1];
        int rc = run(itimestep, 1, u);
        if (par[0] != p0) swap_buffers(0);
        if (par[1] != p1) swap_buffers(1);
        return rc;
    }
    // After a launch of the graph of `kind` (a graph_index): a reorder step
    // has swapped every phase's buffers.
    void launched_step(int kind) {
        if (kind & 1)
            for (int ph = 0; ph < ctx->nphase; ++ph) swap_buffers(ph);
    }
    void after_graph_step(long long launches, int kind) override {
        nfail_slot = 3;
        if (!ctx->prm.single_phase) aliased = true;
        ctx->prof.launches += launches;
        launched_step(kind);
    }
    long long graph_epoch() const override { return epoch; }

    int step_kind(int itimestep) const {
        const sphg_params& p = ctx->prm;
        return ((p.reorder_interval > 0 && itimestep % p.reorder_interval == 0) ? 1 : 0) |
               ((p.volume_fraction_renorm && p.renorm_interval > 0 && itimestep % p.renorm_interval == 0) ? 2 : 0);
    }

    // Launch the captured graph of this kind of step, capturing it first if
    // needed.  If capture is not possible, graphs are switched off and the
    // caller launches the step directly.
    int step_graphed(int itimestep) {
        int rc = prepare();
        if (rc) return rc;
        if ((rc = prime_cells())) return rc;   // a captured step expects the cells counted
        const int kind = graph_index(itimestep);
        if (!graphs[kind]) {
            cudaGraph_t g = nullptr;
            const long long before = ctx->prof.launches;
            if (cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
                cudaGetLastError();
                use_graphs = false;
                return 0;
            }
            rc = capture_step(itimestep);
            cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
            if (rc || e != cudaSuccess || !g) {
                if (g) cudaGraphDestroy(g);
                cudaGetLastError();
                use_graphs = false;
                return rc;
            }
            cudaError_t ei = cudaGraphInstantiate(&graphs[kind], g, 0);
            cudaGraphDestroy(g);
            if (ei != cudaSuccess) { graphs[kind] = nullptr; cudaGetLastError(); use_graphs = false; return 0; }
            launches_per_graph[kind] = ctx->prof.launches - before;
            ctx->prof.launches = before;
        }
        nfail_slot = 3;
        if (!ctx->prm.single_phase) aliased = true;
        CUDA_TRY(cudaGraphLaunch(graphs[kind], ctx->stream));
        ctx->prof.launches += launches_per_graph[kind];
        launched_step(kind);
        return 0;
    }
    long long launches_per_graph[NGRAPH] = {};

    int run(int itimestep, int fh, StepCtl u) {
        const int rc = run_step(itimestep, fh, u);
        if (rc) cells_ready = false;
        return rc;
    }
    int run_step(int itimestep, int fh, StepCtl u) {
        int rc = prepare();
        if (rc) return rc;
        make_sim(itimestep);
        if ((rc = reset_counters())) return rc;
        const sphg_params& p = ctx->prm;
        bool reorder_now = p.reorder_interval > 0 && itimestep > 0 && itimestep % p.reorder_interval == 0;
        if (ctx->nphase == 2 && !p.single_phase) {
            // The soil's cell list, reorder and gather touch soil data only,
            // so they run on the side stream beside the water's (serially
            // while kernels are timed one by one); water_pass_b waits for
            // them (passes).
            cudaStream_t main_stream = ctx->stream;
            cudaStream_t side = ctx->prof.on ? main_stream : ctx->side_stream;
            if (side != main_stream) {
                CUDA_TRY(cudaEventRecord(ctx->ev_fork2, main_stream));
                CUDA_TRY(cudaStreamWaitEvent(side, ctx->ev_fork2, 0));
            }
            ctx->stream = side;
            rc = build_cells(1);
            if (!rc && reorder_now) rc = reorder(1);
            if (!rc) rc = launch_pdl("gather", k_gather<T>, blocks(P[1].n, 256), 256, 0, P[1], sim, 1, sim.yield_dp, fh, 1,
                                 sim.yield_dp, cnt);
            cudaError_t ej = side != main_stream ? cudaEventRecord(ctx->ev_join2, side) : cudaSuccess;
            ctx->stream = main_stream;
            if (rc || ej != cudaSuccess) {
                if (side != main_stream && ej == cudaSuccess) cudaStreamWaitEvent(main_stream, ctx->ev_join2, 0);
                return rc ? rc : SPHG_ERR_CUDA;
            }
            if ((rc = build_cells(0))) return rc;
            if (reorder_now && (rc = reorder(0))) return rc;
        } else {
            for (int ph = 0; ph < ctx->nphase; ++ph) {
                if ((rc = build_cells(ph))) return rc;
                if (reorder_now && (rc = reorder(ph))) return rc;
            }
        }
        switch (p.skf) {
            case 1: rc = passes<1>(fh, u); break;
            case 2: rc = passes<2>(fh, u); break;
            case 3: rc = passes<3>(fh, u); break;
            default: rc = passes<4>(fh, u); break;
        }
        // a step with the corrector has counted the next step's cells
        cells_ready = rc == 0 && u.update != 0;
        if (rc) return rc;
        return launch_pdl("check", k_check, 1, 32, 0, (const DevCounters*)cnt, sticky, (unsigned long long)p.max_interaction,
                          hblk_dev);
    }

    // single_step / single_step_for_water / single_step_for_soil
    int rhs(int itimestep) override {
        StepCtl none{};
        nfail_slot = ctx->prm.plasticity == 3 ? 2 : 1;
        return run(itimestep, 0, none);
    }

    // one leapfrog step of time_integration / _for_water / _for_soil: the
    // predictor runs inside the gathers (not on the first step), the
    // corrector inside the last pass of each phase
    int step(int itimestep) override {
        // regular steps replay a captured graph (not while per-kernel timing is on)
        if (itimestep >= 2 && use_graphs && !ctx->prof.on) {
            int rc = step_graphed(itimestep);
            if (rc || use_graphs) return rc;
        }
        StepCtl u{};
        u.update = 1;
        u.first = itimestep == 1;
        nfail_slot = 3;
        return run(itimestep, itimestep != 1, u);
    }

    int begin_batch() override {
        counters_fresh = false;
        if (!sticky) return 0;
        // the last batch ended in a synchronisation, so no kernel writes the
        // mirror now: the host clears its flags itself
        if (hblk) {
            memset(hblk->sticky, 0, sizeof(hblk->sticky));
            return 0;
        }
        CUDA_TRY(cudaMemsetAsync(sticky, 0, 4 * sizeof(int), ctx->stream));
        return 0;
    }

    // read counters and the sticky flags after a batch
    int finish_batch() override {
        if (!cblk) return 0;   // nothing uploaded yet: no counters
        CounterBlock* hb = hblk ? hblk : &hblk_heap;
        if (!hblk) CUDA_TRY(cudaMemcpyAsync(hb, cblk, sizeof(CounterBlock), cudaMemcpyDeviceToHost, ctx->stream));
        CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        hcnt = hb->c;
        const int* hs = hb->sticky;
        batch_rc = hs[2] ? SPHG_ERR_TIMEOUT : hs[1] ? SPHG_ERR_NONFINITE : hs[0] ? SPHG_ERR_PAIR_OVERFLOW : 0;
        counters_fresh = true;
        return batch_rc;
    }
    // the host copy of the counters matches the device (no launch since the
    // last finish_batch), so sphg_stats needs no second copy and sync
    bool counters_fresh = false;
    int batch_rc = 0;

    // ------------------------------------------------------------- download

    // positions and velocities between the state and caller device arrays in
    // original order, on the context's stream (no host copy, no sync)
    int xv_device(int phase, double* x, double* v, int to_caller) override {
        if (phase < 1 || phase > ctx->nphase) return SPHG_ERR_BAD_ARG;
        int ph = phase - 1;
        if (!have[ph]) return SPHG_ERR_STATE;
        PhaseDev<T>& D = P[ph];
        const int n = D.n;
        double* state[2] = {(double*)D.x, (double*)D.v};
        double* user[2] = {x, v};
        int rc = 0;
        if (!to_caller && x) cells_ready = false;   // new positions
        for (int f = 0; f < 2; ++f) {
            if (!user[f]) continue;
            if (to_caller)
                rc |= launch("xv_device", k_to_original<double>, blocks(n, 256), 256, n, (const int*)D.orig,
                             (const double*)state[f], user[f], 2);
            else
                rc |= launch("xv_device", k_from_original<double>, blocks(n, 256), 256, n, (const int*)D.orig,
                             (const double*)user[f], state[f], 2);
        }
        return rc ? SPHG_ERR_CUDA : SPHG_OK;
    }

    int download_work(int phase, sphg_phase_host* h) {
        if (phase < 1 || phase > ctx->nphase || !h) return SPHG_ERR_BAD_ARG;
        int ph = phase - 1;
        if (!have[ph]) return SPHG_ERR_STATE;
        PhaseDev<T>& D = P[ph];
        int n = D.n, rc = 0;
        const int* o = D.orig;
        h->ntotal = D.ntotal; h->nvirt = n - D.ntotal; h->material = D.material; h->dspp = D.dspp;
        std::vector<DevField> f = {
            {D.x, 2, 1, h->x, nullptr}, {D.v, 2, 1, h->vx, nullptr}, {D.v_min, 2, 1, h->v_min, nullptr},
            {D.dv, 2, 0, h->dvx, nullptr}, {D.av, 2, 0, h->av, nullptr},
            {D.rho, 1, 1, h->rho, nullptr}, {D.rho_min, 1, 1, h->rho_min, nullptr}, {D.drho, 1, 0, h->drho, nullptr},
            {D.p, 1, 1, h->p, nullptr}, {D.c, 1, 1, h->c, nullptr}, {D.mass, 1, 1, h->mass, nullptr},
            {D.hsml, 1, 1, h->hsml, nullptr}, {D.vof, 1, 1, h->vof, nullptr}, {D.vof_min, 1, 1, h->vof_min, nullptr},
            {D.dvof, 1, 0, h->dvof, nullptr}, {D.vof2, 1, 0, h->vof2, nullptr},
            {D.dsxx, 1, 0, h->dsxx, nullptr}, {D.dsxy, 1, 0, h->dsxy, nullptr}, {D.dsyy, 1, 0, h->dsyy, nullptr},
            {D.dp, 1, 0, h->dp, nullptr},
            {D.sxx_min, 1, 1, h->sxx_min, nullptr}, {D.sxy_min, 1, 1, h->sxy_min, nullptr},
            {D.syy_min, 1, 1, h->syy_min, nullptr}, {D.p_min, 1, 1, h->p_min, nullptr},
            {D.eps_p, 1, 1, h->epsilon_p, nullptr}, {D.vcc, 1, 0, h->vcc, nullptr}};
        if (D.material == SPHG_SOIL) {
            f.push_back({D.sxx, 1, 1, h->sxx, nullptr}); f.push_back({D.sxy, 1, 1, h->sxy, nullptr});
            f.push_back({D.syy, 1, 1, h->syy, nullptr});
            f.push_back({D.txx, 1, 0, h->txx, nullptr}); f.push_back({D.tyy, 1, 0, h->tyy, nullptr});
            f.push_back({D.txy, 1, 0, h->txy, nullptr});
        } else {
            // water stress lives in the shared working arrays (sxx => txx, ...)
            f.push_back({D.sxx, 1, 1, h->sxx, h->txx}); f.push_back({D.syy, 1, 1, h->syy, h->tyy});
            f.push_back({D.sxy, 1, 1, h->sxy, h->txy});
        }
        // after a two-phase step the soil pass has overwritten the water's
        // shared working arrays in part (k_alias_soil)
        std::vector<SoilAlias> alias;
        if (D.material == SPHG_WATER && ctx->nphase == 2 && aliased)
            alias = {{D.sxx, P[1].txx, 0}, {D.syy, P[1].tyy, 0}, {D.sxy, P[1].txy, 1}};
        rc = get_fields(n, o, f, alias);
        if (h->itype) {
            rc |= launch("download", k_to_original_i, blocks(n, 256), 256, n, o, (const int*)D.itype, stage_i);
            CUDA_TRY(cudaMemcpyAsync(h->itype, stage_i, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
        }
        if (h->fail) {
            rc |= launch("download", k_to_original_i, blocks(n, 256), 256, n, o, (const int*)D.fail, stage_i);
            CUDA_TRY(cudaMemcpyAsync(h->fail, stage_i, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
        }
        CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        if (rc) return SPHG_ERR_CUDA;
        h->nfail = hcnt.nfail[nfail_slot];
        return 0;
    }

    // ----------------------------------------------------------- pair export
    int export_pairs(int which, int32_t* pi, int32_t* pj, int64_t cap, int64_t* nout) override {
        if (which < 0 || which > 2 || !nout) return SPHG_ERR_BAD_ARG;
        if (which == 1 && ctx->nphase < 2) return SPHG_ERR_BAD_ARG;
        if (which == 2 && ctx->nphase < 2) return SPHG_ERR_BAD_ARG;
        int rc = prepare();
        if (rc) return rc;
        int a = which == 1 ? 1 : 0;
        int b = which == 2 ? 1 : a;
        PhaseDev<T>& A = P[a];
        PhaseDev<T>& B = P[b];
        // the lists of the current positions (the last step's pair search if no
        // step ran since): rebuild sorted positions for both phases
        for (int ph = 0; ph < ctx->nphase; ++ph) {
            if ((rc = build_cells(ph))) { cells_ready = false; return rc; }
            if ((rc = launch("gather", k_gather<T>, blocks(P[ph].n, 256), 256, P[ph], sim, 0, 0, 0, 0, 0, cnt))) {
                cells_ready = false;
                return rc;
            }
        }
        cells_ready = false;   // the counts were consumed
        int n = A.n;
        int* count = stage_i;
        long long* off = stage_l;
        if ((rc = launch("pairs_count", k_pairs_count, blocks(n, SPHG_TPB), SPHG_TPB, n, (const int*)A.perm, (const int*)A.orig,
                         (const double2*)A.xs, (const double*)A.hs, grid, which == 2 ? sc_cross : sc_same,
                         (const int*)B.cell_start, (const double2*)B.xs, (const double*)B.hs, (const int*)B.perm,
                         (const int*)B.orig, which == 2 ? 1 : 0, count, 0, (const long long*)nullptr, (int*)nullptr,
                         (int*)nullptr, 0LL)))
            return rc;
        // exclusive scan of counts (as long long) in original-index order
        std::vector<int> hc((size_t)n);
        CUDA_TRY(cudaMemcpyAsync(hc.data(), count, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
        CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        std::vector<long long> ho((size_t)n + 1, 0);
        for (int i = 0; i < n; ++i) ho[(size_t)i + 1] = ho[(size_t)i] + hc[(size_t)i];
        long long total = ho[(size_t)n];
        *nout = total;
        long long ncopy = std::min<long long>(total, cap);
        if (ncopy <= 0 || !pi || !pj) return 0;
        CUDA_TRY(cudaMemcpyAsync(off, ho.data(), sizeof(long long) * ((size_t)n + 1), cudaMemcpyHostToDevice, ctx->stream));
        int *di = nullptr, *dj = nullptr;
        CUDA_TRY(cudaMalloc(&di, sizeof(int) * (size_t)ncopy));
        CUDA_TRY(cudaMalloc(&dj, sizeof(int) * (size_t)ncopy));
        rc = launch("pairs_write", k_pairs_count, blocks(n, SPHG_TPB), SPHG_TPB, n, (const int*)A.perm, (const int*)A.orig,
                    (const double2*)A.xs, (const double*)A.hs, grid, which == 2 ? sc_cross : sc_same,
                    (const int*)B.cell_start, (const double2*)B.xs, (const double*)B.hs, (const int*)B.perm,
                    (const int*)B.orig, which == 2 ? 1 : 0, count, 1, (const long long*)off, di, dj, ncopy);
        cudaError_t e1 = cudaMemcpyAsync(pi, di, sizeof(int) * (size_t)ncopy, cudaMemcpyDeviceToHost, ctx->stream);
        cudaError_t e2 = cudaMemcpyAsync(pj, dj, sizeof(int) * (size_t)ncopy, cudaMemcpyDeviceToHost, ctx->stream);
        cudaError_t e3 = cudaStreamSynchronize(ctx->stream);
        cudaFree(di);
        cudaFree(dj);
        if (rc) return rc;
        if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) return SPHG_ERR_CUDA;
        return 0;
    }

    int stats(sphg_stats_t* out) override {
        int rc = counters_fresh ? batch_rc : finish_batch();
        memset(out, 0, sizeof(*out));
        out->niac[0] = (int64_t)(hcnt.pairs[0] / 2);
        out->niac[1] = (int64_t)(hcnt.pairs[1] / 2);
        out->niac[2] = (int64_t)hcnt.pairs[2];
        for (int i = 0; i < 2; ++i) {
            out->maxiac[i] = hcnt.maxiac[i];
            out->miniac[i] = hcnt.miniac[i] == 0x7fffffff ? 0 : hcnt.miniac[i];
            out->noiac[i] = hcnt.noiac[i];
        }
        out->nfail = hcnt.nfail[nfail_slot];
        out->n_out_of_domain = hcnt.n_out;
        out->itimestep = ctx->itimestep;
        out->time = ctx->time;
        out->last_step_ms = ctx->last_step_ms;
        return rc == SPHG_ERR_CUDA ? rc : 0;
    }
};

// ============================================================== C ABI
extern "C" {

void sphg_default_params(sphg_params* p) {
    if (!p) return;
    memset(p, 0, sizeof(*p));
    p->abi_version = SPHG_ABI_VERSION;
    p->dim = 2;
    p->skf = 4;                      // m_particles.f90:141
    p->first_material = SPHG_WATER;
    p->average_velocity = 1;         // param.f90:80
    p->visc_artificial = 1;          // :86
    p->artificial_density = 1;       // :95
    p->soil_artificial_stress = 1;   // :96
    p->volume_fraction = 1;          // :98
    p->water_artificial_volume = 1;  // :99
    p->volume_fraction_renorm = 1;   // :100
    p->stress_integration = 1;       // :92
    p->yield_criterion = 2;          // :93
    p->plasticity = 3;               // :94
    p->integrate_scheme = 1;         // :78
    p->precision = SPHG_FP64;
    p->reorder_interval = 10;
    p->renorm_interval = 40;         // declarations_sph.f90:1415
    p->gravity = (double)-9.8f;      // declarations_sph.f90:13 (default-real literal)
    p->numeric_gravity = (double)-9.8f;  // m_particles.f90:40
    p->alpha = 0.1; p->beta = 0.0; p->etq = 0.1;  // :44
    p->dd = 0.1; p->p1 = 12; p->p2 = 4;          // :47
    p->delta = 0.1;                              // :50
    p->epsilon = (double)0.001f;                 // :53
    p->x_min = -10.0; p->x_max = 10.0; p->y_min = -10.0; p->y_max = 10.0;  // param.f90:23-25
    p->max_interaction = 10 * 2000;              // param.f90:14
}

static int validate(const sphg_params* p, int n_phase) {
    if (!p || (n_phase != 1 && n_phase != 2)) return SPHG_ERR_BAD_ARG;
    if (p->abi_version != SPHG_ABI_VERSION || p->dim != 2) return SPHG_ERR_BAD_ARG;
    if (p->skf < 1 || p->skf > 4) return SPHG_ERR_BAD_KERNEL;
    if ((p->single_phase != 0) != (n_phase == 1)) return SPHG_ERR_BAD_ARG;
    if (p->single_phase && p->first_material != SPHG_WATER && p->first_material != SPHG_SOIL) return SPHG_ERR_BAD_ARG;
    if (p->precision != SPHG_FP64 && p->precision != SPHG_FP32) return SPHG_ERR_BAD_ARG;
    if (!(p->forchheimer_b >= 0.0) || !std::isfinite(p->forchheimer_b)) return SPHG_ERR_BAD_ARG;
    // outside the implemented scope: Verlet (param.f90:78 = 2), Mohr-Coulomb
    // (yield_criterion = 1), flow rules 1 and 2, summation density for soil
    if (p->integrate_scheme != 1) return SPHG_ERR_UNSUPPORTED;
    if (p->yield_criterion != 2 && p->yield_criterion != 0) return SPHG_ERR_UNSUPPORTED;
    if (p->plasticity != 3 && p->plasticity != 0) return SPHG_ERR_UNSUPPORTED;
    if (p->stress_integration != 1 && p->stress_integration != 2) return SPHG_ERR_UNSUPPORTED;
    if (p->summation_density && !(p->single_phase && p->first_material == SPHG_WATER)) return SPHG_ERR_UNSUPPORTED;
    if (!(p->dt > 0.0) || p->max_interaction <= 0) return SPHG_ERR_BAD_ARG;
    return SPHG_OK;
}

int sphg_create(const sphg_params* p, int n_phase, sphg_ctx** out) {
    if (!out) return SPHG_ERR_BAD_ARG;
    *out = nullptr;
    int rc = validate(p, n_phase);
    if (rc) return rc;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) { cudaGetLastError(); return SPHG_ERR_NO_DEVICE; }
    sphg_ctx* c = new sphg_ctx();
    c->prm = *p;
    c->nphase = n_phase;
    cudaGetDevice(&c->device);
    if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) { delete c; return SPHG_ERR_CUDA; }
    c->stream = c->own_stream;
    if (cudaStreamCreateWithFlags(&c->side_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_fork2, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_join2, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        if (c->side_stream) cudaStreamDestroy(c->side_stream);
        if (c->ev_fork) cudaEventDestroy(c->ev_fork);
        if (c->ev_join) cudaEventDestroy(c->ev_join);
        if (c->ev_fork2) cudaEventDestroy(c->ev_fork2);
        cudaStreamDestroy(c->own_stream);
        delete c;
        return SPHG_ERR_CUDA;
    }
    if (p->precision == SPHG_FP64) c->eng = new Engine<double>(c);
    else c->eng = new Engine<float>(c);
    *out = c;
    return SPHG_OK;
}

int sphg_upload_phase(sphg_ctx* c, int phase, const sphg_phase_host* v) {
    if (!c) return SPHG_ERR_BAD_ARG;
    if (!v) return SPHG_ERR_BAD_ARG;
    if (c->prm.single_phase && v->material != c->prm.first_material) return SPHG_ERR_BAD_ARG;
    if (c->nphase == 2 && v->material != (phase == 1 ? SPHG_WATER : SPHG_SOIL)) return SPHG_ERR_BAD_ARG;
    cudaSetDevice(c->device);
    return c->eng->upload(phase, v);
}

int sphg_single_step(sphg_ctx* c, int itimestep) {
    if (!c) return SPHG_ERR_BAD_ARG;
    cudaSetDevice(c->device);
    int rc = c->eng->begin_batch();
    if (rc) return rc;
    rc = c->eng->rhs(itimestep);
    // close the batch in every case: it ends in the synchronisation after
    // which the next batch may clear the status flags on the host
    const int rc2 = c->eng->finish_batch();
    return rc ? rc : rc2;
}

int sphg_time_integration(sphg_ctx* c, int maxtimestep, int* itimestep, double* time) {
    if (!c || !itimestep || !time || maxtimestep < 0) return SPHG_ERR_BAD_ARG;
    cudaSetDevice(c->device);
    if (!c->ev_a && (cudaEventCreate(&c->ev_a) != cudaSuccess || cudaEventCreate(&c->ev_b) != cudaSuccess)) {
        cudaGetLastError();
        return SPHG_ERR_CUDA;
    }
    cudaEvent_t a = c->ev_a, b = c->ev_b;
    cudaEventRecord(a, c->stream);
    int rc = c->eng->begin_batch();
    for (int it = 0; it < maxtimestep && rc == 0; ++it) {
        int ts = *itimestep + 1;
        rc = c->eng->step(ts);
        if (rc) break;
        *itimestep = ts;
        *time = *time + c->prm.dt;
    }
    cudaEventRecord(b, c->stream);
    int rc2 = c->eng->finish_batch();
    float ms = 0.f;
    cudaEventSynchronize(b);
    cudaEventElapsedTime(&ms, a, b);
    c->last_step_ms = maxtimestep > 0 ? ms / maxtimestep : 0.0;
    c->itimestep = *itimestep;
    c->time = *time;
    return rc ? rc : rc2;
}

// ------------------------------------------------------- context groups
// One CUDA graph per step for several contexts: each context's step is a
// branch of the graph, forked from and joined back into the stream of the
// first context, so the contexts' kernels can overlap on the GPU.  A graph is
// kept per combination of the contexts' step kinds and recaptured when any
// context has dropped its own graphs (upload, tuning).
struct sphg_group {
    std::vector<sphg_ctx*> ctx;
    int device = 0;     // kept so that destroying the group touches no context
    struct Joint {
        cudaGraphExec_t exec = nullptr;
        std::vector<long long> launches, epochs;
    };
    std::map<std::vector<int>, Joint> joint;   // by the contexts' graph kinds
    std::vector<cudaEvent_t> ev;   // 0: fork; 1..n-1: joins
    bool use_graphs = true;
    ~sphg_group() {
        for (auto& kv : joint) if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
        for (auto e : ev) cudaEventDestroy(e);
    }
};

namespace {

// Capture the joint graph of step `ts`.  On entry every context's stream is
// stream 0 (the stream of context 0); context i > 0 is captured on its
// private stream, forked from and joined into stream 0.
int group_capture(sphg_group* g, int ts, sphg_group::Joint& J) {
    const int n = (int)g->ctx.size();
    cudaStream_t origin = g->ctx[0]->stream;
    std::vector<cudaStream_t> saved(n);
    for (int i = 0; i < n; ++i) saved[i] = g->ctx[i]->stream;
    J.launches.assign(n, 0);
    J.epochs.assign(n, 0);
    if (cudaStreamBeginCapture(origin, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    int rc = 0;
    cudaError_t e = cudaEventRecord(g->ev[0], origin);
    for (int i = 1; i < n && e == cudaSuccess; ++i) {
        g->ctx[i]->stream = g->ctx[i]->own_stream;
        e = cudaStreamWaitEvent(g->ctx[i]->stream, g->ev[0], 0);
    }
    for (int i = 0; i < n && e == cudaSuccess && rc == 0; ++i) {
        const long long before = g->ctx[i]->prof.launches;
        rc = g->ctx[i]->eng->capture_step(ts);
        J.launches[i] = g->ctx[i]->prof.launches - before;
        g->ctx[i]->prof.launches = before;
        J.epochs[i] = g->ctx[i]->eng->graph_epoch();
    }
    for (int i = 1; i < n && e == cudaSuccess; ++i) {
        e = cudaEventRecord(g->ev[i], g->ctx[i]->stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(origin, g->ev[i], 0);
    }
    cudaGraph_t graph = nullptr;
    cudaError_t ee = cudaStreamEndCapture(origin, &graph);
    for (int i = 0; i < n; ++i) g->ctx[i]->stream = saved[i];
    if (rc || e != cudaSuccess || ee != cudaSuccess || !graph) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        return rc ? rc : -1;
    }
    cudaError_t ei = cudaGraphInstantiate(&J.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) { J.exec = nullptr; cudaGetLastError(); return -1; }
    return 0;
}

// One step of every context: a joint graph replay when every context can
// replay one, else each context's own step in turn.
int group_step(sphg_group* g, int ts) {
    const int n = (int)g->ctx.size();
    std::vector<int> key(n, -1);
    bool graphed = g->use_graphs;
    // prepare first: a context that is not prepared reorders (and swaps its
    // buffers) in prepare(), which changes its graph kind
    for (int i = 0; i < n && graphed; ++i) {
        int rc = g->ctx[i]->eng->prepare_graph_step();
        if (rc) return rc;
    }
    for (int i = 0; i < n && graphed; ++i) {
        key[i] = g->ctx[i]->eng->graph_kind(ts);
        if (key[i] < 0) graphed = false;
    }
    if (graphed) {
        auto it = g->joint.find(key);
        if (it != g->joint.end()) {
            bool stale = false;
            for (int i = 0; i < n; ++i) stale |= it->second.epochs[i] != g->ctx[i]->eng->graph_epoch();
            if (stale) {
                if (it->second.exec) cudaGraphExecDestroy(it->second.exec);
                g->joint.erase(it);
                it = g->joint.end();
            }
        }
        if (it == g->joint.end()) {
            sphg_group::Joint J;
            int rc = group_capture(g, ts, J);
            if (rc > 0) return rc;
            if (rc < 0) g->use_graphs = false;
            else it = g->joint.emplace(key, J).first;
        }
        if (g->use_graphs) {
            CUDA_TRY(cudaGraphLaunch(it->second.exec, g->ctx[0]->stream));
            for (int i = 0; i < n; ++i) g->ctx[i]->eng->after_graph_step(it->second.launches[i], key[i]);
            return 0;
        }
    }
    for (int i = 0; i < n; ++i) {
        int rc = g->ctx[i]->eng->step(ts);
        if (rc) return rc;
    }
    return 0;
}

}  // namespace

int sphg_group_create(sphg_ctx* const* ctxs, int n, sphg_group** out) {
    if (!ctxs || !out || n < 1 || n > 32) return SPHG_ERR_BAD_ARG;
    *out = nullptr;
    for (int i = 0; i < n; ++i) {
        if (!ctxs[i] || ctxs[i]->device != ctxs[0]->device) return SPHG_ERR_BAD_ARG;
        for (int j = 0; j < i; ++j) if (ctxs[j] == ctxs[i]) return SPHG_ERR_BAD_ARG;
    }
    cudaSetDevice(ctxs[0]->device);
    sphg_group* g = new sphg_group();
    g->ctx.assign(ctxs, ctxs + n);
    g->device = ctxs[0]->device;
    g->ev.assign(n, nullptr);
    for (int i = 0; i < n; ++i) {
        if (cudaEventCreateWithFlags(&g->ev[i], cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            delete g;
            return SPHG_ERR_CUDA;
        }
    }
    *out = g;
    return SPHG_OK;
}

int sphg_group_time_integration(sphg_group* g, int maxtimestep, int* itimesteps, double* times) {
    if (!g || !itimesteps || !times || maxtimestep < 0) return SPHG_ERR_BAD_ARG;
    const int n = (int)g->ctx.size();
    for (int i = 1; i < n; ++i) if (itimesteps[i] != itimesteps[0]) return SPHG_ERR_BAD_ARG;
    cudaSetDevice(g->ctx[0]->device);
    cudaStream_t origin = g->ctx[0]->stream;
    std::vector<cudaStream_t> own(n);
    for (int i = 0; i < n; ++i) own[i] = g->ctx[i]->stream;
    cudaEvent_t a, b;
    cudaEventCreate(&a); cudaEventCreate(&b);
    int rc = 0;
    for (int i = 0; i < n && rc == 0; ++i) rc = g->ctx[i]->eng->begin_batch();
    // Every step of the group runs on stream 0, graph replays and steps
    // without a graph alike, so that they stay in order; only inside a joint
    // graph do the contexts run as parallel branches.  Stream 0 first waits
    // for the other contexts' earlier work.
    for (int i = 1; i < n; ++i) {
        if (own[i] == origin) continue;
        cudaEventRecord(g->ev[i], own[i]);
        cudaStreamWaitEvent(origin, g->ev[i], 0);
    }
    for (int i = 0; i < n; ++i) g->ctx[i]->stream = origin;
    cudaEventRecord(a, origin);
    for (int it = 0; it < maxtimestep && rc == 0; ++it) {
        const int ts = itimesteps[0] + 1;
        rc = group_step(g, ts);
        if (rc) break;
        for (int i = 0; i < n; ++i) {
            itimesteps[i] = ts;
            times[i] = times[i] + g->ctx[i]->prm.dt;
        }
    }
    cudaEventRecord(b, origin);
    for (int i = 0; i < n; ++i) g->ctx[i]->stream = own[i];
    // the other contexts' later work (statistics, downloads) after stream 0
    for (int i = 1; i < n; ++i) {
        if (own[i] == origin) continue;
        cudaStreamWaitEvent(own[i], b, 0);
    }
    int rc2 = 0;
    for (int i = 0; i < n; ++i) {
        int r = g->ctx[i]->eng->finish_batch();
        if (!rc2) rc2 = r;
    }
    float ms = 0.f;
    cudaEventSynchronize(b);
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a); cudaEventDestroy(b);
    for (int i = 0; i < n; ++i) {
        g->ctx[i]->last_step_ms = maxtimestep > 0 ? ms / maxtimestep : 0.0;
        g->ctx[i]->itimestep = itimesteps[i];
        g->ctx[i]->time = times[i];
    }
    return rc ? rc : rc2;
}

void sphg_group_destroy(sphg_group* g) {
    if (!g) return;
    cudaSetDevice(g->device);
    delete g;
}

int sphg_download_phase(sphg_ctx* c, int phase, sphg_phase_host* v) {
    if (!c) return SPHG_ERR_BAD_ARG;
    cudaSetDevice(c->device);
    return c->eng->download(phase, v);
}

int sphg_export_xv_device(sphg_ctx* c, int phase, double* x_dev, double* v_dev) {
    if (!c) return SPHG_ERR_BAD_ARG;
    cudaSetDevice(c->device);
    return c->eng->xv_device(phase, x_dev, v_dev, 1);
}

int sphg_import_xv_device(sphg_ctx* c, int phase, const double* x_dev, const double* v_dev) {
    if (!c) return SPHG_ERR_BAD_ARG;
    cudaSetDevice(c->device);
    return c->eng->xv_device(phase, (double*)x_dev, (double*)v_dev, 0);
}

int sphg_export_pairs(sphg_ctx* c, int which, int32_t* pi, int32_t* pj, int64_t cap, int64_t* n) {
    if (!c) return SPHG_ERR_BAD_ARG;
    cudaSetDevice(c->device);
    return c->eng->export_pairs(which, pi, pj, cap, n);
}

int sphg_stats(sphg_ctx* c, sphg_stats_t* out) {
    if (!c || !out) return SPHG_ERR_BAD_ARG;
    cudaSetDevice(c->device);
    return c->eng->stats(out);
}

int sphg_set_scenes(sphg_ctx* c, int nscenes, const sphg_scene* scenes) {
    if (!c) return SPHG_ERR_BAD_ARG;
    cudaSetDevice(c->device);
    return c->eng->set_scenes(nscenes, scenes);
}

int sphg_upload_scene_ids(sphg_ctx* c, int phase, const int32_t* scene_id) {
    if (!c) return SPHG_ERR_BAD_ARG;
    cudaSetDevice(c->device);
    return c->eng->upload_scene_ids(phase, scene_id);
}

int sphg_set_tuning(sphg_ctx* c, const sphg_tuning* t) {
    if (!c) return SPHG_ERR_BAD_ARG;
    cudaSetDevice(c->device);
    return c->eng->set_tuning(t);
}

int sphg_write_tecplot(sphg_ctx* c, const char* path_first, const char* path_second, int append,
                       const int32_t* zone_first, const int32_t* zone_second) {
    if (!c || !path_first || (c->nphase == 2 && !path_second)) return SPHG_ERR_BAD_ARG;
    for (int ph = 1; ph <= c->nphase; ++ph) {
        sphg_phase_host h;
        memset(&h, 0, sizeof(h));
        // sizes first
        int rc = c->eng->download(ph, &h);
        if (rc) return rc;
        const size_t n = (size_t)(h.ntotal + h.nvirt);
        std::vector<double> x(2 * n), vx(2 * n), p(n), rho(n), mass(n), vof(n), vof2(n), eps(n), sxx(n), sxy(n), syy(n);
        h.x = x.data(); h.vx = vx.data(); h.p = p.data(); h.rho = rho.data(); h.mass = mass.data();
        h.vof = vof.data(); h.vof2 = vof2.data(); h.epsilon_p = eps.data();
        h.sxx = sxx.data(); h.sxy = sxy.data(); h.syy = syy.data();
        if ((rc = c->eng->download(ph, &h))) return rc;
        rc = sphg_write_tecplot_phase(ph == 1 ? path_first : path_second, append, &h, ph == 1 ? zone_first : zone_second);
        if (rc) return rc;
    }
    return SPHG_OK;
}

int sphg_set_stream(sphg_ctx* c, void* s) {
    if (!c) return SPHG_ERR_BAD_ARG;
    c->stream = s ? (cudaStream_t)s : c->own_stream;
    return SPHG_OK;
}

int sphg_kernel_profile(sphg_ctx* c, int enable) {
    if (!c) return SPHG_ERR_BAD_ARG;
    c->prof.resolve();
    if (enable) c->prof.acc.clear();
    c->prof.on = enable != 0;
    return SPHG_OK;
}

int sphg_kernel_report(sphg_ctx* c, char* buf, int64_t cap) {
    if (!c || !buf || cap <= 0) return SPHG_ERR_BAD_ARG;
    c->prof.resolve();
    std::string s = "{\"launches\": " + std::to_string(c->prof.launches) + ", \"kernels\": {";
    bool first = true;
    for (auto& kv : c->prof.acc) {
        char tmp[256];
        snprintf(tmp, sizeof(tmp), "%s\"%s\": [%lld, %.6f]", first ? "" : ", ", kv.first.c_str(),
                 kv.second.first, kv.second.second);
        s += tmp;
        first = false;
    }
    s += "}}";
    if ((int64_t)s.size() + 1 > cap) return SPHG_ERR_BAD_ARG;
    memcpy(buf, s.c_str(), s.size() + 1);
    return SPHG_OK;
}

void sphg_destroy(sphg_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    c->prof.resolve();
    delete c->eng;
    if (c->ev_a) cudaEventDestroy(c->ev_a);
    if (c->ev_b) cudaEventDestroy(c->ev_b);
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    if (c->ev_fork2) cudaEventDestroy(c->ev_fork2);
    if (c->ev_join2) cudaEventDestroy(c->ev_join2);
    if (c->side_stream) { cudaStreamSynchronize(c->side_stream); cudaStreamDestroy(c->side_stream); }
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
}

const char* sphg_strerror(int code) {
    switch (code) {
        case SPHG_OK: return "ok";
        case SPHG_ERR_PAIR_OVERFLOW: return "too many interactions (pair list exceeds max_interaction)";
        case SPHG_ERR_OUT_OF_DOMAIN: return "particle out of range";
        case SPHG_ERR_BAD_KERNEL: return "no such kernel function (skf)";
        case SPHG_ERR_BAD_ARG: return "bad argument";
        case SPHG_ERR_CUDA: return "CUDA runtime error";
        case SPHG_ERR_TIMEOUT: return "device wait timed out";
        case SPHG_ERR_NONFINITE: return "non-finite particle position";
        case SPHG_ERR_UNSUPPORTED: return "option outside the implemented scope";
        case SPHG_ERR_STATE: return "call out of order (upload every phase first)";
        case SPHG_ERR_NO_DEVICE: return "no CUDA device";
    }
    return "unknown status";
}

}  // extern "C"
