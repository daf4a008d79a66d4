/*
 * sphg.h — C ABI of libsphg, a B200 (sm_100a) implementation of the
 * weakly-compressible two-phase (water/soil) SPH time step of
 * cwang2015/sources.
 *
 * The reference exposes its step as argument-less Fortran module procedures
 * acting on module globals (declarations_sph.f90:13,44-56):
 *     single_step                 declarations_sph.f90:1131  (two-phase RHS)
 *     single_step_for_water       declarations_sph.f90:1439  (water-only RHS)
 *     single_step_for_soil        declarations_sph.f90:1530  (soil-only RHS)
 *     time_integration            declarations_sph.f90:525   (two-phase leapfrog)
 *     time_integration_for_water  declarations_sph.f90:794
 *     time_integration_for_soil   declarations_sph.f90:978
 * called from sph.f90:51-57.  This header replaces those calls with explicit
 * entry points: the Fortran host keeps its arrays and passes plain pointers
 * (ISO_C_BINDING `c_loc`), the library keeps the particle state resident on
 * the GPU between calls.  No torch or CUDA types appear in any signature.
 *
 * Conventions
 *   - Every entry point returns an sphg_status (0 = OK).  The reference's
 *     `stop` statements become status codes; nothing inside the library
 *     aborts the process.
 *   - Host arrays follow the Fortran layouts of the reference's `particles`
 *     type (m_particles.f90:223-300): vectors are x(2,n) interleaved
 *     (x1,y1,x2,y2,...), scalars are (n); index k of a host array is Fortran
 *     particle k+1.  Real particles come first (1..ntotal), virtual (boundary)
 *     particles follow (ntotal+1..ntotal+nvirt), as take_real / take_virtual
 *     build them (m_particles.f90:808-893).
 *   - A context is single-threaded and not re-entrant; several contexts may
 *     coexist (each owns one CUDA stream).
 */
#ifndef SPHG_H
#define SPHG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SPHG_ABI_VERSION 2

/* Status codes.  The reference stops the program where these are returned:
 * pair overflow m_particles.f90:992-993,1053-1054; particle outside the grid
 * :1131-1136; bad kernel id :932. */
typedef enum sphg_status {
    SPHG_OK = 0,
    SPHG_ERR_PAIR_OVERFLOW = 1,   /* a pair list exceeded max_interaction      */
    SPHG_ERR_OUT_OF_DOMAIN = 2,   /* a particle left [x_min,x_max]x[y_min,y_max]*/
    SPHG_ERR_BAD_KERNEL = 3,      /* skf not in 1..4 (get_scale_k)              */
    SPHG_ERR_BAD_ARG = 4,         /* null pointer, bad phase, bad size          */
    SPHG_ERR_CUDA = 5,            /* a CUDA runtime call failed                 */
    SPHG_ERR_TIMEOUT = 6,         /* a bounded device wait gave up              */
    SPHG_ERR_NONFINITE = 7,       /* a NaN/Inf position was met                 */
    SPHG_ERR_UNSUPPORTED = 8,     /* option outside the implemented scope       */
    SPHG_ERR_STATE = 9,           /* call order violated (e.g. step before upload) */
    SPHG_ERR_NO_DEVICE = 10       /* no CUDA device / driver                     */
} sphg_status;

/* Phase materials: `imaterial` of the particles type (m_particles.f90:213). */
enum { SPHG_WATER = 1, SPHG_SOIL = 2 };

/* Arithmetic of the pair kernels.  FP64: every field and sum in double, as
 * the reference.  FP32: pair arithmetic, derivatives and neighbour sums in
 * float; positions, time and the leapfrog-integrated state (x, v, rho, vof,
 * stress, p) stay double. */
enum { SPHG_FP64 = 0, SPHG_FP32 = 1 };

/* Pair lists for sphg_export_pairs. */
enum { SPHG_PAIRS_FIRST = 0,   /* same-phase pairs of phase 1 (direct_find)   */
       SPHG_PAIRS_SECOND = 1,  /* same-phase pairs of phase 2 (direct_find)   */
       SPHG_PAIRS_CROSS = 2 }; /* phase-1 i x phase-2 j (direct_find_2)       */

/* type(material), m_particles.f90:19-29.  Water uses rho0,b,gamma,c,
 * viscosity; soil uses rho0,k,E,niu,c,cohesion,phi,porosity,permeability
 * (case file keys WATER PROPERTY, SOIL PROPERTY, DARCY PARAMETER, SOIL FAILURE
 * CRITERIA, declarations_sph.f90:288-314).  phi is in radians. */
typedef struct sphg_material {
    double rho0, b, gamma, c, viscosity;
    double k, porosity, permeability, G, E, niu, cohesion, phi;
} sphg_material;

/* The three configuration layers of the reference in one POD:
 * param.f90:10-133 module flags, type(numerical) m_particles.f90:31-55, and
 * the case-file values.  sphg_default_params() fills the reference defaults. */
typedef struct sphg_params {
    int32_t abi_version;            /* = SPHG_ABI_VERSION                         */
    int32_t dim;                    /* param.f90:10; only 2 is supported          */
    int32_t skf;                    /* m_particles.f90:141 (1 cubic,2 Gauss,3 quintic,4 Wendland) */
    int32_t single_phase;           /* case file SINGLE PHASE                     */
    int32_t first_material;         /* case file FIRST PHASE (single-phase runs)  */
    int32_t summation_density;      /* param.f90:79                               */
    int32_t average_velocity;       /* param.f90:80                               */
    int32_t visc_artificial;        /* param.f90:86                               */
    int32_t artificial_density;     /* param.f90:95                               */
    int32_t soil_artificial_stress; /* param.f90:96                               */
    int32_t volume_fraction;        /* param.f90:98                               */
    int32_t water_artificial_volume;/* param.f90:99                               */
    int32_t volume_fraction_renorm; /* param.f90:100                              */
    int32_t stress_integration;     /* param.f90:92 (1 Euler, 2 leapfrog)         */
    int32_t yield_criterion;        /* param.f90:93 (2 Drucker-Prager)            */
    int32_t plasticity;             /* param.f90:94 (0 none, 3 flow rule 3)       */
    int32_t integrate_scheme;       /* param.f90:78 (1 leapfrog)                  */
    int32_t precision;              /* SPHG_FP64 / SPHG_FP32                      */
    int32_t reorder_interval;       /* steps between spatial reorders of the device state (0: only at upload) */
    int32_t renorm_interval;        /* vof renormalisation period, 40 in declarations_sph.f90:1415 */
    double gravity;                 /* declarations_sph.f90:13, added to dvx(2)   */
    double numeric_gravity;         /* numerical%gravity m_particles.f90:40, used by darcy_law */
    double alpha, beta, etq;        /* m_particles.f90:44                         */
    double dd, p1, p2;              /* m_particles.f90:47                         */
    double delta;                   /* m_particles.f90:50                         */
    double epsilon;                 /* m_particles.f90:53                         */
    double dt;                      /* case file TIME STEP SIZE                   */
    double x_min, x_max, y_min, y_max; /* x_mingeom.. (m_particles.f90:89-91): neighbour grid extent */
    int64_t max_interaction;        /* param.f90:14: capacity of each pair list   */
    sphg_material water, soil;      /* H2O, SiO2 (declarations_sph.f90:44)        */
    /* Forchheimer coefficient b [s^2/m^2] of the water-soil drag.  The
     * reference's darcy_law (m_particles.f90:3832-3874) is linear: hydraulic
     * gradient i = u/k with u = v_w - v_s.  With b > 0 the drag follows
     * i = u/k + b|u|u, i.e. each pair's Darcy term is scaled by (1 + k b |u|).
     * 0 (the default) is the reference's law, bit for bit. */
    double forchheimer_b;
} sphg_params;

/* Host view of one phase: pointers into the Fortran arrays of a `particles`
 * object.  Vectors are (2,n) interleaved, n = ntotal + nvirt.  On upload,
 * x, vx, rho, p, c, mass, hsml, itype are required; a NULL optional field is
 * taken as zero.  On download, NULL fields are skipped.  txx/tyy/txy return
 * the shared working arrays (declarations_sph.f90:52,371-377,414-415) as the
 * reference leaves them, including the cross-phase aliasing. */
typedef struct sphg_phase_host {
    int32_t ntotal;          /* real particles                                    */
    int32_t nvirt;           /* virtual particles (stored after the real ones)    */
    int32_t material;        /* SPHG_WATER / SPHG_SOIL                            */
    int32_t nfail;           /* download only: soil points on the yield surface   */
    double dspp;             /* initial spacing; r0 of repulsive_force            */
    double *x, *vx, *dvx, *av, *v_min;                 /* (2,n)                   */
    double *rho, *rho_min, *drho, *p, *c, *mass, *hsml; /* (n)                    */
    double *vof, *vof_min, *dvof, *vof2;                /* (n) volume fractions   */
    double *sxx, *sxy, *syy, *dsxx, *dsxy, *dsyy, *dp;  /* (n) soil stress        */
    double *sxx_min, *sxy_min, *syy_min, *p_min;        /* (n) stress_integration=2 */
    double *epsilon_p, *vcc;                            /* (n)                    */
    double *txx, *tyy, *txy;                            /* (n) working arrays     */
    int32_t *itype;          /* >0 real, <0 virtual (setup_itype m_particles.f90:896) */
    int32_t *fail;           /* download only: soil failure flag                  */
} sphg_phase_host;

/* Counters (interaction_statistics m_particles.f90:555-597 and nfail). */
typedef struct sphg_stats_t {
    int64_t niac[3];         /* pairs: phase 1, phase 2, cross (last step)        */
    int32_t maxiac[2], miniac[2], noiac[2]; /* per-particle interaction stats     */
    int32_t nfail;           /* soil points on the yield surface                  */
    int32_t n_out_of_domain; /* particles clamped into the edge cells             */
    int32_t itimestep;
    int32_t _pad;
    double time;
    double last_step_ms;     /* device time per step of the last sphg_time_integration call */
} sphg_stats_t;

typedef struct sphg_ctx sphg_ctx;

/* Fill *p with the reference defaults (param.f90, m_particles.f90:31-55). */
void sphg_default_params(sphg_params* p);

/* Create a context for n_phase phases (1 single-phase, 2 water+soil) on the
 * current CUDA device.  Replaces allocate_sph (declarations_sph.f90:338). */
int sphg_create(const sphg_params* p, int n_phase, sphg_ctx** out);

/* Copy one phase (1-based: 1 = `parts`, 2 = `soil`) to the device.  Uploads
 * and downloads go through one device staging area of up to 37 doubles a
 * particle (at most 512 MB), made at the first transfer of the largest phase
 * and kept until sphg_destroy; pinned host arrays move at the link's speed. */
int sphg_upload_phase(sphg_ctx* ctx, int phase, const sphg_phase_host* v);

/* Right-hand side only: single_step (declarations_sph.f90:1131), or
 * single_step_for_water (:1439) / single_step_for_soil (:1530) in
 * single-phase runs.  itimestep drives the renormalisation period. */
int sphg_single_step(sphg_ctx* ctx, int itimestep);

/* maxtimestep leapfrog steps on the device: time_integration (:525),
 * time_integration_for_water (:794) or time_integration_for_soil (:978).
 * *itimestep and *time are advanced as the module globals are. */
int sphg_time_integration(sphg_ctx* ctx, int maxtimestep, int* itimestep, double* time);

/* A group of contexts stepped together (no counterpart in the reference; the
 * batched ensemble uses it, one context per kind of scene).  Every step of the
 * group after the first replays ONE CUDA graph that holds each context's step
 * as a parallel branch, forked from and joined into the stream of ctxs[0], so
 * the contexts' kernels overlap on the GPU.  The results are those of calling
 * sphg_time_integration on each context in turn.  itimesteps and times hold
 * one entry per context, as sphg_time_integration's arguments, and all
 * itimesteps must be equal.  A group must not be stepped once one of its
 * contexts is destroyed; sphg_group_destroy touches no context, so it may come
 * before or after them. */
typedef struct sphg_group sphg_group;
int sphg_group_create(sphg_ctx* const* ctxs, int n, sphg_group** out);
int sphg_group_time_integration(sphg_group* group, int maxtimestep, int* itimesteps, double* times);
void sphg_group_destroy(sphg_group* group);

/* Copy one phase back into the Fortran arrays (original particle order). */
int sphg_download_phase(sphg_ctx* ctx, int phase, sphg_phase_host* v);

/* Positions and velocities of one phase (2n doubles each, original particle
 * order) copied to (export) or from (import) caller DEVICE arrays on the
 * context's stream, without a host copy or a synchronisation; either
 * pointer may be NULL.  No counterpart in the reference, whose state lives in
 * module arrays the host reads directly: the learned stepper uses these to
 * take rollout snapshots and to hand a stride back to the solver. */
int sphg_export_xv_device(sphg_ctx* ctx, int phase, double* x_dev, double* v_dev);
int sphg_import_xv_device(sphg_ctx* ctx, int phase, const double* x_dev, const double* v_dev);

/* Pair list of the last step as 1-based (i,j), sorted by i then j, as
 * direct_find (m_particles.f90:938) / direct_find_2 (:1004) define it.
 * Writes min(n, cap) pairs and the total count to *n. */
int sphg_export_pairs(sphg_ctx* ctx, int which, int32_t* pair_i, int32_t* pair_j,
                      int64_t cap, int64_t* n);

/* Counters of the last step. */
int sphg_stats(sphg_ctx* ctx, sphg_stats_t* out);

/* Batched ensembles (no counterpart in the reference, whose program holds one
 * scene).  A context may hold several independent scenes side by side: the
 * host places them far enough apart that no pair crosses scenes, uploads
 * them as one phase, and gives each particle the index of its scene.  The
 * parameters that differ between scenes are per-scene; everything else in
 * sphg_params is shared.  soil_phi is the friction angle in radians.  With a
 * scene table, scene s advances by its own dt every step (its time is
 * itimestep * dt_s); *time of sphg_time_integration advances by p->dt. */
typedef struct sphg_scene {
    double dt;        /* TIME STEP SIZE of the scene                        */
    double water_b;   /* WATER PROPERTY b (Tait) of the scene               */
    double water_c;   /* WATER PROPERTY c (reference sound speed)           */
    double soil_phi;  /* SOIL FAILURE CRITERIA phi [rad]                    */
} sphg_scene;
int sphg_set_scenes(sphg_ctx* ctx, int nscenes, const sphg_scene* scenes);
/* scene index (0..nscenes-1) of every particle of a phase, original order */
int sphg_upload_scene_ids(sphg_ctx* ctx, int phase, const int32_t* scene_id);

/* Tuning knobs (no counterpart in the reference): the neighbour-cell edge as
 * a multiple (>= 1) of the support radius, the steps between spatial
 * reorders of the device state, and x_split, the number of cells each row of
 * that edge is cut into along x (1..8; 0 = the library default).  A particle
 * scans 3 rows of 2*x_split+1 cells: finer cells along x test fewer
 * candidates while each row stays one contiguous run of the cell-sorted
 * list.  They change the order in which neighbours are summed, so results
 * agree to rounding, and the pair sets not at all.  state_order picks the
 * order the device state is permuted into at each reorder: 0 = the cell
 * list's own order (rows of cells), 1 = the Morton (Z-order) curve over the
 * support-radius cells; the neighbour search and every sum are the same
 * either way (results bit-identical), only the memory layout differs. */
typedef struct sphg_tuning {
    double cell_factor;
    int32_t reorder_interval;
    int32_t x_split;
    int32_t state_order;
} sphg_tuning;
int sphg_set_tuning(sphg_ctx* ctx, const sphg_tuning* t);

/* The case (steering) file of the reference, read_cas / treat_cmd /
 * usr_def_parameter (declarations_sph.f90:61-335): "NAME = value" commands,
 * '#' comment lines, a trailing ',' continues a command on the next line,
 * a line starting with '&' ends the file.  sphg_read_case fills the
 * matching fields of *p (WATER PROPERTY, SOIL PROPERTY, DARCY PARAMETER,
 * SOIL FAILURE CRITERIA, TIME STEP SIZE, INTEGRATION SCHEME, SINGLE PHASE,
 * FIRST PHASE) and the rest into *c.  Unknown keywords are counted, as the
 * reference reports and skips them; a value that does not parse makes the
 * call return SPHG_ERR_BAD_ARG after reading the whole file. */
typedef struct sphg_case {
    int32_t print_step, save_step, nnps, single_phase, dry_soil, with_nozzle;
    int32_t first_material, second_material;   /* SPHG_WATER / SPHG_SOIL     */
    int32_t unknown_keywords, bad_values;
    double inlet_velocity, dt;
    char results[3][256];                       /* RESULTS FILE: three names  */
    char particle_size[32], operating_mode[32];
} sphg_case;
int sphg_read_case(const char* path, sphg_params* p, sphg_case* c);

/* Tecplot ASCII output of output (declarations_sph.f90:1703-1810): one zone
 * in BLOCK format with the reference's variable list (water: X, Y, Pressure,
 * VoF, vx, vy, rho, zone, VoF2, mass; soil: X, Y, Pressure, VoF, ep, sxy,
 * sxx, syy, vx, vy, rho, mass, sigma_yy = -p + syy, zone).  zone may be NULL
 * (written as 0).  The _phase form writes host arrays (no GPU involved); the
 * context form downloads phase 1 to path_first and, for two-phase contexts,
 * phase 2 to path_second, appending when `append` is set. */
int sphg_write_tecplot_phase(const char* path, int append, const sphg_phase_host* v, const int32_t* zone);
int sphg_write_tecplot(sphg_ctx* ctx, const char* path_first, const char* path_second, int append,
                       const int32_t* zone_first, const int32_t* zone_second);

/* Scene generators: the role of the reference's input_tank.f90 (water
 * column in a tank), input_soilfail.f90 (soil column in a box) and
 * input_mix_Savage.f90 (soil block under water), so that a Fortran host
 * builds its arrays without another layer.  Particles sit on the cell
 * centres of a dx lattice (block%cell_center, m_particles.f90:460-479, x outer
 * and y inner), real particles first, then two layers of virtual particles
 * under the floor and outside both walls (take_real / take_virtual,
 * m_particles.f90:808-893).  The case-file values the reference reads
 * (material constants, initial pressure and stress, dt) follow the choices
 * stated in sphg_scenes.cpp.  Host code only; no GPU needed.
 *   box_w x box_h   tank, box or domain
 *   col_w x col_h   water column, soil column, or soil block at the left wall
 *   water_h         two-phase only: depth of the water layer
 * sphg_scene_default fills the sizes of the three workloads this library is
 * measured on.  sphg_scene_size gives each phase's real and virtual particle
 * counts (n_phase entries each); the host allocates its arrays (x is (2,n))
 * and calls sphg_make_scene, which zeroes every non-NULL array of the views
 * and fills x, hsml, itype, p, c, vof, rho, mass (and sxx, sxy, syy for soil,
 * which are then required), and *p from sphg_default_params plus the scene's
 * values.  ntotal and nvirt of each view must be the counts of
 * sphg_scene_size. */
enum { SPHG_SCENE_DAM_BREAK = 1, SPHG_SCENE_GRANULAR_COLUMN = 2, SPHG_SCENE_TWO_PHASE = 3 };
typedef struct sphg_scene_spec {
    int32_t kind, skf, precision, _pad;
    double dx;
    double box_w, box_h;
    double col_w, col_h;
    double water_h;
    double phi_deg;                  /* soil friction angle [degrees]               */
    double porosity, permeability;   /* two-phase: soil porosity, Darcy k [m/s]     */
    double forchheimer_b;            /* two-phase: sphg_params.forchheimer_b        */
} sphg_scene_spec;
void sphg_scene_default(int kind, sphg_scene_spec* s);
int sphg_scene_size(const sphg_scene_spec* s, int32_t* n_phase, int32_t* ntotal, int32_t* nvirt);
int sphg_make_scene(const sphg_scene_spec* s, sphg_params* p, sphg_phase_host* first, sphg_phase_host* second);

/* Run the context's work on a caller-owned cudaStream_t (passed as void*);
 * NULL restores the context's own stream. */
int sphg_set_stream(sphg_ctx* ctx, void* cuda_stream);

/* Per-kernel CUDA-event timing: enable=1 starts recording, 0 stops.
 * sphg_kernel_report writes a JSON object
 *   {"launches": L, "kernels": {name: [launches, total_ms], ...}}
 * where L counts every kernel the context launched since its creation. */
int sphg_kernel_profile(sphg_ctx* ctx, int enable);
int sphg_kernel_report(sphg_ctx* ctx, char* buf, int64_t cap);

void sphg_destroy(sphg_ctx* ctx);
const char* sphg_strerror(int code);

/* Size limits of sphg_sum_density_noalloc. */
#define SPHG_NOALLOC_MAX_PARTICLES 32768
#define SPHG_NOALLOC_MAX_CELLS 65536

/* No counterpart in the reference: an allocation-free summation density
 * (the Shepard-normalised kernel sum that starts the water-only step) for
 * callers that cannot allocate device memory, e.g. a host whose GPU memory
 * is owned by another runtime's pool allocator, or a solver loop that runs on
 * a fixed memory budget and may not allocate during its time steps.
 * Inputs and the output are DEVICE pointers in the Fortran layout (x is
 * (2,n)); rho_out may alias rho.  Only p->skf, p->dim and the grid extent
 * p->x_min..y_max are read.  Its working memory is one static array of about
 * 4.3 MB that every GPU loading the library keeps until exit: n above
 * SPHG_NOALLOC_MAX_PARTICLES, or a neighbour grid above
 * SPHG_NOALLOC_MAX_CELLS cells, returns SPHG_ERR_BAD_ARG.  All calls share
 * that array, so calls whose GPU work overlaps race and must be serialised.
 * Every call looks up the array's device address with the caller's device
 * current; the first call on a device loads the library's device module and
 * should come before any stream capture.  The call waits on `cuda_stream`
 * once (for the h range and the position check); the result is complete when
 * the stream reaches the end of the call's work.  NaN or infinite positions
 * return SPHG_ERR_NONFINITE, non-positive h SPHG_ERR_BAD_ARG, before any
 * density kernel runs; particles outside the grid extent are clamped into
 * its edge cells, which keeps their pairs exact. */
int sphg_sum_density_noalloc(const sphg_params* p, int32_t n, const double* x_dev, const double* hsml_dev,
                             const double* mass_dev, const double* rho_dev, double* rho_out_dev,
                             void* cuda_stream);

#ifdef __cplusplus
}
#endif
#endif /* SPHG_H */
