/*
 * bld.h -- C ABI of the B200-native time-step engine for BoundaryLayerDynamics.jl.
 *
 * The engine replaces the reference's per-stage Julia closures
 *   rate!(du, u, t)        -> compute_rates!   (src/BoundaryLayerDynamics.jl:149-158,
 *                                               src/Processes.jl:39-62)
 *   projection!(u)         -> apply_projections! (src/BoundaryLayerDynamics.jl:161-165,
 *                                               src/Processes.jl:67-75)
 *   perform_step!/step_to! -> the explicit integrators (src/ODEMethods.jl:100-166,217-234)
 * with hand-written sm_100a kernels.  All entry points are plain C: pointers,
 * sizes and POD structs, no exceptions; every function returns a bld_status.
 *
 * Field layout (host and device): a spectral field is interleaved complex
 * double, column-major (k1, k2, z) exactly like the reference's
 * Array{Complex{Float64},3} of size (k1max+1, 2*k2max+1, n3) with k2 ordered
 * 0..k2max, -k2max..-1 (src/Grids.jl:74-83,91-93).  vel1 and vel2 live on the
 * n3 C nodes, vel3 on the n3-1 I nodes (src/Grids.jl:97-99).
 */
#ifndef BLD_H
#define BLD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BLD_ABI_VERSION 1

/* status codes (no exception crosses the ABI) */
typedef enum {
    BLD_OK = 0,
    BLD_ERR_INVALID_CONFIG = -1,  /* bad sizes / unsupported physical-domain size          */
    BLD_ERR_OUT_OF_MEMORY = -2,   /* cudaMalloc failed                                       */
    BLD_ERR_DIVERGED = -3,        /* a rate was not finite: "The simulation has diverged."
                                     (src/BoundaryLayerDynamics.jl:155-157)                  */
    BLD_ERR_UNSUPPORTED_BC = -4,  /* pressure needs Dirichlet w with equal values
                                     (src/processes/pressure.jl:338-339,357); advection
                                     needs w = 0 (src/processes/momentum_advection.jl:182);
                                     SGS needs rough-wall / free-slip walls
                                     (src/processes/static_smagorinsky.jl:92-98)           */
    BLD_ERR_CUDA = -5,            /* a CUDA runtime call failed (see bld_last_error)         */
    BLD_ERR_TIMEOUT = -6,         /* a bounded device wait expired                           */
    BLD_ERR_ARGUMENT = -7,        /* null pointer / out-of-range argument                    */
    BLD_ERR_NO_DEVICE = -8        /* no CUDA device or the library was not built for it      */
} bld_status;

typedef enum { BLD_BC_DIRICHLET = 0, BLD_BC_NEUMANN = 1 } bld_bc_kind;

/* wall types used by the SGS wall model (src/Domains.jl:181-200) */
typedef enum { BLD_WALL_OTHER = 0, BLD_WALL_ROUGH = 1, BLD_WALL_FREESLIP = 2 } bld_wall_kind;

typedef enum { BLD_FP64 = 0, BLD_MIXED = 1 } bld_precision;

/* src/ODEMethods.jl:21-50 */
typedef enum { BLD_EULER = 0, BLD_AB2 = 1, BLD_SSPRK22 = 2, BLD_SSPRK33 = 3 } bld_method;

/* dealiasing modes of MomentumAdvection / StaticSmagorinskyModel (src/physical_space.jl:42-56) */
typedef enum { BLD_DEALIAS_NONE = 0, BLD_DEALIAS_QUADRATIC = 1, BLD_DEALIAS_EXPLICIT = 2 } bld_dealias;

/*
 * Model description (Model(resolution, domain, processes), src/BoundaryLayerDynamics.jl:72-97).
 * The vertical mapping is passed as tables the caller evaluates from its Domain
 * (src/Domains.jl:97-135): dx3/dzeta at the C nodes and at the n3+1 I
 * positions zeta = 0, 1/n3, ..., 1, and x3 at the C and interior I nodes.
 * Arrays are copied by bld_create; the caller keeps ownership.
 */
typedef struct {
    int32_t n1, n2, n3;            /* resolution (modes x1, modes x2, layers x3), n3 >= 3  */
    int32_t members;               /* independent ensemble members of this size (>= 1)     */
    double l1, l2;                 /* horizontal domain size                               */
    double x3_min, x3_max;         /* vmap(0), vmap(1)                                     */
    const double* dx3_c;           /* [n3]    Dvmap at C nodes                             */
    const double* dx3_i;           /* [n3+1]  Dvmap at I positions incl. both boundaries   */
    const double* x3_c;            /* [n3]    vmap at C nodes                              */
    const double* x3_i;            /* [n3-1]  vmap at interior I nodes                     */
    /* boundary conditions per field (vel1, vel2, vel3) and side (lower, upper);
       for Neumann the value is the gradient d/dx3 (src/boundary_conditions.jl:40-43,55-57) */
    int32_t bc_kind[3][2];
    double bc_value[3][2];
    int32_t wall_kind[2];          /* lower/upper wall type for the SGS wall model         */
    double wall_z0[2];             /* roughness length (RoughWall)                         */
    double wall_kappa[2];          /* von Karman constant (RoughWall)                      */
    /* processes */
    int32_t advection;             /* MomentumAdvection present                            */
    int32_t adv_dealias;           /* bld_dealias                                          */
    int32_t adv_p1, adv_p2;        /* explicit physical size when adv_dealias==EXPLICIT    */
    int32_t diffusion[3];          /* MolecularDiffusion(vel_i, nu_i) present              */
    double diffusivity[3];
    int32_t pressure;              /* Pressure()                                           */
    int32_t source[3];             /* ConstantSource(vel_i, S_i) present                   */
    double source_strength[3];
    int32_t mean[3];               /* ConstantMean(vel_i, Q_i) present (C-node fields)     */
    double mean_value[3];
    int32_t sgs;                   /* StaticSmagorinskyModel present                       */
    int32_t sgs_dealias;           /* bld_dealias                                          */
    int32_t sgs_p1, sgs_p2;
    double sgs_cs;                 /* Cs                                                   */
    int32_t sgs_wall_damping;      /* wall_damping                                         */
    double sgs_wall_damping_exponent;
    int32_t precision;             /* bld_precision                                        */
    int32_t device;                /* CUDA device ordinal                                  */
    /* optional per-member overrides (arrays of length `members`, or NULL) */
    const double* member_cs;           /* Cs of each member                                */
    const double* member_z0_lower;     /* roughness length of the lower rough wall         */
    const double* member_source1;      /* ConstantSource strength for vel1                 */
} bld_config;

typedef struct {
    int32_t k1max, k2max, n3, members;
    int64_t modes_per_layer;       /* (k1max+1)*(2*k2max+1)                                */
    int64_t state_doubles;         /* doubles of one member's (vel1, vel2, vel3) state     */
    int32_t adv_p1, adv_p2;        /* physical size the kernels use for advection (0: off) */
    int32_t adv_ref_p1, adv_ref_p2;/* the reference's pdsize for the same process          */
    int32_t sgs_p1, sgs_p2;        /* physical size used by the SGS kernels (0: off)       */
    int64_t device_bytes;          /* device memory held by the handle                     */
    int32_t precision;
} bld_info;

typedef struct bld_handle bld_handle;

/* library */
int32_t bld_abi_version(void);
const char* bld_status_string(int32_t status);
/* copies the last error message of the calling thread into buf (NUL-terminated) */
int32_t bld_last_error(char* buf, size_t len);

/* Model(resolution, domain, processes) (src/BoundaryLayerDynamics.jl:79-96):
   validates the process set, factorises the pressure matrices
   (src/processes/pressure.jl:231-264) and allocates all device buffers. */
int32_t bld_create(const bld_config* cfg, bld_handle** out);
void bld_destroy(bld_handle* h);
int32_t bld_get_info(const bld_handle* h, bld_info* info);

/* model.state <-> host arrays (interleaved complex, reference layout), one member */
int32_t bld_set_state(bld_handle* h, int32_t member, const double* vel1, const double* vel2, const double* vel3);
int32_t bld_get_state(bld_handle* h, int32_t member, double* vel1, double* vel2, double* vel3);

/* compute_rates!(rates, state, t, processes, ...) + the isfinite scan of rate!
   on host arrays of one member (src/Processes.jl:39-62, src/BoundaryLayerDynamics.jl:149-158).
   Returns BLD_ERR_DIVERGED if any rate is not finite (the rates are still written). */
int32_t bld_compute_rates(bld_handle* h, int32_t member,
                          const double* vel1, const double* vel2, const double* vel3,
                          double* rate1, double* rate2, double* rate3);

/* apply_projections!(state, processes) in place on host arrays of one member
   (src/Processes.jl:67-75: Pressure, then ConstantMean). */
int32_t bld_apply_projections(bld_handle* h, int32_t member, double* vel1, double* vel2, double* vel3);

/* evolve!(model, (t1, t2); dt, method) on the device-resident state of all members
   (src/BoundaryLayerDynamics.jl:190-219): one projection and one rate evaluation,
   then round((t2-t1)/dt) steps, each followed by a rate evaluation. */
int32_t bld_evolve(bld_handle* h, double t1, double t2, double dt, int32_t method);

/* The inner loop of evolve!: `nsteps` steps from the current state and slope,
   replayed from a CUDA graph.  bld_evolve (or bld_prepare) must have run once. */
int32_t bld_prepare(bld_handle* h);                       /* projection + rates  */
int32_t bld_step(bld_handle* h, int64_t nsteps, double dt, int32_t method);

/* Device-pointer variants, stream-ordered on `stream` (a cudaStream_t, or NULL for
   the handle's stream).  Pointers address all members' fields packed as
   [member][vel1 | vel2 | vel3].  They neither synchronise nor check divergence;
   bld_sync reports a non-finite rate seen since the last check. */
int32_t bld_compute_rates_device(bld_handle* h, const void* state, void* rates, void* stream);
int32_t bld_apply_projections_device(bld_handle* h, void* state, void* stream);
int32_t bld_state_device_ptr(bld_handle* h, void** state);
int32_t bld_sync(bld_handle* h);

/* The handle's CUDA stream (cudaStream_t) on which every launch of the handle is
   ordered, so callers can record CUDA events around engine work. */
int32_t bld_get_stream(bld_handle* h, void** stream);

/* bld_step without the trailing synchronisation and divergence check: enqueues
   `nsteps` graph launches and returns; bld_sync reports the outcome. */
int32_t bld_step_async(bld_handle* h, int64_t nsteps, double dt, int32_t method);
/* Non-blocking: *idle = 1 when all work enqueued on the handle's stream has
   finished (then bld_sync returns at once with the divergence check), else 0. */
int32_t bld_stream_idle(bld_handle* h, int32_t* idle);

/* Limit, in SM clock cycles, of the kernels' bounded waits for their own TMA
   copies on `device` (default 2^31, about one second); cycles < 0 restores the
   default.  cycles = 0 is a diagnostic setting: every such wait gives up at once,
   the kernels take their timeout exit (after their copies have landed) and the
   next call that checks the flags returns BLD_ERR_TIMEOUT.  Affects only the
   TMA-staged kernels (k_adv_x2, k_inv_y3, k_project_tile, k_project_pipe,
   k_sgs_x2 and the staged k_sgs_x); the setting is device-wide. */
int32_t bld_set_wait_limit(int32_t device, int64_t cycles);

/* Average device time of each launch kind of one right-hand side, measured with
   CUDA events on the handle's stream over `iters` back-to-back launches of that
   kind on the resident state (index 0: advection space, 1: SGS space). */
typedef struct {
    double inv_y_ms[2];            /* inverse y pass                              */
    double x_ms[2];                /* x transforms + physical-domain products     */
    double fwd_y_ms[2];            /* forward y pass + linear terms               */
    double project_ms;             /* stage update + pressure projection          */
    double linear_ms;              /* linear-only rates (no nonlinear process)    */
    int32_t launches_per_step;     /* kernel launches of one step of the method   */
} bld_phase_times;
int32_t bld_time_phases(bld_handle* h, int32_t iters, int32_t method, bld_phase_times* out);

/* Ensemble slots (continuous batching); no reference counterpart (the reference
   runs one model per process).  All members of a handle share one step graph;
   bld_set_active marks which members bld_step / bld_step_async /
   bld_ensemble_step advance (host array of `members` ints, nonzero = active;
   NULL = all).  Inactive members' blocks exit at once, so a slot costs nothing
   while free, and the mask is read on the device, so changing it needs no new
   graph.  Single-member calls (bld_compute_rates, bld_apply_projections,
   bld_prepare_member, bld_set_field_physical) ignore the mask.
   bld_set_member_params replaces the per-member Cs, lower-wall roughness length
   and vel1 forcing of `member` (NAN keeps a value).  bld_prepare_member runs the
   initial projection and rates (what evolve! does first) for one member after
   its state was set.  Divergence is flagged per member: after a call returned
   BLD_ERR_DIVERGED, bld_get_diverged writes 1 for each member whose rates turned
   non-finite since the previous bld_get_diverged (`members` ints) and clears them. */
int32_t bld_set_active(bld_handle* h, const int32_t* mask);
int32_t bld_set_member_params(bld_handle* h, int32_t member, double cs, double z0_lower, double source1);
int32_t bld_prepare_member(bld_handle* h, int32_t member);
int32_t bld_get_diverged(bld_handle* h, int32_t* out);

/* The kernel variants the autotuner chose for this handle, as a JSON object
   (per physical-domain space: sizes, y-pass and x-pass kernels; the projection
   kernel), NUL-terminated in `buf`.  Diagnostics; no reference counterpart. */
int32_t bld_describe(bld_handle* h, char* buf, size_t len);

/* Advances several handles on one device (e.g. the size classes of an uneven
   ensemble) by `nsteps` steps of `method`: each step is ONE launch of a CUDA
   graph whose child graphs are the handles' step graphs, run as independent
   branches so the classes overlap on the device.  Every handle must have been
   prepared (bld_prepare / bld_evolve).  Synchronises and checks divergence. */
int32_t bld_ensemble_step(bld_handle* const* handles, int32_t n, int64_t nsteps, double dt, int32_t method);

/* Physical-domain fields at the default size (2*k1max+2, 2*k2max+2) of one member:
   initialize!(model; vel = values) (src/State.jl:11-31, set_field! src/physical_space.jl:253-275)
   and model[:vel] (src/State.jl:81-85, get_field src/physical_space.jl:315-319).
   `values` is float64 (P1, P2, nz) column-major (x fastest). field: 0, 1, 2. */
int32_t bld_set_field_physical(bld_handle* h, int32_t member, int32_t field, const double* values);
int32_t bld_get_field_physical(bld_handle* h, int32_t member, int32_t field, double* values);

/* The same at the centres of the grid intervals (x1, x2 shifted by half a grid
   spacing): get_field(...; centered = true) / set_field!(...; centered = true)
   with shift!/unshift! (src/physical_space.jl:277-336), as Snapshots writes and
   initialize!(model, path) reads them (src/logging.jl:582-601, src/State.jl:33-66). */
int32_t bld_get_field_centered(bld_handle* h, int32_t member, int32_t field, double* values);
int32_t bld_set_field_centered(bld_handle* h, int32_t member, int32_t field, const double* values);

/* Seeded initial condition generated on the device: initialize!(model; vel =
   f) (src/State.jl:11-31, set_field! src/physical_space.jl:253-275) for the
   fields f(x1, x2, x3) = base(x3) + scale(x3) r(x1, x2, x3) of the benchmark
   workloads (a mean profile with uniform or Gaussian perturbations), without
   building the physical field on the host.  `base` and `scale` are host arrays
   of the field's nz layers (nz <= 512); r is uniform on [-1, 1) (distribution
   0) or standard normal (1, Box-Muller), drawn from the SplitMix64 output
   function of key + counter with key = splitmix64(seed) ^ splitmix64(field +
   1) and counter 2 i (and 2 i + 1 for the second Box-Muller draw), i = (z P2 +
   y) P1 + x on the default grid, so a host can reproduce every value.  The
   physical values go through the forward transforms as in bld_set_field_physical. */
int32_t bld_init_random_field(bld_handle* h, int32_t member, int32_t field, const double* base, const double* scale,
                              int32_t distribution, uint64_t seed);

/* Mean profiles accumulated on the device (MeanProfiles, src/logging.jl:333-491).
   The horizontal mean of a frequency-space field is the real part of its (0,0)
   mode.  bld_profiles_start(h, 1) zeroes the time integrals and records the
   current state as the first sample; from then on every step (bld_step,
   bld_step_async, bld_evolve, bld_ensemble_step) adds the trapezoid
   (dt/2)(previous sample + new sample) for every member inside the step graph,
   so nothing leaves the device between outputs; bld_evolve records the projected
   initial state as the first sample.  bld_profiles_start(h, 0) stops sampling.
   bld_profiles_read copies member m's integrals and bld_profiles_sample its
   current sample, each 3*(n3+1) doubles: vel1 at the n3 C nodes (one unused
   zero), vel2 likewise, vel3 as lower boundary, the n3-1 I nodes, upper boundary
   (the boundary entries stay zero, as for log_state! of the state). */
int32_t bld_profiles_start(bld_handle* h, int32_t on);
int32_t bld_profiles_read(bld_handle* h, int32_t member, double* out);
int32_t bld_profiles_sample(bld_handle* h, int32_t member, double* out);

/* The statistics ProgressMonitor prints (src/logging.jl:215-276), from one
   member's device-resident state:
   - mean_velocity: sum over layers of Re q(0,0) weighted by dx3 / L3 (vel1,
     vel2 on the C nodes, vel3 on the interior I nodes);
   - mean_ke / turbulent_ke: sum over the C layers of <u>^2 + <v>^2 and of
     <u^2 + v^2> - <u>^2 - <v>^2 (horizontal means; by Parseval from the modes,
     as exact as on the physical grids);
   - advective_timescale: min over the I layers of dx3 / max |w|, with max |w|
     over the largest physical grid of the model (grid_p1 x grid_p2; +inf
     where w vanishes); the Courant number is dt / advective_timescale;
   - wall_stress[i][side]: horizontal mean of the wall-model stress tau_i3 =
     factor u_i sqrt(u_1^2 + u_2^2) at the first C layer next to a rough wall
     (lower, upper), on the Smagorinsky grid (src/processes/static_smagorinsky.jl:
     195-200); 0 elsewhere.
   The first call allocates the handle's scratch for the physical fields. */
typedef struct {
    double mean_velocity[3];
    double mean_ke, turbulent_ke;
    double advective_timescale;
    double wall_stress[2][2];
    int32_t grid_p1, grid_p2;
} bld_progress;
int32_t bld_progress_stats(bld_handle* h, int32_t member, bld_progress* out);

/* Standalone batched symmetric tridiagonal solve (the kernel of
   ldiv!(::DistributedBatchLDLt, b), src/processes/pressure.jl:106-201):
   `nsys` systems of size `n` (1 <= n <= 1024), factor `gamma` [n][nsys] (the
   reference's gamma = 1/(d_z - gamma_{z-1} beta_{z-1}^2), pressure.jl:86-95) and
   off-diagonal `beta` [n-1] shared by all systems, right-hand sides `rhs`
   [n][nsys] solved in place: complex (interleaved double2) or real.  Device
   pointers, stream-ordered. */
int32_t bld_ldlt_solve_device(const double* gamma, const double* beta, void* rhs,
                              int64_t nsys, int32_t n, void* stream);
int32_t bld_ldlt_solve_real_device(const double* gamma, const double* beta, double* rhs,
                                   int64_t nsys, int32_t n, void* stream);

/* Pressure projection that allocates nothing.  No counterpart in the reference:
   it exists for callers that cannot call cudaMalloc -- code whose device memory
   is owned by a host framework's pool (a Julia CuArray pool, an embedding
   application with a fixed memory budget) and that must not have a library
   allocate behind its back.  Such a caller passes every buffer: the velocity
   fields `state` (device, vel1|vel2|vel3 in the reference layout, projected in
   place) and the tables of the Pressure process on the device: `gamma` [n3][F]
   (the LDL^T factor, DistributedBatchLDLt.γ transposed to z-major), `alpha_c`
   [n3] and `alpha_i` [n3-1] (N3/(dx3/dzeta) at C and I nodes), `d1` [k1max+1]
   and `d2` [2*k2max+1] (k*2pi/L).  The forward-sweep scratch of the solve lives
   in one fixed device array inside the library of BLD_NOALLOC_MAX_VALUES
   complex doubles (16 MiB), which every GPU that loads the library holds until
   the process exits; n3 * (k1max+1) * (2*k2max+1) above that limit is rejected
   with BLD_ERR_INVALID_CONFIG.  `w_lo` and `w_hi` are the Dirichlet values of
   vel3 at the lower and upper boundary; like the regular projection, unequal
   values are rejected with BLD_ERR_UNSUPPORTED_BC ("The mean flow must be equal
   at both vertical boundaries.").  Every call outside a stream capture looks up
   the array's device address on the current device (so a device reset does not
   leave a stale address behind); a call during a capture uses the address an
   earlier call on that device found, so the first call on a device must come
   before any stream capture.  All calls share the array: calls that overlap on
   the GPU (other streams, other threads) race, so serialise them.  The solve
   writes every scratch value before reading it, so no clearing is needed
   between calls. */
#define BLD_NOALLOC_MAX_VALUES (1 << 20)
int32_t bld_project_noalloc(int32_t k1max, int32_t k2max, int32_t n3,
                            const double* gamma, const double* alpha_c, const double* alpha_i,
                            const double* d1, const double* d2, double w_lo, double w_hi,
                            void* state, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* BLD_H */
