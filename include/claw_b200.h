/*
 * claw_b200.h — C ABI of the B200-native Clawpack Classic wave-propagation
 * step.  Plain C types only; every function returns an int status:
 *
 *     0        success
 *     2..12    the reference's claw2 info codes (src/2d/claw2.f:288-310):
 *              2  fixed dt does not divide (tend - tstart)
 *              3  cfl_desired > cfl_max with variable dt
 *              5  capa_index > num_aux
 *              6  transverse_waves > order
 *              11 too many time steps (steps_max reached before tend)
 *              12 Courant number too large with fixed dt
 *     < 0      CLAW_E_* below (invalid argument, CUDA failure, ...)
 *
 * Arrays crossing this boundary are host arrays in structure-of-arrays order:
 *     q   : [num_eqn][mz][my][mx]          interior cells only, C order
 *     aux : [num_aux][mz+4][my+4][mx+4]    two ghost layers on every side
 * (1D / 2D drop the absent dimensions.)  The reference's arrays are the
 * Fortran q(meqn, 1-mbc:mx+mbc, 1-mbc:my+mbc): the same values, equation
 * index fastest and ghost cells included; ghost cells of q are produced by
 * the boundary conditions inside the step, exactly as bc2 fills them.
 *
 * A handle owns its device memory and is tied to one CUDA device and one
 * stream; calls on one handle are not reentrant (the reference's step2 /
 * claw2 are not reentrant either, through their COMMON blocks).
 */
#ifndef CLAW_B200_H
#define CLAW_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define CLAW_MAX_WAVES 8

/* Riemann solver plugins (compile-time device functors implementing the
 * rpn2/rpt2 contract of src/2d/claw2.f:312-404 in pointwise form). */
enum claw_solver_id {
    CLAW_SOLVER_ACOUSTICS_2D = 1,    /* q=(p,u,v); params: rho, bulk            */
    CLAW_SOLVER_VC_ADVECTION_2D = 2, /* q=(q); aux=(u edge, v edge, capa)       */
    CLAW_SOLVER_EULER_ROE_2D = 3,    /* q=(rho,rhou,rhov,E); params: gamma      */
    CLAW_SOLVER_ACOUSTICS_1D = 11,   /* q=(p,u); params: rho, bulk              */
    CLAW_SOLVER_VC_ACOUSTICS_1D = 12,/* q=(p,u); aux=(Z,c)                      */
    CLAW_SOLVER_ADVECTION_1D = 13,   /* q=(q); params: u                        */
    CLAW_SOLVER_EULER_ROE_1D = 14,   /* q=(rho,rhou,E); params: gamma           */
    CLAW_SOLVER_VC_ACOUSTICS_3D = 21 /* q=(p,u,v,w); aux=(Z,c)                  */
};

/* Boundary-condition codes beyond claw.data's 0..3: the built-in user BC of
 * examples/acoustics_3d_heterogeneous (bc3.f:282-312) -- a solid wall at
 * z-upper whose centre moves as a piston, w_ghost = 2 s(x,y,t) - w_interior
 * with s = -exp(-500 (x^2+y^2)) exp(-500 t^2) for t < 0.1.  Valid only at
 * bc_upper[2] with CLAW_SOLVER_VC_ACOUSTICS_3D; t is the step's start time. */
enum claw_bc { CLAW_BC_PISTON = 10 };

/* Built-in source terms psi(q) for source_split 1 (Godunov: src after each
 * step over dt) and 2 (Strang: dt/2 before and after), the src1 / src2 hooks
 * of src/1d/claw1.f:486-509 and src/2d/claw2.f:635-738.  The reference's
 * default src routine does nothing, which source_id CLAW_SOURCE_NONE keeps.
 * CLAW_SOURCE_RADIAL is examples/acoustics_2d_radial/1drad/src1.f:18-23: the
 * geometric term of radially symmetric acoustics with x as the radius,
 *     p <- p - dt (ndim - 1) bulk / x_i  u    for cells i = 1 .. mx+2,
 * ndim = source_ndim (2 cylindrical, 3 spherical), bulk = solver_params[1];
 * for CLAW_SOLVER_ACOUSTICS_1D, and for CLAW_SOLVER_ACOUSTICS_2D as the
 * axisymmetric (r, z) form (every row, u the radial velocity). */
enum claw_source_id { CLAW_SOURCE_NONE = 0, CLAW_SOURCE_RADIAL = 1 };

/* Built-in before-step routines: the b4step2 hook of src/2d/claw2.f:626-631,
 * called after bc2 and before each step (retries included) with the step's
 * start time, to set time-dependent aux arrays.  CLAW_B4STEP_NONE is the
 * reference's default (src/2d/b4step2.f90, nothing).  CLAW_B4STEP_REVERSING
 * scales the edge velocities of CLAW_SOLVER_VC_ADVECTION_2D (aux fields 1
 * and 2) by cos(pi t / T), T = b4step_param: the flow runs forward until
 * T/2 and backward to T, where an exact solution is back at its start.  The
 * aux given to claw_set_aux is kept as the unscaled field. */
enum claw_b4step_id { CLAW_B4STEP_NONE = 0, CLAW_B4STEP_REVERSING = 1 };

/* Arithmetic of the Riemann/limiter/update path. */
enum claw_precision {
    CLAW_FP64 = 0,      /* every multiply and add rounded separately: same
                           operation order as the reference, bit-identical to
                           the CPU restatement                                  */
    CLAW_FP64_FMA = 1,  /* fused multiply-add allowed (within 1e-12 relative)  */
    CLAW_FP32 = 2       /* FP32 update; CFL / dt / time stay FP64              */
};

enum claw_error {
    CLAW_E_INVALID = -1,     /* invalid configuration or argument            */
    CLAW_E_CUDA = -2,        /* CUDA runtime failure (see claw_last_error)   */
    CLAW_E_UNSUPPORTED = -3, /* valid for the reference, not built here      */
    CLAW_E_DEVICE = -4,      /* device-side wait gave up (no hang)           */
    CLAW_E_NAN = -5          /* Courant number is NaN                        */
};

/* Mirror of the clawdata fields of ClawRunData that reach claw2ez
 * (src/2d/claw2ez.f:39-156); integer codes as claw.data stores them. */
typedef struct claw_config {
    int num_dim;              /* 1, 2 or 3                                         */
    int num_cells[3];         /* mx, my, mz                                        */
    double lower[3];          /* xlower, ylower, zlower                            */
    double upper[3];          /* xupper, yupper, zupper                            */
    int num_eqn;              /* meqn                                              */
    int num_waves;            /* mwaves                                            */
    int num_aux;              /* maux  (method(7))                                 */
    int capa_index;           /* method(6), 1-based, 0 = none                      */
    int dt_variable;          /* method(1)                                         */
    int order;                /* method(2): 1 or 2                                 */
    int transverse_waves;     /* method(3): 0,1,2 (2D); 0,10,11,20,21,22 (3D)      */
    int dimensional_split;    /* 0 unsplit, 1 Godunov, 2 Strang (3D: Godunov)      */
    int verbosity;            /* method(4)                                         */
    int source_split;         /* method(5): 0 none, 1 Godunov, 2 Strang             */
    int use_fwaves;
    int limiter[CLAW_MAX_WAVES]; /* mthlim: 0 none,1 minmod,2 superbee,3 vanleer,4 MC,5 BW */
    int num_ghost;            /* mbc, must be 2                                    */
    int bc_lower[3];          /* mthbc: 0 user, 1 extrap, 2 periodic, 3 wall,
                                 CLAW_BC_PISTON                                    */
    int bc_upper[3];
    double dt_initial;        /* dtv(1)                                            */
    double dt_max;            /* dtv(2)                                            */
    double cfl_max;           /* cflv(1)                                           */
    double cfl_desired;       /* cflv(2)                                           */
    int steps_max;            /* nv(1)                                             */
    int solver_id;            /* enum claw_solver_id                               */
    double solver_params[8];  /* problem parameters of the solver (setprob)        */
    int precision;            /* enum claw_precision                               */
    int source_id;            /* enum claw_source_id (the src1 / src2 routine)     */
    int source_ndim;          /* CLAW_SOURCE_RADIAL: 2 cylindrical, 3 spherical    */
    int b4step_id;            /* enum claw_b4step_id (the b4step2 routine)         */
    int reserved[2];
    double b4step_param;      /* CLAW_B4STEP_REVERSING: the period T               */
} claw_config;

/* What claw2 returns through dtv / cflv / nv (src/2d/claw2.f:776-781). */
typedef struct claw_stats {
    double t_reached;         /* tend on return (time actually reached)            */
    double dt_min;            /* dtv(3)                                            */
    double dt_max_taken;      /* dtv(4)                                            */
    double dt_next;           /* dtv(5): dt to start the next call with            */
    double cfl_max_seen;      /* cflv(3)                                           */
    double cfl_last;          /* cflv(4)                                           */
    int steps_taken;          /* nv(2)                                             */
    int steps_rejected;
    int info;
    int device_error;
    double device_ms;         /* device time of the call (CUDA events on the
                                 handle's stream), host copies excluded           */
    long long launches;       /* step-kernel launches issued by the call          */
} claw_stats;

typedef struct claw_handle claw_handle;

/* Allocate device state for one grid.  Replaces the allocation of q, aux and
 * work in claw2ez (src/2d/claw2ez.f:182-263). */
int claw_create(const claw_config* cfg, claw_handle** out);
int claw_destroy(claw_handle* h);

/* Copy the interior of q from / to the host (pageable or pinned).  Replaces
 * qinit's fill of q (src/2d/claw2ez.f:244) and the read of q by out2. */
int claw_set_q(claw_handle* h, const double* q);
int claw_get_q(claw_handle* h, double* q);
/* aux with its two ghost layers, as setaux fills it (src/2d/claw2ez.f:224). */
int claw_set_aux(claw_handle* h, const double* aux);

/* One step of length dt from the current q, ghost cells from the boundary
 * conditions: bc2 + copyq2 + step2 (src/2d/claw2.f:622-668,
 * src/2d/step2.f90:2-251; bc3 + step3 in 3D, src/3d/step3.f90:3-873).
 * Writes the Courant number to *cfl and makes the new q current; no
 * accept/reject.  The step starts at the time the last advance reached
 * (0 after claw_create), advanced by dt per claw_step.  With dimensional
 * splitting (dimensional_split 1 or 2) the step is dimsp2 / dimsp3
 * (src/2d/dimsp2.f:1-99, src/3d/dimsp3.f:1-87): when a sweep's Courant
 * number exceeds cfl_max, *cfl is that sweep's number as dimsp2 returns it;
 * the state is then the whole split step (dimsp2 stops part-way, and claw2
 * discards the state either way). */
int claw_step(claw_handle* h, double dt, double* cfl);

/* Advance from tstart to tend with claw2's variable/fixed dt control,
 * rejection and retry (src/2d/claw2.f:494-784; src/1d/claw1.f:394-583 in
 * 1D; src/3d/claw3.f:620-928 in 3D, with chkmth's method check returning
 * info 6).  dt_initial plays dtv(1); the returned stats carry dtv/cflv/nv. */
int claw_advance(claw_handle* h, double tstart, double tend, double dt_initial,
                 claw_stats* stats);

/* claw_set_q + claw_advance + claw_get_q: the whole claw2 call on host arrays
 * (q in, q out), as claw2ez makes it once per output frame. */
int claw_advance_host(claw_handle* h, double* q, double tstart, double tend,
                      double dt_initial, claw_stats* stats);

/* nv(1) of the following claw_advance calls: the most time steps one call
 * takes before it returns info 11 with the state reached (claw2ez passes it
 * to every claw2 call; src/2d/claw2.f:497, 596, 766-769); starts as
 * cfg.steps_max. */
int claw_set_steps_max(claw_handle* h, int steps_max);

/* Device view of the current q (for zero-copy users): pointer, element size,
 * row pitch and field pitch in elements. */
int claw_q_device(claw_handle* h, void** ptr, int* elem_bytes, long long* ld,
                  long long* field_pitch);

/* Number of step-kernel launches issued on this handle so far. */
long long claw_launch_count(claw_handle* h);

/* Test hook for the device-wait failure path (no counterpart in the
 * reference, whose steps have no device waits).  wait_ns limits every
 * device-side wait of the handle's later steps (0: the 2 s default);
 * skip_row >= -2 makes the 2D step kernels of strip 0 skip the copy of that
 * row (-2 .. my+1, ghost rows included), so its wait runs out after wait_ns
 * and nothing faults; skip_row < -2 turns the hook off.  A step whose wait
 * ran out is not accepted: claw_advance / claw_step return CLAW_E_DEVICE and
 * the current q stays that of the last accepted step. */
int claw_debug_fault(claw_handle* h, long long wait_ns, int skip_row);

/* Conserved totals of the current q: totals[m] = sum over interior cells of
 * capa * q_m (capa = 1 without a capacity function), formed in FP64 with
 * Neumaier's compensated summation whatever the storage precision, in a fixed
 * order (the same q gives the same bits).  No counterpart in the reference,
 * whose regression checks sum frames on the host; the FP32 path keeps its
 * conservation sums in FP64 this way. */
int claw_totals(claw_handle* h, double* totals);

/* One 2D step (bc2 + step2, FP64) from caller-owned device buffers, with no
 * device allocation.  No counterpart in the reference: it serves callers that
 * cannot call cudaMalloc -- codes whose device memory all comes from their own
 * pool or arena, memory-capped partitions, time loops that cannot take
 * cudaMalloc's implicit device synchronisation.
 *   q_in, q_out : device arrays [num_eqn][my][q_ld] (q_ld >= mx, even,
 *                 16-byte aligned), distinct; q_out receives the new state
 *   aux         : device array [num_aux][my+4][aux_ld] or NULL
 *   stream      : a cudaStream_t (NULL = the default stream); the call waits
 *                 for it and returns the Courant number in *cfl
 * The step kernel's scratch (its control block) lives in a 256-byte static device
 * array of the library; every call looks up its device address on the
 * current device and resets it, and calls that overlap on the GPU race on
 * it.  Requests whose scratch would exceed the 256-byte maximum are rejected
 * with CLAW_E_INVALID.  Limits:
 *   - it must not be called while the stream is being captured (each call
 *     waits for the stream and uploads the control block from a host
 *     variable): CLAW_E_INVALID;
 *   - no before-step routine (b4step_id must be CLAW_B4STEP_NONE;
 *     otherwise CLAW_E_UNSUPPORTED): the hook needs a copy of the unscaled
 *     aux that this path cannot allocate;
 *   - the caller guarantees a positive capacity field (claw_set_aux checks
 *     it; this path does not): a NaN Courant number returns CLAW_E_NAN. */
int claw_step2d_noalloc(const claw_config* cfg, const double* q_in, double* q_out,
                        long long q_ld, const double* aux, long long aux_ld, double dt,
                        double* cfl, void* stream);

/* ---- Batches: many independent 2D grids advanced together -------------
 * Instances share the solver, its parameters, the method and the boundary
 * conditions; their num_cells, lower/upper and dt limits may differ.  Each
 * instance runs claw2's own dt control from its own Courant number
 * (src/2d/claw2.f:494-784, per instance); one persistent launch per step
 * covers the rows of every instance still advancing.  No counterpart in the
 * reference, whose claw2 advances one grid per call. */
typedef struct claw_batch claw_batch;

/* count instances (1..1024), cfgs[k] for instance k; FP64, 2D. */
int claw_batch_create(const claw_config* cfgs, int count, claw_batch** out);
int claw_batch_destroy(claw_batch* b);
/* q of instance k, [num_eqn][my][mx] as for claw_set_q / claw_get_q */
int claw_batch_set_q(claw_batch* b, int k, const double* q);
int claw_batch_get_q(claw_batch* b, int k, double* q);
/* Advance every instance from tstart to tend.  dt_initial[k] seeds instance
 * k (NULL: cfgs[k].dt_initial); stats[count] receives each instance's claw2
 * returns and info.  Returns 0, or the first nonzero per-instance info. */
int claw_batch_advance(claw_batch* b, double tstart, double tend, const double* dt_initial,
                       claw_stats* stats);

/* Autotuner of the batch launch shape.  It times trial steps from the
 * instances' current q with dt_trial[k] (NULL: each config's dt_initial), min
 * over `repeats`: the CTA count per SM (the resident maximum down to half) on
 * a step of every instance, then the tile height (16 .. 192 rows of a
 * 28-column strip per warp, at least) on a step of the largest instance alone,
 * the regime that ends an uneven ensemble.  It keeps the fastest shape and
 * returns it with the full step's time.  The trial steps leave q and the
 * instances' state as they were.  No counterpart in the reference. */
int claw_batch_autotune(claw_batch* b, const double* dt_trial, int repeats, int* min_rows,
                        int* ctas_per_sm, double* ms_per_step);
/* Set the launch shape directly (a shape kept from an earlier tuning run). */
int claw_batch_set_shape(claw_batch* b, int min_rows, int ctas_per_sm);

/* FP64 fused multiply-add throughput of the current device in TFLOP/s (2
 * flops per FMA; independent FMA chains, best of five timed launches), the
 * ceiling beside HBM bandwidth for the FP64 step kernels.  No counterpart in
 * the reference. */
int claw_probe_fp64(double* tflops, double* ms_best);

/* Test hook: the contracted build's Newton-refined reciprocal and square root
 * (rcp_newton, sqrt_newton: hardware estimate plus Newton-Raphson steps)
 * evaluated on the device for n host values x, so a test can hold them to
 * IEEE 1/x and sqrt(x).  No counterpart in the reference. */
int claw_check_newton(const double* x, int n, double* rcp, double* root);

/* Last error message of the calling thread ("" if none). */
const char* claw_last_error(void);

/* Library / build identification. */
const char* claw_build_info(void);

#ifdef __cplusplus
}
#endif
#endif /* CLAW_B200_H */
