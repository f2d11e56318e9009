/*
 * sp_abi.h -- C ABI of the B200 (sm_100a) advection-diffusion propagator and
 * Parareal driver.
 *
 * The library replaces two C++ classes of andyspiros/StencilParareal:
 *   class Convection   src/Convection/Convection.h:22-108
 *   class Parareal     src/Parareal/Parareal.h:38-289
 * Each entry point below names the reference interface it stands for.  All
 * entry points return an int status (SP_OK = 0, negative = error; they never
 * abort the process); sp_last_error() describes the last failure of the
 * calling thread.  One handle per host thread: a handle is not re-entrant,
 * just as the reference's Convection object mutates its own scalars and joker
 * bindings on every call (Convection.cpp:318-392).
 *
 * Field storage (device memory, owned by the caller).  A field holds the
 * interior ni x nj x nk cells plus a 2-cell periodic halo on every side, i
 * fastest, like the reference's CUDA ConvectionField (Convection.h:13-17:
 * halo 2 in i, j and k; KJI order; i padded for alignment).  sp_field_layout()
 * gives the exact geometry: element (i,j,k), -2 <= i < ni+2 (same for j, k),
 * lives at  origin + k*plane + j*px + i.  Every kernel of this library that
 * writes a field also writes the periodic images of its boundary cells, so a
 * field produced by the library always has a valid halo.  A field written by
 * the caller needs sp_periodicity_apply() (or sp_field_import(), which fills
 * the halo) -- exactly as the reference refreshes the input halo in place
 * before every stencil (Convection.cpp:328-334, Periodicity.h:60-66).
 *
 * Dense arrays (import/export, host entry points): interior only, i fastest,
 * element (i,j,k) at (k*nj + j)*ni + i.
 */
#ifndef SP_ABI_H_
#define SP_ABI_H_

#include <stddef.h>

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define SP_ABI_VERSION 1
#define SP_MAX_ITERS 64

enum {
    SP_OK = 0,
    SP_ERR_INVALID = -1,     /* bad argument (size, pointer, configuration) */
    SP_ERR_CUDA = -2,        /* a CUDA runtime/driver call failed */
    SP_ERR_NOMEM = -3,       /* device allocation failed */
    SP_ERR_UNSUPPORTED = -4, /* not available on this device / build */
    SP_ERR_TIMEOUT = -5,     /* a bounded in-kernel wait gave up (device error word set) */
    SP_ERR_NONFINITE = -6,   /* a Parareal defect became NaN/Inf */
    SP_ERR_STATE = -7        /* call out of order */
};

enum { SP_F64 = 0, SP_F32 = 1 };
enum { SP_COARSE_EULER = 0, SP_COARSE_RK4 = 1 };
enum { SP_TOL_NONE = 0, SP_TOL_DEFECT = 1, SP_TOL_REFERENCE = 2 };

/* PDE parameters: the arguments of Convection::Convection (Convection.h:25)
 * plus the UPWINDADVECTION build switch (CMakeLists.txt:101-105; default on). */
typedef struct {
    int ni, nj, nk;
    double dx, nu0, nufreq, cx, cy, cz;
    int upwind;
} sp_params;

/* Geometry of a field in device memory (element counts). */
typedef struct {
    int ni, nj, nk;
    int lx;            /* columns left of interior i=0 (16 bytes); the halo is the last 2 of them */
    int elem_size;     /* 8 (SP_F64) or 4 (SP_F32) */
    long long px;      /* row pitch (multiple of 32 elements) */
    long long py;      /* rows per plane = nj + 4 */
    long long pz;      /* planes = nk + 4 */
    long long plane;   /* px * py */
    long long origin;  /* offset of interior (0,0,0) = 2*plane + 2*px + lx */
    long long total;   /* elements of one field = plane * pz (a multiple of 32) */
} sp_layout;

/* ---- fields -------------------------------------------------------------- */
int sp_field_layout(int ni, int nj, int nk, int precision, sp_layout* out);

/* ---- propagator: class Convection ----------------------------------------- */
typedef struct sp_convection sp_convection;

/* Convection::Convection (Convection.h:25, Convection.cpp:131-143).  Allocates
 * the propagator's internal work fields on `device` (the reference allocates
 * qInternal_, k1_..k4_, Convection.cpp:159-163). */
int sp_convection_create(const sp_params* p, int device, sp_convection** out);
/* Convection::~Convection (Convection.cpp:145-151). */
int sp_convection_destroy(sp_convection* h);
/* Work is enqueued on this CUDA stream (cudaStream_t; NULL = the handle's own). */
int sp_convection_set_stream(sp_convection* h, void* stream);
/* Waits for the handle's stream and checks the device error word. */
int sp_convection_synchronize(sp_convection* h);

/* Convection::DoRK4 (Convection.h:44-45, Convection.cpp:292-303): `timesteps`
 * RK4 steps from tStart; step 0 reads `in`, later steps run in place on `out`;
 * step i uses nu(tStart + i*dt) (Convection.h:81-84).  timesteps == 0 leaves
 * `out` untouched.  `in` may alias `out`.  FP64 fields. */
int sp_do_rk4(sp_convection* h, const double* in, double* out, double tStart, double dt, int timesteps);
/* Convection::DoEuler (Convection.h:63-64, Convection.cpp:305-316): explicit
 * Euler with the RHS2 stencil (first-order upwind advection when upwind). */
int sp_do_euler(sp_convection* h, const double* in, double* out, double tStart, double dt, int timesteps);
/* Convection::DoRK4Timestep / DoEulerTimestep (Convection.h:69-75). */
int sp_do_rk4_timestep(sp_convection* h, const double* in, double* out, double t, double dt);
int sp_do_euler_timestep(sp_convection* h, const double* in, double* out, double t, double dt);
/* FP32 variants of DoRK4 / DoEuler (the coarse propagator precision). */
int sp_do_rk4_f32(sp_convection* h, const float* in, float* out, double tStart, double dt, int timesteps);
int sp_do_euler_f32(sp_convection* h, const float* in, float* out, double tStart, double dt, int timesteps);

/* Periodicity<T>::Apply (Periodicity.h:60-66, Periodicity.cu:146-214): fills
 * the 2-cell halo of a field from its interior, in place. */
int sp_periodicity_apply(sp_convection* h, void* field, int precision);

/* Dense <-> field copies (fillQ/SynchronizeDevice and SynchronizeHost of the
 * reference's drivers, src/Parareal/main.cpp:212-215).  `dense_on_host` != 0:
 * `dense` is host memory (pinned memory gives full copy bandwidth).  Import
 * fills the halo. */
int sp_field_import(sp_convection* h, const void* dense, void* field, int precision, int dense_on_host);
int sp_field_export(sp_convection* h, const void* field, void* dense, int precision, int dense_on_host);

/* Host-buffer form of DoRK4 for callers without device memory management:
 * dense FP64 host arrays in and out; the host->device copy, the steps and the
 * device->host copy run in one call (the reference's fillQ ->
 * SynchronizeDevice -> DoRK4 -> SynchronizeHost sequence). */
int sp_do_rk4_host(sp_convection* h, const double* in_host, double* out_host, double tStart, double dt,
                   int timesteps);

/* Relative errors of two FP64 fields over the interior (computed on the GPU):
 * max|a-b| / max|a| (computeErrorReference, src/Parareal/main.cpp:98-139) and
 * ||a-b||_2 / ||b||_2. */
int sp_field_errors(sp_convection* h, const double* a, const double* b, double* err_max, double* err_l2);

/* ---- Parareal driver: class Parareal --------------------------------------- */
typedef struct {
    double endTime;
    int timeSlices;        /* P: the reference's MPI communicator size (RuntimeConfiguration.cpp:15) */
    int timeStepsFine;     /* totals; rounded up to a multiple of P (RuntimeConfiguration.cpp:133-151) */
    int timeStepsCoarse;
    int kmax;              /* maximum number of iterations (Parareal.h:116) */
    int async;             /* time sequence of Parareal.h:119-124 (matters only when nufreq != 0) */
    int coarse_scheme;     /* SP_COARSE_EULER (the reference's DoEuler) or SP_COARSE_RK4 */
    int coarse_precision;  /* SP_F64 or SP_F32 */
    int tol_kind;          /* SP_TOL_NONE: run kmax iterations, as the reference does */
    double tol;            /* stop once the chosen relative L2 quantity is below tol */
    int skip_converged;    /* 1: after iteration k, slices < k are exact; skip their fine runs */
    int coarse_delta;      /* 0: U = G(new) + F(old) - G(old), the reference's UpdateStage
                              (Parareal.h:32-33); 1: U = F(old) + G(new - old), equal for this
                              linear G, with G applied to the FP64 increment (use with FP32 G) */
    int first_slice;       /* slice window of this handle: slices [first_slice, first_slice + */
    int slice_count;       /* slice_count) of the timeSlices; 0 = all (one GPU runs everything) */
} sp_parareal_cfg;

typedef struct {
    int iterations;
    int tsFine, tsCoarse;          /* steps per slice after rounding */
    double dtFine, dtCoarse, timeSliceSize;
    double defect[SP_MAX_ITERS];   /* max over slices of ||U^{k+1}-U^k||_2/||U^{k+1}||_2 at slice ends */
    double err_l2[SP_MAX_ITERS];   /* last slice vs `reference` (if given), relative L2 */
    double err_max[SP_MAX_ITERS];  /* same, max-norm relative as in main.cpp:98-139 */
    double seconds;                /* device time of DoParallel (CUDA events) */
    double seconds_fine, seconds_coarse;
    long long fine_cell_updates;   /* cell-updates executed by F */
} sp_parareal_report;

typedef struct sp_parareal sp_parareal;

/* Parareal::Parareal (Parareal.h:48-108): binds the propagator, derives the
 * step counts and allocates every slice's state on the propagator's device. */
int sp_parareal_create(sp_convection* prop, const sp_parareal_cfg* cfg, sp_parareal** out);
int sp_parareal_destroy(sp_parareal* pr);
/* Parareal::DoParallel (Parareal.h:110-171), all P slices on one GPU: fine
 * runs of all slices batched per RK stage, coarse sweep slice by slice, the
 * correction U = G(new) + F(old) - G(old) fused with the defect norms.
 * `initial` and `solution` are FP64 fields; `reference` (may be NULL) is the
 * serial fine solution used for err_l2/err_max and for SP_TOL_REFERENCE.
 * All iterations run in one CUDA-graph launch: a conditional WHILE node repeats
 * the iteration, and a kernel at its end evaluates the defect (and the error
 * against `reference`) and decides on the device whether to go on (kmax, the
 * tolerance, a non-finite defect); the host synchronises once, at the end.  The
 * reference's loop is the same with a fixed kmax (Parareal.h:116). */
int sp_parareal_do_parallel(sp_parareal* pr, const double* initial, double* solution,
                            const double* reference, sp_parareal_report* report);
/* Measurement switch, no counterpart in the reference: host_loop = 1 runs
 * DoParallel as one graph launch per iteration with the stopping test on the
 * host (a device-to-host copy and a synchronisation per iteration); 0 (the
 * default) as one launch for all iterations.  Both give identical fields. */
int sp_parareal_set_host_loop(sp_parareal* pr, int host_loop);
/* Parareal::DoSerial (Parareal.h:250-253): DoRK4(initial, solution, 0, dtF, tsF*P). */
int sp_parareal_do_serial(sp_parareal* pr, const double* initial, double* solution);

/* Many independent Parareal solves at once (grids, parameters, slice counts and
 * step counts may all differ; all handles on one device).  Each instance's
 * iteration (batched fine sweep + coarse sweep) is a child graph; the children
 * run concurrently inside one conditional WHILE node, so the predictors
 * aside the whole run is one graph launch; converged instances are gated off
 * on the device.  This replaces running the reference's MPI job once per
 * instance.
 * run: initial[i], solution[i] (and reference[i], may be NULL) are FP64 fields of
 * instance i; reports[i] (may be NULL) as for sp_parareal_do_parallel; *seconds
 * gets the device time of the whole run. */
typedef struct sp_parareal_batch sp_parareal_batch;
int sp_parareal_batch_create(sp_parareal* const* instances, int n, sp_parareal_batch** out);
int sp_parareal_batch_destroy(sp_parareal_batch* b);
int sp_parareal_batch_run(sp_parareal_batch* b, const double* const* initial, double* const* solution,
                          const double* const* reference, sp_parareal_report* reports, double* seconds);
/* As sp_parareal_set_host_loop, for a batch: 0 (default) runs every iteration of
 * every instance in one graph launch (a conditional WHILE node around the
 * instances' iteration graphs; instances that are done are gated off on the
 * device), 1 one launch and one host synchronisation per iteration. */
int sp_parareal_batch_set_host_loop(sp_parareal_batch* b, int host_loop);

/* Slice-window steps for a Parareal spread over several GPUs (the reference's
 * one-rank-per-slice MPI ring, Parareal.h:110-171, with one rank per slice
 * window).  Per iteration k each window runs window_fine, then -- after the
 * previous window's window_coarse -- window_coarse with that window's last
 * slice result as `u_first_new` (NULL for the window holding slice 0), and
 * passes its own `q_last` on.  window_begin computes the window's predictor
 * (from t = 0, as every reference rank does).  `defect` (may be NULL) gets
 * the window's max relative L2 change of its slice results (synchronises). */
int sp_parareal_window_begin(sp_parareal* pr, const double* initial);
int sp_parareal_window_fine(sp_parareal* pr, int k);
int sp_parareal_window_coarse(sp_parareal* pr, int k, const double* u_first_new, double* q_last, double* defect);

/* ---- adjoint ---------------------------------------------------------------- */
/* Gradient of J = 0.5*||q_n - q_target||^2 through n FP64 RK4 steps (DoRK4
 * from tStart with step dt) with respect to q0, nu0 and (cx, cy, cz).
 * Checkpoints every `checkpoint_every` steps (0 = about sqrt(n)) and
 * recomputes in between.  lambda_n (may be NULL): use this dJ/dq_n instead of
 * q_n - q_target (then q_target may be NULL and *J is not computed).
 * grad_q0 and lambda_n are FP64 fields; grad_par gets 4 doubles. */
int sp_adjoint_rk4(sp_convection* h, const double* q0, const double* q_target, const double* lambda_n,
                   double tStart, double dt, int n, int checkpoint_every, double* J, double* grad_q0,
                   double* grad_par);

/* ---- allocation-free propagation ---------------------------------------------- */
/* No counterpart in the reference: an extra entry point of this library.
 * DoRK4 (same stepping and result as sp_do_rk4) for callers that cannot call
 * cudaMalloc -- e.g. code running inside a process whose GPU memory belongs
 * to another allocator or is fully reserved up front, or a plugin that may
 * only touch the buffers it is given.  It needs no handle and allocates
 * nothing: the three RK4 work fields live in a device array built into the
 * library, SP_NOALLOC_SCRATCH_BYTES on every GPU that loads it, held until the
 * process exits.  Grids whose three FP64 work fields do not fit (beyond about
 * 80^3) are rejected with SP_ERR_INVALID.  `in`/`out` are FP64 fields in the
 * sp_field_layout geometry on the current device; the call runs on `stream`
 * (NULL = legacy default stream) and returns when the steps are done: each
 * call synchronizes `stream` to read back the error word of its bounded
 * in-kernel waits (SP_ERR_TIMEOUT).  The first call on each device looks up
 * the array's device address and sets the kernels' shared-memory limits; make
 * that first call before any stream capture.  A first call that fails leaves
 * nothing behind: the next call on that device sets up again.  GPUs older
 * than sm_100 are rejected with SP_ERR_UNSUPPORTED, as by
 * sp_convection_create.  All calls share the one array: calls whose GPU work
 * overlaps (other streams, other host threads) race on it. */
#define SP_NOALLOC_SCRATCH_BYTES (16u << 20)
int sp_do_rk4_noalloc(const sp_params* p, const double* in, double* out, double tStart, double dt, int timesteps,
                      void* stream);

/* ---- misc ------------------------------------------------------------------- */
const char* sp_last_error(void);
int sp_abi_version(void);
/* Kernel launches issued by this process so far (all handles). */
long long sp_launch_count(void);
/* Launch shape in use for a grid / batch and stage kernel `op` (0..3 = RK4 stages
 * S1..S4, 4 = Euler): tile rows ty, z-chunk, kernel kind (0 direct loads, 1
 * TMA/mbarrier pipeline).  op 9 and 10: the fused stage pairs 1+2 and 3+4 of
 * FP64 RK4 steps: tile rows, planes per CTA (0 = one range per resident CTA),
 * kind 2 when RK4 steps run as fused pairs (4: on 32-column tiles), else 0.
 * op 11: kind 3 when FP64 RK4 propagations run cluster-resident on z-slabs
 * (sp_set_tune kind 3), 5 on (y,z) blocks (kind 5), else 0. */
int sp_tuned_config(sp_convection* h, int precision, int batch, int op, int* ty, int* zchunk, int* kind);
/* Runs the autotuner for this handle's grid at `batch` fields and precision: every
 * stage kernel gets the fastest of its candidate launch shapes, and FP64 RK4
 * steps run as fused pairs when those are more than 2 % faster than the four
 * stages: for batch 1 as timed through sp_do_rk4 (a graph chunk of 50 steps on
 * scratch fields), for larger batches over four consecutive batched steps, each
 * path timed after 0.4 s of running back to back (at the clocks it sustains
 * under the GPU's power cap).  The pairs' shapes are chosen per pair by
 * isolated timing, then compared, in the same sustained way, with both pairs
 * on their best 32 x 16 tiles, which are kept unless more than 1 % slower
 * (they move fewer DRAM bytes, so they hold a higher clock under the cap).
 * Small FP64 fields then take a cluster-resident path (kind 3 or 5 of
 * sp_set_tune) when it is faster.  Takes about 1-3 s. */
int sp_autotune(sp_convection* h, int precision, int batch);
/* Test of the error path of the bounded in-kernel waits: runs one kernel whose
 * wait can never complete and gives up after limit_ms (<= 2000); returns
 * SP_ERR_TIMEOUT, as any kernel of the library would after a wait expires,
 * and leaves the handle usable.  No counterpart in the reference (which has
 * no bounded waits). */
int sp_selftest_wait_timeout(sp_convection* h, double limit_ms);
/* Store-bounds checking, the stand-in for a memory sanitizer: in the library
 * built with -DSP_BOUNDS_CHECK=1 (libstencilparareal_checked.so) every global
 * store of the stencil-producing kernels (stage, fused-pair and widening
 * kernels) is tested against its output allocation and skipped, not made, when
 * it falls outside.  *checked = 1 in that build, 0 otherwise; *count = such
 * stores on the current device since the previous call (then reset), after
 * waiting for the device.  No counterpart in the reference. */
int sp_store_violations(int* checked, long long* count);
/* Median duration in ms of each kernel of an FP64 RK4 step, timed with CUDA
 * events around every launch on the handle's stream over `reps` steps (after
 * one untimed step; all steps enqueued before one synchronisation) run on a
 * copy of `field` (which is left unchanged).  path 0: the kernels the handle's
 * tune runs, 1: the four stage kernels (tuned shapes), 2: the fused pairs.
 * *count = 2 (ms[0..1]: pairs 1+2, 3+4) or 4 (ms[0..3]: stages S1..S4).
 * Measurement support, no counterpart in the reference. */
int sp_kernel_times(sp_convection* h, const double* field, double dt, int reps, int path, float* ms, int* count);
/* Forces one launch shape for a precision and batch.  kind 0 or 1: every
 * single-stage kernel, ty in {4,8,16}, zchunk >= 1, RK4 steps unfused.  kind 2
 * (FP64): RK4 steps as fused pairs with ty in {8,16} and zchunk planes per CTA
 * (0 = automatic) on tiles of 64 columns; kind 4 the same on tiles of 32 x 16
 * cells (ty = 16; no wasted columns on grids such as 96^3).
 * kind 3 (FP64, small fields): every RK4 step of a DoRK4
 * call (or of a Parareal fine sweep) in one launch, each field held in the
 * shared memory of a thread-block cluster (ty and zchunk unused; needs an even
 * ni, at most 2048 cells per plane and nk = C x {2,3,4} with 2 <= C <= 16):
 * CTA c of the cluster holds planes of the field (z-slabs).  kind 5 (FP64,
 * small fields): the same with CTA (ry, rz) holding a block of nj/cy rows and
 * nk/cz planes, cy, cz >= 2, cy x cz <= 16, each block at least 2 x 2: it sends
 * a stage's boundary values to four neighbours, half as many values as the
 * z-slabs at 32^3 on 16 CTAs. */
int sp_set_tune(sp_convection* h, int precision, int batch, int ty, int zchunk, int kind);

#ifdef __cplusplus
}
#endif

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#endif /* SP_ABI_H_ */
