/*
 * sp_oracle.h -- CPU oracle for the advection-diffusion propagator and the
 * Parareal driver.
 *
 * TEST INFRASTRUCTURE ONLY.  This library restates, on the CPU and in plain
 * C++/OpenMP, the algorithm of the reference's FP64 OpenMP path
 * (andyspiros/StencilParareal):
 *   - stencils        src/Convection/ConvectionFunctions.h:4-167
 *   - stage formulas  src/Convection/Convection.cpp:30-127
 *   - time stepping   src/Convection/Convection.cpp:292-392
 *   - periodic halo   src/Communication/Periodicity.cpp:10-135
 *   - Parareal loop   src/Parareal/Parareal.h:110-171,250-253
 *   - step rounding   src/Parareal/RuntimeConfiguration.cpp:133-151
 *   - error metrics   src/Parareal/main.cpp:98-139,
 *                     src/Convection/ConvectionSolution.h:8-103
 * It is used only by the test-suite (as the checker), by the smoke check and
 * by the benchmark's CPU-baseline leg.  The product library never links it.
 *
 * Dense array layout used by every entry point below: interior cells only,
 * i fastest: element (i,j,k) lives at index (k*nj + j)*ni + i, i.e. a C array
 * of shape [nk][nj][ni].  x = (i+1/2)/ni pairs with i, y with j, z with k.
 * Internally the oracle uses the reference's OpenMP storage (JIK order,
 * k contiguous, 2-cell halo) and its separate halo / RHS / Euler / RK passes.
 */
#ifndef SP_ORACLE_H_
#define SP_ORACLE_H_

#ifdef __cplusplus
extern "C" {
#endif

/* PDE parameters, as passed to Convection::Convection (Convection.h:25). */
typedef struct {
    int ni, nj, nk;
    double dx, nu0, nufreq, cx, cy, cz;
    int upwind;        /* 1: Advection2 is first-order upwind (UPWINDADVECTION, the reference default) */
} orc_params;

/* Coarse propagator choices of the Parareal oracle. */
enum {
    ORC_COARSE_EULER_F64 = 0,  /* reference: DoEuler, RHS2, FP64 */
    ORC_COARSE_RK4_F64   = 1,
    ORC_COARSE_RK4_F32   = 2,
    ORC_COARSE_EULER_F32 = 3
};

typedef struct {
    double endTime;
    int timeSlices;
    int timeStepsFine;     /* totals before rounding up to a multiple of timeSlices */
    int timeStepsCoarse;
    int kmax;
    int async;             /* 1: split first fine step as in Parareal.h:119-124 */
    int coarse;            /* ORC_COARSE_* */
    int coarse_delta;      /* 0: U = G(new) + F(old) - G(old) as Parareal.h:32-33;
                              1: U = F(old) + G(new - old) (same value for this linear G) */
} orc_parareal_cfg;

/* Number of OpenMP threads used by the oracle (0 = OpenMP default). */
void orc_set_threads(int n);
int orc_get_threads(void);

/* Convection::DoRK4 / DoEuler (Convection.cpp:292-316): n steps from tStart.
 * n == 0 leaves out untouched. in and out may alias. */
int orc_rk4(const orc_params* p, const double* in, double* out, double tStart, double dt, int n);
int orc_euler(const orc_params* p, const double* in, double* out, double tStart, double dt, int n);
/* Same sequencing computed entirely in FP32 (coarse-propagator variants). */
int orc_rk4_f32(const orc_params* p, const float* in, float* out, double tStart, double dt, int n);
int orc_euler_f32(const orc_params* p, const float* in, float* out, double tStart, double dt, int n);

/* One evaluation of the right-hand side R4 (RHS4Stage) or R2 (RHS2Stage) at time t. */
int orc_rhs4(const orc_params* p, const double* q, double* k, double t);
int orc_rhs2(const orc_params* p, const double* q, double* k, double t);

/* Periodicity::Apply on a halo-padded JIK array, exposed for the halo test:
 * field has (ni+4)*(nj+4)*(nk+4) doubles, index ((j+2)*(ni+4)+(i+2))*(nk+4)+(k+2). */
int orc_periodicity_jik(int ni, int nj, int nk, double* field);

/* RuntimeConfiguration rounding and derived values (RuntimeConfiguration.cpp:133-151,
 * RuntimeConfiguration.h:54-101).  out: [tsFineTotal, tsCoarseTotal, tsFinePerSlice,
 * tsCoarsePerSlice] and dout: [dtFine, dtCoarse, timeSliceSize]. */
int orc_parareal_derived(const orc_parareal_cfg* c, int out[4], double dout[3]);

/* Serial restatement of Parareal::DoSerial + DoParallel (Parareal.h:110-171,250-253).
 * q0: initial field.  q_out: last slice's result after kmax iterations.
 * q_serial (may be NULL): serial fine solution DoRK4(q0, ., 0, dtF, tsF*P).
 * err_max[k], err_l2[k] (may be NULL): after iteration k+1, the max-norm relative
 * error as in main.cpp:98-139 and the relative L2 error, both of the last slice's
 * result against the serial fine solution. */
int orc_parareal(const orc_params* p, const orc_parareal_cfg* c, const double* q0,
                 double* q_out, double* q_serial, double* err_max, double* err_l2);

/* orc_parareal with two more outputs (each may be NULL): defect[k] = max over
 * slices r of ||Q_r^{k+1} - Q_r^k||_2 / ||Q_r^{k+1}||_2, the relative change of
 * every slice's end value in iteration k+1 (Q_r^0: the predictor's slice-end
 * values), and q_iters[k*N .. (k+1)*N) = the last slice's result after
 * iteration k+1 as a dense array (N = ni*nj*nk). */
int orc_parareal_ex(const orc_params* p, const orc_parareal_cfg* c, const double* q0,
                    double* q_out, double* q_serial, double* err_max, double* err_l2,
                    double* defect, double* q_iters);

/* A propagator with its fields allocated once, as the reference's drivers hold
 * a Convection object and its fields across calls (Convection.cpp:131-143,
 * src/Parareal/main.cpp:187-189, timed steps only at main.cpp:218-222):
 * create loads `in`; every run performs DoRK4(in, out, tStart, dt, n) on the
 * held fields; result copies `out` into a dense array. */
typedef struct orc_rk4_session orc_rk4_session;
orc_rk4_session* orc_rk4_session_create(const orc_params* p, const double* in);
int orc_rk4_session_run(orc_rk4_session* s, double tStart, double dt, int n);
int orc_rk4_session_result(const orc_rk4_session* s, double* out);
void orc_rk4_session_destroy(orc_rk4_session* s);

/* Discrete adjoint of n FP64 RK4 steps (Convection.cpp:318-370) for
 * J = 0.5*||q_n - q_target||^2.  Returns J in *J; grad_q0 gets dJ/dq0 and
 * grad_par[0..3] = dJ/d(nu0, cx, cy, cz).  Stores every step (small grids only). */
int orc_adjoint_rk4(const orc_params* p, const double* q0, const double* q_target,
                    double tStart, double dt, int n, double* J, double* grad_q0, double* grad_par);

/* exactQ / fillQ (ConvectionSolution.h:8-52) on the unit cube at time t. */
double orc_exactq(double nu0, double nufreq, double cx, double cy, double cz,
                  double x, double y, double z, double t);
int orc_fillq(const orc_params* p, double t, double* q);

/* computeErrorReference (main.cpp:98-139): max|f-r| / max|f|. */
double orc_error_maxrel(const double* f, const double* r, long n);
/* ||f-r||_2 / ||r||_2 */
double orc_error_l2rel(const double* f, const double* r, long n);

#ifdef __cplusplus
}
#endif
#endif
