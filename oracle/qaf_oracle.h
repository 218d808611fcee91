/*
 * qaf_oracle.h — FP64 host oracle of the reference's pseudo-spectral
 * active-nematic solver. TEST INFRASTRUCTURE ONLY: the tests, smoke() and
 * bench.py's CPU-baseline leg call it as the checker; the product never does.
 *
 * It restates, operation by operation, the reference's algorithm:
 *   wave numbers and 2/3 mask      Basic/Mesh.cuh:6-46
 *   FwdTrans / BwdTrans            FldOp/QFldfuncs.cuh:8-55
 *   derivatives, velocity          FldOp/QFldfuncs.cuh:165-224
 *   IF factors, nonlinear terms    InertialFriction/friction/Qsolver.cuh:20-322
 *   IF-RK4 stages                  TimeIntegration/RK4.cuh:12-74
 *   IF-RK2 / IF-Euler stages       TimeIntegration/IFRK2.cuh:16-51, IFE.cuh:15-25
 *   step order, dealias placement  InertialFriction/friction/friction.cu:212-259
 *   energy, energy spectrum        InertialFriction/post_process/postprocess.cu:54-65,
 *                                  EnergySpec.cu:81-96
 * with its own mixed-radix FFT (twiddles from long-double cosl/sinl of exact
 * rational angles) in place of cuFFT.
 *
 * Layouts are the reference's: physical index i + j*nx, spectral index
 * i + j*(nx/2+1), complex values as interleaved (re, im) doubles.
 *
 * C2R convention: a spectrum that is not Hermitian in the kx = 0 and
 * kx = nx/2 columns is transformed as if those two columns were replaced by
 * their Hermitian parts (equivalently: column complex IDFT, then a row C2R
 * that uses only the real parts of the row's DC and Nyquist terms).
 */
#ifndef QAF_ORACLE_H
#define QAF_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int nx, ny;
    double lx, ly;
    double re, er, rf, lambda;
    double alpha;          /* constant activity Ra, used when no field is given */
    double dt;
    double q_lin;          /* L_Q = -k^2 + q_lin (1.0 in the friction solver) */
    int advect_omega;      /* 1: keep -div(u w) in N_w (friction); 0: drop it */
    int emulate_symmetry;  /* 1: BwdTrans symmetrises its input's kx=0 column in place */
    int no_dealias;        /* 1: steps skip the 2/3 truncation (couple.cu:179-215); 2: truncate w only
                              (dealias/couple.cu:226-229) */
} oracle_params;

enum { ORACLE_IFE = 0, ORACLE_IFRK2 = 1, ORACLE_IFRK4 = 2 };

/* wave-number tables and the 2/3 mask, nxh*ny doubles each (any may be NULL) */
int oracle_tables(const oracle_params* p, double* kx, double* ky, double* k2, double* cutoff);

/* unnormalised R2C of a physical field (FwdTrans) */
int oracle_fwd(int nx, int ny, const double* phys, double* spec);
/* C2R with the 1/(nx*ny) scaling (BwdTrans); spec is not modified */
int oracle_bwd(int nx, int ny, const double* spec, double* phys);
/* the reference's BwdTrans including its in-place symmetrisation of spec */
int oracle_bwd_mutating(int nx, int ny, double* spec, double* phys);

int oracle_xderiv(const oracle_params* p, const double* in, double* out);
int oracle_yderiv(const oracle_params* p, const double* in, double* out);
int oracle_laplacian(const oracle_params* p, const double* in, double* out);
int oracle_vel(const oracle_params* p, const double* w, double* u, double* v);
int oracle_dealias(const oracle_params* p, double* spec);

/* IF tables: which = 0 (w: exp(dt*(-k^2-Rf)/Re)), 1 (Q: exp(dt*(-k^2+q_lin))) */
int oracle_if_tables(const oracle_params* p, int which, double dt, double* IF, double* IFh);

/* Nonlinear right-hand sides of (w, r1, r2) evaluated at the given spectra:
 * curr_func + wnonl_func + r1nonl_func + r2nonl_func. The inputs are copied.
 * alpha_field: nx*ny physical activity, or NULL for the constant p->alpha.
 * phys_out (optional, 9*nx*ny): w, r1, r2, u, v, S, p11, p12, p21 physical. */
int oracle_nonlinear(const oracle_params* p, const double* alpha_field,
                     const double* w, const double* r1, const double* r2,
                     double* wn, double* r1n, double* r2n, double* phys_out);

/* nsteps full steps of the chosen integrator on the spectral state, in place,
 * each ending with dealias (friction.cu:253-259). */
int oracle_step(const oracle_params* p, int integrator, const double* alpha_field,
                double* w, double* r1, double* r2, int nsteps);

/* Diagnostics of a spectral state:
 *   energy    = sum 0.5*(u^2+v^2) dx dy / (Lx Ly)     (postprocess.cu:54-65,158-161)
 *   enstrophy = 0.5 * mean(w^2)
 *   spectrum[s], s < nshells: shell sum of |u^|^2+|v^|^2 over |k| in [k_s, k_s + dk),
 *     k_0 = 0, k_{s+1} = k_s + dk (accumulated), dk = 2 pi / Lx, normalised by 2 dk nx^2 ny^2   (EnergySpec.cu:81-96),
 *     where u^, v^ = vel_func(FwdTrans(BwdTrans(w))), as the post-processor
 *     builds them from a physical vorticity snapshot (EnergySpec.cu:180-186). */
int oracle_diagnostics(const oracle_params* p, const double* w, double* energy,
                       double* enstrophy, double* spectrum, int nshells);

/* IF-RK4 steps with the tangent-linear model (the reference gradient of the
 * discrete adjoint): (w, r1, r2) advance as in oracle_step and (dw, dr1, dr2)
 * as their derivative along the initial tangent and the activity tangent
 * dalpha_field (NULL: zero). loss = mean enstrophy (0.5 mean(w^2)) of the
 * states after the last loss_window steps, dloss its directional derivative. */
int oracle_step_tlm(const oracle_params* p, const double* alpha_field, const double* dalpha_field,
                    double* w, double* r1, double* r2, double* dw, double* dr1, double* dr2,
                    int nsteps, int loss_window, double* loss, double* dloss);

/* the seeded random-Q initial state of include/qaf_init.h (for checking the
 * numpy restatement of the generator) */
void oracle_random_q_init(unsigned long long seed, int nx, int ny, double lo, double hi,
                          double* w, double* r1, double* r2);
/* the coupled-run initial state of include/qaf_init.h on an n x n grid of side L */
void oracle_couple_init(unsigned long long seed, int n, double L, double amp, double* w, double* r1, double* r2);

#ifdef __cplusplus
}
#endif
#endif
