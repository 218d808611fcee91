/*
 * qaf.h — C ABI of the B200 pseudo-spectral active-nematic solver.
 *
 * Plain C: opaque handles, plain pointers and sizes, no C++ or torch types.
 * Every call returns a qaf_status. Device pointers are CUDA device pointers;
 * `stream` is a cudaStream_t passed as void* (NULL = the legacy default
 * stream, like the reference, which runs everything on it).
 *
 * Precision is a property of the mesh (QAF_F64 = the reference's Qreal =
 * double, QAF_F32 = float); every real/complex pointer passed with a mesh
 * points to that mesh's type (complex = interleaved re, im).
 *
 * Layouts are the reference's (Basic/Mesh.cuh:48-129):
 *   physical field  nx*ny reals, index i + j*nx
 *   spectrum        (nx/2+1)*ny complex, index i + j*(nx/2+1)
 *
 * Each entry point below names the reference interface it replaces
 * (file:line in whpy/nature-control).
 *
 * Scratch: a mesh owns its scratch buffers (as the reference's Mesh owns
 * mesh->spec / mesh->phys, Mesh.cuh:66-77), so calls on one mesh must not
 * overlap in time (the same restriction as the reference's FwdTrans/BwdTrans).
 * Different meshes are independent.
 */
#ifndef QAF_H
#define QAF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    QAF_OK = 0,
    QAF_ERR_INVALID = 1,      /* bad argument (null handle/pointer, bad size, bad enum) */
    QAF_ERR_UNSUPPORTED = 2,  /* valid but not built (e.g. a grid size without kernels) */
    QAF_ERR_CUDA = 3,         /* a CUDA runtime call failed; see qaf_last_error() */
    QAF_ERR_NONFINITE = 4,    /* the state holds Inf/NaN (qaf_check_finite) */
    QAF_ERR_ALLOC = 5         /* device allocation failed */
} qaf_status;

typedef enum { QAF_F32 = 0, QAF_F64 = 1 } qaf_dtype;

/* Integrators: IF-Euler (TimeIntegration/IFE.cuh:15-25), IF-RK2
 * (TimeIntegration/IFRK2.cuh:16-51) and IF-RK4 (TimeIntegration/RK4.cuh:12-74). */
typedef enum { QAF_IFE = 0, QAF_IFRK2 = 1, QAF_IFRK4 = 2 } qaf_integrator;

typedef struct {
    int nx, ny;        /* grid points; each a size qaf_supported accepts (nx != ny allowed) */
    double lx, ly;     /* domain lengths */
    qaf_dtype dtype;
} qaf_mesh_desc;

/* Physical parameters of InertialFriction/friction/Qsolver.cuh and friction.cu:100-105. */
typedef struct {
    double re;          /* Re: w viscosity 1/Re, L_w = (-k^2 - Rf)/Re (wlin_func :20-30) */
    double er;          /* Er: active/elastic stress scale 1/(Er Re) (PiDeriv :154-164) */
    double rf;          /* Rf: friction */
    double lambda;      /* flow-alignment parameter */
    double alpha;       /* constant activity Ra, used when alpha_field is NULL */
    const void* alpha_field;  /* optional physical activity field Ra(x), nx*ny reals on the device */
    double dt;
    double q_lin;       /* L_Q = -k^2 + q_lin (hard-wired 1.0 in r1lin_func/r2lin_func :32-54) */
    int advect_omega;   /* 1: keep -div(u w) in N_w (friction variant); 0: drop it (beginning2) */
    int no_dealias;     /* 0: 2/3 truncation of the state after every step (friction.cu:253-255);
                           1: none, as the coupled runs (UnitTest/TimeIntegration/couple/couple.cu:179-215);
                           2: of w only, as UnitTest/TimeIntegration/dealias/couple.cu:226-229 */
} qaf_params;

typedef struct qaf_mesh qaf_mesh;

/* ---- library ---------------------------------------------------------- */
const char* qaf_version(void);
/* message of the last failing call on this host thread ("" if none) */
const char* qaf_last_error(void);
/* 1 if there are kernels for grid size n (as nx or as ny) in this dtype: powers
 * of two in [16, 1024] and 3 * 2^k in [48, 768] */
int qaf_supported(int n, qaf_dtype dtype);

/* ---- mesh (Basic/Mesh.cuh:48-113; Field :115-129) ---------------------- */
qaf_status qaf_mesh_create(const qaf_mesh_desc* desc, qaf_mesh** out);
qaf_status qaf_mesh_destroy(qaf_mesh* mesh);
/* sizes in bytes of one physical field and one spectrum (physsize/specsize, Mesh.cuh:73-75) */
qaf_status qaf_mesh_sizes(const qaf_mesh* mesh, size_t* phys_bytes, size_t* spec_bytes);
/* device allocation of one field pair, like new Field(mesh) (Mesh.cuh:115-129) */
qaf_status qaf_field_alloc(const qaf_mesh* mesh, void** phys, void** spec);
qaf_status qaf_field_free(void* phys, void* spec);
/* kx, ky, k^2 and the 2/3 mask tables, (nx/2+1)*ny reals each, host memory
 * (waveinit / cutoff_func, Mesh.cuh:6-46); any pointer may be NULL */
qaf_status qaf_mesh_tables(const qaf_mesh* mesh, void* kx, void* ky, void* k2, void* cutoff);

/* ---- transforms (FldOp/QFldfuncs.cuh:45-55) ----------------------------- */
/* FwdTrans: unnormalised R2C, phys -> spec */
qaf_status qaf_fwd_trans(qaf_mesh* mesh, const void* phys, void* spec, void* stream);
/* BwdTrans: C2R with the 1/(nx ny) scaling, spec -> phys. The input is not
 * modified; its kx = 0 and kx = nx/2 columns contribute their Hermitian parts
 * (what the reference's cuFFT C2R does). */
qaf_status qaf_bwd_trans(qaf_mesh* mesh, const void* spec, void* phys, void* stream);
/* symmetry_func (QFldfuncs.cuh:18-44): the in-place kx = 0 symmetrisation that
 * the reference's BwdTrans applies to its input, for callers that rely on it */
qaf_status qaf_symmetrize(qaf_mesh* mesh, void* spec, void* stream);

/* ---- spectral operators (QFldfuncs.cuh:165-224) ------------------------- */
qaf_status qaf_xderiv(qaf_mesh* mesh, const void* in, void* out, void* stream);     /* xDeriv */
qaf_status qaf_yderiv(qaf_mesh* mesh, const void* in, void* out, void* stream);     /* yDeriv */
qaf_status qaf_laplacian(qaf_mesh* mesh, const void* in, void* out, void* stream);  /* Laplacian */
qaf_status qaf_vel(qaf_mesh* mesh, const void* w, void* u, void* v, void* stream);  /* vel_func */
/* dealias (Qsolver.cuh:314-322): spec *= 2/3 mask, in place */
qaf_status qaf_dealias(qaf_mesh* mesh, void* spec, void* stream);

/* ---- IF tables and stage kernels ---------------------------------------- */
/* wlin_func (which = 0) / r1lin_func, r2lin_func (which = 1), Qsolver.cuh:20-54:
 * IF = exp(L dt), IFh = exp(L dt / 2), (nx/2+1)*ny reals each, device memory */
qaf_status qaf_if_tables(qaf_mesh* mesh, const qaf_params* p, int which, void* IF, void* IFh, void* stream);
/* integrate_func0D..4D of RK4.cuh:12-74 (integrator QAF_IFRK4, stage 0..4),
 * IF::IFRK2::integrate_func0D..2D (QAF_IFRK2, stage 0..2) and
 * IF::IFE::integrate_func1D (QAF_IFE, stage 1; curr unused) on reference-layout
 * spectra; `nonl` is unused at stage 0 */
qaf_status qaf_integrate(qaf_mesh* mesh, qaf_integrator integ, int stage, const void* old_spec, void* curr_spec,
                         void* new_spec, const void* nonl_spec, const void* IF, const void* IFh, double dt,
                         void* stream);

/* ---- the hot path -------------------------------------------------------- */
/* Nonlinear right-hand sides N_w, N_r1, N_r2 at the given spectra: the
 * reference's curr_func + wnonl_func + r1nonl_func + r2nonl_func
 * (Qsolver.cuh:166-312), fused. Inputs are not modified. */
qaf_status qaf_nonlinear(qaf_mesh* mesh, const qaf_params* p, const void* w, const void* r1, const void* r2,
                         void* w_nl, void* r1_nl, void* r2_nl, void* stream);
/* nsteps steps of the chosen integrator on the spectral state (w, r1, r2),
 * in place, each ending with dealias and old <- new: the loop of
 * InertialFriction/friction/friction.cu:212-259, fused into two kernels per
 * RK stage. Asynchronous on `stream`. */
qaf_status qaf_step(qaf_mesh* mesh, const qaf_params* p, qaf_integrator integ, void* w, void* r1, void* r2,
                    int nsteps, void* stream);
/* The same with the state and result in HOST memory: copies in, steps, copies
 * out, synchronises. */
qaf_status qaf_step_host(qaf_mesh* mesh, const qaf_params* p, qaf_integrator integ, void* w, void* r1, void* r2,
                         int nsteps);
/* Diagnostics of the last qaf_step on this mesh (its final state), after the
 * stream has been synchronised: out[0] = total energy sum 0.5 (u^2+v^2) dx dy /
 * (Lx Ly) (post_process/postprocess.cu:54-65,158-161), out[1] = enstrophy
 * 0.5 <w^2>. Returns QAF_ERR_NONFINITE if a step produced Inf/NaN. */
qaf_status qaf_last_diagnostics(qaf_mesh* mesh, double out[2]);
/* The same two values without synchronising: enqueued on `stream` (after the
 * steps it follows), written to `out` (2 doubles, pinned host or device
 * memory) when the stream reaches it. Where the device can address `out`
 * (device memory, or page-locked host memory mapped under unified
 * addressing) a kernel stores the values there directly, with no copy in
 * the stream; other memory gets a staged copy. No counterpart in the
 * reference. The non-finite status is left to qaf_last_diagnostics /
 * qaf_check_finite. */
qaf_status qaf_last_diagnostics_async(qaf_mesh* mesh, double* out, void* stream);
/* Synchronises `stream` and reports whether any step since the last call
 * produced a non-finite value (the reference's NaN check, friction.cu:280). */
qaf_status qaf_check_finite(qaf_mesh* mesh, void* stream);

/* ---- resident state -------------------------------------------------------
 * The reference keeps its state on the device for the whole run and touches
 * the host only for periodic dumps (friction.cu:212-282). The same here: load
 * a spectral state into the mesh's own buffers once, advance it as often as
 * needed, store it when a snapshot is wanted. qaf_step = load + advance + store. */
qaf_status qaf_state_load(qaf_mesh* mesh, const void* w, const void* r1, const void* r2, void* stream);
qaf_status qaf_state_advance(qaf_mesh* mesh, const qaf_params* p, qaf_integrator integ, int nsteps, void* stream);
qaf_status qaf_state_store(qaf_mesh* mesh, void* w, void* r1, void* r2, void* stream);
/* Exact checkpoint/restart of the resident state (replaces the reference's
 * CSV dumps, friction.cu:262-278, BasicUtils.cuh:38-50, which round the
 * state): a binary file with the grid, precision, domain, a step counter and
 * the three spectra in the reference layout, bit for bit. restore checks that
 * the file matches the mesh and loads the state (as qaf_state_load). */
qaf_status qaf_state_save(qaf_mesh* mesh, const char* path, uint64_t step, void* stream);
qaf_status qaf_state_restore(qaf_mesh* mesh, const char* path, uint64_t* step, void* stream);
/* Advance the resident state by nsteps steps with CUDA events recorded on
 * `stream` around every row and column kernel; out_ms[0] / out_ms[1] = mean
 * duration of one row / one column kernel, out_ms[2] = their launch count.
 * Synchronises `stream`. (Measurement support for the roofline figures.) */
qaf_status qaf_state_advance_timed(qaf_mesh* mesh, const qaf_params* p, qaf_integrator integ, int nsteps,
                                   double out_ms[3], void* stream);
/* Number of kernels this mesh has launched so far. */
uint64_t qaf_launch_count(const qaf_mesh* mesh);
/* Test hook for the bounded copy waits; no counterpart in the reference
 * (whose only failure check is the NaN test, friction.cu:280). The next
 * fused-step column launch of an RK stage in this process (not the launch
 * that first transforms a loaded state) arms slab `slab` (>= 0) of the
 * copy sequence of its queue item 0 but never issues that copy, and every
 * copy wait of that launch gives up after `polls` (>= 1) tries. The CTA whose
 * wait ran out stops at the next item boundary with no copy in flight, and
 * the step reports QAF_ERR_CUDA through qaf_check_finite /
 * qaf_last_diagnostics. One launch only: the hook clears itself. */
qaf_status qaf_test_lose_copy(int slab, unsigned polls);

/* ---- seeded initial state -------------------------------------------------
 * The reference reads its initial Q from CSV files or fills it with libc
 * rand() (friction.cu:21-41, :164-185). Here: r1, r2 ~ U(lo, hi) from the
 * SplitMix64 stream of include/qaf_init.h (r1 first, then r2, in physical order
 * i + j*nx), w = 0, each transformed with FwdTrans into the given spectra. */
qaf_status qaf_init_random_q(qaf_mesh* mesh, uint64_t seed, double lo, double hi, void* w, void* r1, void* r2,
                             void* stream);

/* ---- diagnostics of a spectral state (post_process/) --------------------- */
/* energy and enstrophy as in qaf_last_diagnostics, and the shell spectrum
 * E(k_s), k_s = s dk, s < nshells, dk = 2 pi / Lx (EnergySpec.cu:81-96),
 * written to host memory; `w` is a device spectrum */
qaf_status qaf_diagnostics(qaf_mesh* mesh, const void* w, double* energy, double* enstrophy, double* spectrum,
                           int nshells, void* stream);

/* ---- ensembles -------------------------------------------------------------
 * No counterpart in the reference (one grid per process, friction.cu): many
 * independent instances of mixed grid size, with their own activity Ra
 * (alpha[k]) and friction Rf (rf[k]) and shared Re, Er, lambda, dt, q_lin,
 * advected with IF-RK4 together. Instances of one size share each row/column
 * launch; a step of all sizes is one CUDA graph launch (built at creation).
 * n[k] are the grid sizes (nx = ny = n[k], see qaf_supported). */
typedef struct qaf_ensemble qaf_ensemble;
qaf_status qaf_ensemble_create(int ninst, const int* n, double lx, double ly, qaf_dtype dtype, const qaf_params* p,
                               const double* alpha, const double* rf, qaf_ensemble** out);
qaf_status qaf_ensemble_destroy(qaf_ensemble* ens);
/* seeded random Q per instance (qaf_init_random_q with seeds[k]) */
qaf_status qaf_ensemble_init_random(qaf_ensemble* ens, const uint64_t* seeds, double lo, double hi, void* stream);
/* spectra of instance k in the reference layout (device pointers) */
qaf_status qaf_ensemble_load(qaf_ensemble* ens, int k, const void* w, const void* r1, const void* r2, void* stream);
qaf_status qaf_ensemble_store(qaf_ensemble* ens, int k, void* w, void* r1, void* r2, void* stream);
qaf_status qaf_ensemble_advance(qaf_ensemble* ens, int nsteps, void* stream);
/* new per-instance activity and friction (host arrays of ninst values), effective from the next
 * step enqueued on `stream`; the values are copied before the call returns */
qaf_status qaf_ensemble_set_controls(qaf_ensemble* ens, const double* alpha, const double* rf, void* stream);
/* synchronises `stream`; out[2k], out[2k+1] = energy, enstrophy of instance k after the last step */
qaf_status qaf_ensemble_diagnostics(qaf_ensemble* ens, double* out, void* stream);

/* ---- launch-shape autotuner --------------------------------------------------
 * No counterpart in the reference. The fused step kernels have alternative
 * launch shapes (FP32, grids 64, 128, 256, 1024: FFT radix per thread, rows per
 * CTA); a library-wide table picks one column and one row shape per (precision,
 * n, batched = more than one instance per launch), used by every launch made
 * after the choice (ensembles: those created after it). Default: the built-in
 * shapes.
 * qaf_autotune: times each shape on `ninst` synthetic instances of n x n, keeps
 *   the fastest, and (cache_path != NULL) records it in a JSON-lines file, one
 *   record per (device, precision, n, batched). choice: "col:<name> row:<name>".
 * qaf_autotune_load: applies the records of a cache file that match this GPU
 *   (or whose device is "*"); records naming unknown shapes are skipped.
 * qaf_set_variant / qaf_variant_choice / qaf_variant_list: set, read and list
 *   the shapes by name ("default" or a listed name). */
qaf_status qaf_autotune(int n, qaf_dtype dtype, int ninst, const char* cache_path, char* choice, int choice_len,
                        double* us_per_step);
qaf_status qaf_autotune_load(const char* cache_path);
qaf_status qaf_autotune_reset(void);
qaf_status qaf_set_variant(int n, qaf_dtype dtype, int batched, const char* col, const char* row);
qaf_status qaf_variant_choice(int n, qaf_dtype dtype, int batched, char* buf, int len);
qaf_status qaf_variant_list(int n, qaf_dtype dtype, char* buf, int len);

/* ---- discrete adjoint (IF-RK4) ---------------------------------------------
 * No counterpart in the reference (it has no gradients): reverse-mode
 * derivatives of `nsteps` IF-RK4 steps (qaf_state_advance) with respect to the
 * initial spectra and the activity field Ra(x). The loss is
 *     L = (1/loss_window) * sum of the enstrophy (as qaf_last_diagnostics) of
 *         the states after the last loss_window steps      (0: no loss term)
 * and/or any function of the final state through its gradient.
 * qaf_adjoint_create: allocates checkpoints every `checkpoint_every` steps and
 *   the recording of one segment (4 * checkpoint_every * 9 physical fields);
 *   borrows `mesh`, whose resident state the calls below overwrite.
 * qaf_adjoint_forward: runs the steps from (w0, r1_0, r2_0) (reference-layout
 *   device spectra) with params p (p->alpha_field must stay valid until the
 *   backward call); optional final state out; *loss on return (synchronises).
 * qaf_adjoint_backward: gwT/gr1T/gr2T = dL/d(final state) or NULL (zero),
 *   gloss = dL/d(loss); writes dL/d(initial spectra) (NULL: skipped) and
 *   dL/dRa(x) (nx*ny reals, NULL: skipped). Gradients of complex entries are
 *   dL/dRe + i dL/dIm. */
typedef struct qaf_adjoint qaf_adjoint;
qaf_status qaf_adjoint_create(qaf_mesh* mesh, int nsteps, int checkpoint_every, int loss_window, qaf_adjoint** out);
qaf_status qaf_adjoint_destroy(qaf_adjoint* adj);
qaf_status qaf_adjoint_forward(qaf_adjoint* adj, const qaf_params* p, const void* w0, const void* r1_0,
                               const void* r2_0, void* wT, void* r1T, void* r2T, double* loss, void* stream);
qaf_status qaf_adjoint_backward(qaf_adjoint* adj, const void* gwT, const void* gr1T, const void* gr2T, double gloss,
                                void* gw0, void* gr1_0, void* gr2_0, void* galpha, void* stream);

/* ---- batched adjoint -----------------------------------------------------------
 * No counterpart in the reference. `ninst` instances of one grid size (n <= 256)
 * sharing the parameters p (fixed at creation) but each with its own initial
 * spectra and activity field, stepped and differentiated together: every stage
 * of the forward, the recompute and the adjoint is one launch for the batch.
 * Arrays hold the instances back to back: spectra [ninst][ny][nx/2+1],
 * activity fields and their gradients [ninst][ny][nx]. losses[k] (host) is
 * instance k's mean enstrophy over the last loss_window states; glosses[k]
 * (host, NULL: zero) its weight in the objective. */
typedef struct qaf_adjoint_batch qaf_adjoint_batch;
qaf_status qaf_adjoint_batch_create(int ninst, int n, double lx, double ly, qaf_dtype dtype, const qaf_params* p,
                                    int nsteps, int checkpoint_every, int loss_window, qaf_adjoint_batch** out);
qaf_status qaf_adjoint_batch_destroy(qaf_adjoint_batch* batch);
qaf_status qaf_adjoint_batch_forward(qaf_adjoint_batch* batch, const void* w0, const void* r1_0, const void* r2_0,
                                     const void* alpha, void* wT, void* r1T, void* r2T, double* losses, void* stream);
qaf_status qaf_adjoint_batch_backward(qaf_adjoint_batch* batch, const void* gwT, const void* gr1T, const void* gr2T,
                                      const double* glosses, void* gw0, void* gr1_0, void* gr2_0, void* galpha,
                                      void* stream);

/* ---- allocation-free step --------------------------------------------------
 * No counterpart in the reference (whose Mesh and Field always cudaMalloc).
 * For callers that cannot allocate device memory when they step — work
 * recorded into a CUDA graph while a stream is being captured, plug-ins whose
 * host owns all device memory, real-time loops that must not allocate once
 * running: the same fused IF-RK step as qaf_step on an n x n grid
 * (n a power of two, 16 <= n <= 128; lx, ly as in qaf_mesh_desc), in place on
 * the device spectra w, r1, r2, with every scratch buffer in one fixed 4 MiB
 * device array inside this library (held by each GPU that loads the library
 * until the process exits). Larger grids are rejected with QAF_ERR_INVALID.
 * The first call on a device looks up that array's address with the device
 * current; make that first call before any stream capture. All calls share the
 * one array: calls whose work overlaps on the GPU (other streams, other host
 * threads) race and must be serialised by the caller. The array keeps the last
 * call's contents; each call rebuilds what it needs. Its twiddles and
 * integrating factors are built on the device (sincospi / exp in double),
 * where qaf_step's come from long-double host tables, so the two agree to
 * rounding (last bits), not bit for bit.
 * The call returns once its work is queued on `stream`, so a kernel failure
 * cannot be in its return value: `status` (NULL: not wanted) is a device or
 * page-locked host word that receives, in stream order after the step, the
 * call's status flags — 0 when all went well, bit 0 a non-finite value in the
 * new state, bit 1 a bounded copy wait that gave up (the state is then not
 * valid). Read it once the stream has reached that point. */
qaf_status qaf_step_noalloc(int n, double lx, double ly, qaf_dtype dtype, const qaf_params* p,
                            qaf_integrator integ, void* w, void* r1, void* r2, int nsteps, void* status,
                            void* stream);

#ifdef __cplusplus
}
#endif
#endif /* QAF_H */
