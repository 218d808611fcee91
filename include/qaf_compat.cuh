// qaf_compat.cuh — the reference's C++/CUDA names over the qaf library, so that
// a driver written against the reference's headers (Mesh.cuh, QFldfuncs.cuh,
// friction/Qsolver.cuh, TimeIntegration/{RK4,IFRK2,IFE}.cuh) compiles and runs
// unchanged against libqaf.
//
//   #include "qaf_compat.cuh"       (instead of the reference's headers)
//   nvcc -I include driver.cu -L nature-control_b200/qaf -lqaf
//
// * Mesh / Field keep the reference's public members (Mesh.cuh:48-129). The
//   mesh's wave-number tables and mask are device arrays filled from the
//   library's tables; the destructors free everything the constructors took.
// * FwdTrans / BwdTrans / xDeriv / yDeriv / Laplacian / vel_func map to the
//   library's transforms and operators (QFldfuncs.cuh:45-224). BwdTrans
//   symmetrises its input's kx = 0 column in place first, as the reference's
//   does (QFldfuncs.cuh:50-55).
// * The kernels that reference drivers launch themselves with <<<grid, block>>>
//   (integrate_func*, dealias, SpecSet, FldSet, S_func, the *lin_func tables,
//   ...) are defined here with the reference's signatures and are compiled in
//   the driver's translation unit; they are thin elementwise kernels.
// * curr_func / wnonl_func / r1nonl_func / r2nonl_func give the same spectra
//   and the same curr physical fields (r1, r2, w, u, v, S) as the reference's;
//   each nonlinear function is one fused evaluation of the library
//   (qaf_nonlinear). The scratch fields the reference leaves filled as a side
//   effect (aux, aux1, p11, p12, p21) are not written.
// * Errors: a failing library call prints its message and calls
//   std::terminate(), as the reference does for cuFFT errors (cudaErr.h:54-61).
//
// Precision: Qreal = double (the reference's only precision) unless
// QAF_COMPAT_FP32 is defined before the include.
//
// The fused path for the whole step loop is qaf_step / qaf_state_advance.
#pragma once

#include <cuComplex.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <exception>
#include <vector>

#include "qaf.h"

#ifdef QAF_COMPAT_FP32
typedef float Qreal;
typedef cuComplex Qcomp;
#define QAF_COMPAT_DTYPE QAF_F32
#else
typedef double Qreal;
typedef cuDoubleComplex Qcomp;
#define QAF_COMPAT_DTYPE QAF_F64
#endif

namespace qaf_compat {

inline void check(qaf_status s, const char* what) {
    if (s != QAF_OK) {
        std::fprintf(stderr, "%s failed (status %d): %s\n", what, (int)s, qaf_last_error());
        std::terminate();
    }
}

__host__ __device__ inline Qcomp cx(Qreal re, Qreal im) {
    Qcomp c;
    c.x = re;
    c.y = im;
    return c;
}
__host__ __device__ inline Qcomp operator+(Qcomp a, Qcomp b) { return cx(a.x + b.x, a.y + b.y); }
__host__ __device__ inline Qcomp operator-(Qcomp a, Qcomp b) { return cx(a.x - b.x, a.y - b.y); }
__host__ __device__ inline Qcomp operator*(Qreal s, Qcomp a) { return cx(s * a.x, s * a.y); }
__host__ __device__ inline Qcomp operator*(Qcomp a, Qreal s) { return cx(a.x * s, a.y * s); }
__host__ __device__ inline Qcomp operator/(Qcomp a, Qreal s) { return cx(a.x / s, a.y / s); }

}  // namespace qaf_compat

using qaf_compat::operator+;
using qaf_compat::operator-;
using qaf_compat::operator*;
using qaf_compat::operator/;

// ---------------------------------------------------------------------------
// Mesh and Field (Mesh.cuh:48-129)
// ---------------------------------------------------------------------------
typedef struct Mesh {
    int Nx, Nxh, Ny;
    Qreal Lx, Ly, dx, dy;
    int specsize, physsize, wavesize;
    int BSZ;
    dim3 dimGridp, dimBlockp, dimGridsp, dimBlocksp;
    Qcomp* spec;
    Qreal* phys;
    Qreal *kx, *ky, *k_squared;
    Qreal* cutoff;
    qaf_mesh* handle;   // the library mesh behind this one

    Mesh(int pNx, int pNy, Qreal pLx, Qreal pLy, int pBSZ)
        : Nx(pNx), Nxh(pNx / 2 + 1), Ny(pNy), Lx(pLx), Ly(pLy), dx(pLx / pNx), dy(pLy / pNy), BSZ(pBSZ) {
        specsize = Nxh * Ny * (int)sizeof(Qcomp);
        physsize = Nx * Ny * (int)sizeof(Qreal);
        wavesize = Nxh * Ny * (int)sizeof(Qreal);
        qaf_mesh_desc d = {Nx, Ny, (double)Lx, (double)Ly, QAF_COMPAT_DTYPE};
        qaf_compat::check(qaf_mesh_create(&d, &handle), "Mesh (qaf_mesh_create)");
        dimGridp = dim3((Nx + BSZ - 1) / BSZ, (Ny + BSZ - 1) / BSZ);
        dimBlockp = dim3(BSZ, BSZ);
        dimGridsp = dim3((Nxh + BSZ - 1) / BSZ, (Ny + BSZ - 1) / BSZ);
        dimBlocksp = dim3(BSZ, BSZ);
        cudaMalloc((void**)&spec, specsize);
        cudaMalloc((void**)&phys, physsize);
        cudaMalloc((void**)&kx, wavesize);
        cudaMalloc((void**)&ky, wavesize);
        cudaMalloc((void**)&k_squared, wavesize);
        cudaMalloc((void**)&cutoff, wavesize);
        std::vector<Qreal> hkx(Nxh * Ny), hky(Nxh * Ny), hk2(Nxh * Ny), hc(Nxh * Ny);
        qaf_compat::check(qaf_mesh_tables(handle, hkx.data(), hky.data(), hk2.data(), hc.data()),
                          "Mesh (qaf_mesh_tables)");
        cudaMemcpy(kx, hkx.data(), wavesize, cudaMemcpyHostToDevice);
        cudaMemcpy(ky, hky.data(), wavesize, cudaMemcpyHostToDevice);
        cudaMemcpy(k_squared, hk2.data(), wavesize, cudaMemcpyHostToDevice);
        cudaMemcpy(cutoff, hc.data(), wavesize, cudaMemcpyHostToDevice);
    }
    ~Mesh() {
        cudaFree(spec); cudaFree(phys);
        cudaFree(kx); cudaFree(ky); cudaFree(k_squared); cudaFree(cutoff);
        qaf_mesh_destroy(handle);
    }
    Mesh(const Mesh&) = delete;
    Mesh& operator=(const Mesh&) = delete;
} Mesh;

typedef struct Field {
    Qcomp* spec;
    Qreal* phys;
    Mesh* mesh;
    explicit Field(Mesh* pmesh) : mesh(pmesh) {
        cudaMalloc((void**)&spec, mesh->specsize);
        cudaMalloc((void**)&phys, mesh->physsize);
    }
    ~Field() { cudaFree(spec); cudaFree(phys); }
    Field(const Field&) = delete;
    Field& operator=(const Field&) = delete;
} Field;

// ---------------------------------------------------------------------------
// transforms and spectral operators (QFldfuncs.cuh:45-224)
// ---------------------------------------------------------------------------
inline void FwdTrans(Qcomp* ft, Qreal* f, Mesh* mesh) {
    qaf_compat::check(qaf_fwd_trans(mesh->handle, f, ft, nullptr), "FwdTrans");
}
inline void BwdTrans(Qreal* f, Qcomp* ft, Mesh* mesh) {
    qaf_compat::check(qaf_symmetrize(mesh->handle, ft, nullptr), "BwdTrans (symmetrise)");
    qaf_compat::check(qaf_bwd_trans(mesh->handle, ft, f, nullptr), "BwdTrans");
}
inline void xDeriv(Qcomp* fx, Qcomp* f, Mesh* mesh) { qaf_compat::check(qaf_xderiv(mesh->handle, f, fx, nullptr), "xDeriv"); }
inline void yDeriv(Qcomp* fy, Qcomp* f, Mesh* mesh) { qaf_compat::check(qaf_yderiv(mesh->handle, f, fy, nullptr), "yDeriv"); }
inline void Laplacian(Qcomp* fL, Qcomp* f, Mesh* mesh) {
    qaf_compat::check(qaf_laplacian(mesh->handle, f, fL, nullptr), "Laplacian");
}
inline void vel_func(Qcomp* w_c, Qcomp* u_c, Qcomp* v_c, Mesh* mesh) {
    qaf_compat::check(qaf_vel(mesh->handle, w_c, u_c, v_c, nullptr), "vel_func");
}

// ---------------------------------------------------------------------------
// elementwise kernels launched by drivers (BSZ x BSZ blocks over the grid)
// ---------------------------------------------------------------------------
#define QAF_COMPAT_IJ(NX, NY)                          \
    const int i = blockIdx.x * BSZ + threadIdx.x;       \
    const int j = blockIdx.y * BSZ + threadIdx.y;       \
    if (i >= (NX) || j >= (NY)) return;                 \
    const int index = i + j * (NX);

__global__ void coeff(Qreal* f, int Nx, int Ny, int BSZ) { QAF_COMPAT_IJ(Nx, Ny) f[index] = f[index] / (Qreal)(Nx * Ny); }
__global__ void FldMul(Qreal* pc, Qreal* pa, Qreal* pb, Qreal C, int Nx, int Ny, int BSZ) {
    QAF_COMPAT_IJ(Nx, Ny) pc[index] = C * pa[index] * pb[index];
}
__global__ void FldAdd(Qreal* pc, Qreal a, Qreal* pa, Qreal b, Qreal* pb, int Nx, int Ny, int BSZ) {
    QAF_COMPAT_IJ(Nx, Ny) pc[index] = a * pa[index] + b * pb[index];
}
__global__ void FldAdd(Qreal* pc, Qreal a, Qreal* pa, Qreal b, int Nx, int Ny, int BSZ) {
    QAF_COMPAT_IJ(Nx, Ny) pc[index] = a * pa[index] + b;
}
__global__ void FldSet(Qreal* pf, Qreal c, int Nx, int Ny, int BSZ) { QAF_COMPAT_IJ(Nx, Ny) pf[index] = c; }
__global__ void FldSet(Qreal* pf, Qreal* c, int Nx, int Ny, int BSZ) { QAF_COMPAT_IJ(Nx, Ny) pf[index] = c[index]; }
__global__ void SpecSet(Qcomp* pa, Qcomp* pb, int Nxh, int Ny, int BSZ) { QAF_COMPAT_IJ(Nxh, Ny) pa[index] = pb[index]; }
__global__ void SpecSet(Qcomp* pa, Qcomp c, int Nxh, int Ny, int BSZ) { QAF_COMPAT_IJ(Nxh, Ny) pa[index] = c; }
__global__ void SpecAdd(Qcomp* spc, Qreal a, Qcomp* spa, Qreal b, Qcomp* spb, int Nxh, int Ny, int BSZ) {
    QAF_COMPAT_IJ(Nxh, Ny) spc[index] = a * spa[index] + b * spb[index];
}
__global__ void SpecMul(Qcomp* spc, Qcomp* spa, Qreal C, int Nxh, int Ny, int BSZ) {
    QAF_COMPAT_IJ(Nxh, Ny) spc[index] = C * spa[index];
}

// integrating factors exp(L dt), exp(L dt / 2) (friction/Qsolver.cuh:20-54)
__global__ void wlin_func(Qreal* IFw, Qreal* IFwh, Qreal* k_squared, Qreal Re, Qreal Rf, Qreal dt, int Nxh, int Ny, int BSZ) {
    QAF_COMPAT_IJ(Nxh, Ny)
    const Qreal L = (Qreal)1.0 / Re * (-k_squared[index] - Rf);
    IFw[index] = exp(L * dt);
    IFwh[index] = exp(L * dt / 2);
}
__global__ void r1lin_func(Qreal* IFr1, Qreal* IFr1h, Qreal* k_squared, Qreal dt, int Nxh, int Ny, int BSZ) {
    QAF_COMPAT_IJ(Nxh, Ny)
    const Qreal L = -k_squared[index] + (Qreal)1.0;
    IFr1[index] = exp(L * dt);
    IFr1h[index] = exp(L * dt / 2);
}
__global__ void r2lin_func(Qreal* IFr2, Qreal* IFr2h, Qreal* k_squared, Qreal dt, int Nxh, int Ny, int BSZ) {
    QAF_COMPAT_IJ(Nxh, Ny)
    const Qreal L = -k_squared[index] + (Qreal)1.0;
    IFr2[index] = exp(L * dt);
    IFr2h[index] = exp(L * dt / 2);
}

// physical-space pieces of the nonlinear terms (friction/Qsolver.cuh:63-94, 154-164, 207-215)
__global__ void S_func(Qreal* S, Qreal* r1, Qreal* r2, int Nx, int Ny, int BSZ) {
    QAF_COMPAT_IJ(Nx, Ny) S[index] = 2 * sqrt(r1[index] * r1[index] + r2[index] * r2[index]);
}
__global__ void Rar(Qreal* rar, const Qreal* r, const Qreal* Ra, int Nx, int Ny, int BSZ) {
    QAF_COMPAT_IJ(Nx, Ny) rar[index] = rar[index] - Ra[index] * r[index];
}
__global__ void single1(Qreal* s1, const Qreal* r, const Qreal* S, Qreal lambda, int Nx, int Ny, int BSZ) {
    QAF_COMPAT_IJ(Nx, Ny) s1[index] = s1[index] + lambda * S[index] * (S[index] * S[index] - 1) * r[index];
}
__global__ void S2r(Qreal* rs, Qreal* r, Qreal* S, int Nx, int Ny, int BSZ) {
    QAF_COMPAT_IJ(Nx, Ny) rs[index] = rs[index] - S[index] * S[index] * r[index];
}
__global__ void PiDeriv(Qcomp* dP, Qcomp* p12, Qcomp* p11, Qcomp* p21, Qreal* kx, Qreal* ky, Qreal Er, Qreal Re, int Nxh,
                        int Ny, int BSZ) {
    QAF_COMPAT_IJ(Nxh, Ny)
    dP[index] = dP[index] + (Qreal)1.0 / (Er * Re) *
                                (-kx[index] * kx[index] * p12[index] + 2 * kx[index] * ky[index] * p11[index] +
                                 ky[index] * ky[index] * p21[index]);
}
__global__ void dealias(Qcomp* ft, Qreal* cutoff, int Nxh, int Ny, int BSZ) {
    QAF_COMPAT_IJ(Nxh, Ny) ft[index] = ft[index] * cutoff[index];
}

// IF-RK4 stages (TimeIntegration/RK4.cuh:12-74)
__global__ void integrate_func0D(Qcomp* old_spec, Qcomp* curr_spec, Qcomp* new_spec, Qreal* IF, Qreal* IFh, int Nxh,
                                 int Ny, int BSZ, Qreal dt) {
    QAF_COMPAT_IJ(Nxh, Ny)
    new_spec[index] = old_spec[index] * IF[index];
    curr_spec[index] = old_spec[index];
}
__global__ void integrate_func1D(Qcomp* old_spec, Qcomp* curr_spec, Qcomp* new_spec, Qcomp* nonl_spec, Qreal* IF,
                                 Qreal* IFh, int Nxh, int Ny, int BSZ, Qreal dt) {
    QAF_COMPAT_IJ(Nxh, Ny)
    const Qcomp an = nonl_spec[index] * dt;
    new_spec[index] = new_spec[index] + (Qreal)(1.0 / 6.0) * IF[index] * an;
    curr_spec[index] = (old_spec[index] + an / 2) * IFh[index];
}
__global__ void integrate_func2D(Qcomp* old_spec, Qcomp* curr_spec, Qcomp* new_spec, Qcomp* nonl_spec, Qreal* IF,
                                 Qreal* IFh, int Nxh, int Ny, int BSZ, Qreal dt) {
    QAF_COMPAT_IJ(Nxh, Ny)
    const Qcomp bn = nonl_spec[index] * dt;
    new_spec[index] = new_spec[index] + (Qreal)(1.0 / 3.0) * IFh[index] * bn;
    curr_spec[index] = old_spec[index] * IFh[index] + bn / 2;
}
__global__ void integrate_func3D(Qcomp* old_spec, Qcomp* curr_spec, Qcomp* new_spec, Qcomp* nonl_spec, Qreal* IF,
                                 Qreal* IFh, int Nxh, int Ny, int BSZ, Qreal dt) {
    QAF_COMPAT_IJ(Nxh, Ny)
    const Qcomp cn = nonl_spec[index] * dt;
    new_spec[index] = new_spec[index] + (Qreal)(1.0 / 3.0) * IFh[index] * cn;
    curr_spec[index] = old_spec[index] * IF[index] + cn * IFh[index];
}
__global__ void integrate_func4D(Qcomp* old_spec, Qcomp* curr_spec, Qcomp* new_spec, Qcomp* nonl_spec, Qreal* IF,
                                 Qreal* IFh, int Nxh, int Ny, int BSZ, Qreal dt) {
    QAF_COMPAT_IJ(Nxh, Ny)
    const Qcomp dn = nonl_spec[index] * dt;
    new_spec[index] = new_spec[index] + (Qreal)(1.0 / 6.0) * dn;
}

namespace IF {
// IF-RK2 (TimeIntegration/IFRK2.cuh:16-51); curr uses the factor passed as IFh
namespace IFRK2 {
__global__ void integrate_func0D(Qcomp* old_spec, Qcomp* curr_spec, Qcomp* new_spec, Qreal* IF, Qreal* IFh, int Nxh,
                                 int Ny, int BSZ, Qreal dt) {
    QAF_COMPAT_IJ(Nxh, Ny)
    new_spec[index] = old_spec[index] * IF[index];
    curr_spec[index] = old_spec[index];
}
__global__ void integrate_func1D(Qcomp* old_spec, Qcomp* curr_spec, Qcomp* new_spec, Qcomp* nonl_spec, Qreal* IF,
                                 Qreal* IFh, int Nxh, int Ny, int BSZ, Qreal dt) {
    QAF_COMPAT_IJ(Nxh, Ny)
    const Qcomp an = nonl_spec[index] * dt;
    new_spec[index] = new_spec[index] + (Qreal)0.5 * IF[index] * an;
    curr_spec[index] = (old_spec[index] + an) * IFh[index];
}
__global__ void integrate_func2D(Qcomp* old_spec, Qcomp* curr_spec, Qcomp* new_spec, Qcomp* nonl_spec, Qreal* IF,
                                 Qreal* IFh, int Nxh, int Ny, int BSZ, Qreal dt) {
    QAF_COMPAT_IJ(Nxh, Ny)
    const Qcomp bn = nonl_spec[index] * dt;
    new_spec[index] = new_spec[index] + (Qreal)0.5 * bn;
}
}  // namespace IFRK2
// IF-Euler (TimeIntegration/IFE.cuh:15-25)
namespace IFE {
__global__ void integrate_func1D(Qcomp* old_spec, Qcomp* new_spec, Qcomp* nonl_spec, Qreal* IF, Qreal* IFh, int Nxh,
                                 int Ny, int BSZ, Qreal dt) {
    QAF_COMPAT_IJ(Nxh, Ny)
    new_spec[index] = (old_spec[index] + nonl_spec[index] * dt) * IF[index];
}
}  // namespace IFE
}  // namespace IF

#undef QAF_COMPAT_IJ

// ---------------------------------------------------------------------------
// the friction solver's nonlinear-term functions (friction/Qsolver.cuh:166-312)
// ---------------------------------------------------------------------------
namespace qaf_compat {
inline qaf_params params(Qreal Re, Qreal Er, Qreal lambda, const Qreal* Ra) {
    qaf_params p;
    p.re = Re; p.er = Er; p.rf = 0; p.lambda = lambda; p.alpha = 0; p.alpha_field = Ra;
    p.dt = 1; p.q_lin = 1; p.advect_omega = 1; p.no_dealias = 0;
    return p;
}
}  // namespace qaf_compat

// curr fields: r1, r2, w to physical space (BwdTrans), S, u^ v^ and u, v
inline void curr_func(Field* r1curr, Field* r2curr, Field* wcurr, Field* u, Field* v, Field* S) {
    Mesh* m = wcurr->mesh;
    BwdTrans(r1curr->phys, r1curr->spec, m);
    BwdTrans(r2curr->phys, r2curr->spec, m);
    BwdTrans(wcurr->phys, wcurr->spec, m);
    S_func<<<m->dimGridp, m->dimBlockp>>>(S->phys, r1curr->phys, r2curr->phys, m->Nx, m->Ny, m->BSZ);
    vel_func(wcurr->spec, u->spec, v->spec, m);
    BwdTrans(u->phys, u->spec, m);
    BwdTrans(v->phys, v->spec, m);
}

// N^_w into wnonl->spec (Ra->phys is the activity field)
inline void wnonl_func(Field* wnonl, Field* wcurr, Field* u, Field* v, Field* r1curr, Field* r2curr, Field* Ra, Field* S,
                       Field* p11, Field* p12, Field* p21, Qreal Re, Qreal Er, Qreal lambda, Field* aux, Field* aux1) {
    const qaf_params p = qaf_compat::params(Re, Er, lambda, Ra->phys);
    qaf_compat::check(qaf_nonlinear(wcurr->mesh->handle, &p, wcurr->spec, r1curr->spec, r2curr->spec, wnonl->spec,
                                    aux->spec, aux1->spec, nullptr),
                      "wnonl_func");
}
// N^_r1 into r1nonl->spec
inline void r1nonl_func(Field* r1nonl, Field* wcurr, Field* u, Field* v, Field* r1curr, Field* r2curr, Field* S,
                        Qreal lambda, Field* aux, Field* aux1) {
    const qaf_params p = qaf_compat::params(1, 1, lambda, nullptr);
    qaf_compat::check(qaf_nonlinear(wcurr->mesh->handle, &p, wcurr->spec, r1curr->spec, r2curr->spec, aux->spec,
                                    r1nonl->spec, aux1->spec, nullptr),
                      "r1nonl_func");
}
// N^_r2 into r2nonl->spec
inline void r2nonl_func(Field* r2nonl, Field* wcurr, Field* u, Field* v, Field* r1curr, Field* r2curr, Field* S,
                        Qreal lambda, Field* aux, Field* aux1) {
    const qaf_params p = qaf_compat::params(1, 1, lambda, nullptr);
    qaf_compat::check(qaf_nonlinear(wcurr->mesh->handle, &p, wcurr->spec, r1curr->spec, r2curr->spec, aux->spec,
                                    aux1->spec, r2nonl->spec, nullptr),
                      "r2nonl_func");
}
