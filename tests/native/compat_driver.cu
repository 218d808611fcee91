// A friction.cu-style driver written against the reference's names
// (include/qaf_compat.cuh): the step loop of InertialFriction/friction/
// friction.cu:212-259 launched kernel by kernel, then the same steps through
// the library's fused path (qaf_step), compared field by field.
//
//   compat_driver <N> <nsteps> <integrator: rk4|rk2|ife> [params: test|friction]
// prints one JSON line {"rel_w": .., "rel_r1": .., "rel_r2": .., "energy": ..}.
// params "friction" takes friction.cu's own settings (friction.cu:100-117:
// lambda 0.1, Rf 0.00075, alpha 0.2, Re = Er = 0.1, dt 0.002, Lx = 33 * 2 pi,
// with its Nx = 512 * 3 / 2 = 768 given as N); "test" (the default) Lx = 16 pi,
// Re = Er = 1, Rf = 0.1, alpha 1, dt 1e-3.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "qaf_compat.cuh"
#include "qaf_init.h"

static double rel_l2(const std::vector<Qcomp>& a, const std::vector<Qcomp>& b) {
    double num = 0, den = 0;
    for (size_t k = 0; k < a.size(); ++k) {
        const double dx = (double)a[k].x - b[k].x, dy = (double)a[k].y - b[k].y;
        num += dx * dx + dy * dy;
        den += (double)b[k].x * b[k].x + (double)b[k].y * b[k].y;
    }
    return den > 0 ? std::sqrt(num / den) : std::sqrt(num);
}

static std::vector<Qcomp> fetch(const Qcomp* d, size_t n) {
    std::vector<Qcomp> h(n);
    cudaMemcpy(h.data(), d, n * sizeof(Qcomp), cudaMemcpyDeviceToHost);
    return h;
}

int main(int argc, char** argv) {
    const int Nx = argc > 1 ? std::atoi(argv[1]) : 64;
    const int Ns = argc > 2 ? std::atoi(argv[2]) : 10;
    const std::string integ = argc > 3 ? argv[3] : "rk4";
    const bool friction = argc > 4 && std::string(argv[4]) == "friction";
    const int Ny = Nx, BSZ = 16, Nxh = Nx / 2 + 1;
    const Qreal Lx = friction ? 33 * 2 * M_PI : 16 * M_PI, Ly = Lx;
    const Qreal lambda = 0.1, Rf = friction ? 0.00075 : 0.1, alpha = friction ? 0.2 : 1.0;
    const Qreal Re = friction ? 0.1 : 1.0, Er = friction ? 0.1 : 1.0, dt = friction ? 0.002 : 1e-3;

    Mesh* mesh = new Mesh(Nx, Ny, Lx, Ly, BSZ);
    Field *wold = new Field(mesh), *wcurr = new Field(mesh), *wnew = new Field(mesh), *wnonl = new Field(mesh);
    Field *u = new Field(mesh), *v = new Field(mesh), *S = new Field(mesh);
    Field *r1old = new Field(mesh), *r1curr = new Field(mesh), *r1new = new Field(mesh), *r1nonl = new Field(mesh);
    Field *r2old = new Field(mesh), *r2curr = new Field(mesh), *r2new = new Field(mesh), *r2nonl = new Field(mesh);
    Field *p11 = new Field(mesh), *p12 = new Field(mesh), *p21 = new Field(mesh), *Ra = new Field(mesh);
    Field *aux = new Field(mesh), *aux1 = new Field(mesh);

    // seeded random Q, w = 0, as physical fields; FwdTrans to spectra
    std::vector<double> hw(Nx * Ny), h1(Nx * Ny), h2(Nx * Ny);
    qaf_random_q_init(7, Nx, Ny, -0.01, 0.01, hw.data(), h1.data(), h2.data());
    std::vector<Qreal> tmp(Nx * Ny);
    Field* init[3] = {wold, r1old, r2old};
    const std::vector<double>* src[3] = {&hw, &h1, &h2};
    for (int f = 0; f < 3; ++f) {
        for (int k = 0; k < Nx * Ny; ++k) tmp[k] = (Qreal)(*src[f])[k];
        cudaMemcpy(init[f]->phys, tmp.data(), mesh->physsize, cudaMemcpyHostToDevice);
        FwdTrans(init[f]->spec, init[f]->phys, mesh);
    }
    // the fused path starts from copies of the same spectra
    Qcomp *fw, *f1, *f2;
    cudaMalloc((void**)&fw, mesh->specsize);
    cudaMalloc((void**)&f1, mesh->specsize);
    cudaMalloc((void**)&f2, mesh->specsize);
    cudaMemcpy(fw, wold->spec, mesh->specsize, cudaMemcpyDeviceToDevice);
    cudaMemcpy(f1, r1old->spec, mesh->specsize, cudaMemcpyDeviceToDevice);
    cudaMemcpy(f2, r2old->spec, mesh->specsize, cudaMemcpyDeviceToDevice);

    FldSet<<<mesh->dimGridp, mesh->dimBlockp>>>(Ra->phys, alpha, Nx, Ny, BSZ);
    Qreal *IFw, *IFwh, *IFr1, *IFr1h, *IFr2, *IFr2h;
    cudaMalloc((void**)&IFw, mesh->wavesize); cudaMalloc((void**)&IFwh, mesh->wavesize);
    cudaMalloc((void**)&IFr1, mesh->wavesize); cudaMalloc((void**)&IFr1h, mesh->wavesize);
    cudaMalloc((void**)&IFr2, mesh->wavesize); cudaMalloc((void**)&IFr2h, mesh->wavesize);
    wlin_func<<<mesh->dimGridsp, mesh->dimBlocksp>>>(IFw, IFwh, mesh->k_squared, Re, Rf, dt, Nxh, Ny, BSZ);
    r1lin_func<<<mesh->dimGridsp, mesh->dimBlocksp>>>(IFr1, IFr1h, mesh->k_squared, dt, Nxh, Ny, BSZ);
    r2lin_func<<<mesh->dimGridsp, mesh->dimBlocksp>>>(IFr2, IFr2h, mesh->k_squared, dt, Nxh, Ny, BSZ);

    Field* old_[3] = {wold, r1old, r2old};
    Field* curr_[3] = {wcurr, r1curr, r2curr};
    Field* new_[3] = {wnew, r1new, r2new};
    Field* nonl_[3] = {wnonl, r1nonl, r2nonl};
    Qreal* IF_[3] = {IFw, IFr1, IFr2};
    Qreal* IFh_[3] = {IFwh, IFr1h, IFr2h};
    auto nonlinear = [&]() {
        curr_func(r1curr, r2curr, wcurr, u, v, S);
        wnonl_func(wnonl, wcurr, u, v, r1curr, r2curr, Ra, S, p11, p12, p21, Re, Er, lambda, aux, aux1);
        r1nonl_func(r1nonl, wcurr, u, v, r1curr, r2curr, S, lambda, aux, aux1);
        r2nonl_func(r2nonl, wcurr, u, v, r1curr, r2curr, S, lambda, aux, aux1);
    };
    const dim3 g = mesh->dimGridsp, b = mesh->dimBlocksp;
    for (int m = 0; m < Ns; ++m) {
        if (integ == "rk4") {
            for (int f = 0; f < 3; ++f)
                integrate_func0D<<<g, b>>>(old_[f]->spec, curr_[f]->spec, new_[f]->spec, IF_[f], IFh_[f], Nxh, Ny, BSZ, dt);
            nonlinear();
            for (int f = 0; f < 3; ++f)
                integrate_func1D<<<g, b>>>(old_[f]->spec, curr_[f]->spec, new_[f]->spec, nonl_[f]->spec, IF_[f], IFh_[f], Nxh, Ny, BSZ, dt);
            nonlinear();
            for (int f = 0; f < 3; ++f)
                integrate_func2D<<<g, b>>>(old_[f]->spec, curr_[f]->spec, new_[f]->spec, nonl_[f]->spec, IF_[f], IFh_[f], Nxh, Ny, BSZ, dt);
            nonlinear();
            for (int f = 0; f < 3; ++f)
                integrate_func3D<<<g, b>>>(old_[f]->spec, curr_[f]->spec, new_[f]->spec, nonl_[f]->spec, IF_[f], IFh_[f], Nxh, Ny, BSZ, dt);
            nonlinear();
            for (int f = 0; f < 3; ++f)
                integrate_func4D<<<g, b>>>(old_[f]->spec, curr_[f]->spec, new_[f]->spec, nonl_[f]->spec, IF_[f], IFh_[f], Nxh, Ny, BSZ, dt);
        } else if (integ == "rk2") {
            // Lawson-Heun: the full-step factor as the curr factor
            for (int f = 0; f < 3; ++f)
                IF::IFRK2::integrate_func0D<<<g, b>>>(old_[f]->spec, curr_[f]->spec, new_[f]->spec, IF_[f], IF_[f], Nxh, Ny, BSZ, dt);
            nonlinear();
            for (int f = 0; f < 3; ++f)
                IF::IFRK2::integrate_func1D<<<g, b>>>(old_[f]->spec, curr_[f]->spec, new_[f]->spec, nonl_[f]->spec, IF_[f], IF_[f], Nxh, Ny, BSZ, dt);
            nonlinear();
            for (int f = 0; f < 3; ++f)
                IF::IFRK2::integrate_func2D<<<g, b>>>(old_[f]->spec, curr_[f]->spec, new_[f]->spec, nonl_[f]->spec, IF_[f], IF_[f], Nxh, Ny, BSZ, dt);
        } else {
            for (int f = 0; f < 3; ++f) SpecSet<<<g, b>>>(curr_[f]->spec, old_[f]->spec, Nxh, Ny, BSZ);
            nonlinear();
            for (int f = 0; f < 3; ++f)
                IF::IFE::integrate_func1D<<<g, b>>>(old_[f]->spec, new_[f]->spec, nonl_[f]->spec, IF_[f], IFh_[f], Nxh, Ny, BSZ, dt);
        }
        for (int f = 0; f < 3; ++f) {
            dealias<<<g, b>>>(new_[f]->spec, mesh->cutoff, Nxh, Ny, BSZ);
            SpecSet<<<g, b>>>(old_[f]->spec, new_[f]->spec, Nxh, Ny, BSZ);
        }
    }
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) { std::fprintf(stderr, "CUDA error: %s\n", cudaGetErrorString(e)); return 1; }

    qaf_params p;
    p.re = Re; p.er = Er; p.rf = Rf; p.lambda = lambda; p.alpha = alpha; p.alpha_field = nullptr;
    p.dt = dt; p.q_lin = 1.0; p.advect_omega = 1; p.no_dealias = 0;
    const qaf_integrator qi = integ == "rk4" ? QAF_IFRK4 : (integ == "rk2" ? QAF_IFRK2 : QAF_IFE);
    qaf_compat::check(qaf_step(mesh->handle, &p, qi, fw, f1, f2, Ns, nullptr), "qaf_step");
    cudaDeviceSynchronize();

    const size_t ns = (size_t)Nxh * Ny;
    const double ew = rel_l2(fetch(wold->spec, ns), fetch(fw, ns));
    const double e1 = rel_l2(fetch(r1old->spec, ns), fetch(f1, ns));
    const double e2 = rel_l2(fetch(r2old->spec, ns), fetch(f2, ns));
    std::printf("{\"n\": %d, \"steps\": %d, \"integrator\": \"%s\", \"rel_w\": %.3e, \"rel_r1\": %.3e, \"rel_r2\": %.3e}\n",
                Nx, Ns, integ.c_str(), ew, e1, e2);

    cudaFree(fw); cudaFree(f1); cudaFree(f2);
    cudaFree(IFw); cudaFree(IFwh); cudaFree(IFr1); cudaFree(IFr1h); cudaFree(IFr2); cudaFree(IFr2h);
    Field* all[] = {wold, wcurr, wnew, wnonl, u, v, S, r1old, r1curr, r1new, r1nonl, r2old, r2curr, r2new, r2nonl,
                    p11, p12, p21, Ra, aux, aux1};
    for (Field* f : all) delete f;
    delete mesh;
    return 0;
}
