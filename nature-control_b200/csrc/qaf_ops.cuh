// qaf_ops.cuh — standalone 2D transforms (FwdTrans / BwdTrans of the C ABI)
// and the pointwise spectral kernels of the reference's public surface.
//
// 2D transforms use the packed intermediate T[n*H + k] (x-spectral,
// y-physical, k < H; slot k = 0 holds DC + i*Nyquist of the row):
//   BwdTrans: col_ifft (per kx-column y-IFFT, columns 0 and N/2 projected on
//             their Hermitian parts and packed) -> row_c2r
//   FwdTrans: row_r2c -> col_fft (columns 0 and N/2 unpacked)
#pragma once

#include "qaf_stage.cuh"

namespace qaf {

// N is the column length ny; the nx / 2 columns are the grid (tw: the ny-point twiddles)
template <typename real, int N, int W, int E>
__global__ void __launch_bounds__(W * (N / E))
col_ifft_kernel(const cplx<real>* __restrict__ spec, cplx<real>* __restrict__ T, const cplx<real>* __restrict__ tw, int nx) {
    constexpr int TEAM = N / E;
    const int H = nx / 2, NXH = H + 1;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    cplx<real>* buf = reinterpret_cast<cplx<real>*>(smem_raw);
    const int w = threadIdx.x % W, t = threadIdx.x / W;
    const int i = blockIdx.x * W + w;
    XchgCols<real> x{buf, w, W};
    TeamFFT<real, N, E> fft;
    fft.template init<N>(t, tw);
    const real s = (real)1 / ((real)nx * (real)N);
    cplx<real> v[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int j = t + TEAM * e;
        if (i != 0) {
            v[e] = cscale(spec[(size_t)j * NXH + i], s);
        } else {
            const int jm = (N - j) % N;
            const cplx<real> a0 = spec[(size_t)j * NXH], b0 = spec[(size_t)jm * NXH];
            const cplx<real> aH = spec[(size_t)j * NXH + H], bH = spec[(size_t)jm * NXH + H];
            const cplx<real> P0 = cscale(cadd(a0, cconj(b0)), (real)0.5 * s);
            const cplx<real> PH = cscale(cadd(aH, cconj(bH)), (real)0.5 * s);
            v[e] = cadd(P0, cmul_i(PH));
        }
    }
    fft.template run<true>(t, v, x);
#pragma unroll
    for (int e = 0; e < E; ++e) T[(size_t)(t + TEAM * e) * H + i] = v[e];
}

template <typename real, int N, int W, int E>
__global__ void __launch_bounds__(W * (N / E))
col_fft_kernel(const cplx<real>* __restrict__ T, cplx<real>* __restrict__ spec, const cplx<real>* __restrict__ tw, int nx) {
    constexpr int TEAM = N / E;
    const int H = nx / 2, NXH = H + 1;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    cplx<real>* buf = reinterpret_cast<cplx<real>*>(smem_raw);
    const int w = threadIdx.x % W, t = threadIdx.x / W;
    const int i = blockIdx.x * W + w;
    XchgCols<real> x{buf, w, W};
    TeamFFT<real, N, E> fft;
    fft.template init<N>(t, tw);
    cplx<real> v[E];
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = T[(size_t)(t + TEAM * e) * H + i];
    fft.template run<false>(t, v, x);
    // column 0 holds DC + i*Nyquist sequences: unpack with the partner -j
#pragma unroll
    for (int e = 0; e < E; ++e) x.write(t + TEAM * e, v[e]);
    x.sync();
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int j = t + TEAM * e;
        if (i != 0) {
            spec[(size_t)j * NXH + i] = v[e];
        } else {
            const cplx<real> zm = cconj(x.read((N - j) % N));
            spec[(size_t)j * NXH] = cscale(cadd(v[e], zm), (real)0.5);
            spec[(size_t)j * NXH + H] = cmul_mi(cscale(csub(v[e], zm), (real)0.5));
        }
    }
}

template <typename real, int N, int E, int ROWS>
__global__ void __launch_bounds__(ROWS * (N / 2 / E))
row_c2r_kernel(const cplx<real>* __restrict__ T, real* __restrict__ phys, const cplx<real>* __restrict__ tw) {
    constexpr int H = N / 2, TEAM = H / E;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    cplx<real>* buf = reinterpret_cast<cplx<real>*>(smem_raw);
    const int r = threadIdx.x / TEAM, t = threadIdx.x % TEAM;
    const int n = blockIdx.x * ROWS + r;
    XchgRow<real> x{buf + r * H};
    const cplx<real>* row = T + (size_t)n * H;
    cplx<real> v[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int k = t + TEAM * e;
        if (k == 0) {
            const cplx<real> d = row[0];
            v[e] = mk<real>(d.x + d.y, d.x - d.y);
        } else {
            const cplx<real> A = row[k], B = cconj(row[H - k]);
            v[e] = cadd(cadd(A, B), cmul_i(cmul(cconj(tw[k]), csub(A, B))));
        }
    }
    TeamFFT<real, H, E> fft;
    fft.template init<N>(t, tw);
    fft.template run<true>(t, v, x);
    real* o = phys + (size_t)n * N;
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int m = t + TEAM * e;
        o[2 * m] = v[e].x;
        o[2 * m + 1] = v[e].y;
    }
}

template <typename real, int N, int E, int ROWS>
__global__ void __launch_bounds__(ROWS * (N / 2 / E))
row_r2c_kernel(const real* __restrict__ phys, cplx<real>* __restrict__ T, const cplx<real>* __restrict__ tw) {
    constexpr int H = N / 2, TEAM = H / E;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    cplx<real>* buf = reinterpret_cast<cplx<real>*>(smem_raw);
    const int r = threadIdx.x / TEAM, t = threadIdx.x % TEAM;
    const int n = blockIdx.x * ROWS + r;
    XchgRow<real> x{buf + r * H};
    const real* in = phys + (size_t)n * N;
    cplx<real> v[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int m = t + TEAM * e;
        v[e] = mk<real>(in[2 * m], in[2 * m + 1]);
    }
    TeamFFT<real, H, E> fft;
    fft.template init<N>(t, tw);
    fft.template run<false>(t, v, x);
#pragma unroll
    for (int e = 0; e < E; ++e) x.write(t + TEAM * e, v[e]);
    x.sync();
    cplx<real>* out = T + (size_t)n * H;
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int k = t + TEAM * e;
        const cplx<real> zm = cconj(x.read((H - k) % H));
        if (k == 0) {
            out[0] = mk<real>(v[e].x + v[e].y, v[e].x - v[e].y);
        } else {
            const cplx<real> sum = cscale(cadd(v[e], zm), (real)0.5);
            const cplx<real> dif = cscale(csub(v[e], zm), (real)0.5);
            out[k] = csub(sum, cmul_i(cmul(tw[k], dif)));
        }
    }
}

// ---------------------------------------------------------------------------
// Pointwise kernels on reference-layout spectra (index i + j*nxh). Wave
// numbers are formed as the reference's tables are (waveinit, Mesh.cuh:6-21):
// kx = (2 pi / Lx) i, ky = (2 pi / Ly) (j or j - ny), in double.
// ---------------------------------------------------------------------------
struct Geo {
    int nx, ny, nxh;
    double dkx, dky;
    __device__ double kx(int i) const { return dkx * i; }
    __device__ double ky(int j) const { return j < ny / 2 + 1 ? dky * j : dky * (j - ny); }
};

#define QAF_GRID_LOOP(idx, total) \
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < (total); idx += (size_t)gridDim.x * blockDim.x)

// op 0 xDeriv (QFldfuncs.cuh:165-176), 1 yDeriv (:178-189), 2 Laplacian (:191-202)
template <typename real>
__global__ void spec_unary_kernel(Geo g, int op, const cplx<real>* in, cplx<real>* out) {
    QAF_GRID_LOOP(k, (size_t)g.nxh * g.ny) {
        const int i = (int)(k % g.nxh), j = (int)(k / g.nxh);
        const cplx<real> f = in[k];
        if (op == 0) out[k] = cmul_i(cscale(f, (real)g.kx(i)));
        else if (op == 1) out[k] = cmul_i(cscale(f, (real)g.ky(j)));
        else {
            const real kx = (real)g.kx(i), ky = (real)g.ky(j);
            out[k] = cscale(f, -(kx * kx + ky * ky));
        }
    }
}

// vel_func (QFldfuncs.cuh:204-224)
template <typename real>
__global__ void vel_kernel(Geo g, const cplx<real>* w, cplx<real>* u, cplx<real>* v) {
    QAF_GRID_LOOP(k, (size_t)g.nxh * g.ny) {
        if (k == 0) { u[0] = mk<real>(0, 0); v[0] = mk<real>(0, 0); continue; }
        const int i = (int)(k % g.nxh), j = (int)(k / g.nxh);
        const real kx = (real)g.kx(i), ky = (real)g.ky(j);
        const real k2 = kx * kx + ky * ky;
        const cplx<real> f = w[k];
        const cplx<real> iw = cmul_i(f);
        u[k] = mk<real>(ky * iw.x / k2, ky * iw.y / k2);
        v[k] = mk<real>(-kx * iw.x / k2, -kx * iw.y / k2);
    }
}

// dealias (Qsolver.cuh:314-322) with the mask of cutoff_func (Mesh.cuh:23-46)
template <typename real>
__global__ void dealias_kernel(Geo g, cplx<real>* f) {
    QAF_GRID_LOOP(k, (size_t)g.nxh * g.ny) {
        const int i = (int)(k % g.nxh), j = (int)(k / g.nxh);
        const bool keep = (i < (g.nxh - 1) * 2 / 3 + 1) && ((j < g.ny / 3 + 1) || ((g.ny - j) < g.ny / 3));
        if (!keep) f[k] = mk<real>(0, 0);
    }
}

// symmetry_func (QFldfuncs.cuh:18-44)
template <typename real>
__global__ void symmetrize_kernel(Geo g, cplx<real>* f) {
    QAF_GRID_LOOP(j, (size_t)g.ny) {
        if (j == 0 || (int)j >= g.ny / 2) continue;
        cplx<real>& a = f[j * g.nxh];
        cplx<real>& b = f[(g.ny - j) * g.nxh];
        const cplx<real> mean = cscale(cadd(a, cconj(b)), (real)0.5);
        a = mean;
        b = cconj(mean);
    }
}

// wlin_func / r1lin_func / r2lin_func (Qsolver.cuh:20-54)
template <typename real>
__global__ void if_table_kernel(Geo g, int which, double re, double rf, double q_lin, double dt, real* IF, real* IFh) {
    QAF_GRID_LOOP(k, (size_t)g.nxh * g.ny) {
        const int i = (int)(k % g.nxh), j = (int)(k / g.nxh);
        const double kx = g.kx(i), ky = g.ky(j), k2 = kx * kx + ky * ky;
        const double L = which == 0 ? 1.0 / re * (-1.0 * k2 - rf) : (-1.0 * k2 + q_lin);
        IF[k] = (real)exp(L * dt);
        IFh[k] = (real)exp(L * dt * 0.5);
    }
}

// integrate_func0D..4D (RK4.cuh:12-74), IF::IFRK2 (IFRK2.cuh:16-51), IF::IFE (IFE.cuh:15-25)
template <typename real>
__global__ void integrate_kernel(size_t total, int integ, int stage, const cplx<real>* old, cplx<real>* curr,
                                 cplx<real>* nw, const cplx<real>* nonl, const real* IF, const real* IFh, real dt) {
    QAF_GRID_LOOP(k, total) {
        const real E = IF[k], Eh = IFh[k];
        const cplx<real> o = old[k];
        if (stage == 0) { nw[k] = cscale(o, E); curr[k] = o; continue; }
        const cplx<real> an = cscale(nonl[k], dt);
        if (integ == 2) {
            if (stage == 1) { nw[k] = cadd(nw[k], cscale(an, (real)(1.0 / 6.0) * E)); curr[k] = cscale(cadd(o, cscale(an, (real)0.5)), Eh); }
            else if (stage == 2) { nw[k] = cadd(nw[k], cscale(an, (real)(1.0 / 3.0) * Eh)); curr[k] = cadd(cscale(o, Eh), cscale(an, (real)0.5)); }
            else if (stage == 3) { nw[k] = cadd(nw[k], cscale(an, (real)(1.0 / 3.0) * Eh)); curr[k] = cadd(cscale(o, E), cscale(an, Eh)); }
            else { nw[k] = cadd(nw[k], cscale(an, (real)(1.0 / 6.0))); }
        } else if (integ == 1) {
            if (stage == 1) { nw[k] = cadd(nw[k], cscale(an, (real)0.5 * E)); curr[k] = cscale(cadd(o, an), Eh); }
            else { nw[k] = cadd(nw[k], cscale(an, (real)0.5)); }
        } else {
            nw[k] = cscale(cadd(o, an), E);
        }
    }
}

// Shell energy spectrum, energy and enstrophy of a reference-layout vorticity
// spectrum. Columns kx = 0 and nx/2 enter through their Hermitian parts, as
// a physical snapshot would carry them. Energy/enstrophy use Parseval
// weights (interior kx counted twice); the spectrum sums the stored
// half-plane without doubling, as EnergySpec.cu:81-96 does, over shells
// whose bounds advance by repeated addition k += dk (EnergySpec.cu:194-204).
template <typename real>
__global__ void diag_kernel(Geo g, const cplx<real>* w, double* acc, const double* bounds, int nshells) {
    QAF_GRID_LOOP(k, (size_t)g.nxh * g.ny) {
        const int i = (int)(k % g.nxh), j = (int)(k / g.nxh);
        cplx<real> f = w[k];
        const bool edge = (i == 0 || i == g.nxh - 1);
        if (edge) {
            const int jm = (g.ny - j) % g.ny;
            const cplx<real> b = w[(size_t)jm * g.nxh + i];
            f = cscale(cadd(f, cconj(b)), (real)0.5);
        }
        const double m2 = (double)f.x * f.x + (double)f.y * f.y;
        const double kx = g.kx(i), ky = g.ky(j), k2 = kx * kx + ky * ky;
        const double wgt = edge ? 1.0 : 2.0;
        atomicAdd(&acc[1], wgt * m2);
        if (k2 > 0) {
            atomicAdd(&acc[0], wgt * m2 / k2);
            if (nshells > 0 && k2 < bounds[nshells] * bounds[nshells]) {
                // shell s: bounds[s]^2 <= |k|^2 < bounds[s+1]^2 (bounds accumulated k += dk)
                int lo = 0, hi = nshells;   // invariant: bounds[lo]^2 <= k2 < bounds[hi]^2
                while (hi - lo > 1) {
                    const int mid = (lo + hi) / 2;
                    if (k2 >= bounds[mid] * bounds[mid]) lo = mid; else hi = mid;
                }
                atomicAdd(&acc[2 + lo], m2 / k2);
            }
        }
    }
}

// energy, enstrophy of the last step from its sums (Parseval form), for an asynchronous read-back
static __global__ void diag_finalize_kernel(const double* sums, double* out, double n4) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        out[0] = 0.5 * sums[1] / n4;
        out[1] = 0.5 * sums[0] / n4;
    }
}

}  // namespace qaf
