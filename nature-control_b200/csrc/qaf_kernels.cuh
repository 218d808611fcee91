// qaf_kernels.cuh — column and row kernels of the fused IF-RK stage
// (see qaf_stage.cuh for the data flow and layouts).
#pragma once

#include "qaf_stage.cuh"

namespace qaf {

// ---------------------------------------------------------------------------
// Column kernel, regular tiles: W packed kx-columns i of field f.
// ---------------------------------------------------------------------------
template <typename real, int N, int W, int E>
__device__ __forceinline__ void col_regular(const StageArgs<real>& a, int f, int i, int t, int w, cplx<real>* buf) {
    constexpr int H = N / 2, TEAM = N / E;
    XchgCols<real> x{buf, w, W};
    const real kx = a.dkx * (real)i;
    const real s = (real)1 / ((real)N * (real)N);
    const bool edge_col = (i == 0);   // packed column 0 belongs to the edge CTA
    cplx<real> v[E], nl[E], curr[E];
    const size_t plane = (size_t)N * H;

    if (a.mode != MODE_PROLOGUE) {
        const int gbase = f == 0 ? 0 : (f == 1 ? 3 : 5);
        const int ng = f == 0 ? 3 : 2;
#pragma unroll
        for (int e = 0; e < E; ++e) nl[e] = mk<real>(0, 0);
#pragma unroll 1
        for (int g = 0; g < ng; ++g) {
            const cplx<real>* G = a.G + (size_t)(gbase + g) * plane;
#pragma unroll
            for (int e = 0; e < E; ++e) v[e] = G[(size_t)(t + TEAM * e) * H + i];
            team_fft<real, N, E, false, N>(t, v, a.tw, x);
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const real ky = ky_of<real>(t + TEAM * e, N, a.dky);
                const real m = g == 0 ? (real)1 : (g == 1 ? ky : ky * ky);
                nl[e] = cadd(nl[e], cscale(v[e], m));
            }
        }
        if (a.mode == MODE_NONL) {
            if (!edge_col)
#pragma unroll
                for (int e = 0; e < E; ++e) a.nl_m[f][(size_t)(t + TEAM * e) * H + i] = nl[e];
            return;
        }
    }

    // stage update
    const bool need_old = a.mode == MODE_PROLOGUE || a.integrator == INT_IFE ||
                          (a.integrator == INT_IFRK4 && a.stage <= 3) || (a.integrator == INT_IFRK2 && a.stage == 1);
    const bool need_acc = a.mode == MODE_STAGE && ((a.integrator == INT_IFRK4 && a.stage >= 2) ||
                                                   (a.integrator == INT_IFRK2 && a.stage == 2));
    cplx<real>* om = a.old_m[f];
    cplx<real>* am = a.acc_m[f];
    double zsum = 0, esum = 0;
    bool bad = false;
    if (a.mode == MODE_PROLOGUE) {
#pragma unroll
        for (int e = 0; e < E; ++e) curr[e] = om[(size_t)(t + TEAM * e) * H + i];
    } else {
        const int cls = f == 0 ? 0 : 2;
        const real exf = a.ex[cls * (H + 1) + i] * a.e0[cls];
        const real exh = a.ex[(cls + 1) * (H + 1) + i] * a.e0[cls + 1];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int j = t + TEAM * e;
            const size_t idx = (size_t)j * H + i;
            const real Ef = exf * a.ey[cls * N + j];
            const real Eh = exh * a.ey[(cls + 1) * N + j];
            const cplx<real> o = need_old ? om[idx] : mk<real>(0, 0);
            const cplx<real> ac = need_acc ? am[idx] : mk<real>(0, 0);
            StageUpdate<real> u = stage_update(a, nl[e], o, ac, Ef, Eh, mask_keep(a, i, j));
            if (!edge_col) {
                if (u.write_acc) am[idx] = u.acc;
                if (u.write_old) {
                    om[idx] = u.acc;
                    bad |= !(isfinite(u.acc.x) && isfinite(u.acc.y));
                    if (f == 0 && a.diag) {
                        const real ky = ky_of<real>(j, N, a.dky);
                        const double k2 = (double)kx * kx + (double)ky * ky;
                        const double m2 = (double)u.acc.x * u.acc.x + (double)u.acc.y * u.acc.y;
                        zsum += 2.0 * m2;
                        if (k2 > 0) esum += 2.0 * m2 / k2;
                    }
                }
            }
            curr[e] = u.curr;
        }
        if (a.last_stage) {
            if (a.flags && __any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(a.flags, 1u);
            if (f == 0 && a.diag) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    zsum += __shfl_xor_sync(0xffffffffu, zsum, o);
                    esum += __shfl_xor_sync(0xffffffffu, esum, o);
                }
                if ((threadIdx.x & 31) == 0) { atomicAdd(&a.diag[0], zsum); atomicAdd(&a.diag[1], esum); }
            }
        }
    }

    if (!a.do_inverse) return;
    const int nq = f == 0 ? 4 : 2;
#pragma unroll 1
    for (int qq = 0; qq < nq; ++qq) {
        const int q = f == 0 ? (qq == 0 ? 0 : qq + 2) : (f == 1 ? (qq == 0 ? 1 : 6) : (qq == 0 ? 2 : 7));
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const real ky = ky_of<real>(t + TEAM * e, N, a.dky);
            v[e] = y_mult<real>(q, curr[e], ky, kx * kx + ky * ky, s);
        }
        team_fft<real, N, E, true, N>(t, v, a.tw, x);
        cplx<real>* Y = a.Y + (size_t)q * plane;
#pragma unroll
        for (int e = 0; e < E; ++e) Y[(size_t)(t + TEAM * e) * H + i] = v[e];
    }
}

// ---------------------------------------------------------------------------
// Column kernel, edge CTA of field f: the kx = 0 and kx = N/2 columns.
// W teams share the FFT jobs of the field; team 0 owns the state update.
// ---------------------------------------------------------------------------
template <typename real>
__device__ __forceinline__ void edge_product_mults(int p, real ky, real kN, real ce, int j, int N, int advect,
                                                   cplx<real>& m0, cplx<real>& mH) {
    // multiplier of edge product p in column kx = 0 (m0) and kx = N/2 (mH), as
    // complex numbers applied to the product's column spectrum
    m0 = mk<real>(0, 0);
    mH = mk<real>(0, 0);
    switch (p) {
        case 0:   // -v w: i ky; zeroed at j = N/2 by the round trip of wnonl_func (Qsolver.cuh:184-193)
            if (advect && 2 * j != N) { m0 = mk<real>(0, ky); mH = mk<real>(0, ky); }
            break;
        case 1: mH = mk<real>(2 * ce * kN * ky, 0); break;          // p11: 2 ce kx ky
        case 2: mH = mk<real>(-ce * kN * kN, 0); break;             // p12: -ce kx^2
        case 3: m0 = mk<real>(ce * ky * ky, 0); mH = m0; break;     // p21: ce ky^2
        case 4: case 7: m0 = mk<real>(1, 0); mH = m0; break;        // P1, P2
        case 5: case 8: mH = mk<real>(0, kN); break;                // A1, A2: i kx
        default: m0 = mk<real>(0, ky); mH = m0; break;              // B1, B2: i ky
    }
}

template <typename real, int N, int W, int E>
__device__ __forceinline__ void col_edge(const StageArgs<real>& a, int f, int t, int w, cplx<real>* buf,
                                         cplx<real>* ctab) {
    constexpr int H = N / 2, TEAM = N / E;
    XchgCols<real> x{buf, w, W};
    const real kN = a.dkx * (real)H;
    const real s = (real)1 / ((real)N * (real)N);
    cplx<real> v[E], n0[E], nH[E];
#pragma unroll
    for (int e = 0; e < E; ++e) { n0[e] = mk<real>(0, 0); nH[e] = mk<real>(0, 0); }

    if (a.mode != MODE_PROLOGUE) {
        const int pbase = f == 0 ? 0 : (f == 1 ? 4 : 7);
        const int np = f == 0 ? 4 : 3;
#pragma unroll 1
        for (int base = 0; base < np; base += W) {
            const bool active = base + w < np;
            const int p = pbase + (active ? base + w : 0);
#pragma unroll
            for (int e = 0; e < E; ++e) v[e] = active ? a.Ed[(size_t)p * N + t + TEAM * e] : mk<real>(0, 0);
            team_fft<real, N, E, false, N>(t, v, a.tw, x);
            // unpack the two real sequences: DC = (Z[j] + conj Z[-j]) / 2, NYQ = (Z[j] - conj Z[-j]) / 2i
#pragma unroll
            for (int e = 0; e < E; ++e) x.write(t + TEAM * e, v[e]);
            x.sync();
            cplx<real> c0[E], cH[E];
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int j = t + TEAM * e;
                const cplx<real> zm = cconj(x.read((N - j) % N));
                const cplx<real> dc = cscale(cadd(v[e], zm), (real)0.5);
                const cplx<real> ny = cmul_mi(cscale(csub(v[e], zm), (real)0.5));
                cplx<real> m0, mH;
                edge_product_mults<real>(p, ky_of<real>(j, N, a.dky), kN, a.ce, j, N, a.advect, m0, mH);
                c0[e] = active ? cmul(dc, m0) : mk<real>(0, 0);
                cH[e] = active ? cmul(ny, mH) : mk<real>(0, 0);
            }
            x.sync();
            // sum over teams into team 0
#pragma unroll
            for (int e = 0; e < E; ++e) x.write(t + TEAM * e, c0[e]);
            x.sync();
            if (w == 0)
#pragma unroll
                for (int e = 0; e < E; ++e)
                    for (int ww = 0; ww < W; ++ww) n0[e] = cadd(n0[e], buf[(t + TEAM * e) * W + ww]);
            x.sync();
#pragma unroll
            for (int e = 0; e < E; ++e) x.write(t + TEAM * e, cH[e]);
            x.sync();
            if (w == 0)
#pragma unroll
                for (int e = 0; e < E; ++e)
                    for (int ww = 0; ww < W; ++ww) nH[e] = cadd(nH[e], buf[(t + TEAM * e) * W + ww]);
            x.sync();
        }
    }

    if (w == 0) {
        cplx<real>* om = a.old_m[f];
        cplx<real>* on = a.old_n[f];
        cplx<real>* am = a.acc_m[f];
        cplx<real>* an = a.acc_n[f];
        if (a.mode == MODE_NONL) {
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int j = t + TEAM * e;
                a.nl_m[f][(size_t)j * H] = n0[e];
                a.nl_n[f][j] = nH[e];
            }
        } else if (a.mode == MODE_PROLOGUE) {
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int j = t + TEAM * e;
                ctab[j] = om[(size_t)j * H];
                ctab[N + j] = on[j];
            }
        } else {
            const bool need_old = a.integrator == INT_IFE || (a.integrator == INT_IFRK4 && a.stage <= 3) ||
                                  (a.integrator == INT_IFRK2 && a.stage == 1);
            const bool need_acc = (a.integrator == INT_IFRK4 && a.stage >= 2) || (a.integrator == INT_IFRK2 && a.stage == 2);
            const int cls = f == 0 ? 0 : 2;
            bool bad = false;
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int j = t + TEAM * e;
                const real ky = ky_of<real>(j, N, a.dky);
                const real eyf = a.ey[cls * N + j] * a.e0[cls], eyh = a.ey[(cls + 1) * N + j] * a.e0[cls + 1];
                // column kx = 0
                {
                    const size_t idx = (size_t)j * H;
                    const real Ef = a.ex[cls * (H + 1)] * eyf, Eh = a.ex[(cls + 1) * (H + 1)] * eyh;
                    const cplx<real> o = need_old ? om[idx] : mk<real>(0, 0);
                    const cplx<real> ac = need_acc ? am[idx] : mk<real>(0, 0);
                    StageUpdate<real> u = stage_update(a, n0[e], o, ac, Ef, Eh, mask_keep(a, 0, j));
                    if (u.write_acc) am[idx] = u.acc;
                    if (u.write_old) {
                        om[idx] = u.acc;
                        bad |= !(isfinite(u.acc.x) && isfinite(u.acc.y));
                    }
                    ctab[j] = u.curr;
                }
                // column kx = N/2
                {
                    const real Ef = a.ex[cls * (H + 1) + H] * eyf, Eh = a.ex[(cls + 1) * (H + 1) + H] * eyh;
                    const cplx<real> o = need_old ? on[j] : mk<real>(0, 0);
                    const cplx<real> ac = need_acc ? an[j] : mk<real>(0, 0);
                    StageUpdate<real> u = stage_update(a, nH[e], o, ac, Ef, Eh, mask_keep(a, H, j));
                    if (u.write_acc) an[j] = u.acc;
                    if (u.write_old) {
                        on[j] = u.acc;
                        bad |= !(isfinite(u.acc.x) && isfinite(u.acc.y));
                    }
                    ctab[N + j] = u.curr;
                }
            }
            if (a.last_stage && bad && a.flags) atomicOr(a.flags, 1u);
        }
    }
    __syncthreads();
    // Energy and enstrophy of the new state's kx = 0 and kx = N/2 columns,
    // through their Hermitian parts (what a physical snapshot holds; the
    // asymmetric 2/3 mask leaves the kx = 0 column non-Hermitian at ky = N/3).
    if (a.mode == MODE_STAGE && a.last_stage && f == 0 && a.diag && w == 0) {
        double zsum = 0, esum = 0;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int j = t + TEAM * e, jm = (N - j) % N;
            const double ky = (double)ky_of<real>(j, N, a.dky);
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const cplx<real> p = cscale(cadd(ctab[c * N + j], cconj(ctab[c * N + jm])), (real)0.5);
                const double m2 = (double)p.x * p.x + (double)p.y * p.y;
                const double kx = c == 0 ? 0.0 : (double)kN;
                const double k2 = kx * kx + ky * ky;
                zsum += m2;
                if (k2 > 0) esum += m2 / k2;
            }
        }
        atomicAdd(&a.diag[0], zsum);
        atomicAdd(&a.diag[1], esum);
    }
    if (a.mode == MODE_NONL || !a.do_inverse) return;

    const int no = f == 0 ? 5 : 2;
#pragma unroll 1
    for (int base = 0; base < no; base += W) {
        const bool active = base + w < no;
        const int oi = active ? base + w : 0;
        const int p = f == 0 ? (oi == 0 ? PF_W : PF_U + oi - 1) : (f == 1 ? (oi == 0 ? PF_R1 : PF_LR1)
                                                                         : (oi == 0 ? PF_R2 : PF_LR2));
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int j = t + TEAM * e, jm = (N - j) % N;
            const real kyj = ky_of<real>(j, N, a.dky), kym = ky_of<real>(jm, N, a.dky);
            const cplx<real> v0j = derived<real>(p, ctab[j], (real)0, kyj, kyj * kyj, s);
            const cplx<real> v0m = derived<real>(p, ctab[jm], (real)0, kym, kym * kym, s);
            const cplx<real> vHj = derived<real>(p, ctab[N + j], kN, kyj, kN * kN + kyj * kyj, s);
            const cplx<real> vHm = derived<real>(p, ctab[N + jm], kN, kym, kN * kN + kym * kym, s);
            const cplx<real> P0 = cscale(cadd(v0j, cconj(v0m)), (real)0.5);
            const cplx<real> PH = cscale(cadd(vHj, cconj(vHm)), (real)0.5);
            v[e] = cadd(P0, cmul_i(PH));
        }
        team_fft<real, N, E, true, N>(t, v, a.tw, x);
        if (active)
#pragma unroll
            for (int e = 0; e < E; ++e) a.D[(size_t)p * N + t + TEAM * e] = v[e];
    }
}

template <typename real, int N, int W, int E>
__global__ void __launch_bounds__(W * (N / E)) col_kernel(const StageArgs<real> a) {
    constexpr int H = N / 2, TILES = H / W;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<real>* buf = reinterpret_cast<cplx<real>*>(smem_raw);
    cplx<real>* ctab = buf + N * W;
    const int tid = threadIdx.x, w = tid % W, t = tid / W;
    const int blk = blockIdx.x;
    if (blk < 3 * TILES) {
        const int f = blk / TILES, tile = blk % TILES;
        col_regular<real, N, W, E>(a, f, tile * W + w, t, w, buf);
    } else {
        col_edge<real, N, W, E>(a, blk - 3 * TILES, t, w, buf, ctab);
    }
}

// ---------------------------------------------------------------------------
// Row kernel: ROWS rows per CTA, one team of H/E threads per row.
// ---------------------------------------------------------------------------
template <typename real, int N, int E>
struct RowCtx {
    static constexpr int H = N / 2, TEAM = H / E;
    const StageArgs<real>& a;
    int n, t;
    XchgRow<real> x;

    __device__ cplx<real> yv(int q, int k) const { return a.Y[(size_t)q * N * H + (size_t)n * H + k]; }

    // x-spectrum of physical field p at wave number k in [1, H)
    __device__ cplx<real> xspec(int p, int k) const {
        const real kx = a.dkx * (real)k;
        switch (p) {
            case PF_W: return yv(0, k);
            case PF_R1: return yv(1, k);
            case PF_R2: return yv(2, k);
            case PF_U: return yv(3, k);
            case PF_V: return cmul_i(cscale(yv(4, k), kx));
            case PF_UX: return cmul_i(cscale(yv(3, k), kx));
            case PF_SH: return csub(yv(5, k), cscale(yv(4, k), kx * kx));
            case PF_LR1: return csub(cscale(yv(1, k), -kx * kx), yv(6, k));
            default: return csub(cscale(yv(2, k), -kx * kx), yv(7, k));
        }
    }

    // half-length C2R of field p: out[2e], out[2e+1] = x(2m), x(2m+1), m = t + TEAM e
    __device__ void c2r(int p, real* out) {
        cplx<real> v[E];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int k = t + TEAM * e;
            if (k == 0) {
                const cplx<real> d = a.D[(size_t)p * N + n];
                v[e] = mk<real>(d.x + d.y, d.x - d.y);
            } else {
                const cplx<real> A = xspec(p, k), B = cconj(xspec(p, H - k));
                const cplx<real> wp = cconj(a.tw[k]);    // exp(+2 pi i k / N)
                v[e] = cadd(cadd(A, B), cmul_i(cmul(wp, csub(A, B))));
            }
        }
        team_fft<real, H, E, true, N>(t, v, a.tw, x);
#pragma unroll
        for (int e = 0; e < E; ++e) { out[2 * e] = v[e].x; out[2 * e + 1] = v[e].y; }
    }

    // half-length R2C of the real row `in` (same distribution as c2r's output);
    // F[e] = X[k], k = t + TEAM e (F = 0 at k = 0); edge = (X[0], X[N/2]) packed
    __device__ void r2c(const real* in, cplx<real>* F, cplx<real>& edge) {
        cplx<real> v[E];
#pragma unroll
        for (int e = 0; e < E; ++e) v[e] = mk<real>(in[2 * e], in[2 * e + 1]);
        team_fft<real, H, E, false, N>(t, v, a.tw, x);
#pragma unroll
        for (int e = 0; e < E; ++e) x.write(t + TEAM * e, v[e]);
        x.sync();
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int k = t + TEAM * e;
            const cplx<real> zm = cconj(x.read((H - k) % H));
            if (k == 0) {
                edge = mk<real>(v[e].x + v[e].y, v[e].x - v[e].y);
                F[e] = mk<real>(0, 0);
            } else {
                const cplx<real> sum = cscale(cadd(v[e], zm), (real)0.5);
                const cplx<real> dif = cscale(csub(v[e], zm), (real)0.5);
                F[e] = csub(sum, cmul_i(cmul(a.tw[k], dif)));
            }
        }
        x.sync();
    }

    __device__ void put_edge(int p, cplx<real> edge) const {
        if (t == 0) a.Ed[(size_t)p * N + n] = edge;
    }
    __device__ void put_g(int g, const cplx<real>* F) const {
        cplx<real>* G = a.G + (size_t)g * N * H + (size_t)n * H;
#pragma unroll
        for (int e = 0; e < E; ++e) G[t + TEAM * e] = F[e];
    }
    __device__ real kx_of(int e) const { return a.dkx * (real)(t + TEAM * e); }
    __device__ void dump(int fld, const real* val) const {
        if (!a.phys_out) return;
        real* o = a.phys_out + (size_t)fld * N * N + (size_t)n * N;
#pragma unroll
        for (int e = 0; e < E; ++e) { o[2 * (t + TEAM * e)] = val[2 * e]; o[2 * (t + TEAM * e) + 1] = val[2 * e + 1]; }
    }
};

template <typename real, int N, int E, int ROWS>
__global__ void __launch_bounds__(ROWS * (N / 2 / E)) row_kernel(const StageArgs<real> a) {
    constexpr int H = N / 2, TEAM = H / E, P = 2 * E;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<real>* buf = reinterpret_cast<cplx<real>*>(smem_raw);
    const int r = threadIdx.x / TEAM, t = threadIdx.x % TEAM;
    const int n = blockIdx.x * ROWS + r;
    RowCtx<real, N, E> c{a, n, t, XchgRow<real>{buf + r * H}};
    const real lam = a.lambda, ce = a.ce;

    real r1[P], r2[P], S[P], al[P];
#pragma unroll
    for (int q = 0; q < P; ++q) {
        const int xg = 2 * (t + TEAM * (q / 2)) + (q & 1);
        al[q] = a.alpha_field ? a.alpha_field[(size_t)n * N + xg] : a.alpha;
    }
    c.c2r(PF_R1, r1);
    c.c2r(PF_R2, r2);
#pragma unroll
    for (int q = 0; q < P; ++q) S[q] = 2 * sqrt(r1[q] * r1[q] + r2[q] * r2[q]);   // S_func (Qsolver.cuh:63-71)
    c.dump(PF_R1, r1); c.dump(PF_R2, r2); c.dump(9, S);

    cplx<real> F11[E], F12[E], tmpF[E], edge;
    {
        real L1[P], L2[P], pr[P];
        c.c2r(PF_LR1, L1);
        c.dump(PF_LR1, L1);
        // p11 = -lambda S Lap r1 + lambda S (S^2-1) r1 - Ra r1   (single + Rar, Qsolver.cuh:75-131)
#pragma unroll
        for (int q = 0; q < P; ++q)
            pr[q] = -lam * L1[q] * S[q] + lam * S[q] * (S[q] * S[q] - 1) * r1[q] - al[q] * r1[q];
        c.dump(10, pr);
        c.r2c(pr, F11, edge); c.put_edge(1, edge);
        c.c2r(PF_LR2, L2);
        c.dump(PF_LR2, L2);
        // p12 = single(r2) + 2 Lap r1 r2 - 2 r1 Lap r2 - Ra r2   (p12func, Qsolver.cuh:133-141)
#pragma unroll
        for (int q = 0; q < P; ++q) {
            const real sg = -lam * L2[q] * S[q] + lam * S[q] * (S[q] * S[q] - 1) * r2[q];
            pr[q] = sg + (2 * L1[q] * r2[q] - 2 * r1[q] * L2[q]) - al[q] * r2[q];
        }
        c.dump(11, pr);
        c.r2c(pr, F12, edge); c.put_edge(2, edge);
        // p21 = single(r2) + 2 Lap r2 r1 - 2 r2 Lap r1 - Ra r2   (p21func, Qsolver.cuh:143-151)
#pragma unroll
        for (int q = 0; q < P; ++q) {
            const real sg = -lam * L2[q] * S[q] + lam * S[q] * (S[q] * S[q] - 1) * r2[q];
            pr[q] = sg + (2 * L2[q] * r1[q] - 2 * r2[q] * L1[q]) - al[q] * r2[q];
        }
        c.dump(12, pr);
        c.r2c(pr, tmpF, edge); c.put_edge(3, edge);
#pragma unroll
        for (int e = 0; e < E; ++e) tmpF[e] = cscale(tmpF[e], ce);
        c.put_g(2, tmpF);                                   // G2 = ce F(p21)
    }

    real w[P];
    c.c2r(PF_W, w);
    c.dump(PF_W, w);
    cplx<real> FP1[E], FP2[E];
    {
        real d[P], pr[P];
        c.c2r(PF_UX, d);
        c.dump(PF_UX, d);
        // P1 = -w r2 - S^2 r1 + lambda S du/dx   (r1nonl_func, Qsolver.cuh:217-255)
#pragma unroll
        for (int q = 0; q < P; ++q) pr[q] = (-w[q] * r2[q] - S[q] * S[q] * r1[q]) + lam * S[q] * d[q];
        c.r2c(pr, FP1, edge); c.put_edge(4, edge);
        c.c2r(PF_SH, d);
        c.dump(PF_SH, d);
        // P2 = w r1 - S^2 r2 + lambda/2 S (du/dy + dv/dx)   (r2nonl_func, Qsolver.cuh:257-300)
#pragma unroll
        for (int q = 0; q < P; ++q) pr[q] = (w[q] * r1[q] - S[q] * S[q] * r2[q]) + (real)0.5 * lam * S[q] * d[q];
        c.r2c(pr, FP2, edge); c.put_edge(7, edge);
    }
    {
        real u[P], pr[P];
        c.c2r(PF_U, u);
        c.dump(PF_U, u);
#pragma unroll
        for (int q = 0; q < P; ++q) pr[q] = -u[q] * r1[q];
        c.r2c(pr, tmpF, edge); c.put_edge(5, edge);
#pragma unroll
        for (int e = 0; e < E; ++e) tmpF[e] = cadd(FP1[e], cmul_i(cscale(tmpF[e], c.kx_of(e))));
        c.put_g(3, tmpF);                                   // G3 = F(P1) + i kx F(-u r1)
#pragma unroll
        for (int q = 0; q < P; ++q) pr[q] = -u[q] * r2[q];
        c.r2c(pr, tmpF, edge); c.put_edge(8, edge);
#pragma unroll
        for (int e = 0; e < E; ++e) tmpF[e] = cadd(FP2[e], cmul_i(cscale(tmpF[e], c.kx_of(e))));
        c.put_g(5, tmpF);                                   // G5 = F(P2) + i kx F(-u r2)
        if (a.advect) {
#pragma unroll
            for (int q = 0; q < P; ++q) pr[q] = -u[q] * w[q];
            c.r2c(pr, tmpF, edge);
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const real kx = c.kx_of(e);
                tmpF[e] = cadd(cmul_i(cscale(tmpF[e], kx)), cscale(F12[e], -ce * kx * kx));
            }
        } else {
#pragma unroll
            for (int e = 0; e < E; ++e) { const real kx = c.kx_of(e); tmpF[e] = cscale(F12[e], -ce * kx * kx); }
        }
        c.put_g(0, tmpF);                                   // G0 = i kx F(-u w) - ce kx^2 F(p12)
    }
    {
        real v[P], pr[P];
        c.c2r(PF_V, v);
        c.dump(PF_V, v);
#pragma unroll
        for (int q = 0; q < P; ++q) pr[q] = -v[q] * r1[q];
        c.r2c(pr, tmpF, edge); c.put_edge(6, edge);
#pragma unroll
        for (int e = 0; e < E; ++e) tmpF[e] = cmul_i(tmpF[e]);
        c.put_g(4, tmpF);                                   // G4 = i F(-v r1)
#pragma unroll
        for (int q = 0; q < P; ++q) pr[q] = -v[q] * r2[q];
        c.r2c(pr, tmpF, edge); c.put_edge(9, edge);
#pragma unroll
        for (int e = 0; e < E; ++e) tmpF[e] = cmul_i(tmpF[e]);
        c.put_g(6, tmpF);                                   // G6 = i F(-v r2)
        if (a.advect) {
#pragma unroll
            for (int q = 0; q < P; ++q) pr[q] = -v[q] * w[q];
            c.r2c(pr, tmpF, edge); c.put_edge(0, edge);
#pragma unroll
            for (int e = 0; e < E; ++e)
                tmpF[e] = cadd(cmul_i(tmpF[e]), cscale(F11[e], 2 * ce * c.kx_of(e)));
        } else {
            c.put_edge(0, mk<real>(0, 0));
#pragma unroll
            for (int e = 0; e < E; ++e) tmpF[e] = cscale(F11[e], 2 * ce * c.kx_of(e));
        }
        c.put_g(1, tmpF);                                   // G1 = i F(-v w) + 2 ce kx F(p11)
    }
}

// ---------------------------------------------------------------------------
// Layout conversion between the reference's spectral layout (i + j*(N/2+1))
// and the internal split layout (main[j*H + i], nyq[j]).
// ---------------------------------------------------------------------------
template <typename real>
__global__ void ref_to_internal(const cplx<real>* __restrict__ ref, cplx<real>* __restrict__ m, cplx<real>* __restrict__ nq, int N) {
    const int H = N / 2, nxh = H + 1;
    const size_t total = (size_t)nxh * N;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < total; k += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(k / nxh), i = (int)(k % nxh);
        if (i < H) m[(size_t)j * H + i] = ref[k];
        else nq[j] = ref[k];
    }
}

template <typename real>
__global__ void internal_to_ref(const cplx<real>* __restrict__ m, const cplx<real>* __restrict__ nq, cplx<real>* __restrict__ ref, int N) {
    const int H = N / 2, nxh = H + 1;
    const size_t total = (size_t)nxh * N;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < total; k += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(k / nxh), i = (int)(k % nxh);
        ref[k] = (i < H) ? m[(size_t)j * H + i] : nq[j];
    }
}

}  // namespace qaf
