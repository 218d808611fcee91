// qaf_kernels.cuh — column and row kernels of the fused IF-RK stage
// (see qaf_stage.cuh for the data flow and layouts).
#pragma once

#include "qaf_stage.cuh"

namespace qaf {

// Select one of three pointers without indexing the kernel-parameter array
// with a runtime value (which would copy the array to local memory).
template <typename P>
__device__ __forceinline__ P pick3(const P (&arr)[3], int f) { return f == 0 ? arr[0] : (f == 1 ? arr[1] : arr[2]); }

// ---------------------------------------------------------------------------
// Column kernel, regular tiles: W packed kx-columns i of field f.
// ---------------------------------------------------------------------------
template <typename real, int N, int W, int E>
__device__ __forceinline__ void col_regular(const StageArgs<real>& a, int f, int i, int t, int w, cplx<real>* buf) {
    constexpr int H = N / 2, TEAM = N / E;
    XchgCols<real> x{buf, w, W};
    TeamFFT<real, N, E> fft;
    fft.template init<N>(t, a.tw);
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
            fft.template run<false>(t, v, x);
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
                for (int e = 0; e < E; ++e) pick3(a.nl_m, f)[(size_t)(t + TEAM * e) * H + i] = nl[e];
            return;
        }
    }

    // stage update
    const bool need_old = a.mode == MODE_PROLOGUE || a.integrator == INT_IFE ||
                          (a.integrator == INT_IFRK4 && a.stage <= 3) || (a.integrator == INT_IFRK2 && a.stage == 1);
    const bool need_acc = a.mode == MODE_STAGE && ((a.integrator == INT_IFRK4 && a.stage >= 2) ||
                                                   (a.integrator == INT_IFRK2 && a.stage == 2));
    cplx<real>* om = pick3(a.old_m, f);
    cplx<real>* am = pick3(a.acc_m, f);
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
            // CTAs of the smallest grids hold partial warps: reduce with warp
            // shuffles only when every warp is full
            const bool full_warps = (blockDim.x & 31) == 0;
            if (full_warps) {
                if (a.flags && __any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(a.flags, 1u);
                if (f == 0 && a.diag) {
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) {
                        zsum += __shfl_xor_sync(0xffffffffu, zsum, o);
                        esum += __shfl_xor_sync(0xffffffffu, esum, o);
                    }
                    if ((threadIdx.x & 31) == 0) { atomicAdd(&a.diag[0], zsum); atomicAdd(&a.diag[1], esum); }
                }
            } else {
                if (a.flags && bad) atomicOr(a.flags, 1u);
                if (f == 0 && a.diag) { atomicAdd(&a.diag[0], zsum); atomicAdd(&a.diag[1], esum); }
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
        fft.template run<true>(t, v, x);
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
    TeamFFT<real, N, E> fft;
    fft.template init<N>(t, a.tw);
    const real kN = a.dkx * (real)H;
    const real s = (real)1 / ((real)N * (real)N);
    cplx<real> v[E];
    // N^ of columns kx = 0 (ctab[j]) and kx = N/2 (ctab[N + j]), summed over
    // the products in shared memory; team 0 owns every j of a column
    if (w == 0)
#pragma unroll
        for (int e = 0; e < E; ++e) { ctab[t + TEAM * e] = mk<real>(0, 0); ctab[N + t + TEAM * e] = mk<real>(0, 0); }

    if (a.mode != MODE_PROLOGUE) {
        const int pbase = f == 0 ? 0 : (f == 1 ? 4 : 7);
        const int np = f == 0 ? 4 : 3;
#pragma unroll 1
        for (int base = 0; base < np; base += W) {
            const bool active = base + w < np;
            const int p = pbase + (active ? base + w : 0);
#pragma unroll
            for (int e = 0; e < E; ++e) v[e] = active ? a.Ed[(size_t)p * N + t + TEAM * e] : mk<real>(0, 0);
            fft.template run<false>(t, v, x);
            // unpack the two real sequences: DC = (Z[j] + conj Z[-j]) / 2, NYQ = (Z[j] - conj Z[-j]) / 2i
            cplx<real> zm[E];
#pragma unroll
            for (int e = 0; e < E; ++e) x.write(t + TEAM * e, v[e]);
            x.sync();
#pragma unroll
            for (int e = 0; e < E; ++e) zm[e] = cconj(x.read((N - t - TEAM * e) % N));
            x.sync();
            // the kx = 0 then the kx = N/2 contribution of each team, summed by team 0
#pragma unroll 1
            for (int col = 0; col < 2; ++col) {
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const int j = t + TEAM * e;
                    cplx<real> m0, mH;
                    edge_product_mults<real>(p, ky_of<real>(j, N, a.dky), kN, a.ce, j, N, a.advect, m0, mH);
                    cplx<real> c;
                    if (col == 0) c = cmul(cscale(cadd(v[e], zm[e]), (real)0.5), m0);
                    else c = cmul(cmul_mi(cscale(csub(v[e], zm[e]), (real)0.5)), mH);
                    x.write(j, active ? c : mk<real>(0, 0));
                }
                x.sync();
                if (w == 0)
#pragma unroll
                    for (int e = 0; e < E; ++e) {
                        const int j = t + TEAM * e;
                        cplx<real> acc = ctab[col * N + j];
                        for (int ww = 0; ww < W; ++ww) acc = cadd(acc, buf[j * W + ww]);
                        ctab[col * N + j] = acc;
                    }
                x.sync();
            }
        }
    }

    if (w == 0) {
        cplx<real>* om = pick3(a.old_m, f);
        cplx<real>* on = pick3(a.old_n, f);
        cplx<real>* am = pick3(a.acc_m, f);
        cplx<real>* an = pick3(a.acc_n, f);
        if (a.mode == MODE_NONL) {
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int j = t + TEAM * e;
                pick3(a.nl_m, f)[(size_t)j * H] = ctab[j];
                pick3(a.nl_n, f)[j] = ctab[N + j];
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
                    StageUpdate<real> u = stage_update(a, ctab[j], o, ac, Ef, Eh, mask_keep(a, 0, j));
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
                    StageUpdate<real> u = stage_update(a, ctab[N + j], o, ac, Ef, Eh, mask_keep(a, H, j));
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
        fft.template run<true>(t, v, x);
        if (active)
#pragma unroll
            for (int e = 0; e < E; ++e) a.D[(size_t)p * N + t + TEAM * e] = v[e];
    }
}

template <typename real, int N, int W, int E, int MINB>
__global__ void __launch_bounds__(W * (N / E), MINB) col_kernel(const StageArgs<real> a) {
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
// Row kernel: ROWS rows per CTA, a team of N/E threads per row.
//
// Real transforms are done two at a time as one length-N complex FFT:
//   C2R pair (a, b):  z = IFFT_N(A + i B) = a + i b, with A, B the Hermitian
//                     extensions of the two half spectra
//   R2C pair (p, q):  Z = FFT_N(p + i q); P[k] = (Z[k] + conj Z[N-k]) / 2,
//                     Q[k] = (Z[k] - conj Z[N-k]) / 2i
// so a stage's 9 C2Rs and 11 R2Cs take 5 + 6 transforms. After a transform
// thread t holds the points m = t + TEAM*e, the same for every transform, so
// all physical products are thread-local; the fields needed across
// transforms (r1, r2, w, p21) stay in shared memory at [field][m].
// G arrays fed by two products are completed by a read-modify-write of the
// row the same thread wrote earlier in this kernel.
// ---------------------------------------------------------------------------
template <typename real, int TEAM, bool NAMED>
struct XchgTeam {
    cplx<real>* buf;
    int id;
    __device__ void write(int idx, cplx<real> v) { buf[idx] = v; }
    __device__ cplx<real> read(int idx) const { return buf[idx]; }
    __device__ void sync() {
        if constexpr (NAMED) asm volatile("bar.sync %0, %1;" ::"r"(id), "n"(TEAM) : "memory");
        else __syncthreads();
    }
};

template <typename real, int N, int E, int ROWS>
struct RowKernel {
    static constexpr int H = N / 2, TEAM = N / E, PH = E / 2;
    // a named barrier per row team when teams are whole warps and there is more than one team
    static constexpr bool NAMED = (TEAM % 32 == 0) && ROWS > 1 && ROWS <= 15;
    using X = XchgTeam<real, TEAM, NAMED>;
    static constexpr int NKEEP = 5;   // r1, r2, w, two scratch products
    static constexpr size_t SMEM_PER_ROW = N * sizeof(cplx<real>) + NKEEP * N * sizeof(real);
    static constexpr size_t SMEM = ROWS * SMEM_PER_ROW;

    const StageArgs<real>& a;
    int n, t;
    X x;
    real* keep;            // [NKEEP][N], point m at [slot][m]
    TeamFFT<real, N, E> fft;

    __device__ cplx<real> yv(int q, int k) const { return a.Y[(size_t)q * N * H + (size_t)n * H + k]; }

    // half spectrum of physical field p at x wave number k in [1, H)
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
    // Hermitian-extended spectrum entry k in [0, N) of field p (p < 0: zero field)
    __device__ cplx<real> full(int p, int k, cplx<real> d) const {
        if (p < 0) return mk<real>(0, 0);
        if (k == 0) return mk<real>(d.x, 0);
        if (k == H) return mk<real>(d.y, 0);
        if (k < H) return xspec(p, k);
        return cconj(xspec(p, N - k));
    }

    // C2R pair: v[e] = (field pa, field pb) at point m = t + TEAM e
    __device__ void c2r(int pa, int pb, cplx<real> (&v)[E]) {
        const cplx<real> da = a.D[(size_t)pa * N + n];
        const cplx<real> db = pb >= 0 ? a.D[(size_t)pb * N + n] : mk<real>(0, 0);
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int k = t + TEAM * e;
            const cplx<real> A = full(pa, k, da), B = full(pb, k, db);
            v[e] = mk<real>(A.x - B.y, A.y + B.x);   // A + i B
        }
        fft.template run<true>(t, v, x);
    }

    // R2C pair of v = (p, q): emit(k, P[k], Q[k], ga[e], gb[e]) for k = t + TEAM e in
    // [1, H), with ga, gb rows prefetched by the caller (passed through, so that
    // no lambda captures a register array); the packed (DC, Nyquist) of p and q
    // go to edge slots ep, eq (< 0: none)
    template <class F>
    __device__ void r2c(cplx<real> (&v)[E], int ep, int eq, const cplx<real> (&ga)[PH], const cplx<real> (&gb)[PH],
                        F&& emit) {
        fft.template run<false>(t, v, x);
#pragma unroll
        for (int e = 0; e < E; ++e) x.write(t + TEAM * e, v[e]);
        x.sync();
#pragma unroll
        for (int e = 0; e < PH; ++e) {
            const int k = t + TEAM * e;
            if (k == 0) continue;
            const cplx<real> z = x.read(k), zm = cconj(x.read(N - k));
            emit(k, cscale(cadd(z, zm), (real)0.5), cmul_mi(cscale(csub(z, zm), (real)0.5)), ga[e], gb[e]);
        }
        if (t == 0) {
            const cplx<real> z0 = x.read(0), zh = x.read(H);
            if (ep >= 0) a.Ed[(size_t)ep * N + n] = mk<real>(z0.x, zh.x);
            if (eq >= 0) a.Ed[(size_t)eq * N + n] = mk<real>(z0.y, zh.y);
        }
        x.sync();
    }

    __device__ cplx<real>* grow(int g) const { return a.G + (size_t)g * N * H + (size_t)n * H; }
    __device__ real& kp(int f, int e) const { return keep[f * N + t + TEAM * e]; }
    __device__ void zero_slot0(int g) const { if (t == 0) grow(g)[0] = mk<real>(0, 0); }
    __device__ void dump(int fld, const cplx<real> (&v)[E], bool imag) const {
        if (!a.phys_out) return;
        real* o = a.phys_out + (size_t)fld * N * N + (size_t)n * N;
#pragma unroll
        for (int e = 0; e < E; ++e) o[t + TEAM * e] = imag ? v[e].y : v[e].x;
    }
    __device__ void dump_slot(int fld, int slot) const {
        if (!a.phys_out) return;
        real* o = a.phys_out + (size_t)fld * N * N + (size_t)n * N;
#pragma unroll
        for (int e = 0; e < E; ++e) o[t + TEAM * e] = kp(slot, e);
    }
    __device__ real alpha_at(int e) const {
        return a.alpha_field ? a.alpha_field[(size_t)n * N + t + TEAM * e] : a.alpha;
    }
    __device__ real S_at(int e) const {
        const real r1 = kp(0, e), r2 = kp(1, e);
        return 2 * sqrt(r1 * r1 + r2 * r2);   // S_func (Qsolver.cuh:63-71)
    }

    __device__ void run() {
        const real lam = a.lambda, ce = a.ce, dkx = a.dkx;
        const bool adv = a.advect != 0;
        cplx<real> v[E], g0v[PH], g1v[PH];
#pragma unroll
    for (int e = 0; e < PH; ++e) { g0v[e] = mk<real>(0, 0); g1v[e] = g0v[e]; }
        fft.template init<N>(t, a.tw);
        for (int g = 0; g < NG; ++g) zero_slot0(g);

        // 1. r1, r2 -> slots 0, 1
        c2r(PF_R1, PF_R2, v);
#pragma unroll
        for (int e = 0; e < E; ++e) { kp(0, e) = v[e].x; kp(1, e) = v[e].y; }
        dump(PF_R1, v, false); dump(PF_R2, v, true);

        // 2. Lap r1, Lap r2 -> (p11, p12) transformed now, p21 to slot 4
        //    single + Rar + cross of p11func/p12func/p21func (Qsolver.cuh:75-151)
        c2r(PF_LR1, PF_LR2, v);
        dump(PF_LR1, v, false); dump(PF_LR2, v, true);
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const real r1 = kp(0, e), r2 = kp(1, e), L1 = v[e].x, L2 = v[e].y, al = alpha_at(e);
            const real S = 2 * sqrt(r1 * r1 + r2 * r2);
            const real sgl = lam * S * (S * S - 1);
            const real sg2 = -lam * L2 * S + sgl * r2;
            const real p11 = -lam * L1 * S + sgl * r1 - al * r1;
            const real p12 = sg2 + (2 * L1 * r2 - 2 * r1 * L2) - al * r2;
            kp(4, e) = sg2 + (2 * L2 * r1 - 2 * r2 * L1) - al * r2;
            v[e] = mk<real>(p11, p12);
            if (a.phys_out) kp(3, e) = S;
        }
        if (a.phys_out) { dump_slot(9, 3); dump(10, v, false); dump(11, v, true); dump_slot(12, 4); }
        {
            cplx<real>* g0 = grow(0); cplx<real>* g1 = grow(1);
            r2c(v, 1, 2, g0v, g1v, [=](int k, cplx<real> P, cplx<real> Q, cplx<real>, cplx<real>) {
                const real kx = dkx * (real)k;
                g1[k] = cscale(P, 2 * ce * kx);    // 2 ce kx F(p11)
                g0[k] = cscale(Q, -ce * kx * kx);  // -ce kx^2 F(p12)
            });
        }

        // 3. w, u -> w to slot 2, (-u r1, -u r2) transformed now, then (p21, -u w)
        c2r(PF_W, PF_U, v);
        dump(PF_W, v, false); dump(PF_U, v, true);
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const real w = v[e].x, u = v[e].y, r1 = kp(0, e), r2 = kp(1, e);
            kp(2, e) = w;
            kp(3, e) = adv ? -u * w : (real)0;
            v[e] = mk<real>(-u * r1, -u * r2);
        }
        {
            cplx<real>* g3 = grow(3); cplx<real>* g5 = grow(5);
            r2c(v, 5, 8, g0v, g1v, [=](int k, cplx<real> P, cplx<real> Q, cplx<real>, cplx<real>) {
                const real kx = dkx * (real)k;
                g3[k] = cmul_i(cscale(P, kx));   // i kx F(-u r1)
                g5[k] = cmul_i(cscale(Q, kx));   // i kx F(-u r2)
            });
        }
#pragma unroll
        for (int e = 0; e < E; ++e) v[e] = mk<real>(kp(4, e), kp(3, e));
        {
            cplx<real>* g0 = grow(0); cplx<real>* g2 = grow(2);
#pragma unroll
            for (int e = 0; e < PH; ++e) g0v[e] = g0[t + TEAM * e];
            r2c(v, 3, -1, g0v, g1v, [=](int k, cplx<real> P, cplx<real> Q, cplx<real> ga, cplx<real>) {
                const real kx = dkx * (real)k;
                g2[k] = cscale(P, ce);                                   // ce F(p21)
                g0[k] = adv ? cadd(ga, cmul_i(cscale(Q, kx))) : ga;      // + i kx F(-u w)
            });
        }

        // 4. v, du/dx -> (-v r1, -v r2) transformed now, then (-v w, P1)
        c2r(PF_V, PF_UX, v);
        dump(PF_V, v, false); dump(PF_UX, v, true);
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const real vv = v[e].x, ux = v[e].y, r1 = kp(0, e), r2 = kp(1, e), w = kp(2, e);
            const real S = 2 * sqrt(r1 * r1 + r2 * r2);
            kp(3, e) = adv ? -vv * w : (real)0;
            // P1 = -w r2 - S^2 r1 + lambda S du/dx (r1nonl_func, Qsolver.cuh:217-255)
            kp(4, e) = (-w * r2 - S * S * r1) + lam * S * ux;
            v[e] = mk<real>(-vv * r1, -vv * r2);
        }
        {
            cplx<real>* g4 = grow(4); cplx<real>* g6 = grow(6);
            r2c(v, 6, 9, g0v, g1v, [=](int k, cplx<real> P, cplx<real> Q, cplx<real>, cplx<real>) {
                g4[k] = cmul_i(P);    // i F(-v r1)
                g6[k] = cmul_i(Q);    // i F(-v r2)
            });
        }
#pragma unroll
        for (int e = 0; e < E; ++e) v[e] = mk<real>(kp(3, e), kp(4, e));
        {
            cplx<real>* g1 = grow(1); cplx<real>* g3 = grow(3);
#pragma unroll
            for (int e = 0; e < PH; ++e) { g0v[e] = g1[t + TEAM * e]; g1v[e] = g3[t + TEAM * e]; }
            r2c(v, 0, 4, g0v, g1v, [=](int k, cplx<real> P, cplx<real> Q, cplx<real> ga, cplx<real> gb) {
                g1[k] = adv ? cadd(ga, cmul_i(P)) : ga;   // + i F(-v w)
                g3[k] = cadd(gb, Q);                      // + F(P1)
            });
        }

        // 5. du/dy + dv/dx -> P2
        c2r(PF_SH, -1, v);
        dump(PF_SH, v, false);
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const real sh = v[e].x, r1 = kp(0, e), r2 = kp(1, e), w = kp(2, e);
            const real S = 2 * sqrt(r1 * r1 + r2 * r2);
            // P2 = w r1 - S^2 r2 + lambda/2 S (du/dy + dv/dx) (r2nonl_func, Qsolver.cuh:257-300)
            v[e] = mk<real>((w * r1 - S * S * r2) + (real)0.5 * lam * S * sh, 0);
        }
        {
            cplx<real>* g5 = grow(5);
#pragma unroll
            for (int e = 0; e < PH; ++e) g0v[e] = g5[t + TEAM * e];
            r2c(v, 7, -1, g0v, g1v, [=](int k, cplx<real> P, cplx<real>, cplx<real> ga, cplx<real>) {
                g5[k] = cadd(ga, P);   // + F(P2)
            });
        }
    }
};

template <typename real, int N, int E, int ROWS, int MINB>
__global__ void __launch_bounds__(ROWS * (N / E), MINB) row_kernel(const StageArgs<real> a) {
    using K = RowKernel<real, N, E, ROWS>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int r = threadIdx.x / K::TEAM, t = threadIdx.x % K::TEAM;
    unsigned char* mine = smem_raw + (size_t)r * K::SMEM_PER_ROW;
    K k{a, (int)blockIdx.x * ROWS + r, t,
        typename K::X{reinterpret_cast<cplx<real>*>(mine), 1 + r},
        reinterpret_cast<real*>(mine + N * sizeof(cplx<real>)), {}};
    static_assert(K::PH * K::TEAM == N / 2, "row team layout");
    k.run();
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
