// qaf_adjoint.cuh — discrete adjoint of the IF-RK4 step (two kernels per stage).
//
// The forward map of one step is the reference's literal sequence
// (friction.cu:212-259 with RK4.cuh:12-74 and the nonlinear terms of
// friction/Qsolver.cuh:63-312): spectral multipliers, BwdTrans B = C2R / N^2
// (with the Hermitian projection P of the kx = 0 and kx = N/2 columns that
// cufftExecZ2D applies), pointwise products, FwdTrans F = R2C. Every piece but
// the products is real-linear; under the real inner product
// <a, b> = Re sum conj(a) b over the stored half spectrum
//     F^T(a) = C2R(W a)            W = 1 on the edge columns, 1/2 elsewhere
//     B^T(y) = c R2C(y) / N^2      c = 1 on the edge columns, 2 elsewhere
//     (m .)^T = conj(m) .,  P^T = P,
// so the adjoint of a stage's nonlinear term is (spectral) 11 multiplied
// y-iFFTs -> (row) 11 C2R, the transposed products against the forward
// fields of that stage, 9 R2C -> (spectral) 9 y-FFTs combined with the
// conjugate multipliers. The column kernel also carries the RK4 adjoint
// recursion, so one column launch ends stage s and starts stage s - 1.
//
// With a = M sbar(n+1) (M the 2/3 mask) and E, Eh the full and half-step
// integrating factors of each field, the IF-RK4 adjoint is
//     kb4 = dt/6 a                         cb4 = VJP(c4, kb4)
//     kb3 = dt Eh cb4 + dt/3 Eh a          cb3 = VJP(c3, kb3)
//     kb2 = dt/2 cb3 + dt/3 Eh a           cb2 = VJP(c2, kb2)
//     kb1 = dt/2 Eh cb2 + dt/6 E a         cb1 = VJP(c1, kb1)
//     sbar(n) = E a + E cb4 + Eh cb3 + Eh cb2 + cb1   (+ the loss term of s(n)).
#pragma once

#include "qaf_stage.cuh"

namespace qaf {

// adjoint physical inputs g_q = C2R(W m_q lambda) of the products, in the
// order the forward's nonlinear terms are formed
enum AdjIn : int {
    GA_UW = 0,   // -u w   (wnonl advection, x part; projected)
    GA_VW,       // -v w   (y part; projected)
    GA_P11,      // p11 -> 2 ce kx ky
    GA_P12,      // p12 -> -ce kx^2
    GA_P21,      // p21 -> ce ky^2
    GA_A1,       // -w r2 - S^2 r1 + lambda S du/dx   (r1nonl)
    GA_UR1,      // -u r1  -> i kx
    GA_VR1,      // -v r1  -> i ky
    GA_A2,       // w r1 - S^2 r2 + lambda/2 S (du/dy + dv/dx)   (r2nonl)
    GA_UR2,      // -u r2
    GA_VR2,      // -v r2
    NGA
};

template <typename real>
struct AdjArgs {
    real dkx, dky, dt, lambda, ce;
    int advect, kx_keep, ky_lo, ky_hi;
    int trunc;                 // fields the 2/3 mask truncates: bit f for field f
    const cplx<real>* tw;
    const real* ex;
    const real* ey;
    real e0[4];
    cplx<real>* Tg;            // NGA arrays of N*H: column kernel -> row kernel
    cplx<real>* Tx;            // PF_COUNT arrays of N*H: row kernel -> column kernel
    cplx<real>* abar[3];       // M sbar(n+1), reference layout
    cplx<real>* sacc[3];       // partial sums of sbar(n)
    cplx<real>* sbar[3];       // the adjoint state
    cplx<real>* edge;          // 6 * N scratch: kb of the kx = 0 and kx = N/2 columns
    const cplx<real>* wstate;  // w of the state whose adjoint completes in this launch (loss term) or nullptr
    real loss_w;               // d loss / d enstrophy of that state
    const real* loss_wv;       // per instance instead of loss_w, or nullptr
    int stage;                 // 4..1: Tx holds the transposed products of this stage; 0: start from sbar
    int emit;                  // write Tg for the stage before
    const real* phys;          // the stage input's forward fields (PhysField order, N*N each)
    const real* alpha_field;   // activity field or nullptr (alpha)
    real alpha;
    real* alpha_grad;          // += d loss / d alpha(x), or nullptr
    // batches of instances (field-parallel kernels): instance k's data at these offsets
    int ninst;                 // instances in the launch (1: a single grid)
    size_t s_istride;          // complex elements: abar, sacc, sbar, wstate
    size_t tg_istride;         // complex elements: Tg
    size_t tx_istride;         // complex elements: Tx
    size_t p_istride;          // reals: phys
    size_t a_istride;          // reals: alpha_field (0: one field for all)
    size_t g_istride;          // reals: alpha_grad
};

// conj(multiplier) of the forward field p (derived()) applied to the transform of its adjoint
template <typename real>
__device__ __forceinline__ void adj_combine(int p, cplx<real> v, real kx, real ky, real ik2, cplx<real>& cw,
                                            cplx<real>& c1, cplx<real>& c2) {
    switch (p) {
        case PF_W: cw = cadd(cw, v); break;
        case PF_R1: c1 = cadd(c1, v); break;
        case PF_R2: c2 = cadd(c2, v); break;
        case PF_U: cw = cadd(cw, cmul_mi(cscale(v, ky * ik2))); break;        // conj(i ky / k^2)
        case PF_V: cw = cadd(cw, cmul_i(cscale(v, kx * ik2))); break;         // conj(-i kx / k^2)
        case PF_UX: cw = cadd(cw, cscale(v, -kx * ky * ik2)); break;
        case PF_SH: cw = cadd(cw, cscale(v, (kx * kx - ky * ky) * ik2)); break;
        case PF_LR1: c1 = cadd(c1, cscale(v, -(kx * kx + ky * ky))); break;
        default: c2 = cadd(c2, cscale(v, -(kx * kx + ky * ky))); break;   // PF_LR2
    }
}

// field of the adjoint state that the transposed product p feeds (0 w, 1 r1, 2 r2)
__host__ __device__ constexpr int adj_target(int p) {
    return (p == PF_R1 || p == PF_LR1) ? 1 : ((p == PF_R2 || p == PF_LR2) ? 2 : 0);
}

// conj(multiplier) of the forward field p applied to the transform v of its adjoint
template <typename real>
__device__ __forceinline__ cplx<real> adj_cmult(int p, cplx<real> v, real kx, real ky, real ik2) {
    switch (p) {
        case PF_U: return cmul_mi(cscale(v, ky * ik2));
        case PF_V: return cmul_i(cscale(v, kx * ik2));
        case PF_UX: return cscale(v, -kx * ky * ik2);
        case PF_SH: return cscale(v, (kx * kx - ky * ky) * ik2);
        case PF_LR1: case PF_LR2: return cscale(v, -(kx * kx + ky * ky));
        default: return v;   // PF_W, PF_R1, PF_R2
    }
}

// conj(multiplier) that maps the nonlinear adjoint lambda of field f(q) to g_q's spectrum
template <typename real>
__device__ __forceinline__ cplx<real> adj_emit(int q, cplx<real> lw, cplx<real> l1, cplx<real> l2, real kx, real ky,
                                               real ce) {
    switch (q) {
        case GA_UW: return cmul_mi(cscale(lw, kx));
        case GA_VW: return cmul_mi(cscale(lw, ky));
        case GA_P11: return cscale(lw, 2 * ce * kx * ky);
        case GA_P12: return cscale(lw, -ce * kx * kx);
        case GA_P21: return cscale(lw, ce * ky * ky);
        case GA_A1: return l1;
        case GA_UR1: return cmul_mi(cscale(l1, kx));
        case GA_VR1: return cmul_mi(cscale(l1, ky));
        case GA_A2: return l2;
        case GA_UR2: return cmul_mi(cscale(l2, kx));
        default: return cmul_mi(cscale(l2, ky));                          // GA_VR2
    }
}

// The RK4 adjoint recursion at one spectral point of field f, in two parts:
// adj_rk_load reads the accumulators the stage needs — sbar (stage 0), sacc
// (stage 1), abar and sacc (stages 2-4) — and adj_rk_apply updates them. The
// callers load every field before any field's stores, so that the loads
// overlap (the compiler cannot move them across stores it cannot prove
// disjoint). cb: the VJP of the stage (unused at stage 0); adj_rk_apply
// returns the nonlinear adjoint kb of the stage before. lossg: the loss
// gradient of the state completed here.
template <typename real>
struct AdjHeld {
    cplx<real> x, y;
};

template <typename real>
__device__ __forceinline__ AdjHeld<real> adj_rk_load(const AdjArgs<real>& a, int f, size_t idx) {
    AdjHeld<real> h;
    h.y = mk<real>(0, 0);
    if (a.stage == 0) h.x = pick3(a.sbar, f)[idx];
    else if (a.stage == 1) h.x = pick3(a.sacc, f)[idx];
    else { h.x = pick3(a.abar, f)[idx]; h.y = pick3(a.sacc, f)[idx]; }
    return h;
}

template <typename real>
__device__ __forceinline__ cplx<real> adj_rk_apply(const AdjArgs<real>& a, int f, size_t idx, AdjHeld<real> h,
                                                   cplx<real> cb, real E, real Eh, bool keep, cplx<real> lossg) {
    const real dt = a.dt;
    const real sixth = (real)(1.0 / 6.0), third = (real)(1.0 / 3.0), half = (real)0.5;
    cplx<real> sb;
    if (a.stage == 0) {
        sb = cadd(h.x, lossg);
    } else if (a.stage == 1) {
        sb = cadd(cadd(h.x, cb), lossg);
        pick3(a.sbar, f)[idx] = sb;
    } else {
        const cplx<real> av = h.x;
        cplx<real> sc = h.y;
        cplx<real> kb;
        if (a.stage == 4) {
            sc = cadd(sc, cscale(cb, E));
            kb = cadd(cscale(cb, dt * Eh), cscale(av, third * dt * Eh));
        } else if (a.stage == 3) {
            sc = cadd(sc, cscale(cb, Eh));
            kb = cadd(cscale(cb, half * dt), cscale(av, third * dt * Eh));
        } else {
            sc = cadd(sc, cscale(cb, Eh));
            kb = cadd(cscale(cb, half * dt * Eh), cscale(av, sixth * dt * E));
        }
        pick3(a.sacc, f)[idx] = sc;
        return kb;
    }
    // stages 0 and 1 start the step before: a = M sbar, sacc = E a, kb4 = dt/6 a
    if (!a.emit) return mk<real>(0, 0);
    const cplx<real> av = keep ? sb : mk<real>(0, 0);
    pick3(a.abar, f)[idx] = av;
    pick3(a.sacc, f)[idx] = cscale(av, E);
    return cscale(av, sixth * dt);
}

template <typename real, int N>
__device__ __forceinline__ void adj_factors(const AdjArgs<real>& a, int f, int i, int j, real& E, real& Eh) {
    constexpr int H = N / 2;
    const int cls = f == 0 ? 0 : 2;
    E = __ldg(&a.ex[cls * (H + 1) + i]) * a.e0[cls] * __ldg(&a.ey[cls * N + j]);
    Eh = __ldg(&a.ex[(cls + 1) * (H + 1) + i]) * a.e0[cls + 1] * __ldg(&a.ey[(cls + 1) * N + j]);
}

template <typename real>
__device__ __forceinline__ bool adj_keep(const AdjArgs<real>& a, int f, int i, int j) {
    return !((a.trunc >> f) & 1) || (i <= a.kx_keep && (j <= a.ky_lo || j >= a.ky_hi));
}

// kx = 0 and kx = N/2 columns (packed in slot 0 of the T arrays as DC + i Nyquist), by the first team of the last block
template <typename real, int N, int W, int E>
__device__ void adj_col_edge(const AdjArgs<real>& a, const TeamFFT<real, N, E>& fft, cplx<real>* buf, int w, int t) {
    constexpr int H = N / 2, TEAM = N / E, NXH = H + 1;
    XchgCols<real> x{buf, w, W};
    const bool lead = w == 0;
    const real kN = a.dkx * (real)H;
    const real sc = (real)1 / ((real)N * (real)N);
    const real n4 = sc * sc;
#pragma unroll 1
    for (int c = 0; c < 2; ++c) {
        const int i = c == 0 ? 0 : H;
        const real kx = c == 0 ? (real)0 : kN;
        cplx<real> cw[E], c1[E], c2[E];
#pragma unroll
        for (int e = 0; e < E; ++e) { cw[e] = mk<real>(0, 0); c1[e] = cw[e]; c2[e] = cw[e]; }
        if (a.stage >= 1) {
#pragma unroll 1
            for (int p = 0; p < PF_COUNT; ++p) {
                cplx<real> v[E];
#pragma unroll
                for (int e = 0; e < E; ++e)
                    v[e] = lead ? a.Tx[(size_t)p * N * H + (size_t)(t + TEAM * e) * H] : mk<real>(0, 0);
                fft.template run<false>(t, v, x);
#pragma unroll
                for (int e = 0; e < E; ++e) x.write(t + TEAM * e, v[e]);
                x.sync();
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const int j = t + TEAM * e;
                    const cplx<real> zm = cconj(x.read((N - j) % N));
                    const cplx<real> z = c == 0 ? cscale(cadd(v[e], zm), (real)0.5)
                                                : cmul_mi(cscale(csub(v[e], zm), (real)0.5));
                    const real ky = ky_of<real>(j, N, a.dky);
                    const real k2 = kx * kx + ky * ky;
                    adj_combine<real>(p, z, kx, ky, k2 > 0 ? (real)1 / k2 : (real)0, cw[e], c1[e], c2[e]);
                }
                x.sync();
            }
        }
        if (lead) {
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int j = t + TEAM * e, jm = (N - j) % N;
                const size_t idx = (size_t)j * NXH + i;
                cplx<real> lossg = mk<real>(0, 0);
                if (a.wstate) {
                    const cplx<real> P = cscale(cadd(a.wstate[idx], cconj(a.wstate[(size_t)jm * NXH + i])), (real)0.5);
                    lossg = cscale(P, a.loss_w * n4);
                }
                cplx<real> cb[3] = {cscale(cw[e], sc), cscale(c1[e], sc), cscale(c2[e], sc)};
                real Ef[3], Eh[3];
                AdjHeld<real> held[3];
#pragma unroll
                for (int f = 0; f < 3; ++f) {
                    adj_factors<real, N>(a, f, i, j, Ef[f], Eh[f]);
                    held[f] = adj_rk_load(a, f, idx);
                }
#pragma unroll
                for (int f = 0; f < 3; ++f) {
                    const cplx<real> kb = adj_rk_apply(a, f, idx, held[f], cb[f], Ef[f], Eh[f], adj_keep(a, f, i, j),
                                                       f == 0 ? lossg : mk<real>(0, 0));
                    a.edge[(size_t)(f * 2 + c) * N + j] = kb;
                }
            }
        }
    }
    __syncthreads();
    if (!a.emit) return;
#pragma unroll 1
    for (int q = 0; q < NGA; ++q) {
        if (!a.advect && q <= GA_VW) continue;
        cplx<real> v[E];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            v[e] = mk<real>(0, 0);
            if (!lead) continue;
            const int j = t + TEAM * e;
            cplx<real> P[2];
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const real kx = c == 0 ? (real)0 : kN;
                cplx<real> val[2];
#pragma unroll
                for (int s = 0; s < 2; ++s) {
                    const int jj = s == 0 ? j : (N - j) % N, jp = (N - jj) % N;
                    cplx<real> lw = a.edge[(size_t)c * N + jj];
                    if (q <= GA_VW)   // the advection terms are projected before the derivative's adjoint
                        lw = cscale(cadd(lw, cconj(a.edge[(size_t)c * N + jp])), (real)0.5);
                    const cplx<real> l1 = a.edge[(size_t)(2 + c) * N + jj], l2 = a.edge[(size_t)(4 + c) * N + jj];
                    val[s] = adj_emit<real>(q, lw, l1, l2, kx, ky_of<real>(jj, N, a.dky), a.ce);
                }
                P[c] = cscale(cadd(val[0], cconj(val[1])), (real)0.5);
            }
            v[e] = cadd(P[0], cmul_i(P[1]));
        }
        fft.template run<true>(t, v, x);
        if (lead)
#pragma unroll
            for (int e = 0; e < E; ++e) a.Tg[(size_t)q * N * H + (size_t)(t + TEAM * e) * H] = v[e];
    }
}

// One team of N/E threads per kx-column i in [1, H); the last block takes the edge columns.
template <typename real, int N, int W, int E>
__global__ void __launch_bounds__(W * (N / E)) adj_col_kernel(const __grid_constant__ AdjArgs<real> a) {
    constexpr int H = N / 2, TEAM = N / E, NXH = H + 1;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    cplx<real>* buf = reinterpret_cast<cplx<real>*>(smem_raw);
    const int w = threadIdx.x % W, t = threadIdx.x / W;
    TeamFFT<real, N, E> fft;
    fft.template init<N>(t, a.tw);
    if (blockIdx.x == gridDim.x - 1) {
        adj_col_edge<real, N, W, E>(a, fft, buf, w, t);
        return;
    }
    const int i = blockIdx.x * W + w;
    const bool active = i != 0;
    XchgCols<real> x{buf, w, W};
    const real kx = a.dkx * (real)i;
    const real sc = (real)2 / ((real)N * (real)N);
    cplx<real> cw[E], c1[E], c2[E];
#pragma unroll
    for (int e = 0; e < E; ++e) { cw[e] = mk<real>(0, 0); c1[e] = cw[e]; c2[e] = cw[e]; }
    if (a.stage >= 1) {
#pragma unroll 1
        for (int p = 0; p < PF_COUNT; ++p) {
            cplx<real> v[E];
#pragma unroll
            for (int e = 0; e < E; ++e)
                v[e] = active ? a.Tx[(size_t)p * N * H + (size_t)(t + TEAM * e) * H + i] : mk<real>(0, 0);
            fft.template run<false>(t, v, x);
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const real ky = ky_of<real>(t + TEAM * e, N, a.dky);
                const real k2 = kx * kx + ky * ky;
                adj_combine<real>(p, v[e], kx, ky, k2 > 0 ? (real)1 / k2 : (real)0, cw[e], c1[e], c2[e]);
            }
        }
    }
    if (active) {
        const real n4 = (real)1 / ((real)N * (real)N) / ((real)N * (real)N);
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int j = t + TEAM * e;
            const size_t idx = (size_t)j * NXH + i;
            const cplx<real> lossg = a.wstate ? cscale(a.wstate[idx], 2 * a.loss_w * n4) : mk<real>(0, 0);
            real Ef0, Eh0, Ef, Eh;
            adj_factors<real, N>(a, 0, i, j, Ef0, Eh0);
            adj_factors<real, N>(a, 1, i, j, Ef, Eh);
            const AdjHeld<real> h0 = adj_rk_load(a, 0, idx), h1 = adj_rk_load(a, 1, idx), h2 = adj_rk_load(a, 2, idx);
            cw[e] = adj_rk_apply(a, 0, idx, h0, cscale(cw[e], sc), Ef0, Eh0, adj_keep(a, 0, i, j), lossg);
            c1[e] = adj_rk_apply(a, 1, idx, h1, cscale(c1[e], sc), Ef, Eh, adj_keep(a, 1, i, j), mk<real>(0, 0));
            c2[e] = adj_rk_apply(a, 2, idx, h2, cscale(c2[e], sc), Ef, Eh, adj_keep(a, 2, i, j), mk<real>(0, 0));
        }
    }
    if (!a.emit) return;
#pragma unroll 1
    for (int q = 0; q < NGA; ++q) {
        if (!a.advect && q <= GA_VW) continue;
        cplx<real> v[E];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const real ky = ky_of<real>(t + TEAM * e, N, a.dky);
            v[e] = active ? cscale(adj_emit<real>(q, cw[e], c1[e], c2[e], kx, ky, a.ce), (real)0.5) : mk<real>(0, 0);
        }
        fft.template run<true>(t, v, x);
        if (active)
#pragma unroll
            for (int e = 0; e < E; ++e) a.Tg[(size_t)q * N * H + (size_t)(t + TEAM * e) * H + i] = v[e];
    }
}

// Field-parallel column kernel (grids up to 256^2): one team of N/E threads
// per (transform, kx-column) — NGA teams per column, W columns per CTA — so the
// nine forward and eleven inverse y-FFTs of a column run side by side; the
// nine-to-three combine and the RK4 recursion go through shared memory. The
// last CTA takes the packed kx = 0 / N/2 columns.
template <typename real, int N, int W, int E>
__global__ void __launch_bounds__(NGA * W * (N / E)) adj_colp_kernel(const __grid_constant__ AdjArgs<real> a) {
    constexpr int H = N / 2, TEAM = N / E, NXH = H + 1;
    constexpr int SPAN = N * (W > 1 ? W : 2);   // complex per team buffer (the edge CTA needs 2N)
    constexpr int NTH = NGA * W * TEAM;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    cplx<real>* sm = reinterpret_cast<cplx<real>*>(smem_raw);
    const int tid = threadIdx.x;
    const int f = tid / (W * TEAM), rem = tid % (W * TEAM);
    const int w = rem % W, t = rem / W;
    cplx<real>* buf = sm + (size_t)f * SPAN;
    XchgCols<real> x{buf, w, W};
    TeamFFT<real, N, E> fft;
    fft.template init<N>(t, a.tw);
    constexpr int BPI = H / W + 1;                 // CTAs per instance: H/W column blocks + the edge CTA
    const int inst = blockIdx.x / BPI, lb = blockIdx.x % BPI;
    const size_t so = a.s_istride * inst;
    const cplx<real>* Tx = a.Tx + a.tx_istride * inst;
    cplx<real>* Tg = a.Tg + a.tg_istride * inst;
    const cplx<real>* wst = a.wstate ? a.wstate + so : nullptr;
    const bool edge = lb == BPI - 1;
    const real lw = a.loss_wv ? a.loss_wv[inst] : a.loss_w;
    const bool emit_q = f < NGA && (a.advect || f > GA_VW);
    const real n2 = (real)1 / ((real)N * (real)N);

    if (!edge) {
        const int i = lb * W + w;
        const bool active = i != 0;
        const real kx = a.dkx * (real)i;
        if (a.stage >= 1) {
            const bool mine = f < PF_COUNT && active;
            cplx<real> v[E];
#pragma unroll
            for (int e = 0; e < E; ++e)
                v[e] = mine ? Tx[(size_t)f * N * H + (size_t)(t + TEAM * e) * H + i] : mk<real>(0, 0);
            fft.template run<false>(t, v, x);
            if (f < PF_COUNT)
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const int j = t + TEAM * e;
                    const real ky = ky_of<real>(j, N, a.dky);
                    const real k2 = kx * kx + ky * ky;
                    buf[j * W + w] = adj_cmult<real>(f, v[e], kx, ky, k2 > 0 ? (real)1 / k2 : (real)0);
                }
        }
        __syncthreads();
        for (int pt = tid; pt < N * W; pt += NTH) {
            const int j = pt / W, w2 = pt % W, i2 = lb * W + w2;
            if (i2 == 0) continue;
            cplx<real> cb[3] = {mk<real>(0, 0), mk<real>(0, 0), mk<real>(0, 0)};
            if (a.stage >= 1)
#pragma unroll
                for (int p = 0; p < PF_COUNT; ++p) cb[adj_target(p)] = cadd(cb[adj_target(p)], sm[(size_t)p * SPAN + j * W + w2]);
            const size_t idx = (size_t)j * NXH + i2;
            const cplx<real> lossg = wst ? cscale(wst[idx], 2 * lw * n2 * n2) : mk<real>(0, 0);
            real Ef[3], Eh[3];
            AdjHeld<real> held[3];
#pragma unroll
            for (int g = 0; g < 3; ++g) {
                adj_factors<real, N>(a, g, i2, j, Ef[g], Eh[g]);
                held[g] = adj_rk_load(a, g, so + idx);
            }
#pragma unroll
            for (int g = 0; g < 3; ++g)
                sm[(size_t)g * SPAN + j * W + w2] = adj_rk_apply(a, g, so + idx, held[g], cscale(cb[g], 2 * n2), Ef[g],
                                                                 Eh[g], adj_keep(a, g, i2, j),
                                                                 g == 0 ? lossg : mk<real>(0, 0));
        }
        __syncthreads();
        if (!a.emit) return;
        cplx<real> v[E];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int j = t + TEAM * e;
            v[e] = mk<real>(0, 0);
            if (emit_q && active) {
                const cplx<real> lw = sm[j * W + w], l1 = sm[SPAN + j * W + w], l2 = sm[2 * SPAN + j * W + w];
                v[e] = cscale(adj_emit<real>(f, lw, l1, l2, kx, ky_of<real>(j, N, a.dky), a.ce), (real)0.5);
            }
        }
        __syncthreads();
        fft.template run<true>(t, v, x);
        if (emit_q && active)
#pragma unroll
            for (int e = 0; e < E; ++e) Tg[(size_t)f * N * H + (size_t)(t + TEAM * e) * H + i] = v[e];
        return;
    }

    // ---- the kx = 0 and kx = N/2 columns, packed as DC + i Nyquist; lanes w == 0 of each team
    const bool lead = w == 0;
    const real kN = a.dkx * (real)H;
    {
        const bool mine = f < PF_COUNT && lead && a.stage >= 1;
        cplx<real> v[E];
#pragma unroll
        for (int e = 0; e < E; ++e) v[e] = mine ? Tx[(size_t)f * N * H + (size_t)(t + TEAM * e) * H] : mk<real>(0, 0);
        fft.template run<false>(t, v, x);
        if (lead)
#pragma unroll
            for (int e = 0; e < E; ++e) buf[(t + TEAM * e) * W] = v[e];
        __syncthreads();
        cplx<real> zm[E];
#pragma unroll
        for (int e = 0; e < E; ++e) zm[e] = lead ? cconj(buf[((N - (t + TEAM * e)) % N) * W]) : mk<real>(0, 0);
        __syncthreads();
        if (f < PF_COUNT && lead)
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int j = t + TEAM * e;
                const real ky = ky_of<real>(j, N, a.dky);
                const cplx<real> z0 = a.stage >= 1 ? cscale(cadd(v[e], zm[e]), (real)0.5) : mk<real>(0, 0);
                const cplx<real> zH = a.stage >= 1 ? cmul_mi(cscale(csub(v[e], zm[e]), (real)0.5)) : mk<real>(0, 0);
                const real k2H = kN * kN + ky * ky;
                buf[j] = adj_cmult<real>(f, z0, (real)0, ky, ky != 0 ? (real)1 / (ky * ky) : (real)0);
                buf[N + j] = adj_cmult<real>(f, zH, kN, ky, k2H > 0 ? (real)1 / k2H : (real)0);
            }
    }
    __syncthreads();
    for (int pt = tid; pt < 2 * N; pt += NTH) {
        const int c = pt / N, j = pt % N, jm = (N - j) % N;
        const int i = c == 0 ? 0 : H;
        cplx<real> cb[3] = {mk<real>(0, 0), mk<real>(0, 0), mk<real>(0, 0)};
#pragma unroll
        for (int p = 0; p < PF_COUNT; ++p) cb[adj_target(p)] = cadd(cb[adj_target(p)], sm[(size_t)p * SPAN + c * N + j]);
        const size_t idx = (size_t)j * NXH + i;
        cplx<real> lossg = mk<real>(0, 0);
        if (wst) {
            const cplx<real> P = cscale(cadd(wst[idx], cconj(wst[(size_t)jm * NXH + i])), (real)0.5);
            lossg = cscale(P, lw * n2 * n2);
        }
        real Ef[3], Eh[3];
        AdjHeld<real> held[3];
#pragma unroll
        for (int g = 0; g < 3; ++g) {
            adj_factors<real, N>(a, g, i, j, Ef[g], Eh[g]);
            held[g] = adj_rk_load(a, g, so + idx);
        }
#pragma unroll
        for (int g = 0; g < 3; ++g)
            sm[(size_t)g * SPAN + c * N + j] = adj_rk_apply(a, g, so + idx, held[g], cscale(cb[g], n2), Ef[g], Eh[g],
                                                            adj_keep(a, g, i, j), g == 0 ? lossg : mk<real>(0, 0));
    }
    __syncthreads();
    if (!a.emit) return;
    cplx<real> v[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        v[e] = mk<real>(0, 0);
        if (!(emit_q && lead)) continue;
        const int j = t + TEAM * e;
        cplx<real> P[2];
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            const real kx = c == 0 ? (real)0 : kN;
            cplx<real> val[2];
#pragma unroll
            for (int s2 = 0; s2 < 2; ++s2) {
                const int jj = s2 == 0 ? j : (N - j) % N, jp = (N - jj) % N;
                cplx<real> lw = sm[c * N + jj];
                if (f <= GA_VW) lw = cscale(cadd(lw, cconj(sm[c * N + jp])), (real)0.5);
                const cplx<real> l1 = sm[SPAN + c * N + jj], l2 = sm[2 * SPAN + c * N + jj];
                val[s2] = adj_emit<real>(f, lw, l1, l2, kx, ky_of<real>(jj, N, a.dky), a.ce);
            }
            P[c] = cscale(cadd(val[0], cconj(val[1])), (real)0.5);
        }
        v[e] = cadd(P[0], cmul_i(P[1]));
    }
    __syncthreads();
    fft.template run<true>(t, v, x);
    if (emit_q && lead)
#pragma unroll
        for (int e = 0; e < E; ++e) Tg[(size_t)f * N * H + (size_t)(t + TEAM * e) * H] = v[e];
}

// Field-parallel row kernel: one team of H/E threads per (transform, row),
// NGA teams per row (half-length real transforms): the 11 C2R of the g rows
// side by side, the transposed products at each point of the row against the
// nine recorded forward fields (activity gradient accumulated in place), then
// the 9 R2C side by side. A team's exchange buffer (H complex = N reals) holds
// its real row between the transforms.
template <typename real, int N, int E>
__global__ void __launch_bounds__(NGA * (N / 2 / E)) adj_row_kernel(const __grid_constant__ AdjArgs<real> a) {
    constexpr int H = N / 2, TEAM = H / E, TPR = NGA * TEAM;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    cplx<real>* sm = reinterpret_cast<cplx<real>*>(smem_raw);
    const int q = threadIdx.x / TEAM, t = threadIdx.x % TEAM;
    const int inst = blockIdx.x / N, n = blockIdx.x % N;
    const cplx<real>* Tg = a.Tg + a.tg_istride * inst;
    cplx<real>* Tx = a.Tx + a.tx_istride * inst;
    const real* phys = a.phys + a.p_istride * inst;
    const real* alf = a.alpha_field ? a.alpha_field + a.a_istride * inst : nullptr;
    real* agr = a.alpha_grad ? a.alpha_grad + a.g_istride * inst : nullptr;
    cplx<real>* buf = sm + (size_t)q * H;
    real* row = reinterpret_cast<real*>(buf);
    const real* rows = reinterpret_cast<const real*>(sm);   // field q at rows[q * N + x]
    XchgRow<real> x{buf};
    TeamFFT<real, H, E> fft;
    fft.template init<N>(t, a.tw);
    const bool live = a.advect || q > GA_VW;

    // 1. g_q = C2R of row n of Tg[q] (slot 0 of a T row holds DC + i Nyquist)
    {
        const cplx<real>* tr = Tg + (size_t)q * N * H + (size_t)n * H;
        cplx<real> v[E];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int k = t + TEAM * e;
            v[e] = mk<real>(0, 0);
            if (!live) continue;
            if (k == 0) {
                const cplx<real> d = tr[0];
                v[e] = mk<real>(d.x + d.y, d.x - d.y);
            } else {
                const cplx<real> A = tr[k], B = cconj(tr[H - k]);
                v[e] = cadd(cadd(A, B), cmul_i(cmul(cconj(a.tw[k]), csub(A, B))));
            }
        }
        fft.template run<true>(t, v, x);
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int m = t + TEAM * e;
            row[2 * m] = v[e].x;
            row[2 * m + 1] = v[e].y;
        }
    }
    __syncthreads();

    // 2. transposed products at each point of the row
    const real lam = a.lambda;
    const size_t NN = (size_t)N * N;
    real* rw = reinterpret_cast<real*>(sm);
    for (int xi = threadIdx.x; xi < N; xi += TPR) {
        const size_t pi = (size_t)n * N + xi;
        const real w = phys[PF_W * NN + pi], r1 = phys[PF_R1 * NN + pi], r2 = phys[PF_R2 * NN + pi];
        const real u = phys[PF_U * NN + pi], v = phys[PF_V * NN + pi], ux = phys[PF_UX * NN + pi];
        const real sh = phys[PF_SH * NN + pi], L1 = phys[PF_LR1 * NN + pi], L2 = phys[PF_LR2 * NN + pi];
        const real al = alf ? alf[pi] : a.alpha;
        real g[NGA];
#pragma unroll
        for (int k = 0; k < NGA; ++k) g[k] = rows[k * N + xi];
        const real S = 2 * sqrt(r1 * r1 + r2 * r2);
        const real sgl = lam * S * (S * S - 1);
        const real dsgl = lam * (3 * S * S - 1);
        const real g1221 = g[GA_P12] + g[GA_P21];
        const real Sb = (-lam * L1 + dsgl * r1) * g[GA_P11] + (-lam * L2 + dsgl * r2) * g1221 +
                        (-2 * S * r1 + lam * ux) * g[GA_A1] + (-2 * S * r2 + (real)0.5 * lam * sh) * g[GA_A2];
        const real dS1 = S > 0 ? 4 * r1 / S : (real)0, dS2 = S > 0 ? 4 * r2 / S : (real)0;
        if (agr) agr[pi] += -(r1 * g[GA_P11] + r2 * g1221);
        rw[PF_W * N + xi] = -u * g[GA_UW] - v * g[GA_VW] - r2 * g[GA_A1] + r1 * g[GA_A2];
        rw[PF_R1 * N + xi] = (sgl - al) * g[GA_P11] - 2 * L2 * g[GA_P12] + 2 * L2 * g[GA_P21] - S * S * g[GA_A1] -
                             u * g[GA_UR1] - v * g[GA_VR1] + w * g[GA_A2] + Sb * dS1;
        rw[PF_R2 * N + xi] = (sgl + 2 * L1 - al) * g[GA_P12] + (sgl - 2 * L1 - al) * g[GA_P21] - w * g[GA_A1] -
                             S * S * g[GA_A2] - u * g[GA_UR2] - v * g[GA_VR2] + Sb * dS2;
        rw[PF_U * N + xi] = -w * g[GA_UW] - r1 * g[GA_UR1] - r2 * g[GA_UR2];
        rw[PF_V * N + xi] = -w * g[GA_VW] - r1 * g[GA_VR1] - r2 * g[GA_VR2];
        rw[PF_UX * N + xi] = lam * S * g[GA_A1];
        rw[PF_SH * N + xi] = (real)0.5 * lam * S * g[GA_A2];
        rw[PF_LR1 * N + xi] = -lam * S * g[GA_P11] + 2 * r2 * g[GA_P12] - 2 * r2 * g[GA_P21];
        rw[PF_LR2 * N + xi] = (-lam * S - 2 * r1) * g[GA_P12] + (-lam * S + 2 * r1) * g[GA_P21];
    }
    __syncthreads();

    // 3. R2C of the nine adjoints (teams 0..8) into Tx
    cplx<real> v[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int m = t + TEAM * e;
        v[e] = q < PF_COUNT ? mk<real>(row[2 * m], row[2 * m + 1]) : mk<real>(0, 0);
    }
    __syncthreads();
    fft.template run<false>(t, v, x);
#pragma unroll
    for (int e = 0; e < E; ++e) x.write(t + TEAM * e, v[e]);
    x.sync();
    if (q < PF_COUNT) {
        cplx<real>* out = Tx + (size_t)q * N * H + (size_t)n * H;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const int k = t + TEAM * e;
            const cplx<real> zm = cconj(x.read((H - k) % H));
            if (k == 0) {
                out[0] = mk<real>(v[e].x + v[e].y, v[e].x - v[e].y);
            } else {
                const cplx<real> sum = cscale(cadd(v[e], zm), (real)0.5);
                const cplx<real> dif = cscale(csub(v[e], zm), (real)0.5);
                out[k] = csub(sum, cmul_i(cmul(a.tw[k], dif)));
            }
        }
    }
}

// loss += weight * (0.5 / N^4) * diag[0] (the enstrophy sum of the step's new state); weight carries 1/N^4
static __global__ void adj_loss_accumulate(const double* diag, double* loss, double weight) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *loss += weight * 0.5 * diag[0];
}
// the same for ninst instances (diag: 2 doubles per instance)
static __global__ void adj_loss_accumulate_batch(const double* diag, double* loss, double weight, int ninst) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < ninst) loss[k] += weight * 0.5 * diag[2 * k];
}

}  // namespace qaf
