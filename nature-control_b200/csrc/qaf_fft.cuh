// qaf_fft.cuh — register/shared-memory FFT building blocks for sm_100a.
//
// A length-L transform is computed by a "team" of TEAM = L / E threads; each
// thread holds E complex values in registers. Between Stockham radix passes
// the team exchanges values through shared memory; the last pass leaves every
// thread with the outputs it needs, so an L = R0 * R1 * ... transform costs
// (number of passes - 1) exchanges.
//
// Distribution invariant (entry and exit): thread t holds element t + TEAM*e
// in v[e], e = 0..E-1 (natural order, strided by TEAM), which makes global
// loads/stores of a team coalesced.
//
// The pass, exchange-index and small-DFT routines are __host__ __device__ so
// that the CPU tests can emulate a team (thread loops between the exchange
// phases) and check every index map against a plain DFT.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#define QAF_HD __host__ __device__ __forceinline__
#define QAF_HDC __host__ __device__ constexpr

namespace qaf {

template <typename real> struct cplx_t;
template <> struct cplx_t<float> { using type = float2; };
template <> struct cplx_t<double> { using type = double2; };
template <typename real> using cplx = typename cplx_t<real>::type;

template <typename real> QAF_HD cplx<real> mk(real x, real y) { cplx<real> c; c.x = x; c.y = y; return c; }
template <typename C> QAF_HD C cadd(C a, C b) { C c; c.x = a.x + b.x; c.y = a.y + b.y; return c; }
template <typename C> QAF_HD C csub(C a, C b) { C c; c.x = a.x - b.x; c.y = a.y - b.y; return c; }
template <typename C> QAF_HD C cmul(C a, C b) { C c; c.x = a.x * b.x - a.y * b.y; c.y = a.x * b.y + a.y * b.x; return c; }
template <typename C, typename R> QAF_HD C cscale(C a, R s) { C c; c.x = a.x * s; c.y = a.y * s; return c; }
template <typename C> QAF_HD C cconj(C a) { C c; c.x = a.x; c.y = -a.y; return c; }
// multiply by +i or -i
template <typename C> QAF_HD C cmul_i(C a) { C c; c.x = -a.y; c.y = a.x; return c; }
template <typename C> QAF_HD C cmul_mi(C a) { C c; c.x = a.y; c.y = -a.x; return c; }
// a * conj(w) when INV, a * w otherwise
template <bool INV, typename C> QAF_HD C ctw(C a, C w) { if (INV) w.y = -w.y; return cmul(a, w); }

// cos and sin of 2 pi k / 16, k = 0..15 (mathematical constants to double precision)
QAF_HD double cos16(int k) {
    const double c[16] = {1.0, 0.92387953251128673848, 0.70710678118654752440, 0.38268343236508977173,
                          0.0, -0.38268343236508977173, -0.70710678118654752440, -0.92387953251128673848,
                          -1.0, -0.92387953251128673848, -0.70710678118654752440, -0.38268343236508977173,
                          0.0, 0.38268343236508977173, 0.70710678118654752440, 0.92387953251128673848};
    return c[k & 15];
}
QAF_HD double sin16(int k) { return cos16(k + 12); }   // sin(x) = cos(x - pi/2)

QAF_HDC int ilog2(int n) { return n <= 1 ? 0 : 1 + ilog2(n / 2); }
QAF_HDC int bitrev(int x, int bits) { return bits == 0 ? 0 : ((x & 1) << (bits - 1)) | bitrev(x >> 1, bits - 1); }

// In-register DFT of R = 2, 4, 8 or 16 points: y[r] = sum_q x[q] W_R^{qr},
// W_R = exp(-2 pi i / R) (forward) or exp(+2 pi i / R) (INV). Iterative
// radix-2 on a bit-reversed copy; all indices are compile-time constants.
template <typename real, int R, bool INV>
QAF_HD void small_dft(cplx<real>* x) {
    static_assert(R == 1 || R == 2 || R == 4 || R == 8 || R == 16, "radix");
    if (R == 1) return;
    constexpr int B = ilog2(R);
    cplx<real> y[R];
#pragma unroll
    for (int q = 0; q < R; ++q) y[bitrev(q, B)] = x[q];
#pragma unroll
    for (int m = 2; m <= R; m *= 2) {
#pragma unroll
        for (int g = 0; g < R; g += m) {
#pragma unroll
            for (int k = 0; k < m / 2; ++k) {
                cplx<real> a = y[g + k], b = y[g + k + m / 2];
                const int tk = k * (16 / m);   // W_m^k = W_16^{k*16/m}
                if (tk == 0) {
                } else if (tk == 4) {
                    b = INV ? cmul_i(b) : cmul_mi(b);
                } else {
                    cplx<real> w = mk<real>((real)cos16(tk), (real)(INV ? sin16(tk) : -sin16(tk)));
                    b = cmul(b, w);
                }
                y[g + k] = cadd(a, b);
                y[g + k + m / 2] = csub(a, b);
            }
        }
    }
#pragma unroll
    for (int q = 0; q < R; ++q) x[q] = y[q];
}

// One Stockham pass of radix R on span S (the product of the radices already
// applied) for a length-L transform, E values per thread. Butterfly
// b = t + TEAM*s (s < E/R) reads elements b + q*L/R, i.e. register s + q*(E/R),
// applies W_{S R}^{q k} (k = b mod S), and leaves output r in register
// s + r*(E/R). tw[m] = exp(-2 pi i m / TWN) with TWN a multiple of L.
template <typename real, int L, int E, int R, int S, bool INV, int TWN>
QAF_HD void stockham_pass(int t, cplx<real>* v, const cplx<real>* tw) {
    constexpr int TEAM = L / E;
    constexpr int NB = E / R;
    static_assert(E % R == 0 && L % (S * R) == 0, "pass shape");
#pragma unroll
    for (int s = 0; s < NB; ++s) {
        cplx<real> x[R];
        const int b = t + TEAM * s;
        const int k = b % S;
#pragma unroll
        for (int q = 0; q < R; ++q) {
            x[q] = v[s + q * NB];
            if (S > 1 && q > 0) {
                // W_{S R}^{q k} = W_TWN^{q k TWN/(S R)}, q k < S R
                const int m = q * k * (TWN / (S * R));
                x[q] = ctw<INV>(x[q], tw[m]);
            }
        }
        small_dft<real, R, INV>(x);
#pragma unroll
        for (int r = 0; r < R; ++r) v[s + r * NB] = x[r];
    }
}

// Where register slot (s + r*NB) of thread t lands after the pass above.
template <int L, int E, int R, int S>
QAF_HD int stockham_dest(int t, int slot) {
    constexpr int TEAM = L / E;
    constexpr int NB = E / R;
    const int s = slot % NB, r = slot / NB;
    const int b = t + TEAM * s;
    return (b / S) * S * R + (b % S) + r * S;
}

// Radix schedule for L = 2^m with E = 2^e values per thread: as many radix-E
// passes as fit, then one smaller pass for the remainder.
template <int L, int E>
struct Sched {
    static constexpr int full = ilog2(L) / ilog2(E);
    static constexpr int rem = 1 << (ilog2(L) - full * ilog2(E));
    static constexpr int passes = full + (rem > 1 ? 1 : 0);
    QAF_HD static constexpr int radix(int p) { return p < full ? E : rem; }
    QAF_HD static constexpr int span(int p) {
        int s = 1;
        for (int q = 0; q < p; ++q) s *= radix(q);
        return s;
    }
};

// Team FFT driver. `xchg` provides the team's shared buffer:
//   xchg.write(index, value), xchg.sync(), xchg.read(index) -> value.
// Between passes every thread writes its E values to their destinations,
// the team synchronises, reads back its own E strided elements and
// synchronises again (so the buffer can be reused by the next exchange).
template <typename real, int L, int E, bool INV, int TWN, int P, class X>
QAF_HD void team_pass(int t, cplx<real>* v, const cplx<real>* tw, X& xchg) {
    using Sc = Sched<L, E>;
    constexpr int R = Sc::radix(P);
    constexpr int S = Sc::span(P);
    stockham_pass<real, L, E, R, S, INV, TWN>(t, v, tw);
    if constexpr (P + 1 < Sc::passes) {
        constexpr int TEAM = L / E;
#pragma unroll
        for (int slot = 0; slot < E; ++slot) xchg.write(stockham_dest<L, E, R, S>(t, slot), v[slot]);
        xchg.sync();
#pragma unroll
        for (int e = 0; e < E; ++e) v[e] = xchg.read(t + TEAM * e);
        xchg.sync();
        team_pass<real, L, E, INV, TWN, P + 1, X>(t, v, tw, xchg);
    }
}

template <typename real, int L, int E, bool INV, int TWN, class X>
QAF_HD void team_fft(int t, cplx<real>* v, const cplx<real>* tw, X& xchg) {
    team_pass<real, L, E, INV, TWN, 0, X>(t, v, tw, xchg);
}

}  // namespace qaf
