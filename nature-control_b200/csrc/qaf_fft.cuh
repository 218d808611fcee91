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

// cos and sin of 2 pi k / 48 for any integer k (mathematical constants to
// double precision; the first quadrant is tabulated, the rest by symmetry).
// 48 = 3 * 16 covers every twiddle of the small DFTs below (R | 48).
QAF_HD double cos48(int k) {
    const double c[13] = {1.0, 0.99144486137381041114, 0.96592582628906828675, 0.92387953251128675613,
                          0.86602540378443864676, 0.79335334029123516458, 0.70710678118654752440,
                          0.60876142900872063942, 0.5, 0.38268343236508977173, 0.25881904510252076235,
                          0.13052619222005159155, 0.0};
    k = ((k % 48) + 48) % 48;
    if (k <= 12) return c[k];
    if (k <= 24) return -c[24 - k];
    if (k <= 36) return -c[k - 24];
    return c[48 - k];
}
QAF_HD double sin48(int k) { return cos48(k + 36); }   // sin x = cos(x - pi/2)

QAF_HDC int ilog2(int n) { return n <= 1 ? 0 : 1 + ilog2(n / 2); }
QAF_HDC bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }
// iterative (not recursive) so that, with constant arguments after unrolling,
// the device compiler folds it and register arrays indexed by it stay in registers
QAF_HDC int bitrev(int x, int bits) {
    int r = 0;
    for (int i = 0; i < bits; ++i) { r = (r << 1) | (x & 1); x >>= 1; }
    return r;
}

// a * W_R^m with W_R = exp(-2 pi i / R) (forward) or exp(+2 pi i / R) (INV),
// m a compile-time constant after unrolling, R | 48
template <typename real, int R, bool INV>
QAF_HD cplx<real> rot(cplx<real> a, int m) {
    const int k = ((m % R) + R) % R * (48 / R);   // angle 2 pi k / 48
    if (k == 0) return a;
    if (k == 12) return INV ? cmul_i(a) : cmul_mi(a);
    if (k == 24) return mk<real>(-a.x, -a.y);
    if (k == 36) return INV ? cmul_mi(a) : cmul_i(a);
    const cplx<real> w = mk<real>((real)cos48(k), (real)(INV ? sin48(k) : -sin48(k)));
    return cmul(a, w);
}

// 3-point DFT in place: y_r = sum_q x_q W_3^{qr}
template <typename real, bool INV>
QAF_HD void dft3(cplx<real>& x0, cplx<real>& x1, cplx<real>& x2) {
    const real h = (real)0.86602540378443864676;   // sin(2 pi / 3)
    const cplx<real> t1 = cadd(x1, x2), t2 = csub(x1, x2);
    const cplx<real> m = mk<real>(x0.x - (real)0.5 * t1.x, x0.y - (real)0.5 * t1.y);
    // forward: y1 = m - i h t2, y2 = m + i h t2 (inverse: the signs swap)
    const cplx<real> r = mk<real>(-h * t2.y, h * t2.x);    // i h t2
    x0 = cadd(x0, t1);
    x1 = INV ? cadd(m, r) : csub(m, r);
    x2 = INV ? csub(m, r) : cadd(m, r);
}

// In-register DFT of R points, R = 2^m (m <= 4) or 3 * 2^m (m <= 4):
// y[r] = sum_q x[q] W_R^{qr}, W_R = exp(-2 pi i / R) (forward) or
// exp(+2 pi i / R) (INV). Powers of two: iterative radix-2 on a bit-reversed
// copy. 3 * Q: Cooley-Tukey with n = Q n1 + n2, k = k1 + 3 k2 — three-point
// DFTs over n1, twiddles W_R^{n2 k1}, then Q-point DFTs over n2. All indices
// are compile-time constants.
template <typename real, int R, bool INV>
QAF_HD void small_dft(cplx<real>* x) {
    static_assert(R == 1 || R == 2 || R == 4 || R == 8 || R == 16 || R == 3 || R == 6 || R == 12 || R == 24 ||
                  R == 48, "radix");
    if constexpr (R == 1) {
        return;
    } else if constexpr (R % 3 == 0) {
        constexpr int Q = R / 3;
        cplx<real> a[3][Q];
#pragma unroll
        for (int n2 = 0; n2 < Q; ++n2) {
            cplx<real> t0 = x[n2], t1 = x[Q + n2], t2 = x[2 * Q + n2];
            dft3<real, INV>(t0, t1, t2);
            a[0][n2] = t0;
            a[1][n2] = rot<real, R, INV>(t1, n2);
            a[2][n2] = rot<real, R, INV>(t2, 2 * n2);
        }
#pragma unroll
        for (int k1 = 0; k1 < 3; ++k1) {
            small_dft<real, Q, INV>(a[k1]);
#pragma unroll
            for (int k2 = 0; k2 < Q; ++k2) x[k1 + 3 * k2] = a[k1][k2];
        }
    } else {
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
                    cplx<real> a = y[g + k], b = rot<real, 16, INV>(y[g + k + m / 2], k * (16 / m));   // W_m^k
                    y[g + k] = cadd(a, b);
                    y[g + k + m / 2] = csub(a, b);
                }
            }
        }
#pragma unroll
        for (int q = 0; q < R; ++q) x[q] = y[q];
    }
}

// Values per thread of a length-L team FFT near the power of two e: e itself
// for L = 2^m, 3e/2 for L = 3 * 2^m (the first pass carries the factor 3);
// never more than L. The result divides L.
QAF_HDC int fit_e(int L, int e) {
    return L % 3 == 0 ? (3 * e / 2 < 3 ? 3 : (3 * e / 2 <= L ? 3 * e / 2 : L)) : (e <= L ? e : L);
}
// The power-of-two size whose launch shapes a size L follows: L, or 2L/3 for L = 3 * 2^m.
QAF_HDC int pow2_size(int L) { return L % 3 == 0 ? 2 * L / 3 : L; }

// Where register slot (s + r*NB) of thread t lands after the pass above.
template <int L, int E, int R, int S>
QAF_HD int stockham_dest(int t, int slot) {
    constexpr int TEAM = L / E;
    constexpr int NB = E / R;
    const int s = slot % NB, r = slot / NB;
    const int b = t + TEAM * s;
    return (b / S) * S * R + (b % S) + r * S;
}

// ---------------------------------------------------------------------------
// Exchange-buffer swizzle. A Stockham pass writes its E outputs at stride E
// (first pass) or in groups of S spaced S*R apart, so 8-byte stores of a
// half-warp would pile onto a few banks (up to 16-way); reads are contiguous.
// XOR-ing the element index within each 16-element (128-byte) line with
// (line * 5) mod 16 spreads every write pattern of the team FFTs over the
// banks (worst case 2-way; contiguous reads stay a permutation of one line).
// A bijection of each aligned 16-element line, so buffers whose length is a
// multiple of 16 (or below 16, where it is the identity) stay in bounds.
// ---------------------------------------------------------------------------
QAF_HD int swz(int a) { return a ^ (((a >> 4) * 5) & 15); }

// Radix schedule of a length-L transform with E values per thread.
//   L = 2^m, E = 2^e:        as many radix-E passes as fit, then one smaller
//                            pass for the remainder.
//   L = 3 * 2^m, E = 3 * 2^e: one radix-E pass (it carries the factor 3),
//                            then the power-of-two passes of L / E with
//                            radix 2^e and a remainder.
// Every radix divides E, so each pass is E / R butterflies per thread.
template <int L, int E>
struct Sched {
    static constexpr bool R3 = L % 3 == 0;
    static_assert(R3 ? (E % 3 == 0 && is_pow2(L / 3) && is_pow2(E / 3)) : (is_pow2(L) && is_pow2(E)),
                  "L = 2^m with E = 2^e, or L = 3*2^m with E = 3*2^e");
    static_assert(L % E == 0, "E divides L");
    static constexpr int P2 = R3 ? E / 3 : E;           // radix of the power-of-two passes
    static constexpr int L2 = R3 ? L / E : L;           // length they cover
    static constexpr int first = R3 ? 1 : 0;
    static constexpr int full = P2 > 1 ? ilog2(L2) / ilog2(P2) : 0;
    static constexpr int rem = L2 >> (full * ilog2(P2 > 1 ? P2 : 2));
    static constexpr int passes = first + full + (rem > 1 ? 1 : 0);
    QAF_HD static constexpr int radix(int p) { return (R3 && p == 0) ? E : (p < first + full ? P2 : rem); }
    QAF_HD static constexpr int span(int p) {
        int s = 1;
        for (int q = 0; q < p; ++q) s *= radix(q);
        return s;
    }
};

// Team FFT with per-thread twiddle bases. In pass P (span S, radix R) the
// butterfly b = t + TEAM*s needs W_{S R}^{q k}, q < R, k = b mod S. The base
// W_{S R}^{k} depends only on (t, P, s), not on the data, so a team computes
// its bases once (init) and every transform then forms the powers by complex
// multiplication — no twiddle loads inside a transform. The powers carry a
// rounding error of about q ulps (q < 16).
template <int L, int E>
struct TwLayout {
    using Sc = Sched<L, E>;
    QAF_HD static constexpr int offset(int P) {   // first base of pass P (P >= 1)
        int o = 0;
        for (int p = 1; p < P; ++p) o += E / Sc::radix(p);
        return o;
    }
    static constexpr int count = Sc::passes > 1 ? offset(Sc::passes) : 0;
};

// base: the thread's twiddle bases, base index i at base[i * BS] (BS = 1:
// a register array; BS = TEAM: a shared table [i][t] read at &table[t])
template <typename real, int L, int E, bool INV, int P, int BS = 1>
QAF_HD void stockham_pass_tw(int t, cplx<real>* v, const cplx<real>* base) {
    using Sc = Sched<L, E>;
    constexpr int R = Sc::radix(P), NB = E / R;
#pragma unroll
    for (int s = 0; s < NB; ++s) {
        cplx<real> x[R];
#pragma unroll
        for (int q = 0; q < R; ++q) x[q] = v[s + q * NB];
        if constexpr (P > 0) {
            cplx<real> w = base[(TwLayout<L, E>::offset(P) + s) * BS];
            if (INV) w.y = -w.y;
            cplx<real> wq = w;
#pragma unroll
            for (int q = 1; q < R; ++q) {
                x[q] = cmul(x[q], wq);
                if (q + 1 < R) wq = cmul(wq, w);
            }
        }
        small_dft<real, R, INV>(x);
#pragma unroll
        for (int r = 0; r < R; ++r) v[s + r * NB] = x[r];
    }
}

template <typename real, int L, int E>
struct TeamFFT {
    using Sc = Sched<L, E>;
    static constexpr int TEAM = L / E;
    static constexpr int NBASE = TwLayout<L, E>::count;
    cplx<real> base[NBASE > 0 ? NBASE : 1];

    // tw[m] = exp(-2 pi i m / TWN), TWN a multiple of L
    template <int TWN>
    QAF_HD void init(int t, const cplx<real>* tw) {
        init_pass<TWN, 1>(t, tw);
    }
    template <int TWN, int P>
    QAF_HD void init_pass(int t, const cplx<real>* tw) {
        if constexpr (P < Sc::passes) {
            constexpr int R = Sc::radix(P), S = Sc::span(P), NB = E / R;
#pragma unroll
            for (int s = 0; s < NB; ++s) {
                const int k = (t + TEAM * s) % S;
                base[TwLayout<L, E>::offset(P) + s] = tw[k * (TWN / (S * R))];
            }
            init_pass<TWN, P + 1>(t, tw);
        }
    }

    // In-place transform of v (distribution: thread t holds element t + TEAM*e).
    // `xchg` is the team's shared buffer: write(index, value), sync(), read(index).
    template <bool INV, class X>
    QAF_HD void run(int t, cplx<real>* v, X& xchg) const {
        pass<INV, 0, X>(t, v, xchg);
    }
    template <bool INV, int P, class X>
    QAF_HD void pass(int t, cplx<real>* v, X& xchg) const {
        constexpr int R = Sc::radix(P), S = Sc::span(P);
        stockham_pass_tw<real, L, E, INV, P>(t, v, base);
        if constexpr (P + 1 < Sc::passes) {
#pragma unroll
            for (int slot = 0; slot < E; ++slot) xchg.write(stockham_dest<L, E, R, S>(t, slot), v[slot]);
            xchg.sync();
#pragma unroll
            for (int e = 0; e < E; ++e) v[e] = xchg.read(t + TEAM * e);
            xchg.sync();
            pass<INV, P + 1, X>(t, v, xchg);
        }
    }
};

// The same transform with the twiddle bases in a shared-memory table
// [base index][t] (NBASE * TEAM entries) instead of registers: the table is
// filled once per CTA (fill: one thread per t computes its bases as
// TeamFFT::init does and stores them), teams of several columns share it,
// and a pass reads the thread's bases with consecutive-t (conflict-free,
// broadcast across the teams of a warp) loads. Frees the registers the
// bases would hold for the rest of the kernel's state.
template <typename real, int L, int E>
struct TeamFFTShared {
    using Sc = Sched<L, E>;
    static constexpr int TEAM = L / E;
    static constexpr int NBASE = TwLayout<L, E>::count;
    static constexpr int ENTRIES = (NBASE > 0 ? NBASE : 1) * TEAM;
    const cplx<real>* tab;   // &table[t] of the calling thread

    template <int TWN>
    __device__ static void fill(cplx<real>* table, int t, const cplx<real>* tw) {
        TeamFFT<real, L, E> f;
        f.template init<TWN>(t, tw);
#pragma unroll
        for (int i = 0; i < NBASE; ++i) table[i * TEAM + t] = f.base[i];
    }
    template <bool INV, class X>
    __device__ void run(int t, cplx<real>* v, X& xchg) const {
        pass<INV, 0, X>(t, v, xchg);
    }
    template <bool INV, int P, class X>
    __device__ void pass(int t, cplx<real>* v, X& xchg) const {
        constexpr int R = Sc::radix(P), S = Sc::span(P);
        stockham_pass_tw<real, L, E, INV, P, TEAM>(t, v, tab);
        if constexpr (P + 1 < Sc::passes) {
#pragma unroll
            for (int slot = 0; slot < E; ++slot) xchg.write(stockham_dest<L, E, R, S>(t, slot), v[slot]);
            xchg.sync();
#pragma unroll
            for (int e = 0; e < E; ++e) v[e] = xchg.read(t + TEAM * e);
            xchg.sync();
            pass<INV, P + 1, X>(t, v, xchg);
        }
    }

    // The transform with a double-buffered exchange between interleaved
    // column teams (element idx of team w at buf[idx * W + w]): pass P's
    // outputs go to `ext` (P even) or to `in` (P odd), one barrier per
    // exchange. `in` holds the input the threads loaded before the first
    // pass, so it is free for writing once the first exchange's barrier has
    // passed; an odd number of exchanges ends with a barrier, so that `ext`
    // is free for the next call when this one returns.
    // SWZ (E a multiple of 4): element idx at idx ^ ((idx / E) & 3), which
    // spreads the first pass's stores E t + r of neighbouring t over the banks
    template <bool INV, bool SWZ = false>
    __device__ void run_db(int t, cplx<real>* v, cplx<real>* ext, cplx<real>* in, int w, int W) const {
        pass_db<INV, SWZ, 0>(t, v, ext, in, w, W);
        if constexpr ((Sc::passes - 1) % 2 == 1) __syncthreads();
    }
    template <bool SWZ>
    __device__ static int at(int idx) {
        if constexpr (SWZ) return idx ^ ((idx / E) & 3);
        else return idx;
    }
    template <bool INV, bool SWZ, int P>
    __device__ void pass_db(int t, cplx<real>* v, cplx<real>* ext, cplx<real>* in, int w, int W) const {
        constexpr int R = Sc::radix(P), S = Sc::span(P);
        stockham_pass_tw<real, L, E, INV, P, TEAM>(t, v, tab);
        if constexpr (P + 1 < Sc::passes) {
            cplx<real>* b = (P % 2 == 0) ? ext : in;
#pragma unroll
            for (int slot = 0; slot < E; ++slot) b[at<SWZ>(stockham_dest<L, E, R, S>(t, slot)) * W + w] = v[slot];
            __syncthreads();
#pragma unroll
            for (int e = 0; e < E; ++e) v[e] = b[at<SWZ>(t + TEAM * e) * W + w];
            pass_db<INV, SWZ, P + 1>(t, v, ext, in, w, W);
        }
    }
};

}  // namespace qaf
