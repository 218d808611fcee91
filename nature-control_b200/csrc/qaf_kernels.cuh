// qaf_kernels.cuh — column and row kernels of the fused IF-RK stage
// (see qaf_stage.cuh for the data flow and layouts).
#pragma once

#include "qaf_stage.cuh"

#include <type_traits>

namespace qaf {

// Select one of three pointers without indexing the kernel-parameter array
// with a runtime value (which would copy the array to local memory).
template <typename P>
__device__ __forceinline__ P pick3(const P (&arr)[3], int f) { return f == 0 ? arr[0] : (f == 1 ? arr[1] : arr[2]); }

// ---------------------------------------------------------------------------
// TMA bulk copies (cp.async.bulk) into shared memory, completed on an mbarrier.
// Waits are bounded: a wait that runs out sets FLAG_WAIT_TIMEOUT and returns,
// so a copy that never lands cannot hang the GPU (the data is then garbage and
// the status tells the host).
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    // order this thread's earlier generic-proxy accesses to dst before the async-proxy write
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}"
                 ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}

// 2D tiled TMA load of a box at element coordinates (x, y) of tensor map tm;
// the transaction bytes were announced on bar by the caller
__device__ __forceinline__ void tile_load_2d(void* dst, const CUtensorMap* tm, int x, int y, uint64_t* bar) {
    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
                 ::"r"(smem_u32(dst)), "l"(tm), "r"(x), "r"(y), "r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}"
                 ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return ok != 0;
}

// at most `polls` tries (0: kDefaultPolls; a test lowers it); on a timeout,
// FLAG_WAIT_TIMEOUT in *flags (when given) and false
constexpr unsigned kDefaultPolls = 1u << 22;
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, unsigned* flags, unsigned polls = 0) {
    const unsigned lim = polls ? polls : kDefaultPolls;
    for (unsigned it = 0; it < lim; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    if (flags) atomicOr(flags, FLAG_WAIT_TIMEOUT);
    return false;
}

// ---------------------------------------------------------------------------
// Column kernel (persistent). Work items, largest first:
//   [0, TILES)            the r1 and r2 columns of tile T (4 + 4 y-FFTs)
//   [TILES, 2 TILES)      the w columns of tile T (3 + 4 y-FFTs)
//   [2 TILES, 2 TILES+3)  the kx = 0 / kx = nx/2 edge columns of field f
// (TILES = nx / 2 / TW)
// A tile is TW kx-columns over all N rows, one contiguous slab of each array.
// Every slab an item reads (G arrays, old, acc) is fetched by one TMA bulk
// copy into a ring of three shared-memory buffers, issued up to three slabs
// ahead; a y-FFT runs in the buffer its input arrived in.
//
// A wait that runs out (a copy that never lands) marks the CTA aborted in
// shared memory: its later waits return at once, the CTA finishes the item it
// is on (on whatever the buffers hold), leaves the work loop at the next item
// boundary — where every thread reads the mark after the same barrier, so no
// barrier is left unmatched — and waits, bounded again, for the copies it has
// in flight before it exits. The other CTAs take the remaining items; the
// host sees FLAG_WAIT_TIMEOUT.
// ---------------------------------------------------------------------------
// MODE 0: twiddle bases in registers; the item code inlined whole for FP64 at
// N >= 512 only. MODE 1: twiddle bases in a shared table (TeamFFTShared) and
// the item code always inlined, so no array is passed by reference through a
// call frame (local memory, which the shared-memory carve-out leaves little
// L1 for). MODE 2: MODE 1 plus a fourth slab-sized buffer that makes every
// y-FFT exchange double-buffered (one barrier per exchange instead of two)
// and the integrating factors' ky table in shared memory (for launches of
// one CTA per SM, which leave the room); MODE 3 / 4: MODE 2 with a copy ring
// of 4 / 5 slabs. +16: the double-buffered exchange swizzled (XOR of an
// index's low two bits with bits of idx / E). +64: the item code compiled
// once (ONE_BODY).
//
// N is the column length ny (the y-transforms' length); the number of
// kx-columns H = nx / 2, and with it the tiles and work items, is a launch
// argument.
template <typename real, int N, int E, int MODE = 0, bool SQ = true>
struct ColKernel {
    static constexpr int TEAM = N / E, NTHREADS = TW * TEAM;
    static constexpr size_t SLAB = (size_t)N * TW;   // complex elements of one slab
    static constexpr int BASE = MODE & 15;
    static constexpr bool SB = BASE >= 1;            // shared twiddle bases
    static constexpr bool DB = BASE >= 2;            // double-buffered exchange, ky factors in shared memory
    static constexpr int NBUF = BASE == 3 ? 4 : (BASE >= 4 ? 5 : 3);   // slab buffers in the copy ring
    static constexpr bool SWZ = DB && (MODE & 16) && E % 4 == 0;
    // +64 (with MODE 1 or above): the item code once — the two fields of an
    // item in a loop and both item kinds through one call
    static constexpr bool ONE_BODY = SB && (MODE & 64);
    // elements whose IF factors are fetched ahead of the stage-update stores;
    // at 1024^2 the extra live registers cost more in spills than they save
    static constexpr int PF = N >= 1024 ? 1 : (E < 4 ? E : 4);
    // FP64 at N >= 512: the item code inlined whole, so that the transform
    // state stays in registers rather than in the call frame (measured 9%
    // faster at 1024^2; slower for FP32 and smaller FP64 grids, which keep
    // the compiler's own choice)
    static constexpr bool INLINE_ITEM = SB || (sizeof(real) == 8 && N >= 512);
    // the diagnostics' per-warp sums meet in shared memory and leave with one
    // pair of atomics per CTA, except in the FP32 1024^2 kernel, where the
    // extra barrier measured slower than the per-warp atomics
    static constexpr bool CTA_DIAG = !(sizeof(real) == 4 && N >= 1024);
    // IF table value through the read-only path where it is fetched ahead
    __device__ static real table(const real* p) {
        if constexpr (PF > 1) return __ldg(p);
        else return *p;
    }
    static constexpr int BOXR = g_box_rows(N);         // rows per TMA box (at most 256, divides N)
    static_assert(N % BOXR == 0 && BOXR <= 256, "TMA boxes tile a slab");
    using FFT = std::conditional_t<SB, TeamFFTShared<real, N, E>, TeamFFT<real, N, E>>;
    // MODE 0: slabs | edge table (2N) | mbarriers | ints;
    // MODE 1: slabs | twiddle table | 64 doubles of diagnostic sums | mbarriers | ints
    // (the edge table then lives in slab 1: edge items run with no copy in flight)
    // MODE 2: slabs | extra exchange slab | twiddle table | ky factors (4N) | 64 doubles | mbarriers | ints
    static constexpr size_t SMEM = SB ? (NBUF + (DB ? 1 : 0)) * SLAB * sizeof(cplx<real>) +
                                            TeamFFTShared<real, N, E>::ENTRIES * sizeof(cplx<real>) +
                                            (DB ? 4 * N * sizeof(real) : 0) + 64 * sizeof(double) +
                                            (NBUF + 1) * sizeof(uint64_t) + 16
                                      : 3 * SLAB * sizeof(cplx<real>) + 2 * N * sizeof(cplx<real>) + 4 * sizeof(uint64_t) + 16;
    using X = XchgCols<real>;   // exchange layout of the tile's y-FFTs

    const StageArgs<real>& a;
    const FFT& fft;
    int t, w;
    cplx<real>* bufs;      // three slab buffers back to back
    uint64_t* mbar;        // one mbarrier per buffer
    volatile int* aborted; // shared: a wait of this CTA ran out
    unsigned parity;       // bit b: parity of buffer b's latest issue
    // the current item: fields fa (and fb), tile T; slab sequence per field:
    // its G arrays (none in the prologue), then old and/or acc
    int fa, fb, T, nseq, next, per_a;
    bool need_old, need_acc;
    int inst;              // instance of the current item
    size_t io;             // its buffer offset (complex elements)
    double* red;           // per-warp diagnostic partial sums (the edge table's space, unused by tiles)
    int q_cur;             // queue index of the current item (test hook)
    unsigned armed;        // thread 0: bit b, parity of buffer b's latest armed phase
    cplx<real>* xbuf;      // MODE 2: the extra exchange buffer
    const real* eys;       // MODE 2: the ky factors ey[4][N] in shared memory
    unsigned withheld;     // thread 0: the buffer of the test hook's withheld copy (NBUF: none)

    __device__ cplx<real>* buf(int b) const { return bufs + (size_t)b * SLAB; }
    // kx-columns nx / 2 (the last, kx = nx/2, is an edge column): N / 2 at
    // compile time on a square grid (SQ), which keeps the index arithmetic in
    // shifts and immediates (with the size at run time the 1024^2 kernels
    // spilled), else from the launch arguments
    __device__ __forceinline__ int Hx() const {
        if constexpr (SQ) return N / 2;
        else return a.nx / 2;
    }
    __device__ int nG(int f) const { return a.mode == MODE_PROLOGUE ? 0 : (f == 0 ? 3 : 2); }
    __device__ int per_field(int f) const { return nG(f) + (need_old ? 1 : 0) + (need_acc ? 1 : 0); }
    // slab sidx of the item: a G array (>= 0: its plane index) or a state slab (pointer)
    __device__ int slab_g(int sidx) const {
        const int f = sidx < per_a ? fa : fb;
        const int r = sidx < per_a ? sidx : sidx - per_a;
        return r < nG(f) ? (f == 0 ? 0 : (f == 1 ? 3 : 5)) + r : -1;
    }
    __device__ const cplx<real>* slab_state(int sidx) const {
        const int f = sidx < per_a ? fa : fb;
        const int r = sidx < per_a ? sidx : sidx - per_a;
        const size_t base = io + (size_t)T * SLAB;
        if (r == nG(f) && need_old) return pick3(a.old_m, f) + base;
        return pick3(a.acc_m, f) + base;
    }
    // issue every slab with index < k that has not been issued yet: G arrays
    // (row-major [n][k]) as TMA boxes of TW columns x BOXR rows, state slabs
    // (column-tiled, contiguous) as one bulk copy
    __device__ void issue_upto(int k) {
        if (k > nseq) k = nseq;
        while (next < k) {
            const int b = next % NBUF;
            __syncthreads();   // every thread is done with buffer b
            // an aborted CTA arms nothing more: thread 0 sees the mark once its
            // own wait for buffer b's previous slab gave up or was skipped, so
            // no barrier is re-armed in a phase that has not completed
            if (threadIdx.x == 0 && !*aborted) {
                armed ^= 1u << b;
                const unsigned bytes = (unsigned)(SLAB * sizeof(cplx<real>));
                const int g = slab_g(next);
                if (dropped(next)) {
                    // test hook: the buffer is armed for the slab but the copy
                    // is not issued, so its wait runs out (nothing in flight)
                    expect_tx(&mbar[b], bytes);
                    withheld = (unsigned)b;
                } else if (g >= 0) {
                    expect_tx(&mbar[b], bytes);
                    constexpr int CPE = sizeof(cplx<real>) / 8;   // 8-byte elements per complex
#pragma unroll 1
                    for (int r0 = 0; r0 < N; r0 += BOXR)
                        tile_load_2d(buf(b) + (size_t)r0 * TW, &a.tm_G, T * TW * CPE,
                                     (int)((io / (size_t)Hx()) + (size_t)g * N + r0), &mbar[b]);
                } else {
                    bulk_load(buf(b), slab_state(next), bytes, &mbar[b]);
                }
            }
            parity ^= 1u << b;
            ++next;
        }
    }
    // the test hook's slab of item 0
    __device__ bool dropped(int sidx) const { return a.drop_slab == sidx + 1 && q_cur == 0; }
    __device__ cplx<real>* wait(int sidx) {
        const int b = sidx % NBUF;
        // the default poll limit, or the test's lower one for the copy it withheld
        const unsigned polls = dropped(sidx) ? a.wait_polls : 0u;
        if (!*aborted && !mbar_wait(&mbar[b], ((parity >> b) & 1u) ^ 1u, a.flags, polls)) *aborted = 1;
        return buf(b);
    }
    // before an aborted CTA exits, thread 0 (which issued every copy) waits
    // for the latest armed phase of each buffer, bounded: a consumed or
    // never-armed buffer passes at once, a copy still in flight lands, the
    // phase whose copy never came runs out once more
    __device__ void drain() {
        if (threadIdx.x == 0)
            for (int b = 0; b < NBUF; ++b)
                mbar_wait(&mbar[b], ((armed >> b) & 1u) ^ 1u, nullptr, b == (int)withheld ? a.wait_polls : 0u);
    }

    // forward y-FFT of slab sidx; adds ky^pow * F_y(G) to nl
    __device__ void forward(int sidx, int pow, cplx<real> (&nl)[E]) {
        cplx<real>* b = wait(sidx);
        cplx<real> v[E];
#pragma unroll
        for (int e = 0; e < E; ++e) v[e] = b[(t + TEAM * e) * TW + w];
        if constexpr (DB) {
            fft.template run_db<false, SWZ>(t, v, xbuf, b, w, TW);
        } else {
            X x{b, w, TW};
            x.sync();
            fft.template run<false>(t, v, x);
        }
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const real ky = ky_of<real>(t + TEAM * e, N, a.dky);
            const real m = pow == 0 ? (real)1 : (pow == 1 ? ky : ky * ky);
            nl[e] = cadd(nl[e], cscale(v[e], m));
        }
        issue_upto(sidx + NBUF + 1);
    }

    // field f of the current tile; its slabs start at s0
    __device__ void field(int f, int s0) { field_body(f, s0); }
    __device__ __forceinline__ void field_body(int f, int s0) {
        const int i = T * TW + w;
        const bool edge_col = (i == 0);   // kx = 0 belongs to the edge item
        const real kx = a.dkx * (real)i;
        const real sc = SQ ? (real)1 / ((real)N * (real)N) : (real)1 / ((real)a.nx * (real)a.ny);
        const int ng = nG(f);
        const size_t base = io + (size_t)T * SLAB;
        cplx<real> nl[E], curr[E];
#pragma unroll
        for (int e = 0; e < E; ++e) nl[e] = mk<real>(0, 0);
        for (int g = 0; g < ng; ++g) forward(s0 + g, g, nl);

        if (a.mode == MODE_NONL) {
            cplx<real>* out = pick3(a.nl_m, f) + base;
            if (!edge_col)
#pragma unroll
                for (int e = 0; e < E; ++e) out[(t + TEAM * e) * TW + w] = nl[e];
            return;
        }
        // stage update, old and acc read from their slabs
        const int so = s0 + ng, sa = so + (need_old ? 1 : 0);
        const cplx<real>* ob = need_old ? wait(so) : nullptr;
        const cplx<real>* ab = need_acc ? wait(sa) : nullptr;
        cplx<real>* om = pick3(a.old_m, f) + base;
        cplx<real>* am = pick3(a.acc_m, f) + base;
        double zsum = 0, esum = 0;
        bool bad = false;
        if (a.mode == MODE_PROLOGUE) {
#pragma unroll
            for (int e = 0; e < E; ++e) curr[e] = ob[(t + TEAM * e) * TW + w];
        } else {
            const int cls = f == 0 ? 0 : 2;
            const real* e0 = a.inst_e0 ? a.inst_e0 + 4 * inst : a.e0;
            const real exf = table(&a.ex[cls * (Hx() + 1) + i]) * e0[cls];
            const real exh = table(&a.ex[(cls + 1) * (Hx() + 1) + i]) * e0[cls + 1];
            // the y factors of PF elements at a time first (through the
            // read-only path when PF > 1): fetched inside the loop, each load
            // would wait behind the previous element's stores (the compiler
            // cannot rule out aliasing), exposing the L2 latency once per
            // element
#pragma unroll
            for (int c0 = 0; c0 < E; c0 += PF) {
                real Efs[PF], Ehs[PF];
#pragma unroll
                for (int c = 0; c < PF; ++c) {
                    const int j = t + TEAM * (c0 + c);
                    if constexpr (DB) {
                        Efs[c] = exf * eys[cls * N + j];
                        Ehs[c] = exh * eys[(cls + 1) * N + j];
                    } else {
                        Efs[c] = exf * table(&a.ey[cls * N + j]);
                        Ehs[c] = exh * table(&a.ey[(cls + 1) * N + j]);
                    }
                }
#pragma unroll
                for (int c = 0; c < PF; ++c) {
                    const int e = c0 + c;
                    const int j = t + TEAM * e;
                    const int li = j * TW + w;
                    const real Ef = Efs[c];
                    const real Eh = Ehs[c];
                    const cplx<real> o = need_old ? ob[li] : mk<real>(0, 0);
                    const cplx<real> ac = need_acc ? ab[li] : mk<real>(0, 0);
                    StageUpdate<real> u = stage_update(a, nl[e], o, ac, Ef, Eh, mask_keep(a, f, i, j));
                    if (!edge_col) {
                        if (u.write_acc) am[li] = u.acc;
                        if (u.write_old) {
                            om[li] = u.acc;
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
            }
            if (a.last_stage) {
                const bool full_warps = (blockDim.x & 31) == 0;
                if (full_warps) {
                    if (a.flags && __any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(a.flags, FLAG_NONFINITE);
                    if (f == 0 && a.diag) {
#pragma unroll
                        for (int o = 16; o > 0; o >>= 1) {
                            zsum += __shfl_xor_sync(0xffffffffu, zsum, o);
                            esum += __shfl_xor_sync(0xffffffffu, esum, o);
                        }
                        if constexpr (CTA_DIAG) {
                            const int wid = threadIdx.x >> 5;
                            if ((threadIdx.x & 31) == 0) { red[2 * wid] = zsum; red[2 * wid + 1] = esum; }
                            __syncthreads();
                            if (threadIdx.x == 0) {
                                double z = 0, en = 0;
                                for (int k = 0; k < (int)(blockDim.x >> 5); ++k) { z += red[2 * k]; en += red[2 * k + 1]; }
                                double* dg = a.diag + a.diag_istride * inst;
                                atomicAdd(&dg[0], z); atomicAdd(&dg[1], en);
                            }
                        } else if ((threadIdx.x & 31) == 0) {
                            double* dg = a.diag + a.diag_istride * inst;
                            atomicAdd(&dg[0], zsum); atomicAdd(&dg[1], esum);
                        }
                    }
                } else {
                    if (a.flags && bad) atomicOr(a.flags, FLAG_NONFINITE);
                    if (f == 0 && a.diag) {
                        double* dg = a.diag + a.diag_istride * inst;
                        atomicAdd(&dg[0], zsum); atomicAdd(&dg[1], esum);
                    }
                }
            }
        }
        // the buffer of the last state slab hosts the inverse transforms; the
        // other one is free now
        const int sx = need_acc ? sa : so;
        if (need_old && need_acc) issue_upto(so + NBUF + 1);
        if (!a.do_inverse) { issue_upto(sx + NBUF + 1); return; }
        X x{buf(sx % NBUF), w, TW};
        // every thread has read its old/acc values (MODE 2: the first
        // exchange writes the extra buffer, and its barrier comes first)
        if constexpr (!DB) x.sync();
        const int nq = f == 0 ? 4 : 2;
        for (int qq = 0; qq < nq; ++qq) {
            const int q = f == 0 ? (qq == 0 ? 0 : qq + 2) : (f == 1 ? (qq == 0 ? 1 : 6) : (qq == 0 ? 2 : 7));
            cplx<real> v[E];
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const real ky = ky_of<real>(t + TEAM * e, N, a.dky);
                v[e] = y_mult<real>(q, curr[e], ky, kx * kx + ky * ky, sc);
            }
            if constexpr (DB) fft.template run_db<true, SWZ>(t, v, xbuf, buf(sx % NBUF), w, TW);
            else fft.template run<true>(t, v, x);
            cplx<real>* Y = a.Y + io + (size_t)q * N * Hx() + i;
#pragma unroll
            for (int e = 0; e < E; ++e) Y[(size_t)(t + TEAM * e) * Hx()] = v[e];
            if constexpr (!DB) x.sync();   // the next transform reuses the buffer
        }
        issue_upto(sx + NBUF + 1);
    }

    // a regular item: the fields fa_ (and fb_ >= 0) of tile T_ of instance inst_
    __device__ void item(int fa_, int fb_, int T_, int inst_) { item_body(fa_, fb_, T_, inst_); }
    __device__ __forceinline__ void item_body(int fa_, int fb_, int T_, int inst_) {
        fa = fa_; fb = fb_; T = T_;
        inst = inst_;
        io = (size_t)inst_ * a.istride;
        need_old = a.mode == MODE_PROLOGUE || (a.mode == MODE_STAGE &&
                   (a.integrator == INT_IFE || (a.integrator == INT_IFRK4 && a.stage <= 3) ||
                    (a.integrator == INT_IFRK2 && a.stage == 1)));
        need_acc = a.mode == MODE_STAGE && ((a.integrator == INT_IFRK4 && a.stage >= 2) ||
                                            (a.integrator == INT_IFRK2 && a.stage == 2));
        per_a = per_field(fa);
        nseq = per_a + (fb >= 0 ? per_field(fb) : 0);
        next = 0;
        issue_upto(NBUF);
        if constexpr (ONE_BODY) {
            // one copy of the field code for both fields (and, through the
            // kernel's single call, both item kinds): less code to fetch
#pragma unroll 1
            for (int k = 0; k < 2; ++k) {
                const int f = k == 0 ? fa : fb;
                if (f < 0) break;
                field_body(f, k == 0 ? 0 : per_a);
            }
        } else if constexpr (INLINE_ITEM) {
            field_body(fa, 0);
            if (fb >= 0) field_body(fb, per_a);
        } else {
            field(fa, 0);
            if (fb >= 0) field(fb, per_a);
        }
        __syncthreads();   // buffers free for the next item
    }
};

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

template <typename real, int N, int W, int E, bool SQ = true>
__device__ __forceinline__ void col_edge(const StageArgs<real>& a, int f, int inst, int t, int w, cplx<real>* buf,
                                         cplx<real>* ctab) {
    const size_t io = (size_t)inst * a.istride;
    constexpr int TEAM = N / E;
    const int H = SQ ? N / 2 : a.nx / 2;   // the kx = nx/2 column
    XchgCols<real> x{buf, w, W};
    TeamFFT<real, N, E> fft;
    fft.template init<N>(t, a.tw_y);
    const real kN = a.dkx * (real)H;
    const real s = SQ ? (real)1 / ((real)N * (real)N) : (real)1 / ((real)a.nx * (real)a.ny);
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
            for (int e = 0; e < E; ++e) v[e] = active ? a.Ed[io + (size_t)p * N + t + TEAM * e] : mk<real>(0, 0);
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
                        for (int ww = 0; ww < W; ++ww) acc = cadd(acc, x.read_team(j, ww));
                        ctab[col * N + j] = acc;
                    }
                x.sync();
            }
        }
    }

    if (w == 0) {
        cplx<real>* om = pick3(a.old_m, f) + io;
        cplx<real>* on = pick3(a.old_n, f) + io;
        cplx<real>* am = pick3(a.acc_m, f) + io;
        cplx<real>* an = pick3(a.acc_n, f) + io;
        if (a.mode == MODE_NONL) {
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int j = t + TEAM * e;
                pick3(a.nl_m, f)[io + (size_t)j * TW] = ctab[j];
                pick3(a.nl_n, f)[io + j] = ctab[N + j];
            }
        } else if (a.mode == MODE_PROLOGUE) {
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int j = t + TEAM * e;
                ctab[j] = om[(size_t)j * TW];
                ctab[N + j] = on[j];
            }
        } else {
            const bool need_old = a.integrator == INT_IFE || (a.integrator == INT_IFRK4 && a.stage <= 3) ||
                                  (a.integrator == INT_IFRK2 && a.stage == 1);
            const bool need_acc = (a.integrator == INT_IFRK4 && a.stage >= 2) || (a.integrator == INT_IFRK2 && a.stage == 2);
            const int cls = f == 0 ? 0 : 2;
            bool bad = false;
            const real* e0 = a.inst_e0 ? a.inst_e0 + 4 * inst : a.e0;
            const real f0 = e0[cls], f1 = e0[cls + 1];
            // chunks of C elements: the chunk's factors and state are read
            // before any of its stores, so that their loads overlap (one
            // element at a time at 1024^2, where the registers are short)
            constexpr int C = N >= 1024 ? 1 : (E < 4 ? E : 4);
            auto table = [](const real* p) -> real {
                if constexpr (C > 1) return __ldg(p);
                else return *p;
            };
            const real x0f = table(&a.ex[cls * (H + 1)]), x0h = table(&a.ex[(cls + 1) * (H + 1)]);
            const real xHf = table(&a.ex[cls * (H + 1) + H]), xHh = table(&a.ex[(cls + 1) * (H + 1) + H]);
#pragma unroll
            for (int c0 = 0; c0 < E; c0 += C) {
                real eyf[C], eyh[C];
                cplx<real> o0[C], a0[C], oH[C], aH[C];
#pragma unroll
                for (int c = 0; c < C; ++c) {
                    const int j = t + TEAM * (c0 + c);
                    eyf[c] = table(&a.ey[cls * N + j]) * f0;
                    eyh[c] = table(&a.ey[(cls + 1) * N + j]) * f1;
                    o0[c] = need_old ? om[(size_t)j * TW] : mk<real>(0, 0);   // tile 0, column 0
                    a0[c] = need_acc ? am[(size_t)j * TW] : mk<real>(0, 0);
                    oH[c] = need_old ? on[j] : mk<real>(0, 0);
                    aH[c] = need_acc ? an[j] : mk<real>(0, 0);
                }
#pragma unroll
                for (int c = 0; c < C; ++c) {
                    const int j = t + TEAM * (c0 + c);
                    // column kx = 0
                    {
                        const size_t idx = (size_t)j * TW;
                        const real Ef = x0f * eyf[c], Eh = x0h * eyh[c];
                        StageUpdate<real> u = stage_update(a, ctab[j], o0[c], a0[c], Ef, Eh, mask_keep(a, f, 0, j));
                        if (u.write_acc) am[idx] = u.acc;
                        if (u.write_old) {
                            om[idx] = u.acc;
                            bad |= !(isfinite(u.acc.x) && isfinite(u.acc.y));
                        }
                        ctab[j] = u.curr;
                    }
                    // column kx = N/2
                    {
                        const real Ef = xHf * eyf[c], Eh = xHh * eyh[c];
                        StageUpdate<real> u = stage_update(a, ctab[N + j], oH[c], aH[c], Ef, Eh, mask_keep(a, f, H, j));
                        if (u.write_acc) an[j] = u.acc;
                        if (u.write_old) {
                            on[j] = u.acc;
                            bad |= !(isfinite(u.acc.x) && isfinite(u.acc.y));
                        }
                        ctab[N + j] = u.curr;
                    }
                }
            }
            if (a.last_stage && bad && a.flags) atomicOr(a.flags, FLAG_NONFINITE);
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
        double* dg = a.diag + a.diag_istride * inst;
        atomicAdd(&dg[0], zsum);
        atomicAdd(&dg[1], esum);
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
            for (int e = 0; e < E; ++e) a.D[io + (size_t)p * N + t + TEAM * e] = v[e];
    }
}

// ---------------------------------------------------------------------------
// Field-parallel column pass of one small square grid (32^2, 128^2 or
// 256^2, a single instance). The persistent kernel's CTA runs an item's seven or eight
// y-transforms one after another, and a small grid has too few items to fill
// the GPU with them; here one CTA per kx-column runs all of that column's
// transforms at once — NTF = 8 teams, one per G array in the forward phase
// (the eighth idle), one per Y array in the inverse phase — so a CTA's chain
// is one forward transform, the stage update of the three fields and one
// inverse transform. The last three CTAs take the kx = 0 / N/2 edge columns
// of w, r1 and r2 (col_edge, the persistent kernel's edge item).
// The arithmetic of every value is the persistent kernel's (the same
// transforms, products and stage formulas in the same order); only the
// diagnostics' partial sums are added in another order.
// ---------------------------------------------------------------------------
template <typename real, int N, int E>
struct ColFP {
    static constexpr int TEAM = N / E, NTF = 8, NTHREADS = NTF * TEAM;
    // team buffers [NTF][N] | curr of the three fields [3][N] | 64 doubles of diagnostic sums
    static constexpr size_t SMEM = (size_t)(NTF + 3) * N * sizeof(cplx<real>) + 64 * sizeof(double);
    static_assert(N >= 32 && N <= 256, "small grids (whole warps of threads)");
};

template <typename real, int N, int E>
__global__ void __launch_bounds__(ColFP<real, N, E>::NTHREADS) colfp_kernel(const __grid_constant__ StageArgs<real> a) {
    using K = ColFP<real, N, E>;
    constexpr int TEAM = K::TEAM, NTF = K::NTF, NT = K::NTHREADS, H = N / 2;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    cplx<real>* sm = reinterpret_cast<cplx<real>*>(smem_raw);
    const int tid = threadIdx.x;
    if ((int)blockIdx.x >= H) {   // edge CTAs: field blockIdx.x - H, NTF teams share its transforms
        col_edge<real, N, NTF, E, true>(a, (int)blockIdx.x - H, 0, tid / NTF, tid % NTF, sm, sm + (size_t)N * NTF);
        return;
    }
    const int g = tid / TEAM, t = tid % TEAM;   // team g (G_g forward, Y_g inverse), transform index t
    const int i = (int)blockIdx.x;              // the kx-column
    const bool edge_col = (i == 0);             // kx = 0 belongs to the edge CTAs
    cplx<real>* cur = sm + (size_t)NTF * N;     // curr of field f at cur[f * N + j]
    double* red = reinterpret_cast<double*>(sm + (size_t)(NTF + 3) * N);
    XchgCols<real> x{sm + (size_t)g * N, 0, 1};
    TeamFFT<real, N, E> fft;
    fft.template init<N>(t, a.tw_y);
    const real kx = a.dkx * (real)i;
    const real sc = (real)1 / ((real)N * (real)N);
    cplx<real> v[E];

    // forward: team g < NG transforms column i of G_g and leaves ky^pow F_y(G_g)
    // in its buffer (pow 0, 1, 2 for G0-G2 of w; 0, 1 for G3-G4 of r1 and G5-G6 of r2)
    if (a.mode != MODE_PROLOGUE) {
        const bool act = g < NG;
        const cplx<real>* Gc = a.G + (size_t)(act ? g : 0) * N * H + i;
#pragma unroll
        for (int e = 0; e < E; ++e) v[e] = act ? Gc[(size_t)(t + TEAM * e) * H] : mk<real>(0, 0);
        fft.template run<false>(t, v, x);
        const int pw = (g == 0 || g == 3 || g == 5) ? 0 : (g == 2 ? 2 : 1);
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const real ky = ky_of<real>(t + TEAM * e, N, a.dky);
            const real m = pw == 0 ? (real)1 : (pw == 1 ? ky : ky * ky);
            x.write(t + TEAM * e, cscale(v[e], m));
        }
        __syncthreads();
    }

    // stage update of the three fields at every ky of the column
    const bool need_old = a.mode == MODE_PROLOGUE || (a.mode == MODE_STAGE &&
                          (a.integrator == INT_IFE || (a.integrator == INT_IFRK4 && a.stage <= 3) ||
                           (a.integrator == INT_IFRK2 && a.stage == 1)));
    const bool need_acc = a.mode == MODE_STAGE && ((a.integrator == INT_IFRK4 && a.stage >= 2) ||
                                                   (a.integrator == INT_IFRK2 && a.stage == 2));
    double zsum = 0, esum = 0;
    bool bad = false;
    for (int it = tid; it < 3 * N; it += NT) {
        const int f = it / N, j = it % N;
        const size_t li = tidx(N, i, j);
        cplx<real> nl = mk<real>(0, 0);
        if (a.mode != MODE_PROLOGUE) {
            const int g0 = f == 0 ? 0 : (f == 1 ? 3 : 5), ng = f == 0 ? 3 : 2;
            for (int gg = 0; gg < ng; ++gg) nl = cadd(nl, sm[(size_t)(g0 + gg) * N + j]);
        }
        if (a.mode == MODE_NONL) {
            if (!edge_col) pick3(a.nl_m, f)[li] = nl;
            continue;
        }
        cplx<real> c;
        if (a.mode == MODE_PROLOGUE) {
            c = pick3(a.old_m, f)[li];
        } else {
            const int cls = f == 0 ? 0 : 2;
            const real* e0 = a.inst_e0 ? a.inst_e0 : a.e0;
            const real exf = a.ex[cls * (H + 1) + i] * e0[cls];
            const real exh = a.ex[(cls + 1) * (H + 1) + i] * e0[cls + 1];
            const real Ef = exf * a.ey[cls * N + j], Eh = exh * a.ey[(cls + 1) * N + j];
            const cplx<real> o = need_old ? pick3(a.old_m, f)[li] : mk<real>(0, 0);
            const cplx<real> ac = need_acc ? pick3(a.acc_m, f)[li] : mk<real>(0, 0);
            const StageUpdate<real> u = stage_update(a, nl, o, ac, Ef, Eh, mask_keep(a, f, i, j));
            if (!edge_col) {
                if (u.write_acc) pick3(a.acc_m, f)[li] = u.acc;
                if (u.write_old) {
                    pick3(a.old_m, f)[li] = u.acc;
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
            c = u.curr;
        }
        cur[(size_t)f * N + j] = c;
    }
    if (a.mode == MODE_STAGE && a.last_stage) {
        if (a.flags && __any_sync(0xffffffffu, bad) && (tid & 31) == 0) atomicOr(a.flags, FLAG_NONFINITE);
        if (a.diag) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                zsum += __shfl_xor_sync(0xffffffffu, zsum, o);
                esum += __shfl_xor_sync(0xffffffffu, esum, o);
            }
            if ((tid & 31) == 0) { red[2 * (tid >> 5)] = zsum; red[2 * (tid >> 5) + 1] = esum; }
        }
    }
    __syncthreads();
    if (a.mode == MODE_STAGE && a.last_stage && a.diag && tid == 0) {
        double z = 0, en = 0;
        for (int k = 0; k < NT / 32; ++k) { z += red[2 * k]; en += red[2 * k + 1]; }
        atomicAdd(&a.diag[0], z);
        atomicAdd(&a.diag[1], en);
    }
    if (a.mode == MODE_NONL || !a.do_inverse) return;

    // inverse: team q = g transforms the multiplied curr of its field into Y_q
    const int q = g, fq = (q == 1 || q == 6) ? 1 : ((q == 2 || q == 7) ? 2 : 0);
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int j = t + TEAM * e;
        const real ky = ky_of<real>(j, N, a.dky);
        v[e] = y_mult<real>(q, cur[(size_t)fq * N + j], ky, kx * kx + ky * ky, sc);
    }
    fft.template run<true>(t, v, x);
    cplx<real>* Y = a.Y + (size_t)q * N * H + i;
#pragma unroll
    for (int e = 0; e < E; ++e) Y[(size_t)(t + TEAM * e) * H] = v[e];
}

template <typename real, int N, int E, int MINB, int MODE = 0, bool SQ = true>
__global__ void __launch_bounds__(TW * (N / E), MINB) col_kernel(const __grid_constant__ StageArgs<real> a) {
    using K = ColKernel<real, N, E, MODE, SQ>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    cplx<real>* bufs = reinterpret_cast<cplx<real>*>(smem_raw);
    const int tid = threadIdx.x, w = tid % TW, t = tid / TW;
    cplx<real>* ctab;
    double* red;
    uint64_t* mbar;
    typename K::FFT fft;
    cplx<real>* xbuf = nullptr;
    real* eys = nullptr;
    if constexpr (K::SB) {
        cplx<real>* table = bufs + (K::NBUF + (K::DB ? 1 : 0)) * K::SLAB;
        if constexpr (K::DB) {
            xbuf = bufs + K::NBUF * K::SLAB;
            eys = reinterpret_cast<real*>(table + K::FFT::ENTRIES);
            for (int k = tid; k < 4 * N; k += blockDim.x) eys[k] = a.ey[k];
        }
        ctab = bufs + K::SLAB;
        red = reinterpret_cast<double*>(reinterpret_cast<unsigned char*>(table + K::FFT::ENTRIES) +
                                        (K::DB ? 4 * N * sizeof(real) : 0));
        mbar = reinterpret_cast<uint64_t*>(red + 64);
        if (w == 0) K::FFT::template fill<N>(table, t, a.tw_y);
        fft.tab = table + t;
    } else {
        ctab = bufs + 3 * K::SLAB;
        red = reinterpret_cast<double*>(ctab);
        mbar = reinterpret_cast<uint64_t*>(ctab + 2 * N);
        fft.template init<N>(t, a.tw_y);
    }
    int* item_sh = reinterpret_cast<int*>(mbar + K::NBUF);
    volatile int* aborted = item_sh + 1;
    if (tid == 0) {
        for (int b = 0; b < K::NBUF; ++b) mbar_init(&mbar[b], 1);
        *aborted = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();   // barriers initialised, twiddle table filled
    K k{a, fft, t, w, bufs, mbar, aborted, 0u, 0, 0, 0, 0, 0, 0, false, false};
    k.red = red;
    k.xbuf = xbuf;
    k.eys = eys;
    k.armed = 0u;
    k.withheld = (unsigned)K::NBUF;
    // item q of the launch: kind-major over instances (all r1+r2 tiles of all
    // instances first, then the w tiles, then the edge columns)
    const int tiles = k.Hx() / TW;
    const int total = (2 * tiles + 3) * a.ninst;
    for (;;) {
        if (tid == 0) *item_sh = atomicAdd(a.queue, 1);
        __syncthreads();
        const int q = *item_sh;
        const bool stop = *aborted != 0;   // written before the barrier above
        __syncthreads();
        if (stop) {
            k.drain();
            break;
        }
        if (q >= total) break;
        k.q_cur = q;
        const int local = q / a.ninst, inst = q % a.ninst;
        if (K::ONE_BODY && local < 2 * tiles) {
            const bool rp = local < tiles;   // r1 + r2 of tile `local`, else w of tile local - tiles
            k.item_body(rp ? 1 : 0, rp ? 2 : -1, rp ? local : local - tiles, inst);
        } else if (local < tiles) {
            if constexpr (K::INLINE_ITEM) k.item_body(1, 2, local, inst);
            else k.item(1, 2, local, inst);
        } else if (local < 2 * tiles) {
            if constexpr (K::INLINE_ITEM) k.item_body(0, -1, local - tiles, inst);
            else k.item(0, -1, local - tiles, inst);
        } else {
            col_edge<real, N, TW, E, SQ>(a, local - 2 * tiles, inst, t, w, bufs, ctab);
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------
// Row kernel: ROWS rows per CTA, a team of N/E threads per row. N is the row
// length nx; the number of rows, ny, is a launch argument (ROWS divides it).
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
    __device__ void write(int idx, cplx<real> v) { buf[swz(idx)] = v; }
    __device__ cplx<real> read(int idx) const { return buf[swz(idx)]; }
    __device__ void sync() {
        if constexpr (NAMED) asm volatile("bar.sync %0, %1;" ::"r"(id), "n"(TEAM) : "memory");
        else __syncthreads();
    }
};

// MODE 1: the twiddle bases in a shared table after the rows' regions
// (TeamFFTShared), shared by the CTA's row teams
template <typename real, int N, int E, int ROWS, int MODE = 0, bool SQ = true>
struct RowKernel {
    static constexpr int H = N / 2, TEAM = N / E, PH = E / 2;
    static constexpr bool SB = MODE >= 1;
    // the R2C unpack's partner values by warp shuffle where a team lies within
    // one warp and the CTA is whole warps (N <= 256 at 8 values per thread;
    // measured per step on one box, 85-instance batches: 256^2 1552 -> 1474
    // us, 128^2 593 -> 581, 64^2 177 -> 170)
    static constexpr bool SHFL = TEAM <= 32 && (ROWS * TEAM) % 32 == 0;
    using FFT = std::conditional_t<SB, TeamFFTShared<real, N, E>, TeamFFT<real, N, E>>;
    // a named barrier per row team when teams are whole warps and there is more than one team
    static constexpr bool NAMED = (TEAM % 32 == 0) && ROWS > 1 && ROWS <= 15;
    using X = XchgTeam<real, TEAM, NAMED>;
    static constexpr int NKEEP = 5;   // r1, r2, w, two scratch products
    static constexpr size_t SMEM_PER_ROW = N * sizeof(cplx<real>) + NKEEP * N * sizeof(real);
    static constexpr size_t SMEM = ROWS * SMEM_PER_ROW + (SB ? TeamFFTShared<real, N, E>::ENTRIES * sizeof(cplx<real>) : 0);

    const StageArgs<real>& a;
    int n, t;
    X x;
    real* keep;            // [NKEEP][N], point m at [slot][m]
    int inst;              // instance of this row
    size_t io;             // its buffer offset (complex elements)
    FFT fft;

    // planes of the Y/G arrays hold ny rows of H
    // rows ny: N at compile time on a square grid (SQ), else from the launch arguments
    __device__ __forceinline__ int ny() const {
        if constexpr (SQ) return N;
        else return a.ny;
    }
    __device__ size_t plane() const { return (size_t)ny() * H; }
    __device__ cplx<real> yv(int q, int k) const { return a.Y[io + (size_t)q * plane() + (size_t)n * H + k]; }

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
        const cplx<real> da = a.D[io + (size_t)pa * ny() + n];
        const cplx<real> db = pb >= 0 ? a.D[io + (size_t)pb * ny() + n] : mk<real>(0, 0);
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
        if constexpr (SHFL) {
            // the partner Z[N - k] of k = t + TEAM e sits in lane (TEAM - t) % TEAM
            // of this team, register E - 1 - e (t > 0) or E - e (t = 0, own):
            // one shuffle per value, no shared-memory round trip or barrier
            const int src = (TEAM - t) % TEAM;
#pragma unroll
            for (int e = 0; e < PH; ++e) {
                const real px = __shfl_sync(0xffffffffu, v[E - 1 - e].x, src, TEAM);
                const real py = __shfl_sync(0xffffffffu, v[E - 1 - e].y, src, TEAM);
                const int k = t + TEAM * e;
                if (k == 0) continue;
                const cplx<real> z = v[e];
                const cplx<real> zm = cconj(t == 0 ? v[(E - e) % E] : mk<real>(px, py));
                emit(k, cscale(cadd(z, zm), (real)0.5), cmul_mi(cscale(csub(z, zm), (real)0.5)), ga[e], gb[e]);
            }
            if (t == 0) {
                const cplx<real> z0 = v[0], zh = v[PH];   // Z[0], Z[H]
                if (ep >= 0) a.Ed[io + (size_t)ep * ny() + n] = mk<real>(z0.x, zh.x);
                if (eq >= 0) a.Ed[io + (size_t)eq * ny() + n] = mk<real>(z0.y, zh.y);
            }
            return;
        }
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
            if (ep >= 0) a.Ed[io + (size_t)ep * ny() + n] = mk<real>(z0.x, zh.x);
            if (eq >= 0) a.Ed[io + (size_t)eq * ny() + n] = mk<real>(z0.y, zh.y);
        }
        x.sync();
    }

    __device__ cplx<real>* grow(int g) const { return a.G + io + (size_t)g * plane() + (size_t)n * H; }
    __device__ real& kp(int f, int e) const { return keep[f * N + t + TEAM * e]; }
    __device__ void zero_slot0(int g) const { if (t == 0) grow(g)[0] = mk<real>(0, 0); }
    __device__ void dump(int fld, const cplx<real> (&v)[E], bool imag) const {
        if (!a.phys_out) return;
        real* o = a.phys_out + a.phys_istride * inst + (size_t)fld * N * ny() + (size_t)n * N;
#pragma unroll
        for (int e = 0; e < E; ++e) o[t + TEAM * e] = imag ? v[e].y : v[e].x;
    }
    __device__ void dump_slot(int fld, int slot) const {
        if (!a.phys_out) return;
        real* o = a.phys_out + a.phys_istride * inst + (size_t)fld * N * ny() + (size_t)n * N;
#pragma unroll
        for (int e = 0; e < E; ++e) o[t + TEAM * e] = kp(slot, e);
    }
    __device__ real alpha_at(int e) const {
        if (a.alpha_field) return __ldg(&a.alpha_field[a.alpha_istride * inst + (size_t)n * N + t + TEAM * e]);
        return a.inst_alpha ? a.inst_alpha[inst] : a.alpha;
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
        // the column kernel that follows takes its work items from this counter
        if (a.queue && blockIdx.x == 0 && threadIdx.x == 0) *a.queue = 0;
        if constexpr (!SB) fft.template init<N>(t, a.tw);   // (MODE 1: filled by the kernel)
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
        // the activities first: read in the loop, each would wait behind the
        // previous element's shared-memory stores (possible aliasing)
        real alv[E];
#pragma unroll
        for (int e = 0; e < E; ++e) alv[e] = alpha_at(e);
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const real r1 = kp(0, e), r2 = kp(1, e), L1 = v[e].x, L2 = v[e].y, al = alv[e];
            const real S = 2 * sqrt(r1 * r1 + r2 * r2);
            const real sgl = lam * S * (S * S - 1);
            const real sg2 = -lam * L2 * S + sgl * r2;
            const real p11 = -lam * L1 * S + sgl * r1 - al * r1;
            const real p12 = sg2 + (2 * L1 * r2 - 2 * r1 * L2) - al * r2;
            kp(4, e) = sg2 + (2 * L2 * r1 - 2 * r2 * L1) - al * r2;
            v[e] = mk<real>(p11, p12);
            if (a.phys_out && a.phys_all) kp(3, e) = S;
        }
        if (a.phys_out && a.phys_all) { dump_slot(9, 3); dump(10, v, false); dump(11, v, true); dump_slot(12, 4); }
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

template <typename real, int N, int E, int ROWS, int MINB, int MODE = 0, bool SQ = true>
__global__ void __launch_bounds__(ROWS * (N / E), MINB) row_kernel(const StageArgs<real> a) {
    using K = RowKernel<real, N, E, ROWS, MODE, SQ>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int r = threadIdx.x / K::TEAM, t = threadIdx.x % K::TEAM;
    unsigned char* mine = smem_raw + (size_t)r * K::SMEM_PER_ROW;
    const int BLOCKS_PER_INST = (SQ ? N : a.ny) / ROWS;   // rows of an instance (ny) by ROWS per CTA
    const int inst = (int)blockIdx.x / BLOCKS_PER_INST;
    K k{a, ((int)blockIdx.x % BLOCKS_PER_INST) * ROWS + r, t,
        typename K::X{reinterpret_cast<cplx<real>*>(mine), 1 + r},
        reinterpret_cast<real*>(mine + N * sizeof(cplx<real>)), inst, (size_t)inst * a.istride, {}};
    if constexpr (K::SB) {
        cplx<real>* table = reinterpret_cast<cplx<real>*>(smem_raw + (size_t)ROWS * K::SMEM_PER_ROW);
        if (r == 0) K::FFT::template fill<N>(table, t, a.tw);
        k.fft.tab = table + t;
        __syncthreads();
    }
    static_assert(K::PH * K::TEAM == N / 2, "row team layout");
    k.run();
}

// ---------------------------------------------------------------------------
// Layout conversion between the reference's spectral layout (i + j*(N/2+1))
// and the internal split layout (main[tidx(i, j)], nyq[j]).
// ---------------------------------------------------------------------------
template <typename real>
__global__ void ref_to_internal(const cplx<real>* __restrict__ ref, cplx<real>* __restrict__ m, cplx<real>* __restrict__ nq, int nx,
                                int ny) {
    const int H = nx / 2, nxh = H + 1;
    const size_t total = (size_t)nxh * ny;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < total; k += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(k / nxh), i = (int)(k % nxh);
        if (i < H) m[tidx(ny, i, j)] = ref[k];
        else nq[j] = ref[k];
    }
}

template <typename real>
__global__ void internal_to_ref(const cplx<real>* __restrict__ m, const cplx<real>* __restrict__ nq, cplx<real>* __restrict__ ref, int nx,
                                int ny) {
    const int H = nx / 2, nxh = H + 1;
    const size_t total = (size_t)nxh * ny;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < total; k += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(k / nxh), i = (int)(k % nxh);
        ref[k] = (i < H) ? m[tidx(ny, i, j)] : nq[j];
    }
}

// batched forms: instance k (blockIdx.y) at m + k * istride, nq + k * istride, ref + k * ref_istride
template <typename real>
__global__ void ref_to_internal_batch(const cplx<real>* __restrict__ ref, size_t ref_istride, cplx<real>* __restrict__ m,
                                      cplx<real>* __restrict__ nq, size_t istride, int N) {
    const int H = N / 2, nxh = H + 1;
    const size_t total = (size_t)nxh * N;
    const size_t k0 = blockIdx.y;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < total; k += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(k / nxh), i = (int)(k % nxh);
        const cplx<real> v = ref[k0 * ref_istride + k];
        if (i < H) m[k0 * istride + tidx(N, i, j)] = v;
        else nq[k0 * istride + j] = v;
    }
}
template <typename real>
__global__ void internal_to_ref_batch(const cplx<real>* __restrict__ m, const cplx<real>* __restrict__ nq, size_t istride,
                                      cplx<real>* __restrict__ ref, size_t ref_istride, int N) {
    const int H = N / 2, nxh = H + 1;
    const size_t total = (size_t)nxh * N;
    const size_t k0 = blockIdx.y;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < total; k += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(k / nxh), i = (int)(k % nxh);
        ref[k0 * ref_istride + k] = (i < H) ? m[k0 * istride + tidx(N, i, j)] : nq[k0 * istride + j];
    }
}

}  // namespace qaf
