// qaf_stage.cuh — the fused IF-RK stage of the (w, r1, r2) solver.
//
// One RK stage of the reference (curr_func + wnonl_func + r1nonl_func +
// r2nonl_func + integrate_funcXD, InertialFriction/friction/Qsolver.cuh:166-312,
// TimeIntegration/RK4.cuh:12-74) is two kernels here:
//
//   row kernel     one CTA team per physical row n: 9 half-length C2Rs give
//                  w, r1, r2, u, v, du/dx, du/dy+dv/dx, Lap r1, Lap r2 on the row;
//                  every physical product of the nonlinear terms is formed in
//                  registers; 11 R2Cs, combined with their kx multipliers,
//                  leave 7 "G" arrays (x-spectral, y-physical) and the real
//                  DC/Nyquist values of 10 products ("edge" sequences).
//   column kernel  one CTA per (field, tile of W kx-columns): y-FFTs of the G
//                  arrays, ky multipliers and sum -> N^ for that field; the
//                  IF-RK stage update (dealias and diagnostics at the last
//                  stage); then the inverse y-FFTs of the next stage's
//                  derived spectra -> 8 "Y" arrays for the next row kernel.
//
// The kx = 0 and kx = N/2 columns carry non-Hermitian parts during RK stages
// 2-4. cuFFT's C2R (BwdTrans) sees only their Hermitian parts (measured on the
// B200 with the driver around the reference's build: deviation 2e-16 FP64).
// Those two columns are therefore handled by a dedicated "edge" CTA per field
// that applies every multiplier in full and projects before transforming, so
// the result equals the reference's also where the input is non-Hermitian.
//
// Internal layouts (nx x ny grid, H = nx/2; the row kernel's transforms have
// length nx, the column kernel's length ny). The state is column-tiled so that
// TW adjacent kx columns over all ny rows form one contiguous slab (one TMA
// bulk copy):
//   spectral state, per field: main[tidx(ny, i, j)] for kx index i < H, nyq[j] for i = H,
//   tidx(ny, i, j) = (i / TW) * ny * TW + j * TW + i % TW
//   Y, G arrays: row-major [n * H + k] complex, k = x wave number (k = 0 slot
//   unused); the column kernel fetches TW-column boxes of G with 2D TMA
//   D (9 x ny), Ed (10 x ny): packed (DC + i*Nyquist) per row n
#pragma once

#include "qaf_fft.cuh"

#include <cuda.h>   // CUtensorMap

namespace qaf {

enum StageMode : int { MODE_PROLOGUE = 0, MODE_STAGE = 1, MODE_NONL = 2 };

// kx columns per tile of the column-tiled layouts (32 B of FP32 / 64 B of FP64 complex)
constexpr int TW = 4;
QAF_HD size_t tidx(int N, int i, int j) { return (size_t)(i / TW) * N * TW + (size_t)j * TW + (i % TW); }

// status flags written by the kernels
enum StatusFlag : unsigned { FLAG_NONFINITE = 1u, FLAG_WAIT_TIMEOUT = 2u };
enum Integrator : int { INT_IFE = 0, INT_IFRK2 = 1, INT_IFRK4 = 2 };

// physical fields produced by the row kernel's C2Rs (D slot / field id)
enum PhysField : int { PF_W = 0, PF_R1, PF_R2, PF_U, PF_V, PF_UX, PF_SH, PF_LR1, PF_LR2, PF_COUNT };
// Y arrays (main columns; every entry carries the 1/N^2 of BwdTrans):
//   Y0 w, Y1 r1, Y2 r2, Y3 i ky w/k^2 (= u^), Y4 -w/k^2 (= psi^), Y5 ky^2 psi^, Y6 ky^2 r1, Y7 ky^2 r2
constexpr int NY = 8;
// G arrays (main columns): N^_w = Fy(G0) + ky Fy(G1) + ky^2 Fy(G2),
// N^_r1 = Fy(G3) + ky Fy(G4), N^_r2 = Fy(G5) + ky Fy(G6)
constexpr int NG = 7;
// edge product sequences: 0 -v w, 1 p11, 2 p12, 3 p21, 4 P1, 5 A1=-u r1, 6 B1=-v r1, 7 P2, 8 A2, 9 B2
constexpr int NE = 10;

template <typename real>
struct alignas(64) StageArgs {
    // 2D tensor map over the G arrays viewed as [NG*N rows][H columns] of
    // 8-byte elements (two per FP64 complex), for the column kernel's TMA boxes
    CUtensorMap tm_G;
    // geometry and physics
    int nx, ny;            // grid points along x (rows) and y (columns)
    real dkx, dky;         // 2 pi / Lx, 2 pi / Ly
    real lambda;           // flow alignment
    real ce;               // 1 / (Er Re)
    real alpha;            // constant activity, used when alpha_field == nullptr
    const real* alpha_field;  // N*N physical activity (Ra field) or nullptr
    real dt;
    int advect;            // 1: keep -div(u w) in N_w
    int kx_keep, ky_lo, ky_hi;  // 2/3 mask: keep i <= kx_keep && (j <= ky_lo || j >= ky_hi)
    int trunc;                  // fields the mask truncates after the last stage: bit f for field f
    // spectral state (internal layout)
    cplx<real>* old_m[3];
    cplx<real>* old_n[3];
    cplx<real>* acc_m[3];
    cplx<real>* acc_n[3];
    // nonlinear output (MODE_NONL), internal layout
    cplx<real>* nl_m[3];
    cplx<real>* nl_n[3];
    // intermediates
    cplx<real>* Y;         // NY planes of ny * nx/2
    cplx<real>* D;         // PF_COUNT * ny
    cplx<real>* G;         // NG planes of ny * nx/2
    cplx<real>* Ed;        // NE * ny
    // tables
    const cplx<real>* tw;    // tw[m] = exp(-2 pi i m / nx), m < nx (row transforms)
    const cplx<real>* tw_y;  // tw_y[m] = exp(-2 pi i m / ny), m < ny (column transforms)
    // separable integrating factors: E(i,j) = ex[c][i] * ey[c][j] * e0[c]
    // c = 0: w full step, 1: w half step, 2: Q full step, 3: Q half step
    const real* ex;        // 4 * (nx / 2 + 1)
    const real* ey;        // 4 * ny
    real e0[4];
    // stage control
    int mode, integrator, stage, last_stage, do_inverse;
    // diagnostics / status
    double* diag;          // [0] sum w^2 weights, [1] sum |w|^2/k^2 (half plane, Parseval weights)
    unsigned* flags;       // StatusFlag bits
    unsigned wait_polls;   // tries of a bounded copy wait before it gives up (0: the default)
    int drop_slab;         // test hook, 0: off; k > 0: the column kernel arms slab k - 1 of
                           // queue item 0 (always a tile) without issuing its copy
    int* queue;            // work counter of the persistent column kernel (reset by the row kernel)
    real* phys_out;        // optional: 9 physical fields + S + p11 p12 p21 (13 * nx * ny)
    int phys_all;          // with phys_out: also S, p11, p12, p21 (else the 9 fields only)
    size_t phys_istride;   // reals between instances' phys_out blocks
    // batches of independent instances of the same grid: every buffer above
    // (state, intermediates, D, Ed) of instance k sits istride complex elements
    // after instance k-1's; per-instance parameters come from the inst_ arrays
    int ninst;             // instances in the launch (1: a single grid)
    size_t istride;        // complex elements between instances (a multiple of H)
    const real* inst_alpha;   // constant activity per instance, or nullptr (alpha)
    size_t alpha_istride;     // reals between instances' activity fields (0: shared)
    const real* inst_e0;      // e0[4] per instance, or nullptr (e0)
    size_t diag_istride;      // doubles between instances' diagnostics (0: shared)
};

// Rows per TMA box of the G arrays: at most 256 (the box limit) and a divisor
// of N, so that the boxes of a slab tile its N rows exactly (384 -> 128).
QAF_HDC int g_box_rows(int N) {
    int r = N <= 256 ? N : 256;
    while (N % r != 0) --r;
    return r;
}

template <typename real>
QAF_HD real ky_of(int j, int N, real dky) { return dky * (real)(j <= N / 2 ? j : j - N); }

// ---------------------------------------------------------------------------
// shared-memory exchange for W interleaved teams: element idx of team w at
// buf[idx * W + w] (measured: the exchange swizzle of qaf_fft.cuh slows the
// column kernels, whose interleaved teams already spread the writes)
// ---------------------------------------------------------------------------
template <typename real>
struct XchgCols {
    cplx<real>* buf;
    int w, W;
    __device__ void write(int idx, cplx<real> v) { buf[idx * W + w] = v; }
    __device__ cplx<real> read(int idx) const { return buf[idx * W + w]; }
    __device__ cplx<real> read_team(int idx, int team) const { return buf[idx * W + team]; }
    __device__ void sync() { __syncthreads(); }
};

// one team per row; team r owns buf[r * L ...], element idx at swz(idx)
template <typename real>
struct XchgRow {
    cplx<real>* buf;
    __device__ void write(int idx, cplx<real> v) { buf[swz(idx)] = v; }
    __device__ cplx<real> read(int idx) const { return buf[swz(idx)]; }
    __device__ void sync() { __syncthreads(); }
};

// ---------------------------------------------------------------------------
// IF-RK stage update of one spectral value. Returns the next curr; writes the
// accumulator or (last stage) the dealiased new state.
// ---------------------------------------------------------------------------
template <typename real>
struct StageUpdate {
    cplx<real> curr;
    cplx<real> acc;
    bool write_acc;
    bool write_old;
};

template <typename real>
__device__ __forceinline__ StageUpdate<real> stage_update(const StageArgs<real>& a, cplx<real> nl, cplx<real> old,
                                                           cplx<real> acc, real E, real Eh, bool keep) {
    StageUpdate<real> u;
    u.write_acc = false;
    u.write_old = false;
    const cplx<real> an = cscale(nl, a.dt);
    const real sixth = (real)(1.0 / 6.0), third = (real)(1.0 / 3.0), half = (real)0.5;
    if (a.integrator == INT_IFRK4) {
        if (a.stage == 1) {          // integrate_func0D + 1D (RK4.cuh:12-35)
            u.acc = cadd(cscale(old, E), cscale(an, sixth * E));
            u.curr = cscale(cadd(old, cscale(an, half)), Eh);
            u.write_acc = true;
        } else if (a.stage == 2) {   // integrate_func2D (RK4.cuh:37-48)
            u.acc = cadd(acc, cscale(an, third * Eh));
            u.curr = cadd(cscale(old, Eh), cscale(an, half));
            u.write_acc = true;
        } else if (a.stage == 3) {   // integrate_func3D (RK4.cuh:50-61)
            u.acc = cadd(acc, cscale(an, third * Eh));
            u.curr = cadd(cscale(old, E), cscale(an, Eh));
            u.write_acc = true;
        } else {                     // integrate_func4D + dealias (RK4.cuh:63-74, Qsolver.cuh:314-322)
            cplx<real> nw = cadd(acc, cscale(an, sixth));
            u.acc = keep ? nw : mk<real>(0, 0);
            u.curr = u.acc;
            u.write_old = true;
        }
    } else if (a.integrator == INT_IFRK2) {
        if (a.stage == 1) {          // IF::IFRK2::integrate_func0D + 1D (IFRK2.cuh:16-39), curr factor = E
            u.acc = cadd(cscale(old, E), cscale(an, half * E));
            u.curr = cscale(cadd(old, an), E);
            u.write_acc = true;
        } else {                     // IF::IFRK2::integrate_func2D (IFRK2.cuh:41-51) + dealias
            cplx<real> nw = cadd(acc, cscale(an, half));
            u.acc = keep ? nw : mk<real>(0, 0);
            u.curr = u.acc;
            u.write_old = true;
        }
    } else {                         // IF::IFE::integrate_func1D (IFE.cuh:15-25) + dealias
        cplx<real> nw = cscale(cadd(old, an), E);
        u.acc = keep ? nw : mk<real>(0, 0);
        u.curr = u.acc;
        u.write_old = true;
    }
    return u;
}

template <typename real>
__device__ __forceinline__ bool mask_keep(const StageArgs<real>& a, int f, int i, int j) {
    return !((a.trunc >> f) & 1) || (i <= a.kx_keep && (j <= a.ky_lo || j >= a.ky_hi));
}

// Multiplier (times 1/N^2) that turns the spectral field f into the derived
// spectrum of physical field p, at (kx, ky, k^2).
template <typename real>
__device__ __forceinline__ cplx<real> derived(int p, cplx<real> c, real kx, real ky, real k2, real s) {
    const real ik2 = k2 > (real)0 ? (real)1 / k2 : (real)0;
    switch (p) {
        case PF_W: case PF_R1: case PF_R2: return cscale(c, s);
        case PF_U: return cmul_i(cscale(c, ky * ik2 * s));                    // i ky w / k^2
        case PF_V: return cmul_i(cscale(c, -kx * ik2 * s));                   // -i kx w / k^2
        case PF_UX: return cscale(c, -kx * ky * ik2 * s);                     // i kx u^
        case PF_SH: return cscale(c, (kx * kx - ky * ky) * ik2 * s);          // i ky u^ + i kx v^
        default: return cscale(c, -k2 * s);                                   // Laplacian
    }
}

// The Y arrays a field feeds and their multipliers (main columns)
// (1/k^2 is formed only for the three multipliers that use it)
template <typename real>
__device__ __forceinline__ cplx<real> y_mult(int q, cplx<real> c, real ky, real k2, real s) {
    switch (q) {
        case 0: case 1: case 2: return cscale(c, s);
        case 6: case 7: return cscale(c, ky * ky * s);      // ky^2 r
        default: break;
    }
    const real ik2 = k2 > (real)0 ? (real)1 / k2 : (real)0;
    if (q == 3) return cmul_i(cscale(c, ky * ik2 * s));     // u^ = i ky w / k^2
    if (q == 4) return cscale(c, -ik2 * s);                 // psi^ = -w / k^2
    return cscale(c, -ky * ky * ik2 * s);                   // ky^2 psi^ (q = 5)
}

}  // namespace qaf
