// Host-side emulation of the team FFT in qaf_fft.cuh: every thread of a team
// is run in a loop between the exchange phases, exactly as the kernels
// interleave them with barriers; the result is compared with a direct DFT.
// Built and run by tests/test_native_cpu.py (no GPU needed).
#include "../../nature-control_b200/csrc/qaf_fft.cuh"
#include <cmath>
#include <cstdio>
#include <vector>
#include <complex>

using namespace qaf;

template <typename real, int L, int E, bool INV, int TWN, int P>
void emulate_pass(std::vector<cplx<real>>& regs, const cplx<real>* tw) {
    using Sc = Sched<L, E>;
    constexpr int R = Sc::radix(P), S = Sc::span(P), TEAM = L / E;
    // every thread builds its twiddle bases as the kernels do
    std::vector<TeamFFT<real, L, E>> teams(TEAM);
    for (int t = 0; t < TEAM; ++t) teams[t].template init<TWN>(t, tw);
    for (int t = 0; t < TEAM; ++t) stockham_pass_tw<real, L, E, INV, P>(t, &regs[t * E], teams[t].base);
    if constexpr (P + 1 < Sc::passes) {
        std::vector<cplx<real>> buf(L);
        std::vector<int> hit(L, 0);
        for (int t = 0; t < TEAM; ++t)
            for (int slot = 0; slot < E; ++slot) {
                int d = stockham_dest<L, E, R, S>(t, slot);
                buf[swz(d)] = regs[t * E + slot];   // through the kernels' exchange swizzle
                hit[d]++;
            }
        for (int i = 0; i < L; ++i) if (hit[i] != 1) { std::printf("dest map not a permutation\n"); std::exit(1); }
        for (int t = 0; t < TEAM; ++t)
            for (int e = 0; e < E; ++e) regs[t * E + e] = buf[swz(t + TEAM * e)];
        emulate_pass<real, L, E, INV, TWN, P + 1>(regs, tw);
    }
}

template <typename real, int L, int E, bool INV>
double check() {
    constexpr int TWN = 2 * L, TEAM = L / E;
    std::vector<cplx<real>> tw(TWN);
    for (int m = 0; m < TWN; ++m) {
        long double a = -2.0L * 3.14159265358979323846264338327950288L * m / TWN;
        tw[m] = mk<real>((real)cosl(a), (real)sinl(a));
    }
    std::vector<std::complex<double>> x(L);
    unsigned s = 12345u + L * 7 + E;
    for (int i = 0; i < L; ++i) {
        s = s * 1664525u + 1013904223u; double a = (s >> 8) / 16777216.0 - 0.5;
        s = s * 1664525u + 1013904223u; double b = (s >> 8) / 16777216.0 - 0.5;
        x[i] = {a, b};
    }
    std::vector<cplx<real>> regs(L);
    for (int t = 0; t < TEAM; ++t)
        for (int e = 0; e < E; ++e) regs[t * E + e] = mk<real>((real)x[t + TEAM * e].real(), (real)x[t + TEAM * e].imag());
    emulate_pass<real, L, E, INV, TWN, 0>(regs, tw.data());
    double err = 0, ref = 0;
    for (int k = 0; k < L; ++k) {
        std::complex<long double> acc = 0;
        for (int j = 0; j < L; ++j) {
            long double a = (INV ? 2.0L : -2.0L) * 3.14159265358979323846264338327950288L * ((long long)j * k % L) / L;
            acc += std::complex<long double>(x[j].real(), x[j].imag()) * std::complex<long double>(cosl(a), sinl(a));
        }
        int t = k % TEAM, e = k / TEAM;
        cplx<real> g = regs[t * E + e];
        double dr = (double)g.x - (double)acc.real(), di = (double)g.y - (double)acc.imag();
        err += dr * dr + di * di; ref += (double)(acc.real() * acc.real() + acc.imag() * acc.imag());
    }
    return std::sqrt(err / ref);
}

#define CASE(real, L, E, INV, TOL) do { double e = check<real, L, E, INV>(); \
    std::printf("%-6s L=%-5d E=%-3d inv=%d rel=%.3e\n", #real, L, E, (int)INV, e); if (!(e < TOL)) bad++; } while (0)

// The row kernels' R2C unpack pairs Z[k] (k = t + TEAM e, e < E/2) with
// Z[L - k]; where a team lies within one warp it reads the partner by warp
// shuffle from lane (TEAM - t) % TEAM, register E - 1 - e (t > 0), or from its
// own register (E - e) % E (t = 0), and Z[L/2] from its own register E/2.
// Checks that map against the distribution "thread t holds t + TEAM e".
bool partner_map_ok(int L, int E) {
    const int TEAM = L / E;
    for (int t = 0; t < TEAM; ++t)
        for (int e = 0; e < E / 2; ++e) {
            const int k = t + TEAM * e;
            if (k == 0) continue;
            const int m = (L - k) % L;
            const int lane = (TEAM - t) % TEAM, reg = t == 0 ? (E - e) % E : E - 1 - e;
            if (m % TEAM != lane || m / TEAM != reg) return false;
        }
    return (L / 2) % TEAM == 0 && (L / 2) / TEAM == E / 2;
}

int main() {
    int bad = 0;
    // the shuffle unpack's lanes and registers for the row shapes that use it (team <= 32 threads)
    const int pm[][2] = {{32, 8}, {48, 12}, {64, 8}, {96, 12}, {128, 8}, {192, 12}, {256, 8}, {64, 4}, {128, 4}};
    for (const auto& c : pm)
        if (!partner_map_ok(c[0], c[1])) { std::printf("R2C partner map wrong at L=%d E=%d\n", c[0], c[1]); bad++; }
    // the exchange swizzle permutes every buffer length the kernels use (8 .. 8192 elements)
    for (int len = 8; len <= 8192; len = (len % 3 == 0) ? len * 4 / 3 : (len >= 16 ? len * 3 / 2 : len * 2)) {
        std::vector<int> seen(len, 0);
        for (int a = 0; a < len; ++a) {
            const int p = swz(a);
            if (p < 0 || p >= len || seen[p]++) { std::printf("swizzle not a permutation of [0,%d)\n", len); bad++; break; }
        }
    }
    CASE(double, 8, 8, false, 1e-14);  CASE(double, 16, 8, true, 1e-14);
    CASE(double, 32, 8, false, 1e-14); CASE(double, 64, 8, true, 1e-14);
    CASE(double, 128, 4, false, 1e-14); CASE(double, 256, 16, true, 1e-14);
    CASE(double, 512, 8, false, 1e-14); CASE(double, 1024, 8, true, 1e-14);
    CASE(double, 1024, 16, false, 1e-14); CASE(double, 2048, 8, false, 1e-14);
    CASE(float, 64, 8, false, 1e-6); CASE(float, 512, 8, true, 1e-6); CASE(float, 1024, 4, false, 1e-6);
    // lengths 3 * 2^m (the reference's 768 = 512 * 3 / 2 and its divisors), radix-3E first pass
    CASE(double, 3, 3, false, 1e-14); CASE(double, 6, 6, true, 1e-14); CASE(double, 12, 12, false, 1e-14);
    CASE(double, 24, 24, true, 1e-14); CASE(double, 48, 48, false, 1e-14); CASE(double, 48, 12, true, 1e-14);
    CASE(double, 96, 12, false, 1e-14); CASE(double, 96, 24, true, 1e-14); CASE(double, 192, 12, true, 1e-14);
    CASE(double, 384, 12, false, 1e-14); CASE(double, 384, 24, false, 1e-14); CASE(double, 768, 12, true, 1e-14);
    CASE(double, 768, 24, false, 1e-14); CASE(double, 768, 48, true, 1e-14); CASE(double, 1536, 12, false, 1e-14);
    CASE(double, 96, 6, false, 1e-14); CASE(double, 768, 6, true, 1e-14);
    CASE(float, 768, 12, false, 2e-6); CASE(float, 384, 24, true, 2e-6); CASE(float, 96, 12, false, 2e-6);
    std::printf(bad ? "FAIL\n" : "PASS\n");
    return bad ? 1 : 0;
}
