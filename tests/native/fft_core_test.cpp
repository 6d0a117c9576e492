// CPU check of the Stockham passes and small DFTs of csrc/fft_core.cuh: every
// supported length and both signs against a direct O(N^2) DFT in long double,
// with a tile of several lines in the padded column layout the kernels use.
// Emulates one CTA: all items' load halves of a pass run before any store half.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "fft_core.cuh"

using namespace pdfft;

template <int N, int R, int NS, int S, int L, int LP, int PS = 0, int AS = 0, int KL = 0, int KS = 0>
static void emu_pass(std::vector<double2>& s, const std::vector<double2>& tw) {
    constexpr int WORK = (N / R) * L;
    std::vector<double2> v((size_t)WORK * R);
    for (int w = 0; w < WORK; w++) pass_load<N, R, NS, S, L, LP, PS, AS, KL>(s.data(), tw.data(), w, &v[(size_t)w * R]);
    for (int w = 0; w < WORK; w++) pass_store<N, R, NS, L, LP, PS, AS, KS>(s.data(), w, &v[(size_t)w * R]);
}

// Passes P0..P1-1 of the plan (R0, R1, R2) on NA arrays AS apart (wpasses on the GPU).
template <int N, int S, int PS, int NA, int AS, int R0, int R1, int R2, int P0, int P1, int KL = 0, int KS = 0>
static void emu_passes(std::vector<double2>& s, const std::vector<double2>& tw) {
    constexpr int NP = R2 ? 3 : (R1 ? 2 : 1);
    if constexpr (P0 <= 0 && 0 < P1) emu_pass<N, R0, 1, S, NA, 1, PS, AS, KL, NP == 1 ? KS : 0>(s, tw);
    if constexpr (P0 <= 1 && 1 < P1 && NP > 1) emu_pass<N, R1, R0, S, NA, 1, PS, AS, 0, NP == 2 ? KS : 0>(s, tw);
    if constexpr (P0 <= 2 && 2 < P1 && NP > 2) emu_pass<N, R2, R0 * R1, S, NA, 1, PS, AS, 0, KS>(s, tw);
}

// The x pass's transform chain on one line (three arrays AS apart, band KB = N/3):
// backward transforms of band-limited arrays (first pass reading only the band),
// NL = omega x u at every point, forward transforms of (n1 + i n2) and n3 written
// only in the band; with FusedPlan::fused the third array's last backward pass,
// the product and the first forward pass run per item as the kernel runs them.
// Checked against direct long-double DFTs and the product.
template <int N, int PS>
static double check_xchain() {
    using FP = FusedPlan<N>;
    constexpr int KB = N / 3, AS = (N + (N >> PS) + 7) / 8 * 8 + 4;
    constexpr int R0 = FP::r0, R1 = FP::r1, R2 = FP::r2, NP = FP::np;
    std::vector<double2> tw(N);
    for (int e = 0; e < N; e++) {
        long double a = 6.283185307179586476925286766559005768L * e / N;
        tw[e] = mk((double)cosl(a), -(double)sinl(a));
    }
    std::vector<double2> s((size_t)3 * AS, mk(1e30, 1e30)), x((size_t)3 * N, mk(0.0, 0.0));
    srand(N * 13 + PS);
    for (int p = 0; p < 3; p++)
        for (int n = 0; n < N; n++)
            if (in_band<N, KB>(n)) {
                double2 v = mk(rand() / (double)RAND_MAX - 0.5, rand() / (double)RAND_MAX - 0.5);
                x[(size_t)p * N + n] = v;
                s[(size_t)p * AS + prow<PS>(n)] = v;
            }
    emu_passes<N, +1, PS, 2, AS, R0, R1, R2, 0, NP, KB>(s, tw);
    auto nl = [](double u1, double u2, double u3, double w1, double w2, double w3, double& n3) {
        n3 = u2 * w1 - u1 * w2;
        return mk(u3 * w2 - u2 * w3, u1 * w3 - u3 * w1);
    };
    std::vector<double2> a2(s.begin() + 2 * AS, s.begin() + 3 * AS);
    if constexpr (FP::fused) {
        constexpr int RL = FP::rl, NRL = FP::nrl;
        emu_passes<N, +1, PS, 1, 0, R0, R1, R2, 0, NP - 1, KB>(a2, tw);
        std::vector<double2> v((size_t)NRL * RL), xx((size_t)NRL * RL);
        for (int j = 0; j < NRL; j++) {
            double2* vj = &v[(size_t)j * RL];
            double2* xj = &xx[(size_t)j * RL];
            pass_load<N, RL, NRL, +1, 1, 1, PS, 0>(a2.data(), tw.data(), j, vj);
            for (int r = 0; r < RL; r++) {
                const int n = j + r * NRL;
                const double2 a = s[prow<PS>(n)], b = s[AS + prow<PS>(n)];
                double n3;
                vj[r] = nl(a.x, a.y, b.x, b.y, vj[r].x, vj[r].y, n3);
                xj[r] = mk(n3, 0.0);
            }
            dft<RL, -1>(vj);
            dft<RL, -1>(xj);
        }
        for (int j = 0; j < NRL; j++) {
            pass_store<N, RL, 1, 1, 1, PS, 0>(s.data(), j, &v[(size_t)j * RL]);
            pass_store<N, RL, 1, 1, 1, PS, 0>(s.data() + AS, j, &xx[(size_t)j * RL]);
        }
    } else {
        emu_passes<N, +1, PS, 1, 0, R0, R1, R2, 0, NP, KB>(a2, tw);
        for (int n = 0; n < N; n++) {
            const double2 a = s[prow<PS>(n)], b = s[AS + prow<PS>(n)], c = a2[prow<PS>(n)];
            double n3;
            s[prow<PS>(n)] = nl(a.x, a.y, b.x, b.y, c.x, c.y, n3);
            s[AS + prow<PS>(n)] = mk(n3, 0.0);
        }
    }
    emu_passes<N, -1, PS, 2, AS, FP::f0, FP::f1, FP::f2, FP::fused ? 1 : 0, NP, 0, KB>(s, tw);
    // direct: backward DFTs, product, forward DFTs
    std::vector<long double> ph((size_t)6 * N);
    for (int p = 0; p < 3; p++)
        for (int n = 0; n < N; n++) {
            long double re = 0, im = 0;
            for (int m = 0; m < N; m++) {
                long double ang = 6.283185307179586476925286766559005768L * (long double)((long)m * n % N) / N;
                double2 v = x[(size_t)p * N + m];
                re += v.x * cosl(ang) - v.y * sinl(ang);
                im += v.x * sinl(ang) + v.y * cosl(ang);
            }
            ph[(size_t)(2 * p) * N + n] = re;
            ph[(size_t)(2 * p + 1) * N + n] = im;
        }
    double err = 0, mag = 0;
    for (int k = 0; k < N; k++) {
        if (!in_band<N, KB>(k)) continue;
        long double r0 = 0, i0 = 0, r1 = 0, i1 = 0;
        for (int n = 0; n < N; n++) {
            const long double u1 = ph[n], u2 = ph[N + n], u3 = ph[2 * N + n];
            const long double w1 = ph[3 * N + n], w2 = ph[4 * N + n], w3 = ph[5 * N + n];
            const long double n1 = u3 * w2 - u2 * w3, n2 = u1 * w3 - u3 * w1, n3 = u2 * w1 - u1 * w2;
            long double ang = -6.283185307179586476925286766559005768L * (long double)((long)k * n % N) / N;
            const long double c = cosl(ang), sn = sinl(ang);
            r0 += n1 * c - n2 * sn; i0 += n1 * sn + n2 * c;
            r1 += n3 * c; i1 += n3 * sn;
        }
        const double2 g0 = s[prow<PS>(k)], g1 = s[AS + prow<PS>(k)];
        err = fmax(err, fabs((double)(g0.x - r0)) + fabs((double)(g0.y - i0)));
        err = fmax(err, fabs((double)(g1.x - r1)) + fabs((double)(g1.y - i1)));
        mag = fmax(mag, fabs((double)r0) + fabs((double)i0));
    }
    return err / mag;
}

// Two lines in separate arrays AS elements apart, transformed in lockstep with the
// low-pass warp plan and pad interval PS (the x-pass layout).
template <int N, int S, int PS>
static double check_pair() {
    constexpr int AS = (N + (N >> PS) + 7) / 8 * 8 + 4;
    constexpr int R0 = WPlanL<N>::r0, R1 = WPlanL<N>::r1, R2 = WPlanL<N>::r2;
    std::vector<double2> tw(N);
    for (int e = 0; e < N; e++) {
        long double a = 6.283185307179586476925286766559005768L * e / N;
        tw[e] = mk((double)cosl(a), -(double)sinl(a));
    }
    std::vector<double2> s((size_t)2 * AS), x((size_t)2 * N);
    srand(N * 11 + S + 5);
    for (int l = 0; l < 2; l++)
        for (int n = 0; n < N; n++) {
            double2 v = mk(rand() / (double)RAND_MAX - 0.5, rand() / (double)RAND_MAX - 0.5);
            x[(size_t)l * N + n] = v;
            s[(size_t)l * AS + prow<PS>(n)] = v;
        }
    emu_pass<N, R0, 1, S, 2, 1, PS, AS>(s, tw);
    if constexpr (R1 != 0) emu_pass<N, R1, R0, S, 2, 1, PS, AS>(s, tw);
    if constexpr (R2 != 0) emu_pass<N, R2, R0 * R1, S, 2, 1, PS, AS>(s, tw);
    double err = 0, mag = 0;
    for (int l = 0; l < 2; l++)
        for (int k = 0; k < N; k++) {
            long double re = 0, im = 0;
            for (int n = 0; n < N; n++) {
                long double a = S * 6.283185307179586476925286766559005768L * (long double)((long)k * n % N) / N;
                double2 v = x[(size_t)l * N + n];
                re += v.x * cosl(a) - v.y * sinl(a);
                im += v.x * sinl(a) + v.y * cosl(a);
            }
            double2 g = s[(size_t)l * AS + prow<PS>(k)];
            err = fmax(err, fabs((double)(g.x - re)) + fabs((double)(g.y - im)));
            mag = fmax(mag, fabs((double)re) + fabs((double)im));
        }
    return err / mag;
}

template <int N, int S, int L, int LP, bool WARP, bool LOWPASS = false, bool DIRECT = false>
static double check() {
    static_assert(plan_ok<N>(), "plan");
    std::vector<double2> tw(N);
    for (int e = 0; e < N; e++) {
        long double a = 6.283185307179586476925286766559005768L * e / N;
        tw[e] = mk((double)cosl(a), -(double)sinl(a));
    }
    std::vector<double2> s((size_t)N * LP), x((size_t)N * L);
    srand(N * 7 + S + 3);
    for (int l = 0; l < L; l++)
        for (int n = 0; n < N; n++) {
            double2 v = mk(rand() / (double)RAND_MAX - 0.5, rand() / (double)RAND_MAX - 0.5);
            x[(size_t)l * N + n] = v;
            s[(size_t)n * LP + l] = v;
        }
    if constexpr (WARP) {
        // warp plan, one line per warp: every line is column l of the tile (offset l, L = 1)
        constexpr int R0 = LOWPASS ? WPlanL<N>::r0 : WPlan<N>::r0;
        constexpr int R1 = LOWPASS ? WPlanL<N>::r1 : WPlan<N>::r1;
        constexpr int R2 = LOWPASS ? WPlanL<N>::r2 : WPlan<N>::r2;
        // padded rows (PS = 3) as the kernels use them
        for (int l = 0; l < L; l++) {
            std::vector<double2> col((size_t)tile_rows<N, 3>() * LP);
            for (int n = 0; n < N; n++) col[(size_t)prow<3>(n) * LP] = s[(size_t)n * LP + l];
            emu_pass<N, R0, 1, S, 1, LP, 3>(col, tw);
            if constexpr (R1 != 0) emu_pass<N, R1, R0, S, 1, LP, 3>(col, tw);
            if constexpr (R2 != 0) emu_pass<N, R2, R0 * R1, S, 1, LP, 3>(col, tw);
            for (int n = 0; n < N; n++) s[(size_t)n * LP + l] = col[(size_t)prow<3>(n) * LP];
        }
    } else if constexpr (DIRECT) {
        // direct tile transform: first pass from x, last pass into the tile s, lines
        // interleaved in a scratch tile of pitch L (one CTA emulated pass by pass)
        constexpr int R0 = Plan<N>::r0, R1 = Plan<N>::r1, R2 = Plan<N>::r2;
        std::vector<double2> t((size_t)N * L);
        auto ld = [&](int n, int l) { return x[(size_t)l * N + n]; };
        auto st = [&](int n, int l, double2 v) { s[(size_t)n * LP + l] = v; };
        if constexpr (R1 == 0) {
            for (int l = 0; l < L; l++) pass_only<N, S, L>(l, ld, st);
        } else {
            for (int w = 0; w < (N / R0) * L; w++) pass_first<N, R0, S, L>(t.data(), w, ld);
            if constexpr (R2 != 0) emu_pass<N, R1, R0, S, L, L>(t, tw);
            constexpr int RL = R2 ? R2 : R1;
            for (int w = 0; w < (N / RL) * L; w++) pass_last<N, RL, S, L>(t.data(), tw.data(), w, st);
        }
    } else {
        constexpr int R0 = Plan<N>::r0, R1 = Plan<N>::r1, R2 = Plan<N>::r2;
        emu_pass<N, R0, 1, S, L, LP>(s, tw);
        if constexpr (R1 != 0) emu_pass<N, R1, R0, S, L, LP>(s, tw);
        if constexpr (R2 != 0) emu_pass<N, R2, R0 * R1, S, L, LP>(s, tw);
    }
    double err = 0, mag = 0;
    for (int l = 0; l < L; l++)
        for (int k = 0; k < N; k++) {
            long double re = 0, im = 0;
            for (int n = 0; n < N; n++) {
                long double a = S * 6.283185307179586476925286766559005768L * (long double)((long)k * n % N) / N;
                long double c = cosl(a), sn = sinl(a);
                double2 v = x[(size_t)l * N + n];
                re += v.x * c - v.y * sn;
                im += v.x * sn + v.y * c;
            }
            double2 g = s[(size_t)k * LP + l];
            err = fmax(err, fabs((double)(g.x - re)) + fabs((double)(g.y - im)));
            mag = fmax(mag, fabs((double)re) + fabs((double)im));
        }
    return err / mag;
}

#define RUN(N)                                                                   \
    do {                                                                         \
        double e1 = check<N, -1, 8, 9, false>(), e2 = check<N, +1, 3, 5, false>(); \
        printf("N=%4d fwd %.2e bwd %.2e\n", N, e1, e2);                          \
        if (!(e1 < 1e-14 && e2 < 1e-14)) bad++;                                  \
    } while (0)
#define RUNW(N)                                                                  \
    do {                                                                         \
        double e1 = check<N, -1, 2, 3, true>(), e2 = check<N, +1, 2, 3, true>(); \
        printf("warp N=%4d fwd %.2e bwd %.2e\n", N, e1, e2);                     \
        if (!(e1 < 1e-14 && e2 < 1e-14)) bad++;                                  \
    } while (0)

int main() {
    int bad = 0;
    RUN(16); RUN(24); RUN(32); RUN(40); RUN(48); RUN(56); RUN(64); RUN(80); RUN(96);
    RUN(112); RUN(128); RUN(160); RUN(192); RUN(224); RUN(256); RUN(320); RUN(384);
    RUN(448); RUN(512); RUN(640); RUN(768); RUN(896); RUN(1024);
    RUNW(16); RUNW(24); RUNW(32); RUNW(40); RUNW(48); RUNW(56); RUNW(64); RUNW(80); RUNW(96); RUNW(112);
    RUNW(128); RUNW(160); RUNW(192); RUNW(224); RUNW(256); RUNW(320); RUNW(384); RUNW(448); RUNW(512);
    RUNW(640); RUNW(768); RUNW(896); RUNW(1024);
#define RUNL(N)                                                                             \
    do {                                                                                    \
        double e1 = check<N, -1, 2, 3, true, true>(), e2 = check<N, +1, 2, 3, true, true>();   \
        printf("warp low-pass N=%4d fwd %.2e bwd %.2e\n", N, e1, e2);                       \
        if (!(e1 < 1e-14 && e2 < 1e-14)) bad++;                                             \
    } while (0)
    RUNL(48); RUNL(128); RUNL(256); RUNL(512); RUNL(1024);
#define RUND(N)                                                                                      \
    do {                                                                                             \
        double e1 = check<N, -1, 8, 9, false, false, true>(), e2 = check<N, +1, 8, 9, false, false, true>(); \
        printf("direct tile N=%4d fwd %.2e bwd %.2e\n", N, e1, e2);                                 \
        if (!(e1 < 1e-14 && e2 < 1e-14)) bad++;                                                      \
    } while (0)
    RUND(16); RUND(24); RUND(32); RUND(40); RUND(48); RUND(56); RUND(64); RUND(80); RUND(96); RUND(112);
    RUND(128); RUND(160); RUND(192); RUND(224); RUND(256); RUND(320); RUND(384); RUND(448); RUND(512);
    RUND(640); RUND(768); RUND(896); RUND(1024);
#define RUNP(N, PS)                                                          \
    do {                                                                     \
        double e1 = check_pair<N, -1, PS>(), e2 = check_pair<N, +1, PS>();   \
        printf("pair N=%4d PS=%d fwd %.2e bwd %.2e\n", N, PS, e1, e2);      \
        if (!(e1 < 1e-14 && e2 < 1e-14)) bad++;                              \
    } while (0)
    RUNP(16, 2); RUNP(24, 3); RUNP(32, 2); RUNP(48, 2); RUNP(64, 3); RUNP(96, 3); RUNP(128, 4);
    RUNP(192, 4); RUNP(256, 4); RUNP(512, 5);
#define RUNX(N, PS)                                                              \
    do {                                                                         \
        double e = check_xchain<N, PS>();                                        \
        printf("x chain N=%4d PS=%d fused=%d err %.2e\n", N, PS, (int)FusedPlan<N>::fused, e); \
        if (!(e < 1e-13)) bad++;                                                 \
    } while (0)
    RUNX(16, 2); RUNX(24, 3); RUNX(32, 2); RUNX(48, 2); RUNX(64, 3); RUNX(96, 3); RUNX(128, 4);
    RUNX(192, 4); RUNX(256, 4); RUNX(384, 5); RUNX(512, 5); RUNX(768, 4); RUNX(1024, 5);
    RUNX(40, 4); RUNX(56, 4); RUNX(80, 4); RUNX(112, 4); RUNX(160, 4); RUNX(224, 4); RUNX(320, 4);
    RUNX(448, 4); RUNX(640, 4); RUNX(896, 4);
    printf(bad ? "FAIL\n" : "OK\n");
    return bad ? 1 : 0;
}
