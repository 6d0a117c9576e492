// fft_core.cuh -- building blocks of the batched line FFTs of the RK3 step (FP64
// and FP32).
//
// The reference runs FFTW 1-D plans (src/pf_fftw.f90:199-291): c2c along z and y,
// c2r/r2c along x, FFTW_BACKWARD (e^{+2 pi i kn/N}) unnormalised for
// spectral->physical and FFTW_FORWARD (e^{-2 pi i kn/N}) for physical->spectral.
// Here the same transforms are radix-R Stockham autosort passes (the formulation
// of Govindaraju et al., "High performance discrete Fourier transforms on
// graphics processors", SC 2008) over a tile of L lines held in shared memory
// in column layout: element n of line l sits at s[n*LP + l] (LP >= L, odd pad
// so that the transposing global<->shared copies are bank-conflict free).
// Each pass: load R points of stride N/R, twiddle by W_{Ns R}^{r k}, R-point DFT
// in registers, store at (j/Ns)*Ns*R + j%Ns + r*Ns.
//
// Everything here is __host__ __device__ so that the index arithmetic and the
// small DFTs are exercised on the CPU by the unit test harness (fft_core_test.cpp)
// before they run on a GPU.
#pragma once

#if defined(__CUDACC__)
#include <cuda_runtime.h>
#define PD_HD __host__ __device__ __forceinline__
#else
#include <cstddef>
struct double2 { double x, y; };
struct float2 { float x, y; };
#define PD_HD inline
#endif

namespace pdfft {

// Complex values are double2 (the FP64 form) or float2 (the FP32-mixed form);
// every helper below is generic over the two, the real type following the
// arguments.  Constants are written in FP64 and rounded once to the real type.
template <class T> struct cplx;
template <> struct cplx<double> { using type = double2; };
template <> struct cplx<float> { using type = float2; };
template <class C> using real_of = decltype(C{}.x);

PD_HD double2 mk(double x, double y) { double2 r; r.x = x; r.y = y; return r; }
PD_HD float2 mk(float x, float y) { float2 r; r.x = x; r.y = y; return r; }
// On sm_100 the FP32 form issues its complex arithmetic as packed two-lane FP32
// instructions (__fadd2_rn, __fmul2_rn, __ffma2_rn: per component the same
// rounding as the scalar operation), which halves the instruction count of the
// butterflies.  PD_F32X2 is the device pass for such a target.
#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ >= 1000)
#define PD_F32X2 1
#else
#define PD_F32X2 0
#endif
template <class A, class B> struct same_type { static constexpr bool value = false; };
template <class A> struct same_type<A, A> { static constexpr bool value = true; };
template <class C> constexpr bool packed_f32() { return PD_F32X2 && same_type<C, float2>::value; }

template <class C> PD_HD C add(C a, C b) {
#if PD_F32X2
    if constexpr (packed_f32<C>()) return __fadd2_rn(a, b);
    else
#endif
    return mk(a.x + b.x, a.y + b.y);
}
template <class C> PD_HD C sub(C a, C b) {
#if PD_F32X2
    if constexpr (packed_f32<C>()) return __fadd2_rn(a, mk(-b.x, -b.y));
    else
#endif
    return mk(a.x - b.x, a.y - b.y);
}
template <class C> PD_HD C scl(C a, double s) {
    const real_of<C> t = (real_of<C>)s;
#if PD_F32X2
    if constexpr (packed_f32<C>()) return __fmul2_rn(a, mk(t, t));
    else
#endif
    return mk(a.x * t, a.y * t);
}
// a * b = (a.x, a.x) * b + (a.y, a.y) * (-b.y, b.x)
template <class C> PD_HD C cmul(C a, C b) {
#if PD_F32X2
    if constexpr (packed_f32<C>()) return __ffma2_rn(mk(a.x, a.x), b, __fmul2_rn(mk(a.y, a.y), mk(-b.y, b.x)));
    else
#endif
    return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b) = a * (b.x, b.x) + (a.y, -a.x) * (b.y, b.y)
template <class C> PD_HD C cmulc(C a, C b) {
#if PD_F32X2
    if constexpr (packed_f32<C>()) return __ffma2_rn(a, mk(b.x, b.x), __fmul2_rn(mk(a.y, -a.x), mk(b.y, b.y)));
    else
#endif
    return mk(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

// Sign convention: a DFT of sign S computes X_r = sum_q x_q exp(S * 2 pi i q r / R);
// S = -1 is FFTW_FORWARD, S = +1 is FFTW_BACKWARD.  Twiddle tables hold
// tw[e] = exp(-2 pi i e / N); a sign-S pass multiplies by tw (S=-1) or conj(tw).
template <int S, class C> PD_HD C twmul(C a, C w) { return S < 0 ? cmul(a, w) : cmulc(a, w); }
// a * (S i)
template <int S, class C> PD_HD C mul_si(C a) { return S > 0 ? mk(-a.y, a.x) : mk(a.y, -a.x); }
// a * (c + S i s)
// = a * (cc, cc) + (-a.y, a.x) * (ss, ss)
template <int S, class C> PD_HD C mul_cs(C a, double c, double s) {
    using T = real_of<C>;
    const T cc = (T)c, ss = (T)(S > 0 ? s : -s);
#if PD_F32X2
    if constexpr (packed_f32<C>()) return __ffma2_rn(a, mk(cc, cc), __fmul2_rn(mk(-a.y, a.x), mk(ss, ss)));
    else
#endif
    return mk(a.x * cc - a.y * ss, a.x * ss + a.y * cc);
}

constexpr double kSqrtHalf = 0.7071067811865475244008444;
constexpr double kSin60 = 0.8660254037844386467637232;

template <int S, class C> PD_HD void dft2(C* v) {
    C a = v[0], b = v[1];
    v[0] = add(a, b); v[1] = sub(a, b);
}
template <int S, class C> PD_HD void dft3(C* v) {
    C t = add(v[1], v[2]), d = sub(v[1], v[2]);
    C m = sub(v[0], scl(t, 0.5));
    C e = mul_si<S>(scl(d, kSin60));
    v[0] = add(v[0], t);
    v[1] = add(m, e);
    v[2] = sub(m, e);
}
template <int S, class C> PD_HD void dft4(C* v) {
    C a0 = add(v[0], v[2]), a1 = sub(v[0], v[2]);
    C b0 = add(v[1], v[3]), b1 = mul_si<S>(sub(v[1], v[3]));
    v[0] = add(a0, b0); v[2] = sub(a0, b0);
    v[1] = add(a1, b1); v[3] = sub(a1, b1);
}
template <int S, class C> PD_HD void dft8(C* v) {
    C e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
    dft4<S>(e); dft4<S>(o);
    o[1] = mul_cs<S>(o[1], kSqrtHalf, kSqrtHalf);
    o[2] = mul_si<S>(o[2]);
    o[3] = mul_cs<S>(o[3], -kSqrtHalf, kSqrtHalf);
#pragma unroll
    for (int r = 0; r < 4; r++) { v[r] = add(e[r], o[r]); v[r + 4] = sub(e[r], o[r]); }
}
template <int S, class C> PD_HD void dft16(C* v) {
    C e[8], o[8];
#pragma unroll
    for (int q = 0; q < 8; q++) { e[q] = v[2 * q]; o[q] = v[2 * q + 1]; }
    dft8<S>(e); dft8<S>(o);
    constexpr double c1 = 0.9238795325112867561281832, s1 = 0.38268343236508977172846;
    o[1] = mul_cs<S>(o[1], c1, s1);
    o[2] = mul_cs<S>(o[2], kSqrtHalf, kSqrtHalf);
    o[3] = mul_cs<S>(o[3], s1, c1);
    o[4] = mul_si<S>(o[4]);
    o[5] = mul_cs<S>(o[5], -s1, c1);
    o[6] = mul_cs<S>(o[6], -kSqrtHalf, kSqrtHalf);
    o[7] = mul_cs<S>(o[7], -c1, s1);
#pragma unroll
    for (int r = 0; r < 8; r++) { v[r] = add(e[r], o[r]); v[r + 8] = sub(e[r], o[r]); }
}
// 32 = 2 x 16: radix-2 decimation in time over two length-16 DFTs, twiddles
// W32^(S r) = cos(pi r / 16) + S i sin(pi r / 16) for r = 1..15.
template <int S, class C> PD_HD void dft32(C* v) {
    C e[16], o[16];
#pragma unroll
    for (int q = 0; q < 16; q++) { e[q] = v[2 * q]; o[q] = v[2 * q + 1]; }
    dft16<S>(e); dft16<S>(o);
    constexpr double c1 = 0.9807852804032304491261822, s1 = 0.1950903220161282678482849;
    constexpr double c2 = 0.9238795325112867561281832, s2 = 0.38268343236508977172846;
    constexpr double c3 = 0.8314696123025452370787884, s3 = 0.5555702330196022247428308;
    o[1] = mul_cs<S>(o[1], c1, s1);
    o[2] = mul_cs<S>(o[2], c2, s2);
    o[3] = mul_cs<S>(o[3], c3, s3);
    o[4] = mul_cs<S>(o[4], kSqrtHalf, kSqrtHalf);
    o[5] = mul_cs<S>(o[5], s3, c3);
    o[6] = mul_cs<S>(o[6], s2, c2);
    o[7] = mul_cs<S>(o[7], s1, c1);
    o[8] = mul_si<S>(o[8]);
    o[9] = mul_cs<S>(o[9], -s1, c1);
    o[10] = mul_cs<S>(o[10], -s2, c2);
    o[11] = mul_cs<S>(o[11], -s3, c3);
    o[12] = mul_cs<S>(o[12], -kSqrtHalf, kSqrtHalf);
    o[13] = mul_cs<S>(o[13], -c3, s3);
    o[14] = mul_cs<S>(o[14], -c2, s2);
    o[15] = mul_cs<S>(o[15], -c1, s1);
#pragma unroll
    for (int r = 0; r < 16; r++) { v[r] = add(e[r], o[r]); v[r + 16] = sub(e[r], o[r]); }
}
// 12 = 3 x 4 (Cooley-Tukey): n = 4 n1 + n2, k = k1 + 3 k2.  Length-3 DFTs over n1
// for each n2, twiddles W12^(S n2 k1) (multiples of 30 degrees), length-4 DFTs over
// n2 for each k1.
template <int S, class C> PD_HD void dft12(C* v) {
    C y[4][3];
#pragma unroll
    for (int n2 = 0; n2 < 4; n2++) {
        y[n2][0] = v[n2]; y[n2][1] = v[4 + n2]; y[n2][2] = v[8 + n2];
        dft3<S>(y[n2]);
    }
    // W12^m = cos(30 m deg) + S i sin(30 m deg) for m = n2 k1 in 1..6
    y[1][1] = mul_cs<S>(y[1][1], kSin60, 0.5);            // m = 1
    y[1][2] = mul_cs<S>(y[1][2], 0.5, kSin60);            // m = 2
    y[2][1] = mul_cs<S>(y[2][1], 0.5, kSin60);            // m = 2
    y[2][2] = mul_cs<S>(y[2][2], -0.5, kSin60);           // m = 4
    y[3][1] = mul_si<S>(y[3][1]);                          // m = 3
    y[3][2] = mk(-y[3][2].x, -y[3][2].y);                  // m = 6
#pragma unroll
    for (int k1 = 0; k1 < 3; k1++) {
        C z[4] = {y[0][k1], y[1][k1], y[2][k1], y[3][k1]};
        dft4<S>(z);
#pragma unroll
        for (int k2 = 0; k2 < 4; k2++) v[k1 + 3 * k2] = z[k2];
    }
}
// odd prime R (5, 7): X_r = v0 + sum_{q=1}^{(R-1)/2} [C(qr)(v_q + v_{R-q}) + S i S(qr)(v_q - v_{R-q})]
template <int R> struct PrimeTab;
template <> struct PrimeTab<5> {
    static PD_HD double c(int m) {
        return m == 0 ? 1.0 : (m == 1 || m == 4) ? 0.3090169943749474241022934 : -0.8090169943749474241022934;
    }
    static PD_HD double s(int m) {
        return m == 0 ? 0.0 : m == 1 ? 0.9510565162951535721164393 : m == 2 ? 0.587785252292473129168706
             : m == 3 ? -0.587785252292473129168706 : -0.9510565162951535721164393;
    }
};
template <> struct PrimeTab<7> {
    static PD_HD double c(int m) {
        return m == 0 ? 1.0 : (m == 1 || m == 6) ? 0.6234898018587335305250049
             : (m == 2 || m == 5) ? -0.2225209339563144042889026 : -0.9009688679024191262361023;
    }
    static PD_HD double s(int m) {
        return m == 0 ? 0.0 : m == 1 ? 0.7818314824680298087084445 : m == 2 ? 0.9749279121818236070181317
             : m == 3 ? 0.4338837391175581204757683 : m == 4 ? -0.4338837391175581204757683
             : m == 5 ? -0.9749279121818236070181317 : -0.7818314824680298087084445;
    }
};
template <int R, int S, class C> PD_HD void dft_prime(C* v) {
    C sum[(R - 1) / 2], dif[(R - 1) / 2];
#pragma unroll
    for (int q = 1; q <= (R - 1) / 2; q++) { sum[q - 1] = add(v[q], v[R - q]); dif[q - 1] = sub(v[q], v[R - q]); }
    C out[R];
    C x0 = v[0];
#pragma unroll
    for (int r = 0; r < R; r++) {
        C acc = x0;
#pragma unroll
        for (int q = 1; q <= (R - 1) / 2; q++) {
            const int m = (q * r) % R;
            acc = add(acc, scl(sum[q - 1], PrimeTab<R>::c(m)));
            acc = add(acc, mul_si<S>(scl(dif[q - 1], PrimeTab<R>::s(m))));
        }
        out[r] = acc;
    }
#pragma unroll
    for (int r = 0; r < R; r++) v[r] = out[r];
}

template <int R, int S, class C> PD_HD void dft(C* v) {
    if constexpr (R == 2) dft2<S>(v);
    else if constexpr (R == 3) dft3<S>(v);
    else if constexpr (R == 4) dft4<S>(v);
    else if constexpr (R == 8) dft8<S>(v);
    else if constexpr (R == 16) dft16<S>(v);
    else if constexpr (R == 12) dft12<S>(v);
    else if constexpr (R == 32) dft32<S>(v);
    else if constexpr (R == 5 || R == 7) dft_prime<R, S>(v);
    else static_assert(R == 2, "unsupported radix");
}

// Radix schedule per transform length.  Supported N: 2^a * {1,3,5,7} from 16 to 1024,
// factored into the radices below (2, 3, 4, 5, 7, 8, 12, 16; 32 in warp plans) in at most three passes;
// lengths with a factor 3 take a radix-12 pass where that saves a pass.
template <int N> struct Plan { static constexpr int r0 = 0, r1 = 0, r2 = 0; };
#define PD_PLAN(N_, A, B, C) \
    template <> struct Plan<N_> { static constexpr int r0 = A, r1 = B, r2 = C; };
PD_PLAN(16, 16, 0, 0)
PD_PLAN(24, 3, 8, 0)
PD_PLAN(32, 8, 4, 0)
PD_PLAN(40, 5, 8, 0)
PD_PLAN(48, 3, 16, 0)
PD_PLAN(56, 7, 8, 0)
PD_PLAN(64, 8, 8, 0)
PD_PLAN(80, 5, 16, 0)
PD_PLAN(96, 8, 12, 0)
PD_PLAN(112, 7, 16, 0)
PD_PLAN(128, 8, 16, 0)
PD_PLAN(160, 5, 4, 8)
PD_PLAN(192, 16, 12, 0)
PD_PLAN(224, 7, 4, 8)
PD_PLAN(256, 16, 16, 0)
PD_PLAN(320, 5, 8, 8)
PD_PLAN(384, 3, 8, 16)
PD_PLAN(448, 7, 8, 8)
PD_PLAN(512, 8, 8, 8)
PD_PLAN(640, 5, 8, 16)
PD_PLAN(768, 3, 16, 16)
PD_PLAN(896, 7, 8, 16)
PD_PLAN(1024, 16, 8, 8)
#undef PD_PLAN

template <int N> constexpr bool plan_ok() {
    return Plan<N>::r0 * (Plan<N>::r1 ? Plan<N>::r1 : 1) * (Plan<N>::r2 ? Plan<N>::r2 : 1) == N;
}

// Row of element n in a tile: with PS > 0 one pad row follows every 2^PS rows,
// which spreads the stride-R stores of the first passes over distinct banks
// when a warp owns a single line.
template <int PS> PD_HD int prow(int n) { return PS > 0 ? n + (n >> PS) : n; }
template <int N, int PS> constexpr int tile_rows() { return PS > 0 ? N + (N >> PS) : N; }

// One pass, split into a load/compute half and a store half so that a CPU
// emulator can run all items' first halves before any second half (that is
// what the __syncthreads() between them does on the GPU).
// Element n of line l: interleaved columns (AS = 0, s[prow(n)*LP + l]) or separate
// arrays AS elements apart (s[l*AS + prow(n)]).
template <int LP, int PS, int AS> PD_HD int tidx(int n, int l) {
    return AS ? l * AS + prow<PS>(n) : prow<PS>(n) * LP + l;
}

// Twiddles w[r] = tw[r e] (r = 1..R-1) of one butterfly: the entries at power-of-two
// multiples r = 2^a are read from the table (log2 R loads), the others are products
// w[2^a] w[r - 2^a] of those (at most log2(R) - 1 roundings on a correctly rounded
// entry).  The kernels are bound by load instructions and shared/L1 wavefronts, so
// the table reads are what is saved; the FP arithmetic has room.
template <int R, class C> PD_HD void twiddles(const C* tw, int e, C* w) {
#pragma unroll
    for (int r = 1; r < R; r++) {
        if ((r & (r - 1)) == 0) {
            w[r] = tw[r * e];
        } else {
            int hb = 1;
            while (hb * 2 <= r) hb *= 2;
            w[r] = cmul(w[hb], w[r - hb]);
        }
    }
}

// The band of a 2/3-truncated spectrum on a length-N line: n <= KB or n >= N - KB
// (KB = 0: the whole line).  A pass_load with KB > 0 reads the elements outside
// the band as zero without touching shared memory (first pass of a transform of a
// truncated spectrum); a pass_store with KB > 0 writes only the band (last pass of
// a transform whose outputs outside it are discarded).
template <int N, int KB> PD_HD bool in_band(int n) { return KB == 0 || n <= KB || n >= N - KB; }

template <int N, int R, int NS, int S, int L, int LP, int PS = 0, int AS = 0, int KB = 0, class C>
PD_HD void pass_load(const C* s, const C* tw, int w, C* v) {
    using T = real_of<C>;
    constexpr int NR = N / R;
    const int l = w % L, j = w / L;
#pragma unroll
    for (int r = 0; r < R; r++) {
        if constexpr (KB > 0) v[r] = in_band<N, KB>(j + r * NR) ? s[tidx<LP, PS, AS>(j + r * NR, l)] : mk(T(0), T(0));
        else v[r] = s[tidx<LP, PS, AS>(j + r * NR, l)];
    }
    if constexpr (NS > 1) {
        const int k = j % NS;
        constexpr int step = N / (NS * R);
        C wt[R];
        twiddles<R>(tw, k * step, wt);
#pragma unroll
        for (int r = 1; r < R; r++) v[r] = twmul<S>(v[r], wt[r]);
    }
    dft<R, S>(v);
}
template <int N, int R, int NS, int L, int LP, int PS = 0, int AS = 0, int KB = 0, class C>
PD_HD void pass_store(C* s, int w, const C* v) {
    const int l = w % L, j = w / L;
    const int k = j % NS;
    const int d = (j / NS) * NS * R + k;
#pragma unroll
    for (int r = 0; r < R; r++)
        if (in_band<N, KB>(d + r * NS)) s[tidx<LP, PS, AS>(d + r * NS, l)] = v[r];
}

// Transforms whose first pass reads global memory and whose last pass writes it
// ("direct" tile transforms).  The L lines of a tile are interleaved in shared
// memory, element n of line l at s[n*L + l] with L = 8: the 8 threads of a
// quarter-warp always own the 8 lines of one butterfly, so every shared access of
// every pass is one contiguous 128-byte row (no bank conflicts, no pad rows), and
// the same 8 threads touch 8 lines x 16 bytes of global memory per element.
// The first pass takes element n of line l from ld(n, l); the last pass hands
// output n of line l to st(n, l, value).  A two-pass length costs one shared-memory
// round trip per element instead of four.
template <int N, int R, int S, int L, class C, class Ld>
PD_HD void pass_first(C* s, int w, Ld& ld) {
    constexpr int NR = N / R;
    const int l = w % L, j = w / L;
    C v[R];
#pragma unroll
    for (int r = 0; r < R; r++) v[r] = ld(j + r * NR, l);
    dft<R, S>(v);
#pragma unroll
    for (int r = 0; r < R; r++) s[(j * R + r) * L + l] = v[r];
}
template <int N, int R, int S, int L, class C, class St>
PD_HD void pass_last(const C* s, const C* tw, int w, St& st) {
    constexpr int NS = N / R;
    C v[R];
    pass_load<N, R, NS, S, L, L, 0>(s, tw, w, v);
    const int l = w % L, j = w / L;
#pragma unroll
    for (int r = 0; r < R; r++) st(j + r * NS, l, v[r]);
}
// Single-pass lengths: global to global, no shared memory.
template <int N, int S, int L, class Ld, class St>
PD_HD void pass_only(int l, Ld& ld, St& st) {
    using C = decltype(ld(0, 0));
    C v[N];
#pragma unroll
    for (int r = 0; r < N; r++) v[r] = ld(r, l);
    dft<N, S>(v);
#pragma unroll
    for (int r = 0; r < N; r++) st(r, l, v[r]);
}

// Threads per CTA of a direct tile transform of L = 8 lines: one item per thread
// in the widest pass, at most 512.
// Threads of a tile transform of 8 lines with the radix plan (R0, R1, R2): one
// butterfly per thread in the pass with the most, 64..512.
template <int N, int R0, int R1, int R2> constexpr int tile_threads_for() {
    constexpr int a = N / R0;
    constexpr int b = R1 ? N / R1 : 0;
    constexpr int c = R2 ? N / R2 : 0;
    constexpr int m = 8 * (a > b ? (a > c ? a : c) : (b > c ? b : c));
    return m < 64 ? 64 : (m > 512 ? 512 : m);
}
template <int N> constexpr int tile_threads() { return tile_threads_for<N, Plan<N>::r0, Plan<N>::r1, Plan<N>::r2>(); }

// Radix schedule of the warp-level transforms (one line per warp): radix 8 where
// possible so that a pass has N/8 items, about one per lane.
template <int N> struct WPlan { static constexpr int r0 = 0, r1 = 0, r2 = 0; };
#define PD_WPLAN(N_, A, B, C) \
    template <> struct WPlan<N_> { static constexpr int r0 = A, r1 = B, r2 = C; };
PD_WPLAN(16, 4, 4, 0)
PD_WPLAN(24, 3, 8, 0)
PD_WPLAN(32, 4, 8, 0)
PD_WPLAN(40, 5, 8, 0)
PD_WPLAN(48, 4, 12, 0)
PD_WPLAN(56, 7, 8, 0)
PD_WPLAN(64, 8, 8, 0)
PD_WPLAN(80, 5, 16, 0)
PD_WPLAN(96, 8, 12, 0)
PD_WPLAN(112, 7, 16, 0)
PD_WPLAN(128, 4, 4, 8)
PD_WPLAN(160, 5, 4, 8)
PD_WPLAN(192, 16, 12, 0)
PD_WPLAN(224, 7, 4, 8)
PD_WPLAN(256, 4, 8, 8)
PD_WPLAN(320, 5, 8, 8)
PD_WPLAN(384, 3, 8, 16)
PD_WPLAN(448, 7, 8, 8)
PD_WPLAN(512, 8, 8, 8)
PD_WPLAN(640, 5, 8, 16)
PD_WPLAN(768, 3, 16, 16)
PD_WPLAN(896, 7, 8, 16)
PD_WPLAN(1024, 16, 8, 8)
#undef PD_WPLAN

template <int N> constexpr bool wplan_ok() {
    return WPlan<N>::r0 * (WPlan<N>::r1 ? WPlan<N>::r1 : 1) * (WPlan<N>::r2 ? WPlan<N>::r2 : 1) == N;
}

// Fewer, larger passes (radix 16) for kernels limited by shared-memory bandwidth
// rather than by registers: each pass costs a full read and write of the line.
template <int N> struct WPlanL : WPlan<N> {};
template <> struct WPlanL<128> { static constexpr int r0 = 16, r1 = 8, r2 = 0; };
template <> struct WPlanL<256> { static constexpr int r0 = 16, r1 = 16, r2 = 0; };
template <> struct WPlanL<384> { static constexpr int r0 = 32, r1 = 12, r2 = 0; };
template <> struct WPlanL<512> { static constexpr int r0 = 32, r1 = 16, r2 = 0; };
template <> struct WPlanL<1024> { static constexpr int r0 = 32, r1 = 32, r2 = 0; };

// Plan of a backward transform, a pointwise product and a forward transform run
// by one warp (the x pass): backward (r0, r1[, r2]) = WPlanL; with `fused` the
// forward transform runs the reversed plan, so that the last backward pass and
// the first forward pass see the same elements n = j + r * (N / rl) in item j, and
// the last backward pass of one array, the product and the first forward pass run
// in registers, one item per lane (nrl = N / rl items, 16..32 of them).  Lines
// shorter than 256 keep separate passes and the same plan both ways (measured
// faster at 192: the fused step leaves half the lanes idle there).
template <int N> struct FusedPlan {
    static constexpr int r0 = WPlanL<N>::r0, r1 = WPlanL<N>::r1, r2 = WPlanL<N>::r2;
    static constexpr int np = r2 ? 3 : 2;
    static constexpr int rl = r2 ? r2 : r1;
    static constexpr int nrl = N / rl;
    static constexpr bool fused = N >= 256 && nrl >= 16 && nrl <= 32;
    static constexpr int f0 = fused ? rl : r0;
    static constexpr int f1 = fused ? (r2 ? r1 : r0) : r1;
    static constexpr int f2 = fused ? (r2 ? r0 : 0) : r2;
};

template <int N> constexpr bool wplanl_ok() {
    return WPlanL<N>::r0 * (WPlanL<N>::r1 ? WPlanL<N>::r1 : 1) * (WPlanL<N>::r2 ? WPlanL<N>::r2 : 1) == N;
}

#if defined(__CUDACC__)
// One pass of a single line owned by one warp: the line is column 0 of `s`
// (element n at s[prow<PS>(n)*LP]); only __syncwarp() separates the halves.
template <int N, int R, int NS, int S, int LP, int PS, class C>
__device__ __forceinline__ void wpass(C* s, const C* __restrict__ tw, int lane) {
    constexpr int WORK = N / R;
    constexpr int IT = (WORK + 31) / 32;
    C v[IT][R];
#pragma unroll
    for (int it = 0; it < IT; it++) {
        const int w = lane + it * 32;
        if (WORK % 32 == 0 || w < WORK) pass_load<N, R, NS, S, 1, LP, PS>(s, tw, w, v[it]);
    }
    __syncwarp();
#pragma unroll
    for (int it = 0; it < IT; it++) {
        const int w = lane + it * 32;
        if (WORK % 32 == 0 || w < WORK) pass_store<N, R, NS, 1, LP, PS>(s, w, v[it]);
    }
    __syncwarp();
}

// NA lines transformed in lockstep by one warp (interleaved columns 0..NA-1 for
// AS = 0, else separate arrays AS elements apart): each pass has NA times the
// independent work of a single line, which fills the lanes a radix-16 pass of
// one line leaves idle.
// KL / KS: band of the loads / stores (see in_band).
// W: lanes per line group (32: the whole warp; 32 / W groups of a warp each transform
// their own lines, `lane` being the lane within the group).
template <int N, int R, int NS, int S, int LP, int PS, int NA, int AS = 0, int KL = 0, int KS = 0, int W = 32, class C>
__device__ __forceinline__ void wpass_n(C* s, const C* __restrict__ tw, int lane) {
    constexpr int WORK = (N / R) * NA;
    constexpr int IT = (WORK + W - 1) / W;
    C v[IT][R];
#pragma unroll
    for (int it = 0; it < IT; it++) {
        const int w = lane + it * W;
        if (WORK % W == 0 || w < WORK) pass_load<N, R, NS, S, NA, LP, PS, AS, KL>(s, tw, w, v[it]);
    }
    __syncwarp();
#pragma unroll
    for (int it = 0; it < IT; it++) {
        const int w = lane + it * W;
        if (WORK % W == 0 || w < WORK) pass_store<N, R, NS, NA, LP, PS, AS, KS>(s, w, v[it]);
    }
    __syncwarp();
}

// Passes P0..P1-1 of the radix plan (R0, R1, R2) over NA arrays owned by one
// warp: pass p has radix Rp and NS = the product of the radices before it.  The
// plan's first pass reads the band KL, its last pass writes the band KS.
template <int N, int S, int LP, int PS, int NA, int AS, int R0, int R1, int R2, int P0, int P1,
          int KL = 0, int KS = 0, int W = 32, class C>
__device__ __forceinline__ void wpasses(C* s, const C* __restrict__ tw, int lane) {
    constexpr int NP = R2 ? 3 : (R1 ? 2 : 1);
    if constexpr (P0 <= 0 && 0 < P1) wpass_n<N, R0, 1, S, LP, PS, NA, AS, KL, NP == 1 ? KS : 0, W>(s, tw, lane);
    if constexpr (P0 <= 1 && 1 < P1 && NP > 1) wpass_n<N, R1, R0, S, LP, PS, NA, AS, 0, NP == 2 ? KS : 0, W>(s, tw, lane);
    if constexpr (P0 <= 2 && 2 < P1 && NP > 2) wpass_n<N, R2, R0 * R1, S, LP, PS, NA, AS, 0, KS, W>(s, tw, lane);
}

template <int N, int S, int LP, int PS, int NA, bool LOWPASS = false, int AS = 0, class C>
__device__ __forceinline__ void fft_warp_n(C* s, const C* __restrict__ tw, int lane) {
    static_assert(wplan_ok<N>() && wplanl_ok<N>(), "no warp radix plan for this length");
    constexpr int R0 = LOWPASS ? WPlanL<N>::r0 : WPlan<N>::r0;
    constexpr int R1 = LOWPASS ? WPlanL<N>::r1 : WPlan<N>::r1;
    constexpr int R2 = LOWPASS ? WPlanL<N>::r2 : WPlan<N>::r2;
    wpass_n<N, R0, 1, S, LP, PS, NA, AS>(s, tw, lane);
    if constexpr (R1 != 0) wpass_n<N, R1, R0, S, LP, PS, NA, AS>(s, tw, lane);
    if constexpr (R2 != 0) wpass_n<N, R2, R0 * R1, S, LP, PS, NA, AS>(s, tw, lane);
}

// Full length-N transform of the line at column 0 of `s` by the calling warp
// (the caller makes the line's data visible to the warp before the call).
template <int N, int S, int LP, int PS, bool LOWPASS = false, class C>
__device__ __forceinline__ void fft_warp(C* s, const C* __restrict__ tw, int lane) {
    static_assert(wplan_ok<N>() && wplanl_ok<N>(), "no warp radix plan for this length");
    constexpr int R0 = LOWPASS ? WPlanL<N>::r0 : WPlan<N>::r0;
    constexpr int R1 = LOWPASS ? WPlanL<N>::r1 : WPlan<N>::r1;
    constexpr int R2 = LOWPASS ? WPlanL<N>::r2 : WPlan<N>::r2;
    wpass<N, R0, 1, S, LP, PS>(s, tw, lane);
    if constexpr (R1 != 0) wpass<N, R1, R0, S, LP, PS>(s, tw, lane);
    if constexpr (R2 != 0) wpass<N, R2, R0 * R1, S, LP, PS>(s, tw, lane);
}

// In-place pass over a [N][LP] shared tile with NT threads; items w = tid + it*NT.
template <int N, int R, int NS, int S, int L, int LP, int NT, class C>
__device__ __forceinline__ void pass(C* s, const C* __restrict__ tw, int tid) {
    constexpr int WORK = (N / R) * L;
    constexpr int IT = (WORK + NT - 1) / NT;
    C v[IT][R];
#pragma unroll
    for (int it = 0; it < IT; it++) {
        const int w = tid + it * NT;
        if (WORK % NT == 0 || w < WORK) pass_load<N, R, NS, S, L, LP>(s, tw, w, v[it]);
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < IT; it++) {
        const int w = tid + it * NT;
        if (WORK % NT == 0 || w < WORK) pass_store<N, R, NS, L, LP>(s, w, v[it]);
    }
    __syncthreads();
}

// Direct tile transform of L interleaved lines by NT threads (see pass_first) with
// the radix plan (R0, R1, R2), by default Plan<N>.  The caller makes `s` free
// before the call (a barrier after any earlier use); on return other threads may
// still read `s`.  `mid()` runs once per thread after the first pass (the loads
// of the tile are done and the remaining passes are shared-memory work).
struct NoMid {
    __device__ void operator()() const {}
};
template <int N, int S, int L, int NT, int R0 = Plan<N>::r0, int R1 = Plan<N>::r1, int R2 = Plan<N>::r2,
          class C, class Ld, class St, class Mid = NoMid>
__device__ __forceinline__ void fft_tile_io(C* s, const C* __restrict__ tw, int tid, Ld& ld, St& st,
                                            const Mid& mid = Mid()) {
    static_assert(R0 * (R1 ? R1 : 1) * (R2 ? R2 : 1) == N, "radix plan does not factor N");
    if constexpr (R1 == 0) {
        mid();
        for (int l = tid; l < L; l += NT) pass_only<N, S, L>(l, ld, st);
    } else {
        constexpr int W0 = (N / R0) * L;
#pragma unroll
        for (int w = tid; w < W0; w += NT) pass_first<N, R0, S, L>(s, w, ld);
        __syncthreads();
        mid();
        if constexpr (R2 != 0) pass<N, R1, R0, S, L, L, NT>(s, tw, tid);   // in place, ends with a barrier
        constexpr int RL = R2 ? R2 : R1;
        constexpr int WL = (N / RL) * L;
#pragma unroll
        for (int w = tid; w < WL; w += NT) pass_last<N, RL, S, L>(s, tw, w, st);
    }
}
#endif

}  // namespace pdfft
