// passes_kernels.cuh -- the five HBM passes of one RK3 stage on sm_100a: kernels and
// their configurations (templates on the transform length).  The per-length launchers
// are in passes_n.cuh, instantiated by the passes_n*.cu files (one group of lengths per
// file, so the lengths compile in parallel); kernels_passes.cu dispatches on the length.
//
// Pass structure per stage (replacing f_RK3PrepareRealSpace, f_RK3RealSpace and
// f_RK3SolveNavierStokes, src/pf_rk3.f90:205-329, 960-1237, 1996-2142, whose
// MPI/FFTW pencil transposes collapse into on-chip tile transposes):
//   K1 zpass_inv   u (3 x S)           -> omega, 6 backward z FFTs             -> zb [6][z][j][i]
//   K2 ypass_inv   zb                  -> 6 backward y FFTs                    -> yb [6][z][y][i]
//   K3 xpass       yb (6 half spectra) -> 3 complex c2r (two real lines each), omega x u,
//                                         2 complex r2c, truncate             -> yb fields 0..2
//   K4 ypass_fwd   yb fields 0..2      -> 3 forward y FFTs, truncate j       -> zb fields 0..2
//   K5 zpass_fwd   zb fields 0..2      -> 3 forward z FFTs, x 1/(NX NY NZ), truncate k, then the
//                                         per-mode RHS + low-storage RK3 + continuity fix on u, rk
// Every pass reads and writes HBM once.  The z and y passes (K1, K2, K4, K5a)
// are tile transforms of 8 lines interleaved in shared memory (pdfft::fft_tile_io):
// the first radix pass loads its butterfly inputs straight from HBM (rows of 8
// consecutive i = 128 bytes) and the last pass stores straight to HBM, so a
// two-pass length crosses shared memory once, behind one block barrier.  The x
// pass owns whole lines per warp and needs no block barrier at all.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <type_traits>
#include "fft_core.cuh"
#include "pandora_internal.cuh"
#include "bfrot.cuh"

namespace pd {

using pdfft::mk;
using pdfft::prow;
using pdfft::tile_rows;

// Shared memory of every kernel here, viewed as the kernel's complex type.
extern __shared__ __align__(16) unsigned char pd_smem[];
template <class C> __device__ __forceinline__ C* smem_as() { return reinterpret_cast<C*>(pd_smem); }


// K3 holds three complex arrays per warp, so long lines get fewer warps per CTA.
template <int N> struct Cfg {
    static constexpr int NWX = (N <= 512) ? 8 : 4;
    // K3 CTAs per SM: shared memory allows 2 FP64 CTAs up to N = 256, FP32 twice that
    template <class T> static constexpr int minbx() {
        return sizeof(T) == 8 ? ((N <= 256) ? 2 : 1) : ((N <= 256) ? 3 : (N <= 512 ? 2 : 1));
    }
};

// Transform lengths built: 2^a x {1, 3, 5, 7} from 16 to 1024 (the reference's rule,
// src/pg_domain.f90:274-292), each a radix plan of at most three passes.
#define PD_FOR_EACH_N(X) \
    X(16) X(24) X(32) X(40) X(48) X(56) X(64) X(80) X(96) X(112) X(128) X(160) X(192) X(224) X(256) \
    X(320) X(384) X(448) X(512) X(640) X(768) X(896) X(1024)


// ---------------------------------------------------------------------------
// K3: x pass, one warp per (z,y) line, no block barrier.  The six half spectra
// of the line become three complex backward FFTs (pairs (u1,u2), (u3,w1),
// (w2,w3): the c2r of two real lines at once; the Hermitian extension drops Im
// of the i=0 mode as FFTW's c2r does, src/pf_fftw.f90:646,749-756), then
// NL = omega x u (f_RK3ComputeNonlinearIsotropic, src/pf_rk3.f90:1597-1628),
// then two complex forward FFTs ((n1,n2), (n3,0)) split into the r2c outputs,
// truncated to i = 0..KI (src/pf_fftw.f90:780).  NL overwrites yb fields 0..2 of
// the same line.  Optionally writes the physical velocity (arr_u*_3r,
// src/pf_rk3.f90:1108-1115) and the CFL maximum (src/pf_fluidstats.f90:913-917).
// Warp shared region: three arrays XAS elements apart (XAS = 4 mod 8 in 16-byte
// units), element n of array p at s[p*XAS + prow<XPS>(n)].  Up to N = 512 the
// warp transforms arrays 0 and 1 in lockstep (a radix-16 or radix-32 pass of one
// array leaves lanes idle); with the offset of 4 bank groups between the two
// arrays and XPS chosen per length, those passes are free of bank conflicts.
// The warp plans are two passes up to N = 1024 (radix 32 at 512 and 1024): the
// kernel is bound by shared-memory wavefronts, and each pass is a full read and
// write of the three arrays.
// ---------------------------------------------------------------------------
// Bulk prefetch of [p, p + bytes) into L2 (a hint: no data moves to the SM),
// trimmed inward to the 16-byte boundaries the bulk copy requires.
__device__ __forceinline__ void prefetch_l2(const void* p, size_t bytes) {
    unsigned long long a = (unsigned long long)p, e = a + bytes;
    a = (a + 15) & ~15ull;
    e &= ~15ull;
    if (e > a) asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"((unsigned)(e - a)) : "memory");
}

template <int N> constexpr int xps() {
    return (N == 16 || N == 32 || N == 48) ? 2
         : ((N == 24 || N == 64 || N == 96) ? 3 : ((N == 384 || N == 512 || N == 1024) ? 5 : 4));
}
template <int N> constexpr int xas() { return (tile_rows<N, xps<N>()>() + 7) / 8 * 8 + 4; }
// arrays transformed in lockstep: 2 while a lane's items of a pass fit its registers
template <int N> constexpr int xna() { return N <= 512 ? 2 : 1; }

// NL = omega x u at one point (isotropic or BF-rot); returns (n1, n2) and n3.
template <class T, class C>
__device__ __forceinline__ C nl_point(const BFT<T>& bf, bool shear, T u1, T u2, T u3, T w1, T w2, T w3, T& n3) {
    if (shear) {   // f_RK3ComputeNonlinearBFRot, in the fields' real type
        const T uu[3] = {u1, u2, u3}, om[3] = {w1, w2, w3};
        T nl[3];
        nl_bf(bf, uu, om, nl);
        n3 = nl[2];
        return mk(nl[0], nl[1]);
    }
    n3 = u2 * w1 - u1 * w2;
    return mk(u3 * w2 - u2 * w3, u1 * w3 - u3 * w1);
}

// Real-space statistics of f_FluidstatsRs2D (src/pf_fluidstats.f90:827-958) at one
// point: velocity moments in the laboratory frame (u_lab = binv u for shear), vorticity
// moments, maxima.  acc: [0..5] u1u1 u2u2 u3u3 u1u2 u1u3 u2u3, [6..8] u^3, [9..11] u^4,
// [12..14] w^2, [15..17] w^3, [18..20] w^4; mx: [0] max |u1|+|u2|+|u3|, [1..3] max |w|.
constexpr int kRsSums = 21, kRsMax = 4, kRsSlots = 32, kRsWords = 32;
__device__ __forceinline__ void rs_point(double* acc, double* mx, bool shear, const BF& f, double u1, double u2,
                                         double u3, double w1, double w2, double w3) {
    if (shear) {
        const double um[3] = {u1, u2, u3};
        double ul[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int m = 0; m < 3; m++)
#pragma unroll
            for (int n = 0; n < 3; n++)
                if (bex(m, n)) ul[m] += f.bi[m][n] * um[n];
        u1 = ul[0]; u2 = ul[1]; u3 = ul[2];
    }
    acc[0] += u1 * u1; acc[1] += u2 * u2; acc[2] += u3 * u3;
    acc[3] += u1 * u2; acc[4] += u1 * u3; acc[5] += u2 * u3;
    acc[6] += u1 * u1 * u1; acc[7] += u2 * u2 * u2; acc[8] += u3 * u3 * u3;
    acc[9] += (u1 * u1) * (u1 * u1); acc[10] += (u2 * u2) * (u2 * u2); acc[11] += (u3 * u3) * (u3 * u3);
    acc[12] += w1 * w1; acc[13] += w2 * w2; acc[14] += w3 * w3;
    acc[15] += w1 * w1 * w1; acc[16] += w2 * w2 * w2; acc[17] += w3 * w3 * w3;
    acc[18] += (w1 * w1) * (w1 * w1); acc[19] += (w2 * w2) * (w2 * w2); acc[20] += (w3 * w3) * (w3 * w3);
    mx[0] = fmax(mx[0], fabs(u1) + fabs(u2) + fabs(u3));
    mx[1] = fmax(mx[1], fabs(w1)); mx[2] = fmax(mx[2], fabs(w2)); mx[3] = fmax(mx[3], fabs(w3));
}

// RS: the real-space statistics pass (the same transforms, plus the moments of every
// point, reduced per warp into one of kRsSlots copies of the sums in `rs`).
// LPW: lines per warp (LPW > 1 for short, unfused lines: each group of 32 / LPW lanes
// transforms its own line).
template <int NX, class T, int CAP, bool RS = false, int LPW = 1>
__global__ void __launch_bounds__(32 * Cfg<NX>::NWX, Cfg<NX>::template minbx<T>()) k_xpass(const __grid_constant__ MemberSet<T, CAP> ms,
                                                                                        int want_phys,
                                                                                        int want_cfl,
                                                                                        long long pf_lines,
                                                                                        double* rs) {
    using C = typename FieldsT<T>::C;
    using XP = pdfft::FusedPlan<NX>;
    const Member<T>& mm = ms.m[CAP == 1 ? 0 : blockIdx.y];
    if (!mm.active) return;
    if constexpr (CAP > 1) {   // a batch slot between members
        if (mm.F.clock->status & PD_ST_IDLE) return;
    }
    const FieldsT<T> F = mm.F;
    const Geo g = mm.g;
    constexpr int XPS = xps<NX>(), XAS = xas<NX>(), NA = xna<NX>();
    constexpr int KB = NX / 3;   // the kept band of the x spectrum, i <= KI
    static_assert(LPW == 1 || (!XP::fused && !RS), "several lines per warp: unfused plans, no statistics");
    constexpr int W = 32 / LPW;  // lanes per line
    C* smem = smem_as<C>();
    const int tid = threadIdx.x, lane = (tid & 31) % W, sub = (tid & 31) / W, w = tid >> 5;
    const long long lines = (long long)g.ny * g.nz;
    const C* tw = F.tw_x;
    const long long qw = ((long long)blockIdx.x * Cfg<NX>::NWX + w) * LPW;   // the warp's first line
    if (qw >= lines) return;                      // whole warp; no block barrier follows
    // a group past the last line transforms the last line again and stores nothing
    const bool valid = qw + sub < lines;
    const long long q = valid ? qw + sub : lines - 1;
    C* s = smem + ((size_t)w * LPW + sub) * 3 * XAS;
    constexpr int NKI = NX / 3 + 1, NKIP = (NKI + 7) / 8 * 8;   // g.nki, g.nkip
    const long long fstride = lines * NKIP;       // distance between fields in yb
    C* b = F.yb + q * NKIP;
    BFT<T> bf;
    if (g.shear) bf = bf_as<T>(make_bf(g, F.clock));
    double racc[RS ? kRsSums : 1], rmax[RS ? kRsMax : 1];
    BF brs;
    if constexpr (RS) {
#pragma unroll
        for (int a = 0; a < kRsSums; a++) racc[a] = 0.0;
#pragma unroll
        for (int a = 0; a < kRsMax; a++) rmax[a] = 0.0;
        brs = make_bf(g, F.clock);
    }
    // the band of each array; the first backward pass reads nothing outside it.
    // From 384 points on (registers to spare at one or two CTAs per SM) the loads
    // of up to IB rounds of m are issued before any of their stores, so a line waits
    // on HBM about twice rather than once per round.
    {
        constexpr int ITM = (NX / 3 + 1 + W - 1) / W;     // rounds of m (NKI = NX/3 + 1)
        constexpr int IB = NX >= 384 ? (ITM + 1) / 2 : 1;
#pragma unroll
        for (int i0 = 0; i0 < ITM; i0 += IB) {
            C X[IB][6];
#pragma unroll
            for (int it = 0; it < IB; it++) {
                const int m = lane + W * (i0 + it);
                if (i0 + it < ITM && m < NKI) {
#pragma unroll
                    for (int c = 0; c < 6; c++) X[it][c] = b[c * fstride + m];
                    if constexpr (RS) {
                        // R-conv: the reference's u4..u6 are d(u1,u2,u3)/dx1 (src/pf_rk3.f90:
                        // 422-428), i m times the u rows
                        if (g.rconv) {
                            const T km = (T)m;
#pragma unroll
                            for (int c = 3; c < 6; c++) X[it][c] = mk(-km * X[it][c - 3].y, km * X[it][c - 3].x);
                        }
                    }
                }
            }
#pragma unroll
            for (int it = 0; it < IB; it++) {
                const int m = lane + W * (i0 + it);
                if (i0 + it < ITM && m < NKI) {
#pragma unroll
                    for (int p = 0; p < 3; p++) {
                        C Xp = X[it][2 * p], Yp = X[it][2 * p + 1];
                        if (m == 0) { Xp.y = T(0); Yp.y = T(0); }
                        s[p * XAS + prow<XPS>(m)] = mk(Xp.x - Yp.y, Xp.y + Yp.x);
                        if (m > 0) s[p * XAS + prow<XPS>(NX - m)] = mk(Xp.x + Yp.y, -Xp.y + Yp.x);
                    }
                }
            }
        }
    }
    __syncwarp();
    constexpr int R0 = XP::r0, R1 = XP::r1, R2 = XP::r2, NP = XP::np;
    if constexpr (NA == 2) {
        pdfft::wpasses<NX, +1, 1, XPS, 2, XAS, R0, R1, R2, 0, NP, KB, 0, W>(s, tw, lane);
    } else {   // one array at a time, one copy of the code (instruction-cache footprint)
#pragma unroll 1
        for (int a = 0; a < 2; a++) pdfft::wpasses<NX, +1, 1, XPS, 1, 0, R0, R1, R2, 0, NP, KB, 0, W>(s + a * XAS, tw, lane);
    }
    T umax = T(0);
    if constexpr (XP::fused) {
        constexpr int RL = XP::rl, NRL = XP::nrl;
        pdfft::wpasses<NX, +1, 1, XPS, 1, 0, R0, R1, R2, 0, NP - 1, KB>(s + 2 * XAS, tw, lane);
        C v[RL];
        T n3[RL];
        if (lane < NRL) {
            // last backward pass of array 2: (w2, w3) at n = lane + r * NRL
            pdfft::pass_load<NX, RL, NRL, +1, 1, 1, XPS, 0>(s + 2 * XAS, tw, lane, v);
#pragma unroll
            for (int r = 0; r < RL; r++) {
                const int n = lane + r * NRL;
                const C* e = s + prow<XPS>(n);
                const C a = e[0], bb = e[XAS];
                const T u1 = a.x, u2 = a.y, u3 = bb.x, w1 = bb.y, w2 = v[r].x, w3 = v[r].y;
                if (want_phys) {
                    F.phys[q * NX + n] = u1;
                    F.phys[g.R + q * NX + n] = u2;
                    F.phys[2 * g.R + q * NX + n] = u3;
                }
                if (want_cfl) umax = fmax(umax, fabs(u1) + fabs(u2) + fabs(u3));
                if constexpr (RS) rs_point(racc, rmax, g.shear, brs, u1, u2, u3, w1, w2, w3);
                v[r] = nl_point<T, C>(bf, g.shear && !g.rrot, u1, u2, u3, w1, w2, w3, n3[r]);
            }
        }
        __syncwarp();   // every lane has read arrays 0 and 1
        if (lane < NRL) {
            // first forward pass (NS = 1) of the two product arrays, one at a time
            pdfft::dft<RL, -1>(v);
            pdfft::pass_store<NX, RL, 1, 1, 1, XPS, 0>(s, lane, v);
#pragma unroll
            for (int r = 0; r < RL; r++) v[r] = mk(n3[r], T(0));
            pdfft::dft<RL, -1>(v);
            pdfft::pass_store<NX, RL, 1, 1, 1, XPS, 0>(s + XAS, lane, v);
        }
        __syncwarp();
    } else {
        pdfft::wpasses<NX, +1, 1, XPS, 1, 0, R0, R1, R2, 0, NP, KB, 0, W>(s + 2 * XAS, tw, lane);
        for (int n = lane; n < NX; n += W) {
            C* e = s + prow<XPS>(n);
            const C a = e[0], bb = e[XAS], c = e[2 * XAS];
            const T u1 = a.x, u2 = a.y, u3 = bb.x, w1 = bb.y, w2 = c.x, w3 = c.y;
            if (want_phys && valid) {
                F.phys[q * NX + n] = u1;
                F.phys[g.R + q * NX + n] = u2;
                F.phys[2 * g.R + q * NX + n] = u3;
            }
            if (want_cfl) umax = fmax(umax, fabs(u1) + fabs(u2) + fabs(u3));
            if constexpr (RS) rs_point(racc, rmax, g.shear, brs, u1, u2, u3, w1, w2, w3);
            T n3;
            e[0] = nl_point<T, C>(bf, g.shear && !g.rrot, u1, u2, u3, w1, w2, w3, n3);
            e[XAS] = mk(n3, T(0));
        }
        __syncwarp();
    }
    if (want_cfl) {
        for (int o = 16; o > 0; o >>= 1) umax = fmax(umax, __shfl_xor_sync(0xffffffffu, umax, o));
        if ((tid & 31) == 0) atomicMax(&F.clock->ucfl_bits, (unsigned long long)__double_as_longlong((double)umax));
    }
    if constexpr (RS) {   // the warp's sums into slot q % kRsSlots
        double* slot = rs + (size_t)(q % kRsSlots) * kRsWords;
#pragma unroll
        for (int a = 0; a < kRsSums; a++) {
            double x = racc[a];
            for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
            if (lane == 0) atomicAdd(slot + a, x);
        }
#pragma unroll
        for (int a = 0; a < kRsMax; a++) {
            double x = rmax[a];
            for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_xor_sync(0xffffffffu, x, o));
            if (lane == 0)
                atomicMax(reinterpret_cast<unsigned long long*>(slot + kRsSums + a), (unsigned long long)__double_as_longlong(x));
        }
    }
    // The six input rows of line q + pf_lines (a wave of resident CTAs later, so
    // the CTA that takes it starts about when this one ends) are prefetched into
    // L2, one bulk prefetch per row, while this line's forward transforms run:
    // that CTA's loads then wait on L2 rather than HBM.
    if (pf_lines > 0 && valid && q + pf_lines < lines && lane < 6)
        prefetch_l2(F.yb + lane * fstride + (q + pf_lines) * NKIP, NKI * sizeof(C));
    // forward transforms of the product arrays; only the band is written
    constexpr int F0 = XP::f0, F1 = XP::f1, F2 = XP::f2, P0 = XP::fused ? 1 : 0;
    if constexpr (NA == 2) {
        pdfft::wpasses<NX, -1, 1, XPS, 2, XAS, F0, F1, F2, P0, NP, 0, KB, W>(s, tw, lane);
    } else {
#pragma unroll 1
        for (int a = 0; a < 2; a++) pdfft::wpasses<NX, -1, 1, XPS, 1, 0, F0, F1, F2, P0, NP, 0, KB, W>(s + a * XAS, tw, lane);
    }
    const T half = T(0.5);
    for (int m = lane; m < NKIP && valid; m += W) {
        C n1 = mk(T(0), T(0)), n2 = n1, n3 = n1;
        if (m < NKI) {
            const int mc = (NX - m) % NX;
            const C Z = s[prow<XPS>(m)], Zc = s[prow<XPS>(mc)];
            n1 = mk(half * (Z.x + Zc.x), half * (Z.y - Zc.y));
            n2 = mk(half * (Z.y + Zc.y), -half * (Z.x - Zc.x));
            const C W = s[XAS + prow<XPS>(m)], Wc = s[XAS + prow<XPS>(mc)];
            n3 = mk(half * (W.x + Wc.x), half * (W.y - Wc.y));
        }
        b[m] = n1;
        b[fstride + m] = n2;
        b[2 * fstride + m] = n3;
    }
}

// ---------------------------------------------------------------------------
// K3 of the R-conv form (NS_DEFORMED = NS_R_CONV): the x pass of the twelve fields u1..u3
// and d u_c / d x_d, from the nine rows u, d u / dy, d u / dz of yb (d u_c / dx is i m times
// the x spectrum of u_c, formed here), then f_RK3ComputeNonlinearRConv
// (src/pf_rk3.f90:1717-1774), NL_i = sum_d v_d d u_i / d x_d with v_d = sum_j
// bmat(d,j) u_j, then the forward transforms and split of K3.  One warp per line
// over four arrays: the pairs (u1,u2) and (u3, du1/dx1) first; v and the partial sums
// then stay in the arrays that the later pairs do not use, which are transformed two
// and then one at a time.  Optionally writes the physical velocity (laboratory
// components) for the particles.  Batches: the member is blockIdx.y, as in K3.
// ---------------------------------------------------------------------------
template <int N, class T> struct ConvCfg {
    static constexpr int per_warp = 4 * xas<N>() * (int)sizeof(typename Cplx<T>::type);
    static constexpr int fit = (200 * 1024) / per_warp;
    static constexpr int NW = fit >= 8 ? 8 : (fit < 1 ? 1 : fit);
    static constexpr size_t smem = (size_t)NW * per_warp;
};

template <int NX, class T, int CAP>
__global__ void __launch_bounds__(32 * ConvCfg<NX, T>::NW, 1) k_xpass_conv(const __grid_constant__ MemberSet<T, CAP> ms,
                                                                          int want_phys, int want_cfl, long long pf_lines) {
    using C = typename FieldsT<T>::C;
    using XP = pdfft::FusedPlan<NX>;   // the backward plan r0, r1, r2 (run unfused here)
    const Member<T>& mm = ms.m[CAP == 1 ? 0 : blockIdx.y];
    if (!mm.active) return;
    if constexpr (CAP > 1) {   // a batch slot between members
        if (mm.F.clock->status & PD_ST_IDLE) return;
    }
    const FieldsT<T> F = mm.F;
    const Geo g = mm.g;
    constexpr int XPS = xps<NX>(), XAS = xas<NX>(), NA = xna<NX>(), NW = ConvCfg<NX, T>::NW;
    constexpr int KB = NX / 3;
    constexpr int R0 = XP::r0, R1 = XP::r1, R2 = XP::r2, NP = XP::np;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const long long lines = (long long)g.ny * g.nz;
    const C* tw = F.tw_x;
    const long long q = (long long)blockIdx.x * NW + w;
    if (q >= lines) return;                       // whole warp; no block barrier follows
    C* s = smem_as<C>() + (size_t)w * 4 * XAS;
    constexpr int NKI = NX / 3 + 1, NKIP = (NKI + 7) / 8 * 8;   // g.nki, g.nkip
    const long long fstride = lines * NKIP;
    C* b = F.yb + q * NKIP;
    const BFT<T> bf = bf_as<T>(make_bf(g, F.clock));
    // the Hermitian extension of the half spectra of fields fa and fb into array p, as K3;
    // xa, xb: i m times the field (its x derivative)
    auto build = [&](int p, int fa, bool xa, int fb, bool xb) {
        for (int m = lane; m < NKI; m += 32) {
            C X = b[fa * fstride + m], Y = b[fb * fstride + m];
            const T km = (T)m;
            if (xa) X = mk(-km * X.y, km * X.x);
            if (xb) Y = mk(-km * Y.y, km * Y.x);
            if (m == 0) { X.y = T(0); Y.y = T(0); }
            s[p * XAS + prow<XPS>(m)] = mk(X.x - Y.y, X.y + Y.x);
            if (m > 0) s[p * XAS + prow<XPS>(NX - m)] = mk(X.x + Y.y, -X.y + Y.x);
        }
        __syncwarp();
    };
    auto bwd1 = [&](C* a) { pdfft::wpasses<NX, +1, 1, XPS, 1, 0, R0, R1, R2, 0, NP, KB>(a, tw, lane); };
    auto bwd2 = [&](C* a) {   // arrays a and a + XAS
        if constexpr (NA == 2) pdfft::wpasses<NX, +1, 1, XPS, 2, XAS, R0, R1, R2, 0, NP, KB>(a, tw, lane);
        else {
#pragma unroll 1
            for (int r = 0; r < 2; r++) bwd1(a + r * XAS);
        }
    };
    // (u1,u2), (u3, du1/dx1) -> v = bmat u, NL1 = v1 du1/dx1; arrays 0, 1 = (v1,v2), (v3,NL1)
    build(0, 0, false, 1, false);
    build(1, 2, false, 0, true);
    bwd2(s);
    T umax = T(0);
    for (int n = lane; n < NX; n += 32) {
        C* e = s + prow<XPS>(n);
        const C a = e[0], c1 = e[XAS];
        const T u[3] = {a.x, a.y, c1.x};
        if (want_phys) {
            F.phys[q * NX + n] = u[0];
            F.phys[g.R + q * NX + n] = u[1];
            F.phys[2 * g.R + q * NX + n] = u[2];
        }
        if (want_cfl) umax = fmax(umax, fabs(u[0]) + fabs(u[1]) + fabs(u[2]));
        T v[3];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            v[d] = T(0);
#pragma unroll
            for (int j = 0; j < 3; j++)
                if (bex(d, j)) v[d] += bf.bm[d][j] * u[j];
        }
        e[0] = mk(v[0], v[1]);
        e[XAS] = mk(v[2], v[0] * c1.y);
    }
    // (du2/dx1, du3/dx1), (du1/dx2, du2/dx2); arrays 0..2 = (v2,v3), (NL1,NL2), (NL3,-)
    build(2, 1, true, 2, true);
    build(3, 3, false, 4, false);
    bwd2(s + 2 * XAS);
    for (int n = lane; n < NX; n += 32) {
        C* e = s + prow<XPS>(n);
        const C a = e[0], c1 = e[XAS], g1 = e[2 * XAS], g2 = e[3 * XAS];
        const T v1 = a.x, v2 = a.y, v3 = c1.x;
        const T n1 = c1.y + v2 * g2.x;
        const T n2 = v1 * g1.x + v2 * g2.y;
        const T n3 = v1 * g1.y;
        e[0] = mk(v2, v3);
        e[XAS] = mk(n1, n2);
        e[2 * XAS] = mk(n3, T(0));
    }
    // (du3/dx2, du1/dx3)
    build(3, 5, false, 6, false);
    bwd1(s + 3 * XAS);
    for (int n = lane; n < NX; n += 32) {
        C* e = s + prow<XPS>(n);
        const C a = e[0], c1 = e[XAS], c2 = e[2 * XAS], g1 = e[3 * XAS];
        e[XAS] = mk(c1.x + a.y * g1.y, c1.y);
        e[2 * XAS] = mk(c2.x + a.x * g1.x, T(0));
    }
    // (du2/dx3, du3/dx3); arrays 0, 1 = (NL1,NL2), (NL3,0) for the forward transforms
    build(3, 7, false, 8, false);
    bwd1(s + 3 * XAS);
    for (int n = lane; n < NX; n += 32) {
        C* e = s + prow<XPS>(n);
        const C a = e[0], c1 = e[XAS], c2 = e[2 * XAS], g1 = e[3 * XAS];
        const T v3 = a.y;
        e[0] = mk(c1.x, c1.y + v3 * g1.x);
        e[XAS] = mk(c2.x + v3 * g1.y, T(0));
    }
    __syncwarp();
    if (want_cfl) {
        for (int o = 16; o > 0; o >>= 1) umax = fmax(umax, __shfl_xor_sync(0xffffffffu, umax, o));
        if (threadIdx.x % 32 == 0) atomicMax(&F.clock->ucfl_bits, (unsigned long long)__double_as_longlong((double)umax));
    }
    if (pf_lines > 0 && q + pf_lines < lines && lane < 9)
        prefetch_l2(F.yb + lane * fstride + (q + pf_lines) * NKIP, NKI * sizeof(C));
    if constexpr (NA == 2) {
        pdfft::wpasses<NX, -1, 1, XPS, 2, XAS, R0, R1, R2, 0, NP, 0, KB>(s, tw, lane);
    } else {
#pragma unroll 1
        for (int r = 0; r < 2; r++) pdfft::wpasses<NX, -1, 1, XPS, 1, 0, R0, R1, R2, 0, NP, 0, KB>(s + r * XAS, tw, lane);
    }
    const T half = T(0.5);
    for (int m = lane; m < NKIP; m += 32) {
        C n1 = mk(T(0), T(0)), n2 = n1, n3 = n1;
        if (m < NKI) {
            const int mc = (NX - m) % NX;
            const C Z = s[prow<XPS>(m)], Zc = s[prow<XPS>(mc)];
            n1 = mk(half * (Z.x + Zc.x), half * (Z.y - Zc.y));
            n2 = mk(half * (Z.y + Zc.y), -half * (Z.x - Zc.x));
            const C W = s[XAS + prow<XPS>(m)], Wc = s[XAS + prow<XPS>(mc)];
            n3 = mk(half * (W.x + Wc.x), half * (W.y - Wc.y));
        }
        b[m] = n1;
        b[fstride + m] = n2;
        b[2 * fstride + m] = n3;
    }
}

// ---------------------------------------------------------------------------
// K5: forward z transforms x normalisation, truncate k (f_RK3TransformkRs2Fs +
// f_Fftw_k_Rs2Fs, src/pf_rk3.f90:2242-2316, src/pf_fftw.f90:841-879) into NL-hat
// (K5a), then the per-mode update (K5b).  NL-hat goes to the y-pencil buffer,
// which K4 has finished with; mode 1 writes it into rk instead and stops there
// (the transform test hook of src/ptf_rk3.f90:629-734).  Splitting costs 2 x 3S
// complex words of traffic but lets both halves stream at full occupancy.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void rk_coeffs(int stage, double& beta, double& gamma) {
    if (stage == 1) { beta = 0.0; gamma = 1.0 / 3.0; }
    else if (stage == 2) { beta = -(5.0 / 9.0); gamma = 15.0 / 16.0; }
    else { beta = -(153.0 / 128.0); gamma = 8.0 / 15.0; }
}

template <class C> struct Out3 { C* p[3]; };

// K5b: per mode f_RK3FormFIsotropic / f_RK3FormFBFRot + f_RK3RungeKutta +
// f_RK3ContinuityFixIsotropic (src/pf_rk3.f90:2323-2673, 3457-3531), one thread
// per mode, streaming NL-hat, u and rk.
// Separate instantiations for the isotropic (with forcing) and the BF-rot right-hand
// side: 3 and 4 CTAs of 256 threads per SM, without spills.
// The per-mode arithmetic runs in FP64 registers in both forms (the FP32-mixed
// form loads FP32 values and rounds once on the store).
// FORM: 0 isotropic, 1 BF-rot shear, 2 R-rot shear, 3 isotropic with the integrating
// factor (its own instantiation, so the explicit forms carry no exponent code).
// The update of mode m = (i, j, k) (index in the [i][j][k] layout) from its NL-hat nl[3]:
// the body of K5b.
template <int FORM, class T>
__device__ __forceinline__ void rk_mode(const FieldsT<T>& F, const Geo& g, int stage, long long m, const double2* nl) {
    using C = typename FieldsT<T>::C;
    const int NKK = g.nkk;
    const int k = (int)(m % NKK);
    const long long ij = m / NKK;
    const int j = (int)(ij % g.nkj), i = (int)(ij / g.nkj);
    const double k1 = (double)i, k2 = wvn(j, g.kj), k3 = wvn(k, g.kk);
    const double kmag2 = (k1 * k1) + (k2 * k2) + (k3 * k3);
    if (!(kmag2 > 0.0)) return;
    const double ik2 = 1.0 / kmag2;   // the mode's one FP64 division (products below)
    double beta, gamma;
    rk_coeffs(stage, beta, gamma);
    const double dt = F.clock->dt;
    const double kv[3] = {k1, k2, k3};
    double2 uu[3], tot[3];
#pragma unroll
    for (int c = 0; c < 3; c++) uu[c] = to_d(F.u[c][m]);
    BF bf;
    if constexpr (FORM == 1) {   // f_RK3FormFBFRot, F_SHEAR_DNS (no forcing)
        bf = make_bf(g, F.clock);
        rhs_bf(bf, g.nu, kv, uu, nl, tot);
    } else if constexpr (FORM == 2) {   // f_RK3FormFRRot, F_SHEAR_DNS
        bf = make_bf(g, F.clock);
        rhs_rrot(bf, g.nu, kv, uu, nl, tot);
    } else {
        const double2 kdn = mk(k1 * nl[0].x + k2 * nl[1].x + k3 * nl[2].x,
                               k1 * nl[0].y + k2 * nl[1].y + k3 * nl[2].y);
        double2 force[3] = {mk(0.0, 0.0), mk(0.0, 0.0), mk(0.0, 0.0)};
        const double kmag = sqrt(kmag2);
        if (kmag <= g.force_kf && kmag > 0.0) {
            const int NK = g.fnk, FW = 2 * NK + 1;
            const int jw = (int)k2, kw = (int)k3;
            if (i <= NK && jw >= -NK && jw <= NK && kw >= -NK && kw <= NK) {
                double2 fv[3];
                const long long fi = ((long long)i * FW + (jw + NK)) * FW + (kw + NK);
                const long long fst = (long long)(NK + 1) * FW * FW;
#pragma unroll
                for (int c = 0; c < 3; c++) fv[c] = F.forcing[c * fst + fi];
                const double2 kdb = mk(k1 * fv[0].x + k2 * fv[1].x + k3 * fv[2].x,
                                       k1 * fv[0].y + k2 * fv[1].y + k3 * fv[2].y);
#pragma unroll
                for (int c = 0; c < 3; c++)
                    force[c] = mk(fv[c].x - ((kv[c] * ik2) * kdb.x), fv[c].y - ((kv[c] * ik2) * kdb.y));
            }
        }
        if constexpr (FORM == 3) {   // integrating factor: the viscous term leaves the right-hand side
#pragma unroll
            for (int c = 0; c < 3; c++)
                tot[c] = mk(-nl[c].x + (kv[c] * ik2) * kdn.x + force[c].x,
                            -nl[c].y + (kv[c] * ik2) * kdn.y + force[c].y);
        } else {
#pragma unroll
            for (int c = 0; c < 3; c++)
                tot[c] = mk(-g.nu * kmag2 * uu[c].x - nl[c].x + (kv[c] * ik2) * kdn.x + force[c].x,
                            -g.nu * kmag2 * uu[c].y - nl[c].y + (kv[c] * ik2) * kdn.y + force[c].y);
        }
    }
    // Integrating factor (isotropic flow): E = exp(-nu k^2 (c_{s+1} - c_s) dt), c = 0, 1/3,
    // 3/4, 1, scales the register and u of the stage (FP64 exponent in both precisions)
    constexpr bool vif = FORM == 3;
    double ex = 1.0;
    if constexpr (vif) ex = exp(-(g.nu * kmag2 * (stage == 1 ? 1.0 / 3.0 : (stage == 2 ? 5.0 / 12.0 : 0.25)) * dt));
#pragma unroll
    for (int c = 0; c < 3; c++) {
        double2 r;
        if (stage == 1) r = tot[c];   // beta = 0; registers start at zero (src/pf_arrays.f90:805-832)
        else {
            const double2 r0 = to_d(F.rk[c][m]);
            r = mk((beta * r0.x) + tot[c].x, (beta * r0.y) + tot[c].y);
        }
        if constexpr (vif) {
            r = mk(ex * r.x, ex * r.y);
            uu[c] = mk(ex * uu[c].x, ex * uu[c].y);
        }
        F.rk[c][m] = from_d<C>(r);
        uu[c] = mk(uu[c].x + (gamma * dt * r.x), uu[c].y + (gamma * dt * r.y));
    }
    if constexpr (FORM == 2) {   // f_RK3ContinuityFixRRot
        contfix_rrot(bf, kv, kmag2, uu);
#pragma unroll
        for (int c = 0; c < 3; c++) F.u[c][m] = from_d<C>(uu[c]);
        return;
    }
    const double2 kdu = mk(k1 * uu[0].x + k2 * uu[1].x + k3 * uu[2].x, k1 * uu[0].y + k2 * uu[1].y + k3 * uu[2].y);
#pragma unroll
    for (int c = 0; c < 3; c++)
        F.u[c][m] = from_d<C>(mk(uu[c].x - (kv[c] * kdu.x * ik2), uu[c].y - (kv[c] * kdu.y * ik2)));
}

template <int FORM, class T, int CAP>
__global__ void __launch_bounds__(256, FORM == 1 ? 4 : 3) k_rk_update(const __grid_constant__ MemberSet<T, CAP> ms, int stage) {
    using C = typename FieldsT<T>::C;
    const Member<T>& mm = ms.m[CAP == 1 ? 0 : blockIdx.y];
    if (!mm.active) return;
    if constexpr (CAP > 1) {   // a batch slot between members
        if (mm.F.clock->status & PD_ST_IDLE) return;
    }
    const FieldsT<T> F = mm.F;
    const Geo g = mm.g;
    const C* __restrict__ nlh = F.yb;   // NL-hat from K5a
    const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= g.S) return;
    double2 nl[3];
#pragma unroll
    for (int c = 0; c < 3; c++) nl[c] = to_d(nlh[c * g.S + m]);
    rk_mode<FORM, T>(F, g, stage, m, nl);
}

// ---------------------------------------------------------------------------
// z and y passes: direct-I/O tile transforms (pdfft::fft_tile_io), one field
// per CTA, TCfg::lines interleaved lines, the first radix pass reading its butterfly
// inputs straight from HBM and the last pass writing its outputs straight to
// HBM, so a 256-point line crosses shared memory once (one block barrier).
// ---------------------------------------------------------------------------
template <int N, bool TWO = false> struct TCfg {
    // Radix plan: Plan<N>, or with TWO (the y passes and K5a) for FP32 512-point
    // lines the two-pass (32, 16): one shared-memory round trip instead of two.  An
    // FP64 item of radix 32 does not fit the registers of two CTAs per SM, and K1
    // (vorticity loads in its first pass) measured slower with it.
    template <class T> static constexpr bool two() { return TWO && sizeof(T) == 4 && N == 512; }
    template <class T> static constexpr int r0() { return two<T>() ? 32 : pdfft::Plan<N>::r0; }
    template <class T> static constexpr int r1() { return two<T>() ? 16 : pdfft::Plan<N>::r1; }
    template <class T> static constexpr int r2() { return two<T>() ? 0 : pdfft::Plan<N>::r2; }
    // threads per CTA: one butterfly per thread in the widest pass of a tile of 8 lines
    template <class T> static constexpr int nt() { return pdfft::tile_threads_for<N, r0<T>(), r1<T>(), r2<T>()>(); }
    // Lines per tile: 8 (FP64: one 128-byte row of complex values, so the quarter
    // warp of a shared-memory wavefront owns the lines of one butterfly and every
    // access of a pass is whole rows).  FP32 tiles of 512-point lines take 16 lines,
    // again a 128-byte row per half-warp wavefront (with 8 the stores of a pass have
    // two-way bank conflicts and global rows are 64 bytes); elsewhere the doubled
    // tile costs occupancy (1024) or a half-empty last tile (nkip = 88 at 256) and
    // measured slower.
    template <class T> static constexpr int lines() { return (sizeof(T) == 4 && N == 512) ? 16 : 8; }
    // resident CTAs per SM asked of the register allocator: an FP32 tile of 16 lines
    // holds the registers and shared memory of an FP64 one, of 8 lines half of them
    template <class T> static constexpr int minb() {
        constexpr int NT = nt<T>();
        return (sizeof(T) == 8 || lines<T>() == 16) ? (NT <= 128 ? (N == 192 ? 4 : 5) : (NT <= 256 ? 2 : (N == 512 ? 2 : 1)))
                                                    : (NT <= 128 ? (N == 192 ? 6 : 8) : (NT <= 256 ? 4 : 2));
    }
    template <class T> static constexpr size_t smem() { return sizeof(typename Cplx<T>::type) * (size_t)N * lines<T>(); }
    // tiles along i; with 16 lines the last one may be partial (nkip is a multiple
    // of 8), and its loads and stores stop at nkip
    template <class T> static unsigned tiles(const Geo& g) {
        return (unsigned)((g.nkip + lines<T>() - 1) / lines<T>());
    }
    template <int S, int L, class C, class Ld, class St, class Mid = pdfft::NoMid>
    static __device__ __forceinline__ void transform(C* s, const C* tw, Ld& ld, St& st, const Mid& mid = Mid()) {
        using T = pdfft::real_of<C>;
        pdfft::fft_tile_io<N, S, L, nt<T>(), r0<T>(), r1<T>(), r2<T>()>(s, tw, threadIdx.x, ld, st, mid);
    }
};

// K1: spectral velocity and vorticity, backward z transforms.  Field f =
// blockIdx.x: 0..2 velocity, 3..5 vorticity omega = i k x u, isotropic branch of
// f_RK3PrepareVelocity (src/pf_rk3.f90:402-407,520-525,630-634, derivative
// f_RK3Derivative 3735-3743), or the BF-rot or R-rot vorticity, or (R-conv) the z
// derivatives i k3 u_c; the tile's lines from i0 at one j;
// k is zero-padded into [KK+1, NZ-KK-1] as src/pf_rk3.f90:437-443.  The six CTAs
// of a tile are adjacent in launch order, so the three that read a velocity
// component run together and two of the three reads hit L2.  FORM (compile time, so
// that each instantiation carries only its own derivative code): 0 isotropic, 1 BF-rot,
// 2 R-rot, 3 R-conv.  The batched shear forms at 256 points in FP64 ask for one CTA per SM
// fewer than the others: the member index and frame tensors spilled at five.
template <int NZ, int FORM, class T, int CAP, int CN = 0>
__global__ void __launch_bounds__(TCfg<NZ>::template nt<T>(),
                                  TCfg<NZ>::template minb<T>() - ((CAP > 1 && FORM != 0 && sizeof(T) == 8 && NZ == 256) ? 1 : 0))
    k_zpass_inv(const __grid_constant__ MemberSet<T, CAP> ms, int stage,
                                                                                                   long long pf_ctas) {
    using C = typename FieldsT<T>::C;
    constexpr bool SHEAR = FORM != 0;
    constexpr int nf = FORM == 3 ? 9 : 6;
    const Member<T>& mm = ms.m[CAP == 1 ? 0 : blockIdx.x / nf];
    if (!mm.active) return;
    if constexpr (CAP > 1) {   // a batch slot between members
        if (mm.F.clock->status & PD_ST_IDLE) return;
    }
    const FieldsT<T> F = mm.F;
    const Geo g = mm.g;
    // CN > 0: a cubic grid of CN points a side, every size a compile-time constant
    const int nkj_ = CN ? 2 * (CN / 3) + 1 : g.nkj, kj_ = CN ? CN / 3 : g.kj;
    const int nki_ = CN ? CN / 3 + 1 : g.nki, nkip_ = CN ? (CN / 3 + 1 + 7) / 8 * 8 : g.nkip;
    C* s = smem_as<C>();
    constexpr int LT = TCfg<NZ>::template lines<T>();
    const int f = blockIdx.x % nf, i0 = blockIdx.y * LT, j = blockIdx.z;
    const int lmax = nkip_ - i0;   // lines of this tile inside the i padding
    if (stage == 1 && f == 0 && blockIdx.y == 0 && j == 0 && threadIdx.x == 0) F.clock->ucfl_bits = 0ull;
    constexpr int KK = NZ / 3, NKK = 2 * KK + 1;   // g.kk, g.nkk (the 2/3 rule)
    const int nki = nki_;
    const double k2 = wvn(j, kj_);
    const T k2t = (T)k2;
    const long long istride = (long long)nkj_ * NKK;
    const long long row0 = ((long long)i0 * nkj_ + j) * NKK;
    // velocity: u_f; vorticity omega_{f-3} = i (ka a - kb b): omega1 = i (k2 u3 - k3 u2),
    // omega2 = i (k3 u1 - k1 u3), omega3 = i (k1 u2 - k2 u1).  R-conv: fields 3 + c and
    // 6 + c are d u_c / dy and d u_c / dz (d u_c / dx is formed in the x pass).
    // (selects, not an index into F.u: a computed index would move F to local memory)
    constexpr bool rconv = FORM == 3;
    const int fc = rconv ? f % 3 : -1;
    const C* const pa = rconv ? (fc == 0 ? F.u[0] : (fc == 1 ? F.u[1] : F.u[2]))
                              : ((f == 0 || f == 4) ? F.u[0] : ((f == 1 || f == 5) ? F.u[1] : F.u[2]));
    const C* pb = (f == 3) ? F.u[1] : ((f == 4) ? F.u[2] : F.u[0]);
    BFT<T> bf;
    if constexpr (SHEAR) {
        if (f >= 3) bf = bf_as<T>(make_bf(g, F.clock));
    }
    auto ld = [&](int z, int l) -> C {
        const int i = i0 + l;
        int k;
        if (z <= KK) k = z;
        else if (z >= NZ - KK) k = z - NZ + NKK;
        else return mk(T(0), T(0));
        if (i >= nki) return mk(T(0), T(0));
        const long long m = row0 + l * istride + k;
        if (f < 3) return pa[m];
        if constexpr (FORM == 3) {   // f_RK3Derivative (src/pf_rk3.f90:3735-3743): i k2 u_c or i k3 u_c
            const T kd = f < 6 ? k2t : (T)wvn(k, KK);
            const C uc = pa[m];
            return mk(-kd * uc.y, kd * uc.x);
        } else if constexpr (SHEAR) {
            // BF-rot vorticity (f_RK3VorticityBFRot) or the R-rot sheared curl, in T
            const T kv[3] = {(T)i, k2t, (T)wvn(k, KK)};
            const C zero = mk(T(0), T(0));
            // omega1 has no term in u1 and omega2 none in u2: those loads are skipped
            const C uv[3] = {f != 3 ? F.u[0][m] : zero, f != 4 ? F.u[1][m] : zero, F.u[2][m]};
            C w3[3];
            // only the CTA's own component (f is uniform over the CTA)
            if constexpr (FORM == 2) {
                if (f == 3) vort_rrot<0>(bf, uv, kv, w3);
                else if (f == 4) vort_rrot<1>(bf, uv, kv, w3);
                else vort_rrot<2>(bf, uv, kv, w3);
            } else {
                if (f == 3) vort_bf<0>(bf, uv, kv, w3);
                else if (f == 4) vort_bf<1>(bf, uv, kv, w3);
                else vort_bf<2>(bf, uv, kv, w3);
            }
            return f == 3 ? w3[0] : (f == 4 ? w3[1] : w3[2]);
        } else {
            const T k1 = (T)i, k3 = (T)wvn(k, KK);
            const T ka = (f == 3) ? k2t : ((f == 4) ? k3 : k1);
            const T kb = (f == 3) ? k3 : ((f == 4) ? k1 : k2t);
            const C a = pa[m], b = pb[m];
            return mk((-ka * a.y) - (-kb * b.y), (ka * a.x) - (kb * b.x));
        }
    };
    C* dst = F.zb + (((long long)f * NZ) * nkj_ + j) * nkip_ + i0;
    const long long zs = (long long)nkj_ * nkip_;
    auto st = [&](int z, int l, C v) {
        if (LT > 8 && l >= lmax) return;
        dst[z * zs + l] = v;
    };
    // After the first pass: prefetch into L2 the velocity rows of the CTA a wave of
    // resident CTAs later (single simulations: blocks (f, tile, j) in launch order),
    // so that its loads wait on L2 rather than HBM.  A vorticity CTA's rows are all
    // three components, an R-conv gradient CTA's one.
    const C* const u0 = F.u[0];
    const C* const u1 = F.u[1];
    const C* const u2 = F.u[2];
    const int nkj = nkj_;
    auto mid = [pf_ctas, nki, nkj, NKK, u0, u1, u2]() {
        if (pf_ctas <= 0) return;
        const long long nblk = (long long)nf * gridDim.y * gridDim.z;
        const long long nxt = blockIdx.x + (long long)nf * (blockIdx.y + (long long)gridDim.y * blockIdx.z) + pf_ctas;
        if (nxt >= nblk) return;
        const int f2 = (int)(nxt % nf), ti = (int)((nxt / nf) % gridDim.y), j2 = (int)(nxt / ((long long)nf * gridDim.y));
        const int nc = (f2 < 3 || rconv) ? 1 : 3, t = threadIdx.x;
        if (t >= LT * nc) return;
        const int c = f2 < 3 ? f2 : (rconv ? f2 % 3 : t / LT), i = ti * LT + t % LT;
        const C* uc = c == 0 ? u0 : (c == 1 ? u1 : u2);
        if (i < nki) prefetch_l2(uc + ((long long)i * nkj + j2) * NKK, NKK * sizeof(C));
    };
    TCfg<NZ>::template transform<+1, LT>(s, F.tw_z, ld, st, mid);
}

// ---------------------------------------------------------------------------
// K1 with the velocity rows staged by the tensor-memory accelerator (FP64, single
// simulations, z lines of ZStage<NZ>::enabled lengths).  One CTA per tile (8
// consecutive i at one j) forms every field of the tile: the rows
// u_c[i0..i0+7][j][0..NKK-1] of the three components arrive in shared memory by 3 x NB
// tensor copies (cp.async.bulk.tensor, boxes of BK k x 1 j x 8 i, completion counted on
// one mbarrier; rows past NKI and k past NKK are filled with zeros by the copy engine).
// Each field's backward z transform then takes its first-pass inputs from that staging
// (velocity, or vorticity / gradients formed on the fly) instead of from global memory,
// and stores z rows of 8 i as K1 does.  u is read from HBM once per tile, in whole rows,
// instead of element-wise by each field's CTA.
// ---------------------------------------------------------------------------
template <int NZ> struct ZStage {
    static constexpr int NKK = 2 * (NZ / 3) + 1;
    static constexpr int NB = (NKK + 127) / 128;                 // boxes along k (<= 128 complex each)
    static constexpr int BK0 = (NKK + NB - 1) / NB;
    static constexpr int BK = BK0 + (9 - BK0 % 8) % 8;           // = 1 mod 8: the 8 rows of a box on distinct banks
    static_assert(BK <= 128, "tensor box wider than 256 doubles");
    static constexpr int words = 3 * NB * 8 * BK;                // staged complex values
    static constexpr size_t smem = sizeof(double2) * words + TCfg<NZ>::template smem<double>() + 16;
    // measured at 512 only (one CTA of 512 threads per SM): as fast as the element-wise K1
    // at 512^3, with u read from HBM once per tile in whole rows
    static constexpr bool enabled = NZ == 512;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                 : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
    return ok != 0;
}
// Wait for phase `parity` of the mbarrier for at most `limit` SM clocks.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity, long long limit) {
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > limit) return false;
    return true;
}

template <int NZ, int FORM>
__global__ void __launch_bounds__(TCfg<NZ>::template nt<double>(), 1) k_zpass_inv_tma(const __grid_constant__ MemberSet<double, 1> ms,
                                                                                     const __grid_constant__ ZMaps maps,
                                                                                     int stage) {
    using C = double2;
    using ZS = ZStage<NZ>;
    constexpr int LT = 8, BK = ZS::BK, NB = ZS::NB;
    constexpr int nf = FORM == 3 ? 9 : 6;
    const Member<double>& mm = ms.m[0];
    if (!mm.active) return;
    const Fields F = mm.F;
    const Geo g = mm.g;
    C* stg = smem_as<C>();
    C* s = stg + ZS::words;
    uint64_t* bar = reinterpret_cast<uint64_t*>(s + NZ * LT);
    const int i0 = blockIdx.x * LT, j = blockIdx.y, tid = threadIdx.x;
    if (stage == 1 && blockIdx.x == 0 && j == 0 && tid == 0) F.clock->ucfl_bits = 0ull;
    const uint32_t ba = smem_u32(bar);
    // tensor copies land on 128-byte boundaries: each box is 128 BK bytes from a staging
    // base that must itself be aligned (the dynamic shared memory of this kernel, which has
    // no static shared memory); otherwise no copy is issued and the status records it
    if (smem_u32(stg) & 127u) {
        if (tid == 0) atomicOr(&F.clock->status, PD_ST_TIMEOUT);
        return;
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(ba) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0) {
        constexpr uint32_t bytes = (uint32_t)(sizeof(C) * ZS::words);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(ba), "r"(bytes) : "memory");
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
            for (int b = 0; b < NB; b++)
                asm volatile(
                    "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                    " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(stg + (c * NB + b) * 8 * BK)),
                    "l"(reinterpret_cast<uint64_t>(&maps.u[c])), "r"(2 * b * BK), "r"(j), "r"(i0), "r"(ba)
                    : "memory");
    }
    // bounded wait (about 2 s of SM clocks); on a timeout the status word records it and,
    // after a second bounded wait for the copies in flight, the CTA returns
    constexpr long long kLimit = 4000000000ll;
    if (!mbar_wait_bounded(ba, 0, kLimit)) {
        if (tid == 0) atomicOr(&F.clock->status, PD_ST_TIMEOUT);
        mbar_wait_bounded(ba, 0, kLimit);
        return;
    }
    constexpr int KK = NZ / 3;   // g.kk (the 2/3 rule)
    const double k2 = wvn(j, g.kj);
    BF bf;
    if constexpr (FORM == 1 || FORM == 2) bf = make_bf(g, F.clock);
    // staged value of component c at (line l, k)
    auto su = [&](int c, int l, int k) -> C {
        const int b = k / BK;
        return stg[((c * NB + b) * 8 + l) * BK + (k - b * BK)];
    };
    const long long zs = (long long)g.nkj * g.nkip;
#pragma unroll 1
    for (int f = 0; f < nf; f++) {
        auto ld = [&](int z, int l) -> C {
            int k;
            if (z <= KK) k = z;
            else if (z >= NZ - KK) k = z - NZ + (2 * KK + 1);
            else return mk(0.0, 0.0);
            if constexpr (FORM == 3) {   // u_c, i k2 u_c, i k3 u_c (f_RK3Derivative, src/pf_rk3.f90:3735-3743)
                const int c = f % 3;
                const C uc = su(c, l, k);
                if (f < 3) return uc;
                const double kd = f < 6 ? k2 : wvn(k, KK);
                return mk(-kd * uc.y, kd * uc.x);
            } else {
                if (f < 3) return su(f, l, k);
                const double k1 = (double)(i0 + l), k3 = wvn(k, KK);
                if constexpr (FORM == 1 || FORM == 2) {
                    const double kv[3] = {k1, k2, k3};
                    const C zero = mk(0.0, 0.0);
                    const C uv[3] = {f != 3 ? su(0, l, k) : zero, f != 4 ? su(1, l, k) : zero, su(2, l, k)};
                    C w3[3];
                    if constexpr (FORM == 2) {
                        if (f == 3) vort_rrot<0>(bf, uv, kv, w3);
                        else if (f == 4) vort_rrot<1>(bf, uv, kv, w3);
                        else vort_rrot<2>(bf, uv, kv, w3);
                    } else {
                        if (f == 3) vort_bf<0>(bf, uv, kv, w3);
                        else if (f == 4) vort_bf<1>(bf, uv, kv, w3);
                        else vort_bf<2>(bf, uv, kv, w3);
                    }
                    return f == 3 ? w3[0] : (f == 4 ? w3[1] : w3[2]);
                } else {   // omega = i k x u (f_RK3PrepareVelocity, src/pf_rk3.f90:402-407,520-525,630-634)
                    const double ka = (f == 3) ? k2 : ((f == 4) ? k3 : k1);
                    const double kb = (f == 3) ? k3 : ((f == 4) ? k1 : k2);
                    const int ca = (f == 3) ? 2 : ((f == 4) ? 0 : 1), cb = (f == 3) ? 1 : ((f == 4) ? 2 : 0);
                    const C a = su(ca, l, k), bb = su(cb, l, k);
                    return mk((-ka * a.y) - (-kb * bb.y), (ka * a.x) - (kb * bb.x));
                }
            }
        };
        C* dst = F.zb + (((long long)f * NZ) * g.nkj + j) * g.nkip + i0;
        auto st = [&](int z, int l, C v) { dst[z * zs + l] = v; };
        TCfg<NZ>::template transform<+1, LT>(s, F.tw_z, ld, st);
        __syncthreads();   // the tile buffer is read by the last pass before the next field's first pass
    }
}

// K2: backward y transforms of field f = blockIdx.z, j zero-padded into
// [KJ+1, NY-KJ-1] (f_RK3TransformjiFs2Rs, src/pf_rk3.f90:1458-1473).  nf = six fields, or
// nine in the R-conv form, per member.
template <int NY, class T, int CAP, int CN = 0>
__global__ void __launch_bounds__(TCfg<NY, true>::template nt<T>(), TCfg<NY, true>::template minb<T>()) k_ypass_inv(const __grid_constant__ MemberSet<T, CAP> ms,
                                                                                                          int nf) {
    using C = typename FieldsT<T>::C;
    const Member<T>& mm = ms.m[CAP == 1 ? 0 : blockIdx.z / nf];
    if (!mm.active) return;
    if constexpr (CAP > 1) {   // a batch slot between members
        if (mm.F.clock->status & PD_ST_IDLE) return;
    }
    const FieldsT<T> F = mm.F;
    const Geo g = mm.g;
    // CN > 0: a cubic grid of CN points a side, every size a compile-time constant
    const int nz_ = CN ? CN : g.nz, nkip_ = CN ? (CN / 3 + 1 + 7) / 8 * 8 : g.nkip;
    C* s = smem_as<C>();
    constexpr int LT = TCfg<NY>::template lines<T>();
    const int i0 = blockIdx.x * LT, z = blockIdx.y, f = blockIdx.z % nf;
    const int lmax = nkip_ - i0;
    constexpr int KJ = NY / 3, NKJ = 2 * KJ + 1;   // g.kj, g.nkj (the 2/3 rule)
    const long long rs = nkip_;
    const C* __restrict__ src = F.zb + (((long long)f * nz_ + z) * NKJ) * rs + i0;
    C* dst = F.yb + (((long long)f * nz_ + z) * NY) * rs + i0;
    auto ld = [&](int y, int l) -> C {
        if (LT > 8 && l >= lmax) return mk(T(0), T(0));
        if (y <= KJ) return src[y * rs + l];
        if (y >= NY - KJ) return src[(y - NY + NKJ) * rs + l];
        return mk(T(0), T(0));
    };
    auto st = [&](int y, int l, C v) {
        if (LT > 8 && l >= lmax) return;
        dst[y * rs + l] = v;
    };
    TCfg<NY, true>::template transform<+1, LT>(s, F.tw_y, ld, st);
}

// K4: forward y transforms of NL field f = blockIdx.z, truncated to j
// (f_RK3TransformjiRs2Fs, src/pf_rk3.f90:1902-1938).
template <int NY, class T, int CAP, int CN = 0>
__global__ void __launch_bounds__(TCfg<NY, true>::template nt<T>(), TCfg<NY, true>::template minb<T>()) k_ypass_fwd(const __grid_constant__ MemberSet<T, CAP> ms) {
    using C = typename FieldsT<T>::C;
    const Member<T>& mm = ms.m[CAP == 1 ? 0 : blockIdx.z / 3];
    if (!mm.active) return;
    if constexpr (CAP > 1) {   // a batch slot between members
        if (mm.F.clock->status & PD_ST_IDLE) return;
    }
    const FieldsT<T> F = mm.F;
    const Geo g = mm.g;
    // CN > 0: a cubic grid of CN points a side, every size a compile-time constant
    const int nz_ = CN ? CN : g.nz, nkip_ = CN ? (CN / 3 + 1 + 7) / 8 * 8 : g.nkip;
    C* s = smem_as<C>();
    constexpr int LT = TCfg<NY>::template lines<T>();
    const int i0 = blockIdx.x * LT, z = blockIdx.y, f = blockIdx.z % 3;
    const int lmax = nkip_ - i0;
    constexpr int KJ = NY / 3, NKJ = 2 * KJ + 1;   // g.kj, g.nkj (the 2/3 rule)
    const long long rs = nkip_;
    const C* __restrict__ src = F.yb + (((long long)f * nz_ + z) * NY) * rs + i0;
    C* dst = F.zb + (((long long)f * nz_ + z) * NKJ) * rs + i0;
    auto ld = [&](int y, int l) -> C {
        if (LT > 8 && l >= lmax) return mk(T(0), T(0));
        return src[y * rs + l];
    };
    auto st = [&](int y, int l, C v) {
        if (LT > 8 && l >= lmax) return;
        if (y <= KJ) dst[y * rs + l] = v;
        else if (y >= NY - KJ) dst[(y - NY + NKJ) * rs + l] = v;
    };
    TCfg<NY, true>::template transform<-1, LT>(s, F.tw_y, ld, st);
}

// K5a: forward z transforms of NL field f = blockIdx.z, x 1/(NX NY NZ), truncated
// to k, stored as rows of NL-hat [c][i][j][k].
template <int NZ, class T, int CAP>
__global__ void __launch_bounds__(TCfg<NZ, true>::template nt<T>(), TCfg<NZ, true>::template minb<T>()) k_zpass_fwd(const __grid_constant__ MemberSet<T, CAP> ms, int mode) {
    using C = typename FieldsT<T>::C;
    const Member<T>& mm = ms.m[CAP == 1 ? 0 : blockIdx.z / 3];
    if (!mm.active) return;
    if constexpr (CAP > 1) {   // a batch slot between members
        if (mm.F.clock->status & PD_ST_IDLE) return;
    }
    const FieldsT<T> F = mm.F;
    const Geo g = mm.g;
    C* s = smem_as<C>();
    constexpr int LT = TCfg<NZ>::template lines<T>();
    const int i0 = blockIdx.x * LT, j = blockIdx.y, f = blockIdx.z % 3;
    const int lmax = g.nkip - i0;
    // NL-hat into the y-pencil buffer, or (mode 1) into rk
    Out3<C> nlh;
    for (int c = 0; c < 3; c++) nlh.p[c] = (mode == 1) ? F.rk[c] : F.yb + c * g.S;
    const int KK = g.kk, NKK = g.nkk, nki = g.nki;
    const long long zs = (long long)g.nkj * g.nkip;
    const C* __restrict__ src = F.zb + (((long long)f * NZ) * g.nkj + j) * g.nkip + i0;
    C* dst = (f == 0 ? nlh.p[0] : (f == 1 ? nlh.p[1] : nlh.p[2])) + ((long long)i0 * g.nkj + j) * NKK;
    const long long istride = (long long)g.nkj * NKK;
    const T norm = (T)g.norm;
    auto ld = [&](int z, int l) -> C {
        if (LT > 8 && l >= lmax) return mk(T(0), T(0));
        return src[z * zs + l];
    };
    auto st = [&](int z, int l, C v) {
        if (i0 + l >= nki) return;
        int k;
        if (z <= KK) k = z;
        else if (z >= NZ - KK) k = z - NZ + NKK;
        else return;
        dst[l * istride + k] = mk(v.x * norm, v.y * norm);
    };
    TCfg<NZ, true>::template transform<-1, LT>(s, F.tw_z, ld, st);
}


// x lengths whose x pass has instantiations with several lines per warp (short, unfused
// lines, where one line leaves most lanes idle in its loads and passes).
template <int N> constexpr bool xlpw_len() { return N <= 64; }
// Lines per warp of the x pass when the simulation leaves the choice to the library,
// measured on B200 (decaying flow, FP64): batches of 32 members run 4 lines per warp up to
// 48 points (32^3: 80K -> 106K member-steps/s, 48^3: 22.2K -> 27.1K) and 2 at 64 points
// (17.0K -> 21.2K); a single simulation, whose step is bound by its launches at these
// sizes, 2 from 48 points (64^3: 0.109 -> 0.101 ms per step).
template <int N, class T, int CAP> constexpr int default_xlpw() {
    return CAP > 1 ? (N <= 48 ? 4 : 2) : (N >= 48 ? 2 : 1);
}

// Lengths whose K1, K2 and K4 have instantiations for cubic grids (every size a
// compile-time constant, so the index arithmetic folds): FP32-mixed, the benchmark and
// ensemble sizes.  Measured at 512^3 shear: K1 0.74 -> 0.69, K2 0.70 -> 0.58, K4 0.32 ->
// 0.30 ms per stage; the FP64 passes, bound by their arithmetic, do not gain.
template <int N, class T> constexpr bool cube_len() {
    return std::is_same<T, float>::value && (N == 32 || N == 48 || N == 64 || N == 96 || N == 128 || N == 192 ||
                                             N == 256 || N == 512 || N == 1024);
}
__host__ __device__ inline bool is_cube(const Geo& g, int n) { return g.nx == n && g.ny == n && g.nz == n; }

// Lengths with batched (kBatchChunk-member) instantiations: the ensemble's sizes.
template <int N> constexpr bool batch_len() {
    return N == 32 || N == 48 || N == 64 || N == 96 || N == 128 || N == 192 || N == 256;
}

// Per-length launchers (passes_n.cuh).  Every launcher takes the batch's geometry g
// (grid sizes and flow type, common to all members), the host array M of its B member
// descriptors and the stream; the members go to the kernels by value, kBatchChunk per launch.
template <int N, class T> cudaError_t configure_n(const Geo& g);
template <int N, class T>
cudaError_t zpass_inv_n(const Geo& g, const Member<T>* M, int B, int stage, cudaStream_t st, const ZMaps* maps);
template <int N, class T> cudaError_t ypass_inv_n(const Geo& g, const Member<T>* M, int B, cudaStream_t st);
template <int N, class T>
cudaError_t xpass_n(const Geo& g, const Member<T>* M, int B, int want_phys, int want_cfl, cudaStream_t st);
template <int N, class T> cudaError_t xpass_stats_n(const Geo& g, const Member<T>* M, double* rs, cudaStream_t st);
template <int N, class T> cudaError_t ypass_fwd_n(const Geo& g, const Member<T>* M, int B, cudaStream_t st);
template <int N, class T> cudaError_t zpass_fwd_n(const Geo& g, const Member<T>* M, int B, int mode, cudaStream_t st);

}  // namespace pd
