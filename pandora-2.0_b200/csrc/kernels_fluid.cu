// kernels_fluid.cu -- the five HBM passes of one RK3 stage on sm_100a, plus the
// small kernels around them (statistics, forcing/dt scalars, seeded init).
//
// Pass structure per stage (replacing f_RK3PrepareRealSpace, f_RK3RealSpace and
// f_RK3SolveNavierStokes, src/pf_rk3.f90:205-329, 960-1237, 1996-2142, whose
// MPI/FFTW pencil transposes collapse into on-chip tile transposes):
//   K1 zpass_inv   u (3 x S)          -> omega in registers, 6 backward z FFTs -> zb [6][z][j][i]
//   K2 ypass_inv   zb                 -> 6 backward y FFTs                     -> yb [6][z][y][i]
//   K3 xpass       yb (6 half spectra)-> 3 complex c2r (two real lines each), omega x u,
//                                        2 complex r2c, truncate              -> yb fields 0..2
//   K4 ypass_fwd   yb fields 0..2     -> 3 forward y FFTs, truncate j        -> zb fields 0..2
//   K5 zpass_fwd   zb fields 0..2     -> 3 forward z FFTs, x 1/(NX NY NZ), truncate k, then the
//                                        per-mode RHS + low-storage RK3 + continuity fix on u, rk
// Every pass reads and writes HBM once with coalesced rows; the tile transposes
// between pencil orientations happen in shared memory.
#include <cuda_runtime.h>
#include <math.h>
#include "fft_core.cuh"
#include "pandora_internal.cuh"

namespace pd {

using pdfft::fft_tile;
using pdfft::mk;

constexpr int NT = 256;           // threads per CTA of the FFT passes

// Lines per tile of the strided passes (K1, K2, K4) and of K5, per length.
template <int N> struct Cfg {
    static constexpr int L = 8;                     // K1/K2/K4
    static constexpr int LP = L + 1;
    static constexpr int L5 = (N <= 512) ? 8 : 2;   // K5 keeps 3 truncated fields on chip
    static constexpr int LP5 = L5 + 1;
    static constexpr int LX = (N <= 512) ? 4 : 2;   // K3 lines (x 3 complex arrays)
    static constexpr int LPX = 3 * LX + 1;
};

#define PD_FOR_EACH_N(X) \
    X(16) X(24) X(32) X(48) X(64) X(96) X(128) X(192) X(256) X(384) X(512) X(768) X(1024)

bool supported_length(int n) {
    switch (n) {
#define PD_CASE(N) case N:
        PD_FOR_EACH_N(PD_CASE)
#undef PD_CASE
        return true;
    default:
        return false;
    }
}

// ---------------------------------------------------------------------------
// K1: spectral velocity and vorticity, backward z transforms.
// CTA = (i tile of L lines, one j).  Field f: 0..2 velocity, 3..5 vorticity
// omega = i k x u, isotropic branch of f_RK3PrepareVelocity
// (src/pf_rk3.f90:402-407,520-525,630-634, f_RK3Derivative 3735-3743).
// Zero padding of k into [KK+1, NZ-KK-1] as src/pf_rk3.f90:437-443.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double2 field_value(const double2* const* u, long long m, int f, double k1,
                                               double k2, double k3) {
    if (f < 3) return u[f][m];
    double2 a, b;
    double ka, kb;
    // omega1 = (0 - dv/dz) + dw/dy ; omega2 = du/dz - dw/dx ; omega3 = (-du/dy) + dv/dx
    if (f == 3) { a = u[2][m]; ka = k2; b = u[1][m]; kb = k3; }
    else if (f == 4) { a = u[0][m]; ka = k3; b = u[2][m]; kb = k1; }
    else { a = u[1][m]; ka = k1; b = u[0][m]; kb = k2; }
    // i*ka*a - i*kb*b, with i*k*v = (-k v.y, k v.x)
    return mk((-ka * a.y) - (-kb * b.y), (ka * a.x) - (kb * b.x));
}

template <int NZ>
__global__ void __launch_bounds__(NT) k_zpass_inv(Fields F, Geo g, int stage) {
    constexpr int L = Cfg<NZ>::L, LP = Cfg<NZ>::LP;
    extern __shared__ double2 smem[];
    double2* s = smem;
    const int tid = threadIdx.x;
    const int it = blockIdx.x, j = blockIdx.y;
    const int i0 = it * L;
    if (stage == 1 && it == 0 && j == 0 && tid == 0) F.clock->ucfl_bits = 0ull;
    const double k2 = wvn(j, g.kj);
    const int KK = g.kk, NKK = g.nkk, npad = NZ - NKK;
    const double2* u[3] = {F.u[0], F.u[1], F.u[2]};
    for (int f = 0; f < 6; f++) {
        for (int w = tid; w < npad * L; w += NT) {
            const int l = w % L, z = KK + 1 + w / L;
            s[z * LP + l] = mk(0.0, 0.0);
        }
        for (int w = tid; w < NKK * L; w += NT) {
            const int k = w % NKK, l = w / NKK;
            const int i = i0 + l;
            const int z = (k <= KK) ? k : NZ - NKK + k;
            double2 v = mk(0.0, 0.0);
            if (i < g.nki) {
                const long long m = ((long long)i * g.nkj + j) * NKK + k;
                v = field_value(u, m, f, (double)i, k2, wvn(k, KK));
            }
            s[z * LP + l] = v;
        }
        __syncthreads();
        fft_tile<NZ, +1, L, LP, NT>(s, F.tw_z, tid);
        double2* dst = F.zb + (((long long)f * NZ) * g.nkj + j) * g.nkip + i0;
        for (int w = tid; w < NZ * L; w += NT) {
            const int l = w % L, z = w / L;
            dst[(long long)z * g.nkj * g.nkip + l] = s[z * LP + l];
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// K2: backward y transforms, pad j into [KJ+1, NY-KJ-1] (src/pf_rk3.f90:1458-1473).
// CTA = (i tile, z, field).
// ---------------------------------------------------------------------------
template <int NY>
__global__ void __launch_bounds__(NT) k_ypass_inv(Fields F, Geo g) {
    constexpr int L = Cfg<NY>::L, LP = Cfg<NY>::LP;
    extern __shared__ double2 smem[];
    double2* s = smem;
    const int tid = threadIdx.x;
    const int i0 = blockIdx.x * L, z = blockIdx.y, f = blockIdx.z;
    const int KJ = g.kj, NKJ = g.nkj, npad = NY - NKJ;
    const double2* src = F.zb + (((long long)f * g.nz + z) * NKJ) * g.nkip + i0;
    for (int w = tid; w < npad * L; w += NT) {
        const int l = w % L, y = KJ + 1 + w / L;
        s[y * LP + l] = mk(0.0, 0.0);
    }
    for (int w = tid; w < NKJ * L; w += NT) {
        const int l = w % L, jj = w / L;
        const int y = (jj <= KJ) ? jj : NY - NKJ + jj;
        s[y * LP + l] = src[(long long)jj * g.nkip + l];
    }
    __syncthreads();
    fft_tile<NY, +1, L, LP, NT>(s, F.tw_y, tid);
    double2* dst = F.yb + (((long long)f * g.nz + z) * NY) * g.nkip + i0;
    for (int w = tid; w < NY * L; w += NT) {
        const int l = w % L, y = w / L;
        dst[(long long)y * g.nkip + l] = s[y * LP + l];
    }
}

// ---------------------------------------------------------------------------
// K3: x pass.  Six half spectra per (z,y) line -> three complex backward FFTs
// (pairs (u1,u2), (u3,w1), (w2,w3), each the c2r of two real lines at once; the
// Hermitian extension drops Im of the i=0 mode as FFTW's c2r does,
// src/pf_fftw.f90:646,749-756) -> NL = omega x u (f_RK3ComputeNonlinearIsotropic,
// src/pf_rk3.f90:1597-1628) -> two complex forward FFTs ((n1,n2), (n3,0)) ->
// r2c split, truncate i to 0..KI (src/pf_fftw.f90:780).  Writes NL into yb
// fields 0..2 in place (each CTA owns its lines).  Optionally materialises the
// physical velocity (arr_u*_3r, src/pf_rk3.f90:1108-1115) and the CFL maximum.
// ---------------------------------------------------------------------------
template <int NX>
__global__ void __launch_bounds__(NT) k_xpass(Fields F, Geo g, int want_phys, int want_cfl) {
    constexpr int LX = Cfg<NX>::LX, LPX = Cfg<NX>::LPX;
    extern __shared__ double2 smem[];
    double2* s = smem;
    __shared__ double red[NT / 32];
    const int tid = threadIdx.x;
    const long long q0 = (long long)blockIdx.x * LX;
    const long long lines = (long long)g.ny * g.nz;
    const long long fstride = lines * g.nkip;     // distance between fields in yb
    const int KI = g.ki, NKI = g.nki;
    // build Z = X + iY per pair
    for (int w = tid; w < NKI * LX; w += NT) {
        const int m = w % NKI, l = w / NKI;
        const long long q = q0 + l;
        if (q >= lines) continue;
        const double2* b = F.yb + q * g.nkip + m;
#pragma unroll
        for (int p = 0; p < 3; p++) {
            double2 X = b[(2 * p) * fstride], Y = b[(2 * p + 1) * fstride];
            if (m == 0) { X.y = 0.0; Y.y = 0.0; }
            s[m * LPX + p * LX + l] = mk(X.x - Y.y, X.y + Y.x);
            if (m > 0) s[(NX - m) * LPX + p * LX + l] = mk(X.x + Y.y, -X.y + Y.x);
        }
    }
    for (int w = tid; w < (NX - 2 * KI - 1) * 3 * LX; w += NT) {
        const int c = w % (3 * LX), n = KI + 1 + w / (3 * LX);
        s[n * LPX + c] = mk(0.0, 0.0);
    }
    __syncthreads();
    fft_tile<NX, +1, 3 * LX, LPX, NT>(s, F.tw_x, tid);
    // nonlinear term (and physical velocity / CFL)
    double umax = 0.0;
    for (int w = tid; w < NX * LX; w += NT) {
        const int n = w % NX, l = w / NX;
        const long long q = q0 + l;
        double2 a = s[n * LPX + l], b = s[n * LPX + LX + l], c = s[n * LPX + 2 * LX + l];
        const double u1 = a.x, u2 = a.y, u3 = b.x, w1 = b.y, w2 = c.x, w3 = c.y;
        if (q < lines) {
            if (want_phys) {
                F.phys[q * NX + n] = u1;
                F.phys[g.R + q * NX + n] = u2;
                F.phys[2 * g.R + q * NX + n] = u3;
            }
            if (want_cfl) umax = fmax(umax, fabs(u1) + fabs(u2) + fabs(u3));
        }
        const double n1 = u3 * w2 - u2 * w3;
        const double n2 = u1 * w3 - u3 * w1;
        const double n3 = u2 * w1 - u1 * w2;
        s[n * LPX + l] = mk(n1, n2);
        s[n * LPX + LX + l] = mk(n3, 0.0);
    }
    if (want_cfl) {
        for (int o = 16; o > 0; o >>= 1) umax = fmax(umax, __shfl_xor_sync(0xffffffffu, umax, o));
        if ((tid & 31) == 0) red[tid >> 5] = umax;
    }
    __syncthreads();
    if (want_cfl && tid < 32) {
        double v = (tid < NT / 32) ? red[tid] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (tid == 0) atomicMax(&F.clock->ucfl_bits, (unsigned long long)__double_as_longlong(v));
    }
    fft_tile<NX, -1, 2 * LX, LPX, NT>(s, F.tw_x, tid);
    for (int w = tid; w < g.nkip * LX; w += NT) {
        const int m = w % g.nkip, l = w / g.nkip;
        const long long q = q0 + l;
        if (q >= lines) continue;
        double2 n1 = mk(0.0, 0.0), n2 = n1, n3 = n1;
        if (m < NKI) {
            const int mc = (NX - m) % NX;
            double2 Z = s[m * LPX + l], Zc = s[mc * LPX + l];
            n1 = mk(0.5 * (Z.x + Zc.x), 0.5 * (Z.y - Zc.y));
            n2 = mk(0.5 * (Z.y + Zc.y), -0.5 * (Z.x - Zc.x));
            double2 W = s[m * LPX + LX + l], Wc = s[mc * LPX + LX + l];
            n3 = mk(0.5 * (W.x + Wc.x), 0.5 * (W.y - Wc.y));
        }
        double2* b = F.yb + q * g.nkip + m;
        b[0] = n1;
        b[fstride] = n2;
        b[2 * fstride] = n3;
    }
}

// ---------------------------------------------------------------------------
// K4: forward y transforms of the three NL fields, truncate j
// (f_RK3TransformjiRs2Fs, src/pf_rk3.f90:1902-1938).
// ---------------------------------------------------------------------------
template <int NY>
__global__ void __launch_bounds__(NT) k_ypass_fwd(Fields F, Geo g) {
    constexpr int L = Cfg<NY>::L, LP = Cfg<NY>::LP;
    extern __shared__ double2 smem[];
    double2* s = smem;
    const int tid = threadIdx.x;
    const int i0 = blockIdx.x * L, z = blockIdx.y, f = blockIdx.z;
    const double2* src = F.yb + (((long long)f * g.nz + z) * NY) * g.nkip + i0;
    for (int w = tid; w < NY * L; w += NT) {
        const int l = w % L, y = w / L;
        s[y * LP + l] = src[(long long)y * g.nkip + l];
    }
    __syncthreads();
    fft_tile<NY, -1, L, LP, NT>(s, F.tw_y, tid);
    const int KJ = g.kj, NKJ = g.nkj;
    double2* dst = F.zb + (((long long)f * g.nz + z) * NKJ) * g.nkip + i0;
    for (int w = tid; w < NKJ * L; w += NT) {
        const int l = w % L, jj = w / L;
        const int y = (jj <= KJ) ? jj : NY - NKJ + jj;
        dst[(long long)jj * g.nkip + l] = s[y * LP + l];
    }
}

// ---------------------------------------------------------------------------
// K5: forward z transforms x normalisation, truncate k (f_RK3TransformkRs2Fs +
// f_Fftw_k_Rs2Fs, src/pf_rk3.f90:2242-2316, src/pf_fftw.f90:841-879), then per
// mode f_RK3FormFIsotropic + f_RK3RungeKutta + f_RK3ContinuityFixIsotropic
// (src/pf_rk3.f90:2323-2487, 3457-3531).  mode 1 stores NL-hat into rk instead
// (the transform test hook of src/ptf_rk3.f90:629-734).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void rk_coeffs(int stage, double& beta, double& gamma) {
    if (stage == 1) { beta = 0.0; gamma = 1.0 / 3.0; }
    else if (stage == 2) { beta = -(5.0 / 9.0); gamma = 15.0 / 16.0; }
    else { beta = -(153.0 / 128.0); gamma = 8.0 / 15.0; }
}

template <int NZ>
__global__ void __launch_bounds__(NT) k_zpass_fwd_update(Fields F, Geo g, int stage, int mode) {
    constexpr int L = Cfg<NZ>::L5, LP = Cfg<NZ>::LP5;
    extern __shared__ double2 smem[];
    double2* s = smem;                    // FFT tile [NZ][LP]
    double2* T = smem + NZ * LP;          // truncated NL [3][NKK][LP]
    const int tid = threadIdx.x;
    const int i0 = blockIdx.x * L, j = blockIdx.y;
    const int KK = g.kk, NKK = g.nkk;
    for (int f = 0; f < 3; f++) {
        const double2* src = F.zb + (((long long)f * NZ) * g.nkj + j) * g.nkip + i0;
        for (int w = tid; w < NZ * L; w += NT) {
            const int l = w % L, z = w / L;
            s[z * LP + l] = src[(long long)z * g.nkj * g.nkip + l];
        }
        __syncthreads();
        fft_tile<NZ, -1, L, LP, NT>(s, F.tw_z, tid);
        for (int w = tid; w < NKK * L; w += NT) {
            const int k = w % NKK, l = w / NKK;
            const int z = (k <= KK) ? k : NZ - NKK + k;
            double2 v = s[z * LP + l];
            T[(f * NKK + k) * LP + l] = mk(v.x * g.norm, v.y * g.norm);
        }
        __syncthreads();
    }
    const double dt = F.clock->dt;
    double beta, gamma;
    rk_coeffs(stage, beta, gamma);
    const double k2 = wvn(j, g.kj);
    const int NK = g.fnk, FW = 2 * NK + 1;
    for (int w = tid; w < NKK * L; w += NT) {
        const int k = w % NKK, l = w / NKK;
        const int i = i0 + l;
        if (i >= g.nki) continue;
        const long long m = ((long long)i * g.nkj + j) * NKK + k;
        double2 nl[3];
#pragma unroll
        for (int c = 0; c < 3; c++) nl[c] = T[(c * NKK + k) * LP + l];
        if (mode == 1) {
#pragma unroll
            for (int c = 0; c < 3; c++) F.rk[c][m] = nl[c];
            continue;
        }
        const double k1 = (double)i, k3 = wvn(k, KK);
        const double kmag2 = (k1 * k1) + (k2 * k2) + (k3 * k3);
        if (!(kmag2 > 0.0)) continue;
        const double kv[3] = {k1, k2, k3};
        const double2 kdn = mk(k1 * nl[0].x + k2 * nl[1].x + k3 * nl[2].x,
                               k1 * nl[0].y + k2 * nl[1].y + k3 * nl[2].y);
        double2 force[3] = {mk(0, 0), mk(0, 0), mk(0, 0)};
        const double kmag = sqrt(kmag2);
        if (kmag <= g.force_kf && kmag > 0.0) {
            const int jw = (int)k2, kw = (int)k3;
            if (i <= NK && jw >= -NK && jw <= NK && kw >= -NK && kw <= NK) {
                double2 fv[3];
                const long long fi = ((long long)i * FW + (jw + NK)) * FW + (kw + NK);
                const long long fstride = (long long)(NK + 1) * FW * FW;
#pragma unroll
                for (int c = 0; c < 3; c++) fv[c] = F.forcing[c * fstride + fi];
                const double2 kdb = mk(k1 * fv[0].x + k2 * fv[1].x + k3 * fv[2].x,
                                       k1 * fv[0].y + k2 * fv[1].y + k3 * fv[2].y);
#pragma unroll
                for (int c = 0; c < 3; c++)
                    force[c] = mk(fv[c].x - ((kv[c] / kmag2) * kdb.x), fv[c].y - ((kv[c] / kmag2) * kdb.y));
            }
        }
        double2 uu[3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            uu[c] = F.u[c][m];
            const double2 tot = mk(-g.nu * kmag2 * uu[c].x - nl[c].x + (kv[c] / kmag2) * kdn.x + force[c].x,
                                   -g.nu * kmag2 * uu[c].y - nl[c].y + (kv[c] / kmag2) * kdn.y + force[c].y);
            double2 r;
            if (stage == 1) r = tot;   // beta = 0; registers start at zero (src/pf_arrays.f90:805-832)
            else {
                const double2 r0 = F.rk[c][m];
                r = mk((beta * r0.x) + tot.x, (beta * r0.y) + tot.y);
            }
            F.rk[c][m] = r;
            uu[c] = mk(uu[c].x + (gamma * dt * r.x), uu[c].y + (gamma * dt * r.y));
        }
        const double2 kdu = mk(k1 * uu[0].x + k2 * uu[1].x + k3 * uu[2].x,
                               k1 * uu[0].y + k2 * uu[1].y + k3 * uu[2].y);
#pragma unroll
        for (int c = 0; c < 3; c++)
            F.u[c][m] = mk(uu[c].x - (kv[c] * kdu.x / kmag2), uu[c].y - (kv[c] * kdu.y / kmag2));
    }
}

// ---------------------------------------------------------------------------
// E(k), dissipation and Reynolds-stress sums, f_FluidstatsFsPrimaryQuants
// (src/pf_fluidstats.f90:1423-1576): per mode e = (phi11+phi22+phi33)/2 (x2 for
// i != 0), d = 2 k^2 nu e, binned in [kk-1/2, kk+1/2).  Raw sums; the host
// divides by the mode density.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_stats(Fields F, Geo g) {
    extern __shared__ double sh[];
    const int K = g.kkmax;
    double* se = sh;            // [K+1]
    double* sd = sh + (K + 1);  // [K+1]
    double* sp = sh + 2 * (K + 1);
    for (int q = threadIdx.x; q < 2 * (K + 1) + 3; q += blockDim.x) sh[q] = 0.0;
    __syncthreads();
    double p11 = 0, p22 = 0, p33 = 0;
    const long long total = g.S;
    for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < total;
         m += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(m % g.nkk);
        const long long ij = m / g.nkk;
        const int jj = (int)(ij % g.nkj), i = (int)(ij / g.nkj);
        const double a = (double)i, b = wvn(jj, g.kj), c = wvn(k, g.kk);
        const double km = sqrt((a * a) + (b * b) + (c * c));
        const double2 u1 = F.u[0][m], u2 = F.u[1][m], u3 = F.u[2][m];
        double q11 = u1.x * u1.x + u1.y * u1.y, q22 = u2.x * u2.x + u2.y * u2.y;
        double q33 = u3.x * u3.x + u3.y * u3.y;
        if (i != 0) { q11 *= 2.0; q22 *= 2.0; q33 *= 2.0; }
        p11 += q11; p22 += q22; p33 += q33;
        const double e = 0.5 * (q11 + q22 + q33);
        if (!isfinite(e)) atomicOr(&F.clock->status, PD_ST_NAN);
        const double d = 2.0 * km * km * g.nu * e;
        const int kc = (int)floor(km + 0.5);
        for (int q = kc - 1; q <= kc + 1; q++) {
            if (q < 1 || q > K) continue;
            if (km >= (double)q - 0.5 && km < (double)q + 0.5) {
                atomicAdd(&se[q], e);
                atomicAdd(&sd[q], d);
            }
        }
    }
    atomicAdd(&sp[0], p11);
    atomicAdd(&sp[1], p22);
    atomicAdd(&sp[2], p33);
    __syncthreads();
    for (int q = threadIdx.x; q < 2 * (K + 1) + 3; q += blockDim.x)
        if (sh[q] != 0.0) atomicAdd(&F.shell[q], sh[q]);
}

// ---------------------------------------------------------------------------
// Stage scalars: dt (f_RK3Tstep, src/pf_rk3.f90:3852-3948) at stage 1 and the OU
// forcing update f_ForceCalc (src/pf_force.f90:106-268) at every stage with the
// project RNG: normal-pair call c of a stage draws from sub-stream c.  The
// normal pairs are generated in parallel, the OU update replays the reference's
// loop order in one thread (it overwrites entries of the i=0 plane).
// ---------------------------------------------------------------------------
__device__ int normal_pair(uint64_t key, uint64_t call, double& r1, double& r2) {
    const uint64_t sub = mix64(key + (call + 1) * PD_GOLDEN);
    double x1 = 0.0, x2 = 0.0, w = 2.0;
    int a = 0;
    while (w >= 1.0) {
        if (a >= kMaxPolarTries) { r1 = 0.0; r2 = 0.0; return -1; }
        x1 = uniform(sub, 2 * (uint64_t)a);
        x2 = uniform(sub, 2 * (uint64_t)a + 1);
        x1 = __dsub_rn(__dmul_rn(2.0, x1), 1.0);
        x2 = __dsub_rn(__dmul_rn(2.0, x2), 1.0);
        w = __dadd_rn(__dmul_rn(x1, x1), __dmul_rn(x2, x2));
        a++;
    }
    w = sqrt((-2.0 * log(w)) / w);
    r1 = x1 * w;
    r2 = x2 * w;
    return 0;
}

__global__ void __launch_bounds__(256) k_stage_scalars(Fields F, Geo g, StepParams sp, ForceParams fp,
                                                       int stage) {
    extern __shared__ double nrm[];   // [2 * calls]
    Clock* ck = F.clock;
    const int tid = threadIdx.x;
    if (stage == 1 && tid == 0) {
        const double ucfl = __longlong_as_double((long long)ck->ucfl_bits);
        double dt = sp.rk3_dt;
        if (sp.rk3_timestep == PANDORA_RK3_TIMESTEP_FIXED) {
            dt = sp.rk3_dt;
        } else if (sp.rk3_timestep == PANDORA_RK3_TIMESTEP_CFL) {
            dt = (ucfl == 0.0) ? 0.02 : sp.rk3_cfl * g.dx / ucfl;
        } else if (sp.rk3_timestep == PANDORA_RK3_TIMESTEP_DECIDE) {
            if (sp.f_type == PANDORA_F_ISOTROPIC) {
                if (ucfl == 0.0) dt = 0.02;
                else { dt = sp.rk3_cfl * g.dx / ucfl; if (dt > sp.force_tf) dt = sp.force_tf; }
            } else if (sp.f_type == PANDORA_F_ISOTROPIC_DEFORMED) {
                const double m = fmin(fmin(g.dx, g.dy), g.dz);
                if (ucfl == 0.0) dt = 0.02;
                else { dt = sp.rk3_cfl * m / ucfl; if (dt > sp.force_tf) dt = sp.force_tf; }
            } else {
                dt = ((0.5 / sp.f_deform_s) / (double)sp.f_remesh_t);
            }
        }
        ck->dt = dt;
    }
    __syncthreads();
    const int NK = g.fnk, FW = 2 * NK + 1;
    const long long fstride = (long long)(NK + 1) * FW * FW;
    const int tstep = ck->tstep;
    if (tstep >= fp.stop) {
        for (long long q = tid; q < 3 * fstride; q += blockDim.x) F.forcing[q] = mk(0.0, 0.0);
        return;
    }
    const long long calls = fp.calls_per_stage;
    const uint64_t base = ((uint64_t)tstep * 3 + (uint64_t)(stage - 1)) * (uint64_t)calls;
    unsigned int bad = 0;
    for (long long c = tid; c < calls; c += blockDim.x) {
        double r1, r2;
        if (normal_pair(fp.key, base + (uint64_t)c, r1, r2)) bad = 1;
        nrm[2 * c] = r1;
        nrm[2 * c + 1] = r2;
    }
    if (bad) atomicOr(&ck->status, PD_ST_POLAR);
    __syncthreads();
    if (tid != 0) return;
    const double dt_over_TF = ck->dt / fp.tf;
    const double amp = sqrt(2.0 * (fp.sigma * fp.sigma) * dt_over_TF);
    const double decay = 1.0 - dt_over_TF;
    long long c = 0;
    double2* ff = F.forcing;
    auto at = [&](int comp, int i, int jw, int kw) -> double2& {
        return ff[comp * fstride + ((long long)i * FW + (jw + NK)) * FW + (kw + NK)];
    };
    auto ou = [&](int i, int jw, int kw) {
        for (int comp = 0; comp < 3; comp++) {
            double2& v = at(comp, i, jw, kw);
            const double re = nrm[2 * (c + comp)], im = nrm[2 * (c + comp) + 1];
            v = mk(v.x * decay + re * amp, v.y * decay + im * amp);
        }
        c += 3;
    };
    auto conj_copy = [&](int jd, int kd, int js, int ks) {
        for (int comp = 0; comp < 3; comp++) {
            const double2 sv = at(comp, 0, js, ks);
            at(comp, 0, jd, kd) = mk(sv.x, -sv.y);
        }
    };
    for (int jw = 0; jw <= NK; jw++)
        for (int kw = 0; kw <= NK; kw++) {
            ou(0, jw, kw);
            conj_copy(-jw, -kw, jw, kw);
            if (jw > 0) {
                ou(0, -jw, kw);
                conj_copy(jw, -kw, -jw, kw);
            }
        }
    for (int i = 1; i <= NK; i++)
        for (int jw = -NK; jw <= NK; jw++)
            for (int kw = -NK; kw <= NK; kw++) ou(i, jw, kw);
}

// simtime after stage s: t0 + {1/3, 3/4, 1} dt (src/pg_rk3.f90:109-127); the step
// counter advances after stage 3.
__global__ void k_advance_time(Fields F, int stage) {
    Clock* ck = F.clock;
    if (stage == 1) ck->simtime = ck->t0 + (1.0 / 3.0) * ck->dt;
    else if (stage == 2) ck->simtime = ck->t0 + (3.0 / 4.0) * ck->dt;
    else {
        ck->simtime = ck->t0 + ck->dt;
        ck->t0 = ck->simtime;
        ck->tstep += 1;
    }
}

// ---------------------------------------------------------------------------
// Seeded initial field, f_InitialiseFluid (src/pf_initialise.f90:97-512).  The
// draw index of every mode is known in closed form (the reference loops run
// one index past the stored range, and the i=0 plane draws a second triple for
// k != 0), so each thread builds its modes independently.
// ---------------------------------------------------------------------------
__device__ double init_spec(const InitParams& p, double kmag) {
    const double pi = 3.14159265358979323846264338327950288;
    switch (p.type) {
    case PANDORA_F_INIT_GAUSS:
        return (p.u0 / (p.kv * sqrt(4.0 * asin(1.0)))) *
               exp(-((kmag - p.kp) * (kmag - p.kp)) / (2.0 * (p.kv * p.kv)));
    case PANDORA_F_INIT_KERR:
        return (p.u0 / (4.0 * asin(1.0))) * (kmag * kmag * kmag * kmag) * exp(-(2.0 * kmag * kmag) / (p.kp * p.kp));
    case PANDORA_F_INIT_PULSE:
        return (sqrt((kmag - p.kp) * (kmag - p.kp)) < p.kv) ? p.u0 : 0.0;
    case PANDORA_F_INIT_SQUARE:
        return (kmag > p.kstart && kmag < p.kend) ? 1.0 : 0.0;
    case PANDORA_F_INIT_MINUSFIVETHIRD:
        if (kmag < p.kstart)
            return 1.5 * pow(p.epsilon, 2.0 / 3.0) * pow(p.kstart, -5.0 / 3.0) * ((kmag / p.kstart) * (kmag / p.kstart));
        if (kmag < p.kend)
            return 1.5 * pow(p.epsilon, 2.0 / 3.0) * pow(p.kstart, -5.0 / 3.0) * pow(kmag / p.kstart, -5.0 / 3.0);
        return 0.0;
    case PANDORA_F_INIT_MATSUMOTO:
        if (kmag < p.kstart) return p.u0 * (kmag * kmag);
        if (kmag < p.kend) return p.u0 * pow(p.kstart, 11.0 / 3.0) * pow(kmag, -5.0 / 3.0);
        return 0.0;
    case PANDORA_F_INIT_AHMED_ELGHOBASHI: {
        const double k4 = (kmag * kmag) * (kmag * kmag);
        const double kp5 = p.kp * p.kp * p.kp * p.kp * p.kp;
        return 16.0 * pow(2.0 / pi, 0.5) * 1.5 * p.u0 * (k4 / kp5) * exp(-(2.0 * kmag * kmag) / (p.kp * p.kp));
    }
    default:
        return 0.0;
    }
}

__device__ void rogallo_mode(const InitParams& p, double k1, double k2, double k3, double kmag, double r1,
                             double r2, double r3, double2 t[3]) {
    const double twopi = 6.283185307179586476925286766559005768;
    const double fourpi = 12.566370614359172953850573533118011536;
    r1 = twopi * r1; r2 = twopi * r2; r3 = twopi * r3;
    const double k2d = (k1 * k1) + (k2 * k2);
    t[0] = t[1] = t[2] = mk(0.0, 0.0);
    if (!(kmag > 0.0)) return;
    const double ek = init_spec(p, kmag);
    const double factor = sqrt(ek / (fourpi * kmag * kmag));
    const double2 al = mk(factor * cos(r1) * cos(r3), factor * sin(r1) * cos(r3));
    const double2 be = mk(factor * cos(r2) * sin(r3), factor * sin(r2) * sin(r3));
    if (!(k2d > 0.0)) return;
    const double den = kmag * sqrt(k2d);
    t[0] = mk((al.x * kmag * k2 + be.x * k1 * k3) / den, (al.y * kmag * k2 + be.y * k1 * k3) / den);
    t[1] = mk((be.x * k2 * k3 - al.x * kmag * k1) / den, (be.y * k2 * k3 - al.y * kmag * k1) / den);
    t[2] = mk(-(be.x * sqrt(k2d)) / kmag, -(be.y * sqrt(k2d)) / kmag);
}

__global__ void k_init_fluid(Fields F, Geo g, InitParams ip) {
    const int KJ = g.kj, KK = g.kk, NKJ = g.nkj, NKK = g.nkk;
    const long long plane0 = (long long)(KJ + 1) * (KK + 1);
    const long long rest = (long long)g.ki * NKJ * NKK;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    auto U = [&](int c, int i, int j, int k) -> double2& {
        return F.u[c][((long long)i * NKJ + j) * NKK + k];
    };
    if (idx < plane0) {
        const int j = (int)(idx / (KK + 1)), k = (int)(idx % (KK + 1));
        const uint64_t n = (uint64_t)j * 3 * (2 * KK + 1) + (k == 0 ? 0 : 3 + 6 * (uint64_t)(k - 1));
        const double k1 = 0.0, k2 = wvn(j, KJ), k3 = wvn(k, KK);
        const double kmag = sqrt((k1 * k1) + (k2 * k2) + (k3 * k3));
        double2 t[3];
        rogallo_mode(ip, k1, k2, k3, kmag, uniform(ip.key, n), uniform(ip.key, n + 1), uniform(ip.key, n + 2), t);
        const int jj = (j != 0) ? NKJ - j : j, kk = (k != 0) ? NKK - k : k;
        for (int c = 0; c < 3; c++) U(c, 0, j, k) = t[c];
        for (int c = 0; c < 3; c++) U(c, 0, jj, kk) = mk(t[c].x, -t[c].y);
        if (k != 0) {
            double k2n = wvn(jj, KJ);
            if (ip.b220 > 1) k2n = k2n / (double)ip.b220;
            rogallo_mode(ip, k1, k2n, k3, kmag, uniform(ip.key, n + 3), uniform(ip.key, n + 4),
                         uniform(ip.key, n + 5), t);
            for (int c = 0; c < 3; c++) U(c, 0, jj, k) = t[c];
            for (int c = 0; c < 3; c++) U(c, 0, j, kk) = mk(t[c].x, -t[c].y);
        }
        return;
    }
    const long long r = idx - plane0;
    if (r >= rest) return;
    const int k = (int)(r % NKK);
    const long long r2 = r / NKK;
    const int j = (int)(r2 % NKJ), i = 1 + (int)(r2 / NKJ);
    const uint64_t base1 = (uint64_t)(KJ + 1) * 3 * (2 * KK + 1);
    const uint64_t n = base1 + 3 * ((((uint64_t)(i - 1) * (NKJ + 1)) + j) * (NKK + 1) + k);
    const double a = (double)i, b = wvn(j, KJ), c3 = wvn(k, KK);
    const double kmag = sqrt((a * a) + (b * b) + (c3 * c3));
    double2 t[3];
    rogallo_mode(ip, a, b, c3, kmag, uniform(ip.key, n), uniform(ip.key, n + 1), uniform(ip.key, n + 2), t);
    for (int c = 0; c < 3; c++) U(c, i, j, k) = t[c];
}

// Non-finite check of the spectral state (sets PD_ST_NAN).
__global__ void k_check_finite(Fields F, Geo g) {
    bool bad = false;
    for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < g.S;
         m += (long long)gridDim.x * blockDim.x) {
        for (int c = 0; c < 3; c++) {
            const double2 v = F.u[c][m];
            if (!isfinite(v.x) || !isfinite(v.y)) bad = true;
        }
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(&F.clock->status, PD_ST_NAN);
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
template <int N> static size_t smem_k1() { return sizeof(double2) * N * Cfg<N>::LP; }
template <int N> static size_t smem_kx() { return sizeof(double2) * N * Cfg<N>::LPX; }
template <int N> static size_t smem_k5(const Geo& g) {
    return sizeof(double2) * ((size_t)N * Cfg<N>::LP5 + (size_t)3 * g.nkk * Cfg<N>::LP5);
}

static int sm_count() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

cudaError_t configure_kernels(const Geo& g) {
    cudaError_t e = cudaSuccess;
#define PD_CFG(N)                                                                                   \
    if (g.nz == N || g.ny == N || g.nx == N) {                                                      \
        e = cudaFuncSetAttribute(k_zpass_inv<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,       \
                                 (int)smem_k1<N>());                                                \
        if (e) return e;                                                                            \
        e = cudaFuncSetAttribute(k_ypass_inv<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,       \
                                 (int)smem_k1<N>());                                                \
        if (e) return e;                                                                            \
        e = cudaFuncSetAttribute(k_ypass_fwd<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,       \
                                 (int)smem_k1<N>());                                                \
        if (e) return e;                                                                            \
        e = cudaFuncSetAttribute(k_xpass<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,           \
                                 (int)smem_kx<N>());                                                \
        if (e) return e;                                                                            \
        e = cudaFuncSetAttribute(k_zpass_fwd_update<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,\
                                 (int)smem_k5<N>(g));                                               \
        if (e) return e;                                                                            \
    }
    PD_FOR_EACH_N(PD_CFG)
#undef PD_CFG
    return cudaSuccess;
}

cudaError_t launch_zpass_inv(const Geo& g, const Fields& f, int stage, cudaStream_t st) {
    switch (g.nz) {
#define PD_L(N)                                                                              \
    case N: {                                                                                \
        dim3 grid(g.nkip / Cfg<N>::L, g.nkj);                                                \
        k_zpass_inv<N><<<grid, NT, smem_k1<N>(), st>>>(f, g, stage);                         \
        break;                                                                               \
    }
        PD_FOR_EACH_N(PD_L)
#undef PD_L
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_ypass_inv(const Geo& g, const Fields& f, cudaStream_t st) {
    switch (g.ny) {
#define PD_L(N)                                                                              \
    case N: {                                                                                \
        dim3 grid(g.nkip / Cfg<N>::L, g.nz, 6);                                              \
        k_ypass_inv<N><<<grid, NT, smem_k1<N>(), st>>>(f, g);                                \
        break;                                                                               \
    }
        PD_FOR_EACH_N(PD_L)
#undef PD_L
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_xpass(const Geo& g, const Fields& f, int want_phys, int want_cfl, cudaStream_t st) {
    const long long lines = (long long)g.ny * g.nz;
    switch (g.nx) {
#define PD_L(N)                                                                              \
    case N: {                                                                                \
        const long long nb = (lines + Cfg<N>::LX - 1) / Cfg<N>::LX;                          \
        k_xpass<N><<<(unsigned)nb, NT, smem_kx<N>(), st>>>(f, g, want_phys, want_cfl);      \
        break;                                                                               \
    }
        PD_FOR_EACH_N(PD_L)
#undef PD_L
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_ypass_fwd(const Geo& g, const Fields& f, cudaStream_t st) {
    switch (g.ny) {
#define PD_L(N)                                                                              \
    case N: {                                                                                \
        dim3 grid(g.nkip / Cfg<N>::L, g.nz, 3);                                              \
        k_ypass_fwd<N><<<grid, NT, smem_k1<N>(), st>>>(f, g);                                \
        break;                                                                               \
    }
        PD_FOR_EACH_N(PD_L)
#undef PD_L
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_zpass_fwd_update(const Geo& g, const Fields& f, int stage, int mode, cudaStream_t st) {
    switch (g.nz) {
#define PD_L(N)                                                                              \
    case N: {                                                                                \
        dim3 grid((g.nki + Cfg<N>::L5 - 1) / Cfg<N>::L5, g.nkj);                             \
        k_zpass_fwd_update<N><<<grid, NT, smem_k5<N>(g), st>>>(f, g, stage, mode);           \
        break;                                                                               \
    }
        PD_FOR_EACH_N(PD_L)
#undef PD_L
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_stats(const Geo& g, const Fields& f, cudaStream_t st) {
    const size_t nsh = (size_t)2 * (g.kkmax + 1) + 3;
    cudaError_t e = cudaMemsetAsync(f.shell, 0, sizeof(double) * nsh, st);
    if (e) return e;
    long long nb = (g.S + 255) / 256;
    const long long cap = 4LL * sm_count();
    if (nb > cap) nb = cap;
    k_stats<<<(unsigned)nb, 256, sizeof(double) * nsh, st>>>(f, g);
    return cudaGetLastError();
}

cudaError_t launch_stage_scalars(const Geo& g, const Fields& f, const StepParams& sp, const ForceParams& fp,
                                 int stage, cudaStream_t st) {
    const size_t sm = sizeof(double) * 2 * (size_t)fp.calls_per_stage;
    k_stage_scalars<<<1, 256, sm, st>>>(f, g, sp, fp, stage);
    return cudaGetLastError();
}

cudaError_t launch_advance_time(const Fields& f, int stage, cudaStream_t st) {
    k_advance_time<<<1, 1, 0, st>>>(f, stage);
    return cudaGetLastError();
}

cudaError_t launch_init_fluid(const Geo& g, const Fields& f, const InitParams& ip, cudaStream_t st) {
    const long long total = (long long)(g.kj + 1) * (g.kk + 1) + (long long)g.ki * g.nkj * g.nkk;
    for (int c = 0; c < 3; c++) {
        cudaError_t e = cudaMemsetAsync(f.u[c], 0, sizeof(double2) * g.S, st);
        if (e) return e;
    }
    k_init_fluid<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(f, g, ip);
    return cudaGetLastError();
}

cudaError_t launch_check_finite(const Geo& g, const Fields& f, cudaStream_t st) {
    long long nb = (g.S + 255) / 256;
    const long long cap = 4LL * sm_count();
    if (nb > cap) nb = cap;
    k_check_finite<<<(unsigned)nb, 256, 0, st>>>(f, g);
    return cudaGetLastError();
}

}  // namespace pd
