// kernels_fluid.cu -- the small kernels around the five HBM passes of an RK3
// stage (kernels_passes.cu): statistics, dt and forcing scalars, time advance,
// seeded initial field, non-finite check.

#include <cuda_runtime.h>
#include <math.h>
#include <algorithm>
#include <atomic>
#include <type_traits>
#include "fft_core.cuh"
#include "pandora_internal.cuh"
#include "bfrot.cuh"

namespace pd {

using pdfft::mk;

// ---------------------------------------------------------------------------
// E(k), dissipation and Reynolds-stress sums, f_FluidstatsFsPrimaryQuants
// (src/pf_fluidstats.f90:1423-1576): per mode e = (phi11+phi22+phi33)/2 (x2 for
// i != 0), d = 2 k^2 nu e, binned in [kk-1/2, kk+1/2).  Raw sums; the host
// divides by the mode density.
// ---------------------------------------------------------------------------
size_t shell_words(const Geo& g) { return (size_t)3 * (g.kkmax + 1) + 3; }

// Compensated (Neumaier) accumulation: s + c carries the sum of the added terms
// to about one rounding, whatever their count and order of magnitude.
__device__ __forceinline__ void neumaier(double& s, double& c, double x) {
    const double t = s + x;
    c += (fabs(s) >= fabs(x)) ? ((s - t) + x) : ((x - t) + s);
    s = t;
}

// Shear flow: the same sums in the laboratory frame, k_lab = B^T k and
// u_lab = B^-1 u (f_FluidstatsFsPrimaryQuantsBFRot, src/pf_fluidstats.f90:1586-1960),
// with the per-shell mode counts of f_FluidstatsModeDensityBFRot
// (src/pf_fluidstats.f90:1977-2229), which change with B every step.
//
// Two launches.  k_stats: G CTAs of 8 warps, CTA b owning the contiguous rows
// [b R / G, (b+1) R / G) of (i, j), one warp per row, 32 consecutive k at a time.
// Along a row the shell index is monotone on each half of k, so the lanes of a shell
// form runs; a segmented sum over the runs (a fixed shuffle tree) leaves one
// shared-memory update per run.  Each CTA writes its sums to the free y-pencil
// buffer (G x nsh doubles).  k_stats_reduce adds the G partial sums of every output
// word in CTA order with Neumaier compensation: the cross-CTA sum, where the terms
// are many and of every size, carries about one rounding, and the result does not
// depend on the order in which CTAs finish.
template <class T, int CAP>
__global__ void __launch_bounds__(256) k_stats(const __grid_constant__ MemberSet<T, CAP> ms, int G) {
    const Member<T>& mm = ms.m[CAP == 1 ? 0 : blockIdx.y];
    if (!mm.active) return;
    if constexpr (CAP > 1) {   // a batch slot between members
        if (mm.F.clock->status & PD_ST_IDLE) return;
    }
    const FieldsT<T> F = mm.F;
    const Geo g = mm.g;
    extern __shared__ double sh[];
    const int K = g.kkmax;
    double* se = sh;                // [K+1]
    double* sd = sh + (K + 1);      // [K+1]
    double* sp = sh + 2 * (K + 1);  // [3]
    double* sc = sp + 3;            // [K+1] mode counts
    const int nsh = 3 * (K + 1) + 3;
    for (int q = threadIdx.x; q < nsh; q += blockDim.x) sh[q] = 0.0;
    __syncthreads();
    BF bf;
    if (g.shear) bf = make_bf(g, F.clock);
    double p11 = 0, p22 = 0, p33 = 0;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int NKK = g.nkk;
    const long long rows = (long long)g.nki * g.nkj;
    const long long r0 = rows * blockIdx.x / G, r1 = rows * (blockIdx.x + 1) / G;
    for (long long r = r0 + wib; r < r1; r += nw) {
        const int i = (int)(r / g.nkj), jj = (int)(r - (long long)i * g.nkj);
        const double k1 = (double)i, k2 = wvn(jj, g.kj);
        const double wgt = (i != 0) ? 2.0 : 1.0;
        for (int k0 = 0; k0 < NKK; k0 += 32) {
            const int k = k0 + lane;
            double e = 0.0, d = 0.0;
            int q = -1;   // shell, -1: none
            if (k < NKK) {
                const long long m = r * NKK + k;
                double kv[3] = {k1, k2, wvn(k, g.kk)};
                double2 uv[3] = {to_d(F.u[0][m]), to_d(F.u[1][m]), to_d(F.u[2][m])};
                if (g.shear) {
                    double kl[3] = {0.0, 0.0, 0.0};
                    double2 ul[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
#pragma unroll
                    for (int a = 0; a < 3; a++)
#pragma unroll
                        for (int b = 0; b < 3; b++)
                            if (bex(a, b)) {
                                kl[b] += bf.bm[a][b] * kv[a];
                                ul[a].x += bf.bi[a][b] * uv[b].x;
                                ul[a].y += bf.bi[a][b] * uv[b].y;
                            }
                    // R-rot holds laboratory components already (f_FluidstatsFsPrimaryQuantsRRot)
#pragma unroll
                    for (int a = 0; a < 3; a++) { kv[a] = kl[a]; if (!g.rrot) uv[a] = ul[a]; }
                }
                const double km = sqrt((kv[0] * kv[0]) + (kv[1] * kv[1]) + (kv[2] * kv[2]));
                double q11 = uv[0].x * uv[0].x + uv[0].y * uv[0].y, q22 = uv[1].x * uv[1].x + uv[1].y * uv[1].y;
                double q33 = uv[2].x * uv[2].x + uv[2].y * uv[2].y;
                if (i != 0) { q11 *= 2.0; q22 *= 2.0; q33 *= 2.0; }
                p11 += q11; p22 += q22; p33 += q33;
                e = 0.5 * (q11 + q22 + q33);
                if (!isfinite(e)) atomicOr(&F.clock->status, PD_ST_NAN);
                d = 2.0 * km * km * g.nu * e;
                // bin [q - 1/2, q + 1/2), q = 1..K
                int qc = (int)floor(km + 0.5);
                if (km < (double)qc - 0.5) qc--;
                else if (km >= (double)qc + 0.5) qc++;
                if (qc >= 1 && qc <= K) q = qc;
            }
            // runs of equal q in lane order: start lane of this lane's run
            const int prevq = __shfl_up_sync(0xffffffffu, q, 1);
            int start = (lane == 0 || prevq != q) ? lane : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) start = max(start, __shfl_up_sync(0xffffffffu, start, o));
            double c = (q >= 0) ? wgt : 0.0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const double e2 = __shfl_up_sync(0xffffffffu, e, o), d2 = __shfl_up_sync(0xffffffffu, d, o);
                const double c2 = __shfl_up_sync(0xffffffffu, c, o);
                if (lane - o >= start) { e += e2; d += d2; c += c2; }
            }
            const int nextq = __shfl_down_sync(0xffffffffu, q, 1);
            if (((lane == 31) || (nextq != q)) && q >= 1) {
                atomicAdd(&se[q], e);
                atomicAdd(&sd[q], d);
                if (g.shear) atomicAdd(&sc[q], c);
            }
        }
    }
    // the three second moments: summed within each warp, then the warps' sums added in warp
    // order by one thread (not 256 atomics on the same three shared words)
    __shared__ double wp[8][3];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        p11 += __shfl_xor_sync(0xffffffffu, p11, o);
        p22 += __shfl_xor_sync(0xffffffffu, p22, o);
        p33 += __shfl_xor_sync(0xffffffffu, p33, o);
    }
    if (lane == 0) { wp[wib][0] = p11; wp[wib][1] = p22; wp[wib][2] = p33; }
    __syncthreads();
    if (threadIdx.x < 3) {
        double a = 0.0;
        for (int v = 0; v < nw; v++) a += wp[v][threadIdx.x];
        sp[threadIdx.x] = a;
    }
    __syncthreads();
    double* part = reinterpret_cast<double*>(F.yb) + (size_t)blockIdx.x * nsh;
    for (int q = threadIdx.x; q < nsh; q += blockDim.x) part[q] = sh[q];
}

// One CTA per 32 output words: lane l of warp v adds, compensated, the partials of
// word w0 + l from CTAs v, v + 8, v + 16, ...; the 8 pairs of a word then fold in warp
// order.
template <class T, int CAP>
__global__ void __launch_bounds__(256) k_stats_reduce(const __grid_constant__ MemberSet<T, CAP> ms, int G) {
    const Member<T>& mm = ms.m[CAP == 1 ? 0 : blockIdx.y];
    if (!mm.active) return;
    if constexpr (CAP > 1) {   // a batch slot between members
        if (mm.F.clock->status & PD_ST_IDLE) return;
    }
    const FieldsT<T> F = mm.F;
    const int nsh = 3 * (mm.g.kkmax + 1) + 3;
    __shared__ double ps[8][32], pc[8][32];
    const int lane = threadIdx.x & 31, v = threadIdx.x >> 5;
    const int w = blockIdx.x * 32 + lane;
    const double* part = reinterpret_cast<const double*>(F.yb);
    double s = 0.0, c = 0.0;
    if (w < nsh)
        for (int b = v; b < G; b += 8) neumaier(s, c, part[(size_t)b * nsh + w]);
    ps[v][lane] = s;
    pc[v][lane] = c;
    __syncthreads();
    if (v == 0 && w < nsh) {
        double S = 0.0, Cc = 0.0;
        for (int u = 0; u < 8; u++) { neumaier(S, Cc, ps[u][lane]); Cc += pc[u][lane]; }
        F.shell[w] = S + Cc;
    }
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

template <class T, int CAP>
__global__ void __launch_bounds__(256) k_stage_scalars(const __grid_constant__ MemberSet<T, CAP> ms, int stage) {
    const Member<T>& mm = ms.m[CAP == 1 ? 0 : blockIdx.x];
    if (!mm.active) return;
    if constexpr (CAP > 1) {   // a batch slot between members
        if (mm.F.clock->status & PD_ST_IDLE) return;
    }
    const FieldsT<T> F = mm.F;
    const Geo g = mm.g;
    const StepParams sp = mm.sp;
    const ForceParams fp = mm.fp;
    extern __shared__ double nrm[];   // [2 * calls] normal pairs, then the i = 0 plane [3][FW][FW]
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
    const double dt_over_TF = ck->dt / fp.tf;
    const double amp = sqrt(2.0 * (fp.sigma * fp.sigma) * dt_over_TF);
    const double decay = 1.0 - dt_over_TF;
    double2* ff = F.forcing;
    const int plane = FW * FW;
    // Modes i >= 1 take normal pairs c0 + 3q.. in the order i, jw, kw (all from -NK):
    // independent of each other, updated in parallel.
    const long long c0 = 3LL * (NK + 1) * (2 * NK + 1);
    for (int q = tid; q < NK * plane; q += blockDim.x) {
        const long long m = (long long)plane + q;   // (i*FW + jw+NK)*FW + kw+NK with i >= 1
        const long long c = c0 + 3LL * q;
#pragma unroll
        for (int comp = 0; comp < 3; comp++) {
            double2& v = ff[comp * fstride + m];
            v = mk(v.x * decay + nrm[2 * (c + comp)] * amp, v.y * decay + nrm[2 * (c + comp) + 1] * amp);
        }
    }
    // The i = 0 plane: the OU update of the half jw >= 0 (and jw < 0 for kw >= 0)
    // interleaved with conjugate copies that later steps overwrite again, so it
    // runs in its original order, on a shared-memory copy of the plane.
    double2* pl = (double2*)(nrm + 2 * calls);   // [3][FW][FW]
    for (int q = tid; q < 3 * plane; q += blockDim.x) pl[q] = ff[(q / plane) * fstride + q % plane];
    __syncthreads();
    if (tid == 0) {
        long long c = 0;
        auto at = [&](int comp, int jw, int kw) -> double2& { return pl[comp * plane + (jw + NK) * FW + (kw + NK)]; };
        auto ou = [&](int jw, int kw) {
            for (int comp = 0; comp < 3; comp++) {
                double2& v = at(comp, jw, kw);
                const double re = nrm[2 * (c + comp)], im = nrm[2 * (c + comp) + 1];
                v = mk(v.x * decay + re * amp, v.y * decay + im * amp);
            }
            c += 3;
        };
        auto conj_copy = [&](int jd, int kd, int js, int ks) {
            for (int comp = 0; comp < 3; comp++) {
                const double2 sv = at(comp, js, ks);
                at(comp, jd, kd) = mk(sv.x, -sv.y);
            }
        };
        for (int jw = 0; jw <= NK; jw++)
            for (int kw = 0; kw <= NK; kw++) {
                ou(jw, kw);
                conj_copy(-jw, -kw, jw, kw);
                if (jw > 0) {
                    ou(-jw, kw);
                    conj_copy(jw, -kw, -jw, kw);
                }
            }
    }
    __syncthreads();
    for (int q = tid; q < 3 * plane; q += blockDim.x) ff[(q / plane) * fstride + q % plane] = pl[q];
}

// simtime after stage s: t0 + {1/3, 3/4, 1} dt (src/pg_rk3.f90:109-127); the step
// counter advances after stage 3.
template <class T, int CAP>
__global__ void k_advance_time(const __grid_constant__ MemberSet<T, CAP> ms, int stage) {
    const Member<T>& mm = ms.m[CAP == 1 ? 0 : blockIdx.x];
    if (!mm.active) return;
    if constexpr (CAP > 1) {   // a batch slot between members
        if (mm.F.clock->status & PD_ST_IDLE) return;
    }
    const FieldsT<T> F = mm.F;
    const Geo g = mm.g;

    Clock* ck = F.clock;
    if (stage == 1) ck->simtime = ck->t0 + (1.0 / 3.0) * ck->dt;
    else if (stage == 2) ck->simtime = ck->t0 + (3.0 / 4.0) * ck->dt;
    else ck->simtime = ck->t0 + ck->dt;
    if (g.shear) update_b(g, ck->tstep, ck->simtime, ck->b13, ck->bi13);
    if (stage == 3) {
        ck->t0 = ck->simtime;
        ck->tstep += 1;
    }
}

// A fresh clock (step tstep at time t, frame tensors b13 / bi13), set on the
// device in stream order with the values as launch parameters.
__global__ void k_reset_clock(Clock* ck, int tstep, double t, double b13, double bi13) {
    Clock c{};
    c.tstep = tstep;
    c.simtime = t;
    c.t0 = t;
    c.b13 = b13;
    c.bi13 = bi13;
    *ck = c;
}
cudaError_t launch_reset_clock(Clock* ck, int tstep, double t, double b13, double bi13, cudaStream_t st) {
    k_reset_clock<<<1, 1, 0, st>>>(ck, tstep, t, b13, bi13);
    return cudaGetLastError();
}
// Marks a batch slot free (batched kernels skip it from the next launch on).
__global__ void k_set_idle(Clock* ck) { ck->status |= PD_ST_IDLE; }
cudaError_t launch_set_idle(Clock* ck, cudaStream_t st) {
    k_set_idle<<<1, 1, 0, st>>>(ck);
    return cudaGetLastError();
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
                             double r2, double r3, double2 t[3], double fdiv) {
    const double twopi = 6.283185307179586476925286766559005768;
    const double fourpi = 12.566370614359172953850573533118011536;
    r1 = twopi * r1; r2 = twopi * r2; r3 = twopi * r3;
    const double k2d = (k1 * k1) + (k2 * k2);
    t[0] = t[1] = t[2] = mk(0.0, 0.0);
    if (!(kmag > 0.0)) return;
    const double ek = init_spec(p, kmag);
    double factor = sqrt(ek / (fourpi * kmag * kmag));
    if (fdiv != 1.0) factor = factor / fdiv;
    const double2 al = mk(factor * cos(r1) * cos(r3), factor * sin(r1) * cos(r3));
    const double2 be = mk(factor * cos(r2) * sin(r3), factor * sin(r2) * sin(r3));
    if (!(k2d > 0.0)) return;
    const double den = kmag * sqrt(k2d);
    t[0] = mk((al.x * kmag * k2 + be.x * k1 * k3) / den, (al.y * kmag * k2 + be.y * k1 * k3) / den);
    t[1] = mk((be.x * k2 * k3 - al.x * kmag * k1) / den, (be.y * k2 * k3 - al.y * kmag * k1) / den);
    t[2] = mk(-(be.x * sqrt(k2d)) / kmag, -(be.y * sqrt(k2d)) / kmag);
}

// Deformed grid (f_InitialiseFluidDeformed, src/pf_initialise.f90:520-990): the
// construction above in laboratory wavenumbers k/B, amplitude divided by
// (B110 B220 B330)^(1/2), velocity mapped by bmat (diagonal at t = 0).
__device__ __forceinline__ void deform_map(const Geo& g, double2 t[3]) {
    for (int c = 0; c < 3; c++) t[c] = mk(g.bdiag[c] * t[c].x, g.bdiag[c] * t[c].y);
}

__global__ void k_init_fluid(Fields F, Geo g, InitParams ip) {
    const int KJ = g.kj, KK = g.kk, NKJ = g.nkj, NKK = g.nkk;
    const long long plane0 = (long long)(KJ + 1) * (KK + 1);
    const long long rest = (long long)g.ki * NKJ * NKK;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const double b1 = ip.deformed ? (double)ip.b110 : 1.0, b2 = ip.deformed ? (double)ip.b220 : 1.0;
    const double b3 = ip.deformed ? (double)ip.b330 : 1.0;
    const double fdiv = ip.deformed ? pow((double)ip.b110 * (double)ip.b220 * (double)ip.b330, 0.5) : 1.0;
    auto U = [&](int c, int i, int j, int k) -> double2& {
        return F.u[c][((long long)i * NKJ + j) * NKK + k];
    };
    if (idx < plane0) {
        const int j = (int)(idx / (KK + 1)), k = (int)(idx % (KK + 1));
        const uint64_t n = (uint64_t)j * 3 * (2 * KK + 1) + (k == 0 ? 0 : 3 + 6 * (uint64_t)(k - 1));
        const double k1 = 0.0 / b1, k2 = wvn(j, KJ) / b2, k3 = wvn(k, KK) / b3;
        const double kmag = sqrt((k1 * k1) + (k2 * k2) + (k3 * k3));
        double2 t[3];
        rogallo_mode(ip, k1, k2, k3, kmag, uniform(ip.key, n), uniform(ip.key, n + 1), uniform(ip.key, n + 2), t,
                     fdiv);
        if (ip.deformed) deform_map(g, t);
        const int jj = (j != 0) ? NKJ - j : j, kk = (k != 0) ? NKK - k : k;
        for (int c = 0; c < 3; c++) U(c, 0, j, k) = t[c];
        for (int c = 0; c < 3; c++) U(c, 0, jj, kk) = mk(t[c].x, -t[c].y);
        if (k != 0) {
            double k2n = wvn(jj, KJ);
            if (ip.deformed || ip.b220 > 1) k2n = k2n / (double)ip.b220;
            rogallo_mode(ip, k1, k2n, k3, kmag, uniform(ip.key, n + 3), uniform(ip.key, n + 4),
                         uniform(ip.key, n + 5), t, fdiv);
            if (ip.deformed) deform_map(g, t);
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
    const double a = (double)i / b1, b = wvn(j, KJ) / b2, c3 = wvn(k, KK) / b3;
    const double kmag = sqrt((a * a) + (b * b) + (c3 * c3));
    double2 t[3];
    rogallo_mode(ip, a, b, c3, kmag, uniform(ip.key, n), uniform(ip.key, n + 1), uniform(ip.key, n + 2), t, fdiv);
    if (ip.deformed) deform_map(g, t);
    for (int c = 0; c < 3; c++) U(c, i, j, k) = t[c];
}

// Wave-space remesh at stage 1 of a remesh step (f_RK3Remesh / f_RK3RemeshWaveSpace,
// src/pf_rk3.f90:3958-4178): per (i,j) row k3 <- k3 - k1, modes below -KK
// dropped, BF-rot u1 += u3; the frame jumps from S t = +B110/2 to -B110/2.  The
// step number is read on the device, so the launch sits in every step's graph
// and returns at once on the other steps.  One CTA per row, row staged in shared memory.
template <class T, int CAP>
__global__ void __launch_bounds__(256) k_remesh(const __grid_constant__ MemberSet<T, CAP> ms) {
    const Member<T>& mm = ms.m[CAP == 1 ? 0 : blockIdx.y];
    if (!mm.active) return;
    if constexpr (CAP > 1) {   // a batch slot between members
        if (mm.F.clock->status & PD_ST_IDLE) return;
    }
    const FieldsT<T> F = mm.F;
    const Geo g = mm.g;

    using C = typename FieldsT<T>::C;
    Clock* ck = F.clock;
    if (!remesh_due(g, ck->tstep)) return;
    extern __shared__ double2 rowbuf[];   // [3][NKK]
    const long long ij = blockIdx.x;
    const int i = (int)(ij / g.nkj), jj = (int)(ij - (long long)i * g.nkj);
    const int KK = g.kk, NKK = g.nkk, nodes = 2 * KK + 1;
    // DEALIASING 2/3: modes outside the cutoff are dropped in the frame before the
    // remesh and again in the frame after it (src/pf_rk3.f90:3999-4025); the frame
    // itself is reset by k_remesh_frame after this kernel
    const bool dealias = g.dealias_cut > 0.0;
    BF fold, fnew;
    if (dealias) {
        fold = make_bf(g, ck);
        fnew = fold;
        fnew.bm[0][2] = -g.bdiag[0] * (-(double)g.b110 * 0.5);
    }
    const double k1 = (double)i, k2 = wvn(jj, g.kj);
    for (int q = threadIdx.x; q < 3 * NKK; q += blockDim.x) rowbuf[q] = mk(0.0, 0.0);
    __syncthreads();
    for (int k = threadIdx.x; k < NKK; k += blockDim.x) {
        const int actualk = k > KK ? k - nodes : k;
        int knew = actualk - i;
        if (knew >= -KK) {
            if (knew < 0) knew += nodes;
            const bool drop = dealias && dealias_drop(g, fold, k1, k2, (double)actualk);
            for (int c = 0; c < 3; c++)
                rowbuf[c * NKK + knew] = drop ? mk(0.0, 0.0) : to_d(F.u[c][ij * NKK + k]);
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < NKK; k += blockDim.x) {
        const double2 a = rowbuf[k], b3 = rowbuf[2 * NKK + k];
        if (dealias && dealias_drop(g, fnew, k1, k2, wvn(k, KK))) {
            for (int c = 0; c < 3; c++) F.u[c][ij * NKK + k] = from_d<C>(mk(0.0, 0.0));
            continue;
        }
        // BF-rot: u1 += u3; R-rot keeps the components (src/pf_rk3.f90:4150-4162)
        F.u[0][ij * NKK + k] = from_d<C>(g.rrot ? a : mk(a.x + b3.x, a.y + b3.y));
        F.u[1][ij * NKK + k] = from_d<C>(rowbuf[NKK + k]);
        F.u[2][ij * NKK + k] = from_d<C>(b3);
    }
}

// The frame jump of the remesh (bmat/binv (1,3) to S t = -B110/2), after k_remesh:
// every CTA of k_remesh reads the frame from before the remesh.
template <class T, int CAP>
__global__ void k_remesh_frame(const __grid_constant__ MemberSet<T, CAP> ms) {
    const Member<T>& mm = ms.m[CAP == 1 ? 0 : blockIdx.x];
    if (!mm.active) return;
    Clock* ck = mm.F.clock;
    if constexpr (CAP > 1) {
        if (ck->status & PD_ST_IDLE) return;
    }
    const Geo& g = mm.g;
    if (!remesh_due(g, ck->tstep)) return;
    const double half_b = (double)g.b110 * 0.5;
    ck->b13 = -g.bdiag[0] * (-half_b);
    ck->bi13 = (-half_b) / g.bdiag[2];
}

// DEALIASING 2/3 applied to the state in place (after the initial field,
// src/pf_initialise.f90:75-83).
template <class T, int CAP>
__global__ void k_dealias(const __grid_constant__ MemberSet<T, CAP> ms) {
    const Member<T>& mm = ms.m[CAP == 1 ? 0 : blockIdx.y];
    if (!mm.active) return;
    const FieldsT<T> F = mm.F;
    const Geo g = mm.g;
    using C = typename FieldsT<T>::C;
    const BF bf = make_bf(g, F.clock);
    for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < g.S; m += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(m % g.nkk);
        const long long ij = m / g.nkk;
        const int j = (int)(ij % g.nkj), i = (int)(ij / g.nkj);
        if (dealias_drop(g, bf, (double)i, wvn(j, g.kj), wvn(k, g.kk)))
            for (int c = 0; c < 3; c++) F.u[c][m] = C{};
    }
}

// Particle positions at the remesh (p_MPIRemeshPosition, src/pp_mpi.f90:1062-1092).
template <class T, int CAP>
__global__ void k_remesh_particles(const __grid_constant__ MemberSet<T, CAP> ms) {
    const Member<T>& mm = ms.m[CAP == 1 ? 0 : blockIdx.y];
    if (!mm.active) return;
    if constexpr (CAP > 1) {   // a batch slot between members
        if (mm.F.clock->status & PD_ST_IDLE) return;
    }
    const Particles P = mm.P;
    const Geo g = mm.g;
    const Clock* ck = mm.F.clock;
    if (!remesh_due(g, ck->tstep)) return;
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= P.np) return;
    const double x1min = -0.5 * g.dx, x1max = x1min + g.lx;
    double x = P.xp[0][n] + P.xp[2][n];
    if (x < x1min) x = x + g.lx;
    if (x >= x1max) x = x - g.lx;
    P.xp[0][n] = x;
}

// np: particles per member (0: none)
#define PD_CAP(S) std::decay_t<decltype(S)>::cap
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

template <class T>
cudaError_t launch_remesh(const Geo& g, const Member<T>* M, int B, long long np, cudaStream_t st) {
    return for_member_sets(M, B, [&](const auto& ms, int nb) {
        constexpr int CAP = PD_CAP(ms);
        if (np > 0) k_remesh_particles<T, CAP><<<dim3((unsigned)((np + 255) / 256), nb), 256, 0, st>>>(ms);
        k_remesh<T, CAP><<<dim3((unsigned)((long long)g.nki * g.nkj), nb), 256, sizeof(double2) * 3 * g.nkk, st>>>(ms);
        k_remesh_frame<T, CAP><<<nb, 1, 0, st>>>(ms);
    });
}

template <class T>
cudaError_t launch_dealias(const Geo& g, const Member<T>* M, int B, cudaStream_t st) {
    if (!(g.dealias_cut > 0.0)) return cudaSuccess;
    long long nb = (g.S + 255) / 256;
    if (nb > 4LL * sm_count()) nb = 4LL * sm_count();
    return for_member_sets(M, B, [&](const auto& ms, int nm) {
        k_dealias<T, PD_CAP(ms)><<<dim3((unsigned)nb, nm), 256, 0, st>>>(ms);
    });
}

// Non-finite check of the spectral state (sets PD_ST_NAN).
template <class T, int CAP>
__global__ void k_check_finite(const __grid_constant__ MemberSet<T, CAP> ms) {
    const Member<T>& mm = ms.m[CAP == 1 ? 0 : blockIdx.y];
    if (!mm.active) return;
    if constexpr (CAP > 1) {   // a batch slot between members
        if (mm.F.clock->status & PD_ST_IDLE) return;
    }
    const FieldsT<T> F = mm.F;
    const Geo g = mm.g;

    bool bad = false;
    for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < g.S;
         m += (long long)gridDim.x * blockDim.x) {
        for (int c = 0; c < 3; c++) {
            const double2 v = to_d(F.u[c][m]);
            if (!isfinite(v.x) || !isfinite(v.y)) bad = true;
        }
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(&F.clock->status, PD_ST_NAN);
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------

// Statistics of every member into its own F.shell (shell_words doubles); the
// per-CTA partial sums live in the member's y-pencil buffer, free at stage 1 and
// between steps.
template <class T>
cudaError_t launch_stats(const Geo& g, const Member<T>* M, int B, double* shell, cudaStream_t st) {
    (void)shell;
    const size_t nsh = shell_words(g);
    const long long rows = (long long)g.nki * g.nkj;
    const size_t yb_bytes = sizeof(typename Cplx<T>::type) * 6 * (size_t)g.nz * g.ny * g.nkip;
    long long G = std::min<long long>(4LL * sm_count(), std::max<long long>(1, rows / 8));
    G = std::min<long long>(G, (long long)(yb_bytes / (sizeof(double) * nsh)));
    if (G < 1) return cudaErrorInvalidValue;
    const int gi = (int)G;
    cudaError_t e = for_member_sets(M, B, [&](const auto& ms, int nm) {
        k_stats<T, PD_CAP(ms)><<<dim3((unsigned)gi, nm), 256, sizeof(double) * nsh, st>>>(ms, gi);
    });
    if (e) return e;
    return for_member_sets(M, B, [&](const auto& ms, int nm) {
        k_stats_reduce<T, PD_CAP(ms)><<<dim3((unsigned)((nsh + 31) / 32), nm), 256, 0, st>>>(ms, gi);
    });
}

// Shared memory of k_stage_scalars: the normal pairs of one stage, then the i = 0
// forcing plane (about 132 KB at the largest forcing radius, FORCE_KF = 8).
static size_t stage_scalars_smem(const Geo& g, const ForceParams& fp) {
    const int fw = 2 * g.fnk + 1;
    return sizeof(double) * 2 * (size_t)fp.calls_per_stage + sizeof(double2) * 3 * (size_t)fw * fw;
}

// The dynamic shared memory limits only ever grow: the attribute is per function for
// the whole process, and handles of several geometries live side by side.
template <typename K> static cudaError_t raise_smem(K kernel, int bytes, std::atomic<int>& have) {
    int cur = have.load();
    if (bytes <= cur) return cudaSuccess;
    const cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess)
        while (cur < bytes && !have.compare_exchange_weak(cur, bytes)) {}
    return e;
}

cudaError_t configure_fluid_kernels(const Geo& g, const ForceParams& fp) {
    static std::atomic<int> ss[4], st[4];   // zero-initialised (static storage)
    const int b = (int)stage_scalars_smem(g, fp);
    const int bs = (int)(sizeof(double) * shell_words(g));   // statistics' shell sums
    cudaError_t e;
    if ((e = raise_smem(k_stage_scalars<double, 1>, b, ss[0])) || (e = raise_smem(k_stage_scalars<float, 1>, b, ss[1])) ||
        (e = raise_smem(k_stage_scalars<double, kBatchChunk>, b, ss[2])) ||
        (e = raise_smem(k_stage_scalars<float, kBatchChunk>, b, ss[3])) || (e = raise_smem(k_stats<double, 1>, bs, st[0])) ||
        (e = raise_smem(k_stats<float, 1>, bs, st[1])) || (e = raise_smem(k_stats<double, kBatchChunk>, bs, st[2])))
        return e;
    return raise_smem(k_stats<float, kBatchChunk>, bs, st[3]);
}

template <class T>
cudaError_t launch_stage_scalars(const Geo& g, const Member<T>* M, int B, const ForceParams& fp, int stage,
                                 cudaStream_t st) {
    return for_member_sets(M, B, [&](const auto& ms, int nm) {
        k_stage_scalars<T, PD_CAP(ms)><<<nm, 256, stage_scalars_smem(g, fp), st>>>(ms, stage);
    });
}

template <class T>
cudaError_t launch_advance_time(const Geo& g, const Member<T>* M, int B, int stage, cudaStream_t st) {
    return for_member_sets(M, B, [&](const auto& ms, int nm) {
        k_advance_time<T, PD_CAP(ms)><<<nm, 1, 0, st>>>(ms, stage);
    });
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

template <class T> cudaError_t launch_check_finite(const Geo& g, const Member<T>* M, int B, cudaStream_t st) {
    long long nb = (g.S + 255) / 256;
    const long long cap = 4LL * sm_count();
    if (nb > cap) nb = cap;
    return for_member_sets(M, B, [&](const auto& ms, int nm) {
        k_check_finite<T, PD_CAP(ms)><<<dim3((unsigned)nb, nm), 256, 0, st>>>(ms);
    });
}

#undef PD_CAP

// TS_CORR's longitudinal autocorrelation (f_FluidstatsRs2D, src/pf_fluidstats.f90:933-945)
// in wave space.  The sum over the grid of a(x) b(x + l dx) is N^3 sum_k a^(k) conj(b^(k))
// e^{-2 pi i m l / NX} over the full spectrum, so per x wavenumber m the co-spectrum
// P_m = sum_{j,k} a^ conj(b^) of a = u1 in the laboratory frame (binv u for shear, as
// the reference's real-space statistics take it) and b = the stored u1 carries all of
// it; the modes DEALIASING 2/3 drops are left out, as the real-space field holds none.
// One CTA per m plane with a fixed-order block sum: P[2m], P[2m+1] = Re, Im.
template <class T>
__global__ void __launch_bounds__(256) k_xcorr_cospec(const __grid_constant__ MemberSet<T, 1> ms, double* P) {
    const FieldsT<T> F = ms.m[0].F;
    const Geo g = ms.m[0].g;
    const BF bf = make_bf(g, F.clock);
    const bool dealias = g.dealias_cut > 0.0;
    const int i = blockIdx.x;
    const long long plane = (long long)g.nkj * g.nkk, base = (long long)i * plane;
    double re = 0.0, im = 0.0;
    for (long long q = threadIdx.x; q < plane; q += blockDim.x) {
        const int j = (int)(q / g.nkk), k = (int)(q % g.nkk);
        if (dealias && dealias_drop(g, bf, (double)i, wvn(j, g.kj), wvn(k, g.kk))) continue;
        const double2 b = to_d(F.u[0][base + q]);
        double2 a = b;
        if (g.shear) {
            const double2 u3 = to_d(F.u[2][base + q]);
            a = make_double2(bf.bi[0][0] * b.x + bf.bi[0][2] * u3.x, bf.bi[0][0] * b.y + bf.bi[0][2] * u3.y);
        }
        re += a.x * b.x + a.y * b.y;
        im += a.y * b.x - a.x * b.y;
    }
    __shared__ double sr[8], si[8];
    for (int o = 16; o > 0; o >>= 1) {
        re += __shfl_xor_sync(0xffffffffu, re, o);
        im += __shfl_xor_sync(0xffffffffu, im, o);
    }
    if ((threadIdx.x & 31) == 0) { sr[threadIdx.x >> 5] = re; si[threadIdx.x >> 5] = im; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double tr = 0.0, ti = 0.0;
        for (int w = 0; w < 8; w++) { tr += sr[w]; ti += si[w]; }
        P[2 * i] = tr;
        P[2 * i + 1] = ti;
    }
}

template <class T> cudaError_t launch_xcorr_cospec(const Member<T>& m, double* P, cudaStream_t st) {
    MemberSet<T, 1> one;
    one.m[0] = m;
    k_xcorr_cospec<T><<<(unsigned)m.g.nki, 256, 0, st>>>(one, P);
    return cudaGetLastError();
}

#define PD_INST(T)                                                                                   \
    template cudaError_t launch_xcorr_cospec<T>(const Member<T>&, double*, cudaStream_t);            \
    template cudaError_t launch_stats<T>(const Geo&, const Member<T>*, int, double*, cudaStream_t);  \
    template cudaError_t launch_stage_scalars<T>(const Geo&, const Member<T>*, int, const ForceParams&, int, \
                                                 cudaStream_t);                                      \
    template cudaError_t launch_advance_time<T>(const Geo&, const Member<T>*, int, int, cudaStream_t); \
    template cudaError_t launch_check_finite<T>(const Geo&, const Member<T>*, int, cudaStream_t);    \
    template cudaError_t launch_remesh<T>(const Geo&, const Member<T>*, int, long long, cudaStream_t);  \
    template cudaError_t launch_dealias<T>(const Geo&, const Member<T>*, int, cudaStream_t);
PD_INST(double)
PD_INST(float)
#undef PD_INST

}  // namespace pd
