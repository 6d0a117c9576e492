// kernels_particles.cu -- Lagrangian particle advance on sm_100a.
//
// One thread per particle: tensor-product Lagrange interpolation of order ORD
// of the physical velocity of the current stage (the reference evaluates the
// same polynomial by Neville's scheme, p_InterpInterpolate3D / FindMolecule /
// Neville3D, src/pp_interp.f90:313-560), the tracer or Stokes-drag RK3 update
// (p_RK3SolveParticle, src/pp_rk3.f90:57-165, drag 927-946) and the periodic
// wrap (p_MPICorrectPosition, src/pp_mpi.f90:1011-1057; x3 uses '>' where x1
// and x2 use '>=').  The reference fetches a halo of NHALO = order/2 planes by
// DMGlobalToLocal (src/pp_interp.f90:115-264); on one GPU the stencil indices
// wrap modulo N.  Physical velocity layout: [c][z][y][x].
//
// Particles are kept sorted by spatial bin (z slowest), re-sorted once per step,
// so that a wave of threads reads a compact set of velocity rows that stays in
// L2 instead of gathering at random from a field larger than L2.
#include <cuda_runtime.h>
#include <algorithm>
#include <type_traits>
#include "pandora_internal.cuh"
#include "bfrot.cuh"

namespace pd {

constexpr int kMaxOrder = 6;

// Lagrange basis weight m at x over the ORD nodes: prod_{n != m} (x - x_n) / (x_m - x_n),
// formed as one quotient of the two products (one FP64 division per weight).
template <int ORD>
__device__ __forceinline__ double lagrange_weight(double x, const double* nodes, int m) {
    double xm = nodes[0];
#pragma unroll
    for (int n = 1; n < ORD; n++)
        if (n == m) xm = nodes[n];   // m may be a run-time value: select, do not index
    double num = 1.0, den = 1.0;
#pragma unroll
    for (int n = 0; n < ORD; n++)
        if (n != m) { num *= x - nodes[n]; den *= xm - nodes[n]; }
    return num / den;
}

// G threads per particle (G = the power of two at or above ORD): thread `sub` of a
// group gathers the stencil column x = i0 + sub (threads sub >= ORD add nothing),
// so one warp load touches 32/G particles' rows of consecutive values instead of
// 32 scattered rows; the group sums its partial results with shuffles and its
// first thread does the update.
template <int ORD> constexpr int part_group() { return ORD <= 1 ? 1 : (ORD <= 2 ? 2 : (ORD <= 4 ? 4 : 8)); }

// T: precision of the stored physical velocity (the particle state and its
// arithmetic are FP64 in both forms).
template <int ORD, class T, int CAP>
__global__ void __launch_bounds__(256, 2) k_particles(const __grid_constant__ MemberSet<T, CAP> ms, int stage) {
    constexpr int G = part_group<ORD>();
    const Member<T>& mm = ms.m[CAP == 1 ? 0 : blockIdx.y];
    if (!mm.active) return;
    if constexpr (CAP > 1) {   // a batch slot between members
        if (mm.F.clock->status & PD_ST_IDLE) return;
    }                             // uniform over the CTA
    const Particles P = mm.P;
    const Geo g = mm.g;
    const T* __restrict__ phys = mm.F.phys;
    Clock* ck = mm.F.clock;
    const PartParams pp = mm.pp;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long n = t / G;
    const int sub = (int)(t % G);
    const int tstep = ck->tstep;
    if (tstep < pp.release) return;                     // uniform over the member
    if (G == 1 && n >= P.np) return;
    // With G > 1 every lane of a warp reaches the shuffles: lanes past the last
    // particle (whole groups at the tail) gather for the last particle and store nothing.
    const bool valid = n < P.np;
    const long long nn = valid ? n : P.np - 1;
    const double dt = ck->dt;
    double beta, gamma;
    if (stage == 1) { beta = 0.0; gamma = 1.0 / 3.0; }
    else if (stage == 2) { beta = -(5.0 / 9.0); gamma = 15.0 / 16.0; }
    else { beta = -(153.0 / 128.0); gamma = 8.0 / 15.0; }
    constexpr int nh = ORD / 2;
    const double D[3] = {g.dx, g.dy, g.dz};
    const int NN[3] = {g.nx, g.ny, g.nz};
    double xp[3];
#pragma unroll
    for (int c = 0; c < 3; c++) xp[c] = P.xp[c][nn];
    // p_InterpFindMolecule: stencil start from the same rounded arithmetic
    double w[3][ORD];
    int idx[3][ORD];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        double halo = __dmul_rn((double)nh, D[c]);
        double xd;
        if ((ORD & 1) == 0) {
            halo = __dsub_rn(halo, __dmul_rn(0.5, D[c]));
            xd = __dadd_rn(__dadd_rn(__dadd_rn(xp[c], halo), D[c]), __dmul_rn(0.5, D[c]));
        } else {
            xd = __dadd_rn(__dadd_rn(xp[c], halo), __dmul_rn(0.5, D[c]));
        }
        const int i0 = (int)__ddiv_rn(xd, D[c]) - nh - nh;
        double nodes[ORD];
#pragma unroll
        for (int m = 0; m < ORD; m++) {
            nodes[m] = __dmul_rn((double)(i0 + m), D[c]);
            int q = (i0 + m) % NN[c];
            idx[c][m] = q < 0 ? q + NN[c] : q;
        }
        if constexpr (G == 1) {
#pragma unroll
            for (int m = 0; m < ORD; m++) w[c][m] = lagrange_weight<ORD>(xp[c], nodes, m);
        } else {
            // each thread of the group forms the weight of its own offset; the
            // group exchanges them (lanes of a group are consecutive)
            const double mine = lagrange_weight<ORD>(xp[c], nodes, sub < ORD ? sub : ORD - 1);
            const int base = (threadIdx.x & 31) & ~(G - 1);
#pragma unroll
            for (int m = 0; m < ORD; m++) w[c][m] = __shfl_sync(0xffffffffu, mine, base + m);
        }
    }
    double uf[3];
    if constexpr (G == 1) {
        long long rowoff[ORD][ORD];
#pragma unroll
        for (int zi = 0; zi < ORD; zi++)
#pragma unroll
            for (int yi = 0; yi < ORD; yi++) rowoff[zi][yi] = ((long long)idx[2][zi] * g.ny + idx[1][yi]) * g.nx;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const T* f = phys + (long long)c * g.R;
            double acc_z = 0.0;
#pragma unroll
            for (int zi = 0; zi < ORD; zi++) {
                double acc_y = 0.0;
#pragma unroll
                for (int yi = 0; yi < ORD; yi++) {
                    const T* row = f + rowoff[zi][yi];
                    double acc_x = 0.0;
#pragma unroll
                    for (int xi = 0; xi < ORD; xi++) acc_x += w[0][xi] * (double)__ldg(row + idx[0][xi]);
                    acc_y += w[1][yi] * acc_x;
                }
                acc_z += w[2][zi] * acc_y;
            }
            uf[c] = acc_z;
        }
    } else {
        // column x = idx[0][sub]; the x weights are applied before the group sum
        int xs = idx[0][0];
        double wx = (sub == 0) ? w[0][0] : 0.0;
#pragma unroll
        for (int xi = 1; xi < ORD; xi++)
            if (sub == xi) { xs = idx[0][xi]; wx = w[0][xi]; }
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const T* f = phys + (long long)c * g.R + xs;
            double acc_z = 0.0;
#pragma unroll
            for (int zi = 0; zi < ORD; zi++) {
                double acc_y = 0.0;
#pragma unroll
                for (int yi = 0; yi < ORD; yi++)
                    acc_y += w[1][yi] * (double)__ldg(f + ((long long)idx[2][zi] * g.ny + idx[1][yi]) * g.nx);
                acc_z += w[2][zi] * acc_y;
            }
            double v = wx * acc_z;
#pragma unroll
            for (int o = 1; o < G; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            uf[c] = v;
        }
        if (sub != 0 || !valid) return;
    }
    // the particle's RK3 state, read only by the thread that updates it, after the
    // gather (not held in registers across it)
    double up[3], ur[3], pr[3];
#pragma unroll
    for (int c = 0; c < 3; c++) { up[c] = P.up[c][nn]; ur[c] = P.uprk[c][nn]; pr[c] = P.prk[c][nn]; }
    double xw[3] = {xp[0], xp[1], xp[2]};   // frame in which the RK3 update runs
    // BF-rot shear transforms to the laboratory frame and back; the R forms
    // (p_RK3SolveParticleR, src/pp_rk3.f90:307-403, dispatched at src/pp_control.f90:
    // 568-571) interpolate laboratory components and advance the moving position with
    // them directly, the isotropic arithmetic
    const bool bfrot = g.shear && !g.rrot;
    if (bfrot) {
        // p_RK3SolveParticleBF (src/pp_rk3.f90:169-303): velocity and position to
        // the laboratory frame (p_RK3Mov2Lab, src/pp_rk3.f90:989-1014), RK3 there,
        // back with p_RK3Lab2Mov (1016-1042) at the same B.
        const BF bf = make_bf(g, ck);
        double xl[3] = {0.0, 0.0, 0.0}, ul[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
            for (int b = 0; b < 3; b++)
                if (bex(a, b)) { xl[a] += bf.bi[a][b] * xp[b]; ul[a] += bf.bi[a][b] * uf[b]; }
#pragma unroll
        for (int c = 0; c < 3; c++) { xw[c] = xl[c]; uf[c] = ul[c]; }
    }
    // p_ControlInitPartVelocity(BF) at the release step (src/pp_control.f90:378-516)
    if (tstep == pp.release && stage == 1) {
#pragma unroll
        for (int c = 0; c < 3; c++) { up[c] = uf[c]; pr[c] = 0.0; ur[c] = 0.0; }
    }
    const double dpv = P.dp[n];
    if (dpv > 0.0) {
        const double tau = ((dpv * dpv) / (18.0 * pp.f_nu)) * (pp.p_rho / pp.f_rho);
        // shear: minus the homogeneous source amat up (p_RK3ComputeHomogeneousSourceTerm,
        // src/pp_rk3.f90:1080-1102); amat has the single entry (1,3)
        const double hs0 = bfrot ? g.shear_s * up[2] : 0.0;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const double acc = ((uf[c] - up[c]) / tau) - (c == 0 ? hs0 : 0.0);
            pr[c] = (beta * pr[c]) + acc;
            up[c] = up[c] + (gamma * dt * pr[c]);
        }
    } else {
#pragma unroll
        for (int c = 0; c < 3; c++) up[c] = uf[c];
    }
#pragma unroll
    for (int c = 0; c < 3; c++) {
        ur[c] = (beta * ur[c]) + up[c];
        xw[c] = xw[c] + (gamma * dt * ur[c]);
    }
    if (bfrot) {
        const BF bf = make_bf(g, ck);
#pragma unroll
        for (int a = 0; a < 3; a++) {
            double v = 0.0;
#pragma unroll
            for (int b = 0; b < 3; b++)
                if (bex(a, b)) v += bf.bm[a][b] * xw[b];
            xp[a] = v;
        }
    } else {
#pragma unroll
        for (int c = 0; c < 3; c++) xp[c] = xw[c];
    }
    const double x1min = -0.5 * g.dx, x2min = -0.5 * g.dy, x3min = -0.5 * g.dz;
    const double x1max = x1min + g.lx, x2max = x2min + g.ly, x3max = x3min + g.lz;
    if (xp[0] < x1min) xp[0] = xp[0] + g.lx;
    if (xp[0] >= x1max) xp[0] = xp[0] - g.lx;
    if (xp[1] < x2min) xp[1] = xp[1] + g.ly;
    if (xp[1] >= x2max) xp[1] = xp[1] - g.ly;
    if (xp[2] < x3min) xp[2] = xp[2] + g.lz;
    if (xp[2] > x3max) xp[2] = xp[2] - g.lz;
    const double ymin = -(0.5 * g.dy), ymax = (double)g.ny * g.dy - (0.5 * g.dy);
    const double zmin = -(0.5 * g.dz), zmax = (double)g.nz * g.dz - (0.5 * g.dz);
    if (!(xp[1] >= ymin && xp[1] < ymax && xp[2] >= zmin && xp[2] < zmax)) atomicOr(&ck->status, PD_ST_LOST);
#pragma unroll
    for (int c = 0; c < 3; c++) {
        P.xp[c][n] = xp[c]; P.up[c][n] = up[c]; P.uprk[c][n] = ur[c]; P.prk[c][n] = pr[c];
    }
}

// P_INIT_RANDOM (src/pp_control.f90:663-707): three draws per particle, in order.
__global__ void k_init_particles(Particles P, Geo g, uint64_t key, double dia) {
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= P.np) return;
    const double L[3] = {g.lx, g.ly, g.lz}, D[3] = {g.dx, g.dy, g.dz};
    for (int c = 0; c < 3; c++) {
        const double rn = uniform(key, (uint64_t)(3 * n + c));
        P.xp[c][n] = __dsub_rn(__dmul_rn(rn, L[c]), __dmul_rn(D[c], 0.5));
        P.up[c][n] = 0.0; P.uprk[c][n] = 0.0; P.prk[c][n] = 0.0;
    }
    P.dp[n] = dia;
    P.pid[n] = n;
}

// ---------------------------------------------------------------------------
// Spatial sort: counting sort by bin (z slowest, then y, then x).  Bins are
// whole blocks of cells; positions lie in [-d/2, L-d/2) after the wrap, so
// x + d/2 is in [0, L).  Order inside a bin follows atomics; every particle's
// update is independent of the order, and pid keeps the caller's numbering.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int bin_of(double x, double d, int cells, int nb) {
    int b = (int)floor((x + 0.5 * d) / (d * cells));
    return b < 0 ? 0 : (b >= nb ? nb - 1 : b);
}

__global__ void k_part_key(Particles P, Geo g, PartSort s) {
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= P.np) return;
    const int bx = bin_of(P.xp[0][n], g.dx, s.bin_cells[0], s.nb[0]);
    const int by = bin_of(P.xp[1][n], g.dy, s.bin_cells[1], s.nb[1]);
    const int bz = bin_of(P.xp[2][n], g.dz, s.bin_cells[2], s.nb[2]);
    const unsigned k = ((unsigned)bz * s.nb[1] + by) * s.nb[0] + bx;
    s.key[n] = k;
    atomicAdd(&s.count[k], 1u);
}

// exclusive scan of count[0..n) in place: per-block scan of 1024 entries ...
__device__ __forceinline__ unsigned block_exclusive_scan(unsigned v, unsigned* warp_tot, unsigned& total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    unsigned x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[wid] = x;
    __syncthreads();
    if (wid == 0) {
        unsigned t = (lane < (int)(blockDim.x >> 5)) ? warp_tot[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        warp_tot[lane] = t;   // inclusive prefix of warp totals
    }
    __syncthreads();
    total = warp_tot[(blockDim.x >> 5) - 1];
    const unsigned base = wid ? warp_tot[wid - 1] : 0u;
    return base + x - v;
}

__global__ void __launch_bounds__(1024) k_scan_blocks(unsigned* a, unsigned* sums, long long n) {
    __shared__ unsigned wt[32];
    const long long i = (long long)blockIdx.x * 1024 + threadIdx.x;
    const unsigned v = i < n ? a[i] : 0u;
    unsigned total;
    const unsigned ex = block_exclusive_scan(v, wt, total);
    if (i < n) a[i] = ex;
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// ... one block scans the block totals (at most 1024 of them) ...
__global__ void __launch_bounds__(1024) k_scan_sums(unsigned* sums, int nblocks) {
    __shared__ unsigned wt[32];
    const unsigned v = threadIdx.x < (unsigned)nblocks ? sums[threadIdx.x] : 0u;
    unsigned total;
    const unsigned ex = block_exclusive_scan(v, wt, total);
    if (threadIdx.x < (unsigned)nblocks) sums[threadIdx.x] = ex;
}

// ... and the block offsets are added back.
__global__ void __launch_bounds__(1024) k_scan_add(unsigned* a, const unsigned* sums, long long n) {
    const long long i = (long long)blockIdx.x * 1024 + threadIdx.x;
    if (i < n) a[i] += sums[blockIdx.x];
}

__global__ void k_part_scatter(Particles src, PartSort s) {
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= src.np) return;
    const long long d = atomicAdd(&s.count[s.key[n]], 1u);
    const Particles& t = s.tmp;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        t.xp[c][d] = src.xp[c][n]; t.up[c][d] = src.up[c][n];
        t.uprk[c][d] = src.uprk[c][n]; t.prk[c][d] = src.prk[c][n];
    }
    t.dp[d] = src.dp[n];
    t.pid[d] = src.pid[n];
}

template <class T>
cudaError_t launch_particles(const Geo& g, const Member<T>* M, int B, long long np, int order, int stage,
                             cudaStream_t st) {
    if (np == 0) return cudaSuccess;
    switch (order) {
#define PD_ORD(O)                                                                                  \
    case O:                                                                                        \
        return for_member_sets(M, B, [&](const auto& ms, int nm) {                                 \
            constexpr int CAP = std::decay_t<decltype(ms)>::cap;                                   \
            k_particles<O, T, CAP><<<dim3((unsigned)((np * part_group<O>() + 255) / 256), nm), 256, 0, st>>>(ms, stage); \
        });
        PD_ORD(1) PD_ORD(2) PD_ORD(3) PD_ORD(4) PD_ORD(5) PD_ORD(6)
#undef PD_ORD
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_init_particles(const Geo& g, const Particles& p, uint64_t key, double dia, cudaStream_t st) {
    if (p.np == 0) return cudaSuccess;
    const long long nb = (p.np + 255) / 256;
    k_init_particles<<<(unsigned)nb, 256, 0, st>>>(p, g, key, dia);
    return cudaGetLastError();
}

// Sorts P by bin into s.tmp, then copies back into P's storage (so that the
// pointers captured in the step's CUDA graph stay valid).
cudaError_t launch_particle_sort(const Geo& g, const Particles& P, const PartSort& s, cudaStream_t st,
                                 int* nlaunch) {
    if (P.np == 0) return cudaSuccess;
    const long long nbins = (long long)s.nb[0] * s.nb[1] * s.nb[2];
    const int nblk = (int)((nbins + 1023) / 1024);
    if (nblk > 1024) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(s.count, 0, sizeof(unsigned) * nbins, st);
    if (e) return e;
    const unsigned pb = (unsigned)((P.np + 255) / 256);
    k_part_key<<<pb, 256, 0, st>>>(P, g, s);
    k_scan_blocks<<<nblk, 1024, 0, st>>>(s.count, s.block_sums, nbins);
    k_scan_sums<<<1, 1024, 0, st>>>(s.block_sums, nblk);
    k_scan_add<<<nblk, 1024, 0, st>>>(s.count, s.block_sums, nbins);
    k_part_scatter<<<pb, 256, 0, st>>>(P, s);
    if ((e = cudaGetLastError())) return e;
    // the 13 double arrays and pid are contiguous in both buffers (14 * np words)
    e = cudaMemcpyAsync(P.xp[0], s.tmp.xp[0], sizeof(double) * 14 * (size_t)P.np, cudaMemcpyDeviceToDevice, st);
    if (nlaunch) *nlaunch += 5;
    return e;
}

// p_StatsPrimary (src/pp_stats.f90:119-200): the sums over particles of up_i up_j and of
// the kinetic energy (1/2)(pi/6 dp^3 P_RHO)|up|^2; the caller divides by P_NP_GLOBAL.
__global__ void __launch_bounds__(256) k_part_stats(Particles p, long long np, double rho_p, double* acc) {
    double s[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    const double c = 3.14159265358979323846264338327950288 / 6.0;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < np; n += (long long)gridDim.x * blockDim.x) {
        const double u1 = p.up[0][n], u2 = p.up[1][n], u3 = p.up[2][n], d = p.dp[n];
        s[0] += u1 * u1; s[1] += u2 * u2; s[2] += u3 * u3;
        s[3] += u1 * u2; s[4] += u1 * u3; s[5] += u2 * u3;
        s[6] += 0.5 * ((c * (d * d * d)) * rho_p) * ((u1 * u1) + (u2 * u2) + (u3 * u3));
    }
    __shared__ double red[8][7];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int a = 0; a < 7; a++) {
        double x = s[a];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) red[w][a] = x;
    }
    __syncthreads();
    if (threadIdx.x < 7) {
        double x = 0.0;
        for (int v = 0; v < (int)(blockDim.x >> 5); v++) x += red[v][threadIdx.x];
        atomicAdd(acc + threadIdx.x, x);
    }
}

cudaError_t launch_particle_stats(const Particles& p, long long np, double rho_p, double* acc, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(acc, 0, sizeof(double) * 7, st);
    if (e || np <= 0) return e;
    unsigned nb = (unsigned)std::min<long long>((np + 255) / 256, 1024);
    k_part_stats<<<nb, 256, 0, st>>>(p, np, rho_p, acc);
    return cudaGetLastError();
}

template cudaError_t launch_particles<double>(const Geo&, const Member<double>*, int, long long, int, int,
                                             cudaStream_t);
template cudaError_t launch_particles<float>(const Geo&, const Member<float>*, int, long long, int, int,
                                            cudaStream_t);

}  // namespace pd
