// kernels_particles.cu -- Lagrangian particle advance on sm_100a.
//
// One thread per particle: tensor-product Neville interpolation of the physical
// velocity of the current stage (p_InterpInterpolate3D / FindMolecule /
// Neville3D, src/pp_interp.f90:313-560), the tracer or Stokes-drag RK3 update
// (p_RK3SolveParticle, src/pp_rk3.f90:57-165, drag 927-946) and the periodic
// wrap (p_MPICorrectPosition, src/pp_mpi.f90:1011-1057; x3 uses '>' where x1
// and x2 use '>=').  The reference fetches a halo of NHALO = order/2 planes by
// DMGlobalToLocal (src/pp_interp.f90:115-264); on one GPU the stencil indices
// simply wrap modulo N.  Physical velocity layout: [c][z][y][x].
#include <cuda_runtime.h>
#include "pandora_internal.cuh"

namespace pd {

constexpr int kMaxOrder = 6;

__global__ void __launch_bounds__(256) k_particles(Particles P, Geo g, const double* __restrict__ phys,
                                                   Clock* ck, PartParams pp, int stage) {
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int tstep = ck->tstep;
    if (n >= P.np || tstep < pp.release) return;
    const double dt = ck->dt;
    double beta, gamma;
    if (stage == 1) { beta = 0.0; gamma = 1.0 / 3.0; }
    else if (stage == 2) { beta = -(5.0 / 9.0); gamma = 15.0 / 16.0; }
    else { beta = -(153.0 / 128.0); gamma = 8.0 / 15.0; }
    const int ord = pp.order, nh = ord / 2;
    const double D[3] = {g.dx, g.dy, g.dz};
    const int NN[3] = {g.nx, g.ny, g.nz};
    double xp[3], up[3], ur[3], pr[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        xp[c] = P.xp[c][n]; up[c] = P.up[c][n]; ur[c] = P.uprk[c][n]; pr[c] = P.prk[c][n];
    }
    // p_InterpFindMolecule: index arithmetic with explicit rounding (no contraction)
    int i0[3];
    double nodes[3][kMaxOrder];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        double halo = __dmul_rn((double)nh, D[c]);
        double xd;
        if ((ord & 1) == 0) {
            halo = __dsub_rn(halo, __dmul_rn(0.5, D[c]));
            xd = __dadd_rn(__dadd_rn(__dadd_rn(xp[c], halo), D[c]), __dmul_rn(0.5, D[c]));
        } else {
            xd = __dadd_rn(__dadd_rn(xp[c], halo), __dmul_rn(0.5, D[c]));
        }
        const int idx = (int)__ddiv_rn(xd, D[c]) - nh - nh;
        i0[c] = idx;
        for (int m = 0; m < ord; m++) nodes[c][m] = __dmul_rn((double)(idx + m), D[c]);
    }
    int X[kMaxOrder], Y[kMaxOrder], Z[kMaxOrder];
    for (int m = 0; m < ord; m++) {
        X[m] = ((i0[0] + m) % NN[0] + NN[0]) % NN[0];
        Y[m] = ((i0[1] + m) % NN[1] + NN[1]) % NN[1];
        Z[m] = ((i0[2] + m) % NN[2] + NN[2]) % NN[2];
    }
    // p_InterpNeville3D: along y for every (x, z), then along z for every x, then x.
    double uf[3];
    for (int c = 0; c < 3; c++) {
        const double* f = phys + (long long)c * g.R;
        double vz[kMaxOrder][kMaxOrder];   // [xi][zi] after the y sweep
        for (int zi = 0; zi < ord; zi++) {
            for (int xi = 0; xi < ord; xi++) {
                double v[kMaxOrder];
                for (int yi = 0; yi < ord; yi++)
                    v[yi] = __ldg(&f[((long long)Z[zi] * g.ny + Y[yi]) * g.nx + X[xi]]);
                for (int col = 1; col <= ord - 1; col++)
                    for (int nv = 0; nv < ord - col; nv++) {
                        const double d1 = xp[1] - nodes[1][nv + col], d2 = nodes[1][nv] - xp[1];
                        const double d3 = nodes[1][nv] - nodes[1][nv + col];
                        v[nv] = ((d1 * v[nv]) + (d2 * v[nv + 1])) / d3;
                    }
                vz[xi][zi] = v[0];
            }
        }
        double vx[kMaxOrder];
        for (int xi = 0; xi < ord; xi++) {
            for (int col = 1; col <= ord - 1; col++)
                for (int nv = 0; nv < ord - col; nv++) {
                    const double d1 = xp[2] - nodes[2][nv + col], d2 = nodes[2][nv] - xp[2];
                    const double d3 = nodes[2][nv] - nodes[2][nv + col];
                    vz[xi][nv] = ((d1 * vz[xi][nv]) + (d2 * vz[xi][nv + 1])) / d3;
                }
            vx[xi] = vz[xi][0];
        }
        for (int col = 1; col <= ord - 1; col++)
            for (int nv = 0; nv < ord - col; nv++) {
                const double d1 = xp[0] - nodes[0][nv + col], d2 = nodes[0][nv] - xp[0];
                const double d3 = nodes[0][nv] - nodes[0][nv + col];
                vx[nv] = ((d1 * vx[nv]) + (d2 * vx[nv + 1])) / d3;
            }
        uf[c] = vx[0];
    }
    // p_ControlInitPartVelocity at the release step (src/pp_control.f90:378-416)
    if (tstep == pp.release && stage == 1) {
        for (int c = 0; c < 3; c++) { up[c] = uf[c]; pr[c] = 0.0; ur[c] = 0.0; }
    }
    const double dpv = P.dp[n];
    if (dpv > 0.0) {
        const double tau = ((dpv * dpv) / (18.0 * pp.f_nu)) * (pp.p_rho / pp.f_rho);
        for (int c = 0; c < 3; c++) {
            const double acc = (uf[c] - up[c]) / tau;
            pr[c] = (beta * pr[c]) + acc;
            up[c] = up[c] + (gamma * dt * pr[c]);
        }
    } else {
        for (int c = 0; c < 3; c++) up[c] = uf[c];
    }
    for (int c = 0; c < 3; c++) {
        ur[c] = (beta * ur[c]) + up[c];
        xp[c] = xp[c] + (gamma * dt * ur[c]);
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
}

cudaError_t launch_particles(const Geo& g, const Fields& f, const Particles& p, const PartParams& pp, int stage,
                             cudaStream_t st) {
    if (p.np == 0) return cudaSuccess;
    if (pp.order < 1 || pp.order > kMaxOrder) return cudaErrorInvalidValue;
    const long long nb = (p.np + 255) / 256;
    k_particles<<<(unsigned)nb, 256, 0, st>>>(p, g, f.phys, f.clock, pp, stage);
    return cudaGetLastError();
}

cudaError_t launch_init_particles(const Geo& g, const Particles& p, uint64_t key, double dia, cudaStream_t st) {
    if (p.np == 0) return cudaSuccess;
    const long long nb = (p.np + 255) / 256;
    k_init_particles<<<(unsigned)nb, 256, 0, st>>>(p, g, key, dia);
    return cudaGetLastError();
}

}  // namespace pd
