// pandora_internal.cuh -- device-side structures shared by the kernels and the
// C-ABI layer.  Not part of the public boundary (include/pandora_gpu.h is).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/pandora_gpu.h"

namespace pd {

// Geometry and constants of one simulation, passed by value to every kernel.
// Sizes follow g_DomainCalc (src/pg_domain.f90:147-243): KI = NX/3 etc., the
// stored spectral extents NKI = KI+1, NKJ = 2KJ+1, NKK = 2KK+1.  Intermediate
// pencils pad the i extent to NKIP (a multiple of 8) so that every tile row
// starts on a 128-byte boundary.
struct Geo {
    int nx, ny, nz;
    int ki, kj, kk;
    int nki, nkj, nkk, nkip;
    long long S;          // modes per component
    long long R;          // physical points
    double nu;            // F_NU
    double norm;          // 1 / (NX NY NZ)
    double dx, dy, dz, lx, ly, lz;
    double force_kf;
    int fnk;              // aint(FORCE_KF)
    int kkmax;            // E(k) shells
    // homogeneous shear (F_TYPE = F_SHEAR_DNS); zero for isotropic flow
    int shear;
    int rrot;             // shear in a Rogallo form (NS_DEFORMED = NS_R_ROT or NS_R_CONV), else BF-rot
    int rconv;            // ... the convective one (NS_R_CONV): u and its nine gradients in real space
    double bdiag[3];      // bmat(1,1), bmat(2,2), bmat(3,3) = 1/B110, 1/B220, 1/B330
    double bidiag[3];     // binv diagonal = B110, B220, B330
    double shear_s;       // F_DEFORM_S = amat(1,3)
    int b110, remesh_t, rk3_decide;
    double bvol;          // B110 B220 B330
    // DEALIASING 2 (2/3 sphere) or 3 (LES cutoff): modes with |k_lab| above this are
    // zeroed (src/pf_arrays.f90:1865-1987); 0 for the 2/3 rule alone
    double dealias_cut;
    // PANDORA_VISCOUS_INTEGRATING_FACTOR: the viscous term as exp(-nu k^2 dc dt) factors
    // of u and the register per stage (isotropic flow), else explicit
    int visc_if;
    // x lines per warp of the x pass (0: the library's choice for the length)
    int xlpw;
};

// Scalars of the running step kept in device memory so that a whole step can
// be replayed from a CUDA graph without host involvement.
struct Clock {
    double simtime;                 // time of the current stage (g_RK3Calc's simtime)
    double t0;                      // time at the start of the step
    double dt;                      // dt of the step (f_RK3Tstep at stage 1)
    unsigned long long ucfl_bits;   // max |u1|+|u2|+|u3| of stage 1, as ordered bits
    int tstep;                      // number of the step being taken
    unsigned int status;            // PD_ST_* bits
    double b13, bi13;               // bmat(1,3), binv(1,3) of the moving frame (shear)
};

enum : unsigned int {
    PD_ST_NAN = 1u,
    PD_ST_POLAR = 2u,       // bounded polar rejection loop gave up
    PD_ST_LOST = 4u,        // particle outside the domain after the wrap
    PD_ST_TIMEOUT = 8u,
    PD_ST_IDLE = 16u,       // batch slot without a member: batched kernels return at once
};

// ---- project RNG (SplitMix64 finaliser over a stream index; the oracle
//      restates the same definition) ----
#define PD_GOLDEN 0x9E3779B97F4A7C15ULL
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
__host__ __device__ __forceinline__ uint64_t stream_key(uint64_t seed, uint64_t tag) {
    return mix64(seed * PD_GOLDEN + tag * 0xD1B54A32D192ED03ULL + 0x632BE59BD9B4E019ULL);
}
__host__ __device__ __forceinline__ double uniform(uint64_t key, uint64_t n) {
    return (double)(mix64(key + (n + 1) * PD_GOLDEN) >> 11) * 0x1.0p-53;
}
enum : uint64_t { TAG_FLUID = 1, TAG_FORCE = 2, TAG_PART = 3 };
constexpr int kMaxPolarTries = 64;

__host__ __device__ __forceinline__ double wvn(int idx, int K) {
    return (double)(idx <= K ? idx : idx - (2 * K + 1));
}

// Device buffers of one simulation.  T is the real type of the fields and of the
// transforms: double for the FP64 form, float for the FP32-mixed form, whose
// forcing coefficients, clock and shell sums stay FP64.
template <class T> struct Cplx;
template <> struct Cplx<double> { using type = double2; };
template <> struct Cplx<float> { using type = float2; };

template <class T> struct FieldsT {
    using C = typename Cplx<T>::type;
    C* u[3];
    C* rk[3];
    C* zb;              // [6][NZ][NKJ][NKIP]  after the z pass
    C* yb;              // [6][NZ][NY][NKIP]   after the y pass; NL written into fields 0..2
    T* phys;            // [3][NZ][NY][NX]     physical velocity (particles), may be null
    double2* forcing;   // [3][NK+1][2NK+1][2NK+1]
    const C *tw_x, *tw_y, *tw_z;
    Clock* clock;
    double* shell;      // [3*(kkmax+1) + 3] shell sums (e, d), p11,p22,p33, mode counts
};
using Fields = FieldsT<double>;

// FP64 view of a stored value and its rounding back (identity for the FP64 form).
__host__ __device__ __forceinline__ double2 to_d(double2 v) { return v; }
__host__ __device__ __forceinline__ double2 to_d(float2 v) { return make_double2(v.x, v.y); }
template <class C> __host__ __device__ __forceinline__ C from_d(double2 v);
template <> __host__ __device__ __forceinline__ double2 from_d<double2>(double2 v) { return v; }
template <> __host__ __device__ __forceinline__ float2 from_d<float2>(double2 v) {
    return make_float2((float)v.x, (float)v.y);
}

// Launchers (kernels_*.cu), instantiated for T = double and float.  All enqueue
// on `st` and return cudaGetLastError().

// Particle arrays, structure of arrays: 13 doubles + the particle's index in
// the caller's order (pid).  The device keeps them sorted by spatial bin.
struct Particles {
    long long np;
    double* xp[3];
    double* up[3];
    double* uprk[3];
    double* prk[3];
    double* dp;
    long long* pid;
};

// Scratch of the per-step spatial sort of the particles.
struct PartSort {
    int nb[3];                 // bins per direction
    int bin_cells[3];          // cells per bin per direction
    unsigned* key;             // [np]
    unsigned* count;           // [nbins] counts, then exclusive offsets
    unsigned* block_sums;      // [ceil(nbins/1024)]
    Particles tmp;             // destination of the scatter
};

struct ForceParams {
    double tf, sigma;
    int stop;
    uint64_t key;
    long long calls_per_stage;
};

struct StepParams {
    int rk3_timestep;
    int f_type;
    double rk3_dt, rk3_cfl, force_tf, f_deform_s;
    int f_remesh_t;
};

struct PartParams {
    int order;
    int release;
    double f_nu, p_rho, f_rho;
};

struct InitParams {
    int type;
    double u0, kp, kv, kstart, kend, epsilon;
    int b110, b220, b330;
    int deformed;       // B110 + B220 + B330 > 3: f_InitialiseFluidDeformed
    uint64_t key;
};

// One simulation as the step kernels see it.  Every kernel of the step takes a
// set of these as a __grid_constant__ parameter (constant bank: read at CTA start
// without a trip to memory) and finds its member from a grid dimension, so one
// launch serves up to kBatchChunk members of a batch (same grid size, precision and
// flow type); a single simulation is a set of one.  A member with active == 0 (a
// free slot) returns at once in every kernel.
template <class T> struct Member {
    FieldsT<T> F;
    Geo g;
    Particles P;
    StepParams sp;
    ForceParams fp;
    PartParams pp;
    int active;
};
constexpr int kBatchChunk = 32;   // members per launch of a batch (about 18 KB of parameters)
template <class T, int CAP> struct MemberSet {
    static constexpr int cap = CAP;
    Member<T> m[CAP];
};

bool supported_length(int n);
// Lengths whose kernels have batched (multi-member) instantiations: the ensemble's sizes.
bool batched_length(int n);

// Records "where: <CUDA error string>" as the message pandora_strerror returns for
// PANDORA_ERR_CUDA (thread-local, the last failure wins) and returns PANDORA_ERR_CUDA.
int cuda_fail_msg(cudaError_t e, const char* where);

// Fields through the inverse z and y passes (zb, yb): velocity and vorticity, or in the
// R-conv form velocity, d u / dy and d u / dz (d u / dx is formed in the x pass).
__host__ __device__ __forceinline__ int pass_fields(const Geo& g) { return g.rconv ? 9 : 6; }

// Calls f(set, n) for each chunk of at most kBatchChunk members of the B in M: a
// MemberSet<T, 1> for a single simulation, MemberSet<T, kBatchChunk> (unused
// entries inactive) otherwise.  f launches one kernel with the set as parameter
// and n as the member extent of its grid.
template <class T, class Fn> inline cudaError_t for_member_sets(const Member<T>* M, int B, Fn f) {
    if (B == 1) {
        MemberSet<T, 1> one;
        one.m[0] = M[0];
        f(one, 1);
        return cudaGetLastError();
    }
    static thread_local MemberSet<T, kBatchChunk> set;   // 18 KB, copied into the launch
    for (int c0 = 0; c0 < B; c0 += kBatchChunk) {
        const int n = (B - c0) < kBatchChunk ? (B - c0) : kBatchChunk;
        for (int i = 0; i < kBatchChunk; i++) {
            if (i < n) set.m[i] = M[c0 + i];
            else set.m[i].active = 0;
        }
        f(set, n);
        cudaError_t e = cudaGetLastError();
        if (e) return e;
    }
    return cudaSuccess;
}

// Launchers of the step kernels: g is the batch's geometry (grid sizes and flow
// type, common to its members), M a host array of its B member descriptors
// (passed by value to the kernels, kBatchChunk members per launch).
// Tensor maps of the three FP64 velocity components in the [i][j][k] layout (dims k as
// 2 NKK doubles, j, i; boxes of BK k x 1 j x 8 i), for the K1 whose velocity rows are
// staged by tensor copies.
struct ZMaps {
    CUtensorMap u[3];
};
// Fills *out for a single FP64 simulation whose z length has the staged K1; *ok = false
// (and cudaSuccess) where it does not, or where the driver has no tensor-map encoder.
cudaError_t make_zmaps(const Geo& g, double2* const* u, ZMaps* out, bool* ok);
// K1: with `maps` (a single FP64 simulation, make_zmaps ok) the staged kernel, else the
// kernel that reads its inputs element-wise from global memory.
template <class T>
cudaError_t launch_zpass_inv(const Geo& g, const Member<T>* M, int B, int stage, cudaStream_t st,
                             const ZMaps* maps = nullptr);
template <class T> cudaError_t launch_ypass_inv(const Geo& g, const Member<T>* M, int B, cudaStream_t st);
template <class T>
cudaError_t launch_xpass(const Geo& g, const Member<T>* M, int B, int want_phys, int want_cfl, cudaStream_t st);
template <class T> cudaError_t launch_ypass_fwd(const Geo& g, const Member<T>* M, int B, cudaStream_t st);
template <class T>
cudaError_t launch_zpass_fwd_update(const Geo& g, const Member<T>* M, int B, int stage, int mode, cudaStream_t st);
template <class T>
cudaError_t launch_stats(const Geo& g, const Member<T>* M, int B, double* shell, cudaStream_t st);
template <class T>
cudaError_t launch_stage_scalars(const Geo& g, const Member<T>* M, int B, const ForceParams& fp, int stage,
                                 cudaStream_t st);
template <class T> cudaError_t launch_advance_time(const Geo& g, const Member<T>* M, int B, int stage, cudaStream_t st);
template <class T>
cudaError_t launch_particles(const Geo& g, const Member<T>* M, int B, long long np, int order, int stage,
                             cudaStream_t st);
template <class T> cudaError_t launch_check_finite(const Geo& g, const Member<T>* M, int B, cudaStream_t st);
template <class T>
cudaError_t launch_remesh(const Geo& g, const Member<T>* M, int B, long long np, cudaStream_t st);
// The x pass with the real-space statistics of every point (single simulation):
// kRsSlots (32) copies of 21 moment sums and 4 maxima (as ordered bits), 32 doubles each.
template <class T>
cudaError_t launch_xpass_stats(const Geo& g, const Member<T>* M, double* rs, cudaStream_t st);
// Particle moments: sum up_i up_j (6) and the kinetic energy sum (1) into acc[7].
cudaError_t launch_particle_stats(const Particles& p, long long np, double rho_p, double* acc, cudaStream_t st);
// DEALIASING 2/3 applied to the members' state in place (no-op for the 2/3 rule)
template <class T>
cudaError_t launch_dealias(const Geo& g, const Member<T>* M, int B, cudaStream_t st);
// P[2m], P[2m+1] (m = 0..NKI-1): the x co-spectrum of u1 (laboratory) and u1 (stored)
template <class T> cudaError_t launch_xcorr_cospec(const Member<T>& m, double* P, cudaStream_t st);
// Per simulation (not batched): initial field (generated in FP64; the FP32-mixed
// form converts it), particle initialisation and the per-step spatial sort.
cudaError_t launch_init_fluid(const Geo& g, const Fields& f, const InitParams& ip, cudaStream_t st);
cudaError_t launch_reset_clock(Clock* ck, int tstep, double t, double b13, double bi13, cudaStream_t st);
cudaError_t launch_set_idle(Clock* ck, cudaStream_t st);
cudaError_t launch_init_particles(const Geo& g, const Particles& p, uint64_t key, double dia,
                                  cudaStream_t st);
cudaError_t launch_particle_sort(const Geo& g, const Particles& p, const PartSort& s, cudaStream_t st,
                                 int* nlaunch);
// n complex values from one precision to the other (FP64 <-> FP32 at the boundary).
cudaError_t launch_convert(const double2* in, float2* out, long long n, cudaStream_t st);
cudaError_t launch_convert(const float2* in, double2* out, long long n, cudaStream_t st);
size_t shell_words(const Geo& g);

// Shared-memory configuration (set once per process per device).
template <class T> cudaError_t configure_kernels(const Geo& g);
cudaError_t configure_fluid_kernels(const Geo& g, const ForceParams& fp);

}  // namespace pd
