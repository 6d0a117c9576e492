// pandora_capi.cu -- the extern "C" boundary (include/pandora_gpu.h).
//
// Replaces the module-global state and the stage sequencing of g_RK3Calc /
// f_RK3Stage{1,2,3} (src/pg_rk3.f90:82-129, src/pf_rk3.f90:40-200): one handle
// owns the resident device fields, the twiddle tables, the clock scalars and a
// CUDA graph that holds one whole time step.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <algorithm>
#include <cmath>
#include <new>
#include <vector>
#include "pandora_internal.cuh"
#include "bfrot.cuh"

using namespace pd;

struct pandora_handle {
    pandora_params p;
    Geo g;
    int dev = 0;
    cudaStream_t own = nullptr;
    cudaStream_t st = nullptr;
    cudaStream_t side = nullptr;      // particle branch of a stage (forked from st, joined back)
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    int timing = 0;                   // pandora_set_pass_timing: bit p-1 times pass p
    bool timed[3][6] = {};
    cudaEvent_t tev[3][6][2] = {};
    Fields F{};                       // FP64 view of the buffers (and the FP64 scratch of the mixed form)
    FieldsT<float> Ff{};              // FP32 view of the same buffers (FP32-mixed form)
    bool mixed = false;               // PANDORA_PREC_FP32_MIXED
    size_t celem = sizeof(double2);   // bytes of one stored complex value
    void* fbuf = nullptr;             // u[3], rk[3] contiguous
    void* tw = nullptr;               // tw_x | tw_y | tw_z
    Clock* clock = nullptr;
    Clock* clock_host = nullptr;      // pinned mirror
    double* shell_step = nullptr;     // stats of the state at stage 1 of the last step
    double* shell_now = nullptr;      // stats of pandora_stats()
    double* shell_host = nullptr;     // pinned
    std::vector<double> dens_mod;     // [kkmax + 1]
    long long nforce = 0;             // complex entries per forcing component
    StepParams sp{};
    ForceParams fp{};
    PartParams pp{};
    Particles P{};
    double* pbuf = nullptr;           // 13 * np doubles + np pid
    double* pbuf2 = nullptr;          // sort destination, same layout
    PartSort sort{};
    void* nlbuf = nullptr;            // scratch for pandora_nonlinear
    double* rsbuf = nullptr;          // real-space / particle statistics sums (32 x 32)
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool use_graph = true;
    int launches_per_step = 0;
    bool particles_on = false;
    ZMaps zmaps{};                    // tensor maps of u for the staged K1 (FP64, z lengths that have it)
    bool zmaps_ok = false;
};

static thread_local char g_errmsg[256];

static int cuda_fail(cudaError_t e, const char* where) {
    snprintf(g_errmsg, sizeof(g_errmsg), "%s: %s", where, cudaGetErrorString(e));
    return PANDORA_ERR_CUDA;
}
namespace pd {
int cuda_fail_msg(cudaError_t e, const char* where) { return cuda_fail(e, where); }
}  // namespace pd
#define PD_CK(x)                                          \
    do {                                                  \
        cudaError_t _e = (x);                             \
        if (_e != cudaSuccess) return cuda_fail(_e, #x);  \
    } while (0)

extern "C" const char* pandora_strerror(int s) {
    switch (s) {
    case PANDORA_OK: return "ok";
    case PANDORA_ERR_INVALID_ARG: return "invalid argument";
    case PANDORA_ERR_OOM: return "device allocation failed";
    case PANDORA_ERR_CUDA: return g_errmsg[0] ? g_errmsg : "CUDA error";
    case PANDORA_ERR_NAN: return "non-finite value in the state";
    case PANDORA_ERR_TIMEOUT: return "bounded device wait gave up";
    case PANDORA_ERR_BAD_LAYOUT: return "grid size not supported by the transform plan";
    case PANDORA_ERR_CFL: return "RK3_CFL >= 1";
    case PANDORA_ERR_PARTICLE_LOST: return "particle left the domain after the wrap";
    case PANDORA_ERR_NO_DEVICE: return "no CUDA device";
    case PANDORA_ERR_UNSUPPORTED: return "option not supported by this library";
    default: return "unknown status";
    }
}

extern "C" int pandora_params_sizeof(void) { return (int)sizeof(pandora_params); }

extern "C" int pandora_device_count(int* count) {
    if (!count) return PANDORA_ERR_INVALID_ARG;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) { *count = 0; cudaGetLastError(); return PANDORA_ERR_NO_DEVICE; }
    *count = n;
    return PANDORA_OK;
}

extern "C" int pandora_params_default(pandora_params* p) {
    if (!p) return PANDORA_ERR_INVALID_ARG;
    memset(p, 0, sizeof(*p));
    p->nodes_x = p->nodes_y = p->nodes_z = 32;
    p->b110 = p->b220 = p->b330 = 1;
    p->f_rho = 1.0; p->f_nu = 0.025;
    p->f_type = PANDORA_F_ISOTROPIC; p->f_deform_s = 28.3; p->f_remesh_t = 32;
    p->rk3_timestep = PANDORA_RK3_TIMESTEP_DECIDE; p->rk3_cfl = 0.75; p->rk3_dt = 0.01;
    p->ns_deformed = PANDORA_NS_BF_ROT; p->dealiasing = 1; p->tsteps = 10;
    p->f_init_type = PANDORA_F_INIT_KERR; p->f_init_u0 = 0.1; p->f_init_kp = 11.0; p->f_init_kv = 20.0;
    p->f_init_kstart = 5.0; p->f_init_kend = 10.0;
    p->force_tf = 0.2; p->force_sigma = 0.03743; p->force_kf = 2.829; p->force_stop = 99999;
    p->p_track_part = 0; p->p_init_type = PANDORA_P_INIT_RANDOM; p->p_np_global = 10;
    p->p_interp_order = 4; p->p_ts_release = 1000; p->p_rho = 1000.0; p->p_dia_vals = 0.01514314;
    p->seed_fluid = 1; p->seed_force = 2; p->seed_particles = 3;
    p->precision = PANDORA_PREC_FP64;
    p->les_cutoff = 1.0;
    return PANDORA_OK;
}

static int kkmax_of(int ki, int kj, int kk) {
    const double kmax = sqrt((double)((long long)ki * ki + (long long)kj * kj + (long long)kk * kk));
    return (int)lround(kmax / 1.0);
}
// src/pf_fluidstats.f90:356-366: deformed domains scale k_max by 1/B
static int kkmax_of(const pandora_params* p) {
    const int ki = p->nodes_x / 3, kj = p->nodes_y / 3, kk = p->nodes_z / 3;
    if (p->f_type == PANDORA_F_ISOTROPIC) return kkmax_of(ki, kj, kk);
    const double kmax = sqrt((double)((double)ki * ki / (double)(p->b110 * p->b110) +
                                      (double)kj * kj / (double)(p->b220 * p->b220) +
                                      (double)kk * kk / (double)(p->b330 * p->b330)));
    return (int)lround(kmax / 1.0);
}

extern "C" int pandora_sizes(const pandora_params* p, int32_t* nki, int32_t* nkj, int32_t* nkk, int64_t* modes,
                             int32_t* kkmax) {
    if (!p || p->nodes_x < 3 || p->nodes_y < 3 || p->nodes_z < 3) return PANDORA_ERR_INVALID_ARG;
    const int ki = p->nodes_x / 3, kj = p->nodes_y / 3, kk = p->nodes_z / 3;
    if (nki) *nki = ki + 1;
    if (nkj) *nkj = 2 * kj + 1;
    if (nkk) *nkk = 2 * kk + 1;
    if (modes) *modes = (int64_t)(ki + 1) * (2 * kj + 1) * (2 * kk + 1);
    if (kkmax) *kkmax = kkmax_of(p);
    return PANDORA_OK;
}

static long long force_calls(int NK) {
    return 3LL * ((long long)(NK + 1) * (NK + 1) + (long long)NK * (NK + 1)) +
           3LL * NK * (2LL * NK + 1) * (2LL * NK + 1);
}

static void release(pandora_handle* h) {
    if (!h) return;
    cudaSetDevice(h->dev);
    if (h->exec) cudaGraphExecDestroy(h->exec);
    if (h->graph) cudaGraphDestroy(h->graph);
    cudaFree(h->fbuf); cudaFree(h->F.zb); cudaFree(h->F.yb); cudaFree(h->F.phys);
    cudaFree(h->F.forcing); cudaFree(h->tw); cudaFree(h->clock); cudaFree(h->shell_step);
    cudaFree(h->shell_now); cudaFree(h->pbuf); cudaFree(h->pbuf2); cudaFree(h->nlbuf); cudaFree(h->rsbuf);
    cudaFree(h->sort.key); cudaFree(h->sort.count); cudaFree(h->sort.block_sums);
    if (h->clock_host) cudaFreeHost(h->clock_host);
    if (h->shell_host) cudaFreeHost(h->shell_host);
    for (auto& st3 : h->tev)
        for (auto& pr : st3)
            for (cudaEvent_t e : pr)
                if (e) cudaEventDestroy(e);
    if (h->ev_fork) cudaEventDestroy(h->ev_fork);
    if (h->ev_join) cudaEventDestroy(h->ev_join);
    if (h->side) cudaStreamDestroy(h->side);
    if (h->own) cudaStreamDestroy(h->own);
    delete h;
}

// The handle's buffers as fields of the stored precision.
template <class T> static FieldsT<T>& fields(pandora_handle* h);
template <> FieldsT<double>& fields<double>(pandora_handle* h) { return h->F; }
template <> FieldsT<float>& fields<float>(pandora_handle* h) { return h->Ff; }

// This simulation as a batch of one (every step kernel takes a member array).
template <class T> static Member<T> member_of(pandora_handle* h, const FieldsT<T>& F) {
    Member<T> m{};
    m.F = F;
    m.g = h->g;
    m.P = h->P;
    m.sp = h->sp;
    m.fp = h->fp;
    m.pp = h->pp;
    m.active = 1;
    return m;
}
template <class T> static Member<T> self_of(pandora_handle* h) { return member_of<T>(h, fields<T>(h)); }

static int validate(const pandora_params* p) {
    if (!p) return PANDORA_ERR_INVALID_ARG;
    if (p->precision != PANDORA_PREC_FP64 && p->precision != PANDORA_PREC_FP32_MIXED) return PANDORA_ERR_UNSUPPORTED;
    if (p->f_type != PANDORA_F_ISOTROPIC && p->f_type != PANDORA_F_SHEAR_DNS) return PANDORA_ERR_UNSUPPORTED;
    if (p->f_type == PANDORA_F_SHEAR_DNS) {
        if (p->ns_deformed != PANDORA_NS_BF_ROT && p->ns_deformed != PANDORA_NS_R_ROT &&
            p->ns_deformed != PANDORA_NS_R_CONV)
            return PANDORA_ERR_UNSUPPORTED;
        if (p->b110 < 1 || p->b220 < 1 || p->b330 < 1 || p->f_deform_s == 0.0 || p->f_remesh_t < 1)
            return PANDORA_ERR_INVALID_ARG;
    }
    if (p->rk3_viscous != PANDORA_VISCOUS_EXPLICIT && p->rk3_viscous != PANDORA_VISCOUS_INTEGRATING_FACTOR)
        return PANDORA_ERR_INVALID_ARG;
    // the integrating factor of a sheared frame would need the time integral of its moving k^2
    if (p->rk3_viscous == PANDORA_VISCOUS_INTEGRATING_FACTOR && p->f_type != PANDORA_F_ISOTROPIC)
        return PANDORA_ERR_UNSUPPORTED;
    if (p->dealiasing < PANDORA_DEALIASING_23 || p->dealiasing > PANDORA_DEALIASING_LES) return PANDORA_ERR_UNSUPPORTED;
    if (p->x_lines_per_warp != 0 && p->x_lines_per_warp != 1 && p->x_lines_per_warp != 2 && p->x_lines_per_warp != 4)
        return PANDORA_ERR_INVALID_ARG;
    if (p->x_lines_per_warp > 1 && p->nodes_x > 64) return PANDORA_ERR_INVALID_ARG;
    if (p->dealiasing == PANDORA_DEALIASING_LES && !(p->les_cutoff > 0.0)) return PANDORA_ERR_INVALID_ARG;
    if (!supported_length(p->nodes_x) || !supported_length(p->nodes_y) || !supported_length(p->nodes_z))
        return PANDORA_ERR_BAD_LAYOUT;
    if (p->rk3_cfl >= 1.0) return PANDORA_ERR_CFL;   // g_RK3Check, src/pg_rk3.f90:240-267
    if (p->rk3_timestep < 1 || p->rk3_timestep > 3) return PANDORA_ERR_INVALID_ARG;
    if (p->force_kf < 0.0 || p->force_kf > 8.0 || p->force_tf <= 0.0) return PANDORA_ERR_INVALID_ARG;
    if (p->f_nu < 0.0) return PANDORA_ERR_INVALID_ARG;
    if (p->p_track_part) {
        if (p->p_np_global < 0 || p->p_interp_order < 1 || p->p_interp_order > 6) return PANDORA_ERR_INVALID_ARG;
        // the spatial sort counts and offsets particles in 32 bits
        if (p->p_np_global > 0x7fffffffll) return PANDORA_ERR_INVALID_ARG;
        if (p->p_dia_vals > 0.0 && (p->f_nu <= 0.0 || p->f_rho <= 0.0)) return PANDORA_ERR_INVALID_ARG;
    }
    return PANDORA_OK;
}

extern "C" int pandora_create(const pandora_params* p, pandora_handle** out) {
    if (!out) return PANDORA_ERR_INVALID_ARG;
    *out = nullptr;
    int rc = validate(p);
    if (rc) return rc;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { cudaGetLastError(); return PANDORA_ERR_NO_DEVICE; }
    pandora_handle* h = new (std::nothrow) pandora_handle();
    if (!h) return PANDORA_ERR_OOM;
    h->p = *p;
    cudaGetDevice(&h->dev);
    Geo& g = h->g;
    g.nx = p->nodes_x; g.ny = p->nodes_y; g.nz = p->nodes_z;
    g.ki = g.nx / 3; g.kj = g.ny / 3; g.kk = g.nz / 3;
    g.nki = g.ki + 1; g.nkj = 2 * g.kj + 1; g.nkk = 2 * g.kk + 1;
    g.nkip = (g.nki + 7) / 8 * 8;
    g.S = (long long)g.nki * g.nkj * g.nkk;
    g.R = (long long)g.nx * g.ny * g.nz;
    g.nu = p->f_nu;
    g.norm = 1.0 / ((double)g.nx * (double)g.ny * (double)g.nz);
    const double twopi = 6.283185307179586476925286766559005768;
    g.lx = twopi; g.ly = twopi; g.lz = twopi;
    g.dx = g.lx / (double)g.nx; g.dy = g.ly / (double)g.ny; g.dz = g.lz / (double)g.nz;
    g.force_kf = p->force_kf;
    g.fnk = (int)p->force_kf;
    g.kkmax = kkmax_of(p);
    g.shear = (p->f_type == PANDORA_F_SHEAR_DNS) ? 1 : 0;
    g.rrot = (g.shear && (p->ns_deformed == PANDORA_NS_R_ROT || p->ns_deformed == PANDORA_NS_R_CONV)) ? 1 : 0;
    g.rconv = (g.shear && p->ns_deformed == PANDORA_NS_R_CONV) ? 1 : 0;
    g.bdiag[0] = 1.0 / (double)p->b110; g.bdiag[1] = 1.0 / (double)p->b220; g.bdiag[2] = 1.0 / (double)p->b330;
    g.bidiag[0] = (double)p->b110; g.bidiag[1] = (double)p->b220; g.bidiag[2] = (double)p->b330;
    g.shear_s = p->f_deform_s;
    g.b110 = p->b110; g.remesh_t = p->f_remesh_t;
    g.rk3_decide = (p->rk3_timestep == PANDORA_RK3_TIMESTEP_DECIDE) ? 1 : 0;
    g.bvol = (double)p->b110 * (double)p->b220 * (double)p->b330;
    g.visc_if = p->rk3_viscous == PANDORA_VISCOUS_INTEGRATING_FACTOR ? 1 : 0;
    g.xlpw = p->x_lines_per_warp;
    {   // KMAX = min(KI_MAX, KJ_MAX, KK_MAX) (src/pg_domain.f90:231)
        const double kmax = (double)std::min(g.ki, std::min(g.kj, g.kk));
        g.dealias_cut = p->dealiasing == PANDORA_DEALIASING_SPHERICAL ? kmax
                      : (p->dealiasing == PANDORA_DEALIASING_LES ? p->les_cutoff * kmax : 0.0);
    }
    h->nforce = (long long)(g.fnk + 1) * (2 * g.fnk + 1) * (2 * g.fnk + 1);
    h->particles_on = p->p_track_part != 0;
    h->mixed = p->precision == PANDORA_PREC_FP32_MIXED;
    h->celem = h->mixed ? sizeof(float2) : sizeof(double2);
    const size_t ce = h->celem;

    cudaError_t e;
#define PD_ALLOC(ptr, bytes)                                              \
    do {                                                                  \
        e = cudaMalloc((void**)&(ptr), (bytes));                          \
        if (e != cudaSuccess) { cudaGetLastError(); release(h); return PANDORA_ERR_OOM; } \
    } while (0)
    // fields in the stored precision; zb (6 x NZ x NKJ x NKIP values, NZ >= NKK and
    // NKIP >= NKI) always holds 3S FP64 values, the conversion scratch of the mixed form.
    // The R-conv form carries 9 fields through the inverse z and y passes.
    PD_ALLOC(h->fbuf, ce * 6 * (size_t)g.S);
    PD_ALLOC(h->F.zb, ce * (size_t)pass_fields(g) * g.nz * g.nkj * g.nkip);
    PD_ALLOC(h->F.yb, ce * (size_t)pass_fields(g) * g.nz * g.ny * g.nkip);
    if (h->particles_on) PD_ALLOC(h->F.phys, ce / 2 * 3 * (size_t)g.R);
    PD_ALLOC(h->F.forcing, sizeof(double2) * 3 * (size_t)h->nforce);
    PD_ALLOC(h->tw, ce * (size_t)(g.nx + g.ny + g.nz));
    PD_ALLOC(h->clock, sizeof(Clock));
    const size_t nsh = shell_words(g);
    PD_ALLOC(h->shell_step, sizeof(double) * nsh);
    PD_ALLOC(h->shell_now, sizeof(double) * nsh);
#undef PD_ALLOC
    if (cudaMallocHost((void**)&h->clock_host, sizeof(Clock)) != cudaSuccess ||
        cudaMallocHost((void**)&h->shell_host, sizeof(double) * nsh) != cudaSuccess) {
        cudaGetLastError(); release(h); return PANDORA_ERR_OOM;
    }
    if ((e = cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming)) != cudaSuccess) {
        release(h); return cuda_fail(e, "cudaStreamCreate");
    }
    h->st = h->own;
    // twiddles tw[e] = exp(-2 pi i e / N), long double on the host, rounded once to
    // the stored precision
    {
        const size_t ntw = (size_t)(g.nx + g.ny + g.nz);
        std::vector<double2> tw(ntw);
        std::vector<float2> twf(ntw);
        int off = 0;
        const int lens[3] = {g.nx, g.ny, g.nz};
        const int offs[3] = {0, g.nx, g.nx + g.ny};
        for (int d = 0; d < 3; d++) {
            const int n = lens[d];
            for (int q = 0; q < n; q++) {
                const long double a = 6.283185307179586476925286766559005768L * (long double)q / (long double)n;
                tw[off + q] = make_double2((double)cosl(a), -(double)sinl(a));
                twf[off + q] = make_float2((float)cosl(a), -(float)sinl(a));
            }
            off += n;
        }
        const double2* twd = (const double2*)h->tw;
        const float2* tws = (const float2*)h->tw;
        h->F.tw_x = twd + offs[0]; h->F.tw_y = twd + offs[1]; h->F.tw_z = twd + offs[2];
        h->Ff.tw_x = tws + offs[0]; h->Ff.tw_y = tws + offs[1]; h->Ff.tw_z = tws + offs[2];
        e = h->mixed ? cudaMemcpy(h->tw, twf.data(), sizeof(float2) * ntw, cudaMemcpyHostToDevice)
                     : cudaMemcpy(h->tw, tw.data(), sizeof(double2) * ntw, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) { release(h); return cuda_fail(e, "twiddles"); }
    }
    // mode density (src/pf_fluidstats.f90:696-780), integer counts -> exact
    h->dens_mod.assign(g.kkmax + 1, 0.0);
    {
        std::vector<long long> cnt(g.kkmax + 2, 0);
        for (int i = 0; i < g.nki; i++)
            for (int j = 0; j < g.nkj; j++)
                for (int k = 0; k < g.nkk; k++) {
                    const double a = i, b = wvn(j, g.kj), c = wvn(k, g.kk);
                    const double km = sqrt((a * a) + (b * b) + (c * c));
                    const int kc = (int)floor(km + 0.5);
                    for (int q = kc - 1; q <= kc + 1; q++) {
                        if (q < 1 || q > g.kkmax) continue;
                        if (km >= (double)q - 0.5 && km < (double)q + 0.5) cnt[q] += (i != 0) ? 2 : 1;
                    }
                }
        const double pi = 3.14159265358979323846264338327950288;
        for (int q = 1; q <= g.kkmax; q++) {
            const double up = (double)q + 0.5, lo = (double)q - 0.5;
            h->dens_mod[q] = (double)cnt[q] / (4.0 / 3.0 * pi * (up * up * up - lo * lo * lo));
        }
    }
    for (int c = 0; c < 3; c++) {
        h->F.u[c] = (double2*)h->fbuf + c * g.S; h->F.rk[c] = (double2*)h->fbuf + (3 + c) * g.S;
        h->Ff.u[c] = (float2*)h->fbuf + c * g.S; h->Ff.rk[c] = (float2*)h->fbuf + (3 + c) * g.S;
    }
    h->Ff.zb = (float2*)h->F.zb; h->Ff.yb = (float2*)h->F.yb; h->Ff.phys = (float*)h->F.phys;
    h->Ff.forcing = h->F.forcing;
    h->F.clock = h->clock; h->Ff.clock = h->clock;
    h->F.shell = h->shell_step; h->Ff.shell = h->shell_step;
    h->sp.rk3_timestep = p->rk3_timestep; h->sp.f_type = p->f_type; h->sp.rk3_dt = p->rk3_dt;
    h->sp.rk3_cfl = p->rk3_cfl; h->sp.force_tf = p->force_tf; h->sp.f_deform_s = p->f_deform_s;
    h->sp.f_remesh_t = p->f_remesh_t;
    h->fp.tf = p->force_tf; h->fp.sigma = p->force_sigma; h->fp.stop = p->force_stop;
    h->fp.key = stream_key(p->seed_force, TAG_FORCE);
    h->fp.calls_per_stage = force_calls(g.fnk);
    h->pp.order = p->p_interp_order; h->pp.release = p->p_ts_release; h->pp.f_nu = p->f_nu;
    h->pp.p_rho = p->p_rho; h->pp.f_rho = p->f_rho;
    if ((e = h->mixed ? configure_kernels<float>(g) : configure_kernels<double>(g)) != cudaSuccess) {
        release(h); return cuda_fail(e, "configure_kernels");
    }
    if ((e = configure_fluid_kernels(g, h->fp)) != cudaSuccess) {
        release(h); return cuda_fail(e, "configure_fluid_kernels");
    }
    if (!h->mixed && (e = make_zmaps(g, h->F.u, &h->zmaps, &h->zmaps_ok)) != cudaSuccess) {
        release(h); return cuda_fail(e, "make_zmaps");
    }
    // zero state (the reference zero-initialises its Vecs and rk3 registers)
    if ((e = cudaMemsetAsync(h->fbuf, 0, ce * 6 * (size_t)g.S, h->st)) != cudaSuccess ||
        (e = cudaMemsetAsync(h->F.forcing, 0, sizeof(double2) * 3 * (size_t)h->nforce, h->st)) != cudaSuccess ||
        (e = cudaMemsetAsync(h->clock, 0, sizeof(Clock), h->st)) != cudaSuccess ||
        (e = cudaMemsetAsync(h->shell_step, 0, sizeof(double) * nsh, h->st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(h->st)) != cudaSuccess) {
        release(h); return cuda_fail(e, "zero state");
    }
    if (h->particles_on && p->p_np_global > 0) {
        const long long np = p->p_np_global;
        PartSort& so = h->sort;
        const int lens[3] = {g.nx, g.ny, g.nz};
        long long nbins = 1;
        for (int d = 0; d < 3; d++) {
            int cells = 4;
            while ((lens[d] + cells - 1) / cells > 64) cells *= 2;
            so.bin_cells[d] = cells;
            so.nb[d] = (lens[d] + cells - 1) / cells;
            nbins *= so.nb[d];
        }
        const size_t pbytes = sizeof(double) * 14 * (size_t)np;
        if (cudaMalloc((void**)&h->pbuf, pbytes) != cudaSuccess ||
            cudaMalloc((void**)&h->pbuf2, pbytes) != cudaSuccess ||
            cudaMalloc((void**)&so.key, sizeof(unsigned) * (size_t)np) != cudaSuccess ||
            cudaMalloc((void**)&so.count, sizeof(unsigned) * (size_t)nbins) != cudaSuccess ||
            cudaMalloc((void**)&so.block_sums, sizeof(unsigned) * 1024) != cudaSuccess) {
            cudaGetLastError(); release(h); return PANDORA_ERR_OOM;
        }
        cudaMemsetAsync(h->pbuf, 0, pbytes, h->st);
        auto bind = [np](Particles& P, double* b) {
            P.np = np;
            for (int c = 0; c < 3; c++) {
                P.xp[c] = b + (0 + c) * np; P.up[c] = b + (3 + c) * np;
                P.uprk[c] = b + (6 + c) * np; P.prk[c] = b + (9 + c) * np;
            }
            P.dp = b + 12 * np;
            P.pid = (long long*)(b + 13 * np);
        };
        bind(h->P, h->pbuf);
        bind(so.tmp, h->pbuf2);
        std::vector<long long> ids((size_t)np);
        for (long long n = 0; n < np; n++) ids[(size_t)n] = n;
        if (cudaMemcpy(h->P.pid, ids.data(), sizeof(long long) * np, cudaMemcpyHostToDevice) != cudaSuccess) {
            release(h); return PANDORA_ERR_CUDA;
        }
    }
    *out = h;
    return PANDORA_OK;
}

extern "C" int pandora_destroy(pandora_handle* h) {
    if (!h) return PANDORA_ERR_INVALID_ARG;
    release(h);
    return PANDORA_OK;
}

static void drop_graph(pandora_handle* h) {
    if (h->exec) { cudaGraphExecDestroy(h->exec); h->exec = nullptr; }
    if (h->graph) { cudaGraphDestroy(h->graph); h->graph = nullptr; }
}

extern "C" int pandora_set_stream(pandora_handle* h, void* s) {
    if (!h) return PANDORA_ERR_INVALID_ARG;
    cudaSetDevice(h->dev);
    PD_CK(cudaStreamSynchronize(h->st));
    h->st = s ? (cudaStream_t)s : h->own;
    return PANDORA_OK;
}

static int copy3(pandora_handle* h, double2* const* dev, const double* a, const double* b, const double* c,
                 size_t n, bool to_dev) {
    if (!h || !a || !b || !c) return PANDORA_ERR_INVALID_ARG;
    cudaSetDevice(h->dev);
    const double* src[3] = {a, b, c};
    for (int q = 0; q < 3; q++) {
        if (to_dev) PD_CK(cudaMemcpyAsync(dev[q], src[q], sizeof(double2) * n, cudaMemcpyHostToDevice, h->st));
        else PD_CK(cudaMemcpyAsync((void*)src[q], dev[q], sizeof(double2) * n, cudaMemcpyDeviceToHost, h->st));
    }
    PD_CK(cudaStreamSynchronize(h->st));
    return PANDORA_OK;
}

// Three spectral fields of S complex values at the FP64 boundary.  The mixed form
// stores FP32: the host's FP64 values pass through the z-pencil buffer (free between
// steps) and are converted on the device in either direction.
static int copy_fields(pandora_handle* h, double2* const* dev64, float2* const* dev32, const double* a,
                       const double* b, const double* c, bool to_dev) {
    if (!a || !b || !c) return PANDORA_ERR_INVALID_ARG;
    if (!h->mixed) return copy3(h, dev64, a, b, c, (size_t)h->g.S, to_dev);
    cudaSetDevice(h->dev);
    const long long S = h->g.S;
    double2* scr[3] = {h->F.zb, h->F.zb + S, h->F.zb + 2 * S};
    if (to_dev) {
        int rc = copy3(h, scr, a, b, c, (size_t)S, true);
        if (rc) return rc;
        for (int q = 0; q < 3; q++) PD_CK(launch_convert(scr[q], dev32[q], S, h->st));
        PD_CK(cudaStreamSynchronize(h->st));
        return PANDORA_OK;
    }
    for (int q = 0; q < 3; q++) PD_CK(launch_convert(dev32[q], scr[q], S, h->st));
    return copy3(h, scr, a, b, c, (size_t)S, false);
}

extern "C" int pandora_set_state(pandora_handle* h, const double* u1, const double* u2, const double* u3) {
    if (!h) return PANDORA_ERR_INVALID_ARG;
    return copy_fields(h, h->F.u, h->Ff.u, u1, u2, u3, true);
}
extern "C" int pandora_get_state(pandora_handle* h, double* u1, double* u2, double* u3) {
    if (!h) return PANDORA_ERR_INVALID_ARG;
    return copy_fields(h, h->F.u, h->Ff.u, u1, u2, u3, false);
}
extern "C" int pandora_set_rk(pandora_handle* h, const double* r1, const double* r2, const double* r3) {
    if (!h) return PANDORA_ERR_INVALID_ARG;
    return copy_fields(h, h->F.rk, h->Ff.rk, r1, r2, r3, true);
}
extern "C" int pandora_get_rk(pandora_handle* h, double* r1, double* r2, double* r3) {
    if (!h) return PANDORA_ERR_INVALID_ARG;
    return copy_fields(h, h->F.rk, h->Ff.rk, r1, r2, r3, false);
}
extern "C" int pandora_forcing_size(pandora_handle* h, int64_t* n) {
    if (!h || !n) return PANDORA_ERR_INVALID_ARG;
    *n = 2 * h->nforce;
    return PANDORA_OK;
}
extern "C" int pandora_set_forcing(pandora_handle* h, const double* f1, const double* f2, const double* f3) {
    if (!h) return PANDORA_ERR_INVALID_ARG;
    double2* d[3] = {h->F.forcing, h->F.forcing + h->nforce, h->F.forcing + 2 * h->nforce};
    return copy3(h, d, f1, f2, f3, (size_t)h->nforce, true);
}
extern "C" int pandora_get_forcing(pandora_handle* h, double* f1, double* f2, double* f3) {
    if (!h) return PANDORA_ERR_INVALID_ARG;
    double2* d[3] = {h->F.forcing, h->F.forcing + h->nforce, h->F.forcing + 2 * h->nforce};
    return copy3(h, d, f1, f2, f3, (size_t)h->nforce, false);
}
extern "C" int pandora_state_device_ptrs(pandora_handle* h, void** u1, void** u2, void** u3) {
    if (!h || !u1 || !u2 || !u3) return PANDORA_ERR_INVALID_ARG;
    if (h->mixed) { *u1 = h->Ff.u[0]; *u2 = h->Ff.u[1]; *u3 = h->Ff.u[2]; }
    else { *u1 = h->F.u[0]; *u2 = h->F.u[1]; *u3 = h->F.u[2]; }
    return PANDORA_OK;
}

// The seeded initial field, enqueued on the handle's stream (no host wait).
static int init_fluid_async(pandora_handle* h) {
    InitParams ip{};
    ip.type = h->p.f_init_type; ip.u0 = h->p.f_init_u0; ip.kp = h->p.f_init_kp; ip.kv = h->p.f_init_kv;
    ip.kstart = h->p.f_init_kstart; ip.kend = h->p.f_init_kend; ip.epsilon = h->p.f_init_epsilon;
    ip.b110 = h->p.b110; ip.b220 = h->p.b220; ip.b330 = h->p.b330;
    ip.deformed = (h->p.b110 + h->p.b220 + h->p.b330) > 3 ? 1 : 0;
    ip.key = stream_key(h->p.seed_fluid, TAG_FLUID);
    if (h->mixed) {   // generated in FP64 into the z-pencil buffer, then rounded once
        Fields Fd = h->F;
        for (int c = 0; c < 3; c++) Fd.u[c] = h->F.zb + c * h->g.S;
        PD_CK(launch_init_fluid(h->g, Fd, ip, h->st));
        for (int c = 0; c < 3; c++) PD_CK(launch_convert(Fd.u[c], h->Ff.u[c], h->g.S, h->st));
        const Member<float> m = self_of<float>(h);
        PD_CK(launch_dealias(h->g, &m, 1, h->st));   // DEALIASING 2/3 after the initial field
    } else {
        PD_CK(launch_init_fluid(h->g, h->F, ip, h->st));
        const Member<double> m = self_of<double>(h);
        PD_CK(launch_dealias(h->g, &m, 1, h->st));
    }
    return PANDORA_OK;
}

extern "C" int pandora_init_fluid(pandora_handle* h) {
    if (!h) return PANDORA_ERR_INVALID_ARG;
    cudaSetDevice(h->dev);
    int rc = init_fluid_async(h);
    if (rc) return rc;
    PD_CK(cudaStreamSynchronize(h->st));
    return PANDORA_OK;
}

// ---- particles ----
static int part_check(pandora_handle* h, int64_t np) {
    if (!h) return PANDORA_ERR_INVALID_ARG;
    if (!h->particles_on || np != h->P.np) return PANDORA_ERR_INVALID_ARG;
    return PANDORA_OK;
}
extern "C" int pandora_set_particles(pandora_handle* h, int64_t np, const double* xp, const double* up,
                                     const double* up_rk3, const double* rk3, const double* dp) {
    int rc = part_check(h, np);
    if (rc) return rc;
    if (np == 0) return PANDORA_OK;
    cudaSetDevice(h->dev);
    std::vector<double> soa((size_t)13 * np, 0.0);
    // SoA order in pbuf: xp(0..2) up(3..5) uprk(6..8) prk(9..11) dp(12)
    const double* srcs[4] = {xp, up, up_rk3, rk3};
    for (int a = 0; a < 4; a++) {
        if (!srcs[a]) continue;
        for (int64_t n = 0; n < np; n++)
            for (int c = 0; c < 3; c++) soa[(size_t)(3 * a + c) * np + n] = srcs[a][3 * n + c];
    }
    if (dp) memcpy(&soa[(size_t)12 * np], dp, sizeof(double) * np);
    std::vector<long long> ids((size_t)np);
    for (int64_t n = 0; n < np; n++) ids[(size_t)n] = n;
    PD_CK(cudaMemcpyAsync(h->pbuf, soa.data(), sizeof(double) * soa.size(), cudaMemcpyHostToDevice, h->st));
    PD_CK(cudaMemcpyAsync(h->P.pid, ids.data(), sizeof(long long) * np, cudaMemcpyHostToDevice, h->st));
    PD_CK(cudaStreamSynchronize(h->st));
    return PANDORA_OK;
}
extern "C" int pandora_get_particles(pandora_handle* h, int64_t np, double* xp, double* up, double* up_rk3,
                                     double* rk3, double* dp) {
    int rc = part_check(h, np);
    if (rc) return rc;
    if (np == 0) return PANDORA_OK;
    cudaSetDevice(h->dev);
    std::vector<double> soa((size_t)13 * np);
    std::vector<long long> ids((size_t)np);
    PD_CK(cudaMemcpyAsync(soa.data(), h->pbuf, sizeof(double) * soa.size(), cudaMemcpyDeviceToHost, h->st));
    PD_CK(cudaMemcpyAsync(ids.data(), h->P.pid, sizeof(long long) * np, cudaMemcpyDeviceToHost, h->st));
    PD_CK(cudaStreamSynchronize(h->st));
    // the device keeps particles sorted by bin; pid maps back to the caller's order
    double* dsts[4] = {xp, up, up_rk3, rk3};
    for (int64_t n = 0; n < np; n++) {
        const long long q = ids[(size_t)n];
        if (q < 0 || q >= np) return PANDORA_ERR_INVALID_ARG;
        for (int a = 0; a < 4; a++) {
            if (!dsts[a]) continue;
            for (int c = 0; c < 3; c++) dsts[a][3 * q + c] = soa[(size_t)(3 * a + c) * np + n];
        }
        if (dp) dp[q] = soa[(size_t)12 * np + n];
    }
    return PANDORA_OK;
}
extern "C" int pandora_init_particles(pandora_handle* h) {
    if (!h || !h->particles_on) return PANDORA_ERR_INVALID_ARG;
    cudaSetDevice(h->dev);
    PD_CK(launch_init_particles(h->g, h->P, stream_key(h->p.seed_particles, TAG_PART), h->p.p_dia_vals, h->st));
    PD_CK(cudaStreamSynchronize(h->st));
    return PANDORA_OK;
}

// ---- stage sequencing ----
// f_RK3Stage{s} (src/pf_rk3.f90:40-200): [s=1: statistics of the state],
// vorticity + z pass, y pass, x pass with NL (and CFL / physical velocity),
// dt + forcing, particles, forward y, forward z + RK update, time advance.
// One stage.  With particles, stage 1 forks a second stream: the spatial sort of
// the particles runs beside the statistics and the first three passes and joins
// the main stream before the particle advance.  Captured into the step graph, the
// fork and join become graph edges.
// What one stage of a batch needs: the batch's geometry, its device member array
// of B slots, the particles per member, the shell sums (B x shell_words,
// contiguous), the streams, and for a single simulation the particle sort and the
// pass-timing events.
template <class T> struct StepCtx {
    const Geo* g;
    const Member<T>* M;
    int B;
    long long np;
    int order;
    const ForceParams* fp;
    double* shell;
    cudaStream_t st, side;
    cudaEvent_t ev_fork, ev_join;
    const PartSort* sort;        // null: no per-step particle sort (batches)
    const Particles* sortP;      // the particles the sort reorders
    pandora_handle* timing;      // null: no pass timing
    const ZMaps* zmaps;          // null: K1 reads u element-wise (batches, FP32, other lengths)
};

template <class T> static int enqueue_stage_ctx(const StepCtx<T>& c, int stage, int* nlaunch) {
    const Geo& g = *c.g;
    const Member<T>* M = c.M;
    const int B = c.B;
    int n = 0;
    const bool part = c.np > 0;
    if (stage == 1 && g.shear) {
        PD_CK(launch_remesh(g, M, B, c.np, c.st)); n += part ? 2 : 1;
    }
    const bool sorted = stage == 1 && part && c.sort;
    if (sorted) {   // the spatial sort runs beside the statistics and K1-K3, joined before the advance
        PD_CK(cudaEventRecord(c.ev_fork, c.st));
        PD_CK(cudaStreamWaitEvent(c.side, c.ev_fork, 0));
        PD_CK(launch_particle_sort(g, *c.sortP, *c.sort, c.side, &n));
        PD_CK(cudaEventRecord(c.ev_join, c.side));
    }
    if (stage == 1) {
        PD_CK(launch_stats(g, M, B, c.shell, c.st)); n += 1;   // one kernel (plus a memset node)
    }
    // instrumentation: event pair around pass `ps` (1..6) when pass timing is on
    pandora_handle* h = c.timing;
    auto mark = [&](int ps, int end, cudaStream_t s) -> cudaError_t {
        if (!h || !(h->timing & (1 << (ps - 1)))) return cudaSuccess;
        h->timed[stage - 1][ps - 1] = true;
        // External: captured as an event record node (a plain record inside a capture
        // only orders the streams and never fires the event)
        return cudaEventRecordWithFlags(h->tev[stage - 1][ps - 1][end], s, cudaEventRecordExternal);
    };
    PD_CK(mark(1, 0, c.st));
    PD_CK(launch_zpass_inv(g, M, B, stage, c.st, c.zmaps)); n += g.dealias_cut > 0.0 ? 2 : 1;   // k_dealias first
    PD_CK(mark(1, 1, c.st));
    PD_CK(mark(2, 0, c.st));
    PD_CK(launch_ypass_inv(g, M, B, c.st)); n++;
    PD_CK(mark(2, 1, c.st));
    PD_CK(mark(3, 0, c.st));
    PD_CK(launch_xpass(g, M, B, part ? 1 : 0, stage == 1 ? 1 : 0, c.st)); n++;
    PD_CK(mark(3, 1, c.st));
    PD_CK(launch_stage_scalars(g, M, B, *c.fp, stage, c.st)); n++;
    // The particle advance (it needs K3's physical velocity and the stage's dt) runs in
    // the main stream between K3 and K4: on a second stream beside K4/K5 it slowed them
    // by more than its own time (512^3 shear: K4 0.62 -> 0.85 ms beside a 0.08 ms advance).
    if (part) {
        if (sorted) PD_CK(cudaStreamWaitEvent(c.st, c.ev_join, 0));
        PD_CK(mark(6, 0, c.st));
        PD_CK(launch_particles(g, M, B, c.np, c.order, stage, c.st)); n++;
        PD_CK(mark(6, 1, c.st));
    }
    PD_CK(mark(4, 0, c.st));
    PD_CK(launch_ypass_fwd(g, M, B, c.st)); n++;
    PD_CK(mark(4, 1, c.st));
    PD_CK(mark(5, 0, c.st));
    PD_CK(launch_zpass_fwd_update(g, M, B, stage, 0, c.st)); n += 2;   // forward z FFT, RK update
    PD_CK(mark(5, 1, c.st));
    PD_CK(launch_advance_time(g, M, B, stage, c.st)); n++;
    if (nlaunch) *nlaunch += n;
    return PANDORA_OK;
}

template <class T> static int enqueue_stage_t(pandora_handle* h, int stage, int* nlaunch) {
    const Member<T> self = self_of<T>(h);   // copied into each launch's parameters
    StepCtx<T> c{};
    c.g = &h->g;
    c.M = &self;
    c.B = 1;
    c.np = (h->particles_on && h->P.np > 0) ? h->P.np : 0;
    c.order = h->pp.order;
    c.fp = &h->fp;
    c.shell = h->shell_step;
    c.st = h->st;
    c.side = h->side;
    c.ev_fork = h->ev_fork;
    c.ev_join = h->ev_join;
    c.sort = &h->sort;
    c.sortP = &h->P;
    c.timing = h;
    c.zmaps = (h->zmaps_ok && !h->mixed) ? &h->zmaps : nullptr;
    return enqueue_stage_ctx(c, stage, nlaunch);
}

static int enqueue_stage(pandora_handle* h, int stage, int* nlaunch) {
    return h->mixed ? enqueue_stage_t<float>(h, stage, nlaunch) : enqueue_stage_t<double>(h, stage, nlaunch);
}

static int enqueue_step(pandora_handle* h) {
    int n = 0;
    for (int s = 1; s <= 3; s++) {
        int rc = enqueue_stage(h, s, &n);
        if (rc) return rc;
    }
    h->launches_per_step = n;
    return PANDORA_OK;
}

static int build_graph(pandora_handle* h) {
    if (h->exec) return PANDORA_OK;
    PD_CK(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_step(h);
    cudaGraph_t gr = nullptr;
    cudaError_t e = cudaStreamEndCapture(h->st, &gr);
    if (rc) { if (gr) cudaGraphDestroy(gr); return rc; }
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    h->graph = gr;
    e = cudaGraphInstantiate(&h->exec, gr, 0);
    if (e != cudaSuccess) { drop_graph(h); return cuda_fail(e, "cudaGraphInstantiate"); }
    return PANDORA_OK;
}

static int status_to_rc(unsigned int st) {
    if (st & PD_ST_NAN) return PANDORA_ERR_NAN;
    if (st & PD_ST_LOST) return PANDORA_ERR_PARTICLE_LOST;
    if (st & (PD_ST_POLAR | PD_ST_TIMEOUT)) return PANDORA_ERR_TIMEOUT;
    return PANDORA_OK;
}

static int set_clock(pandora_handle* h, int tstep, double simtime) {
    // keep dt / ucfl / status from the device copy
    PD_CK(cudaMemcpyAsync(h->clock_host, h->clock, sizeof(Clock), cudaMemcpyDeviceToHost, h->st));
    PD_CK(cudaStreamSynchronize(h->st));
    h->clock_host->tstep = tstep;
    h->clock_host->simtime = simtime;
    h->clock_host->t0 = simtime;
    if (h->g.shear) {
        // the frame of stage 1 of step tstep is the one g_RK3UpdateB set at the end of step tstep-1
        update_b(h->g, tstep - 1, simtime, h->clock_host->b13, h->clock_host->bi13);
    }
    PD_CK(cudaMemcpyAsync(h->clock, h->clock_host, sizeof(Clock), cudaMemcpyHostToDevice, h->st));
    return PANDORA_OK;
}

extern "C" int pandora_rk3_advance(pandora_handle* h, int32_t tstep0, int32_t nsteps, int32_t sync,
                                   double* simtime) {
    if (!h || nsteps < 0 || !simtime) return PANDORA_ERR_INVALID_ARG;
    cudaSetDevice(h->dev);
    int rc = set_clock(h, tstep0, *simtime);
    if (rc) return rc;
    if (h->use_graph) {
        rc = build_graph(h);
        if (rc) return rc;
        for (int s = 0; s < nsteps; s++) PD_CK(cudaGraphLaunch(h->exec, h->st));
    } else {
        for (int s = 0; s < nsteps; s++) if ((rc = enqueue_step(h))) return rc;
    }
    if (!sync) return PANDORA_OK;
    PD_CK(cudaMemcpyAsync(h->clock_host, h->clock, sizeof(Clock), cudaMemcpyDeviceToHost, h->st));
    PD_CK(cudaStreamSynchronize(h->st));
    *simtime = h->clock_host->simtime;
    return status_to_rc(h->clock_host->status);
}

extern "C" int pandora_rk3_step(pandora_handle* h, int32_t tstep, double* simtime, double* dt) {
    if (!h || !simtime) return PANDORA_ERR_INVALID_ARG;
    int rc = pandora_rk3_advance(h, tstep, 1, 1, simtime);
    if (dt) *dt = h->clock_host->dt;
    return rc;
}

extern "C" int pandora_rk3_stage(pandora_handle* h, int32_t stage, int32_t tstep, double time, double* dt) {
    if (!h || stage < 1 || stage > 3 || !dt) return PANDORA_ERR_INVALID_ARG;
    cudaSetDevice(h->dev);
    PD_CK(cudaMemcpyAsync(h->clock_host, h->clock, sizeof(Clock), cudaMemcpyDeviceToHost, h->st));
    PD_CK(cudaStreamSynchronize(h->st));
    h->clock_host->tstep = tstep;
    h->clock_host->simtime = time;
    if (stage == 1) h->clock_host->t0 = time;
    h->clock_host->dt = *dt;
    PD_CK(cudaMemcpyAsync(h->clock, h->clock_host, sizeof(Clock), cudaMemcpyHostToDevice, h->st));
    int rc = enqueue_stage(h, stage, nullptr);
    if (rc) return rc;
    PD_CK(cudaMemcpyAsync(h->clock_host, h->clock, sizeof(Clock), cudaMemcpyDeviceToHost, h->st));
    PD_CK(cudaStreamSynchronize(h->st));
    *dt = h->clock_host->dt;
    return status_to_rc(h->clock_host->status);
}

// ---- statistics ----
static void finish_stats(pandora_handle* h, const double* sh, double* ek, int32_t kkmax, double* tke,
                         double* eps) {
    const int K = h->g.kkmax;
    const double* se = sh;
    const double* sd = sh + (K + 1);
    const double* sp = sh + 2 * (K + 1);
    const double* sc = sp + 3;
    if (h->g.shear) {   // f_FluidstatsModeDensityBFRot: counts of this B, / (B110 B220 B330)
        const double pi = 3.14159265358979323846264338327950288;
        for (int q = 1; q <= K; q++) {
            const double up = (double)q + 0.5, lo = (double)q - 0.5;
            h->dens_mod[q] = sc[q] / (4.0 / 3.0 * pi * (up * up * up - lo * lo * lo)) / h->g.bvol;
        }
    }
    double fdis = 0.0;
    for (int q = 1; q <= K; q++) {
        if (h->dens_mod[q] != 0.0) {
            fdis += sd[q];
            if (ek && q - 1 < kkmax) ek[q - 1] = se[q] / h->dens_mod[q];
        } else if (ek && q - 1 < kkmax) {
            ek[q - 1] = se[q];
        }
    }
    if (tke) *tke = 0.5 * (sp[0] + sp[1] + sp[2]);
    if (eps) *eps = fdis;
}

extern "C" int pandora_stats(pandora_handle* h, double* ek, int32_t kkmax, double* tke, double* eps,
                             double* ucfl) {
    if (!h) return PANDORA_ERR_INVALID_ARG;
    cudaSetDevice(h->dev);
    if (h->mixed) {
        FieldsT<float> Fs = h->Ff;
        Fs.shell = h->shell_now;
        const Member<float> mv = member_of<float>(h, Fs);
        PD_CK(launch_stats(h->g, &mv, 1, h->shell_now, h->st));
    } else {
        Fields Fs = h->F;
        Fs.shell = h->shell_now;
        const Member<double> mv = member_of<double>(h, Fs);
        PD_CK(launch_stats(h->g, &mv, 1, h->shell_now, h->st));
    }
    const size_t nsh = shell_words(h->g);
    PD_CK(cudaMemcpyAsync(h->shell_host, h->shell_now, sizeof(double) * nsh, cudaMemcpyDeviceToHost, h->st));
    PD_CK(cudaMemcpyAsync(h->clock_host, h->clock, sizeof(Clock), cudaMemcpyDeviceToHost, h->st));
    PD_CK(cudaStreamSynchronize(h->st));
    finish_stats(h, h->shell_host, ek, kkmax, tke, eps);
    if (ucfl) memcpy(ucfl, &h->clock_host->ucfl_bits, sizeof(double));
    return PANDORA_OK;
}

extern "C" int pandora_last_step_stats(pandora_handle* h, double* ek, int32_t kkmax, double* tke, double* eps,
                                       double* ucfl) {
    if (!h) return PANDORA_ERR_INVALID_ARG;
    cudaSetDevice(h->dev);
    const size_t nsh = shell_words(h->g);
    PD_CK(cudaMemcpyAsync(h->shell_host, h->shell_step, sizeof(double) * nsh, cudaMemcpyDeviceToHost, h->st));
    PD_CK(cudaMemcpyAsync(h->clock_host, h->clock, sizeof(Clock), cudaMemcpyDeviceToHost, h->st));
    PD_CK(cudaStreamSynchronize(h->st));
    finish_stats(h, h->shell_host, ek, kkmax, tke, eps);
    if (ucfl) memcpy(ucfl, &h->clock_host->ucfl_bits, sizeof(double));
    return PANDORA_OK;
}

extern "C" int pandora_nonlinear(pandora_handle* h, double* n1, double* n2, double* n3) {
    if (!h || !n1 || !n2 || !n3) return PANDORA_ERR_INVALID_ARG;
    cudaSetDevice(h->dev);
    if (!h->nlbuf) {
        if (cudaMalloc((void**)&h->nlbuf, h->celem * 3 * (size_t)h->g.S) != cudaSuccess) {
            cudaGetLastError(); return PANDORA_ERR_OOM;
        }
    }
    if (h->mixed) {
        FieldsT<float> Fn = h->Ff;
        for (int c = 0; c < 3; c++) Fn.rk[c] = (float2*)h->nlbuf + c * h->g.S;
        const Member<float> mv = member_of<float>(h, Fn);
        const Member<float>* Mv = &mv;
        PD_CK(launch_zpass_inv(h->g, Mv, 1, 0, h->st));
        PD_CK(launch_ypass_inv(h->g, Mv, 1, h->st));
        PD_CK(launch_xpass(h->g, Mv, 1, 0, 0, h->st));
        PD_CK(launch_ypass_fwd(h->g, Mv, 1, h->st));
        PD_CK(launch_zpass_fwd_update(h->g, Mv, 1, 1, 1, h->st));
        double2* none[3] = {nullptr, nullptr, nullptr};
        return copy_fields(h, none, Fn.rk, n1, n2, n3, false);
    }
    Fields Fn = h->F;
    for (int c = 0; c < 3; c++) Fn.rk[c] = (double2*)h->nlbuf + c * h->g.S;
    const Member<double> mv = member_of<double>(h, Fn);
    const Member<double>* Mv = &mv;
    PD_CK(launch_zpass_inv(h->g, Mv, 1, 0, h->st, h->zmaps_ok ? &h->zmaps : nullptr));
    PD_CK(launch_ypass_inv(h->g, Mv, 1, h->st));
    PD_CK(launch_xpass(h->g, Mv, 1, 0, 0, h->st));
    PD_CK(launch_ypass_fwd(h->g, Mv, 1, h->st));
    PD_CK(launch_zpass_fwd_update(h->g, Mv, 1, 1, 1, h->st));
    return copy3(h, Fn.rk, n1, n2, n3, (size_t)h->g.S, false);
}

// f_FluidstatsRs2D's sums over the physical field of the current state
// (src/pf_fluidstats.f90:827-958): out[0..20] the raw sums of u1u1 u2u2 u3u3 u1u2 u1u3
// u2u3, u^3 (3), u^4 (3) (laboratory frame), w^2 (3), w^3 (3), w^4 (3); out[21] max
// |u1|+|u2|+|u3|; out[22..24] max |w_i|.  The caller normalises as
// f_FluidstatsRsCollect does (src/pf_fluidstats.f90:960-1100).
extern "C" int pandora_realspace_stats(pandora_handle* h, double* out, int32_t n) {
    if (!h || !out || n < 25) return PANDORA_ERR_INVALID_ARG;
    // R-conv: the reference's u4..u6 in real space are d(u1,u2,u3)/dx1 (src/pf_rk3.f90:422-428,
    // 476-482, 538-544), and its vorticity moments are taken of those; so are these
    cudaSetDevice(h->dev);
    const size_t words = 32 * 32;
    if (!h->rsbuf) {
        if (cudaMalloc((void**)&h->rsbuf, sizeof(double) * words) != cudaSuccess) { cudaGetLastError(); return PANDORA_ERR_OOM; }
    }
    PD_CK(cudaMemsetAsync(h->rsbuf, 0, sizeof(double) * words, h->st));
    if (h->mixed) {
        const Member<float> mv = self_of<float>(h);
        PD_CK(launch_zpass_inv(h->g, &mv, 1, 0, h->st));
        PD_CK(launch_ypass_inv(h->g, &mv, 1, h->st));
        PD_CK(launch_xpass_stats(h->g, &mv, h->rsbuf, h->st));
    } else {
        const Member<double> mv = self_of<double>(h);
        PD_CK(launch_zpass_inv(h->g, &mv, 1, 0, h->st));
        PD_CK(launch_ypass_inv(h->g, &mv, 1, h->st));
        PD_CK(launch_xpass_stats(h->g, &mv, h->rsbuf, h->st));
    }
    std::vector<double> hb(words);
    PD_CK(cudaMemcpyAsync(hb.data(), h->rsbuf, sizeof(double) * words, cudaMemcpyDeviceToHost, h->st));
    PD_CK(cudaStreamSynchronize(h->st));
    for (int a = 0; a < 25; a++) out[a] = 0.0;
    for (int slot = 0; slot < 32; slot++) {
        for (int a = 0; a < 21; a++) out[a] += hb[(size_t)slot * 32 + a];
        for (int a = 21; a < 25; a++) out[a] = std::max(out[a], hb[(size_t)slot * 32 + a]);
    }
    return PANDORA_OK;
}

// TS_CORR's longitudinal autocorrelation (f_FluidstatsRs2D, src/pf_fluidstats.f90:933-945):
// r[l] = sum over the grid of u1(x) u1(x + l dx), l = 0..NX/2, with u1(x) in the laboratory
// frame for shear and u1(x + l dx) the stored component (the reference's temp_r1i before
// f_FluidstatsRsCollect divides it).  From the x co-spectrum P_m of the current state:
// r[l] = NX NY NZ sum_m c_m Re(P_m e^{-2 pi i m l / NX}), c_0 = 1, c_m = 2 (the -m half).
extern "C" int pandora_x_correlation(pandora_handle* h, double* r, int32_t n) {
    if (!h || !r) return PANDORA_ERR_INVALID_ARG;
    const int nx = h->g.nx, nl = nx / 2 + 1, nki = h->g.nki;
    if (n < nl) return PANDORA_ERR_INVALID_ARG;
    cudaSetDevice(h->dev);
    if (!h->rsbuf) {   // 1024 words: 2 NKI <= 684 for NX <= 1024
        if (cudaMalloc((void**)&h->rsbuf, sizeof(double) * 32 * 32) != cudaSuccess) { cudaGetLastError(); return PANDORA_ERR_OOM; }
    }
    if (h->mixed) PD_CK(launch_xcorr_cospec(self_of<float>(h), h->rsbuf, h->st));
    else PD_CK(launch_xcorr_cospec(self_of<double>(h), h->rsbuf, h->st));
    std::vector<double> P((size_t)2 * nki);
    PD_CK(cudaMemcpyAsync(P.data(), h->rsbuf, sizeof(double) * 2 * nki, cudaMemcpyDeviceToHost, h->st));
    PD_CK(cudaStreamSynchronize(h->st));
    const double npts = (double)h->g.R, w = 6.283185307179586476925286766559005768 / (double)nx;
    for (int l = 0; l < nl; l++) {
        double acc = 0.0;
        for (int m = 0; m < nki; m++) {
            const double th = w * (double)(((long long)m * l) % nx);   // the phase reduced exactly
            const double t = P[2 * m] * std::cos(th) + P[2 * m + 1] * std::sin(th);
            acc += m == 0 ? t : 2.0 * t;
        }
        r[l] = npts * acc;
    }
    return PANDORA_OK;
}

// p_StatsPrimary's sums over the particles (src/pp_stats.f90:119-200): out[0..5] the
// sums of up_i up_j (u1u1 u2u2 u3u3 u1u2 u1u3 u2u3), out[6] the sum of the particles'
// kinetic energy (1/2)(pi/6 dp^3 P_RHO)|up|^2; divided by P_NP_GLOBAL by the caller.
extern "C" int pandora_particle_stats(pandora_handle* h, double* out, int32_t n) {
    if (!h || !out || n < 7) return PANDORA_ERR_INVALID_ARG;
    if (!h->particles_on || h->P.np <= 0) return PANDORA_ERR_UNSUPPORTED;
    cudaSetDevice(h->dev);
    if (!h->rsbuf) {
        if (cudaMalloc((void**)&h->rsbuf, sizeof(double) * 32 * 32) != cudaSuccess) { cudaGetLastError(); return PANDORA_ERR_OOM; }
    }
    PD_CK(launch_particle_stats(h->P, h->P.np, h->p.p_rho, h->rsbuf, h->st));
    PD_CK(cudaMemcpyAsync(out, h->rsbuf, sizeof(double) * 7, cudaMemcpyDeviceToHost, h->st));
    PD_CK(cudaStreamSynchronize(h->st));
    return PANDORA_OK;
}

extern "C" int pandora_get_physical_velocity(pandora_handle* h, double* u1, double* u2, double* u3) {
    if (!h || !u1 || !u2 || !u3) return PANDORA_ERR_INVALID_ARG;
    if (!h->F.phys) return PANDORA_ERR_UNSUPPORTED;
    cudaSetDevice(h->dev);
    double* d[3] = {u1, u2, u3};
    if (h->mixed) {   // stored FP32: widened on the host
        std::vector<float> tmp((size_t)h->g.R);
        for (int c = 0; c < 3; c++) {
            PD_CK(cudaMemcpyAsync(tmp.data(), h->Ff.phys + c * h->g.R, sizeof(float) * h->g.R,
                                  cudaMemcpyDeviceToHost, h->st));
            PD_CK(cudaStreamSynchronize(h->st));
            for (long long q = 0; q < h->g.R; q++) d[c][q] = tmp[(size_t)q];
        }
        return PANDORA_OK;
    }
    for (int c = 0; c < 3; c++)
        PD_CK(cudaMemcpyAsync(d[c], h->F.phys + c * h->g.R, sizeof(double) * h->g.R, cudaMemcpyDeviceToHost, h->st));
    PD_CK(cudaStreamSynchronize(h->st));
    return PANDORA_OK;
}

extern "C" int pandora_check_status(pandora_handle* h) {
    if (!h) return PANDORA_ERR_INVALID_ARG;
    cudaSetDevice(h->dev);
    if (h->mixed) {
        const Member<float> self = self_of<float>(h);
        PD_CK(launch_check_finite(h->g, &self, 1, h->st));
    } else {
        const Member<double> self = self_of<double>(h);
        PD_CK(launch_check_finite(h->g, &self, 1, h->st));
    }
    PD_CK(cudaMemcpyAsync(h->clock_host, h->clock, sizeof(Clock), cudaMemcpyDeviceToHost, h->st));
    PD_CK(cudaStreamSynchronize(h->st));
    const unsigned int st = h->clock_host->status;
    h->clock_host->status = 0;
    PD_CK(cudaMemcpyAsync(&h->clock->status, &h->clock_host->status, sizeof(unsigned int),
                          cudaMemcpyHostToDevice, h->st));
    PD_CK(cudaStreamSynchronize(h->st));
    return status_to_rc(st);
}

extern "C" int pandora_launches_per_step(pandora_handle* h, int32_t* n) {
    if (!h || !n) return PANDORA_ERR_INVALID_ARG;
    if (!h->launches_per_step) {
        // count without launching: same sequence as enqueue_step
        const bool part = h->particles_on && h->P.np > 0;
        h->launches_per_step = 1 + 3 * (8 + (part ? 1 : 0)) + (part ? 5 : 0) + (h->g.shear ? (part ? 2 : 1) : 0);
    }
    *n = h->launches_per_step;
    return PANDORA_OK;
}

extern "C" int pandora_set_pass_timing(pandora_handle* h, int32_t passes) {
    if (!h || passes < 0 || passes > 0x3F) return PANDORA_ERR_INVALID_ARG;
    cudaSetDevice(h->dev);
    PD_CK(cudaStreamSynchronize(h->st));
    if (passes && !h->tev[0][0][0]) {
        for (auto& st3 : h->tev)
            for (auto& pr : st3)
                for (cudaEvent_t& e : pr) PD_CK(cudaEventCreate(&e));
    }
    h->timing = passes;
    for (auto& st3 : h->timed)
        for (bool& t : st3) t = false;
    drop_graph(h);   // the next step captures the graph with (or without) the event nodes
    return PANDORA_OK;
}

extern "C" int pandora_pass_times(pandora_handle* h, float* ms) {
    if (!h || !ms) return PANDORA_ERR_INVALID_ARG;
    cudaSetDevice(h->dev);
    PD_CK(cudaStreamSynchronize(h->st));
    for (int st = 0; st < 3; st++)
        for (int ps = 0; ps < 6; ps++) {
            float v = -1.0f;
            if ((h->timing & (1 << ps)) && h->timed[st][ps]) PD_CK(cudaEventElapsedTime(&v, h->tev[st][ps][0], h->tev[st][ps][1]));
            ms[st * 6 + ps] = v;
        }
    return PANDORA_OK;
}

template <class T> static int profile_pass_t(pandora_handle* h, int32_t pass, int32_t reps) {
    const bool part = h->particles_on && h->P.np > 0;
    const Member<T> self = self_of<T>(h);
    const Member<T>* M = &self;
    FieldsT<T> Fs = fields<T>(h);
    Fs.shell = h->shell_now;
    const Member<T> mv = member_of<T>(h, Fs);
    const Member<T>* Mv = &mv;
    for (int r = 0; r < reps; r++) {
        switch (pass) {
        case 1: PD_CK(launch_zpass_inv(h->g, M, 1, 2, h->st, (h->zmaps_ok && !h->mixed) ? &h->zmaps : nullptr)); break;
        case 2: PD_CK(launch_ypass_inv(h->g, M, 1, h->st)); break;
        case 3: PD_CK(launch_xpass(h->g, M, 1, part ? 1 : 0, 0, h->st)); break;
        case 4: PD_CK(launch_ypass_fwd(h->g, M, 1, h->st)); break;
        case 5: PD_CK(launch_zpass_fwd_update(h->g, M, 1, 2, 0, h->st)); break;
        case 6:
            if (!part) return PANDORA_ERR_INVALID_ARG;
            PD_CK(launch_particles(h->g, M, 1, h->P.np, h->pp.order, 2, h->st));
            break;
        case 7: PD_CK(launch_stats(h->g, Mv, 1, h->shell_now, h->st)); break;
        default: return PANDORA_ERR_INVALID_ARG;
        }
    }
    return PANDORA_OK;
}

extern "C" int pandora_profile_pass(pandora_handle* h, int32_t pass, int32_t reps) {
    if (!h || reps < 0) return PANDORA_ERR_INVALID_ARG;
    cudaSetDevice(h->dev);
    return h->mixed ? profile_pass_t<float>(h, pass, reps) : profile_pass_t<double>(h, pass, reps);
}

extern "C" int pandora_pass_bytes(pandora_handle* h, int32_t pass, double* bytes) {
    if (!h || !bytes) return PANDORA_ERR_INVALID_ARG;
    const Geo& g = h->g;
    const double c16 = (double)h->celem;          // one stored complex value
    const double r8 = (double)h->celem / 2.0;     // one stored real value
    const double S = (double)g.S;
    const double Z = (double)g.nz * g.nkj * g.nki;
    const double Y = (double)g.nz * g.ny * g.nki;
    const double R = (double)g.R;
    const bool part = h->particles_on && h->P.np > 0;
    switch (pass) {
    case 1: *bytes = c16 * (3 * S + pass_fields(g) * Z); break;   // 6 fields, 9 in the R-conv form
    case 2: *bytes = c16 * (pass_fields(g) * Z + pass_fields(g) * Y); break;
    case 3: *bytes = c16 * (pass_fields(g) * Y + 3 * Y) + (part ? r8 * 3 * R : 0.0); break;
    case 4: *bytes = c16 * (3 * Y + 3 * Z); break;
    case 5: *bytes = c16 * (3 * Z + 3 * S) + c16 * (3 * S + 6 * S + 6 * S); break;   // K5a + K5b
    case 6: {   // the field values the stencils need (each read once at most) and the particle state
        const double ord = (double)h->pp.order, np = (double)h->P.np;
        *bytes = part ? r8 * 3 * std::min(R, np * ord * ord * ord) + 8.0 * 24.0 * np : 0.0;
        break;
    }
    case 7: *bytes = c16 * 3 * S; break;
    default: return PANDORA_ERR_INVALID_ARG;
    }
    return PANDORA_OK;
}

extern "C" int pandora_frame(pandora_handle* h, double* bmat13, double* binv13) {
    if (!h || !bmat13 || !binv13) return PANDORA_ERR_INVALID_ARG;
    cudaSetDevice(h->dev);
    PD_CK(cudaMemcpyAsync(h->clock_host, h->clock, sizeof(Clock), cudaMemcpyDeviceToHost, h->st));
    PD_CK(cudaStreamSynchronize(h->st));
    *bmat13 = h->clock_host->b13;
    *binv13 = h->clock_host->bi13;
    return PANDORA_OK;
}

// ===========================================================================
// Batches of simulations (the ensemble server's device side; no counterpart in
// the reference).  A batch holds `capacity` slots of one class: grid size,
// precision, flow type (isotropic or BF-rot shear with its B110..B330), particles
// per member, interpolation order and forcing radius.  Each slot is a full
// simulation (its own fields, scratch pencils, clock, forcing and particles);
// what may differ between members is everything else: seeds, viscosity, dt, the
// forcing amplitude and time scale, the shear rate.  One step of the batch is a
// CUDA graph captured once over all slots: every kernel launch of the step
// serves every member (the member index is a grid dimension), and members at
// different step numbers advance side by side because each carries its own device
// clock.  Free slots carry an idle bit in their device clock and return at once.
// Admitting a member (seeding, clock reset) and finishing one (idle bit, copy of
// its statistics to pinned host memory) are enqueued in the batch's stream order
// and never wait on the host; the slot descriptors (kernel parameters) change, and
// the graph is re-captured, only when a member's constant parameters differ from
// those of its slot.  Every step and finish call records a ticket (an event) the
// host can poll.
// ===========================================================================
struct pandora_batch {
    pandora_params cls{};
    Geo g{};                               // class geometry (grid sizes and flow type)
    bool mixed = false;
    int cap = 0;
    int dev = 0;
    std::vector<pandora_handle*> m;        // the slots' simulations
    std::vector<int> active;
    std::vector<Member<double>> md;        // slot descriptors (FP64 form)
    std::vector<Member<float>> mf;         // slot descriptors (FP32-mixed form)
    bool dirty = true;                     // descriptors changed since the graph was captured
    std::vector<pandora_params> slot_p;    // the parameters each slot's descriptor was built from
    double* shell_host = nullptr;          // pinned [cap][shell_words]: statistics of finished members
    static constexpr int kTickets = 512;
    cudaEvent_t ev[kTickets] = {};
    long long ticket = 0;                  // number of tickets recorded
    double* shell = nullptr;               // [cap][shell_words]
    size_t nsh = 0;
    cudaStream_t st = nullptr, side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int launches_per_step = 0;
};

static void batch_release(pandora_batch* b) {
    if (!b) return;
    cudaSetDevice(b->dev);
    if (b->st) cudaStreamSynchronize(b->st);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (pandora_handle* h : b->m) release(h);
    for (cudaEvent_t e : b->ev)
        if (e) cudaEventDestroy(e);
    if (b->shell_host) cudaFreeHost(b->shell_host);
    cudaFree(b->shell);
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    if (b->ev_join) cudaEventDestroy(b->ev_join);
    if (b->side) cudaStreamDestroy(b->side);
    if (b->st) cudaStreamDestroy(b->st);
    delete b;
}

// The per-member parameters of a simulation (those a batch member may change).
static void derive_member(pandora_handle* h, const pandora_params* p) {
    h->p = *p;
    Geo& g = h->g;
    g.nu = p->f_nu;
    g.shear_s = p->f_deform_s;
    g.remesh_t = p->f_remesh_t;
    g.rk3_decide = (p->rk3_timestep == PANDORA_RK3_TIMESTEP_DECIDE) ? 1 : 0;
    h->sp.rk3_timestep = p->rk3_timestep; h->sp.f_type = p->f_type; h->sp.rk3_dt = p->rk3_dt;
    h->sp.rk3_cfl = p->rk3_cfl; h->sp.force_tf = p->force_tf; h->sp.f_deform_s = p->f_deform_s;
    h->sp.f_remesh_t = p->f_remesh_t;
    h->fp.tf = p->force_tf; h->fp.sigma = p->force_sigma; h->fp.stop = p->force_stop;
    h->fp.key = stream_key(p->seed_force, TAG_FORCE);
    h->pp.release = p->p_ts_release; h->pp.f_nu = p->f_nu;
    h->pp.p_rho = p->p_rho; h->pp.f_rho = p->f_rho;
}

// Do two parameter sets describe the same batch class?
static bool same_class(const pandora_params* a, const pandora_params* b) {
    const long long na = a->p_track_part ? a->p_np_global : 0, nb = b->p_track_part ? b->p_np_global : 0;
    return a->nodes_x == b->nodes_x && a->nodes_y == b->nodes_y && a->nodes_z == b->nodes_z &&
           a->precision == b->precision && a->f_type == b->f_type && a->ns_deformed == b->ns_deformed &&
           a->b110 == b->b110 && a->b220 == b->b220 && a->b330 == b->b330 && a->dealiasing == b->dealiasing && a->les_cutoff == b->les_cutoff &&
           a->rk3_viscous == b->rk3_viscous &&   // one update kernel per launch
           na == nb && (na == 0 || a->p_interp_order == b->p_interp_order) &&
           a->force_kf == b->force_kf;   // the forcing radius of the class geometry (mask kmag <= kf)
}

template <class T> static Member<T> slot_member(pandora_batch* b, int slot, int on) {
    pandora_handle* h = b->m[slot];
    FieldsT<T> F = fields<T>(h);
    F.shell = b->shell + (size_t)slot * b->nsh;
    Member<T> mm = member_of<T>(h, F);
    mm.active = on;
    return mm;
}
// Do two members of a class give the same slot descriptor?  (The descriptor holds
// the slot's buffers and the member's constant parameters: viscosity, time step,
// shear rate, forcing -- its random key only where forcing runs -- and particle
// properties; seeds of the initial field and particles are not in it.)
static bool same_descriptor(const pandora_params& a, const pandora_params& b) {
    const bool fa = a.force_stop > 0, fb = b.force_stop > 0;
    return a.f_nu == b.f_nu && a.f_deform_s == b.f_deform_s && a.f_remesh_t == b.f_remesh_t &&
           a.rk3_timestep == b.rk3_timestep && a.rk3_dt == b.rk3_dt && a.rk3_cfl == b.rk3_cfl &&
           a.force_stop == b.force_stop && (!fa || (a.force_tf == b.force_tf && a.force_sigma == b.force_sigma &&
                                                     a.seed_force == b.seed_force)) &&
           fa == fb && a.p_ts_release == b.p_ts_release && a.p_rho == b.p_rho && a.f_rho == b.f_rho;
}
// The slot's descriptor for the member now in it (re-capture only if it changed).
static void set_slot(pandora_batch* b, int slot, bool force = false) {
    pandora_handle* h = b->m[slot];
    if (!force && same_descriptor(b->slot_p[slot], h->p)) return;
    b->slot_p[slot] = h->p;
    if (b->mixed) b->mf[slot] = slot_member<float>(b, slot, 1);
    else b->md[slot] = slot_member<double>(b, slot, 1);
    b->dirty = true;
}
static cudaError_t record_ticket(pandora_batch* b) {
    const cudaError_t e = cudaEventRecord(b->ev[b->ticket % pandora_batch::kTickets], b->st);
    if (e == cudaSuccess) b->ticket++;
    return e;
}

template <class T> static int batch_enqueue_step(pandora_batch* b, int* nlaunch) {
    StepCtx<T> c{};
    c.g = &b->g;
    c.M = b->mixed ? (const Member<T>*)(const void*)b->mf.data() : (const Member<T>*)(const void*)b->md.data();
    c.B = b->cap;
    c.np = b->cls.p_track_part ? b->cls.p_np_global : 0;
    c.order = b->cls.p_interp_order;
    c.fp = &b->m[0]->fp;         // only its size (the forcing radius) is used at launch
    c.shell = b->shell;
    c.st = b->st;
    c.side = b->side;
    c.ev_fork = b->ev_fork;
    c.ev_join = b->ev_join;
    for (int s = 1; s <= 3; s++) {
        int rc = enqueue_stage_ctx(c, s, nlaunch);
        if (rc) return rc;
    }
    return PANDORA_OK;
}

extern "C" int pandora_batch_bytes(const pandora_params* p, int32_t capacity, int64_t* bytes) {
    if (!p || capacity < 1 || !bytes) return PANDORA_ERR_INVALID_ARG;
    int rc = validate(p);
    if (rc) return rc;
    const long long nx = p->nodes_x, ny = p->nodes_y, nz = p->nodes_z;
    const long long nki = nx / 3 + 1, nkj = 2 * (ny / 3) + 1, nkk = 2 * (nz / 3) + 1, nkip = (nki + 7) / 8 * 8;
    const long long S = nki * nkj * nkk, R = nx * ny * nz;
    const long long ce = p->precision == PANDORA_PREC_FP32_MIXED ? 8 : 16;
    const long long np = p->p_track_part ? p->p_np_global : 0;
    const long long nfb = (p->f_type == PANDORA_F_SHEAR_DNS && p->ns_deformed == PANDORA_NS_R_CONV) ? 9 : 6;
    long long per = ce * 6 * S + ce * nfb * nz * nkj * nkip + ce * nfb * nz * ny * nkip + ce * (nx + ny + nz);
    if (p->p_track_part) per += ce / 2 * 3 * R + 2 * 8 * 14 * np + 4 * np;
    per += 1 << 20;   // clock, forcing, shells, member descriptors, allocator granularity
    *bytes = per * capacity;
    return PANDORA_OK;
}

extern "C" int pandora_batch_create(const pandora_params* cls, int32_t capacity, pandora_batch** out) {
    if (!cls || !out || capacity < 1 || capacity > 4096) return PANDORA_ERR_INVALID_ARG;
    *out = nullptr;
    int rc = validate(cls);
    if (rc) return rc;
    // more than one member per launch needs the batched kernels of every axis length
    if (capacity > 1 && !(batched_length(cls->nodes_x) && batched_length(cls->nodes_y) && batched_length(cls->nodes_z)))
        return PANDORA_ERR_UNSUPPORTED;
    pandora_batch* b = new (std::nothrow) pandora_batch();
    if (!b) return PANDORA_ERR_OOM;
    cudaGetDevice(&b->dev);
    b->cls = *cls;
    b->mixed = cls->precision == PANDORA_PREC_FP32_MIXED;
    b->cap = capacity;
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming)) != cudaSuccess) {
        batch_release(b); return cuda_fail(e, "batch streams");
    }
    b->m.assign(capacity, nullptr);
    b->active.assign(capacity, 0);
    for (int i = 0; i < capacity; i++) {
        rc = pandora_create(cls, &b->m[i]);
        if (rc) { batch_release(b); return rc; }
        b->m[i]->st = b->st;      // every member's copies run in the batch's stream order
    }
    b->g = b->m[0]->g;
    b->nsh = shell_words(b->g);
    if (cudaMalloc((void**)&b->shell, sizeof(double) * b->nsh * capacity) != cudaSuccess ||
        cudaMallocHost((void**)&b->shell_host, sizeof(double) * b->nsh * capacity) != cudaSuccess) {
        cudaGetLastError(); batch_release(b); return PANDORA_ERR_OOM;
    }
    for (cudaEvent_t& ev : b->ev)
        if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) {
            batch_release(b); return cuda_fail(e, "batch events");
        }
    b->md.resize(b->mixed ? 0 : capacity);
    b->mf.resize(b->mixed ? capacity : 0);
    b->slot_p.assign(capacity, *cls);
    for (int i = 0; i < capacity; i++) {
        set_slot(b, i, true);
        if ((e = launch_set_idle(b->m[i]->clock, b->st)) != cudaSuccess) { batch_release(b); return cuda_fail(e, "idle"); }
    }
    if ((e = cudaStreamSynchronize(b->st)) != cudaSuccess) { batch_release(b); return cuda_fail(e, "batch"); }
    *out = b;
    return PANDORA_OK;
}

extern "C" int pandora_batch_destroy(pandora_batch* b) {
    if (!b) return PANDORA_ERR_INVALID_ARG;
    batch_release(b);
    return PANDORA_OK;
}

extern "C" int pandora_batch_capacity(pandora_batch* b, int32_t* capacity, int32_t* free_slots) {
    if (!b) return PANDORA_ERR_INVALID_ARG;
    int nfree = 0;
    for (int a : b->active) nfree += a ? 0 : 1;
    if (capacity) *capacity = b->cap;
    if (free_slots) *free_slots = nfree;
    return PANDORA_OK;
}

extern "C" int pandora_batch_admit(pandora_batch* b, const pandora_params* p, int32_t* slot) {
    if (!b || !p || !slot) return PANDORA_ERR_INVALID_ARG;
    int rc = validate(p);
    if (rc) return rc;
    if (!same_class(p, &b->cls)) return PANDORA_ERR_BAD_LAYOUT;
    int s = -1;
    if (*slot >= 0) {              // the caller's choice of a free slot
        if (*slot >= b->cap || b->active[*slot]) return PANDORA_ERR_INVALID_ARG;
        s = *slot;
    } else {
        for (int i = 0; i < b->cap; i++)
            if (!b->active[i]) { s = i; break; }
    }
    if (s < 0) return PANDORA_ERR_OOM;
    cudaSetDevice(b->dev);
    pandora_handle* h = b->m[s];
    derive_member(h, p);
    // a fresh simulation in the slot: zero state and registers, seeded field and
    // particles, clock at step 1 (all in the batch's stream order, no host wait)
    PD_CK(cudaMemsetAsync(h->fbuf, 0, h->celem * 6 * (size_t)h->g.S, h->st));
    PD_CK(cudaMemsetAsync(h->F.forcing, 0, sizeof(double2) * 3 * (size_t)h->nforce, h->st));
    rc = init_fluid_async(h);
    if (rc) return rc;
    if (h->particles_on && h->P.np > 0)
        PD_CK(launch_init_particles(h->g, h->P, stream_key(p->seed_particles, TAG_PART), p->p_dia_vals, h->st));
    // clock of step 1 at time 0 (frame of the initial state for shear)
    double b13 = 0.0, bi13 = 0.0;
    if (h->g.shear) update_b(h->g, 0, 0.0, b13, bi13);
    PD_CK(launch_reset_clock(h->clock, 1, 0.0, b13, bi13, h->st));
    set_slot(b, s);
    b->active[s] = 1;
    *slot = s;
    return PANDORA_OK;
}

extern "C" int pandora_batch_release(pandora_batch* b, int32_t slot) {
    if (!b || slot < 0 || slot >= b->cap || !b->active[slot]) return PANDORA_ERR_INVALID_ARG;
    cudaSetDevice(b->dev);
    PD_CK(launch_set_idle(b->m[slot]->clock, b->st));
    b->active[slot] = 0;
    return PANDORA_OK;
}

extern "C" int pandora_batch_finish(pandora_batch* b, int32_t slot, int64_t* ticket) {
    if (!b || slot < 0 || slot >= b->cap || !b->active[slot]) return PANDORA_ERR_INVALID_ARG;
    cudaSetDevice(b->dev);
    PD_CK(cudaMemcpyAsync(b->shell_host + (size_t)slot * b->nsh, b->shell + (size_t)slot * b->nsh,
                          sizeof(double) * b->nsh, cudaMemcpyDeviceToHost, b->st));
    PD_CK(launch_set_idle(b->m[slot]->clock, b->st));
    PD_CK(record_ticket(b));
    b->active[slot] = 0;
    if (ticket) *ticket = b->ticket - 1;
    return PANDORA_OK;
}

extern "C" int pandora_batch_ticket_done(pandora_batch* b, int64_t ticket, int32_t* done) {
    if (!b || !done || ticket < 0 || ticket >= b->ticket) return PANDORA_ERR_INVALID_ARG;
    // The slot of an old ticket may hold a newer record on the same stream; that one
    // completes after the old one, so its completion still implies the old ticket's
    // (a not-ready answer is then conservative).
    const cudaError_t e = cudaEventQuery(b->ev[ticket % pandora_batch::kTickets]);
    if (e == cudaErrorNotReady) { cudaGetLastError(); *done = 0; return PANDORA_OK; }
    PD_CK(e);
    *done = 1;
    return PANDORA_OK;
}

extern "C" int pandora_batch_result_stats(pandora_batch* b, int32_t slot, double* ek, int32_t kkmax, double* tke,
                                          double* eps) {
    if (!b || slot < 0 || slot >= b->cap) return PANDORA_ERR_INVALID_ARG;
    finish_stats(b->m[slot], b->shell_host + (size_t)slot * b->nsh, ek, kkmax, tke, eps);
    return PANDORA_OK;
}

extern "C" int pandora_batch_step(pandora_batch* b, int32_t nsteps, int64_t* ticket) {
    if (!b || nsteps < 0) return PANDORA_ERR_INVALID_ARG;
    cudaSetDevice(b->dev);
    if (b->dirty) {
        // the slot descriptors are kernel parameters: capture the step again and
        // update the executable graph (same topology) once earlier launches are done
        PD_CK(cudaStreamSynchronize(b->st));
        PD_CK(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
        int n = 0;
        int rc = b->mixed ? batch_enqueue_step<float>(b, &n) : batch_enqueue_step<double>(b, &n);
        cudaGraph_t gr = nullptr;
        cudaError_t e = cudaStreamEndCapture(b->st, &gr);
        if (rc) { if (gr) cudaGraphDestroy(gr); return rc; }
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
        bool updated = false;
        if (b->exec) {
            cudaGraphExecUpdateResultInfo info;
            updated = cudaGraphExecUpdate(b->exec, gr, &info) == cudaSuccess;
            if (!updated) { cudaGetLastError(); cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
        }
        if (!updated && (e = cudaGraphInstantiate(&b->exec, gr, 0)) != cudaSuccess) {
            cudaGraphDestroy(gr);
            return cuda_fail(e, "cudaGraphInstantiate");
        }
        if (b->graph) cudaGraphDestroy(b->graph);
        b->graph = gr;
        b->launches_per_step = n;
        b->dirty = false;
    }
    for (int i = 0; i < nsteps; i++) PD_CK(cudaGraphLaunch(b->exec, b->st));
    PD_CK(record_ticket(b));
    if (ticket) *ticket = b->ticket - 1;
    return PANDORA_OK;
}

extern "C" int pandora_batch_sync(pandora_batch* b) {
    if (!b) return PANDORA_ERR_INVALID_ARG;
    cudaSetDevice(b->dev);
    PD_CK(cudaStreamSynchronize(b->st));
    return PANDORA_OK;
}

extern "C" int pandora_batch_launches_per_step(pandora_batch* b, int32_t* n) {
    if (!b || !n) return PANDORA_ERR_INVALID_ARG;
    *n = b->launches_per_step;
    return PANDORA_OK;
}

static int batch_slot(pandora_batch* b, int32_t slot, pandora_handle** h) {
    if (!b || slot < 0 || slot >= b->cap) return PANDORA_ERR_INVALID_ARG;
    *h = b->m[slot];
    return PANDORA_OK;
}

extern "C" int pandora_batch_member_time(pandora_batch* b, int32_t slot, int32_t* tstep, double* simtime,
                                         double* dt) {
    pandora_handle* h;
    int rc = batch_slot(b, slot, &h);
    if (rc) return rc;
    cudaSetDevice(b->dev);
    PD_CK(cudaMemcpyAsync(h->clock_host, h->clock, sizeof(Clock), cudaMemcpyDeviceToHost, b->st));
    PD_CK(cudaStreamSynchronize(b->st));
    if (tstep) *tstep = h->clock_host->tstep;
    if (simtime) *simtime = h->clock_host->simtime;
    if (dt) *dt = h->clock_host->dt;
    return status_to_rc(h->clock_host->status);
}

extern "C" int pandora_batch_get_state(pandora_batch* b, int32_t slot, double* u1, double* u2, double* u3) {
    pandora_handle* h;
    int rc = batch_slot(b, slot, &h);
    if (rc) return rc;
    return pandora_get_state(h, u1, u2, u3);
}

extern "C" int pandora_batch_get_particles(pandora_batch* b, int32_t slot, int64_t np, double* xp, double* up,
                                           double* up_rk3, double* rk3, double* dp) {
    pandora_handle* h;
    int rc = batch_slot(b, slot, &h);
    if (rc) return rc;
    return pandora_get_particles(h, np, xp, up, up_rk3, rk3, dp);
}

extern "C" int pandora_batch_last_step_stats(pandora_batch* b, int32_t slot, double* ek, int32_t kkmax, double* tke,
                                             double* eps) {
    pandora_handle* h;
    int rc = batch_slot(b, slot, &h);
    if (rc) return rc;
    cudaSetDevice(b->dev);
    PD_CK(cudaMemcpyAsync(h->shell_host, b->shell + (size_t)slot * b->nsh, sizeof(double) * b->nsh,
                          cudaMemcpyDeviceToHost, b->st));
    PD_CK(cudaStreamSynchronize(b->st));
    finish_stats(h, h->shell_host, ek, kkmax, tke, eps);
    return PANDORA_OK;
}
