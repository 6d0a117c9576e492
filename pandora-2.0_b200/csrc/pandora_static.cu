// pandora_static.cu -- pandora_nonlinear_static: the nonlinear term of a
// spectral velocity field, computed without allocating any memory.
//
// Who needs it: callers that may not call cudaMalloc -- a driver that runs inside
// a pre-reserved memory pool or a memory budget it does not own, or code that
// must not take the device allocator's locks while other work is in flight.
// They pass their own input and output buffers; everything else this
// computation needs (the two pencil buffers between the transform passes, the
// twiddle tables and the scalar block the kernels read) lives in file-scope
// __device__ arrays of fixed size, sized for grids up to kStaticMaxN points per
// direction.  Every GPU that loads the library holds these arrays (about 16 MB)
// until the process exits.
//
// The arrays are shared by every call: calls that overlap on the GPU (two host
// threads, or two streams) race on them, so callers serialise their calls.  Each
// call overwrites the whole scratch before reading it, so nothing has to start at
// zero.  The first call on a device looks up the device addresses of the arrays
// (cudaGetSymbolAddress, with that device current) and caches them; make that
// first call before any stream capture on the device.
#include <cuda_runtime.h>
#include <math.h>
#include <mutex>
#include "pandora_internal.cuh"

namespace {

constexpr int kStaticMaxN = 64;                         // points per direction, at most
constexpr int kStaticMaxNkip = (kStaticMaxN / 3 + 1 + 7) / 8 * 8;
constexpr int kStaticMaxNkj = 2 * (kStaticMaxN / 3) + 1;
constexpr size_t kZbWords = (size_t)6 * kStaticMaxN * kStaticMaxNkj * kStaticMaxNkip;
constexpr size_t kYbWords = (size_t)6 * kStaticMaxN * kStaticMaxN * kStaticMaxNkip;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double2 g_static_zb[kZbWords];
static __device__ __align__(256) double2 g_static_yb[kYbWords];
static __device__ __align__(256) double2 g_static_tw[3 * kStaticMaxN];
static __device__ __align__(256) pd::Clock g_static_clock;

struct StaticPtrs {
    bool ready = false;
    double2* zb = nullptr;
    double2* yb = nullptr;
    double2* tw = nullptr;
    pd::Clock* clock = nullptr;
};
StaticPtrs g_ptrs[kMaxDevices];
std::mutex g_mutex;

// Device addresses of the static arrays on the current device (set up once per device).
int static_ptrs(int dev, StaticPtrs** out) {
    if (dev < 0 || dev >= kMaxDevices) return PANDORA_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_mutex);
    StaticPtrs& s = g_ptrs[dev];
    if (!s.ready) {
        cudaError_t e;
        if ((e = cudaGetSymbolAddress((void**)&s.zb, g_static_zb)) != cudaSuccess ||
            (e = cudaGetSymbolAddress((void**)&s.yb, g_static_yb)) != cudaSuccess ||
            (e = cudaGetSymbolAddress((void**)&s.tw, g_static_tw)) != cudaSuccess ||
            (e = cudaGetSymbolAddress((void**)&s.clock, g_static_clock)) != cudaSuccess) {
            cudaGetLastError();
            return pd::cuda_fail_msg(e, "pandora_nonlinear_static: cudaGetSymbolAddress");
        }
        if ((e = cudaMemset(s.clock, 0, sizeof(pd::Clock))) != cudaSuccess) {
            cudaGetLastError();
            return pd::cuda_fail_msg(e, "pandora_nonlinear_static: clearing the scalar block");
        }
        s.ready = true;
    }
    *out = &s;
    return PANDORA_OK;
}

}  // namespace

// Declared in include/pandora_gpu.h.
extern "C" int pandora_nonlinear_static(const pandora_params* p, const double* u1, const double* u2,
                                        const double* u3, double* n1, double* n2, double* n3,
                                        void* cuda_stream) {
    if (!p || !u1 || !u2 || !u3 || !n1 || !n2 || !n3) return PANDORA_ERR_INVALID_ARG;
    if (p->f_type != PANDORA_F_ISOTROPIC || p->precision != PANDORA_PREC_FP64 || p->dealiasing != PANDORA_DEALIASING_23)
        return PANDORA_ERR_UNSUPPORTED;
    const int nx = p->nodes_x, ny = p->nodes_y, nz = p->nodes_z;
    if (nx > kStaticMaxN || ny > kStaticMaxN || nz > kStaticMaxN) return PANDORA_ERR_BAD_LAYOUT;
    if (!pd::supported_length(nx) || !pd::supported_length(ny) || !pd::supported_length(nz))
        return PANDORA_ERR_BAD_LAYOUT;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); return PANDORA_ERR_NO_DEVICE; }
    StaticPtrs* sp = nullptr;
    int rc = static_ptrs(dev, &sp);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)cuda_stream;

    pd::Geo g{};
    g.nx = nx; g.ny = ny; g.nz = nz;
    g.ki = nx / 3; g.kj = ny / 3; g.kk = nz / 3;
    g.nki = g.ki + 1; g.nkj = 2 * g.kj + 1; g.nkk = 2 * g.kk + 1;
    g.nkip = (g.nki + 7) / 8 * 8;
    g.S = (long long)g.nki * g.nkj * g.nkk;
    g.R = (long long)nx * ny * nz;
    g.norm = 1.0 / ((double)nx * (double)ny * (double)nz);
    g.nu = p->f_nu;
    g.dx = 6.283185307179586476925286766559005768 / nx;
    g.dy = 6.283185307179586476925286766559005768 / ny;
    g.dz = 6.283185307179586476925286766559005768 / nz;

    // twiddles tw[e] = exp(-2 pi i e / N) from a fixed host table (no heap)
    double2 tw[3 * kStaticMaxN];
    const int lens[3] = {nx, ny, nz};
    int off = 0;
    for (int d = 0; d < 3; d++) {
        for (int q = 0; q < lens[d]; q++) {
            const long double a = 6.283185307179586476925286766559005768L * (long double)q / (long double)lens[d];
            tw[off + q] = make_double2((double)cosl(a), -(double)sinl(a));
        }
        off += lens[d];
    }
    cudaError_t e;
    if ((e = cudaMemcpyAsync(sp->tw, tw, sizeof(double2) * off, cudaMemcpyHostToDevice, st)) != cudaSuccess) {
        cudaGetLastError();
        return pd::cuda_fail_msg(e, "pandora_nonlinear_static: twiddle upload");
    }
    if ((e = pd::configure_kernels<double>(g)) != cudaSuccess) {
        cudaGetLastError();
        return pd::cuda_fail_msg(e, "pandora_nonlinear_static: kernel attributes");
    }
    pd::Fields F{};
    F.u[0] = (double2*)u1; F.u[1] = (double2*)u2; F.u[2] = (double2*)u3;
    F.rk[0] = (double2*)n1; F.rk[1] = (double2*)n2; F.rk[2] = (double2*)n3;
    F.zb = sp->zb;
    F.yb = sp->yb;
    F.tw_x = sp->tw; F.tw_y = sp->tw + nx; F.tw_z = sp->tw + nx + ny;
    F.clock = sp->clock;
    pd::Member<double> m{};
    m.F = F;
    m.g = g;
    m.active = 1;
    const pd::Member<double>* M = &m;   // passed to the kernels by value
    // the same five passes as the step, with the last one storing NL-hat instead of updating
    if ((e = pd::launch_zpass_inv(g, M, 1, 0, st)) != cudaSuccess ||
        (e = pd::launch_ypass_inv(g, M, 1, st)) != cudaSuccess ||
        (e = pd::launch_xpass(g, M, 1, 0, 0, st)) != cudaSuccess ||
        (e = pd::launch_ypass_fwd(g, M, 1, st)) != cudaSuccess ||
        (e = pd::launch_zpass_fwd_update(g, M, 1, 1, 1, st)) != cudaSuccess) {
        cudaGetLastError();
        return pd::cuda_fail_msg(e, "pandora_nonlinear_static: transform pass launch");
    }
    // the host twiddle table must outlive the copy
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) {
        cudaGetLastError();
        return pd::cuda_fail_msg(e, "pandora_nonlinear_static: stream synchronise");
    }
    return PANDORA_OK;
}
