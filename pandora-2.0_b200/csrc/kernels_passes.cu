// kernels_passes.cu -- the five HBM passes of one RK3 stage on sm_100a: dispatch on the
// transform length to the per-length launchers (passes_n.cuh, instantiated by the
// passes_n*.cu files), the per-mode RK update (K5b), the tensor maps of the staged K1
// and the FP64 <-> FP32 conversions of the mixed form's boundary.  The kernels and
// the pass structure are described in passes_kernels.cuh.
#include "passes_kernels.cuh"

namespace pd {

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

bool batched_length(int n) {
    switch (n) {
#define PD_CASE(N) \
    case N: return batch_len<N>();
        PD_FOR_EACH_N(PD_CASE)
#undef PD_CASE
    default:
        return false;
    }
}

template <class T> cudaError_t configure_kernels(const Geo& g) {
    cudaError_t e;
#define PD_C(N)                                                 \
    if (g.nx == N || g.ny == N || g.nz == N) {                  \
        if ((e = configure_n<N, T>(g)) != cudaSuccess) return e; \
    }
    PD_FOR_EACH_N(PD_C)
#undef PD_C
    return cudaSuccess;
}

template <class T>
cudaError_t launch_zpass_inv(const Geo& g, const Member<T>* M, int B, int stage, cudaStream_t st, const ZMaps* maps) {
    // DEALIASING 2/3: f_RK3PrepareRealSpace first zeroes the modes outside the cutoff
    // (src/pf_rk3.f90:269-277): k_dealias writes those zeros (it reads nothing) ahead of
    // K1, whose loads then carry no mask test
    if (g.dealias_cut > 0.0) {
        const cudaError_t e = launch_dealias(g, M, B, st);
        if (e != cudaSuccess) return e;
    }
    switch (g.nz) {
#define PD_L(N) case N: return zpass_inv_n<N, T>(g, M, B, stage, st, maps);
        PD_FOR_EACH_N(PD_L)
#undef PD_L
    default: return cudaErrorInvalidValue;
    }
}

template <class T> cudaError_t launch_ypass_inv(const Geo& g, const Member<T>* M, int B, cudaStream_t st) {
    switch (g.ny) {
#define PD_L(N) case N: return ypass_inv_n<N, T>(g, M, B, st);
        PD_FOR_EACH_N(PD_L)
#undef PD_L
    default: return cudaErrorInvalidValue;
    }
}

template <class T>
cudaError_t launch_xpass(const Geo& g, const Member<T>* M, int B, int want_phys, int want_cfl, cudaStream_t st) {
    switch (g.nx) {
#define PD_L(N) case N: return xpass_n<N, T>(g, M, B, want_phys, want_cfl, st);
        PD_FOR_EACH_N(PD_L)
#undef PD_L
    default: return cudaErrorInvalidValue;
    }
}

template <class T>
cudaError_t launch_xpass_stats(const Geo& g, const Member<T>* M, double* rs, cudaStream_t st) {
    switch (g.nx) {
#define PD_L(N) case N: return xpass_stats_n<N, T>(g, M, rs, st);
        PD_FOR_EACH_N(PD_L)
#undef PD_L
    default: return cudaErrorInvalidValue;
    }
}

template <class T> cudaError_t launch_ypass_fwd(const Geo& g, const Member<T>* M, int B, cudaStream_t st) {
    switch (g.ny) {
#define PD_L(N) case N: return ypass_fwd_n<N, T>(g, M, B, st);
        PD_FOR_EACH_N(PD_L)
#undef PD_L
    default: return cudaErrorInvalidValue;
    }
}

template <class T>
cudaError_t launch_zpass_fwd_update(const Geo& g, const Member<T>* M, int B, int stage, int mode, cudaStream_t st) {
    cudaError_t e = cudaErrorInvalidValue;
    switch (g.nz) {
#define PD_L(N)                                    \
    case N:                                        \
        e = zpass_fwd_n<N, T>(g, M, B, mode, st);  \
        break;
        PD_FOR_EACH_N(PD_L)
#undef PD_L
    default: return cudaErrorInvalidValue;
    }
    if (e || mode == 1) return e;
    return for_member_sets(M, B, [&](const auto& ms, int nb) {
        constexpr int CAP = std::decay_t<decltype(ms)>::cap;
        const dim3 grid((unsigned)((g.S + 255) / 256), nb);
        if (g.rrot) k_rk_update<2, T, CAP><<<grid, 256, 0, st>>>(ms, stage);
        else if (g.shear) k_rk_update<1, T, CAP><<<grid, 256, 0, st>>>(ms, stage);
        else if (g.visc_if) k_rk_update<3, T, CAP><<<grid, 256, 0, st>>>(ms, stage);
        else k_rk_update<0, T, CAP><<<grid, 256, 0, st>>>(ms, stage);
    });
}

// Tensor maps of the staged K1 (host).  The encoder is the driver's
// cuTensorMapEncodeTiled, looked up through the runtime (no link against libcuda).
typedef CUresult (*TensorMapEncodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                         const cuuint64_t*, const cuuint32_t*, const cuuint32_t*,
                                         CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                         CUtensorMapFloatOOBfill);

cudaError_t make_zmaps(const Geo& g, double2* const* u, ZMaps* out, bool* ok) {
    *ok = false;
    int bk = 0;
    switch (g.nz) {
#define PD_L(N)                                               \
    case N:                                                   \
        if constexpr (ZStage<N>::enabled) bk = ZStage<N>::BK; \
        break;
        PD_FOR_EACH_N(PD_L)
#undef PD_L
    default: break;
    }
    if (bk == 0) return cudaSuccess;
    static TensorMapEncodeTiled encode = nullptr;
    if (!encode) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn) {
            cudaGetLastError();
            return cudaSuccess;
        }
        encode = (TensorMapEncodeTiled)fn;
    }
    // u_c as a 3-D tensor of doubles: dim 0 the 2 NKK reals of a k row, dim 1 j, dim 2 i
    const cuuint64_t dims[3] = {(cuuint64_t)2 * g.nkk, (cuuint64_t)g.nkj, (cuuint64_t)g.nki};
    const cuuint64_t strides[2] = {(cuuint64_t)2 * g.nkk * sizeof(double),
                                   (cuuint64_t)2 * g.nkk * g.nkj * sizeof(double)};
    const cuuint32_t box[3] = {(cuuint32_t)(2 * bk), 1u, 8u};
    const cuuint32_t estr[3] = {1u, 1u, 1u};
    for (int c = 0; c < 3; c++) {
        if (encode(&out->u[c], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, (void*)u[c], dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return cudaSuccess;
    }
    *ok = true;
    return cudaSuccess;
}

// conversions at the FP64 boundary of the FP32-mixed form
__global__ void k_to_f32(const double2* __restrict__ in, float2* __restrict__ out, long long n) {
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        out[q] = make_float2((float)in[q].x, (float)in[q].y);
}
__global__ void k_to_f64(const float2* __restrict__ in, double2* __restrict__ out, long long n) {
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        out[q] = make_double2(in[q].x, in[q].y);
}
static unsigned conv_blocks(long long n) {
    const long long b = (n + 255) / 256;
    return (unsigned)(b < 4096 ? (b > 0 ? b : 1) : 4096);
}
cudaError_t launch_convert(const double2* in, float2* out, long long n, cudaStream_t st) {
    k_to_f32<<<conv_blocks(n), 256, 0, st>>>(in, out, n);
    return cudaGetLastError();
}
cudaError_t launch_convert(const float2* in, double2* out, long long n, cudaStream_t st) {
    k_to_f64<<<conv_blocks(n), 256, 0, st>>>(in, out, n);
    return cudaGetLastError();
}

#define PD_INST(T)                                                                                       \
    template cudaError_t configure_kernels<T>(const Geo&);                                               \
    template cudaError_t launch_zpass_inv<T>(const Geo&, const Member<T>*, int, int, cudaStream_t, const ZMaps*); \
    template cudaError_t launch_ypass_inv<T>(const Geo&, const Member<T>*, int, cudaStream_t);           \
    template cudaError_t launch_xpass<T>(const Geo&, const Member<T>*, int, int, int, cudaStream_t);     \
    template cudaError_t launch_xpass_stats<T>(const Geo&, const Member<T>*, double*, cudaStream_t);    \
    template cudaError_t launch_ypass_fwd<T>(const Geo&, const Member<T>*, int, cudaStream_t);           \
    template cudaError_t launch_zpass_fwd_update<T>(const Geo&, const Member<T>*, int, int, int, cudaStream_t);
PD_INST(double)
PD_INST(float)
#undef PD_INST

}  // namespace pd
