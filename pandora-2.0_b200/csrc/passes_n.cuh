// passes_n.cuh -- the launchers of the five passes for one transform length N (host
// code), instantiated per group of lengths by the passes_n*.cu files.
#pragma once
#include "passes_kernels.cuh"

namespace pd {

template <int N, class T, int LPW = 1> static size_t smem_kx() {
    return sizeof(typename Cplx<T>::type) * ((size_t)Cfg<N>::NWX * LPW * 3 * xas<N>());
}

// CTAs of `kernel` resident on the whole device at once.
template <typename K> static long long resident_ctas(K kernel, int threads, size_t smem) {
    int dev = 0, nsm = 1, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem) != cudaSuccess || per < 1) {
        cudaGetLastError();
        per = 1;
    }
    return (long long)nsm * per;
}

template <typename K> static cudaError_t set_smem(K kernel, size_t bytes) {
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

#define PD_CAP(S) std::decay_t<decltype(S)>::cap

// Dynamic shared memory limits of the kernels of length N that the geometry uses, for
// member sets of CAP.
template <int N, class T, int CAP> static cudaError_t configure_cap(const Geo& g) {
    cudaError_t e;
    if constexpr (cube_len<N, T>()) {
        if (is_cube(g, N)) {
            if ((e = set_smem(k_zpass_inv<N, 0, T, CAP, N>, TCfg<N>::template smem<T>()))) return e;
            if ((e = set_smem(k_zpass_inv<N, 1, T, CAP, N>, TCfg<N>::template smem<T>()))) return e;
            if ((e = set_smem(k_zpass_inv<N, 2, T, CAP, N>, TCfg<N>::template smem<T>()))) return e;
            if ((e = set_smem(k_zpass_inv<N, 3, T, CAP, N>, TCfg<N>::template smem<T>()))) return e;
            if ((e = set_smem(k_ypass_inv<N, T, CAP, N>, TCfg<N, true>::template smem<T>()))) return e;
            if ((e = set_smem(k_ypass_fwd<N, T, CAP, N>, TCfg<N, true>::template smem<T>()))) return e;
        }
    }
    if (g.nz == N) {
        if ((e = set_smem(k_zpass_inv<N, 0, T, CAP>, TCfg<N>::template smem<T>()))) return e;
        if ((e = set_smem(k_zpass_inv<N, 1, T, CAP>, TCfg<N>::template smem<T>()))) return e;
        if ((e = set_smem(k_zpass_inv<N, 2, T, CAP>, TCfg<N>::template smem<T>()))) return e;
        if ((e = set_smem(k_zpass_inv<N, 3, T, CAP>, TCfg<N>::template smem<T>()))) return e;
        if ((e = set_smem(k_zpass_fwd<N, T, CAP>, TCfg<N, true>::template smem<T>()))) return e;
    }
    if (g.ny == N) {
        if ((e = set_smem(k_ypass_inv<N, T, CAP>, TCfg<N, true>::template smem<T>()))) return e;
        if ((e = set_smem(k_ypass_fwd<N, T, CAP>, TCfg<N, true>::template smem<T>()))) return e;
    }
    if (g.nx == N) {
        if ((e = set_smem(k_xpass<N, T, CAP>, smem_kx<N, T>()))) return e;
        if constexpr (xlpw_len<N>()) {
            if ((e = set_smem(k_xpass<N, T, CAP, false, 2>, smem_kx<N, T, 2>()))) return e;
            if ((e = set_smem(k_xpass<N, T, CAP, false, 4>, smem_kx<N, T, 4>()))) return e;
        }
        if (g.rconv && (e = set_smem(k_xpass_conv<N, T, CAP>, ConvCfg<N, T>::smem))) return e;
    }
    return cudaSuccess;
}

template <int N, class T> cudaError_t configure_n(const Geo& g) {
    cudaError_t e;
    if constexpr (std::is_same<T, double>::value && ZStage<N>::enabled) {
        if (g.nz == N) {
            if ((e = set_smem(k_zpass_inv_tma<N, 0>, ZStage<N>::smem))) return e;
            if ((e = set_smem(k_zpass_inv_tma<N, 1>, ZStage<N>::smem))) return e;
            if ((e = set_smem(k_zpass_inv_tma<N, 2>, ZStage<N>::smem))) return e;
            if ((e = set_smem(k_zpass_inv_tma<N, 3>, ZStage<N>::smem))) return e;
        }
    }
    if ((e = configure_cap<N, T, 1>(g))) return e;
    if constexpr (batch_len<N>()) {
        if ((e = configure_cap<N, T, kBatchChunk>(g))) return e;
    }
    return cudaSuccess;
}

// K1 (z length N): the staged kernel for a single FP64 simulation with tensor maps, else
// the element-wise kernel of the flow's form.
template <int N, class T>
cudaError_t zpass_inv_n(const Geo& g, const Member<T>* M, int B, int stage, cudaStream_t st, const ZMaps* maps) {
    if constexpr (std::is_same<T, double>::value && ZStage<N>::enabled) {
        if (maps && B == 1) {
            MemberSet<double, 1> one;
            one.m[0] = M[0];
            const dim3 grid(TCfg<N>::template tiles<double>(g), g.nkj);
            constexpr int NT = TCfg<N>::template nt<double>();
            constexpr size_t sm = ZStage<N>::smem;
            if (!g.shear) k_zpass_inv_tma<N, 0><<<grid, NT, sm, st>>>(one, *maps, stage);
            else if (!g.rrot) k_zpass_inv_tma<N, 1><<<grid, NT, sm, st>>>(one, *maps, stage);
            else if (!g.rconv) k_zpass_inv_tma<N, 2><<<grid, NT, sm, st>>>(one, *maps, stage);
            else k_zpass_inv_tma<N, 3><<<grid, NT, sm, st>>>(one, *maps, stage);
            return cudaGetLastError();
        }
    }
    return for_member_sets(M, B, [&](const auto& ms, int nb) {
        constexpr int CAP = PD_CAP(ms);
        if constexpr (CAP == 1 || batch_len<N>()) {
            const dim3 grid(pass_fields(g) * nb, TCfg<N>::template tiles<T>(g), g.nkj);
            constexpr int NT = TCfg<N>::template nt<T>();
            const size_t sm = TCfg<N>::template smem<T>();
            auto go = [&](auto kern) {
                const long long pf = CAP == 1 ? resident_ctas(kern, NT, sm) : 0;
                kern<<<grid, NT, sm, st>>>(ms, stage, pf);
            };
            auto form = [&](auto cn) {
                constexpr int CN = decltype(cn)::value;
                if (!g.shear) go(k_zpass_inv<N, 0, T, CAP, CN>);
                else if (!g.rrot) go(k_zpass_inv<N, 1, T, CAP, CN>);
                else if (!g.rconv) go(k_zpass_inv<N, 2, T, CAP, CN>);
                else go(k_zpass_inv<N, 3, T, CAP, CN>);
            };
            if constexpr (cube_len<N, T>()) {
                if (is_cube(g, N)) { form(std::integral_constant<int, N>{}); return; }
            }
            form(std::integral_constant<int, 0>{});
        }
    });
}

template <int N, class T> cudaError_t ypass_inv_n(const Geo& g, const Member<T>* M, int B, cudaStream_t st) {
    return for_member_sets(M, B, [&](const auto& ms, int nb) {
        constexpr int CAP = PD_CAP(ms);
        if constexpr (CAP == 1 || batch_len<N>()) {
            const dim3 grid(TCfg<N, true>::template tiles<T>(g), g.nz, pass_fields(g) * nb);
            constexpr int NT = TCfg<N, true>::template nt<T>();
            constexpr size_t sm = TCfg<N, true>::template smem<T>();
            if constexpr (cube_len<N, T>()) {
                if (is_cube(g, N)) { k_ypass_inv<N, T, CAP, N><<<grid, NT, sm, st>>>(ms, pass_fields(g)); return; }
            }
            k_ypass_inv<N, T, CAP><<<grid, NT, sm, st>>>(ms, pass_fields(g));
        }
    });
}

template <int N, class T>
cudaError_t xpass_n(const Geo& g, const Member<T>* M, int B, int want_phys, int want_cfl, cudaStream_t st) {
    const long long lines = (long long)g.ny * g.nz;
    return for_member_sets(M, B, [&](const auto& ms, int nb) {
        constexpr int CAP = PD_CAP(ms);
        if constexpr (CAP == 1 || batch_len<N>()) {
            if (g.rconv) {   // R-conv: its own x pass
                constexpr int NW = ConvCfg<N, T>::NW;
                const long long nl = (lines + NW - 1) / NW;
                const long long pf = CAP == 1 ? NW * resident_ctas(k_xpass_conv<N, T, CAP>, 32 * NW, ConvCfg<N, T>::smem) : 0;
                k_xpass_conv<N, T, CAP><<<dim3((unsigned)nl, nb), 32 * NW, ConvCfg<N, T>::smem, st>>>(ms, want_phys,
                                                                                                  want_cfl, pf);
                return;
            }
            auto go = [&](auto lpwc) {
                constexpr int LPW = decltype(lpwc)::value;
                constexpr int LB = Cfg<N>::NWX * LPW;   // lines per CTA
                const long long nl = (lines + LB - 1) / LB;
                // L2 prefetch distance: one wave of resident CTAs (single simulations)
                const long long pf = CAP == 1 ? LB * resident_ctas(k_xpass<N, T, CAP, false, LPW>, 32 * Cfg<N>::NWX,
                                                                   smem_kx<N, T, LPW>())
                                              : 0;
                k_xpass<N, T, CAP, false, LPW><<<dim3((unsigned)nl, nb), 32 * Cfg<N>::NWX, smem_kx<N, T, LPW>(), st>>>(
                    ms, want_phys, want_cfl, pf, nullptr);
            };
            if constexpr (xlpw_len<N>()) {
                const int lpw = g.xlpw > 0 ? g.xlpw : default_xlpw<N, T, CAP>();
                if (lpw == 4) go(std::integral_constant<int, 4>{});
                else if (lpw == 2) go(std::integral_constant<int, 2>{});
                else go(std::integral_constant<int, 1>{});
            } else {
                go(std::integral_constant<int, 1>{});
            }
        }
    });
}

// The x pass of the real-space statistics (single simulation): the moments of every
// point into `rs` (kRsSlots x kRsWords doubles, zeroed by the caller).
template <int N, class T> cudaError_t xpass_stats_n(const Geo& g, const Member<T>* M, double* rs, cudaStream_t st) {
    const long long lines = (long long)g.ny * g.nz;
    cudaError_t e = set_smem(k_xpass<N, T, 1, true>, smem_kx<N, T>());
    if (e) return e;
    MemberSet<T, 1> ms;
    ms.m[0] = M[0];
    const long long nl = (lines + Cfg<N>::NWX - 1) / Cfg<N>::NWX;
    k_xpass<N, T, 1, true><<<dim3((unsigned)nl, 1), 32 * Cfg<N>::NWX, smem_kx<N, T>(), st>>>(ms, 0, 0, 0, rs);
    return cudaGetLastError();
}

template <int N, class T> cudaError_t ypass_fwd_n(const Geo& g, const Member<T>* M, int B, cudaStream_t st) {
    return for_member_sets(M, B, [&](const auto& ms, int nb) {
        constexpr int CAP = PD_CAP(ms);
        if constexpr (CAP == 1 || batch_len<N>()) {
            const dim3 grid(TCfg<N, true>::template tiles<T>(g), g.nz, 3 * nb);
            constexpr int NT = TCfg<N, true>::template nt<T>();
            constexpr size_t sm = TCfg<N, true>::template smem<T>();
            if constexpr (cube_len<N, T>()) {
                if (is_cube(g, N)) { k_ypass_fwd<N, T, CAP, N><<<grid, NT, sm, st>>>(ms); return; }
            }
            k_ypass_fwd<N, T, CAP><<<grid, NT, sm, st>>>(ms);
        }
    });
}

// K5a: forward z transforms (mode 1: NL-hat into rk, the transform test hook).
template <int N, class T>
cudaError_t zpass_fwd_n(const Geo& g, const Member<T>* M, int B, int mode, cudaStream_t st) {
    return for_member_sets(M, B, [&](const auto& ms, int nb) {
        constexpr int CAP = PD_CAP(ms);
        if constexpr (CAP == 1 || batch_len<N>())
            k_zpass_fwd<N, T, CAP><<<dim3(TCfg<N, true>::template tiles<T>(g), g.nkj, 3 * nb),
                                     TCfg<N, true>::template nt<T>(), TCfg<N, true>::template smem<T>(), st>>>(ms, mode);
    });
}
#undef PD_CAP

#define PD_PASSES_INST_T(N, T)                                                                            \
    template cudaError_t configure_n<N, T>(const Geo&);                                                   \
    template cudaError_t zpass_inv_n<N, T>(const Geo&, const Member<T>*, int, int, cudaStream_t, const ZMaps*); \
    template cudaError_t ypass_inv_n<N, T>(const Geo&, const Member<T>*, int, cudaStream_t);              \
    template cudaError_t xpass_n<N, T>(const Geo&, const Member<T>*, int, int, int, cudaStream_t);        \
    template cudaError_t xpass_stats_n<N, T>(const Geo&, const Member<T>*, double*, cudaStream_t);        \
    template cudaError_t ypass_fwd_n<N, T>(const Geo&, const Member<T>*, int, cudaStream_t);              \
    template cudaError_t zpass_fwd_n<N, T>(const Geo&, const Member<T>*, int, int, cudaStream_t);
#define PD_PASSES_INST(N) PD_PASSES_INST_T(N, double) PD_PASSES_INST_T(N, float)

}  // namespace pd
