// march.cu -- instantiations of the persistent IRK march kernel for one Ntau
// (PCC_MARCH_N, set by the build: one translation unit per Ntau so that the
// fifteen shapes compile in parallel) and, with PCC_MARCH_DISPATCH, the
// launcher that selects among them.
#include "pcc_internal.h"

namespace pcc {

namespace {

template <int N, int S>
constexpr int min_blocks()
{
    // The radix-8 RHS needs ~230 registers per thread without spilling, so a
    // 128-thread CTA reaches two resident CTAs per SM and wider CTAs one.
    constexpr int nt = MarchShape<N, S>::NT;
    return nt <= 128 ? 2 : 1;
}

template <int N, int S>
cudaError_t launch_shape(const MarchParams& P, int max_ctas, cudaStream_t st, MarchLaunchInfo* info)
{
    using K = MarchShape<N, S>;
    auto kern = march_kernel<N, S, min_blocks<N, S>()>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)K::SMEM);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0, per_sm = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, K::NT, K::SMEM)) != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    int ctas = sms * per_sm;
    if (max_ctas > 0 && ctas > max_ctas) ctas = max_ctas;
    const int needed = (P.n_items + K::SPC - 1) / K::SPC;
    if (ctas > needed) ctas = needed;
    if (ctas < 1) ctas = 1;
    if (info) {
        info->ctas = ctas;
        info->sweeps_per_cta = K::SPC;
        info->threads = K::NT;
        info->smem = K::SMEM;
        info->ctas_per_sm = per_sm;
    }
    kern<<<ctas, K::NT, K::SMEM, st>>>(P);
    return cudaGetLastError();
}

template <int N>
cudaError_t launch_n(int stages, const MarchParams& P, int max_ctas, cudaStream_t st, MarchLaunchInfo* info)
{
    switch (stages) {
        case 1: return launch_shape<N, 1>(P, max_ctas, st, info);
        case 2: return launch_shape<N, 2>(P, max_ctas, st, info);
        case 3: return launch_shape<N, 3>(P, max_ctas, st, info);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace

#ifdef PCC_MARCH_N
#define PCC_CAT2(a, b) a##b
#define PCC_CAT(a, b) PCC_CAT2(a, b)
cudaError_t PCC_CAT(launch_march_n, PCC_MARCH_N)(int stages, const MarchParams& P, int max_ctas, cudaStream_t st,
                                                 MarchLaunchInfo* info)
{
    return launch_n<PCC_MARCH_N>(stages, P, max_ctas, st, info);
}
#endif

#ifdef PCC_MARCH_BATCH
bool march_batch_supported(int ntau, int stages)
{
    return stages == 2 && (ntau == 128 || ntau == 256 || ntau == 512 || ntau == 1024);
}

cudaError_t launch_march_batch(const BatchParams& B, int max_ctas, cudaStream_t st, MarchLaunchInfo* info)
{
    using K = BatchShape<2>;
    auto kern = march_batch_kernel<2>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)K::SMEM);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0, per_sm = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, K::NT, K::SMEM)) != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    int ctas = sms * per_sm;
    if (max_ctas > 0 && ctas > max_ctas) ctas = max_ctas;
    if (info) {
        info->ctas = ctas;
        info->sweeps_per_cta = 0;  // depends on the class
        info->threads = K::NT;
        info->smem = K::SMEM;
        info->ctas_per_sm = per_sm;
    }
    kern<<<ctas, K::NT, K::SMEM, st>>>(B);
    return cudaGetLastError();
}
#endif

#ifdef PCC_MARCH_DISPATCH
cudaError_t launch_march_n128(int, const MarchParams&, int, cudaStream_t, MarchLaunchInfo*);
cudaError_t launch_march_n256(int, const MarchParams&, int, cudaStream_t, MarchLaunchInfo*);
cudaError_t launch_march_n512(int, const MarchParams&, int, cudaStream_t, MarchLaunchInfo*);
cudaError_t launch_march_n1024(int, const MarchParams&, int, cudaStream_t, MarchLaunchInfo*);
cudaError_t launch_march_n2048(int, const MarchParams&, int, cudaStream_t, MarchLaunchInfo*);

bool march_supported(int ntau, int stages)
{
    const bool n_ok = ntau == 128 || ntau == 256 || ntau == 512 || ntau == 1024 || ntau == 2048;
    return n_ok && stages >= 1 && stages <= 3;
}

cudaError_t launch_march(int ntau, int stages, const MarchParams& P, int max_ctas, cudaStream_t st,
                         MarchLaunchInfo* info)
{
    switch (ntau) {
        case 128: return launch_march_n128(stages, P, max_ctas, st, info);
        case 256: return launch_march_n256(stages, P, max_ctas, st, info);
        case 512: return launch_march_n512(stages, P, max_ctas, st, info);
        case 1024: return launch_march_n1024(stages, P, max_ctas, st, info);
        case 2048: return launch_march_n2048(stages, P, max_ctas, st, info);
        default: return cudaErrorInvalidValue;
    }
}
#endif

}  // namespace pcc
