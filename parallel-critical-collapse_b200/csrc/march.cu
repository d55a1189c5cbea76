// march.cu -- instantiations of the persistent IRK march kernel for one Ntau
// and one transform schedule (PCC_MARCH_N, PCC_MARCH_PAIR, set by the build:
// one translation unit each so that the shapes compile in parallel) and, with
// PCC_MARCH_DISPATCH, the launcher that selects among them and the autotuner
// that picks the schedule per (device, Ntau, stages).
#include <cmath>
#include <cstdlib>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "pcc_internal.h"

namespace pcc {

namespace {

template <int N, int S, int PAIR>
constexpr int min_blocks()
{
    // The radix-8 RHS needs ~230 registers per thread without spilling, so a
    // 128-thread CTA reaches two resident CTAs per SM and wider CTAs one.
    constexpr int nt = MarchShape<N, S, PAIR>::NT;
    return nt <= 128 ? 2 : 1;
}

template <int N, int S, int PAIR>
cudaError_t launch_shape(const MarchParams& P, int max_ctas, cudaStream_t st, MarchLaunchInfo* info)
{
    using K = MarchShape<N, S, PAIR>;
    auto kern = march_kernel<N, S, min_blocks<N, S, PAIR>(), PAIR>;
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

template <int N, int PAIR>
cudaError_t launch_n(int stages, const MarchParams& P, int max_ctas, cudaStream_t st, MarchLaunchInfo* info)
{
    switch (stages) {
        case 1: return launch_shape<N, 1, PAIR>(P, max_ctas, st, info);
        case 2: return launch_shape<N, 2, PAIR>(P, max_ctas, st, info);
        case 3: return launch_shape<N, 3, PAIR>(P, max_ctas, st, info);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace

#ifdef PCC_MARCH_N
#define PCC_CAT2(a, b) a##b
#define PCC_CAT(a, b) PCC_CAT2(a, b)
#define PCC_CAT4(a, b, c, d) PCC_CAT(PCC_CAT(a, b), PCC_CAT(c, d))
cudaError_t PCC_CAT4(launch_march_n, PCC_MARCH_N, _p, PCC_MARCH_PAIR)(int stages, const MarchParams& P,
                                                                     int max_ctas, cudaStream_t st,
                                                                     MarchLaunchInfo* info)
{
    return launch_n<PCC_MARCH_N, PCC_MARCH_PAIR>(stages, P, max_ctas, st, info);
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
#define PCC_DECL(n)                                                                                      \
    cudaError_t launch_march_n##n##_p0(int, const MarchParams&, int, cudaStream_t, MarchLaunchInfo*);    \
    cudaError_t launch_march_n##n##_p1(int, const MarchParams&, int, cudaStream_t, MarchLaunchInfo*);
PCC_DECL(128)
PCC_DECL(256)
PCC_DECL(512)
PCC_DECL(1024)
PCC_DECL(2048)
#undef PCC_DECL
cudaError_t launch_march_n1024_p2(int, const MarchParams&, int, cudaStream_t, MarchLaunchInfo*);

bool march_supported(int ntau, int stages)
{
    const bool n_ok = ntau == 128 || ntau == 256 || ntau == 512 || ntau == 1024 || ntau == 2048;
    return n_ok && stages >= 1 && stages <= 3;
}

namespace {

// Autotuned transform schedule per (device, Ntau, stages): 0 single, 1
// paired, 2 paired with the warp-exchange transforms (Ntau 1024, 2 stages).
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int>, MarchTuning> g_tuned;

bool schedule_available(int ntau, int stages, int sched)
{
    return sched == 0 || sched == 1 || (sched == 2 && ntau == 1024 && stages == 2);
}

cudaError_t launch_variant(int ntau, int stages, const MarchParams& P, int max_ctas, cudaStream_t st,
                           MarchLaunchInfo* info, int sched)
{
    if (sched == 2 && schedule_available(ntau, stages, 2)) return launch_march_n1024_p2(stages, P, max_ctas, st, info);
    const bool pair = sched != 0;
#define PCC_CASE(n)                                                                                           \
    case n:                                                                                                   \
        return pair ? launch_march_n##n##_p1(stages, P, max_ctas, st, info)                                   \
                    : launch_march_n##n##_p0(stages, P, max_ctas, st, info);
    switch (ntau) {
        PCC_CASE(128)
        PCC_CASE(256)
        PCC_CASE(512)
        PCC_CASE(1024)
        PCC_CASE(2048)
        default: return cudaErrorInvalidValue;
    }
#undef PCC_CASE
}

}  // namespace

bool march_tuning(int device, int ntau, int stages, MarchTuning* out)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tuned.find(std::make_tuple(device, ntau, stages));
    if (it == g_tuned.end()) return false;
    if (out) *out = it->second;
    return true;
}

void march_set_tuning(int device, int ntau, int stages, const MarchTuning& t)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tuned[std::make_tuple(device, ntau, stages)] = t;
}

cudaError_t launch_march(int ntau, int stages, const MarchParams& P, int max_ctas, cudaStream_t st,
                         MarchLaunchInfo* info)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    MarchTuning t{};
    int sched = march_tuning(dev, ntau, stages, &t) ? t.pair : 1;  // untuned: paired
    if (const char* f = std::getenv("PCC_MARCH_SCHEDULE")) {
        // a fixed schedule for every shape that has it (0, 1 or 2)
        const int v = std::atoi(f);
        if (schedule_available(ntau, stages, v)) sched = v;
    }
    return launch_variant(ntau, stages, P, max_ctas, st, info, sched);
}

// Times the transform schedules of the shape on the kernel's single-RHS mode:
// items marching no step, one RHS evaluation each, over sixteen waves of
// sweep slots (about half a millisecond at Ntau = 1024), from a smooth
// synthetic state (Delta = 3.4 in its slot), best of five.  The paired
// schedule is kept unless another one is more than 3 % faster: on a full
// march the schedules differ by a few per cent, less than a short probe's
// noise.  The choice is recorded for (device, Ntau, stages).  Allocates and
// frees its own buffers.
cudaError_t march_autotune(int ntau, int stages, const double2* tw, cudaStream_t st, MarchTuning* out)
{
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    const int items = 16 * 2 * sms * (ntau >= 1024 ? 1 : 1024 / ntau);
    std::vector<double> y((size_t)items * ntau, 0.0), xs(items, 0.5);
    for (int i = 0; i < items; ++i) {
        double* s = &y[(size_t)i * ntau];
        for (int m = 0; m < ntau / 2; ++m) s[2 * m] = 1e-2 * std::exp(-0.5 * m) * (1.0 + 0.01 * (i % 7));
        s[4] = 3.4;  // Re Y[2]: the echoing period
    }
    double *d_y = nullptr, *d_out = nullptr, *d_x = nullptr;
    int* d_cnt = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    const size_t by = y.size() * sizeof(double);
    e = cudaMalloc(&d_y, by);
    if (e == cudaSuccess) e = cudaMalloc(&d_out, by);
    if (e == cudaSuccess) e = cudaMalloc(&d_x, items * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&d_cnt, sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_y, y.data(), by, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_x, xs.data(), items * sizeof(double), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaEventCreate(&a);
    if (e == cudaSuccess) e = cudaEventCreate(&b);
    double ms[3] = {0.0, 0.0, 0.0};
    for (int v = 0; v < 3 && e == cudaSuccess; ++v) {
        if (!schedule_available(ntau, stages, v)) continue;
        MarchParams P{};
        P.n_items = items;
        P.mode = 1;
        P.yinit = d_y;
        P.yfinal = d_out;
        P.dim = 4.0;
        P.dim_m2_cubed = 8.0;
        P.prec = 1e-15;
        P.max_its = 100;
        P.stages = stages;
        P.twN = tw;
        P.x_in = d_x;
        P.work_counter = d_cnt;
        float best = 1e30f;
        for (int rep = 0; rep < 6 && e == cudaSuccess; ++rep) {  // one warm-up, best of five
            e = cudaMemsetAsync(d_cnt, 0, sizeof(int), st);
            if (e == cudaSuccess) e = cudaEventRecord(a, st);
            if (e == cudaSuccess) e = launch_variant(ntau, stages, P, 0, st, nullptr, v);
            if (e == cudaSuccess) e = cudaEventRecord(b, st);
            if (e == cudaSuccess) e = cudaEventSynchronize(b);
            float t = 0.0f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&t, a, b);
            if (rep > 0 && t < best) best = t;
        }
        ms[v] = best;
    }
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    cudaFree(d_y);
    cudaFree(d_out);
    cudaFree(d_x);
    cudaFree(d_cnt);
    if (e != cudaSuccess) return e;
    MarchTuning t{};
    t.pair = 1;
    double best = 0.97 * ms[1];
    for (int v : {0, 2})
        if (ms[v] > 0.0 && ms[v] < best) {
            best = ms[v];
            t.pair = v;
        }
    t.ms_single = ms[0];
    t.ms_pair = ms[1];
    t.ms_wx = ms[2];
    march_set_tuning(dev, ntau, stages, t);
    if (out) *out = t;
    return cudaSuccess;
}
#endif

}  // namespace pcc
