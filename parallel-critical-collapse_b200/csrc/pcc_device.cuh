// pcc_device.cuh -- device helpers shared by the boundary kernels and the
// IRK march kernel: complex arithmetic on double2, the twiddle table layout,
// and sweep-local synchronisation.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pcc {

constexpr double kPi = 3.14159265358979323846;

__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
// a * (s i) for s = +1/-1 : (x + iy)(s i) = (-s y, s x)
template <int S>
__host__ __device__ __forceinline__ double2 cmul_si(double2 a)
{
    return S > 0 ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
}

// (a + ib) / (c + id) in the operation order of libgcc's __divdc3 (Smith's
// method with the subnormal-ratio variant), which is what std::complex<double>
// division compiles to in the reference (SpectralTransformer.cpp:173-186).
__host__ __device__ __forceinline__ double2 cdiv(double a, double b, double c, double d)
{
    double x, y;
    if (fabs(c) < fabs(d)) {
        const double ratio = c / d;
        const double denom = (c * ratio) + d;
        if (fabs(ratio) > 2.2250738585072014e-308) {
            x = ((a * ratio) + b) / denom;
            y = ((b * ratio) - a) / denom;
        } else {
            x = ((c * (a / d)) + b) / denom;
            y = ((c * (b / d)) - a) / denom;
        }
    } else {
        const double ratio = d / c;
        const double denom = (d * ratio) + c;
        if (fabs(ratio) > 2.2250738585072014e-308) {
            x = ((b * ratio) + a) / denom;
            y = (b - (a * ratio)) / denom;
        } else {
            x = (a + (d * (b / c))) / denom;
            y = (b - (d * (a / c))) / denom;
        }
    }
    return make_double2(x, y);
}

// Shared-memory index padding: one complex of padding per 8, which makes the
// 16-byte accesses of 8 consecutive lanes hit 8 distinct bank groups for
// every Stockham stride used here.
__host__ __device__ __forceinline__ int pad8(int i) { return i + (i >> 3); }

// The same property without padding: XOR the low three bits of a complex
// index with bits 3..5.  Every access pattern of the radix-8 Stockham passes
// (stride-8 writes, span-8/64/512 writes, unit-stride reads of 8 lanes)
// then maps 8 consecutive lanes to 8 distinct 16-byte bank groups.
__host__ __device__ __forceinline__ int swz8(int i) { return i ^ ((i >> 3) & 7); }

// Synchronisation of a group of threads (a sweep, or one stage group of it).
// Groups of at most 32 threads live inside one warp and use __syncwarp on
// their lane mask; wider groups (WIDE, fixed by the kernel's shape at compile
// time) use a named barrier (id >= 1) over their own warps.
template <bool WIDE>
struct SweepSync {
    unsigned mask;  // lane mask (all lanes for wide groups)
    int bar_id;     // named barrier id (wide groups)
    int nthreads;   // threads taking part (multiple of 32 for wide groups)
    __device__ __forceinline__ void sync() const
    {
        if constexpr (WIDE) {
            asm volatile("bar.sync %0, %1;" ::"r"(bar_id), "r"(nthreads) : "memory");
        } else {
            __syncwarp(mask);
        }
    }
};

}  // namespace pcc
