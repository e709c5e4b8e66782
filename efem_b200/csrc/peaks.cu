// CUDA-core FMA throughput of the current device, the compute roof of the
// element residual kernels (FP64, or FP32 in mixed precision), which run on
// the FMA pipes and not on the tensor cores.  The reference has no
// counterpart: this is a measurement helper for the roofline figures.
//
// Every thread runs kChains independent FMA chains x <- x * a + b (a just
// below 1, so the values stay bounded), enough independent work per warp to
// keep the pipe issuing every cycle; the grid fills every SM with 2048
// resident threads.  The result is stored only when it equals a value it
// cannot take, so the compiler keeps the work.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "efem_internal.h"

namespace efem {
namespace {

constexpr int kChains = 8;
constexpr int kPeakThreads = 256;

__device__ __forceinline__ double fma_rn(double x, double a, double b) { return __fma_rn(x, a, b); }
__device__ __forceinline__ float fma_rn(float x, float a, float b) { return __fmaf_rn(x, a, b); }

template <typename T>
__global__ void __launch_bounds__(kPeakThreads) k_fma_peak(T* out, int iters, T a, T b)
{
    T x[kChains];
#pragma unroll
    for (int k = 0; k < kChains; k++) x[k] = static_cast<T>(threadIdx.x) * static_cast<T>(1e-3) + static_cast<T>(k);
    for (int i = 0; i < iters; i++)
#pragma unroll
        for (int k = 0; k < kChains; k++) x[k] = fma_rn(x[k], a, b);
    T s = 0;
#pragma unroll
    for (int k = 0; k < kChains; k++) s += x[k];
    if (s == static_cast<T>(-1)) out[0] = s;  // never true: x stays positive
}

template <typename T>
efem_status fma_peak(double* gflops)
{
    int dev = 0, sms = 0;
    EFEM_CUDA(cudaGetDevice(&dev));
    EFEM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int grid = sms * (2048 / kPeakThreads);
    const int iters = 4096;
    T* out = nullptr;
    EFEM_CUDA(cudaMalloc(&out, sizeof(T)));
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    efem_status s = EFEM_OK;
    std::vector<float> ms;
    auto fail = [&](cudaError_t e, const char* what) {
        set_error(std::string(what) + ": " + cudaGetErrorString(e));
        s = EFEM_ERR_CUDA;
    };
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) != cudaSuccess) fail(e, "cudaStreamCreate");
    if (s == EFEM_OK && (e = cudaEventCreate(&e0)) != cudaSuccess) fail(e, "cudaEventCreate");
    if (s == EFEM_OK && (e = cudaEventCreate(&e1)) != cudaSuccess) fail(e, "cudaEventCreate");
    for (int rep = 0; rep < 8 && s == EFEM_OK; rep++) {
        cudaEventRecord(e0, st);
        k_fma_peak<T><<<grid, kPeakThreads, 0, st>>>(out, iters, static_cast<T>(0.999999), static_cast<T>(1e-6));
        cudaEventRecord(e1, st);
        if ((e = cudaEventSynchronize(e1)) != cudaSuccess) {
            fail(e, "k_fma_peak");
            break;
        }
        float t = 0.0f;
        cudaEventElapsedTime(&t, e0, e1);
        if (rep >= 3) ms.push_back(t);  // three warm-up launches
    }
    if (e1) cudaEventDestroy(e1);
    if (e0) cudaEventDestroy(e0);
    if (st) cudaStreamDestroy(st);
    cudaFree(out);
    if (s != EFEM_OK) return s;
    std::sort(ms.begin(), ms.end());
    const double med = ms[ms.size() / 2];
    const double flops = 2.0 * kChains * static_cast<double>(iters) * grid * kPeakThreads;
    *gflops = flops / (med * 1e-3) / 1e9;
    return EFEM_OK;
}

}  // namespace
}  // namespace efem

extern "C" efem_status efem_fma_peak(int fp32, double* gflops)
{
    if (!gflops) {
        efem::set_error("efem_fma_peak: gflops is NULL");
        return EFEM_ERR_ARG;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        efem::set_error("no CUDA device is visible; this library has no CPU path");
        return EFEM_ERR_NO_DEVICE;
    }
    return fp32 ? efem::fma_peak<float>(gflops) : efem::fma_peak<double>(gflops);
}
