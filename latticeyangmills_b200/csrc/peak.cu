// Measured CUDA-core FMA throughput: the denominator of the flow kernels'
// arithmetic roofline (the stage kernels are 3x3 complex products with no
// tensor-core shape, so their ceiling is the FP32 or FP64 FMA pipe).
//
// Each thread runs 8 independent FMA chains (enough instruction-level
// parallelism to cover the pipe latency at full occupancy) for `iters` x 16
// rounds; the grid fills every SM several times over.  A result that is never
// true keeps the compiler from dropping the chains.
#include <cuda_runtime.h>

#include <string>

#include "api_util.h"
#include "ymflow.h"

namespace ym {
namespace {

constexpr int kChains = 8;
constexpr int kUnroll = 16;

template <class T>
__global__ void __launch_bounds__(256) fma_peak_kernel(T* out, T a, T b, int iters) {
    T x[kChains];
#pragma unroll
    for (int i = 0; i < kChains; i++) x[i] = T(threadIdx.x) * T(1e-3) + T(i);
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int k = 0; k < kUnroll; k++)
#pragma unroll
            for (int i = 0; i < kChains; i++) x[i] = fma(x[i], a, b);
    }
    T s = T(0);
#pragma unroll
    for (int i = 0; i < kChains; i++) s += x[i];
    if (s == T(-1.25)) out[blockIdx.x] = s;
}

template <class T>
cudaError_t time_peak(int sms, double* tflops) {
    T* out = nullptr;
    cudaError_t e = cudaMalloc(&out, sizeof(T) * 4096);
    if (e != cudaSuccess) return e;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int block = 256, grid = sms * 8, iters = 4096;
    float best = 1e30f;
    for (int rep = 0; rep < 12 && e == cudaSuccess; rep++) {  // first launch is a warm-up; best of the rest
        cudaEventRecord(e0);
        fma_peak_kernel<T><<<grid, block>>>(out, T(0.999999), T(1e-7), iters);
        cudaEventRecord(e1);
        e = cudaEventSynchronize(e1);
        if (e == cudaSuccess) e = cudaGetLastError();
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (e == cudaSuccess) {
        const double fmas = double(grid) * block * double(iters) * kUnroll * kChains;
        *tflops = 2.0 * fmas / (double(best) * 1e-3) / 1e12;
    }
    return e;
}

}  // namespace
}  // namespace ym

using namespace ym;

extern "C" int ymflow_fma_peak(int device, int precision, double* tflops) {
    if (!tflops || (precision != YMFLOW_FP64 && precision != YMFLOW_FP32_18 && precision != YMFLOW_FP32_12))
        return YMFLOW_ERR_ARG;
    std::string why;
    if (!device_usable(device, &why)) return YMFLOW_ERR_NODEVICE;
    DeviceGuard guard(device);
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
        cudaGetLastError();
        return YMFLOW_ERR_CUDA;
    }
    const cudaError_t e = precision == YMFLOW_FP64 ? time_peak<double>(sms, tflops) : time_peak<float>(sms, tflops);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return status_of(e);
    }
    return YMFLOW_OK;
}
