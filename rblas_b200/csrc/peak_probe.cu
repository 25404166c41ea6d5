// peak_probe.cu -- measures the FP32 and FP64 FMA throughput of the current
// GPU (the roofline denominators for the plain SIMT forms, which the
// tensor-core peak figures do not cover). Each thread runs 8 independent FMA
// chains; the grid is a multiple of the SM count; the result is written back
// so the compiler cannot drop the work.
#include <cuda_runtime.h>

#include "../../include/rblas_b200.h"
#include "rb_internal.h"

namespace rb {

template <typename T>
__global__ void __launch_bounds__(256) fma_peak_kernel(T* out, int iters, T x, T y) {
    T a0 = x + threadIdx.x, a1 = a0 + T(1), a2 = a0 + T(2), a3 = a0 + T(3);
    T a4 = a0 + T(4), a5 = a0 + T(5), a6 = a0 + T(6), a7 = a0 + T(7);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            a0 = fma(a0, y, x); a1 = fma(a1, y, x); a2 = fma(a2, y, x); a3 = fma(a3, y, x);
            a4 = fma(a4, y, x); a5 = fma(a5, y, x); a6 = fma(a6, y, x); a7 = fma(a7, y, x);
        }
    }
    const T s = ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + (a6 + a7));
    if (s == T(-12345.0)) out[blockIdx.x] = s;  // never true for these inputs
}

template <typename T>
static double probe(int iters) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int blocks = sms * 8;
    T* out = nullptr;
    if (dev_alloc(reinterpret_cast<void**>(&out), blocks * sizeof(T)) != cudaSuccess) return -1.0;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    fma_peak_kernel<T><<<blocks, 256>>>(out, 16, T(0.5), T(0.999));  // warm-up
    count_launch();
    cudaEventRecord(e0);
    fma_peak_kernel<T><<<blocks, 256>>>(out, iters, T(0.5), T(0.999));
    count_launch();
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (cudaGetLastError() != cudaSuccess || ms <= 0.f) return -1.0;
    const double flops = 2.0 * 8 * 16 * double(iters) * blocks * 256;
    return flops / (ms * 1e-3) / 1e12;
}

}  // namespace rb

extern "C" double rb_probe_tensor_peak_tflops(int is_i8, int iters) {
    if (iters <= 0) iters = 65536;
    return rb::probe_umma_peak(is_i8, iters);
}

extern "C" double rb_probe_fma_peak_tflops(int is_f64, int iters) {
    if (iters <= 0) iters = 4096;
    return is_f64 ? rb::probe<double>(iters) : rb::probe<float>(iters);
}
