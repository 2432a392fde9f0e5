// FP32 and FP64 FMA-chain throughput of this GPU: the pipe ceilings the
// radiation kernels are compared against (the driver's peak file carries HBM
// bandwidth and bf16 tensor throughput only).
//
// Each thread runs CHAINS independent multiply-add chains of ITERS steps
// (enough independent work to keep the pipe busy), on a grid of
// 8 CTAs x 256 threads per SM.  FLOPs = 2 x threads x CHAINS x ITERS; time
// from CUDA events around REPS launches after one warm-up launch.  The
// result is written to stdout as one JSON line.
#include <cuda_runtime.h>

#include <cstdio>

namespace {

constexpr int CHAINS = 8;
constexpr int ITERS = 4096;
constexpr int REPS = 20;

template <class T>
__global__ void __launch_bounds__(256) fma_chains(T *out, T a, T b) {
    T x[CHAINS];
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) x[c] = (T)(threadIdx.x + c);
    for (int i = 0; i < ITERS; ++i) {
#pragma unroll
        for (int c = 0; c < CHAINS; ++c) x[c] = fma(x[c], a, b);
    }
    T s = 0;
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) s += x[c];
    if (s == (T)-1.2345) out[blockIdx.x * blockDim.x + threadIdx.x] = s;   // keeps the chains live
}

template <class T>
double measure(int sms, double *ms_out) {
    const int blocks = sms * 8, threads = 256;
    T *out = nullptr;
    if (cudaMalloc(&out, sizeof(T) * blocks * threads) != cudaSuccess) return -1.0;
    const T a = (T)0.999999, b = (T)1e-7;
    fma_chains<T><<<blocks, threads>>>(out, a, b);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    for (int r = 0; r < REPS; ++r) fma_chains<T><<<blocks, threads>>>(out, a, b);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (cudaGetLastError() != cudaSuccess) return -1.0;
    const double flops = 2.0 * blocks * threads * (double)CHAINS * ITERS * REPS;
    *ms_out = ms;
    return flops / (ms * 1e-3) / 1e12;
}

}  // namespace

int main() {
    cudaDeviceProp p{};
    if (cudaGetDeviceProperties(&p, 0) != cudaSuccess) {
        std::printf("{\"error\": \"no CUDA device\"}\n");
        return 1;
    }
    double ms32 = 0, ms64 = 0;
    const double f32 = measure<float>(p.multiProcessorCount, &ms32);
    const double f64 = measure<double>(p.multiProcessorCount, &ms64);
    int clk = 0;
    cudaDeviceGetAttribute(&clk, cudaDevAttrClockRate, 0);
    std::printf(
        "{\"device\": \"%s\", \"sms\": %d, \"fp32_fma_tflops\": %.2f, \"fp64_fma_tflops\": %.2f, "
        "\"fp32_ms\": %.3f, \"fp64_ms\": %.3f, \"max_sm_clock_mhz\": %d, "
        "\"method\": \"%d independent FMA chains x %d steps per thread, %d CTAs x 256 threads per SM, "
        "%d launches timed with CUDA events\"}\n",
        p.name, p.multiProcessorCount, f32, f64, ms32, ms64, clk / 1000, CHAINS, ITERS, 8, REPS);
    return (f32 > 0 && f64 > 0) ? 0 : 1;
}
