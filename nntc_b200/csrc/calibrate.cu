// calibrate.cu: the measured issue peaks of the FP64 and FP32 vector pipes on this device, the denominators of the
// compute fractions bench.py reports beside the HBM fraction for the kernels those pipes bind (the objective, the
// gathers, the site terms): a grid of four resident blocks per SM, each thread running eight independent chains of
// fused multiply-adds (no loads, no dependences between chains), timed with CUDA events after one warm-up launch.

#include "device.cuh"

namespace nb
{

constexpr int CAL_CHAINS = 8;
constexpr int CAL_THREADS = 256;

// Where a chain's sum would go if it ever took the impossible value the kernel tests for: keeps the chains live.
static __device__ double g_cal_sink;

template <typename T>
__global__ void __launch_bounds__(CAL_THREADS) k_fma_peak(int iters, T a, T b)
{
    T x[CAL_CHAINS];
#pragma unroll
    for (int c = 0; c < CAL_CHAINS; c++)
        x[c] = (T)(threadIdx.x + c) * (T)1e-3;
    for (int i = 0; i < iters; i++)
#pragma unroll
        for (int c = 0; c < CAL_CHAINS; c++)
            x[c] = fma(x[c], a, b);
    T s = 0;
#pragma unroll
    for (int c = 0; c < CAL_CHAINS; c++)
        s += x[c];
    if (s == (T)-12345.0)   // never (the chains converge to b / (1 - a) > 0)
        g_cal_sink = (double)s;
}

template <typename T>
static int time_peak(double* tflops)
{
    int dev = 0, sms = 0;
    NB_CUDA(cudaGetDevice(&dev));
    NB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int blocks = sms * 4, iters = 1 << 14;
    cudaEvent_t a, b;
    NB_CUDA(cudaEventCreate(&a));
    NB_CUDA(cudaEventCreate(&b));
    k_fma_peak<T><<<blocks, CAL_THREADS>>>(256, (T)0.999, (T)1e-4);
    NB_LAUNCHED();
    NB_CUDA(cudaEventRecord(a));
    k_fma_peak<T><<<blocks, CAL_THREADS>>>(iters, (T)0.999, (T)1e-4);
    NB_LAUNCHED();
    NB_CUDA(cudaEventRecord(b));
    NB_CUDA(cudaEventSynchronize(b));
    float ms = 0.0f;
    NB_CUDA(cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    const double flops = 2.0 * CAL_CHAINS * (double)iters * (double)blocks * CAL_THREADS;
    *tflops = flops / (ms * 1e-3) / 1e12;
    return NNTC_B200_OK;
}

}   // namespace nb

extern "C" int nntc_b200_measure_fma_peaks(double* fp64_tflops, double* fp32_tflops)
{
    NB_TRY(nb::time_peak<double>(fp64_tflops));
    return nb::time_peak<float>(fp32_tflops);
}
