// FP32 FMA throughput probe: the measured denominator of the FP32-pipe
// rooflines (dictionary, Gauss-Newton and FP32 matching kernels), as a copy
// kernel and a BF16 GEMM are for the memory and tensor-core rooflines.
// Built into its own library (libsnapmrf_probe.so), loaded only by the
// benchmark; the matching and dictionary library does not contain it.
//
// Each thread runs eight independent FMA chains; the only memory traffic is
// one store per thread.
#include <cuda_runtime.h>

namespace {

__global__ void fma_chains_kernel(float *out, int iters, float a, float b) {
    float x[8];
#pragma unroll
    for (int i = 0; i < 8; i++) x[i] = threadIdx.x * 1e-3f + i;
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int r = 0; r < 16; r++)
#pragma unroll
            for (int i = 0; i < 8; i++) x[i] = fmaf(x[i], a, b);
    }
    float s = 0.f;
#pragma unroll
    for (int i = 0; i < 8; i++) s += x[i];
    out[blockIdx.x * (long long)blockDim.x + threadIdx.x] = s;
}

}  // namespace

// Best of `reps` timed launches (after one warm-up) of FMA chains on the
// current device, 8 CTAs of 256 threads per SM; *tflops = 2 flop per FMA.
// Returns 0, or the CUDA error code.
extern "C" int snapmrf_probe_fp32_fma(int reps, double *tflops) {
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return (int)e;
    const int block = 256, grid = sms * 8, iters = 2048;
    float *out = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    double best = 0.0;
    if ((e = cudaMalloc(&out, sizeof(float) * (size_t)grid * block)) != cudaSuccess) return (int)e;
    if ((e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) == cudaSuccess &&
        (e = cudaEventCreate(&e0)) == cudaSuccess && (e = cudaEventCreate(&e1)) == cudaSuccess) {
        for (int r = 0; r <= reps && e == cudaSuccess; r++) {
            cudaEventRecord(e0, st);
            fma_chains_kernel<<<grid, block, 0, st>>>(out, iters, 0.999f, 1e-3f);
            cudaEventRecord(e1, st);
            if ((e = cudaEventSynchronize(e1)) != cudaSuccess) break;
            if ((e = cudaGetLastError()) != cudaSuccess) break;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            const double fmas = (double)grid * block * iters * 16 * 8;
            if (r > 0 && ms > 0.f) best = fmax(best, 2.0 * fmas / (ms * 1e-3) / 1e12);
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) cudaStreamDestroy(st);
    cudaFree(out);
    *tflops = best;
    return (int)e;
}
