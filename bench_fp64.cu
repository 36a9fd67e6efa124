// bench_fp64.cu -- FP64 FMA throughput probe, bench support.  The roofline
// of the solver's arithmetic kernels is the GPU's non-tensor FP64 rate,
// which the measured-peaks file (HBM and bf16 figures) does not carry, so
// bench.py measures it with this kernel: every thread runs 8 independent
// DFMA chains.  Built into libbench_fp64.so beside bench.py; the solver
// does not link it.
#include <cuda_runtime.h>

__global__ void k_dfma(int iters, double *out) {
    double a[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        a[q] = 1.0 + 1e-9 * (threadIdx.x + q);
    }
    const double m = 0.999999999, c = 1e-12;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            a[q] = fma(a[q], m, c);
        }
    }
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        s += a[q];
    }
    if (s == 12345.0) {
        out[0] = s; // keeps the chains alive
    }
}

// Returns the achieved FP64 rate in GFLOP/s (2 flops per FMA), or a
// negative CUDA error code.
extern "C" double brdc_probe_dfma_gflops(int blocks, int threads, int iters) {
    double *out = nullptr;
    if (cudaMalloc(&out, sizeof(double)) != cudaSuccess) {
        return -1.0;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    k_dfma<<<blocks, threads>>>(iters / 10, out); // warm-up
    cudaEventRecord(e0);
    k_dfma<<<blocks, threads>>>(iters, out);
    cudaEventRecord(e1);
    const cudaError_t st = cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (st != cudaSuccess || ms <= 0.0f) {
        return -(double)st;
    }
    const double flops = 2.0 * 8.0 * (double)blocks * threads * (double)iters;
    return flops / (ms * 1e-3) / 1e9;
}
