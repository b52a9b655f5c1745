// int_peak.cu -- measured integer-ALU peak, the roofline denominator of the banded DP.
//
// The DP cell update is a chain of 32-bit adds and maxes.  This kernel runs
// eight independent add+max chains per thread over a full grid and reports the
// achieved rate, counting the add and the max as one op each.  Built as its own
// small library (libhero_peak.so); it is not part of the correction path.
#include <cuda_runtime.h>
#include <stdint.h>

__global__ void __launch_bounds__(256) k_int_peak(int iters, int seed, int *sink) {
    int a[8];
    const int b = seed ^ int(threadIdx.x);
#pragma unroll
    for (int j = 0; j < 8; j++) a[j] = int(threadIdx.x) * (j + 1) + seed;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int j = 0; j < 8; j++) a[j] = max(a[j] + b, i - j);
    }
    int s = 0;
#pragma unroll
    for (int j = 0; j < 8; j++) s ^= a[j];
    if (s == 0x7f3a91c5) sink[0] = s;
}

// Returns the best of `reps` runs in tera-ops/s (add and max each count 1), or
// a negative value on a CUDA error.
extern "C" double hero_int_peak_tops(int device, int reps) {
    if (cudaSetDevice(device) != cudaSuccess) return -1;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    int *sink = nullptr;
    if (cudaMalloc(&sink, sizeof(int)) != cudaSuccess) return -1;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = sms * 8, threads = 256, iters = 16384;
    k_int_peak<<<blocks, threads>>>(64, 1, sink);  // warm-up
    double best = 0;
    for (int r = 0; r < reps; r++) {
        cudaEventRecord(e0);
        k_int_peak<<<blocks, threads>>>(iters, r + 2, sink);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        const double ops = double(blocks) * threads * double(iters) * 8.0 * 2.0;
        const double tops = ops / (double(ms) * 1e-3) / 1e12;
        if (tops > best) best = tops;
    }
    cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    return err == cudaSuccess ? best : -2;
}

// Packed 16-bit DPX throughput: eight independent chains of
// max(a + b, c) on s16x2 (2 lanes x 2 ops per instruction) and of the 3-input
// max.  Reported in tera-ops/s counting every lane's add and max.
__global__ void __launch_bounds__(256) k_dpx_peak(int iters, int seed, int *sink) {
    unsigned a[8];
    const unsigned b = 0x00010001u * unsigned(seed & 7);
#pragma unroll
    for (int j = 0; j < 8; j++) a[j] = (threadIdx.x * (j + 1)) & 0x0fff0fffu;
    for (int i = 0; i < iters; i++) {
        const unsigned c = 0x00010001u * unsigned(i & 0xff);
#pragma unroll
        for (int j = 0; j < 8; j++) a[j] = __viaddmax_s16x2(a[j], b, c);
    }
    unsigned s = 0;
#pragma unroll
    for (int j = 0; j < 8; j++) s ^= a[j];
    if (s == 0x7f3a91c5u) sink[0] = int(s);
}

extern "C" double hero_dpx_peak_tops(int device, int reps) {
    if (cudaSetDevice(device) != cudaSuccess) return -1;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    int *sink = nullptr;
    if (cudaMalloc(&sink, sizeof(int)) != cudaSuccess) return -1;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = sms * 8, threads = 256, iters = 16384;
    k_dpx_peak<<<blocks, threads>>>(64, 1, sink);
    double best = 0;
    for (int r = 0; r < reps; r++) {
        cudaEventRecord(e0);
        k_dpx_peak<<<blocks, threads>>>(iters, r + 2, sink);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        const double ops = double(blocks) * threads * double(iters) * 8.0 * 4.0;
        const double tops = ops / (double(ms) * 1e-3) / 1e12;
        if (tops > best) best = tops;
    }
    cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    return err == cudaSuccess ? best : -2;
}
