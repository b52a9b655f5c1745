// int_peak.cu -- measured integer-ALU peaks, the roofline denominators of the banded DP.
//
// The DP cell update is a chain of 32-bit adds and maxes, which the kernel
// issues as DPX instructions (__viaddmax_s32: max(a + b, c); __vimax3_s32:
// max(a, b, c)) plus plain adds and compares.  Each microbenchmark below runs
// eight independent chains of one instruction form per thread over a full grid
// and reports the achieved rate in tera-ops/s, counting every lane's
// arithmetic: an add or a max is one op, so __viaddmax_s32 and __vimax3_s32
// are two ops per lane and the packed s16x2 forms four.  Built as its own small
// library (libhero_peak.so); it is not part of the correction path.
#include <cuda_runtime.h>
#include <stdint.h>

namespace {

enum Form : int {
    F_ADD_MAX = 0,   // max(a + b, c) written as plain C (the compiler picks the instructions)
    F_VIADDMAX = 1,  // __viaddmax_s32
    F_VIMAX3 = 2,    // __vimax3_s32
    F_VIADDMAX2 = 3, // __viaddmax_s16x2
    F_VIMAX3_2 = 4,  // __vimax3_s16x2
};

constexpr double kOpsPerLane[] = {2.0, 2.0, 2.0, 4.0, 4.0};

template <int FORM>
__global__ void __launch_bounds__(256) k_peak(int iters, int seed, int *sink) {
    int a[8];
    const int b = (seed & 7) ^ int(threadIdx.x & 1u);
#pragma unroll
    for (int j = 0; j < 8; j++) a[j] = (int(threadIdx.x) * (j + 1) + seed) & 0x0fff0fff;
    for (int i = 0; i < iters; i++) {
        const int c = (i - 16) & 0x00ff00ff;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            if (FORM == F_ADD_MAX) a[j] = max(a[j] + b, i - j);
            if (FORM == F_VIADDMAX) a[j] = __viaddmax_s32(a[j], b, c);
            if (FORM == F_VIMAX3) a[j] = __vimax3_s32(a[j], b + j, c);
            if (FORM == F_VIADDMAX2)
                a[j] = int(__viaddmax_s16x2(unsigned(a[j]), 0x00010001u * unsigned(b), unsigned(c)));
            if (FORM == F_VIMAX3_2)
                a[j] = int(__vimax3_s16x2(unsigned(a[j]), unsigned(b + j), unsigned(c)));
        }
    }
    int s = 0;
#pragma unroll
    for (int j = 0; j < 8; j++) s ^= a[j];
    if (s == 0x7f3a91c5) sink[0] = s;
}

template <int FORM>
double run_peak(int device, int reps) {
    if (cudaSetDevice(device) != cudaSuccess) return -1;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    int *sink = nullptr;
    if (cudaMalloc(&sink, sizeof(int)) != cudaSuccess) return -1;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = sms * 8, threads = 256, iters = 16384;
    k_peak<FORM><<<blocks, threads>>>(64, 1, sink);  // warm-up
    double best = 0;
    for (int r = 0; r < reps; r++) {
        cudaEventRecord(e0);
        k_peak<FORM><<<blocks, threads>>>(iters, r + 2, sink);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        const double ops = double(blocks) * threads * double(iters) * 8.0 * kOpsPerLane[FORM];
        const double tops = ops / (double(ms) * 1e-3) / 1e12;
        if (tops > best) best = tops;
    }
    cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    return err == cudaSuccess ? best : -2;
}

}  // namespace

// max(a + b, c) in plain C, add and max one op each: the best of `reps` runs in
// tera-ops/s, or a negative value on a CUDA error.
extern "C" double hero_int_peak_tops(int device, int reps) { return run_peak<F_ADD_MAX>(device, reps); }

// One instruction form by number: 0 max(a + b, c) in plain C, 1 __viaddmax_s32,
// 2 __vimax3_s32, 3 __viaddmax_s16x2, 4 __vimax3_s16x2.  Tera-ops/s counting
// every lane's adds and maxes (2 per lane for forms 0-2, 4 for the packed ones).
extern "C" double hero_form_peak_tops(int device, int form, int reps) {
    switch (form) {
        case F_ADD_MAX: return run_peak<F_ADD_MAX>(device, reps);
        case F_VIADDMAX: return run_peak<F_VIADDMAX>(device, reps);
        case F_VIMAX3: return run_peak<F_VIMAX3>(device, reps);
        case F_VIADDMAX2: return run_peak<F_VIADDMAX2>(device, reps);
        case F_VIMAX3_2: return run_peak<F_VIMAX3_2>(device, reps);
        default: return -3;
    }
}

// Packed 16-bit DPX (__viaddmax_s16x2), kept for callers of the earlier name.
extern "C" double hero_dpx_peak_tops(int device, int reps) { return run_peak<F_VIADDMAX2>(device, reps); }
