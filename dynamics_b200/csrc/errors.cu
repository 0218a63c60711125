// Error reporting and small library-wide entry points.
#include <cstdio>
#include <string>

#include "common.cuh"

namespace dyn {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char* what) {
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    if (e == cudaErrorMemoryAllocation) return DYN_ERR_OOM;
    return DYN_ERR_CUDA;
}

}  // namespace dyn

extern "C" const char* dyn_last_error(void) { return dyn::g_last_error.c_str(); }

extern "C" int dyn_version(void) { return 1; }

extern "C" int dyn_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

// ---------------------------------------------------------------------------
// FP32 FMA throughput probe: the denominator of the pair kernel's roofline
// (the measured-peaks file holds HBM and tensor-core figures only).  Every
// thread runs 8 independent FMA chains; the result is stored so the work is
// not eliminated.
// ---------------------------------------------------------------------------
__global__ void k_fma_probe(float* out, int iters, float a, float b) {
    float x0 = threadIdx.x * 1e-3f, x1 = x0 + 1.f, x2 = x0 + 2.f, x3 = x0 + 3.f;
    float x4 = x0 + 4.f, x5 = x0 + 5.f, x6 = x0 + 6.f, x7 = x0 + 7.f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            x0 = fmaf(x0, a, b); x1 = fmaf(x1, a, b); x2 = fmaf(x2, a, b); x3 = fmaf(x3, a, b);
            x4 = fmaf(x4, a, b); x5 = fmaf(x5, a, b); x6 = fmaf(x6, a, b); x7 = fmaf(x7, a, b);
        }
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
}

extern "C" int dyn_probe_fp32_peak(void* stream, double* tflops) {
    DYN_CHECK(tflops, DYN_ERR_INVALID, "dyn_probe_fp32_peak: NULL argument");
    int dev = 0, sms = 0;
    DYN_CUDA(cudaGetDevice(&dev));
    DYN_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    cudaStream_t st = (cudaStream_t)stream;
    const int threads = 512, blocks = sms * 4, iters = 4096;
    float* out = nullptr;
    DYN_CUDA(cudaMalloc(&out, (size_t)threads * blocks * sizeof(float)));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    k_fma_probe<<<blocks, threads, 0, st>>>(out, 64, 0.999f, 1e-4f);  // warm-up
    float best = 1e30f;
    for (int r = 0; r < 5; ++r) {
        cudaEventRecord(e0, st);
        k_fma_probe<<<blocks, threads, 0, st>>>(out, iters, 0.999f, 1e-4f);
        cudaEventRecord(e1, st);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        best = ms < best ? ms : best;
    }
    cudaError_t e = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (e != cudaSuccess) return dyn::cuda_fail(e, "k_fma_probe");
    const double flops = 2.0 * 8.0 * 16.0 * iters * (double)threads * blocks;
    *tflops = flops / (best * 1e-3) / 1e12;
    return DYN_OK;
}
