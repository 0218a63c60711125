// Shared device/host helpers for the dynb200 engine (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>

#include "../../include/dynb200.h"

// ---------------------------------------------------------------------------
// error plumbing (host)
// ---------------------------------------------------------------------------
namespace dyn {

void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

}  // namespace dyn

#define DYN_CUDA(call)                                              \
    do {                                                            \
        cudaError_t _e = (call);                                    \
        if (_e != cudaSuccess) return dyn::cuda_fail(_e, #call);    \
    } while (0)

#define DYN_CHECK(cond, code, msg)                                  \
    do {                                                            \
        if (!(cond)) return dyn::fail((code), (msg));               \
    } while (0)

// ---------------------------------------------------------------------------
// fixed point: forces are accumulated as int64 with 2^-32 kcal/mol/A
// resolution, so the sum is independent of accumulation order.
// ---------------------------------------------------------------------------
#define DYN_FIX_SCALE 4294967296.0
#define DYN_FIX_SCALE_F 4294967296.0f
#define DYN_FIX_INV (1.0 / 4294967296.0)

__device__ __forceinline__ long long fix_from_float(float f) {
    return __float2ll_rn(f * DYN_FIX_SCALE_F);
}
__device__ __forceinline__ long long fix_from_double(double f) {
    return __double2ll_rn(f * DYN_FIX_SCALE);
}
__device__ __forceinline__ void fix_atomic_add(long long* p, long long v) {
    atomicAdd(reinterpret_cast<unsigned long long*>(p), static_cast<unsigned long long>(v));
}
__device__ __forceinline__ float fix_to_float(long long v) {
    return (float)((double)v * DYN_FIX_INV);
}

// ---------------------------------------------------------------------------
// small vector helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
// The library is compiled without automatic multiply-add contraction
// (-fmad=false), so that a kernel body rounds identically in its
// single-system and batched instantiations; fused multiply-adds are written
// out where they are wanted.
__device__ __forceinline__ float dot3(float3 a, float3 b) { return fmaf(a.z, b.z, fmaf(a.y, b.y, a.x * b.x)); }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
    return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float3 xyz(float4 a) { return f3(a.x, a.y, a.z); }

// Device copy of the periodic box; kernels read it from memory so that a
// captured CUDA graph stays valid when the barostat rescales the box.
struct BoxDev {
    float lo[3];
    float ext[3];
    float inv_ext[3];
    float pad;
};

__device__ __forceinline__ float3 min_image_rint(float3 d, const BoxDev& b) {
    d.x -= rintf(d.x * b.inv_ext[0]) * b.ext[0];
    d.y -= rintf(d.y * b.inv_ext[1]) * b.ext[1];
    d.z -= rintf(d.z * b.inv_ext[2]) * b.ext[2];
    return d;
}

// ---------------------------------------------------------------------------
// warp / block reductions (deterministic: fixed shuffle tree)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum_d(double x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}
__device__ __forceinline__ float warp_sum_f(float x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}
__device__ __forceinline__ float warp_max_f(float x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = fmaxf(x, __shfl_xor_sync(0xffffffffu, x, o));
    return x;
}

// Block-wide sum of NV doubles; result valid in thread 0.  blockDim.x must be
// a multiple of 32 and at most 1024.
template <int NV>
__device__ __forceinline__ void block_sum_d(double (&v)[NV]) {
    __shared__ double sh[32][NV];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = warp_sum_d(v[k]);
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) sh[wid][k] = v[k];
    }
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x >> 5;
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double x = lane < nw ? sh[lane][k] : 0.0;
            v[k] = warp_sum_d(x);
        }
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon et al., SC'11); matches oracle/philox.py
// ---------------------------------------------------------------------------
struct Philox4 { uint32_t x[4]; };

__device__ __forceinline__ Philox4 philox4x32(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                               uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
        const uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
        const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    Philox4 r; r.x[0] = c0; r.x[1] = c1; r.x[2] = c2; r.x[3] = c3;
    return r;
}

#define DYN_STREAM_OU 1u
#define DYN_STREAM_CSVR 2u
#define DYN_STREAM_BARO 3u

__device__ __forceinline__ float uniform24f(uint32_t x) {
    return ((float)(x >> 8) + 0.5f) * 5.9604644775390625e-08f;  // 2^-24
}
__device__ __forceinline__ double uniform24d(uint32_t x) {
    return ((double)(x >> 8) + 0.5) * 5.9604644775390625e-08;
}

// Three standard normals (Box-Muller) for particle `pid` at step `step`.
__device__ __forceinline__ float3 ou_normals(uint32_t pid, uint64_t step, uint64_t seed) {
    const Philox4 r = philox4x32(pid, (uint32_t)step, DYN_STREAM_OU, (uint32_t)(step >> 32),
                                 (uint32_t)seed, (uint32_t)(seed >> 32));
    const float u0 = uniform24f(r.x[0]), v0 = uniform24f(r.x[1]);
    const float u1 = uniform24f(r.x[2]), v1 = uniform24f(r.x[3]);
    const float a = sqrtf(-2.0f * logf(u0));
    const float b = sqrtf(-2.0f * logf(u1));
    float s0, c0, s1, c1;
    sincospif(2.0f * v0, &s0, &c0);
    sincospif(2.0f * v1, &s1, &c1);
    return f3(a * c0, a * s0, b * c1);
}

// ---------------------------------------------------------------------------
// OPC water constants (src/solvent/mod.rs:58-94, src/solvent/opc_settle.rs:41)
// ---------------------------------------------------------------------------
#define OPC_O_MASS 16.0f
#define OPC_H_MASS 1.008f
#define OPC_MASS_MOL (16.0f + 2.0f * 1.008f)
#define OPC_O_EP_R 0.15939833f
#define OPC_O_H_R 0.87243313f
#define OPC_HOH_THETA 1.808161105066f
#define OPC_RA 0.5395199719801114f
#define CHARGE_UNIT_SCALER 18.2223f
#define OPC_Q_H (0.6791f * CHARGE_UNIT_SCALER)
#define OPC_Q_EP (-2.0f * OPC_Q_H)
#define OPC_O_SIGMA (1.777167268f * (2.0f / 1.122462048309373f))
#define OPC_O_EPS 0.2128008130f
#define OPC_C_H ((OPC_O_EP_R / OPC_RA) / 2.0f)
#define OPC_C_O (1.0f - 2.0f * OPC_C_H)
#define KCAL_TO_NATIVE 418.4f
#define KB_NATIVE 0.83144626f       // amu A^2 ps^-2 K^-1 (src/thermostat.rs:19)
#define GAS_CONST_R 0.0019872041    // kcal/mol/K (src/thermostat.rs:15)
#define BAR_PER_KCAL_MOL_A3 69476.95457055373
#define KB_BAR_A3 138.0649
#define INV_SQRT_PI_F 0.5641895835477563f
#define MAX_ACCEL 1.0e5f            // src/integrate.rs:26
// A water site lies within this distance of its O (the O-H bond).
#define OPC_SITE_REACH 0.8725f
