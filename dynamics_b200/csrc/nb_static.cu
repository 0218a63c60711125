// dyn_nb_forces_static: the flat-pair-list force evaluation of dyn_nb_forces
// for callers that must not allocate.
//
// Who needs it: code that runs where a device allocation is not allowed or
// not wanted -- a host framework that owns every device buffer through its
// own pool, a step enqueued from a callback that must not block on the
// allocator, or a process that has reserved the whole device for another
// engine.  The handle-based entry points allocate their staging and
// accumulator buffers at dyn_nb_create / dyn_nb_set_pairs time; this one
// takes every input and output as a device array from the caller and keeps
// its only scratch (the 64-bit fixed-point force accumulators, the per-block
// partial sums and a skipped-pair counter) in one file-scope device array of
// fixed size, so it calls no cudaMalloc, cudaFree or allocating library
// routine.
//
// Limits and sharing: the scratch holds DYN_NB_STATIC_MAX_SITES sites
// (atoms + 4 x waters) and is loaded on every device that loads this
// library, until the process exits.  All calls on a device share it and it
// keeps the last call's contents; each call clears the part it uses before
// accumulating.  Calls whose kernels overlap on one device (different
// streams with no ordering between them) race on the scratch and give wrong
// results.  The first call on each device sets that device up with it
// current: it looks up the scratch's device address (cudaGetSymbolAddress)
// and loads this entry point's kernels.  With the runtime's lazy module
// loading that first call is when the driver places the scratch in device
// memory, so make it before reserving the rest of the device for other
// work, and before any stream capture on that device.  The address is kept
// for the life of the process: after cudaDeviceReset the module is gone and
// this entry point must not be called again in that process.
#include <mutex>

#include "common.cuh"

namespace {

constexpr uint32_t ST_BLOCK = 256;
constexpr uint32_t ST_MAX_BLOCKS = 148 * 8;
constexpr uint32_t ST_MAX_DEVICES = 64;

// scratch layout in 64-bit words:
//   [0, 3*MAX_SITES)                      fixed-point forces, bodies back to back
//   [3*MAX_SITES, +2*ST_MAX_BLOCKS)       per-block (virial, energy) partials
//   [.. + 2*ST_MAX_BLOCKS]                skipped-pair counter
constexpr size_t ST_FORCE_WORDS = 3 * (size_t)DYN_NB_STATIC_MAX_SITES;
constexpr size_t ST_PART_WORDS = 2 * (size_t)ST_MAX_BLOCKS;
constexpr size_t ST_WORDS = ST_FORCE_WORDS + ST_PART_WORDS + 32;

// In host code this name is only a handle for cudaGetSymbolAddress, not a
// device address.
static __device__ __align__(256) long long g_nb_scratch[ST_WORDS];

std::mutex g_mu;
void* g_scratch_ptr[ST_MAX_DEVICES] = {};

struct StPos { const float* p[5]; };
struct StOut { double* f[5]; };
struct StSizes { uint32_t n[5]; uint32_t off[5]; };  // sites per body, word offset / 3

__device__ __forceinline__ float st_round_half_away(float q) {
    const float t = truncf(q);
    const float fr = __fsub_rn(q, t);
    return fabsf(fr) >= 0.5f ? t + copysignf(1.0f, q) : t;
}

// Pair arithmetic identical to the handle-based kernel (the reference CUDA
// kernel's conventions for CPU_SEM = false, src/cuda/cuda.cu:239-316; the
// CPU path's for CPU_SEM = true, src/non_bonded.rs:967-1054), reading the
// reference's unpacked per-pair arrays directly.
template <bool CPU_SEM>
__global__ void __launch_bounds__(ST_BLOCK) st_pair_kernel(
    StPos pos, StSizes sz, const uint32_t* __restrict__ tgt, const uint32_t* __restrict__ src,
    const float* __restrict__ sig, const float* __restrict__ eps, const float* __restrict__ qt,
    const float* __restrict__ qs, const uint8_t* __restrict__ btv, const uint8_t* __restrict__ bsv,
    const uint8_t* __restrict__ flv, uint64_t n, float3 ext, float3 inv_ext, float rc, float alpha,
    float ljc, uint32_t ovr, long long* __restrict__ scratch) {
    long long* fix = scratch;
    double* partials = reinterpret_cast<double*>(scratch + ST_FORCE_WORDS);
    unsigned long long* skipped = reinterpret_cast<unsigned long long*>(scratch + ST_FORCE_WORDS + ST_PART_WORDS);
    double w_acc = 0.0, e_acc = 0.0;
    const bool lj_off = ovr & DYN_OVR_LJ_DISABLED;
    const bool co_off = ovr & DYN_OVR_COULOMB_DISABLED;
    for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
         p += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t bt = btv[p], bs = bsv[p];
        const uint32_t it = tgt[p], is = src[p];
        if (bt > 4 || bs > 4 || it >= sz.n[bt] || is >= sz.n[bs]) {
            atomicAdd(skipped, 1ull);
            continue;
        }
        const uint32_t fl = flv[p];
        const bool scale14 = fl & DYN_PAIR_SCALE14, sym = fl & DYN_PAIR_SYMMETRIC;
        const float* at = pos.p[bt] + 3 * (size_t)it;
        const float* as = pos.p[bs] + 3 * (size_t)is;
        const float3 pt = f3(at[0], at[1], at[2]);
        const float3 ps = f3(as[0], as[1], as[2]);
        float3 d = pt - ps;
        if (CPU_SEM) {
            d.x = __fsub_rn(d.x, __fmul_rn(st_round_half_away(__fdiv_rn(d.x, ext.x)), ext.x));
            d.y = __fsub_rn(d.y, __fmul_rn(st_round_half_away(__fdiv_rn(d.y, ext.y)), ext.y));
            d.z = __fsub_rn(d.z, __fmul_rn(st_round_half_away(__fdiv_rn(d.z, ext.z)), ext.z));
        } else {
            d.x -= rintf(d.x * inv_ext.x) * ext.x;
            d.y -= rintf(d.y * inv_ext.y) * ext.y;
            d.z -= rintf(d.z * inv_ext.z) * ext.z;
        }
        const float r2 = d.x * d.x + d.y * d.y + d.z * d.z;
        if (r2 < (CPU_SEM ? 1e-12f : 1e-16f)) continue;
        const float inv_r = rsqrtf(r2);
        const float r = r2 * inv_r;
        const float2 lj = make_float2(sig[p], (fl & DYN_PAIR_LJ) ? eps[p] : 0.f);
        float fmag = 0.f, e = 0.f;
        if (!lj_off && lj.y != 0.f && (!CPU_SEM || r <= ljc)) {
            const float sr = lj.x * inv_r;
            const float sr2 = sr * sr;
            const float sr6 = sr2 * sr2 * sr2;
            const float sr12 = sr6 * sr6;
            float fl_ = 24.0f * lj.y * fmaf(2.f, sr12, -sr6) * inv_r;
            float el = 4.f * lj.y * (sr12 - sr6);
            if (scale14) { fl_ *= 0.5f; el *= 0.5f; }
            fmag += fl_; e += el;
        }
        const float qq = (fl & DYN_PAIR_COULOMB) ? __fmul_rn(qt[p], qs[p]) : 0.f;
        if (!co_off && qq != 0.f && r < rc) {
            const float ar = alpha * r;
            const float ec = erfcf(ar);
            const float ex = expf(-(ar * ar));
            float fc = qq * fmaf(ec, inv_r * inv_r, 2.0f * alpha * ex * INV_SQRT_PI_F * inv_r);
            float eco = qq * inv_r * ec;
            if (scale14) { fc *= 0.833333333f; eco *= 0.833333333f; }
            fmag += fc; e += eco;
        }
        const float3 f = d * (fmag * inv_r);
        w_acc += (double)d.x * (double)f.x + (double)d.y * (double)f.y + (double)d.z * (double)f.z;
        if (CPU_SEM ? (bt == 0 || bs == 0) : (bt == 0)) e_acc += (double)e;
        long long* ft = fix + 3 * ((size_t)sz.off[bt] + it);
        fix_atomic_add(ft + 0, fix_from_float(f.x));
        fix_atomic_add(ft + 1, fix_from_float(f.y));
        fix_atomic_add(ft + 2, fix_from_float(f.z));
        if (sym) {
            long long* fs = fix + 3 * ((size_t)sz.off[bs] + is);
            fix_atomic_add(fs + 0, -fix_from_float(f.x));
            fix_atomic_add(fs + 1, -fix_from_float(f.y));
            fix_atomic_add(fs + 2, -fix_from_float(f.z));
        }
    }
    double v[2] = {w_acc, e_acc};
    block_sum_d<2>(v);
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x + 0] = v[0];
        partials[2 * blockIdx.x + 1] = v[1];
    }
}

// Fixed-point scratch -> the caller's float64 force arrays.
__global__ void st_forces_out(StSizes sz, StOut out, const long long* __restrict__ scratch) {
    const size_t total = 3 * ((size_t)sz.off[4] + sz.n[4]);
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (size_t)gridDim.x * blockDim.x) {
        const size_t site = k / 3;
        int a = 4;
        while (a > 0 && site < sz.off[a]) --a;
        out.f[a][k - 3 * (size_t)sz.off[a]] = (double)scratch[k] * DYN_FIX_INV;
    }
}

// Block partials summed in a fixed order (deterministic); scalars receive
// virial, energy and the number of pairs skipped for a bad body code or index.
__global__ void st_scalars_out(int nblocks, const long long* __restrict__ scratch, double* __restrict__ scalars) {
    const double* partials = reinterpret_cast<const double*>(scratch + ST_FORCE_WORDS);
    const unsigned long long* skipped =
        reinterpret_cast<const unsigned long long*>(scratch + ST_FORCE_WORDS + ST_PART_WORDS);
    double v[2] = {0.0, 0.0};
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
        v[0] += partials[2 * b];
        v[1] += partials[2 * b + 1];
    }
    block_sum_d<2>(v);
    if (threadIdx.x == 0) {
        scalars[0] = v[0];
        scalars[1] = v[1];
        scalars[2] = (double)*skipped;
    }
}

// Set-up of the current device, once per device: the scratch's device
// address, and the device code of this entry point.  The CUDA runtime loads
// a module's code and its __device__ arrays lazily (CUDA_MODULE_LOADING=LAZY
// is the default since CUDA 12.2): the symbol lookup makes the driver load
// the scratch (its one allocation, made by the driver, not by this call's
// work), and querying each kernel's attributes loads the kernels, so that no
// later call loads anything -- not inside a stream capture either.
int scratch_for_current_device(long long** out) {
    int dev = 0;
    DYN_CUDA(cudaGetDevice(&dev));
    DYN_CHECK(dev >= 0 && (uint32_t)dev < ST_MAX_DEVICES, DYN_ERR_UNSUPPORTED,
              "dyn_nb_forces_static: device ordinal beyond 63");
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_nb_scratch);
        if (e != cudaSuccess) return dyn::cuda_fail(e, "dyn_nb_forces_static: cudaGetSymbolAddress");
        const void* ks[4] = {(const void*)st_pair_kernel<true>, (const void*)st_pair_kernel<false>,
                             (const void*)st_forces_out, (const void*)st_scalars_out};
        for (const void* k : ks) {
            cudaFuncAttributes fa;
            e = cudaFuncGetAttributes(&fa, k);
            if (e != cudaSuccess) return dyn::cuda_fail(e, "dyn_nb_forces_static: loading its kernels");
        }
        g_scratch_ptr[dev] = p;
    }
    *out = (long long*)g_scratch_ptr[dev];
    return DYN_OK;
}

}  // namespace

extern "C" int dyn_nb_forces_static(void* stream, uint32_t n_dyn, uint32_t n_water,
                                    const float* pos_dyn, const float* pos_w_o, const float* pos_w_m,
                                    const float* pos_w_h0, const float* pos_w_h1, uint64_t n_pairs,
                                    const uint32_t* tgt, const uint32_t* src, const float* sigma,
                                    const float* eps, const float* q_tgt, const float* q_src,
                                    const uint8_t* body_tgt, const uint8_t* body_src,
                                    const uint8_t* flags, const float cell_extent[3],
                                    float cutoff_ewald, float alpha_ewald, float lj_cutoff,
                                    uint32_t override_bits, double* f_dyn, double* f_w_o,
                                    double* f_w_m, double* f_w_h0, double* f_w_h1, double* scalars) {
    DYN_CHECK(cell_extent && scalars, DYN_ERR_INVALID, "dyn_nb_forces_static: NULL argument");
    DYN_CHECK(cutoff_ewald > 0.f && alpha_ewald > 0.f, DYN_ERR_INVALID,
              "dyn_nb_forces_static: cutoff and alpha must be > 0");
    for (int k = 0; k < 3; ++k)
        DYN_CHECK(cell_extent[k] > 0.f, DYN_ERR_INVALID, "dyn_nb_forces_static: extent must be > 0");
    const uint64_t sites = (uint64_t)n_dyn + 4ull * n_water;
    DYN_CHECK(sites <= DYN_NB_STATIC_MAX_SITES, DYN_ERR_INVALID,
              "dyn_nb_forces_static: n_dyn + 4*n_water exceeds DYN_NB_STATIC_MAX_SITES (131072)");
    const float* in[5] = {pos_dyn, pos_w_o, pos_w_m, pos_w_h0, pos_w_h1};
    double* outp[5] = {f_dyn, f_w_o, f_w_m, f_w_h0, f_w_h1};
    StPos pp;
    StOut op;
    StSizes sz;
    uint32_t off = 0;
    for (int a = 0; a < 5; ++a) {
        sz.n[a] = a == 0 ? n_dyn : n_water;
        sz.off[a] = off;
        off += sz.n[a];
        if (sz.n[a] > 0)
            DYN_CHECK(in[a] && outp[a], DYN_ERR_INVALID, "dyn_nb_forces_static: NULL position or force array");
        pp.p[a] = in[a];
        op.f[a] = outp[a];
    }
    if (n_pairs > 0)
        DYN_CHECK(tgt && src && sigma && eps && q_tgt && q_src && body_tgt && body_src && flags,
                  DYN_ERR_INVALID, "dyn_nb_forces_static: NULL pair array");
    long long* scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    // the forces in use, the partials and the counter start at zero
    DYN_CUDA(cudaMemsetAsync(scratch, 0, 3 * sites * sizeof(long long), st));
    DYN_CUDA(cudaMemsetAsync(scratch + ST_FORCE_WORDS, 0, (ST_PART_WORDS + 1) * sizeof(long long), st));
    const float3 ext = make_float3(cell_extent[0], cell_extent[1], cell_extent[2]);
    const float3 inv_ext = make_float3(1.0f / ext.x, 1.0f / ext.y, 1.0f / ext.z);
    int blocks = (int)std::min<uint64_t>((n_pairs + ST_BLOCK - 1) / ST_BLOCK, ST_MAX_BLOCKS);
    if (blocks < 1) blocks = 1;
    if (lj_cutoff > 0.f)
        st_pair_kernel<true><<<blocks, ST_BLOCK, 0, st>>>(pp, sz, tgt, src, sigma, eps, q_tgt, q_src, body_tgt,
                                                          body_src, flags, n_pairs, ext, inv_ext, cutoff_ewald,
                                                          alpha_ewald, lj_cutoff, override_bits, scratch);
    else
        st_pair_kernel<false><<<blocks, ST_BLOCK, 0, st>>>(pp, sz, tgt, src, sigma, eps, q_tgt, q_src, body_tgt,
                                                           body_src, flags, n_pairs, ext, inv_ext, cutoff_ewald,
                                                           alpha_ewald, lj_cutoff, override_bits, scratch);
    DYN_CUDA(cudaGetLastError());
    if (sites > 0) {
        const int ob = (int)std::min<uint64_t>((3 * sites + ST_BLOCK - 1) / ST_BLOCK, ST_MAX_BLOCKS);
        st_forces_out<<<ob, ST_BLOCK, 0, st>>>(sz, op, scratch);
        DYN_CUDA(cudaGetLastError());
    }
    st_scalars_out<<<1, ST_BLOCK, 0, st>>>(blocks, scratch, scalars);
    DYN_CUDA(cudaGetLastError());
    return DYN_OK;
}
