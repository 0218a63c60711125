// Layer 1 of the C ABI: a drop-in for src/gpu_interface.rs.
//
// The reference uploads 33 bytes of per-pair metadata (15 arrays) and
// evaluates one pair per thread with float atomics
// (src/cuda/cuda.cu:185-362).  Here the same flat pair list is re-packed to
// 20 bytes per pair (two 32-bit words holding index, body code and flag,
// (sigma, eps) and the product q_t q_s), evaluated one pair per thread with
// the reference's float32 pair math, and accumulated into 64-bit fixed-point
// forces, so results are bit-identical run to run.  The pair-list build
// (dyn_nb_build_pairs) replaces the reference's O(N^2) host rebuild with a
// GPU brute-force scan in the reference's exact float32 arithmetic.
// Pairs flagged alchemical (DYN_PAIR_ALCH, or marked by dyn_nb_mark_alch)
// take the reference's soft-core LJ and scaled Coulomb on the staged
// decoupling schedule (nonbonded_force_alchemical_kernel,
// src/cuda/cuda.cu:367-566; f_nonbonded_cpu, src/non_bonded.rs:950-1057).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"

namespace {

// packed pair words: w.x = target index (bits 0-26) | alchemical (27) |
// body (28-30) | scale14 (31); w.y = source index (0-27) | body | symmetric
constexpr uint32_t IDX_MASK = 0x0FFFFFFFu;
constexpr uint32_t TGT_MASK = 0x07FFFFFFu;
constexpr uint32_t ALCH_BIT = 0x08000000u;
constexpr int NB_PART = 3;  // virial, energy, dH/dlambda per block
constexpr int NB_BLOCK = 256;
constexpr int NB_MAX_BLOCKS = 148 * 8;

}  // namespace

struct dyn_nb_s {
    cudaStream_t stream = nullptr;
    uint32_t n_dyn = 0, n_water = 0;
    float rc = 10.f, alpha = 0.3f, ljc = 0.f;
    float* d_pos[5] = {};          // dyn, O, M, H0, H1: [3n] floats
    long long* d_f[5] = {};        // fixed-point forces [3n]
    double* d_partials = nullptr;  // [NB_MAX_BLOCKS * NB_PART]
    double* d_scalars = nullptr;   // virial, energy, dH/dlambda
    uint64_t n_alch = 0;           // installed pairs with the alchemical bit
    uint64_t n_pairs = 0, cap_pairs = 0;
    uint2* d_pidx = nullptr;       // packed target/source words
    float2* d_plj = nullptr;       // sigma, eps
    float* d_pqq = nullptr;        // q_t * q_s
    float* h_pos[5] = {};          // pinned staging
    long long* h_f[5] = {};
    double* h_scalars = nullptr;
    uint32_t n_of(int a) const { return a == 0 ? n_dyn : n_water; }
};

// ---------------------------------------------------------------------------
// pair evaluation
// ---------------------------------------------------------------------------

__device__ __forceinline__ float3 ld_pos(const float* const* pos, uint32_t body, uint32_t i) {
    // body 0 = atom array, 1..4 = water O, M, H0, H1 arrays
    const float* a = pos[body];
    return f3(a[3 * i + 0], a[3 * i + 1], a[3 * i + 2]);
}

__device__ __forceinline__ float round_half_away(float q) {
    const float t = truncf(q);
    const float fr = __fsub_rn(q, t);
    return fabsf(fr) >= 0.5f ? t + copysignf(1.0f, q) : t;
}

struct PosPtrs { const float* p[5]; };
struct ForcePtrs { long long* f[5]; };

// The staged decoupling schedule of one lambda (staged_decoupling_schedule,
// src/alchemical.rs:77-100): Coulomb scale and its lambda derivative over
// lambda 0..0.5, then the soft-core LJ lambda and its derivative over 0.5..1.
struct AlchSched { float cs, dcs, ll, dll; };

AlchSched alch_schedule(double lambda) {
    float l = (float)lambda;
    l = std::min(1.0f, std::max(0.0f, l));
    if (l < 0.5f) return {1.0f - 2.0f * l, -2.0f, 0.0f, 0.0f};
    return {0.0f, 0.0f, 2.0f * l - 1.0f, 2.0f};
}

// Beutler soft-core LJ of a decoupled pair (alchemical_lj_soft_core_decouple,
// src/non_bonded.rs:883-941; sc-alpha 0.5, power 1, soft-core sigma >= 3 A,
// src/alchemical.rs:55-65): V = (1 - l) V_LJ(r_sc), r_sc^6 = r^6 + 0.5 s^6 l.
// Returns the force magnitude along the pair direction (F_LJ(r_sc) (1 - l)
// (r / r_sc)^5), the energy and dV/dl = -V_LJ(r_sc) - (1 - l) F_LJ(r_sc)
// 0.5 s^6 / (6 r_sc^5).  r2 = 0 gives the energy at contact and no force.
__device__ __forceinline__ void soft_core(float r2, float sig, float eps, float lam, float& fmag,
                                          float& e, float& dvdl) {
    fmag = 0.f; e = 0.f; dvdl = 0.f;
    if (eps == 0.f || !isfinite(eps) || !isfinite(sig)) return;
    const float ss = fmaxf(sig, 3.0f), ss2 = ss * ss;
    const float ss6 = ss2 * ss2 * ss2;
    const float rsc6 = fmaf(0.5f * ss6, lam, r2 * r2 * r2);
    if (!(rsc6 > 0.f) || !isfinite(rsc6)) return;
    const float rsc = sqrtf(cbrtf(rsc6));
    const float inv_rsc = 1.0f / rsc;
    const float sr = sig * inv_rsc, sr2 = sr * sr;
    const float sr6 = sr2 * sr2 * sr2, sr12 = sr6 * sr6;
    const float hf = 24.0f * eps * fmaf(2.0f, sr12, -sr6) * inv_rsc;
    const float he = 4.0f * eps * (sr12 - sr6);
    const float scale = 1.0f - lam;
    const float q = sqrtf(r2) * inv_rsc, q2 = q * q;
    fmag = hf * scale * (q2 * q2 * q);
    e = he * scale;
    dvdl = -he - scale * hf * (0.5f * ss6) / (6.0f * (rsc6 * inv_rsc));
}

// CPU_SEM = false: the reference CUDA kernel's conventions
//   (src/cuda/cuda.cu:239-316, alchemical form 367-566): rint min-image by
//   multiplication, r^2 < 1e-16 skip, no LJ cutoff, energy only for atom
//   targets.
// CPU_SEM = true: f_nonbonded_cpu's conventions (src/non_bonded.rs:967-1054):
//   min-image by division with ties away from zero, r^2 < 1e-12 skip (an
//   alchemical pair there keeps its soft-core contact energy), LJ only for
//   r <= lj_cutoff, energy when either body is an atom.
// ALCH: pairs with the alchemical bit take soft-core LJ at the schedule's LJ
//   lambda and Coulomb times its scale; their dH/dlambda is summed.
template <bool CPU_SEM, bool ALCH>
__global__ void __launch_bounds__(NB_BLOCK) nb_pair_kernel(
    PosPtrs pos, ForcePtrs out, const uint2* __restrict__ pidx, const float2* __restrict__ plj,
    const float* __restrict__ pqq, uint64_t n, float3 ext, float3 inv_ext, float rc, float alpha,
    float ljc, uint32_t ovr, AlchSched al, double* __restrict__ partials) {
    double w_acc = 0.0, e_acc = 0.0, h_acc = 0.0;
    const bool lj_off = ovr & DYN_OVR_LJ_DISABLED;
    const bool co_off = ovr & DYN_OVR_COULOMB_DISABLED;
    for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
         p += (uint64_t)gridDim.x * blockDim.x) {
        const uint2 w = pidx[p];
        const uint32_t bt = (w.x >> 28) & 7u, bs = (w.y >> 28) & 7u;
        const uint32_t it = w.x & TGT_MASK, is = w.y & IDX_MASK;
        const bool scale14 = w.x >> 31, sym = w.y >> 31;
        const bool alch = ALCH && (w.x & ALCH_BIT);
        const bool e_counts = CPU_SEM ? (bt == 0 || bs == 0) : (bt == 0);
        const float3 pt = ld_pos(pos.p, bt, it);
        const float3 ps = ld_pos(pos.p, bs, is);
        float3 d = pt - ps;
        if (CPU_SEM) {
            d.x = __fsub_rn(d.x, __fmul_rn(round_half_away(__fdiv_rn(d.x, ext.x)), ext.x));
            d.y = __fsub_rn(d.y, __fmul_rn(round_half_away(__fdiv_rn(d.y, ext.y)), ext.y));
            d.z = __fsub_rn(d.z, __fmul_rn(round_half_away(__fdiv_rn(d.z, ext.z)), ext.z));
        } else {
            d.x -= rintf(d.x * inv_ext.x) * ext.x;
            d.y -= rintf(d.y * inv_ext.y) * ext.y;
            d.z -= rintf(d.z * inv_ext.z) * ext.z;
        }
        const float r2 = d.x * d.x + d.y * d.y + d.z * d.z;
        const float2 lj = plj[p];
        if (r2 < (CPU_SEM ? 1e-12f : 1e-16f)) {
            if (CPU_SEM && alch && !lj_off && lj.y != 0.f) {
                float fs, es, dv;
                soft_core(0.f, lj.x, lj.y, al.ll, fs, es, dv);
                if (scale14) { es *= 0.5f; dv *= 0.5f; }
                if (e_counts) e_acc += (double)es;
                h_acc += (double)(dv * al.dll);
            }
            continue;
        }
        const float inv_r = rsqrtf(r2);
        const float r = r2 * inv_r;
        float fmag = 0.f, e = 0.f, dh = 0.f;
        if (!lj_off && lj.y != 0.f && (!CPU_SEM || r <= ljc)) {
            float fl, el;
            if (alch) {
                soft_core(r2, lj.x, lj.y, al.ll, fl, el, dh);
                dh *= al.dll;
            } else {
                const float sr = lj.x * inv_r;
                const float sr2 = sr * sr;
                const float sr6 = sr2 * sr2 * sr2;
                const float sr12 = sr6 * sr6;
                fl = 24.0f * lj.y * fmaf(2.f, sr12, -sr6) * inv_r;
                el = 4.f * lj.y * (sr12 - sr6);
            }
            if (scale14) { fl *= 0.5f; el *= 0.5f; dh *= 0.5f; }
            fmag += fl; e += el;
        }
        const float qq = pqq[p];
        if (!co_off && qq != 0.f && r < rc) {
            const float ar = alpha * r;
            const float ec = erfcf(ar);
            const float ex = expf(-(ar * ar));
            float fc = qq * fmaf(ec, inv_r * inv_r, 2.0f * alpha * ex * INV_SQRT_PI_F * inv_r);
            float eco = qq * inv_r * ec;
            if (scale14) { fc *= 0.833333333f; eco *= 0.833333333f; }
            if (alch) {
                fmag += fc * al.cs; e += eco * al.cs;
                dh += eco * al.dcs;
            } else {
                fmag += fc; e += eco;
            }
        }
        const float3 f = d * (fmag * inv_r);
        w_acc += (double)d.x * (double)f.x + (double)d.y * (double)f.y + (double)d.z * (double)f.z;
        if (e_counts) e_acc += (double)e;
        if (ALCH) h_acc += (double)dh;
        long long* ft = out.f[bt] + 3 * (size_t)it;
        fix_atomic_add(ft + 0, fix_from_float(f.x));
        fix_atomic_add(ft + 1, fix_from_float(f.y));
        fix_atomic_add(ft + 2, fix_from_float(f.z));
        if (sym) {
            long long* fs = out.f[bs] + 3 * (size_t)is;
            fix_atomic_add(fs + 0, -fix_from_float(f.x));
            fix_atomic_add(fs + 1, -fix_from_float(f.y));
            fix_atomic_add(fs + 2, -fix_from_float(f.z));
        }
    }
    double v[NB_PART] = {w_acc, e_acc, h_acc};
    block_sum_d<NB_PART>(v);
    if (threadIdx.x == 0)
        for (int k = 0; k < NB_PART; ++k) partials[NB_PART * blockIdx.x + k] = v[k];
}

// Sums block partials in a fixed order (deterministic).
__global__ void nb_finalize_kernel(const double* __restrict__ partials, int nblocks,
                                   double* __restrict__ scalars) {
    double v[NB_PART] = {0.0, 0.0, 0.0};
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
        for (int k = 0; k < NB_PART; ++k) v[k] += partials[NB_PART * b + k];
    block_sum_d<NB_PART>(v);
    if (threadIdx.x == 0)
        for (int k = 0; k < NB_PART; ++k) scalars[k] = v[k];
}

// Marks the installed pairs that cross the boundary of the atom range
// [lo, hi) as alchemical, as setup_pairs does for the alchemical molecule
// (src/non_bonded.rs:581-612): atom-atom pairs with exactly one end inside,
// atom-water pairs whose atom is inside; water-water pairs never.  Clears
// the bit on every other pair and counts the marked ones.
__global__ void mark_alch_kernel(uint64_t n, uint32_t lo, uint32_t hi, uint2* __restrict__ pidx,
                                 unsigned long long* __restrict__ count) {
    uint32_t c = 0;
    for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
         p += (uint64_t)gridDim.x * blockDim.x) {
        uint2 w = pidx[p];
        const uint32_t bt = (w.x >> 28) & 7u, bs = (w.y >> 28) & 7u;
        const uint32_t it = w.x & TGT_MASK, is = w.y & IDX_MASK;
        const bool in_t = bt == 0 && it >= lo && it < hi;
        const bool in_s = bs == 0 && is >= lo && is < hi;
        const bool a = in_t != in_s;
        w.x = a ? (w.x | ALCH_BIT) : (w.x & ~ALCH_BIT);
        pidx[p] = w;
        c += a;
    }
    c = __reduce_add_sync(0xffffffffu, c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, (unsigned long long)c);
}

__global__ void pack_pairs_kernel(uint64_t n, const uint32_t* __restrict__ tgt,
                                  const uint32_t* __restrict__ src, const float* __restrict__ sig,
                                  const float* __restrict__ eps, const float* __restrict__ qt,
                                  const float* __restrict__ qs, const uint8_t* __restrict__ bt,
                                  const uint8_t* __restrict__ bs, const uint8_t* __restrict__ fl,
                                  uint2* __restrict__ pidx, float2* __restrict__ plj,
                                  float* __restrict__ pqq) {
    for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
         p += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t f = fl[p];
        uint2 w;
        w.x = (tgt[p] & TGT_MASK) | ((uint32_t)(bt[p] & 7u) << 28) |
              ((f & DYN_PAIR_SCALE14) ? 0x80000000u : 0u) | ((f & DYN_PAIR_ALCH) ? ALCH_BIT : 0u);
        w.y = (src[p] & IDX_MASK) | ((uint32_t)(bs[p] & 7u) << 28) | ((f & DYN_PAIR_SYMMETRIC) ? 0x80000000u : 0u);
        pidx[p] = w;
        plj[p] = make_float2(sig[p], (f & DYN_PAIR_LJ) ? eps[p] : 0.f);
        pqq[p] = (f & DYN_PAIR_COULOMB) ? __fmul_rn(qt[p], qs[p]) : 0.f;
    }
}

// ---------------------------------------------------------------------------
// reference-exact neighbour lists (src/neighbors.rs:180-281) + setup_pairs
// ---------------------------------------------------------------------------

// SimBox::min_image in float32, no contraction (src/barostat.rs:162-170).
__device__ __forceinline__ float mi1(float dv, float e) {
    return __fsub_rn(dv, __fmul_rn(round_half_away(__fdiv_rn(dv, e)), e));
}
__device__ __forceinline__ float dist2_ref(float3 a, float3 b, float3 ext) {
    const float x = mi1(__fsub_rn(a.x, b.x), ext.x);
    const float y = mi1(__fsub_rn(a.y, b.y), ext.y);
    const float z = mi1(__fsub_rn(a.z, b.z), ext.z);
    return __fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), __fmul_rn(z, z));
}
// SimBox::wrap (src/barostat.rs:141-157): rem_euclid then + lo.
__device__ __forceinline__ float wrap1(float p, float lo, float e) {
    float r = fmodf(__fsub_rn(p, lo), e);
    if (r < 0.f) r = __fadd_rn(r, fabsf(e));
    return __fadd_rn(r, lo);
}

__global__ void wrap_o_kernel(uint32_t nw, const float* __restrict__ o, float3 lo, float3 ext,
                              float* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nw) return;
    out[3 * i + 0] = wrap1(o[3 * i + 0], lo.x, ext.x);
    out[3 * i + 1] = wrap1(o[3 * i + 1], lo.y, ext.y);
    out[3 * i + 2] = wrap1(o[3 * i + 2], lo.z, ext.z);
}

__device__ __forceinline__ bool in_sorted(const uint32_t* a, uint32_t n, uint32_t v) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t m = (lo + hi) >> 1;
        if (a[m] < v) lo = m + 1; else hi = m;
    }
    return lo < n && a[lo] == v;
}

struct ListArgs {
    const float* outer;    // [3*n_outer]
    const float* inner;    // [3*n_inner]
    uint32_t n_outer, n_inner;
    int mode;              // 0 std-std (half, j>i), 1 std-water, 2 water-water (half)
    float thr;             // (cutoff+skin)^2
    float3 ext;
    const uint8_t* is_static;
    const uint8_t* bonded_only;
    const uint32_t* ex_off; const uint32_t* ex_idx;   // exclusions CSR (std-std)
    const uint32_t* s14_off; const uint32_t* s14_idx; // 1-4 CSR
};

// One warp per outer row; inner indices are scanned in ascending order and
// compacted with ballots, so rows come out sorted, as in the reference.
// PASS 0 counts pairs per row; PASS 1 writes them at row offsets.
template <int PASS>
__global__ void ref_list_kernel(ListArgs a, uint32_t* __restrict__ row_count,
                                const uint64_t* __restrict__ row_off, uint32_t* __restrict__ out_j,
                                uint8_t* __restrict__ out_s14) {
    const int lane = threadIdx.x & 31;
    const uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (row >= a.n_outer) return;
    const float3 pi = f3(a.outer[3 * row], a.outer[3 * row + 1], a.outer[3 * row + 2]);
    const uint32_t j0 = (a.mode == 1) ? 0u : row + 1;
    uint32_t cnt = 0;
    uint64_t base = PASS ? row_off[row] : 0;
    for (uint32_t jb = j0; jb < a.n_inner; jb += 32) {
        const uint32_t j = jb + lane;
        bool hit = false;
        bool s14 = false;
        if (j < a.n_inner) {
            const float3 pj = f3(a.inner[3 * j], a.inner[3 * j + 1], a.inner[3 * j + 2]);
            bool skip = false;
            if (a.mode == 0) {
                if (a.is_static && a.is_static[row] && a.is_static[j]) skip = true;
            }
            if (!skip) hit = dist2_ref(pi, pj, a.ext) < a.thr;
            if (hit && a.mode == 0) {
                // setup_pairs filters (src/non_bonded.rs:572-580)
                if (a.bonded_only && (a.bonded_only[row] || a.bonded_only[j])) hit = false;
                if (hit && a.ex_off &&
                    in_sorted(a.ex_idx + a.ex_off[row], a.ex_off[row + 1] - a.ex_off[row], j))
                    hit = false;
                if (hit && a.s14_off)
                    s14 = in_sorted(a.s14_idx + a.s14_off[row], a.s14_off[row + 1] - a.s14_off[row], j);
            }
        }
        const uint32_t m = __ballot_sync(0xffffffffu, hit);
        if (PASS && hit) {
            const uint32_t k = cnt + __popc(m & ((1u << lane) - 1u));
            out_j[base + k] = j;
            if (out_s14) out_s14[base + k] = s14;
        }
        cnt += __popc(m);
    }
    if (!PASS && lane == 0) row_count[row] = cnt;
}

// Emits the flat SoA of setup_pairs from the per-row neighbour arrays.
struct EmitArgs {
    uint32_t n_std, n_water;
    const uint64_t* ss_off; const uint32_t* ss_j; const uint8_t* ss_s14;
    const uint64_t* sw_off; const uint32_t* sw_j;
    const uint64_t* ww_off; const uint32_t* ww_j;
    uint64_t base_sw, base_ww;
    const float* q; const float* sig; const float* eps;
};

// water site codes in setup_pairs' iteration order O, M, H0, H1
__device__ __forceinline__ float site_q(uint32_t s) {
    return s == DYN_BODY_W_O ? 0.f : (s == DYN_BODY_W_M ? OPC_Q_EP : OPC_Q_H);
}

__global__ void emit_ss_kernel(EmitArgs a, uint2* pidx, float2* plj, float* pqq) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_std) return;
    for (uint64_t k = a.ss_off[i]; k < a.ss_off[i + 1]; ++k) {
        const uint32_t j = a.ss_j[k];
        const bool s14 = a.ss_s14[k];
        pidx[k] = make_uint2(i | (s14 ? 0x80000000u : 0u), j | 0x80000000u);
        // combine_lj_params (src/non_bonded.rs:1081-1086)
        plj[k] = make_float2(__fmul_rn(0.5f, __fadd_rn(a.sig[i], a.sig[j])),
                             __fsqrt_rn(__fmul_rn(a.eps[i], a.eps[j])));
        pqq[k] = __fmul_rn(a.q[i], a.q[j]);
    }
}

__global__ void emit_sw_kernel(EmitArgs a, uint2* pidx, float2* plj, float* pqq) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_std) return;
    // water_std row of LjTables (src/non_bonded.rs:139-145)
    const float sg = __fmul_rn(0.5f, __fadd_rn(a.sig[i], OPC_O_SIGMA));
    const float ep = __fsqrt_rn(__fmul_rn(a.eps[i], OPC_O_EPS));
    for (uint64_t k = a.sw_off[i]; k < a.sw_off[i + 1]; ++k) {
        const uint32_t w = a.sw_j[k];
        const uint64_t o = a.base_sw + 4 * k;
        const uint32_t sites[4] = {DYN_BODY_W_O, DYN_BODY_W_M, DYN_BODY_W_H0, DYN_BODY_W_H1};
        for (int s = 0; s < 4; ++s) {
            pidx[o + s] = make_uint2(i, w | (sites[s] << 28) | 0x80000000u);
            plj[o + s] = make_float2(sg, s == 0 ? ep : 0.f);
            pqq[o + s] = s == 0 ? 0.f : __fmul_rn(a.q[i], site_q(sites[s]));
        }
    }
}

__global__ void emit_ww_kernel(EmitArgs a, uint2* pidx, float2* plj, float* pqq) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_water) return;
    const uint32_t sites[4] = {DYN_BODY_W_O, DYN_BODY_W_M, DYN_BODY_W_H0, DYN_BODY_W_H1};
    for (uint64_t k = a.ww_off[i]; k < a.ww_off[i + 1]; ++k) {
        const uint32_t j = a.ww_j[k];
        uint64_t o = a.base_ww + 10 * k;
        for (int s0 = 0; s0 < 4; ++s0)
            for (int s1 = 0; s1 < 4; ++s1) {
                const bool lj = s0 == 0 && s1 == 0;
                const bool co = s0 != 0 && s1 != 0;
                if (!(lj || co)) continue;
                pidx[o] = make_uint2(i | (sites[s0] << 28), j | (sites[s1] << 28) | 0x80000000u);
                plj[o] = make_float2(OPC_O_SIGMA, lj ? OPC_O_EPS : 0.f);
                pqq[o] = co ? __fmul_rn(site_q(sites[s0]), site_q(sites[s1])) : 0.f;
                ++o;
            }
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
namespace {

template <typename T>
int dalloc(T** p, size_t n) {
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
    if (e != cudaSuccess) return dyn::cuda_fail(e, "cudaMalloc");
    return DYN_OK;
}
template <typename T>
int halloc(T** p, size_t n) {
    if (n == 0) n = 1;
    cudaError_t e = cudaMallocHost((void**)p, n * sizeof(T));
    if (e != cudaSuccess) return dyn::cuda_fail(e, "cudaMallocHost");
    return DYN_OK;
}

int ensure_pair_capacity(dyn_nb_s* h, uint64_t n) {
    if (n <= h->cap_pairs) return DYN_OK;
    cudaFree(h->d_pidx); cudaFree(h->d_plj); cudaFree(h->d_pqq);
    h->d_pidx = nullptr; h->d_plj = nullptr; h->d_pqq = nullptr; h->cap_pairs = 0;
    int rc;
    if ((rc = dalloc(&h->d_pidx, n)) || (rc = dalloc(&h->d_plj, n)) || (rc = dalloc(&h->d_pqq, n)))
        return rc;
    h->cap_pairs = n;
    return DYN_OK;
}

void build_csr(uint32_t n, uint64_t m, const uint32_t* pairs, std::vector<uint32_t>& off,
               std::vector<uint32_t>& idx) {
    // symmetric CSR of (i, j) pairs, each row sorted ascending
    std::vector<std::vector<uint32_t>> rows(n);
    for (uint64_t k = 0; k < m; ++k) {
        const uint32_t i = pairs[2 * k], j = pairs[2 * k + 1];
        if (i < n && j < n) { rows[i].push_back(j); rows[j].push_back(i); }
    }
    off.assign(n + 1, 0);
    idx.clear();
    for (uint32_t i = 0; i < n; ++i) {
        std::sort(rows[i].begin(), rows[i].end());
        rows[i].erase(std::unique(rows[i].begin(), rows[i].end()), rows[i].end());
        off[i + 1] = off[i] + (uint32_t)rows[i].size();
        idx.insert(idx.end(), rows[i].begin(), rows[i].end());
    }
}

// exclusive scan of row counts on the host (rows are few relative to pairs)
int scan_rows(cudaStream_t st, const uint32_t* d_cnt, uint32_t n, uint64_t* d_off,
              uint64_t* total) {
    std::vector<uint32_t> c(n);
    std::vector<uint64_t> o(n + 1, 0);
    if (n) DYN_CUDA(cudaMemcpyAsync(c.data(), d_cnt, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    DYN_CUDA(cudaStreamSynchronize(st));
    for (uint32_t i = 0; i < n; ++i) o[i + 1] = o[i] + c[i];
    DYN_CUDA(cudaMemcpyAsync(d_off, o.data(), (n + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
    DYN_CUDA(cudaStreamSynchronize(st));
    *total = o[n];
    return DYN_OK;
}

}  // namespace

extern "C" int dyn_nb_create(void* stream, uint32_t n_dyn, uint32_t n_water, float cutoff_ewald,
                             float alpha_ewald, float lj_cutoff, dyn_nb_t* out) {
    DYN_CHECK(out != nullptr, DYN_ERR_INVALID, "dyn_nb_create: out is NULL");
    DYN_CHECK(cutoff_ewald > 0.f && alpha_ewald > 0.f, DYN_ERR_INVALID,
              "dyn_nb_create: cutoff and alpha must be > 0");
    DYN_CHECK(n_dyn < (1u << 27) && n_water < (1u << 27), DYN_ERR_INVALID,
              "dyn_nb_create: fewer than 2^27 atoms / waters");
    *out = nullptr;
    dyn_nb_s* h = new dyn_nb_s();
    h->stream = (cudaStream_t)stream;
    h->n_dyn = n_dyn; h->n_water = n_water;
    h->rc = cutoff_ewald; h->alpha = alpha_ewald; h->ljc = lj_cutoff;
    int rc = DYN_OK;
    for (int a = 0; a < 5 && rc == DYN_OK; ++a) {
        const size_t n3 = 3 * (size_t)std::max(1u, h->n_of(a));
        if ((rc = dalloc(&h->d_pos[a], n3)) || (rc = dalloc(&h->d_f[a], n3)) ||
            (rc = halloc(&h->h_pos[a], n3)) || (rc = halloc(&h->h_f[a], n3)))
            break;
    }
    if (rc == DYN_OK) rc = dalloc(&h->d_partials, NB_PART * NB_MAX_BLOCKS);
    if (rc == DYN_OK) rc = dalloc(&h->d_scalars, NB_PART);
    if (rc == DYN_OK) rc = halloc(&h->h_scalars, NB_PART);
    if (rc != DYN_OK) {
        dyn_nb_destroy(h);
        return rc;
    }
    *out = h;
    return DYN_OK;
}

extern "C" int dyn_nb_destroy(dyn_nb_t h) {
    if (!h) return DYN_OK;
    if (h->stream) cudaStreamSynchronize(h->stream); else cudaDeviceSynchronize();
    for (int a = 0; a < 5; ++a) {
        cudaFree(h->d_pos[a]); cudaFree(h->d_f[a]);
        cudaFreeHost(h->h_pos[a]); cudaFreeHost(h->h_f[a]);
    }
    cudaFree(h->d_partials); cudaFree(h->d_scalars); cudaFreeHost(h->h_scalars);
    cudaFree(h->d_pidx); cudaFree(h->d_plj); cudaFree(h->d_pqq);
    delete h;
    return DYN_OK;
}

extern "C" int dyn_nb_set_pairs(dyn_nb_t h, uint64_t n, const uint32_t* tgt, const uint32_t* src,
                                const float* sigma, const float* eps, const float* q_tgt,
                                const float* q_src, const uint8_t* body_tgt,
                                const uint8_t* body_src, const uint8_t* flags) {
    DYN_CHECK(h, DYN_ERR_INVALID, "dyn_nb_set_pairs: NULL handle");
    if (n > 0)
        DYN_CHECK(tgt && src && sigma && eps && q_tgt && q_src && body_tgt && body_src && flags,
                  DYN_ERR_INVALID, "dyn_nb_set_pairs: NULL array");
    for (uint64_t p = 0; p < n; ++p) {
        const uint32_t bt = body_tgt[p], bs = body_src[p];
        if (bt > 4 || bs > 4) return dyn::fail(DYN_ERR_INVALID, "dyn_nb_set_pairs: body code > 4");
        if (tgt[p] >= (bt ? h->n_water : h->n_dyn) || src[p] >= (bs ? h->n_water : h->n_dyn))
            return dyn::fail(DYN_ERR_INVALID, "dyn_nb_set_pairs: pair index out of range");
    }
    int rc = ensure_pair_capacity(h, n);
    if (rc) return rc;
    h->n_pairs = n;
    h->n_alch = 0;
    for (uint64_t p = 0; p < n; ++p) h->n_alch += (flags[p] & DYN_PAIR_ALCH) != 0;
    if (n == 0) return DYN_OK;
    // stage through temporary device buffers, then pack
    void* tmp = nullptr;
    const size_t bytes = n * (4 + 4 + 4 + 4 + 4 + 4 + 1 + 1 + 1);
    DYN_CUDA(cudaMalloc(&tmp, bytes));
    char* b = (char*)tmp;
    uint32_t* dt = (uint32_t*)b; b += 4 * n;
    uint32_t* ds = (uint32_t*)b; b += 4 * n;
    float* dsg = (float*)b; b += 4 * n;
    float* dep = (float*)b; b += 4 * n;
    float* dqt = (float*)b; b += 4 * n;
    float* dqs = (float*)b; b += 4 * n;
    uint8_t* dbt = (uint8_t*)b; b += n;
    uint8_t* dbs = (uint8_t*)b; b += n;
    uint8_t* dfl = (uint8_t*)b;
    cudaStream_t st = h->stream;
    cudaMemcpyAsync(dt, tgt, 4 * n, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(ds, src, 4 * n, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dsg, sigma, 4 * n, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dep, eps, 4 * n, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dqt, q_tgt, 4 * n, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dqs, q_src, 4 * n, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dbt, body_tgt, n, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dbs, body_src, n, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dfl, flags, n, cudaMemcpyHostToDevice, st);
    const int blocks = (int)std::min<uint64_t>((n + 255) / 256, 148 * 16);
    pack_pairs_kernel<<<blocks, 256, 0, st>>>(n, dt, ds, dsg, dep, dqt, dqs, dbt, dbs, dfl,
                                              h->d_pidx, h->d_plj, h->d_pqq);
    DYN_CUDA(cudaGetLastError());
    DYN_CUDA(cudaStreamSynchronize(st));
    cudaFree(tmp);
    return DYN_OK;
}

extern "C" int dyn_nb_get_pairs(dyn_nb_t h, uint64_t n, uint32_t* tgt, uint32_t* src,
                                float* sigma, float* eps, float* q_tgt, float* q_src,
                                uint8_t* body_tgt, uint8_t* body_src, uint8_t* flags) {
    DYN_CHECK(h, DYN_ERR_INVALID, "dyn_nb_get_pairs: NULL handle");
    DYN_CHECK(n <= h->n_pairs, DYN_ERR_INVALID, "dyn_nb_get_pairs: n exceeds installed pairs");
    if (n == 0) return DYN_OK;
    std::vector<uint2> idx(n);
    std::vector<float2> lj(n);
    std::vector<float> qq(n);
    cudaStream_t st = h->stream;
    DYN_CUDA(cudaMemcpyAsync(idx.data(), h->d_pidx, n * sizeof(uint2), cudaMemcpyDeviceToHost, st));
    DYN_CUDA(cudaMemcpyAsync(lj.data(), h->d_plj, n * sizeof(float2), cudaMemcpyDeviceToHost, st));
    DYN_CUDA(cudaMemcpyAsync(qq.data(), h->d_pqq, n * sizeof(float), cudaMemcpyDeviceToHost, st));
    DYN_CUDA(cudaStreamSynchronize(st));
    for (uint64_t p = 0; p < n; ++p) {
        const uint32_t bt = (idx[p].x >> 28) & 7u, bs = (idx[p].y >> 28) & 7u;
        if (tgt) tgt[p] = idx[p].x & TGT_MASK;
        if (src) src[p] = idx[p].y & IDX_MASK;
        if (body_tgt) body_tgt[p] = (uint8_t)bt;
        if (body_src) body_src[p] = (uint8_t)bs;
        if (sigma) sigma[p] = lj[p].x;
        if (eps) eps[p] = lj[p].y;
        if (q_tgt) q_tgt[p] = qq[p];   // the product q_t q_s is what is stored
        if (q_src) q_src[p] = 1.0f;
        if (flags) {
            uint8_t f = 0;
            if (idx[p].x >> 31) f |= DYN_PAIR_SCALE14;
            if (idx[p].y >> 31) f |= DYN_PAIR_SYMMETRIC;
            if (idx[p].x & ALCH_BIT) f |= DYN_PAIR_ALCH;
            if (lj[p].y != 0.f) f |= DYN_PAIR_LJ;
            // setup_pairs sets calc_coulomb for every pair but water O ones
            const bool o_t = bt == DYN_BODY_W_O, o_s = bs == DYN_BODY_W_O;
            if (!(o_t || o_s)) f |= DYN_PAIR_COULOMB;
            flags[p] = f;
        }
    }
    return DYN_OK;
}

extern "C" int dyn_nb_build_pairs(dyn_nb_t h, const float* pos_dyn, const float* pos_w_o,
                                  const float* atom_q, const float* atom_sigma,
                                  const float* atom_eps, const uint8_t* is_static,
                                  const uint8_t* bonded_only, uint64_t n_excl,
                                  const uint32_t* excl, uint64_t n_pair14, const uint32_t* pair14,
                                  const float box_lo[3], const float box_hi[3], float skin,
                                  uint64_t* n_pairs_out) {
    DYN_CHECK(h && box_lo && box_hi, DYN_ERR_INVALID, "dyn_nb_build_pairs: NULL argument");
    DYN_CHECK(h->n_dyn == 0 || (pos_dyn && atom_q && atom_sigma && atom_eps), DYN_ERR_INVALID,
              "dyn_nb_build_pairs: atom arrays required");
    DYN_CHECK(h->n_water == 0 || pos_w_o, DYN_ERR_INVALID, "dyn_nb_build_pairs: water O required");
    DYN_CHECK(skin >= 0.f, DYN_ERR_INVALID, "dyn_nb_build_pairs: skin < 0");
    const uint32_t ns = h->n_dyn, nw = h->n_water;
    cudaStream_t st = h->stream;
    // float32 exactly as the reference: extent = hi - lo, thr = (c+s)*(c+s)
    float ext_h[3], lo_h[3];
    for (int k = 0; k < 3; ++k) {
        lo_h[k] = box_lo[k];
        volatile float e = box_hi[k] - box_lo[k];
        ext_h[k] = e;
        DYN_CHECK(ext_h[k] > 0.f, DYN_ERR_INVALID, "dyn_nb_build_pairs: box extent must be > 0");
    }
    volatile float cs = h->rc + skin;
    const float thr = cs * cs;
    const float3 ext = make_float3(ext_h[0], ext_h[1], ext_h[2]);
    // exclusion / 1-4 CSR
    std::vector<uint32_t> ex_off, ex_idx, s_off, s_idx;
    build_csr(ns, n_excl, excl, ex_off, ex_idx);
    build_csr(ns, n_pair14, pair14, s_off, s_idx);
    // device scratch
    float *d_atoms = nullptr, *d_wo = nullptr, *d_wo_raw = nullptr, *d_q = nullptr, *d_sig = nullptr,
          *d_eps = nullptr;
    uint8_t *d_static = nullptr, *d_bonly = nullptr, *d_s14 = nullptr;
    uint32_t *d_exo = nullptr, *d_exi = nullptr, *d_so = nullptr, *d_si = nullptr, *d_cnt = nullptr,
             *d_ssj = nullptr, *d_swj = nullptr, *d_wwj = nullptr;
    uint64_t *d_sso = nullptr, *d_swo = nullptr, *d_wwo = nullptr;
    int rc = DYN_OK;
    auto cleanup = [&]() {
        cudaFree(d_atoms); cudaFree(d_wo); cudaFree(d_wo_raw); cudaFree(d_q); cudaFree(d_sig);
        cudaFree(d_eps); cudaFree(d_static); cudaFree(d_bonly); cudaFree(d_s14); cudaFree(d_exo);
        cudaFree(d_exi); cudaFree(d_so); cudaFree(d_si); cudaFree(d_cnt); cudaFree(d_ssj);
        cudaFree(d_swj); cudaFree(d_wwj); cudaFree(d_sso); cudaFree(d_swo); cudaFree(d_wwo);
    };
#define TRY(x) do { if ((rc = (x)) != DYN_OK) { cleanup(); return rc; } } while (0)
#define TRYC(x) do { cudaError_t _e = (x); if (_e != cudaSuccess) { cleanup(); return dyn::cuda_fail(_e, #x); } } while (0)
    TRY(dalloc(&d_atoms, 3 * (size_t)ns)); TRY(dalloc(&d_q, ns)); TRY(dalloc(&d_sig, ns));
    TRY(dalloc(&d_eps, ns)); TRY(dalloc(&d_wo, 3 * (size_t)nw)); TRY(dalloc(&d_wo_raw, 3 * (size_t)nw));
    TRY(dalloc(&d_exo, ns + 1)); TRY(dalloc(&d_exi, ex_idx.size())); TRY(dalloc(&d_so, ns + 1));
    TRY(dalloc(&d_si, s_idx.size())); TRY(dalloc(&d_cnt, std::max(ns, nw)));
    TRY(dalloc(&d_sso, ns + 1)); TRY(dalloc(&d_swo, ns + 1)); TRY(dalloc(&d_wwo, nw + 1));
    if (is_static) { TRY(dalloc(&d_static, ns)); TRYC(cudaMemcpyAsync(d_static, is_static, ns, cudaMemcpyHostToDevice, st)); }
    if (bonded_only) { TRY(dalloc(&d_bonly, ns)); TRYC(cudaMemcpyAsync(d_bonly, bonded_only, ns, cudaMemcpyHostToDevice, st)); }
    if (ns) {
        TRYC(cudaMemcpyAsync(d_atoms, pos_dyn, 12 * (size_t)ns, cudaMemcpyHostToDevice, st));
        TRYC(cudaMemcpyAsync(d_q, atom_q, 4 * (size_t)ns, cudaMemcpyHostToDevice, st));
        TRYC(cudaMemcpyAsync(d_sig, atom_sigma, 4 * (size_t)ns, cudaMemcpyHostToDevice, st));
        TRYC(cudaMemcpyAsync(d_eps, atom_eps, 4 * (size_t)ns, cudaMemcpyHostToDevice, st));
    }
    TRYC(cudaMemcpyAsync(d_exo, ex_off.data(), 4 * ex_off.size(), cudaMemcpyHostToDevice, st));
    if (!ex_idx.empty()) TRYC(cudaMemcpyAsync(d_exi, ex_idx.data(), 4 * ex_idx.size(), cudaMemcpyHostToDevice, st));
    TRYC(cudaMemcpyAsync(d_so, s_off.data(), 4 * s_off.size(), cudaMemcpyHostToDevice, st));
    if (!s_idx.empty()) TRYC(cudaMemcpyAsync(d_si, s_idx.data(), 4 * s_idx.size(), cudaMemcpyHostToDevice, st));
    if (nw) {
        TRYC(cudaMemcpyAsync(d_wo_raw, pos_w_o, 12 * (size_t)nw, cudaMemcpyHostToDevice, st));
        wrap_o_kernel<<<(nw + 255) / 256, 256, 0, st>>>(nw, d_wo_raw, make_float3(lo_h[0], lo_h[1], lo_h[2]), ext, d_wo);
        TRYC(cudaGetLastError());
    }
    uint64_t n_ss = 0, n_sw = 0, n_ww = 0;
    ListArgs la{};
    la.thr = thr; la.ext = ext;
    la.is_static = d_static; la.bonded_only = d_bonly;
    la.ex_off = d_exo; la.ex_idx = d_exi; la.s14_off = d_so; la.s14_idx = d_si;
    auto run_list = [&](const float* outer, const float* inner, uint32_t no, uint32_t ni, int mode,
                        uint64_t* d_off, uint32_t** d_j, uint8_t** d_s14o, uint64_t* total) -> int {
        ListArgs a = la;
        a.outer = outer; a.inner = inner; a.n_outer = no; a.n_inner = ni; a.mode = mode;
        if (mode != 0) { a.ex_off = nullptr; a.s14_off = nullptr; a.bonded_only = nullptr; a.is_static = nullptr; }
        const int threads = 256;
        const int blocks = (int)(((uint64_t)no * 32 + threads - 1) / threads);
        if (no) {
            ref_list_kernel<0><<<blocks, threads, 0, st>>>(a, d_cnt, nullptr, nullptr, nullptr);
            DYN_CUDA(cudaGetLastError());
        }
        int r = scan_rows(st, d_cnt, no, d_off, total);
        if (r) return r;
        if ((r = dalloc(d_j, *total))) return r;
        if (d_s14o && (r = dalloc(d_s14o, *total))) return r;
        if (no) {
            ref_list_kernel<1><<<blocks, threads, 0, st>>>(a, nullptr, d_off, *d_j, d_s14o ? *d_s14o : nullptr);
            DYN_CUDA(cudaGetLastError());
        }
        return DYN_OK;
    };
    TRY(run_list(d_atoms, d_atoms, ns, ns, 0, d_sso, &d_ssj, &d_s14, &n_ss));
    TRY(run_list(d_atoms, d_wo, ns, nw, 1, d_swo, &d_swj, nullptr, &n_sw));
    TRY(run_list(d_wo, d_wo, nw, nw, 2, d_wwo, &d_wwj, nullptr, &n_ww));
    const uint64_t total = n_ss + 4 * n_sw + 10 * n_ww;
    TRY(ensure_pair_capacity(h, total));
    EmitArgs ea{};
    ea.n_std = ns; ea.n_water = nw;
    ea.ss_off = d_sso; ea.ss_j = d_ssj; ea.ss_s14 = d_s14;
    ea.sw_off = d_swo; ea.sw_j = d_swj; ea.ww_off = d_wwo; ea.ww_j = d_wwj;
    ea.base_sw = n_ss; ea.base_ww = n_ss + 4 * n_sw;
    ea.q = d_q; ea.sig = d_sig; ea.eps = d_eps;
    if (ns) {
        emit_ss_kernel<<<(ns + 127) / 128, 128, 0, st>>>(ea, h->d_pidx, h->d_plj, h->d_pqq);
        emit_sw_kernel<<<(ns + 127) / 128, 128, 0, st>>>(ea, h->d_pidx, h->d_plj, h->d_pqq);
    }
    if (nw) emit_ww_kernel<<<(nw + 127) / 128, 128, 0, st>>>(ea, h->d_pidx, h->d_plj, h->d_pqq);
    TRYC(cudaGetLastError());
    TRYC(cudaStreamSynchronize(st));
    h->n_pairs = total;
    h->n_alch = 0;
    if (n_pairs_out) *n_pairs_out = total;
    cleanup();
#undef TRY
#undef TRYC
    return DYN_OK;
}

namespace {

int nb_forces(dyn_nb_t h, const float* pos_dyn, const float* pos_w_o,
                             const float* pos_w_m, const float* pos_w_h0, const float* pos_w_h1,
                             const float cell_extent[3], uint32_t override_bits, double* f_dyn,
                             double* f_w_o, double* f_w_m, double* f_w_h0, double* f_w_h1,
                             double* virial, double* energy, double lambda, double* dh_dl) {
    DYN_CHECK(h && cell_extent, DYN_ERR_INVALID, "dyn_nb_forces: NULL argument");
    const float* in[5] = {pos_dyn, pos_w_o, pos_w_m, pos_w_h0, pos_w_h1};
    double* outp[5] = {f_dyn, f_w_o, f_w_m, f_w_h0, f_w_h1};
    for (int a = 0; a < 5; ++a)
        if (h->n_of(a) > 0)
            DYN_CHECK(in[a] != nullptr, DYN_ERR_INVALID, "dyn_nb_forces: NULL position array");
    for (int k = 0; k < 3; ++k)
        DYN_CHECK(cell_extent[k] > 0.f, DYN_ERR_INVALID, "dyn_nb_forces: extent must be > 0");
    cudaStream_t st = h->stream;
    // upload_positions (src/gpu_interface.rs:414-455) via pinned staging
    for (int a = 0; a < 5; ++a) {
        const size_t n3 = 3 * (size_t)h->n_of(a);
        if (!n3) continue;
        std::memcpy(h->h_pos[a], in[a], n3 * sizeof(float));
        DYN_CUDA(cudaMemcpyAsync(h->d_pos[a], h->h_pos[a], n3 * sizeof(float), cudaMemcpyHostToDevice, st));
    }
    // zero_forces_and_accums (src/gpu_interface.rs:635-645)
    for (int a = 0; a < 5; ++a)
        DYN_CUDA(cudaMemsetAsync(h->d_f[a], 0, 3 * (size_t)std::max(1u, h->n_of(a)) * sizeof(long long), st));
    const float3 ext = make_float3(cell_extent[0], cell_extent[1], cell_extent[2]);
    // the reference computes the reciprocal extent on the host in float32
    const float3 inv_ext = make_float3(1.0f / ext.x, 1.0f / ext.y, 1.0f / ext.z);
    int blocks = (int)std::min<uint64_t>((h->n_pairs + NB_BLOCK - 1) / NB_BLOCK, NB_MAX_BLOCKS);
    if (blocks < 1) blocks = 1;
    PosPtrs pp;
    ForcePtrs fp;
    for (int a = 0; a < 5; ++a) { pp.p[a] = h->d_pos[a]; fp.f[a] = h->d_f[a]; }
    // the alchemical kernel runs when any installed pair is alchemical, as
    // force_nonbonded_gpu picks it (src/gpu_interface.rs:488-499)
    const AlchSched al = alch_schedule(lambda);
    const bool cpu = h->ljc > 0.f, alch = h->n_alch > 0;
    auto kern = cpu ? (alch ? nb_pair_kernel<true, true> : nb_pair_kernel<true, false>)
                    : (alch ? nb_pair_kernel<false, true> : nb_pair_kernel<false, false>);
    kern<<<blocks, NB_BLOCK, 0, st>>>(pp, fp, h->d_pidx, h->d_plj, h->d_pqq, h->n_pairs, ext, inv_ext,
                                      h->rc, h->alpha, h->ljc, override_bits, al, h->d_partials);
    DYN_CUDA(cudaGetLastError());
    nb_finalize_kernel<<<1, 256, 0, st>>>(h->d_partials, blocks, h->d_scalars);
    DYN_CUDA(cudaGetLastError());
    for (int a = 0; a < 5; ++a) {
        const size_t n3 = 3 * (size_t)h->n_of(a);
        if (!n3) continue;
        DYN_CUDA(cudaMemcpyAsync(h->h_f[a], h->d_f[a], n3 * sizeof(long long), cudaMemcpyDeviceToHost, st));
    }
    DYN_CUDA(cudaMemcpyAsync(h->h_scalars, h->d_scalars, NB_PART * sizeof(double), cudaMemcpyDeviceToHost, st));
    DYN_CUDA(cudaStreamSynchronize(st));
    for (int a = 0; a < 5; ++a) {
        const size_t n3 = 3 * (size_t)h->n_of(a);
        if (!outp[a]) continue;
        for (size_t k = 0; k < n3; ++k) outp[a][k] = (double)h->h_f[a][k] * DYN_FIX_INV;
    }
    if (virial) *virial = h->h_scalars[0];
    if (energy) *energy = h->h_scalars[1];
    if (dh_dl) *dh_dl = alch ? h->h_scalars[2] : 0.0;
    return DYN_OK;
}

}  // namespace

extern "C" int dyn_nb_forces(dyn_nb_t h, const float* pos_dyn, const float* pos_w_o,
                             const float* pos_w_m, const float* pos_w_h0, const float* pos_w_h1,
                             const float cell_extent[3], uint32_t override_bits, double* f_dyn,
                             double* f_w_o, double* f_w_m, double* f_w_h0, double* f_w_h1,
                             double* virial, double* energy) {
    return nb_forces(h, pos_dyn, pos_w_o, pos_w_m, pos_w_h0, pos_w_h1, cell_extent, override_bits,
                     f_dyn, f_w_o, f_w_m, f_w_h0, f_w_h1, virial, energy, 0.0, nullptr);
}

extern "C" int dyn_nb_forces_alch(dyn_nb_t h, const float* pos_dyn, const float* pos_w_o,
                                  const float* pos_w_m, const float* pos_w_h0,
                                  const float* pos_w_h1, const float cell_extent[3],
                                  uint32_t override_bits, double lambda_alch, double* f_dyn,
                                  double* f_w_o, double* f_w_m, double* f_w_h0, double* f_w_h1,
                                  double* virial, double* energy, double* dh_dl) {
    DYN_CHECK(std::isfinite(lambda_alch), DYN_ERR_INVALID, "dyn_nb_forces_alch: lambda is not finite");
    return nb_forces(h, pos_dyn, pos_w_o, pos_w_m, pos_w_h0, pos_w_h1, cell_extent, override_bits,
                     f_dyn, f_w_o, f_w_m, f_w_h0, f_w_h1, virial, energy, lambda_alch, dh_dl);
}

extern "C" int dyn_nb_mark_alch(dyn_nb_t h, uint32_t atom_begin, uint32_t atom_end,
                                uint64_t* n_marked) {
    DYN_CHECK(h, DYN_ERR_INVALID, "dyn_nb_mark_alch: NULL handle");
    DYN_CHECK(atom_begin <= atom_end && atom_end <= h->n_dyn, DYN_ERR_INVALID,
              "dyn_nb_mark_alch: range outside the atoms");
    cudaStream_t st = h->stream;
    unsigned long long* d_cnt = nullptr;
    DYN_CUDA(cudaMalloc(&d_cnt, sizeof(unsigned long long)));
    cudaError_t e = cudaMemsetAsync(d_cnt, 0, sizeof(unsigned long long), st);
    if (e == cudaSuccess && h->n_pairs) {
        const int blocks = (int)std::min<uint64_t>((h->n_pairs + 255) / 256, 148 * 8);
        mark_alch_kernel<<<blocks, 256, 0, st>>>(h->n_pairs, atom_begin, atom_end, h->d_pidx, d_cnt);
        e = cudaGetLastError();
    }
    unsigned long long c = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&c, d_cnt, sizeof(c), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(d_cnt);
    if (e != cudaSuccess) return dyn::cuda_fail(e, "dyn_nb_mark_alch");
    h->n_alch = c;
    if (n_marked) *n_marked = c;
    return DYN_OK;
}
