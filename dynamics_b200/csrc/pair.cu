// Short-range LJ + erfc-screened Coulomb over cluster pairs.
//
// Replaces the reference's one-thread-per-pair kernel over a flat list
// (src/cuda/cuda.cu:185-362) and its CPU twin (src/non_bonded.rs:258-412,
// 950-1057).  The physics is the reference CPU path's: LJ for r <= lj_cutoff
// between sites that carry LJ, erfc(alpha r)/r Coulomb for r < cutoff
// between charged sites, 1-2/1-3 exclusions, no intra-water pairs; 1-4 pairs
// are excluded here and evaluated (scaled) by k_pair14.
//
// Work decomposition.  Water-water (full list, no atomics): one CTA per
// 32-water i-group, j sites staged in shared memory, LPW lanes per i-water
// over its compact molecule list (k_pair_ww_tile).  Atom-water and atom-atom
// (half lists: every pair once): one warp per work item (an 8-body
// i-cluster and up to ch_mix entries of its list); lane = (ii, jq) with
// ii = lane & 7 and jq = lane >> 3 evaluates i-body ii against j-atoms jq and
// jq + 4 of every j-cluster in the item.  Water pairs are
// handled as molecule pairs: one min-image shift from the O-O vector serves
// all site pairs, valid because the cutoff plus twice the O-H reach is below
// half the box.  i-forces stay in registers over the whole list, are reduced
// over the lanes sharing an i-body with shuffles and written once as int64
// fixed point; the water-water kernel stores (first writer), the others add,
// and j-side forces go out as integer atomics after a reduce-scatter over
// the lanes of a j-body.  Integer sums do not depend on order, so the
// result is deterministic.
#include <algorithm>

#include "engine.cuh"

namespace {

constexpr int PT = 128;  // threads per block (4 warps)

// e_lj, e_c accumulate per-pair energies in float64 (energy steps only);
// w sums the virial of one list entry (a molecule pair, or an i-body
// against a j-cluster's atoms) in float32, and wd the entries' sums in
// float64, so no long float32 chain feeds the pressure
struct Acc3 {
    double e_lj, e_c;
    float w;
    double wd;
    __device__ __forceinline__ void flush_w() { wd += (double)w; w = 0.f; }
};

// erfc-screened Coulomb between site pi and site pj shifted by sh
// (d = pi - (pj - sh)), branch-free: force q q (r^-3 + g(r^2)) d with
// g(z) = 2 d/dz [erf(alpha sqrt z) / sqrt z] from the host-fitted polynomial
// in t = 2 r^2 / rc^2 - 1 (no square root needed for the argument); zero for
// r >= rc (src/cuda/cuda.cu:160-164).  On energy steps the energy
// qqe erfc(alpha r) / r is added in float64.
template <bool ENERGY>
__device__ __forceinline__ void coul(float3 pi, float3 pj, float3 sh, float qq, double qqe, const SysView& v,
                                     float3& f, Acc3& a) {
    const float3 d = pi - (pj - sh);
    const float r2 = dot3(d, d);
    const float rinv = rsqrtf(r2);
    const float t = fmaf(r2, v.two_over_rc2, -1.0f);
    float g = v.poly_g[NPOLY_G - 1];
#pragma unroll
    for (int k = NPOLY_G - 2; k >= 0; --k) g = fmaf(g, t, v.poly_g[k]);
    float fs = qq * fmaf(rinv * rinv, rinv, g);
    fs = r2 < v.rc2 ? fs : 0.0f;
    f.x = fmaf(fs, d.x, f.x); f.y = fmaf(fs, d.y, f.y); f.z = fmaf(fs, d.z, f.z);
    a.w = fmaf(fs, r2, a.w);
    if (ENERGY && r2 < v.rc2) {
        // erfc(alpha r) / r in float32 from the force's r^2 and 1/r, scaled by
        // the float64 charge product and summed in float64: per-pair errors
        // of a few ulp with no common sign
        const float re = r2 * rinv;
        a.e_c += qqe * (double)(erfcf(v.alpha * re) * rinv);
    }
}

// 12-6 LJ (force_e_lj, src/forces.rs:10-21) between pi and pj shifted by sh,
// branch-free, r <= lj_cutoff; energy summed in float64.
template <bool ENERGY>
__device__ __forceinline__ void lj(float3 pi, float3 pj, float3 sh, float sig2, float eps, float ljc2,
                                   float scale, float3& f, Acc3& a) {
    const float3 d = pi - (pj - sh);
    const float r2 = dot3(d, d);
    const bool in = r2 <= ljc2;
    const float ir2 = __frcp_rn(in ? r2 : 1.0f);
    const float sr2 = sig2 * ir2;
    const float sr6 = sr2 * sr2 * sr2;
    float fs = scale * 24.0f * eps * fmaf(2.f, sr6 * sr6, -sr6) * ir2;
    fs = in ? fs : 0.0f;
    f.x = fmaf(fs, d.x, f.x); f.y = fmaf(fs, d.y, f.y); f.z = fmaf(fs, d.z, f.z);
    a.w = fmaf(fs, r2, a.w);
    if (ENERGY && in) {
        const double s6 = (double)sr6;
        a.e_lj += 4.0 * (double)scale * (double)eps * (s6 * s6 - s6);
    }
}

// Soft-core LJ of a pair between the alchemical molecule and the rest
// (Beutler et al., Chem. Phys. Lett. 222, 529 (1994), as
// alchemical_lj_soft_core_decouple, src/non_bonded.rs:883-941, with the
// reference's sc-alpha 0.5, power 1 and soft-core sigma >= 3 A,
// src/alchemical.rs:55-65): V = (1 - l) V_LJ(r_sc) with
// r_sc^6 = r^6 + 0.5 s^6 l, s = max(sigma, 3); force (1 - l) F_LJ(r_sc)
// (r / r_sc)^5; dV/dl = -V_LJ(r_sc) - (1 - l) F_LJ(r_sc) 0.5 s^6 / (6 r_sc^5),
// times dl/dlambda of the schedule (dlam) into dh.
template <bool ENERGY>
__device__ __forceinline__ void lj_soft(float3 pi, float3 pj, float3 sh, float sig, float eps, float ljc2,
                                        float lam, float dlam, float3& f, Acc3& a, double& dh) {
    const float3 d = pi - (pj - sh);
    const float r2 = dot3(d, d);
    if (!(r2 <= ljc2) || !(r2 > 0.f) || eps == 0.f) return;
    const float ss = fmaxf(sig, 3.0f), ss2 = ss * ss;
    const float ss6 = ss2 * ss2 * ss2;
    const float rsc6 = fmaf(0.5f * ss6, lam, r2 * r2 * r2);
    const float rsc = sqrtf(cbrtf(rsc6));
    const float inv_rsc = 1.0f / rsc;
    const float sr = sig * inv_rsc, sr2 = sr * sr;
    const float sr6 = sr2 * sr2 * sr2, sr12 = sr6 * sr6;
    const float hf = 24.0f * eps * fmaf(2.0f, sr12, -sr6) * inv_rsc;
    const float he = 4.0f * eps * (sr12 - sr6);
    const float scale = 1.0f - lam;
    const float r = sqrtf(r2);
    const float q = r * inv_rsc, q2 = q * q;
    const float fs = hf * scale * (q2 * q2 * q) / r;
    f.x = fmaf(fs, d.x, f.x); f.y = fmaf(fs, d.y, f.y); f.z = fmaf(fs, d.z, f.z);
    a.w = fmaf(fs, r2, a.w);
    if (ENERGY) {
        const double rsc5 = (double)rsc6 / (double)rsc;
        a.e_lj += (double)scale * (double)he;
        dh += (double)dlam * (-(double)he - (double)scale * (double)hf * (0.5 * (double)ss6) / (6.0 * rsc5));
    }
}

__device__ __forceinline__ float3 shift_of(float3 d, const BoxDev& b) {
    return f3(-rintf(d.x * b.inv_ext[0]) * b.ext[0], -rintf(d.y * b.inv_ext[1]) * b.ext[1],
              -rintf(d.z * b.inv_ext[2]) * b.ext[2]);
}

__device__ __forceinline__ float red4(float x) {
    x += __shfl_xor_sync(0xffffffffu, x, 8);
    x += __shfl_xor_sync(0xffffffffu, x, 16);
    return x;
}

__device__ __forceinline__ void add_fix3(long long* p, float3 f) {
    fix_atomic_add(p + 0, fix_from_float(f.x));
    fix_atomic_add(p + 1, fix_from_float(f.y));
    fix_atomic_add(p + 2, fix_from_float(f.z));
}

template <bool ENERGY>
__device__ __forceinline__ void write_partials(const SysView& v, Blk bk, int region, double el,
                                               double ec, double w, double dh = 0.0) {
    double x[4] = {el, ec, w, dh};
    block_sum_d<4>(x);
    if (threadIdx.x == 0) {
        double* p = v.partials + ((size_t)region * v.max_blocks + bk.idx) * 4;
        p[0] = x[0]; p[1] = x[1]; p[2] = x[2]; p[3] = x[3];
    }
}

// ---------------------------------------------------------------------------
// Staging for the water-water kernel (k_pair_ww_tile, below): a group's
// union of j-waters, stored as runs of consecutive slots, is copied global
// -> shared with one cp.async.bulk per run, completing on an mbarrier, with
// bounded waits; the kernel then reads the j sites from shared memory
// (4 x 16-byte loads per molecule pair).
// ---------------------------------------------------------------------------
constexpr int WT = GRPW * LPW;  // threads per CTA
constexpr uint32_t WAIT_LIMIT = 1u << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait: gives up after WAIT_LIMIT polls and reports it
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, unsigned int* timeout_flag) {
    for (uint32_t it = 0; it < WAIT_LIMIT; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    atomicExch(timeout_flag, 1u);
    return false;
}

// Issues the bulk copies that bring union entries [lo, hi) of group g (from
// its runs of consecutive slots) into buf; one lane per run.  Called by one
// whole warp; lane 0 arms the barrier with the byte count.
__device__ __forceinline__ uint32_t stage_chunk(const SysView& v, uint32_t g, uint32_t lo, uint32_t hi,
                                                float4* buf, uint64_t* bar, int lane, uint32_t* uslot = nullptr) {
    const uint32_t nloc = v.grp_nloc[g], nrun = v.grp_nrun[g];
    const uint2* runs = v.grp_run + (size_t)g * v.cap_run;
    if (lane == 0) mbar_expect_tx(bar, (hi - lo) * (uint32_t)(4 * sizeof(float4)));
    __syncwarp();
    for (uint32_t t = lane; t < nrun; t += 32) {
        const uint2 r = runs[t];
        const uint32_t end = t + 1 < nrun ? runs[t + 1].y : nloc;
        const uint32_t a = max(r.y, lo), e = min(end, hi);
        if (a < e) {
            bulk_g2s(buf + (size_t)(a - lo) * 4, v.wpos + (size_t)(r.x + (a - r.y)) * 4,
                     (e - a) * (uint32_t)(4 * sizeof(float4)), bar);
            if (uslot)
                for (uint32_t u = a; u < e; ++u) uslot[u - lo] = r.x + (u - r.y);
        }
    }
    return hi - lo;
}

// Screened Coulomb of one site pair of a molecule pair, both sides: the
// pair force fs d (d = pi - pj) is added to the i-site sum fi and to the
// j-site sum gj (the j site receives -gj).
template <bool ENERGY>
__device__ __forceinline__ void coul2(float3 pi, float3 pj, float qq, double qqe, const SysView& v, float3& fi,
                                      float3& gj, Acc3& a) {
    const float3 d = pi - pj;
    const float r2 = dot3(d, d);
    const float rinv = rsqrtf(r2);
    const float t = fmaf(r2, v.two_over_rc2, -1.0f);
    float g = v.poly_g[NPOLY_G - 1];
#pragma unroll
    for (int k = NPOLY_G - 2; k >= 0; --k) g = fmaf(g, t, v.poly_g[k]);
    float fs = qq * fmaf(rinv * rinv, rinv, g);
    fs = r2 < v.rc2 ? fs : 0.0f;
    fi.x = fmaf(fs, d.x, fi.x); fi.y = fmaf(fs, d.y, fi.y); fi.z = fmaf(fs, d.z, fi.z);
    gj.x = fmaf(fs, d.x, gj.x); gj.y = fmaf(fs, d.y, gj.y); gj.z = fmaf(fs, d.z, gj.z);
    a.w = fmaf(fs, r2, a.w);
    if (ENERGY && r2 < v.rc2) {
        const float re = r2 * rinv;
        a.e_c += qqe * (double)(erfcf(v.alpha * re) * rinv);
    }
}

// j-side forces of union water u are added to the CTA's int32 sums; a
// molecule pair with a component too large for them (|f| >= JFIX_MAX: 32
// such contributions stay below 2^15 kcal/mol/A, the int32 range at
// 2^-16) goes to the slot's int64 overflow sums instead.  Which path a pair
// takes depends only on its values, and both are integer sums, so the
// result stays deterministic.
constexpr float JFIX_SCALE = (float)(1 << WW_JFIX_SHIFT);
constexpr float JFIX_MAX = 1000.0f;

__device__ __noinline__ void jforce_big(const SysView& v, uint32_t g, uint32_t u, int c, float f) {
    const uint32_t slot = v.grp_uslot[(size_t)g * v.cap_union + u];
    fix_atomic_add(v.wforce + (size_t)slot * 12 + c, fix_from_float(f));
}

// The 12 j-side components of one molecule pair (the forces on the j
// water's O, H0, H1, M); one range check for all of them.
__device__ __forceinline__ void jforce_add12(const SysView& v, int* jacc, uint32_t cs, uint32_t g, uint32_t u,
                                             uint32_t ul, const float (&f)[12]) {
    float m = 0.f;
#pragma unroll
    for (int c = 0; c < 12; ++c) m = fmaxf(m, fabsf(f[c]));
    if (m < JFIX_MAX) {
#pragma unroll
        for (int c = 0; c < 12; ++c) atomicAdd(jacc + (size_t)c * cs + ul, __float2int_rn(f[c] * JFIX_SCALE));
    } else {
        for (int c = 0; c < 12; ++c) jforce_big(v, g, u, c, f[c]);
    }
}

// Per-warp partials (the atom pair kernels' warps run independent work
// items: no block barrier at the end); fixed shuffle order, so the sums are
// deterministic.  The region holds blocks x PT/32 entries.
template <bool ENERGY>
__device__ __forceinline__ void write_partials_warp(const SysView& v, Blk bk, int region, double el, double ec,
                                                    double w, double dh) {
    el = warp_sum_d(el); ec = warp_sum_d(ec); w = warp_sum_d(w); dh = warp_sum_d(dh);
    if ((threadIdx.x & 31) == 0) {
        const size_t e = (size_t)bk.idx * (blockDim.x >> 5) + (threadIdx.x >> 5);
        double* p = v.partials + ((size_t)region * v.max_blocks + e) * 4;
        p[0] = el; p[1] = ec; p[2] = w; p[3] = dh;
    }
}

// ---------------------------------------------------------------------------
// water(i) - water(j), tile form, half lists.  One CTA per 32-water
// i-group.  The waters the group's lists reach (its union, stored as runs
// of consecutive slots) are copied global -> shared with one cp.async.bulk
// per run, completing on an mbarrier, union_chunk waters at a time (one
// chunk for most groups; sized so that three CTAs fit on an SM, with 80
// registers per thread; the batch form, which reads its SysView from global
// memory, spills at 80 and runs two CTAs per SM instead).  The lists hold
// every water pair once (in the list of the lower slot), so
// their lengths vary several-fold across a group; the chunk's entries of
// all 32 lists are therefore dealt out as one sequence, an equal
// contiguous share per thread, whatever list they come from.  A thread
// keeps the i-water's forces in registers while its share stays in one
// list and adds them to the water forces (int64 reductions) when it moves
// to the next list.  All 10 site pairs of a molecule pair use one
// min-image shift.  The j-side forces are summed per union water in shared
// memory (int32 fixed point, 12 components, component-major with a stride
// of chunk + 1 words, so that both the threads' adds and the flush's reads
// spread over the banks), then added to the union waters' forces with one
// coalesced run of int64 reductions per chunk (the union's slots are noted
// in shared memory while the copies are issued).  The shares depend only on
// the lists and the chunk size, and every sum across threads is an integer
// sum: the forces are the same bits run to run.  The list lengths of a group
// whose union fits one chunk (almost every group) are read while its copies
// are in flight; larger unions find each chunk's entries by binary search.
// A system with fewer groups than the GPU has SMs gives each group ww_split
// CTAs, each staging the union and taking an equal slice of the entries.
// ---------------------------------------------------------------------------
DYN_KERNEL_T2((bool ENERGY), (ENERGY), __launch_bounds__(WT, 3), __launch_bounds__(WT, 2), k_pair_ww_tile, (), ()) {
    extern __shared__ __align__(128) float4 tile[];  // union_chunk waters x 4 float4, then the j sums
    __shared__ __align__(8) uint64_t bar;
    __shared__ float4 ipos[GRPW * 4];   // the group's i-water sites
    __shared__ uint32_t woff[GRPW + 1]; // first share position of each list's chunk entries
    __shared__ uint32_t wbeg[GRPW];     // each list's first entry in the chunk
    __shared__ uint32_t wend[GRPW];     // ... and one past its last
    __shared__ uint32_t wlen[GRPW];     // list lengths
    const int tid = threadIdx.x;
    const uint32_t nwc = v.sc->n_wclus;
    const uint32_t ng = (nwc + GRPW / WCL - 1) / (GRPW / WCL);
    const uint32_t nslots = nwc * WCL;
    const uint32_t chunk = v.union_chunk;
    const uint32_t cs = chunk + 1;  // component stride of the j sums
    int* jacc = reinterpret_cast<int*>(tile + 4 * (size_t)chunk);  // [12][chunk + 1]
    uint32_t* uslot = reinterpret_cast<uint32_t*>(jacc + 12 * (size_t)cs);  // [chunk] union entry -> slot
    const BoxDev b = *v.box;
    const float ljc2 = v.ljc2;
    const float sig2 = OPC_O_SIGMA * OPC_O_SIGMA;
    const float qhh = OPC_Q_H * OPC_Q_H, qhm = OPC_Q_H * OPC_Q_EP, qmm = OPC_Q_EP * OPC_Q_EP;
    const double ehh = (double)OPC_Q_H * (double)OPC_Q_H, ehm = (double)OPC_Q_H * (double)OPC_Q_EP,
                 emm = (double)OPC_Q_EP * (double)OPC_Q_EP;
    if (tid == 0) mbar_init(&bar, 1);
    // the j sums start at zero; each chunk's flush zeroes what it read
    for (uint32_t t = tid; t < 12 * cs; t += WT) jacc[t] = 0;
    __syncthreads();
    uint32_t parity = 0;
    Acc3 a{0.0, 0.0, 0.f, 0.0};
    bool alive = true;
    // inclusive scan of a count over the 32 lanes of a warp
    auto scan32 = [](uint32_t x, int l) {
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (l >= o) x += y;
        }
        return x;
    };
    const uint32_t split = v.ww_split;
    for (uint32_t q = bk.idx; q < ng * split && alive; q += bk.cnt) {
        const uint32_t g = q / split, part = q - g * split;
        const uint32_t nloc = v.grp_nloc[g];
        if (tid < GRPW * 4) {
            const uint32_t s = g * GRPW + tid / 4;
            ipos[tid] = s < nslots ? v.wpos[(size_t)4 * g * GRPW + tid] : make_float4(0.f, 0.f, 0.f, 0.f);
        }
        const bool single = nloc <= chunk;
        if (tid >= 32 && tid < 32 + GRPW) {
            const int w = tid - 32;
            const uint32_t s = g * GRPW + w;
            const uint32_t n = s < nslots ? v.winb_n[s] : 0u;
            wlen[w] = n;
            wend[w] = 0u;
            if (single) {
                // one chunk: every entry of every list
                const uint32_t x = scan32(n, w);
                wbeg[w] = 0u;
                woff[w + 1] = x;
                if (w == 0) woff[0] = 0u;
            }
        }
        for (uint32_t lo = 0; lo < nloc; lo += chunk) {
            const uint32_t hi = min(nloc, lo + chunk);
            if (tid < 32) stage_chunk(v, g, lo, hi, tile, &bar, tid, uslot);
            __syncthreads();  // the lengths and wend of the previous chunk are visible
            if (!single && tid >= 32 && tid < 32 + GRPW) {
                // the list entries of this chunk: from where the previous
                // chunk stopped to the first union index >= hi (lists ascend)
                const int w = tid - 32;
                const uint16_t* lst = v.winb + (size_t)(g * GRPW + w) * v.cap_nb;
                const uint32_t b0 = wend[w];
                uint32_t l0 = b0, l1 = wlen[w];
                while (l0 < l1) {
                    const uint32_t m = (l0 + l1) >> 1;
                    if ((uint32_t)lst[m] < hi) l0 = m + 1; else l1 = m;
                }
                const uint32_t x = scan32(l0 - b0, w);
                wbeg[w] = b0;
                woff[w + 1] = x;
                if (w == 0) woff[0] = 0u;
                wend[w] = l0;
            }
            const bool ok = mbar_wait(&bar, parity, &v.sc->timeout);
            if (!__syncthreads_and(ok)) {
                // give the copies in flight one more bounded chance, then stop
                if (!ok) mbar_wait(&bar, parity, &v.sc->timeout);
                alive = false;
                break;
            }
            parity ^= 1u;
            // this CTA's slice of the chunk's entries, and this thread's
            // share [e0, e1) of the slice
            const uint32_t total = woff[GRPW];
            const uint32_t s0 = (uint32_t)(((uint64_t)part * total) / split);
            const uint32_t slen = (uint32_t)(((uint64_t)(part + 1) * total) / split) - s0;
            const uint32_t e0 = s0 + (uint32_t)(((uint64_t)tid * slen) / WT);
            const uint32_t e1 = s0 + (uint32_t)(((uint64_t)(tid + 1) * slen) / WT);
            int w = 0;
            while (w < GRPW - 1 && woff[w + 1] <= e0) ++w;
            float3 iO = f3(0, 0, 0), iH0 = iO, iH1 = iO, iM = iO;
            float3 fO = iO, fH0 = iO, fH1 = iO, fM = iO;
            const uint16_t* lst = v.winb;
            uint32_t wstop = 0;  // share position where list w ends
            auto enter = [&](int wn) {
                w = wn;
                iO = xyz(ipos[4 * w + 0]); iH0 = xyz(ipos[4 * w + 1]);
                iH1 = xyz(ipos[4 * w + 2]); iM = xyz(ipos[4 * w + 3]);
                // lst[e] is the entry at list position wbeg[w] + (e - woff[w])
                lst = v.winb + ((size_t)(g * GRPW + w) * v.cap_nb + wbeg[w]) - woff[w];
                wstop = woff[w + 1];
            };
            auto leave = [&]() {
                long long* p = v.wforce + (size_t)(g * GRPW + w) * 12;
                add_fix3(p + 0, fO); add_fix3(p + 3, fH0); add_fix3(p + 6, fH1); add_fix3(p + 9, fM);
                fO = f3(0, 0, 0); fH0 = fO; fH1 = fO; fM = fO;
            };
            if (e0 < e1) enter(w);
            // the next entry's index is loaded one iteration ahead, so the
            // global-memory latency of the list overlaps the arithmetic
            uint32_t idx_next = e0 < e1 ? (uint32_t)lst[e0] : 0u;
            for (uint32_t e = e0; e < e1; ++e) {
                if (e >= wstop) {
                    leave();
                    int wn = w + 1;
                    while (woff[wn + 1] <= e) ++wn;
                    enter(wn);
                    idx_next = (uint32_t)lst[e];
                }
                const uint32_t idx = idx_next;
                if (e + 1 < e1 && e + 1 < wstop) idx_next = (uint32_t)lst[e + 1];
                const float4* jw = tile + 4 * (idx - lo);
                const float3 jO = xyz(jw[0]);
                const float3 sh = shift_of(iO - jO, b);
                // the j sites moved by the shift once, then zero shift
                const float3 z0 = f3(0.f, 0.f, 0.f);
                const float3 sO = jO - sh, sH0 = xyz(jw[1]) - sh, sH1 = xyz(jw[2]) - sh, sM = xyz(jw[3]) - sh;
                float3 gO = z0, gH0 = z0, gH1 = z0, gM = z0;
                {
                    float3 t = z0;
                    lj<ENERGY>(iO, sO, z0, sig2, OPC_O_EPS, ljc2, 1.0f, t, a);
                    fO = fO + t;
                    gO = t;
                }
                coul2<ENERGY>(iH0, sH0, qhh, ehh, v, fH0, gH0, a);
                coul2<ENERGY>(iH0, sH1, qhh, ehh, v, fH0, gH1, a);
                coul2<ENERGY>(iH0, sM, qhm, ehm, v, fH0, gM, a);
                coul2<ENERGY>(iH1, sH0, qhh, ehh, v, fH1, gH0, a);
                coul2<ENERGY>(iH1, sH1, qhh, ehh, v, fH1, gH1, a);
                coul2<ENERGY>(iH1, sM, qhm, ehm, v, fH1, gM, a);
                coul2<ENERGY>(iM, sH0, qhm, ehm, v, fM, gH0, a);
                coul2<ENERGY>(iM, sH1, qhm, ehm, v, fM, gH1, a);
                coul2<ENERGY>(iM, sM, qmm, emm, v, fM, gM, a);
                a.flush_w();
                // the j waters receive the opposite forces (sites O, H0, H1, M)
                const float jf[12] = {-gO.x, -gO.y, -gO.z, -gH0.x, -gH0.y, -gH0.z,
                                      -gH1.x, -gH1.y, -gH1.z, -gM.x, -gM.y, -gM.z};
                jforce_add12(v, jacc, cs, g, idx, idx - lo, jf);
            }
            if (e0 < e1) leave();
            __syncthreads();  // every j sum of the chunk is in
            // the chunk's sums -> the union waters' forces (2^-16 -> 2^-32
            // fixed point); consecutive union entries of a run are
            // consecutive slots, so the reductions are coalesced
            for (uint32_t t = tid; t < 12 * (hi - lo); t += WT) {
                const uint32_t u = t / 12, c = t - 12 * u;
                const int val = jacc[c * cs + u];
                if (val != 0) {
                    jacc[c * cs + u] = 0;
                    fix_atomic_add(v.wforce + 12 * (size_t)uslot[u] + c,
                                   (long long)val * (1ll << (32 - WW_JFIX_SHIFT)));
                }
            }
            __syncthreads();  // the tile and the sums are refilled by the next chunk or group
        }
    }
    write_partials<ENERGY>(v, bk, REG_WW, ENERGY ? a.e_lj : 0.0, ENERGY ? a.e_c : 0.0, a.wd);
}


// Reduce-scatter over the 8 lanes that share jq (lane bits 0-2): N values
// per lane in, N/8 out; lane ii ends with the sums of values
// [ii N/8, (ii + 1) N/8).  The pairing order is fixed, so the result is
// deterministic.
template <int N>
__device__ __forceinline__ void reduce_scatter8(float (&x)[N], int ii) {
#pragma unroll
    for (int m = 4, h = N / 2; m >= 1; m >>= 1, h >>= 1) {
        const bool up = (ii & m) != 0;
#pragma unroll
        for (int k = 0; k < h; ++k) {
            const float keep = up ? x[k + h] : x[k];
            const float send = up ? x[k] : x[k + h];
            x[k] = keep + __shfl_xor_sync(0xffffffffu, send, m);
        }
    }
}

__device__ __forceinline__ void add_fix(long long* p, float f) {
    if (f != 0.0f) fix_atomic_add(p, fix_from_float(f));
}

// j-atom data of one list entry for lane group jq: atoms jq and jq + 4 of
// cluster cj (position + charge, sigma/eps, home index or INVALID_ID)
struct JAtoms { float4 p0, p1; float2 l0, l1; uint32_t a0, a1; };
__device__ __forceinline__ JAtoms load_jatoms(const SysView& v, uint32_t cj, int jq) {
    const uint32_t s = cj * ACL + jq;
    return JAtoms{v.spos[s], v.spos[s + 4], v.slj[s], v.slj[s + 4], v.sidx[s], v.sidx[s + 4]};
}

// ---------------------------------------------------------------------------
// water(i) - atom(j), each pair once.  One warp per work item (a water
// i-cluster and ch_mix entries of its atom-cluster list); the list entries
// are read once per item (one per lane) and the next entry's j-atoms are
// loaded while the current one is evaluated.  The water forces stay in
// registers over the item; the j-atom forces (the opposite of the pair
// forces) are reduce-scattered over the 8 water lanes of a j-group and added
// with integer atomics (24 per entry).
// ---------------------------------------------------------------------------
DYN_KERNEL_T((bool ENERGY, bool ALCH), (ENERGY, ALCH), __launch_bounds__(PT, 4), k_pair_ws, (), ()) {
    const int lane = threadIdx.x & 31;
    const int ii = lane & 7, jq = lane >> 3;
    const uint32_t nwarps = (bk.cnt * blockDim.x) >> 5;
    const uint32_t nit = v.sc->n_ws_items;
    const uint32_t first_single = v.sc->a_sparse_base / ACL;  // first single-atom cluster
    const BoxDev b = *v.box;
    const float ljc2 = v.ljc2;
    double el = 0.0, ec = 0.0, ew = 0.0, dh = 0.0;
    for (uint32_t it = ((bk.idx * blockDim.x + threadIdx.x) >> 5); it < nit; it += nwarps) {
        const uint2 item = v.ws_item[it];
        const uint32_t ci = item.x, k0 = item.y;
        const uint32_t n = min(v.ws_n[ci], k0 + v.ch_mix) - k0;
        const uint32_t si = ci * WCL + ii;
        const bool vi = v.wid[si] != INVALID_ID;
        const float3 iO = xyz(v.wpos[4 * si + 0]), iH0 = xyz(v.wpos[4 * si + 1]);
        const float3 iH1 = xyz(v.wpos[4 * si + 2]), iM = xyz(v.wpos[4 * si + 3]);
        float3 fO = f3(0, 0, 0), fH0 = fO, fH1 = fO, fM = fO;
        Acc3 a{0.0, 0.0, 0.f, 0.0};
        const uint32_t my_j = (uint32_t)lane < n ? v.ws_j[(size_t)ci * v.cap_ws + k0 + lane] : 0u;
        // Single-atom clusters (ions) come last in every list.  Four of them
        // are taken per iteration, one per lane group jq (its atom in the
        // h = 0 slot), instead of one cluster with seven empty slots.
        auto load_at = [&](uint32_t k) -> JAtoms {
            const uint32_t c0 = __shfl_sync(0xffffffffu, my_j, k);
            const uint32_t kk = k + (uint32_t)jq;
            const uint32_t cq = __shfl_sync(0xffffffffu, my_j, kk < n ? kk : k);
            if (c0 < first_single) return load_jatoms(v, c0, jq);
            const uint32_t sq = cq * ACL;
            return JAtoms{v.spos[sq], make_float4(0.f, 0.f, 0.f, 0.f), v.slj[sq], make_float2(0.f, 0.f),
                          kk < n ? v.sidx[sq] : INVALID_ID, INVALID_ID};
        };
        auto advance = [&](uint32_t k) -> uint32_t {
            return __shfl_sync(0xffffffffu, my_j, k) < first_single ? 1u : 4u;
        };
        JAtoms nx = load_at(0);
        for (uint32_t k = 0; k < n;) {
            const JAtoms cur = nx;
            k += advance(k);
            if (k < n) nx = load_at(k);
            // the cluster boxes met within r_ws; skip the entry when no lane's
            // water O lies within cutoff + O-H reach of its atoms
            {
                const float r2 = v.r_ws_skip2;
                bool near = false;
                if (vi && cur.a0 != INVALID_ID) {
                    const float3 d = min_image_rint(iO - xyz(cur.p0), b);
                    near = dot3(d, d) < r2;
                }
                if (vi && cur.a1 != INVALID_ID) {
                    const float3 d = min_image_rint(iO - xyz(cur.p1), b);
                    near = near || dot3(d, d) < r2;
                }
                if (!__any_sync(0xffffffffu, near)) continue;
            }
            float jf[8];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const float4 pj = h ? cur.p1 : cur.p0;
                const float2 lj_j = h ? cur.l1 : cur.l0;
                const uint32_t aj = h ? cur.a1 : cur.a0;
                float3 fo = f3(0, 0, 0), f0 = fo, f1 = fo, fm = fo;
                if (vi && aj != INVALID_ID) {
                    const float3 jp = xyz(pj);
                    // the atom moved by the shift once, then zero shift
                    const float3 js = jp - shift_of(iO - jp, b), z0 = f3(0.f, 0.f, 0.f);
                    const float sg = 0.5f * (OPC_O_SIGMA + lj_j.x);
                    const float ep = sqrtf(OPC_O_EPS * lj_j.y);
                    const double qe = (double)pj.w;
                    if (ALCH && aj >= v.alch_lo && aj < v.alch_hi) {
                        // a water and an atom of the alchemical molecule
                        lj_soft<ENERGY>(iO, js, z0, sg, ep, ljc2, v.alch_ll, v.alch_dll, fo, a, dh);
                        Acc3 t{0.0, 0.0, 0.f, 0.0};
                        coul<ENERGY>(iH0, js, z0, OPC_Q_H * pj.w, (double)OPC_Q_H * qe, v, f0, t);
                        coul<ENERGY>(iH1, js, z0, OPC_Q_H * pj.w, (double)OPC_Q_H * qe, v, f1, t);
                        coul<ENERGY>(iM, js, z0, OPC_Q_EP * pj.w, (double)OPC_Q_EP * qe, v, fm, t);
                        const float cs = v.alch_cs;
                        f0 = f0 * cs; f1 = f1 * cs; fm = fm * cs;
                        a.w = fmaf(cs, t.w, a.w);
                        if (ENERGY) { a.e_c += (double)cs * t.e_c; dh += (double)v.alch_dcs * t.e_c; }
                    } else {
                        lj<ENERGY>(iO, js, z0, sg * sg, ep, ljc2, 1.0f, fo, a);
                        coul<ENERGY>(iH0, js, z0, OPC_Q_H * pj.w, (double)OPC_Q_H * qe, v, f0, a);
                        coul<ENERGY>(iH1, js, z0, OPC_Q_H * pj.w, (double)OPC_Q_H * qe, v, f1, a);
                        coul<ENERGY>(iM, js, z0, OPC_Q_EP * pj.w, (double)OPC_Q_EP * qe, v, fm, a);
                    }
                }
                fO = fO + fo; fH0 = fH0 + f0; fH1 = fH1 + f1; fM = fM + fm;
                const float3 t = (fo + f0) + (f1 + fm);
                jf[3 * h + 0] = -t.x; jf[3 * h + 1] = -t.y; jf[3 * h + 2] = -t.z;
            }
            jf[6] = 0.f; jf[7] = 0.f;
            a.flush_w();
            // lane ii < 6 now holds component ii % 3 of the group's j-atom a0 (ii < 3) or a1
            reduce_scatter8(jf, ii);
            if (ii < 6) {
                const uint32_t aj = ii < 3 ? cur.a0 : cur.a1;
                if (aj != INVALID_ID) add_fix(v.aforce + 3 * (size_t)aj + ii % 3, jf[0]);
            }
        }
        fO = f3(red4(fO.x), red4(fO.y), red4(fO.z));
        fH0 = f3(red4(fH0.x), red4(fH0.y), red4(fH0.z));
        fH1 = f3(red4(fH1.x), red4(fH1.y), red4(fH1.z));
        fM = f3(red4(fM.x), red4(fM.y), red4(fM.z));
        if (jq == 0 && vi) {
            long long* p = v.wforce + (size_t)si * 12;
            add_fix3(p + 0, fO); add_fix3(p + 3, fH0); add_fix3(p + 6, fH1); add_fix3(p + 9, fM);
        }
        if (ENERGY) { el += a.e_lj; ec += a.e_c; }
        a.flush_w();
        ew += a.wd;
    }
    write_partials_warp<ENERGY>(v, bk, REG_WS, el, ec, ew, dh);
}

// ---------------------------------------------------------------------------
// atom(i) - atom(j), each pair once (cluster pairs with cj >= ci; the
// interaction mask from the list build holds jj > ii on the diagonal and
// drops exclusions); work items, prefetch and j-side atomics as above.
// ---------------------------------------------------------------------------
DYN_KERNEL_T((bool ENERGY, bool ALCH), (ENERGY, ALCH), __launch_bounds__(PT), k_pair_ss, (), ()) {
    const int lane = threadIdx.x & 31;
    const int ii = lane & 7, jq = lane >> 3;
    const uint32_t nwarps = (bk.cnt * blockDim.x) >> 5;
    const uint32_t nit = v.sc->n_ss_items;
    const BoxDev b = *v.box;
    const float ljc2 = v.ljc2;
    double el = 0.0, ec = 0.0, ew = 0.0, dh = 0.0;
    for (uint32_t it = ((bk.idx * blockDim.x + threadIdx.x) >> 5); it < nit; it += nwarps) {
        const uint2 item = v.ss_item[it];
        const uint32_t ci = item.x, k0 = item.y;
        const uint32_t n = min(v.ss_n[ci], k0 + v.ch_mix) - k0;
        const uint32_t si = ci * ACL + ii;
        const uint32_t ai = v.sidx[si];
        const float4 pi = v.spos[si];
        const float2 lji = v.slj[si];
        float3 f = f3(0, 0, 0);
        Acc3 a{0.0, 0.0, 0.f, 0.0};
        const size_t row = (size_t)ci * v.cap_ss + k0;
        const uint32_t my_j = (uint32_t)lane < n ? v.ss_j[row + lane] : 0u;
        const unsigned long long my_m = (uint32_t)lane < n ? v.ss_mask[row + lane] : 0ull;
        JAtoms nx = load_jatoms(v, __shfl_sync(0xffffffffu, my_j, 0), jq);
        for (uint32_t k = 0; k < n; ++k) {
            const JAtoms cur = nx;
            const unsigned long long m = __shfl_sync(0xffffffffu, my_m, k);
            if (k + 1 < n) nx = load_jatoms(v, __shfl_sync(0xffffffffu, my_j, k + 1), jq);
            float jf[8];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int jj = jq + 4 * h;
                const float4 pj = h ? cur.p1 : cur.p0;
                const float2 ljj = h ? cur.l1 : cur.l0;
                float3 fp = f3(0, 0, 0);
                if ((m >> (ii * ACL + jj)) & 1ull) {
                    const float3 s = shift_of(xyz(pi) - xyz(pj), b);
                    const float sg = 0.5f * (lji.x + ljj.x);
                    const uint32_t aj = h ? cur.a1 : cur.a0;
                    if (ALCH && ((ai >= v.alch_lo && ai < v.alch_hi) != (aj >= v.alch_lo && aj < v.alch_hi))) {
                        // exactly one atom of the pair in the alchemical molecule
                        lj_soft<ENERGY>(xyz(pi), xyz(pj), s, sg, sqrtf(lji.y * ljj.y), ljc2, v.alch_ll, v.alch_dll,
                                        fp, a, dh);
                        Acc3 t{0.0, 0.0, 0.f, 0.0};
                        float3 fc = f3(0.f, 0.f, 0.f);
                        coul<ENERGY>(xyz(pi), xyz(pj), s, pi.w * pj.w, (double)pi.w * (double)pj.w, v, fc, t);
                        const float cs = v.alch_cs;
                        fp = fp + fc * cs;
                        a.w = fmaf(cs, t.w, a.w);
                        if (ENERGY) { a.e_c += (double)cs * t.e_c; dh += (double)v.alch_dcs * t.e_c; }
                    } else {
                        lj<ENERGY>(xyz(pi), xyz(pj), s, sg * sg, sqrtf(lji.y * ljj.y), ljc2, 1.0f, fp, a);
                        coul<ENERGY>(xyz(pi), xyz(pj), s, pi.w * pj.w, (double)pi.w * (double)pj.w, v, fp, a);
                    }
                }
                f = f + fp;
                jf[3 * h + 0] = -fp.x; jf[3 * h + 1] = -fp.y; jf[3 * h + 2] = -fp.z;
            }
            jf[6] = 0.f; jf[7] = 0.f;
            a.flush_w();
            // lane ii < 6 now holds component ii % 3 of atom jq + 4 (ii / 3)
            reduce_scatter8(jf, ii);
            if (ii < 6) {
                const uint32_t aj = ii < 3 ? cur.a0 : cur.a1;
                if (aj != INVALID_ID) add_fix(v.aforce + 3 * (size_t)aj + ii % 3, jf[0]);
            }
        }
        f = f3(red4(f.x), red4(f.y), red4(f.z));
        if (jq == 0 && ai != INVALID_ID) add_fix3(v.aforce + 3 * (size_t)ai, f);
        if (ENERGY) { el += a.e_lj; ec += a.e_c; }
        a.flush_w();
        ew += a.wd;
    }
    write_partials_warp<ENERGY>(v, bk, REG_SS, el, ec, ew, dh);
}

// ---------------------------------------------------------------------------
// 1-4 pairs: LJ x0.5, Coulomb x1/1.2 (src/non_bonded.rs:55-56,1014-1042)
// ---------------------------------------------------------------------------
DYN_KERNEL_T((bool ENERGY), (ENERGY), , k_pair14, (), ()) {
    const BoxDev b = *v.box;
    double e_acc = 0.0, w_acc = 0.0;
    for (uint32_t k = bk.idx * blockDim.x + threadIdx.x; k < v.n14; k += bk.cnt * blockDim.x) {
        const uint2 p = v.p14[k];
        const float4 par = v.p14_par[k];  // sigma, eps, qq
        const float4 pa = v.apos[p.x], pb = v.apos[p.y];
        const float3 sh = shift_of(xyz(pa) - xyz(pb), b);
        float3 f = f3(0, 0, 0);
        Acc3 a{0.0, 0.0, 0.f, 0.0};
        lj<ENERGY>(xyz(pa), xyz(pb), sh, par.x * par.x, par.y, v.ljc2, 0.5f, f, a);
        float3 fc = f3(0, 0, 0);
        Acc3 ac{0.0, 0.0, 0.f, 0.0};
        coul<ENERGY>(xyz(pa), xyz(pb), sh, par.z, (double)pa.w * (double)pb.w, v, fc, ac);
        const float s = 0.833333333f;
        f = f + fc * s;
        add_fix3(v.aforce + 3 * (size_t)p.x, f);
        add_fix3(v.aforce + 3 * (size_t)p.y, f3(-f.x, -f.y, -f.z));
        if (ENERGY) e_acc += a.e_lj + ac.e_c / 1.2;
        w_acc += (double)a.w + (double)ac.w * s;
    }
    write_partials<ENERGY>(v, bk, REG_14, e_acc, 0.0, w_acc);
}

// Blocks of the atom pair kernels: one per 4 work items, at most one
// resident wave (4 blocks per SM; the kernels loop over the items), which
// also bounds the block partials the step finalisation sums.
inline int pblocks(const SysView& v, uint64_t warps) {
    uint64_t bl = (warps * 32 + PT - 1) / PT;
    if (bl < 1) bl = 1;
    // at most max_blocks / 4: the kernels write one partial per warp
    const uint64_t cap = std::min<uint64_t>(v.max_blocks / (PT / 32), 148u * 4u);
    return (int)(bl < cap ? bl : cap);
}

}  // namespace

namespace dyn {

int pair_blocks_ws(const SysView& v) { return pblocks(v, v.ws_item_cap); }

int ww_tile_blocks(const SysView& v) {
    const uint64_t n = (uint64_t)v.ngrp_cap * v.ww_split;
    return (int)(n < v.max_blocks ? n : v.max_blocks);
}

// per union water: 4 float4 positions, 12 int32 j sums (+ the stride pad) and its slot
size_t ww_tile_smem(const SysView& v) {
    return (size_t)v.union_chunk * (4 * sizeof(float4) + 13 * sizeof(int)) + 12 * sizeof(int);
}

// The limit is a property of the kernel, shared by every system in the
// process, so it is raised to the device maximum once rather than set to one
// system's chunk size (which would break systems with larger chunks).
int pair_ww_setup(const SysView& v) {
    int dev = 0, optin = 0;
    DYN_CUDA(cudaGetDevice(&dev));
    DYN_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const void* ks[4] = {(const void*)k_pair_ww_tile<true>, (const void*)k_pair_ww_tile<false>,
                         (const void*)k_pair_ww_tile_batch<true>, (const void*)k_pair_ww_tile_batch<false>};
    for (const void* k : ks) {
        cudaFuncAttributes fa;
        DYN_CUDA(cudaFuncGetAttributes(&fa, k));
        const int lim = optin - (int)fa.sharedSizeBytes;
        DYN_CHECK(ww_tile_smem(v) <= (size_t)lim, DYN_ERR_UNSUPPORTED, "water-water chunk exceeds shared memory");
        DYN_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
    }
    return DYN_OK;
}
int pair_blocks_ss(const SysView& v) { return pblocks(v, v.ss_item_cap); }
int pair14_blocks(const SysView& v) {
    uint64_t bl = (v.n14 + 255) / 256;
    if (bl < 1) bl = 1;
    return (int)(bl < v.max_blocks ? bl : v.max_blocks);
}

void launch_pairs(const Target& t, bool energy) {
    launch_pairs_water(t, energy);
    launch_pairs_atoms(t, energy);
}

// the alchemical variants wherever a system decouples a molecule
inline bool any_alch(const Target& t) {
    return t.any([](const SysView& v) { return v.alch_on != 0u; });
}

void launch_pairs_atoms(const Target& t, bool energy) {
    auto ss = [](const SysView& v) { return v.na ? pair_blocks_ss(v) : 0; };
    const bool al = any_alch(t);
    if (energy && al) t.launch(k_pair_ss<true, true>, k_pair_ss_batch<true, true>, ss, PT, 0);
    else if (energy) t.launch(k_pair_ss<true, false>, k_pair_ss_batch<true, false>, ss, PT, 0);
    else if (al) t.launch(k_pair_ss<false, true>, k_pair_ss_batch<false, true>, ss, PT, 0);
    else t.launch(k_pair_ss<false, false>, k_pair_ss_batch<false, false>, ss, PT, 0);
}

void launch_pairs_ww(const Target& t, bool energy) {
    const size_t sm = t.max_over([](const SysView& v) { return v.nw ? ww_tile_smem(v) : (size_t)0; });
    // water-water short-range energy is part of the potential only with
    // DYN_FLAG_FULL_ENERGY (the reference leaves it out,
    // src/non_bonded.rs:335-342), so other energy steps skip it
    auto eww = [energy](const SysView& v) { return energy && (v.flags & DYN_FLAG_FULL_ENERGY); };
    t.launch(k_pair_ww_tile<true>, k_pair_ww_tile_batch<true>,
             [&](const SysView& v) { return v.nw && eww(v) ? ww_tile_blocks(v) : 0; }, WT, sm);
    t.launch(k_pair_ww_tile<false>, k_pair_ww_tile_batch<false>,
             [&](const SysView& v) { return v.nw && !eww(v) ? ww_tile_blocks(v) : 0; }, WT, sm);
}

void launch_pairs_water(const Target& t, bool energy) {
    launch_pairs_ww(t, energy);
    launch_pairs_ws(t, energy);
}

void launch_pairs_ws(const Target& t, bool energy) {
    auto ws = [](const SysView& v) { return v.nw && v.na ? pair_blocks_ws(v) : 0; };
    const bool al = any_alch(t);
    if (energy && al) t.launch(k_pair_ws<true, true>, k_pair_ws_batch<true, true>, ws, PT, 0);
    else if (energy) t.launch(k_pair_ws<true, false>, k_pair_ws_batch<true, false>, ws, PT, 0);
    else if (al) t.launch(k_pair_ws<false, true>, k_pair_ws_batch<false, true>, ws, PT, 0);
    else t.launch(k_pair_ws<false, false>, k_pair_ws_batch<false, false>, ws, PT, 0);
}

void launch_pair14(const Target& t, bool energy) {
    auto g = [](const SysView& v) { return v.n14 ? pair14_blocks(v) : 0; };
    if (energy) t.launch(k_pair14<true>, k_pair14_batch<true>, g, 256, 0);
    else t.launch(k_pair14<false>, k_pair14_batch<false>, g, 256, 0);
}

}  // namespace dyn
