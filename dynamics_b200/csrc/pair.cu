// Short-range LJ + erfc-screened Coulomb over cluster pairs.
//
// Replaces the reference's one-thread-per-pair kernel over a flat list
// (src/cuda/cuda.cu:185-362) and its CPU twin (src/non_bonded.rs:258-412,
// 950-1057).  The physics is the reference CPU path's: LJ for r <= lj_cutoff
// between sites that carry LJ, erfc(alpha r)/r Coulomb for r < cutoff
// between charged sites, 1-2/1-3 exclusions, no intra-water pairs; 1-4 pairs
// are excluded here and evaluated (scaled) by k_pair14.
//
// Work decomposition (one warp per i-cluster, full lists, no atomics on the
// i side): a warp owns 8 i-waters (or 8 atoms); lane = (ii, jq) with
// ii = lane & 7 and jq = lane >> 3, so each lane evaluates i-body ii against
// j-bodies jq and jq + 4 of every j-cluster in the list.  Water pairs are
// handled as molecule pairs: one min-image shift from the O-O vector serves
// all 10 site pairs (1 LJ + 9 Coulomb), valid because the cutoff plus twice
// the O-H reach is below half the box.  i-forces stay in registers over the
// whole list, are reduced over the 4 lanes sharing ii with two shuffles and
// stored once as int64 fixed point; the water-water and atom-atom kernels
// store (first writers), the mixed kernels add.
#include "engine.cuh"

namespace {

constexpr int PT = 128;  // threads per block (4 warps)

struct Acc3 { float e_lj, e_c, w; };

template <bool ENERGY>
__device__ __forceinline__ void coul(float3 d, float qq, float rc2, float alpha, float c2a,
                                     float3& f, Acc3& a) {
    const float r2 = dot3(d, d);
    if (r2 < rc2) {
        const float rinv = rsqrtf(r2);
        const float r = r2 * rinv;
        const float ar = alpha * r;
        const float ex = __expf(-ar * ar);
        const float ec = erfcf(ar);
        const float fs = qq * fmaf(ec, rinv, c2a * ex) * (rinv * rinv);
        f.x = fmaf(fs, d.x, f.x); f.y = fmaf(fs, d.y, f.y); f.z = fmaf(fs, d.z, f.z);
        a.w = fmaf(fs, r2, a.w);
        if (ENERGY) a.e_c = fmaf(qq * rinv, ec, a.e_c);
    }
}

template <bool ENERGY>
__device__ __forceinline__ void lj(float3 d, float sig2, float eps, float ljc2, float scale,
                                   float3& f, Acc3& a) {
    const float r2 = dot3(d, d);
    if (r2 <= ljc2 && eps != 0.f) {
        const float ir2 = __frcp_rn(r2);
        const float sr2 = sig2 * ir2;
        const float sr6 = sr2 * sr2 * sr2;
        const float fs = scale * 24.0f * eps * fmaf(2.f, sr6 * sr6, -sr6) * ir2;
        f.x = fmaf(fs, d.x, f.x); f.y = fmaf(fs, d.y, f.y); f.z = fmaf(fs, d.z, f.z);
        a.w = fmaf(fs, r2, a.w);
        if (ENERGY) a.e_lj = fmaf(scale * 4.0f * eps, sr6 * sr6 - sr6, a.e_lj);
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

__device__ __forceinline__ void store_fix3(long long* p, float3 f) {
    p[0] = fix_from_float(f.x); p[1] = fix_from_float(f.y); p[2] = fix_from_float(f.z);
}
__device__ __forceinline__ void add_fix3(long long* p, float3 f) {
    fix_atomic_add(p + 0, fix_from_float(f.x));
    fix_atomic_add(p + 1, fix_from_float(f.y));
    fix_atomic_add(p + 2, fix_from_float(f.z));
}

template <bool ENERGY>
__device__ __forceinline__ void write_partials(const SysView& v, int region, double el, double ec,
                                               double w) {
    double x[3] = {el, ec, w};
    block_sum_d<3>(x);
    if (threadIdx.x == 0) {
        double* p = v.partials + ((size_t)region * v.max_blocks + blockIdx.x) * 4;
        p[0] = x[0]; p[1] = x[1]; p[2] = x[2]; p[3] = 0.0;
    }
}

// ---------------------------------------------------------------------------
// water(i) - water(j)
// ---------------------------------------------------------------------------
template <bool ENERGY>
__global__ void __launch_bounds__(PT) k_pair_ww(SysView v) {
    const int lane = threadIdx.x & 31;
    const int ii = lane & 7, jq = lane >> 3;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t nwc = v.sc->n_wclus;
    const BoxDev b = *v.box;
    const float rc2 = v.rc2, ljc2 = v.ljc2, alpha = v.alpha;
    const float c2a = 2.0f * alpha * INV_SQRT_PI_F;
    const float sig2 = OPC_O_SIGMA * OPC_O_SIGMA;
    const float qhh = OPC_Q_H * OPC_Q_H, qhm = OPC_Q_H * OPC_Q_EP, qmm = OPC_Q_EP * OPC_Q_EP;
    double el = 0.0, ec = 0.0, ew = 0.0;
    for (uint32_t ci = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); ci < nwc; ci += nwarps) {
        const uint32_t si = ci * WCL + ii;
        const bool vi = v.wid[si] != INVALID_ID;
        const float3 iO = xyz(v.wpos[4 * si + 0]), iH0 = xyz(v.wpos[4 * si + 1]);
        const float3 iH1 = xyz(v.wpos[4 * si + 2]), iM = xyz(v.wpos[4 * si + 3]);
        float3 fO = f3(0, 0, 0), fH0 = fO, fH1 = fO, fM = fO;
        Acc3 a{0.f, 0.f, 0.f};
        const uint32_t n = v.ww_n[ci];
        const uint32_t* lst = v.ww_j + (size_t)ci * v.cap_ww;
        for (uint32_t k = 0; k < n; ++k) {
            const uint32_t cj = lst[k];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int jj = jq + 4 * h;
                const uint32_t sj = cj * WCL + jj;
                const bool ok = vi && v.wid[sj] != INVALID_ID && !(cj == ci && jj == ii);
                if (!ok) continue;
                const float3 jO = xyz(v.wpos[4 * sj + 0]), jH0 = xyz(v.wpos[4 * sj + 1]);
                const float3 jH1 = xyz(v.wpos[4 * sj + 2]), jM = xyz(v.wpos[4 * sj + 3]);
                const float3 s = shift_of(iO - jO, b);
                const float3 jOs = jO - s, jH0s = jH0 - s, jH1s = jH1 - s, jMs = jM - s;
                lj<ENERGY>(iO - jOs, sig2, OPC_O_EPS, ljc2, 1.0f, fO, a);
                coul<ENERGY>(iH0 - jH0s, qhh, rc2, alpha, c2a, fH0, a);
                coul<ENERGY>(iH0 - jH1s, qhh, rc2, alpha, c2a, fH0, a);
                coul<ENERGY>(iH0 - jMs, qhm, rc2, alpha, c2a, fH0, a);
                coul<ENERGY>(iH1 - jH0s, qhh, rc2, alpha, c2a, fH1, a);
                coul<ENERGY>(iH1 - jH1s, qhh, rc2, alpha, c2a, fH1, a);
                coul<ENERGY>(iH1 - jMs, qhm, rc2, alpha, c2a, fH1, a);
                coul<ENERGY>(iM - jH0s, qhm, rc2, alpha, c2a, fM, a);
                coul<ENERGY>(iM - jH1s, qhm, rc2, alpha, c2a, fM, a);
                coul<ENERGY>(iM - jMs, qmm, rc2, alpha, c2a, fM, a);
            }
        }
        fO = f3(red4(fO.x), red4(fO.y), red4(fO.z));
        fH0 = f3(red4(fH0.x), red4(fH0.y), red4(fH0.z));
        fH1 = f3(red4(fH1.x), red4(fH1.y), red4(fH1.z));
        fM = f3(red4(fM.x), red4(fM.y), red4(fM.z));
        if (jq == 0) {
            long long* p = v.wforce + (size_t)si * 12;
            store_fix3(p + 0, fO); store_fix3(p + 3, fH0); store_fix3(p + 6, fH1); store_fix3(p + 9, fM);
        }
        if (ENERGY) { el += a.e_lj; ec += a.e_c; }
        ew += a.w;
    }
    write_partials<ENERGY>(v, REG_WW, el, ec, ew);
}

// ---------------------------------------------------------------------------
// water(i) - atom(j): forces on the water sites
// ---------------------------------------------------------------------------
template <bool ENERGY>
__global__ void __launch_bounds__(PT) k_pair_ws(SysView v) {
    const int lane = threadIdx.x & 31;
    const int ii = lane & 7, jq = lane >> 3;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t nwc = v.sc->n_wclus;
    const BoxDev b = *v.box;
    const float rc2 = v.rc2, ljc2 = v.ljc2, alpha = v.alpha;
    const float c2a = 2.0f * alpha * INV_SQRT_PI_F;
    double el = 0.0, ec = 0.0, ew = 0.0;
    for (uint32_t ci = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); ci < nwc; ci += nwarps) {
        const uint32_t n = v.ws_n[ci];
        if (n == 0) continue;
        const uint32_t si = ci * WCL + ii;
        const bool vi = v.wid[si] != INVALID_ID;
        const float3 iO = xyz(v.wpos[4 * si + 0]), iH0 = xyz(v.wpos[4 * si + 1]);
        const float3 iH1 = xyz(v.wpos[4 * si + 2]), iM = xyz(v.wpos[4 * si + 3]);
        float3 fO = f3(0, 0, 0), fH0 = fO, fH1 = fO, fM = fO;
        Acc3 a{0.f, 0.f, 0.f};
        const uint32_t* lst = v.ws_j + (size_t)ci * v.cap_ws;
        for (uint32_t k = 0; k < n; ++k) {
            const uint32_t cj = lst[k];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const uint32_t sj = cj * ACL + jq + 4 * h;
                if (!vi || v.sidx[sj] == INVALID_ID) continue;
                const float4 pj = v.spos[sj];
                const float2 lj_j = v.slj[sj];
                const float3 s = shift_of(iO - xyz(pj), b);
                const float3 jp = xyz(pj) - s;
                const float sg = 0.5f * (OPC_O_SIGMA + lj_j.x);
                const float ep = sqrtf(OPC_O_EPS * lj_j.y);
                lj<ENERGY>(iO - jp, sg * sg, ep, ljc2, 1.0f, fO, a);
                coul<ENERGY>(iH0 - jp, OPC_Q_H * pj.w, rc2, alpha, c2a, fH0, a);
                coul<ENERGY>(iH1 - jp, OPC_Q_H * pj.w, rc2, alpha, c2a, fH1, a);
                coul<ENERGY>(iM - jp, OPC_Q_EP * pj.w, rc2, alpha, c2a, fM, a);
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
        ew += a.w;
    }
    write_partials<ENERGY>(v, REG_WS, el, ec, ew);
}

// ---------------------------------------------------------------------------
// atom(i) - water(j): forces on the atoms
// ---------------------------------------------------------------------------
template <bool ENERGY>
__global__ void __launch_bounds__(PT) k_pair_sw(SysView v) {
    const int lane = threadIdx.x & 31;
    const int ii = lane & 7, jq = lane >> 3;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t nac = v.sc->n_aclus;
    const BoxDev b = *v.box;
    const float rc2 = v.rc2, ljc2 = v.ljc2, alpha = v.alpha;
    const float c2a = 2.0f * alpha * INV_SQRT_PI_F;
    double el = 0.0, ec = 0.0, ew = 0.0;
    for (uint32_t ci = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); ci < nac; ci += nwarps) {
        const uint32_t n = v.sw_n[ci];
        if (n == 0) continue;
        const uint32_t si = ci * ACL + ii;
        const uint32_t ai = v.sidx[si];
        const bool vi = ai != INVALID_ID;
        const float4 pi = v.spos[si];
        const float2 lji = v.slj[si];
        const float sg = 0.5f * (OPC_O_SIGMA + lji.x);
        const float ep = sqrtf(OPC_O_EPS * lji.y);
        float3 f = f3(0, 0, 0);
        Acc3 a{0.f, 0.f, 0.f};
        const uint32_t* lst = v.sw_j + (size_t)ci * v.cap_sw;
        for (uint32_t k = 0; k < n; ++k) {
            const uint32_t cj = lst[k];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const uint32_t sj = cj * WCL + jq + 4 * h;
                if (!vi || v.wid[sj] == INVALID_ID) continue;
                const float3 jO = xyz(v.wpos[4 * sj + 0]);
                const float3 s = shift_of(xyz(pi) - jO, b);
                lj<ENERGY>(xyz(pi) - (jO - s), sg * sg, ep, ljc2, 1.0f, f, a);
                coul<ENERGY>(xyz(pi) - (xyz(v.wpos[4 * sj + 1]) - s), pi.w * OPC_Q_H, rc2, alpha, c2a, f, a);
                coul<ENERGY>(xyz(pi) - (xyz(v.wpos[4 * sj + 2]) - s), pi.w * OPC_Q_H, rc2, alpha, c2a, f, a);
                coul<ENERGY>(xyz(pi) - (xyz(v.wpos[4 * sj + 3]) - s), pi.w * OPC_Q_EP, rc2, alpha, c2a, f, a);
            }
        }
        f = f3(red4(f.x), red4(f.y), red4(f.z));
        if (jq == 0 && vi) add_fix3(v.aforce + 3 * (size_t)ai, f);
        if (ENERGY) { el += a.e_lj; ec += a.e_c; }
        ew += a.w;
    }
    write_partials<ENERGY>(v, REG_SW, el, ec, ew);
}

// ---------------------------------------------------------------------------
// atom(i) - atom(j): interaction mask from the list build
// ---------------------------------------------------------------------------
template <bool ENERGY>
__global__ void __launch_bounds__(PT) k_pair_ss(SysView v) {
    const int lane = threadIdx.x & 31;
    const int ii = lane & 7, jq = lane >> 3;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t nac = v.sc->n_aclus;
    const BoxDev b = *v.box;
    const float rc2 = v.rc2, ljc2 = v.ljc2, alpha = v.alpha;
    const float c2a = 2.0f * alpha * INV_SQRT_PI_F;
    double el = 0.0, ec = 0.0, ew = 0.0;
    for (uint32_t ci = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); ci < nac; ci += nwarps) {
        const uint32_t si = ci * ACL + ii;
        const uint32_t ai = v.sidx[si];
        const float4 pi = v.spos[si];
        const float2 lji = v.slj[si];
        float3 f = f3(0, 0, 0);
        Acc3 a{0.f, 0.f, 0.f};
        const uint32_t n = v.ss_n[ci];
        const uint32_t* lst = v.ss_j + (size_t)ci * v.cap_ss;
        const unsigned long long* msk = v.ss_mask + (size_t)ci * v.cap_ss;
        for (uint32_t k = 0; k < n; ++k) {
            const uint32_t cj = lst[k];
            const unsigned long long m = msk[k];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int jj = jq + 4 * h;
                if (!((m >> (ii * ACL + jj)) & 1ull)) continue;
                const uint32_t sj = cj * ACL + jj;
                const float4 pj = v.spos[sj];
                const float2 ljj = v.slj[sj];
                const float3 d = min_image_rint(xyz(pi) - xyz(pj), b);
                const float sg = 0.5f * (lji.x + ljj.x);
                lj<ENERGY>(d, sg * sg, sqrtf(lji.y * ljj.y), ljc2, 1.0f, f, a);
                coul<ENERGY>(d, pi.w * pj.w, rc2, alpha, c2a, f, a);
            }
        }
        f = f3(red4(f.x), red4(f.y), red4(f.z));
        if (jq == 0 && ai != INVALID_ID) store_fix3(v.aforce + 3 * (size_t)ai, f);
        if (ENERGY) { el += a.e_lj; ec += a.e_c; }
        ew += a.w;
    }
    write_partials<ENERGY>(v, REG_SS, el, ec, ew);
}

// ---------------------------------------------------------------------------
// 1-4 pairs: LJ x0.5, Coulomb x1/1.2 (src/non_bonded.rs:55-56,1014-1042)
// ---------------------------------------------------------------------------
template <bool ENERGY>
__global__ void k_pair14(SysView v) {
    const BoxDev b = *v.box;
    const float c2a = 2.0f * v.alpha * INV_SQRT_PI_F;
    double e_acc = 0.0, w_acc = 0.0;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < v.n14; k += gridDim.x * blockDim.x) {
        const uint2 p = v.p14[k];
        const float4 par = v.p14_par[k];  // sigma, eps, qq
        const float3 d = min_image_rint(xyz(v.apos[p.x]) - xyz(v.apos[p.y]), b);
        float3 f = f3(0, 0, 0);
        Acc3 a{0.f, 0.f, 0.f};
        lj<ENERGY>(d, par.x * par.x, par.y, v.ljc2, 0.5f, f, a);
        float3 fc = f3(0, 0, 0);
        Acc3 ac{0.f, 0.f, 0.f};
        coul<ENERGY>(d, par.z, v.rc2, v.alpha, c2a, fc, ac);
        const float s = 0.833333333f;
        f = f + fc * s;
        add_fix3(v.aforce + 3 * (size_t)p.x, f);
        add_fix3(v.aforce + 3 * (size_t)p.y, f3(-f.x, -f.y, -f.z));
        if (ENERGY) e_acc += (double)a.e_lj + (double)ac.e_c * s;
        w_acc += (double)a.w + (double)ac.w * s;
    }
    write_partials<ENERGY>(v, REG_14, e_acc, 0.0, w_acc);
}

inline int pblocks(const SysView& v, uint64_t warps) {
    uint64_t bl = (warps * 32 + PT - 1) / PT;
    if (bl < 1) bl = 1;
    return (int)(bl < v.max_blocks ? bl : v.max_blocks);
}

}  // namespace

namespace dyn {

int pair_blocks_ww(const SysView& v) { return pblocks(v, v.nwclus_cap); }
int pair_blocks_ss(const SysView& v) { return pblocks(v, v.naclus_cap); }
int pair14_blocks(const SysView& v) {
    uint64_t bl = (v.n14 + 255) / 256;
    if (bl < 1) bl = 1;
    return (int)(bl < v.max_blocks ? bl : v.max_blocks);
}

void launch_pairs(const SysView& v, cudaStream_t st, bool energy) {
    const int bw = pblocks(v, v.nwclus_cap), ba = pblocks(v, v.naclus_cap);
    if (energy) {
        if (v.nw) k_pair_ww<true><<<bw, PT, 0, st>>>(v);
        if (v.na) k_pair_ss<true><<<ba, PT, 0, st>>>(v);
        if (v.nw && v.na) {
            k_pair_ws<true><<<bw, PT, 0, st>>>(v);
            k_pair_sw<true><<<ba, PT, 0, st>>>(v);
        }
    } else {
        if (v.nw) k_pair_ww<false><<<bw, PT, 0, st>>>(v);
        if (v.na) k_pair_ss<false><<<ba, PT, 0, st>>>(v);
        if (v.nw && v.na) {
            k_pair_ws<false><<<bw, PT, 0, st>>>(v);
            k_pair_sw<false><<<ba, PT, 0, st>>>(v);
        }
    }
}

void launch_pair14(const SysView& v, cudaStream_t st, bool energy) {
    if (!v.n14) return;
    if (energy) k_pair14<true><<<pair14_blocks(v), 256, 0, st>>>(v);
    else k_pair14<false><<<pair14_blocks(v), 256, 0, st>>>(v);
}

}  // namespace dyn
