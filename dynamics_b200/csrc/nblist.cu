// Cluster neighbour lists of the resident engine.
//
// The reference rebuilds O(N^2) Verlet lists with a 4 A skin on the host and
// re-uploads 33 B per pair (src/neighbors.rs:102-281,
// src/gpu_interface.rs:243-410).  Here the rebuild runs on the device:
//   1. molecules / atoms are binned into columns of an xy grid and ranked by
//      z inside each column (deterministic: ties broken by index);
//   2. waters are physically permuted into that order, columns padded to a
//      multiple of 8, so every aligned 8-slot group is a compact cluster;
//   3. cluster bounding boxes are tested against each other (all pairs,
//      min-image on centres) and each i-cluster's hits are compacted with
//      warp ballots into a fixed-capacity list, ascending in j;
//   4. for water-water, 32-water groups get a tile of j-clusters and every
//      water a compact list of tile-local molecule indices (O-O distance
//      below cutoff + twice the O-H reach + buffer).
// Every kernel of the rebuild returns immediately unless the displacement
// check raised Scalars::need_rebuild; inside a captured step graph the
// rebuild kernels also sit under a conditional (IF) node that the check
// sets, so steps without a rebuild launch none of them.  The rebuild criterion is the reference's: max displacement since
// the last rebuild >= buffer / 2 (src/neighbors.rs:159-169), tracking water
// O only (src/neighbors.rs:71-82); water list radii add twice the O-H reach.
#include <algorithm>

#include "engine.cuh"

namespace {

__device__ __forceinline__ bool rebuild_on(const SysView& v, bool force) {
    return force || v.sc->need_rebuild;
}

__device__ __forceinline__ float frac_box(float x, float lo, float inv_ext) {
    float f = (x - lo) * inv_ext;
    f -= floorf(f);
    return f >= 1.0f ? 0.0f : f;
}

// Column rank along a boustrophedon path over the xy grid, and the sort key
// inside the column: z ascending in even-ranked columns, descending in odd
// ones, so consecutive slots are neighbours in space across column ends too.
__device__ __forceinline__ uint32_t column_of(float3 p, const BoxDev& b, uint32_t ncx, uint32_t ncy,
                                              float* key) {
    const float fx = frac_box(p.x, b.lo[0], b.inv_ext[0]);
    const float fy = frac_box(p.y, b.lo[1], b.inv_ext[1]);
    const float fz = frac_box(p.z, b.lo[2], b.inv_ext[2]);
    const uint32_t cx = min((uint32_t)(fx * ncx), ncx - 1);
    const uint32_t cy = min((uint32_t)(fy * ncy), ncy - 1);
    const uint32_t rank = cy * ncx + ((cy & 1u) ? (ncx - 1 - cx) : cx);
    *key = (rank & 1u) ? 1.0f - fz : fz;
    return rank;
}

// ---------------------------------------------------------------------------
// displacement check
// ---------------------------------------------------------------------------
DYN_KERNEL(, k_disp_check, (), ()) {
    const BoxDev b = *v.box;
    float m = 0.f, mp = 0.f;
    const uint32_t tid = bk.idx * blockDim.x + threadIdx.x;
    const uint32_t stride = bk.cnt * blockDim.x;
    for (uint32_t s = tid; s < v.nw_cap; s += stride) {
        if (v.wid[s] == INVALID_ID) continue;
        const float3 o = xyz(v.wpos[4 * s]);
        const float3 d = min_image_rint(o - xyz(v.wref[s]), b);
        const float d2 = dot3(d, d);
        m = fmaxf(m, isfinite(d2) ? d2 : 1e30f);
        // since the last prune of the water-water lists
        const float3 dp = min_image_rint(o - xyz(v.wprune[s]), b);
        const float dp2 = dot3(dp, dp);
        mp = fmaxf(mp, isfinite(dp2) ? dp2 : 1e30f);
    }
    for (uint32_t a = tid; a < v.na; a += stride) {
        const float3 d = xyz(v.apos[a]) - xyz(v.aref[a]);
        const float d2 = dot3(d, d);
        m = fmaxf(m, isfinite(d2) ? d2 : 1e30f);
    }
    m = warp_max_f(m);
    mp = warp_max_f(mp);
    if ((threadIdx.x & 31) == 0 && m > 0.f) atomicMax(&v.sc->max_disp2_bits, __float_as_uint(m));
    if ((threadIdx.x & 31) == 0 && mp > 0.f) atomicMax(&v.sc->max_dprune_bits, __float_as_uint(mp));
    __threadfence();
    __syncthreads();
    if (threadIdx.x != 0) return;
    if (atomicAdd(&v.sc->ctr_disp, 1u) != bk.cnt - 1) return;
    // the last block to finish sees every block's maximum and decides:
    // rebuild when the largest displacement reaches half the buffer
    __threadfence();
    const float mx = __uint_as_float(atomicExch(&v.sc->max_disp2_bits, 0u));
    const float mxp = __uint_as_float(atomicExch(&v.sc->max_dprune_bits, 0u));
    const float h = 0.5f * v.buffer;
    unsigned int need = v.sc->need_rebuild;
    if (mx >= h * h) need = 1u;
    v.sc->need_rebuild = need;
    // new outer lists are pruned at once; otherwise prune when a water has
    // moved half the inner buffer
    const float hp = 0.5f * v.prune_buf;
    unsigned int need_p = v.sc->need_prune | need;
    if (mxp >= hp * hp) need_p = 1u;
    v.sc->need_prune = need_p;
    if (mx >= 1e29f || mxp >= 1e29f) v.sc->nonfinite = 1u;
    v.sc->ctr_disp = 0u;
    if (v.use_cond && need) cudaGraphSetConditional(v.cond_rebuild, 1u);
    if (v.use_cond && need_p) cudaGraphSetConditional(v.cond_prune, 1u);
}

// ---------------------------------------------------------------------------
// column binning
// ---------------------------------------------------------------------------
DYN_KERNEL(, k_col_clear, (, bool force), (, force)) {
    if (!rebuild_on(v, force)) return;
    if (bk.idx == 0 && threadIdx.x == 0) {
        v.sc->list_pairs = 0ull;
        v.sc->union_max = 0u;
    }
    const uint32_t nc = v.ncol > v.ancol ? v.ncol : v.ancol;
    for (uint32_t c = bk.idx * blockDim.x + threadIdx.x; c < nc; c += bk.cnt * blockDim.x) {
        if (c < v.ncol) { v.col_count[c] = 0; v.col_fill[c] = 0; }
        if (c < v.ancol) { v.acol_count[c] = 0; v.acol_fill[c] = 0; }
    }
}

DYN_KERNEL(, k_col_assign, (, bool force), (, force)) {
    if (!rebuild_on(v, force)) return;
    const BoxDev b = *v.box;
    const uint32_t tid = bk.idx * blockDim.x + threadIdx.x;
    const uint32_t stride = bk.cnt * blockDim.x;
    for (uint32_t s = tid; s < v.nw_cap; s += stride) {
        if (v.wid[s] == INVALID_ID) continue;
        float zf;
        const uint32_t c = column_of(xyz(v.wpos[4 * s]), b, v.ncx, v.ncy, &zf);
        v.wcol[s] = c;
        v.wkey[s] = zf;
        atomicAdd(&v.col_count[c], 1u);
    }
    for (uint32_t a = tid; a < v.na; a += stride) {
        if (v.asparse[a] != INVALID_ID) continue;
        float zf;
        const uint32_t c = column_of(xyz(v.apos[a]), b, v.ancx, v.ancy, &zf);
        v.acol[a] = c;
        v.akey[a] = zf;
        atomicAdd(&v.acol_count[c], 1u);
    }
}

// Serial scan over columns in path order (only at rebuilds; a few hundred
// columns).  Slots are contiguous along the path; padding sits at the end.
DYN_KERNEL(, k_col_scan, (, bool force), (, force)) {
    if (!rebuild_on(v, force)) return;
    if (threadIdx.x == 0) {
        uint32_t q = 0;
        for (uint32_t c = 0; c < v.ncol; ++c) {
            v.col_off[c] = q; v.col_boff[c] = q;
            q += v.col_count[c];
        }
        v.col_off[v.ncol] = q; v.col_boff[v.ncol] = q;
        v.sc->n_wclus = (q + WCL - 1) / WCL;
    } else if (threadIdx.x == 32) {
        uint32_t q = 0;
        for (uint32_t c = 0; c < v.ancol; ++c) {
            v.acol_off[c] = q; v.acol_boff[c] = q;
            q += v.acol_count[c];
        }
        v.acol_off[v.ancol] = q; v.acol_boff[v.ancol] = q;
        // clustered atoms fill whole clusters from slot 0; each atom without
        // bonds then gets a cluster of its own
        const uint32_t base = (q + ACL - 1) / ACL * ACL;
        v.sc->a_sparse_base = base;
        v.sc->n_aclus = base / ACL + v.n_sparse;
    }
}

DYN_KERNEL(, k_col_bucket, (, bool force), (, force)) {
    if (!rebuild_on(v, force)) return;
    const uint32_t tid = bk.idx * blockDim.x + threadIdx.x;
    const uint32_t stride = bk.cnt * blockDim.x;
    for (uint32_t s = tid; s < v.nw_cap; s += stride) {
        if (v.wid[s] == INVALID_ID) continue;
        const uint32_t c = v.wcol[s];
        v.bucket[v.col_boff[c] + atomicAdd(&v.col_fill[c], 1u)] = s;
    }
    for (uint32_t a = tid; a < v.na; a += stride) {
        if (v.asparse[a] != INVALID_ID) continue;
        const uint32_t c = v.acol[a];
        v.abucket[v.acol_boff[c] + atomicAdd(&v.acol_fill[c], 1u)] = a;
    }
}

// Rank inside the column by (z, original index): deterministic order.
DYN_KERNEL(, k_col_rank, (, bool force), (, force)) {
    if (!rebuild_on(v, force)) return;
    const uint32_t tid = bk.idx * blockDim.x + threadIdx.x;
    const uint32_t stride = bk.cnt * blockDim.x;
    for (uint32_t s = tid; s < v.nw_cap; s += stride) {
        if (v.wid[s] == INVALID_ID) continue;
        const uint32_t c = v.wcol[s];
        const float z = v.wkey[s];
        const uint32_t id = v.wid[s];
        uint32_t r = 0;
        for (uint32_t k = v.col_boff[c]; k < v.col_boff[c + 1]; ++k) {
            const uint32_t m = v.bucket[k];
            const float zm = v.wkey[m];
            r += (zm < z) || (zm == z && v.wid[m] < id);
        }
        v.wnew[s] = v.col_off[c] + r;
    }
    for (uint32_t a = tid; a < v.na; a += stride) {
        if (v.asparse[a] != INVALID_ID) {
            v.aslot[a] = v.sc->a_sparse_base + ACL * v.asparse[a];
            continue;
        }
        const uint32_t c = v.acol[a];
        const float z = v.akey[a];
        uint32_t r = 0;
        for (uint32_t k = v.acol_boff[c]; k < v.acol_boff[c + 1]; ++k) {
            const uint32_t m = v.abucket[k];
            const float zm = v.akey[m];
            r += (zm < z) || (zm == z && m < a);
        }
        v.aslot[a] = v.acol_off[c] + r;
    }
}

DYN_KERNEL(, k_perm_init, (, bool force), (, force)) {
    if (!rebuild_on(v, force)) return;
    const uint32_t tid = bk.idx * blockDim.x + threadIdx.x;
    const uint32_t stride = bk.cnt * blockDim.x;
    for (uint32_t s = tid; s < v.nw_cap; s += stride) {
        v.wtmp_id[s] = INVALID_ID;
        for (int k = 0; k < 10; ++k) v.wtmp[10 * s + k] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    for (uint32_t s = tid; s < v.na_cap; s += stride) {
        v.sidx[s] = INVALID_ID;
        v.slj[s] = make_float2(0.f, 0.f);
        v.spos[s] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
}

DYN_KERNEL(, k_perm_scatter, (, bool force), (, force)) {
    if (!rebuild_on(v, force)) return;
    const uint32_t tid = bk.idx * blockDim.x + threadIdx.x;
    const uint32_t stride = bk.cnt * blockDim.x;
    for (uint32_t s = tid; s < v.nw_cap; s += stride) {
        if (v.wid[s] == INVALID_ID) continue;
        const uint32_t n = v.wnew[s];
        for (int k = 0; k < 4; ++k) v.wtmp[10 * n + k] = v.wpos[4 * s + k];
        for (int k = 0; k < 3; ++k) v.wtmp[10 * n + 4 + k] = v.wvel[3 * s + k];
        for (int k = 0; k < 3; ++k) v.wtmp[10 * n + 7 + k] = v.wacc[3 * s + k];
        v.wtmp_id[n] = v.wid[s];
    }
    for (uint32_t a = tid; a < v.na; a += stride) {
        const uint32_t s = v.aslot[a];
        v.sidx[s] = a;
        v.slj[s] = v.alj[a];
        v.spos[s] = v.apos[a];
        v.aref[a] = v.apos[a];
    }
}

DYN_KERNEL(, k_perm_copyback, (, bool force), (, force)) {
    if (!rebuild_on(v, force)) return;
    const uint32_t tid = bk.idx * blockDim.x + threadIdx.x;
    const uint32_t stride = bk.cnt * blockDim.x;
    for (uint32_t s = tid; s < v.nw_cap; s += stride) {
        for (int k = 0; k < 4; ++k) v.wpos[4 * s + k] = v.wtmp[10 * s + k];
        for (int k = 0; k < 3; ++k) v.wvel[3 * s + k] = v.wtmp[10 * s + 4 + k];
        for (int k = 0; k < 3; ++k) v.wacc[3 * s + k] = v.wtmp[10 * s + 7 + k];
        v.wid[s] = v.wtmp_id[s];
        v.wref[s] = v.wtmp[10 * s];
    }
}

// Bounding boxes of water clusters (O positions) and atom clusters.
DYN_KERNEL(, k_bbox, (, bool force), (, force)) {
    if (!rebuild_on(v, force)) return;
    const BoxDev b = *v.box;
    const uint32_t nwc = v.sc->n_wclus, nac = v.sc->n_aclus;
    const uint32_t tid = bk.idx * blockDim.x + threadIdx.x;
    const uint32_t stride = bk.cnt * blockDim.x;
    for (uint32_t c = tid; c < nwc + nac; c += stride) {
        float3 lo = f3(1e30f, 1e30f, 1e30f), hi = f3(-1e30f, -1e30f, -1e30f);
        const bool is_w = c < nwc;
        const uint32_t cl = is_w ? c : c - nwc;
        // reference point: first valid member; others are min-imaged to it so
        // a cluster straddling a periodic face still gets a compact box
        bool have = false;
        float3 ref = f3(0.f, 0.f, 0.f);
        for (int k = 0; k < 8; ++k) {
            float3 p;
            if (is_w) {
                const uint32_t s = cl * WCL + k;
                if (v.wid[s] == INVALID_ID) continue;
                p = xyz(v.wpos[4 * s]);
            } else {
                const uint32_t s = cl * ACL + k;
                if (v.sidx[s] == INVALID_ID) continue;
                p = xyz(v.spos[s]);
            }
            if (!have) { ref = p; have = true; }
            p = ref + min_image_rint(p - ref, b);
            lo = f3(fminf(lo.x, p.x), fminf(lo.y, p.y), fminf(lo.z, p.z));
            hi = f3(fmaxf(hi.x, p.x), fmaxf(hi.y, p.y), fmaxf(hi.z, p.z));
        }
        if (!have) { lo = f3(0.f, 0.f, 0.f); hi = lo; }
        const float4 cen = make_float4(0.5f * (lo.x + hi.x), 0.5f * (lo.y + hi.y), 0.5f * (lo.z + hi.z), 0.f);
        const float4 half = make_float4(0.5f * (hi.x - lo.x), 0.5f * (hi.y - lo.y), 0.5f * (hi.z - lo.z), 0.f);
        if (is_w) { v.wbb_c[cl] = cen; v.wbb_h[cl] = half; }
        else { v.abb_c[cl] = cen; v.abb_h[cl] = half; }
    }
}

__device__ __forceinline__ float bb_dist2(float4 ci, float4 hi, float4 cj, float4 hj, const BoxDev& b) {
    float3 d = f3(ci.x - cj.x, ci.y - cj.y, ci.z - cj.z);
    d = min_image_rint(d, b);
    const float gx = fmaxf(0.f, fabsf(d.x) - hi.x - hj.x);
    const float gy = fmaxf(0.f, fabsf(d.y) - hi.y - hj.y);
    const float gz = fmaxf(0.f, fabsf(d.z) - hi.z - hj.z);
    return gx * gx + gy * gy + gz * gz;
}

__device__ __forceinline__ bool excluded(const SysView& v, uint32_t a, uint32_t b) {
    uint32_t lo = v.ex_off[a], hi = v.ex_off[a + 1];
    while (lo < hi) {
        const uint32_t m = (lo + hi) >> 1;
        if (v.ex_idx[m] < b) lo = m + 1; else hi = m;
    }
    return lo < v.ex_off[a + 1] && v.ex_idx[lo] == b;
}

// One warp per i-cluster.  MODE 1: water i-clusters against atom
// j-clusters; MODE 3: atom i-clusters against atom j-clusters with cj >= ci
// (each cluster pair once), with the interaction mask of the cluster pair
// (jj > ii on the diagonal, exclusions removed).
DYN_KERNEL_T((int MODE), (MODE), , k_list, (, bool force), (, force)) {
    if (!rebuild_on(v, force)) return;
    const BoxDev b = *v.box;
    const int lane = threadIdx.x & 31;
    const uint32_t ci = (bk.idx * blockDim.x + threadIdx.x) >> 5;
    const uint32_t ni = MODE == 1 ? v.sc->n_wclus : v.sc->n_aclus;
    const uint32_t nj = v.sc->n_aclus;
    if (ci >= ni) return;
    const float4* bcj = v.abb_c;
    const float4* bhj = v.abb_h;
    const float r = MODE == 3 ? v.r_ss : v.r_ws;
    const float r2 = r * r;
    const uint32_t cap = MODE == 1 ? v.cap_ws : v.cap_ss;
    uint32_t* out = MODE == 1 ? v.ws_j : v.ss_j;
    uint32_t* outn = MODE == 1 ? v.ws_n : v.ss_n;
    const float4 c0 = MODE == 1 ? v.wbb_c[ci] : v.abb_c[ci];
    const float4 h0 = MODE == 1 ? v.wbb_h[ci] : v.abb_h[ci];
    uint32_t cnt = 0;
    for (uint32_t jb = MODE == 3 ? (ci & ~31u) : 0u; jb < nj; jb += 32) {
        const uint32_t cj = jb + lane;
        bool hit = false;
        if (cj < nj && (MODE != 3 || cj >= ci)) hit = bb_dist2(c0, h0, bcj[cj], bhj[cj], b) < r2;
        const uint32_t m = __ballot_sync(0xffffffffu, hit);
        if (hit) {
            const uint32_t k = cnt + __popc(m & ((1u << lane) - 1u));
            if (k < cap) out[(size_t)ci * cap + k] = cj;
        }
        if (MODE == 3) {
            // interaction masks, one hit at a time with the whole warp: lane
            // decides the pairs (ii, jj) = (lane / 8, lane % 8) and
            // (lane / 8 + 4, lane % 8); bit ii * 8 + jj
            for (uint32_t mm = m; mm; mm &= mm - 1u) {
                const int src = __ffs(mm) - 1;
                const uint32_t k = cnt + __popc(m & ((1u << src) - 1u));
                const uint32_t cjh = jb + (uint32_t)src;
                bool pb[2];
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int ii = (lane >> 3) + 4 * h, jj = lane & 7;
                    const uint32_t a = v.sidx[ci * ACL + ii];
                    const uint32_t c = v.sidx[cjh * ACL + jj];
                    bool on = a != INVALID_ID && c != INVALID_ID && !(cjh == ci && jj <= ii);
                    if (on && v.astatic && v.astatic[a] && v.astatic[c]) on = false;
                    if (on && v.ex_off && excluded(v, a, c)) on = false;
                    pb[h] = on;
                }
                const uint32_t lo = __ballot_sync(0xffffffffu, pb[0]);
                const uint32_t hi = __ballot_sync(0xffffffffu, pb[1]);
                if (lane == 0 && k < cap) v.ss_mask[(size_t)ci * cap + k] = (unsigned long long)hi << 32 | lo;
            }
        }
        cnt += __popc(m);
    }
    if (lane == 0) {
        outn[ci] = min(cnt, cap);
        if (cnt > cap) atomicMax(&v.sc->overflow, cnt);
        atomicAdd(&v.sc->list_pairs, (unsigned long long)min(cnt, cap));
    }
}

// Work items of the atom pair kernels: for every i-cluster (in order) one
// item per ch_mix entries of its list, {cluster, first entry}.  One block;
// an exclusive scan of the per-cluster item counts, tile by tile.
constexpr int IT_T = 1024;
DYN_KERNEL_T((int MODE), (MODE), __launch_bounds__(IT_T), k_items, (, bool force), (, force)) {
    if (!rebuild_on(v, force)) return;
    const uint32_t ni = MODE == 1 ? v.sc->n_wclus : v.sc->n_aclus;
    const uint32_t* cnt = MODE == 1 ? v.ws_n : v.ss_n;
    uint2* items = MODE == 1 ? v.ws_item : v.ss_item;
    const uint32_t icap = MODE == 1 ? v.ws_item_cap : v.ss_item_cap;
    __shared__ uint32_t wsum[IT_T / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t base = 0;
    for (uint32_t c0 = 0; c0 < ni; c0 += IT_T) {
        const uint32_t c = c0 + threadIdx.x;
        const uint32_t k = c < ni ? (cnt[c] + v.ch_mix - 1) / v.ch_mix : 0u;
        uint32_t x = k;  // inclusive scan inside the warp
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[w] = x;
        __syncthreads();
        if (w == 0) {
            uint32_t t = lane < IT_T / 32 ? wsum[lane] : 0u;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += y;
            }
            if (lane < IT_T / 32) wsum[lane] = t;  // inclusive warp totals
        }
        __syncthreads();
        const uint32_t off = base + (w ? wsum[w - 1] : 0u) + x - k;
        for (uint32_t t = 0; t < k; ++t)
            if (off + t < icap) items[off + t] = make_uint2(c, t * v.ch_mix);
        base += wsum[IT_T / 32 - 1];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        if (MODE == 1) v.sc->n_ws_items = min(base, icap);
        else v.sc->n_ss_items = min(base, icap);
    }
}

// Group bounding boxes over the O positions of the group's waters,
// min-imaged to the first one.
DYN_KERNEL(, k_group_bbox, (, bool force), (, force)) {
    if (!rebuild_on(v, force)) return;
    const BoxDev b = *v.box;
    const uint32_t nwc = v.sc->n_wclus;
    const uint32_t ng = (nwc + GRPW / WCL - 1) / (GRPW / WCL);
    for (uint32_t g = bk.idx * blockDim.x + threadIdx.x; g < ng; g += bk.cnt * blockDim.x) {
        float3 lo = f3(1e30f, 1e30f, 1e30f), hi = f3(-1e30f, -1e30f, -1e30f);
        bool have = false;
        float3 ref = f3(0.f, 0.f, 0.f);
        for (uint32_t k = 0; k < GRPW; ++k) {
            const uint32_t s = g * GRPW + k;
            if (s >= v.nw_cap || v.wid[s] == INVALID_ID) continue;
            float3 p = xyz(v.wpos[4 * s]);
            if (!have) { ref = p; have = true; }
            p = ref + min_image_rint(p - ref, b);
            lo = f3(fminf(lo.x, p.x), fminf(lo.y, p.y), fminf(lo.z, p.z));
            hi = f3(fmaxf(hi.x, p.x), fmaxf(hi.y, p.y), fmaxf(hi.z, p.z));
        }
        if (!have) { lo = f3(0.f, 0.f, 0.f); hi = lo; }
        v.gbb_c[g] = make_float4(0.5f * (lo.x + hi.x), 0.5f * (lo.y + hi.y), 0.5f * (lo.z + hi.z), 0.f);
        v.gbb_h[g] = make_float4(0.5f * (hi.x - lo.x), 0.5f * (hi.y - lo.y), 0.5f * (hi.z - lo.z), 0.f);
    }
}

// j-cluster tile of every group: clusters within the water list radius of
// the group box, ascending (one warp per group, ballot compaction).  The
// molecule lists are half lists (a pair belongs to its lower slot), so only
// clusters from the group's own first cluster on can hold a partner.
DYN_KERNEL(, k_tile_list, (, bool force), (, force)) {
    if (!rebuild_on(v, force)) return;
    const BoxDev b = *v.box;
    const int lane = threadIdx.x & 31;
    const uint32_t nwc = v.sc->n_wclus;
    const uint32_t ng = (nwc + GRPW / WCL - 1) / (GRPW / WCL);
    const uint32_t g = (bk.idx * blockDim.x + threadIdx.x) >> 5;
    if (g >= ng) return;
    const float4 c0 = v.gbb_c[g], h0 = v.gbb_h[g];
    const float r2 = v.r_ww * v.r_ww;
    const uint32_t c_first = g * (GRPW / WCL);
    uint32_t cnt = 0;
    for (uint32_t jb = c_first & ~31u; jb < nwc; jb += 32) {
        const uint32_t cj = jb + lane;
        const bool hit = cj < nwc && cj >= c_first && bb_dist2(c0, h0, v.wbb_c[cj], v.wbb_h[cj], b) < r2;
        const uint32_t m = __ballot_sync(0xffffffffu, hit);
        if (hit) {
            const uint32_t k = cnt + __popc(m & ((1u << lane) - 1u));
            if (k < v.cap_tile) v.tile_j[(size_t)g * v.cap_tile + k] = cj;
        }
        cnt += __popc(m);
    }
    if (lane == 0) {
        v.tile_n[g] = min(cnt, v.cap_tile);
        if (cnt > v.cap_tile) atomicMax(&v.sc->overflow, cnt);
    }
}

// Union of the waters an i-group needs, as runs of consecutive slots, and
// per i-water lists of indices into that union.  One CTA (256 threads) per
// group.  Pass 1 marks every candidate water (waters of the group's tile
// clusters, ascending slot order) that lies within the list radius of any
// group member and numbers the marked ones with a block-wide scan; run
// starts (a marked water whose predecessor is unmarked or not the previous
// slot) get a run record.  Pass 2: 8 lanes per i-water test 8 consecutive
// candidates at a time and compact hits with a ballot, so every list is in
// ascending order.  Everything is deterministic.
constexpr int UT = 256;

DYN_KERNEL(__launch_bounds__(UT), k_group_union, (, bool force), (, force)) {
    if (!rebuild_on(v, force)) return;
    const BoxDev b = *v.box;
    const float r2 = v.r_ww * v.r_ww;
    const uint32_t nwc = v.sc->n_wclus;
    const uint32_t ng = (nwc + GRPW / WCL - 1) / (GRPW / WCL);
    const int tid = threadIdx.x, lane = tid & 31, wid_ = tid >> 5;
    __shared__ float4 io[GRPW];
    __shared__ uint32_t wn[UT / 32], wr[UT / 32];
    __shared__ uint8_t sh_need[UT];
    __shared__ uint32_t sh_slot[UT];
    __shared__ uint32_t base_cnt, base_run, carry_slot;
    __shared__ uint8_t carry_need;
    for (uint32_t g = bk.idx; g < ng; g += bk.cnt) {
        if (tid < GRPW) {
            const uint32_t s = g * GRPW + tid;
            const bool ok = s < v.nw_cap && v.wid[s] != INVALID_ID;
            const float4 p = ok ? v.wpos[4 * s] : make_float4(0.f, 0.f, 0.f, 0.f);
            io[tid] = make_float4(p.x, p.y, p.z, ok ? 1.f : 0.f);
        }
        if (tid == 0) { base_cnt = 0; base_run = 0; carry_need = 0; carry_slot = INVALID_ID; }
        __syncthreads();
        const uint32_t nt = v.tile_n[g];
        const uint32_t ncand = nt * WCL;
        const uint32_t* tl = v.tile_j + (size_t)g * v.cap_tile;
        uint16_t* cl = v.cand_loc + (size_t)g * v.cap_tile * WCL;
        for (uint32_t c0 = 0; c0 < ncand; c0 += UT) {
            const uint32_t k = c0 + tid;
            bool need = false;
            uint32_t slot = INVALID_ID;
            if (k < ncand) {
                slot = tl[k / WCL] * WCL + (k % WCL);
                if (v.wid[slot] != INVALID_ID) {
                    const float3 o = xyz(v.wpos[4 * slot]);
                    // members below the candidate's slot (half lists)
                    const int ilim = slot > g * GRPW ? (int)min(slot - g * GRPW, (uint32_t)GRPW) : 0;
                    for (int i = 0; i < ilim && !need; ++i) {
                        const float4 q = io[i];
                        if (q.w == 0.f) continue;
                        const float3 d = min_image_rint(o - xyz(q), b);
                        need = dot3(d, d) < r2;
                    }
                }
            }
            sh_need[tid] = need;
            sh_slot[tid] = slot;
            __syncthreads();
            const bool pn = tid ? sh_need[tid - 1] != 0 : carry_need != 0;
            const uint32_t ps = tid ? sh_slot[tid - 1] : carry_slot;
            const bool start = need && (!pn || slot != ps + 1u);
            const uint32_t mn = __ballot_sync(0xffffffffu, need), ms = __ballot_sync(0xffffffffu, start);
            if (lane == 0) { wn[wid_] = __popc(mn); wr[wid_] = __popc(ms); }
            __syncthreads();
            uint32_t on = 0, os = 0;
            for (int w = 0; w < wid_; ++w) { on += wn[w]; os += wr[w]; }
            const uint32_t lm = (1u << lane) - 1u;
            const uint32_t loc = base_cnt + on + __popc(mn & lm);
            const uint32_t rid = base_run + os + __popc(ms & lm);
            if (k < ncand) cl[k] = need && loc < v.cap_union ? (uint16_t)loc : (uint16_t)0xFFFFu;
            if (need && loc < v.cap_union) {
                v.grp_uslot[(size_t)g * v.cap_union + loc] = slot;
            }
            if (start && rid < v.cap_run) v.grp_run[(size_t)g * v.cap_run + rid] = make_uint2(slot, loc);
            __syncthreads();
            if (tid == 0) {
                uint32_t tn = 0, ts = 0;
                for (int w = 0; w < UT / 32; ++w) { tn += wn[w]; ts += wr[w]; }
                base_cnt += tn; base_run += ts;
                carry_need = sh_need[UT - 1]; carry_slot = sh_slot[UT - 1];
            }
            __syncthreads();
        }
        if (tid == 0) {
            v.grp_nloc[g] = min(base_cnt, v.cap_union);
            v.grp_nrun[g] = min(base_run, v.cap_run);
            if (base_cnt > v.cap_union) atomicMax(&v.sc->overflow, base_cnt);
            atomicMax(&v.sc->union_max, base_cnt);
            if (base_run > v.cap_run) atomicMax(&v.sc->overflow, base_run);
        }
        __syncthreads();
        // pass 2: per i-water lists, LPW lanes per i-water
        const int il = tid / LPW, l = tid % LPW;
        const uint32_t si = g * GRPW + il;
        const float4 qi = io[il];
        const unsigned gmask = ((1u << LPW) - 1u) << ((lane / LPW) * LPW);
        uint32_t cnt = 0;
        uint16_t* out = v.wnb + (size_t)si * v.cap_nb;
        for (uint32_t c0 = 0; c0 < ncand; c0 += LPW) {
            const uint32_t k = c0 + l;
            bool hit = false;
            uint16_t loc = 0xFFFFu;
            if (k < ncand && qi.w != 0.f) {
                loc = cl[k];
                const uint32_t slot = tl[k / WCL] * WCL + (k % WCL);
                if (loc != 0xFFFFu && slot > si) {
                    const float3 d = min_image_rint(xyz(qi) - xyz(v.wpos[4 * slot]), b);
                    hit = dot3(d, d) < r2;
                }
            }
            const uint32_t m = __ballot_sync(0xffffffffu, hit) & gmask;
            if (hit) {
                const uint32_t pos = cnt + __popc(m & ((1u << lane) - 1u));
                if (pos < v.cap_nb) out[pos] = loc;
            }
            cnt += __popc(m);
        }
        if (l == 0 && si < v.nw_cap) {
            v.wnb_n[si] = qi.w != 0.f ? min(cnt, v.cap_nb) : 0u;
            if (cnt > v.cap_nb) atomicMax(&v.sc->overflow, cnt);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Pruning of the water-water lists (a dual pair list: Pall, Zhmurov,
// Bauer, Abraham, Lundborg, Gray, Hess, Lindahl, J. Chem. Phys. 153, 134110
// (2020)).  The rebuild's lists hold the molecule pairs with an O-O distance
// below r_ww = cutoff + 2 reach + buffer; the kernel walks these pruned to
// r_in = cutoff + 2 reach + prune buffer, which stay complete until some
// water has moved half the prune buffer since the prune.  One CTA per group:
// the union's O positions are staged in shared memory (PR_CHUNK at a time)
// and LPW lanes per water test its list entries in order, compacting the
// hits with ballots over the water's lanes (the pruned lists stay
// ascending).  The group's O positions are recorded for the next check.
// ---------------------------------------------------------------------------
constexpr int PRT = GRPW * LPW;
constexpr uint32_t PR_CHUNK = 1024;

DYN_KERNEL(__launch_bounds__(PRT), k_ww_prune, (, bool force), (, force)) {
    if (!(force || v.sc->need_prune)) return;
    __shared__ float4 uo[PR_CHUNK];
    const BoxDev b = *v.box;
    const float r2 = v.r_in * v.r_in;
    const uint32_t ng = (v.sc->n_wclus + GRPW / WCL - 1) / (GRPW / WCL);
    const int tid = threadIdx.x, lane = tid & 31;
    const int il = tid / LPW, l = tid % LPW;
    const unsigned gmask = ((1u << LPW) - 1u) << ((lane / LPW) * LPW);
    for (uint32_t g = bk.idx; g < ng; g += bk.cnt) {
        const uint32_t nloc = v.grp_nloc[g];
        const uint32_t s = g * GRPW + il;
        const bool valid = s < v.nw_cap && v.wid[s] != INVALID_ID;
        const float3 io = valid ? xyz(v.wpos[4 * s]) : f3(0.f, 0.f, 0.f);
        const uint32_t n = valid ? v.wnb_n[s] : 0u;
        const uint16_t* in = v.wnb + (size_t)s * v.cap_nb;
        uint16_t* out = v.winb + (size_t)s * v.cap_nb;
        uint32_t cnt = 0, k0 = 0;
        for (uint32_t lo = 0; lo < nloc; lo += PR_CHUNK) {
            const uint32_t hi = min(nloc, lo + PR_CHUNK);
            for (uint32_t t = tid; t < hi - lo; t += PRT)
                uo[t] = v.wpos[4 * (size_t)v.grp_uslot[(size_t)g * v.cap_union + lo + t]];
            __syncthreads();
            // this water's entries in [lo, hi): a prefix of what is left
            for (;;) {
                const uint32_t k = k0 + (uint32_t)l;
                const uint32_t idx = k < n ? (uint32_t)in[k] : 0xFFFFFFFFu;
                const bool here = idx < hi;
                bool hit = false;
                if (here) {
                    const float3 d = min_image_rint(io - xyz(uo[idx - lo]), b);
                    hit = dot3(d, d) < r2;
                }
                const uint32_t mh = __ballot_sync(gmask, hit) & gmask;
                if (hit) out[cnt + __popc(mh & ((1u << lane) - 1u))] = (uint16_t)idx;
                cnt += __popc(mh);
                const uint32_t adv = __popc(__ballot_sync(gmask, here) & gmask);
                k0 += adv;
                if (adv < (uint32_t)LPW) break;
            }
            __syncthreads();
        }
        if (l == 0 && s < v.nw_cap) v.winb_n[s] = valid ? cnt : 0u;
        if (tid < GRPW && g * GRPW + tid < v.nw_cap) v.wprune[g * GRPW + tid] = v.wpos[4 * (g * GRPW + tid)];
    }
}

DYN_KERNEL(, k_prune_done, (, bool force), (, force)) {
    if (!(force || v.sc->need_prune)) return;
    v.sc->need_prune = 0u;
    v.sc->prunes += 1ull;
}

DYN_KERNEL(, k_rebuild_done, (, bool force), (, force)) {
    if (!rebuild_on(v, force)) return;
    v.sc->need_rebuild = 0u;
    v.sc->rebuilds += 1ull;
}

// Copies positions into cluster order and zeroes the atoms' and the
// waters' short-range force accumulators (every pair kernel adds to them).
DYN_KERNEL(, k_gather_atoms, (), ()) {
    const uint32_t t0 = bk.idx * blockDim.x + threadIdx.x, stride = bk.cnt * blockDim.x;
    for (uint32_t s = t0; s < v.na_cap; s += stride) {
        const uint32_t a = v.sidx[s];
        if (a != INVALID_ID) {
            v.spos[s] = v.apos[a];
            v.aforce[3 * (size_t)a + 0] = 0; v.aforce[3 * (size_t)a + 1] = 0; v.aforce[3 * (size_t)a + 2] = 0;
        }
    }
    int4* wf = reinterpret_cast<int4*>(v.wforce);  // 12 int64 = 6 int4 per slot
    for (uint32_t t = t0; t < 6 * v.nw_cap; t += stride) wf[t] = make_int4(0, 0, 0, 0);
}

inline int nblocks(uint64_t n, int threads, int cap = 148 * 8) {
    uint64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    return (int)(b < (uint64_t)cap ? b : cap);
}

}  // namespace

namespace dyn {

void launch_displacement_check(const Target& t) {
    t.launch(k_disp_check, k_disp_check_batch, [](const SysView& v) { return nblocks(v.nw_cap + v.na, 256); },
             256, 0);
}

void launch_rebuild(const Target& t, bool force) {
    const int T = 256;
    auto nmax = [](const SysView& v) { return v.nw_cap > v.na_cap ? v.nw_cap : v.na_cap; };
    t.launch(k_col_clear, k_col_clear_batch,
             [](const SysView& v) { return nblocks((v.ncol > v.ancol ? v.ncol : v.ancol) + 1, 256); }, T, 0, force);
    t.launch(k_col_assign, k_col_assign_batch, [&](const SysView& v) { return nblocks(nmax(v), 256); }, T, 0, force);
    t.launch(k_col_scan, k_col_scan_batch, [](const SysView&) { return 1; }, 64, 0, force);
    t.launch(k_col_bucket, k_col_bucket_batch, [&](const SysView& v) { return nblocks(nmax(v), 256); }, T, 0, force);
    t.launch(k_col_rank, k_col_rank_batch, [&](const SysView& v) { return nblocks(nmax(v), 256); }, T, 0, force);
    t.launch(k_perm_init, k_perm_init_batch, [&](const SysView& v) { return nblocks(nmax(v), 256); }, T, 0, force);
    t.launch(k_perm_scatter, k_perm_scatter_batch, [&](const SysView& v) { return nblocks(nmax(v), 256); }, T, 0,
             force);
    t.launch(k_perm_copyback, k_perm_copyback_batch, [](const SysView& v) { return nblocks(v.nw_cap, 256); }, T, 0,
             force);
    t.launch(k_bbox, k_bbox_batch, [](const SysView& v) { return nblocks(v.nwclus_cap + v.naclus_cap, 256); }, T, 0,
             force);
    const int LT = 128;  // 4 warps per block, one i-cluster per warp
    t.launch(k_group_bbox, k_group_bbox_batch, [](const SysView& v) { return v.nw ? nblocks(v.ngrp_cap, 256) : 0; },
             T, 0, force);
    t.launch(k_tile_list, k_tile_list_batch,
             [](const SysView& v) { return v.nw ? nblocks((uint64_t)v.ngrp_cap * 32, 128, 1 << 30) : 0; }, LT, 0,
             force);
    t.launch(k_group_union, k_group_union_batch,
             [](const SysView& v) { return v.nw ? (int)std::min<uint32_t>(v.ngrp_cap, 148 * 8) : 0; }, UT, 0, force);
    t.launch(k_list<1>, k_list_batch<1>,
             [](const SysView& v) { return v.nw && v.na ? nblocks((uint64_t)v.nwclus_cap * 32, 128, 1 << 30) : 0; },
             LT, 0, force);
    t.launch(k_list<3>, k_list_batch<3>,
             [](const SysView& v) { return v.na ? nblocks((uint64_t)v.naclus_cap * 32, 128, 1 << 30) : 0; }, LT, 0,
             force);
    t.launch(k_items<1>, k_items_batch<1>, [](const SysView& v) { return v.nw && v.na ? 1 : 0; }, IT_T, 0, force);
    t.launch(k_items<3>, k_items_batch<3>, [](const SysView& v) { return v.na ? 1 : 0; }, IT_T, 0, force);
    t.launch(k_rebuild_done, k_rebuild_done_batch, [](const SysView&) { return 1; }, 1, 0, force);
}

void launch_prune(const Target& t, bool force) {
    t.launch(k_ww_prune, k_ww_prune_batch,
             [](const SysView& v) { return v.nw ? (int)std::min<uint32_t>(v.ngrp_cap, 148 * 8) : 0; }, PRT, 0, force);
    t.launch(k_prune_done, k_prune_done_batch, [](const SysView&) { return 1; }, 1, 0, force);
}

void launch_gather_atoms(const Target& t) {
    t.launch(k_gather_atoms, k_gather_atoms_batch,
             [](const SysView& v) { return nblocks(std::max<uint64_t>(v.na_cap, 6ull * v.nw_cap), 256); }, 256, 0);
}

}  // namespace dyn
