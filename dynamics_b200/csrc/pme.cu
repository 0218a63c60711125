// Smooth PME on the device: spread -> cuFFT R2C -> fused convolution (energy
// and virial in float64) -> cuFFT C2R -> gather.
//
// The reference hands wrapped positions and charges to the external crate
// ``ewald`` (src/non_bonded.rs:681-846); this is the published method
// (Essmann et al. 1995, order-4 cardinal B-splines) on the same grid.
// Determinism: charges are spread as 64-bit fixed point (2^-32 e-units), so
// the grid, and everything downstream, is bit-identical run to run.
// Reciprocal forces (plus the exclusion corrections) are written to a cache
// indexed by original particle id and added by the kick kernels on every
// step, which implements the reference's SPME-every-n-steps reuse
// (src/lib.rs:1282-1341).
#include <algorithm>
#include <cmath>
#include <vector>

#include "engine.cuh"

namespace {

constexpr int GT = 256;

__device__ __forceinline__ void bspline4(float w, float* th, float* dth) {
    const float w2 = w * w, w3 = w2 * w, om = 1.0f - w;
    th[0] = om * om * om * (1.0f / 6.0f);
    th[1] = (3.0f * w3 - 6.0f * w2 + 4.0f) * (1.0f / 6.0f);
    th[2] = (-3.0f * w3 + 3.0f * w2 + 3.0f * w + 1.0f) * (1.0f / 6.0f);
    th[3] = w3 * (1.0f / 6.0f);
    if (dth) {
        dth[0] = -0.5f * om * om;
        dth[1] = 1.5f * w2 - 2.0f * w;
        dth[2] = -1.5f * w2 + w + 0.5f;
        dth[3] = 0.5f * w2;
    }
}

// grid coordinate of a position: u = K * frac((x - lo) / L), in float64 (a
// float32 u near K = 96 is only good to ~4e-6 grid units, which would put
// relative errors of 1e-6 into the B-spline weights); base[a] = floor(u),
// w[a] = u - floor(u)
__device__ __forceinline__ void grid_coord(float3 p, const BoxDev& b, const uint32_t* K, int* base,
                                           double* w) {
    const float c[3] = {p.x, p.y, p.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        double f = ((double)c[a] - (double)b.lo[a]) / (double)b.ext[a];
        f -= floor(f);
        const double u = f * (double)K[a];
        int i = (int)floor(u);
        const double ww = u - (double)i;
        if (i >= (int)K[a]) { i -= K[a]; }
        if (i < 0) { i += K[a]; }
        base[a] = i;
        w[a] = ww;
    }
}

__device__ __forceinline__ void bspline4d(double w, double* th) {
    const double w2 = w * w, w3 = w2 * w, om = 1.0 - w;
    th[0] = om * om * om * (1.0 / 6.0);
    th[1] = (3.0 * w3 - 6.0 * w2 + 4.0) * (1.0 / 6.0);
    th[2] = (-3.0 * w3 + 3.0 * w2 + 3.0 * w + 1.0) * (1.0 / 6.0);
    th[3] = w3 * (1.0 / 6.0);
}

// Which charges an SPME pass spreads and gathers: pass 0 all of them;
// with an alchemical molecule, pass 1 all but the molecule's (the
// environment) and pass 2 the molecule's only (src/non_bonded.rs:709-743).
__device__ __forceinline__ bool pass_has_atom(const SysView& v, int pass, uint32_t a) {
    if (pass == 0) return true;
    const bool in = a >= v.alch_lo && a < v.alch_hi;
    return pass == 1 ? !in : in;
}
// weight of a pass in the mixed forces / energies: lambda-scaled full
// evaluation plus the unscaled environment and molecule evaluations
__device__ __forceinline__ float pass_weight(const SysView& v, int pass) {
    if (!v.alch_on) return 1.0f;
    return pass == 0 ? v.alch_cs : 1.0f - v.alch_cs;
}

// ---------------------------------------------------------------------------
// Spread and gather by grid bricks.
//
// Every SPME pass first bins the charged sites (water H0, H1, M and the
// charged atoms) by the PME_BRICK^3 brick that holds their stencil base,
// one record each (fractional grid coordinates, charge, base).  A site with
// base b covers grid points b-3 .. b in each dimension, so the points of a
// brick receive charge only from sites based in it or in the next bricks
// up (up to 3 points on).  The spread gives each brick to one CTA, which
// adds those sites' stencils in shared memory, exactly, and writes its
// points once, converted to float: no global atomics and no separate
// conversion pass.  The gather stages a brick with its 3-point halo and
// evaluates its own sites' stencils from shared memory.  Sites beyond a
// brick's capacity (rare: a capacity of about twice the mean) go to an
// overflow list, spread with global fixed-point atomics that the brick's
// CTA folds in, and gathered from the global grid, with the same values.
// ---------------------------------------------------------------------------
constexpr int SB_T = 256;                               // spread: threads per CTA
constexpr int GB_T = 128;                               // gather: threads per CTA
constexpr int BR3 = PME_BRICK * PME_BRICK * PME_BRICK;
constexpr int HB = PME_BRICK + 3;                       // gather tile edge (brick + halo)
constexpr int OVF_BLOCKS = 8;                           // gather CTAs for the overflow list

__device__ __forceinline__ void rec_base(uint32_t b, int* base) {
    base[0] = (int)(b & 1023u);
    base[1] = (int)((b >> 10) & 1023u);
    base[2] = (int)(b >> 20);
}

__device__ __forceinline__ SiteRec make_rec(float3 p, float q, const BoxDev& b, const uint32_t* K) {
    int base[3];
    double w[3];
    grid_coord(p, b, K, base, w);
    SiteRec r;
    r.w[0] = w[0]; r.w[1] = w[1]; r.w[2] = w[2];
    r.q = q;
    r.base = (uint32_t)base[0] | ((uint32_t)base[1] << 10) | ((uint32_t)base[2] << 20);
    return r;
}

__device__ __forceinline__ uint32_t brick_index(const SysView& v, int x, int y, int z) {
    return ((uint32_t)(x / PME_BRICK) * v.nbrick[1] + (uint32_t)(y / PME_BRICK)) * v.nbrick[2] +
           (uint32_t)(z / PME_BRICK);
}

__device__ __forceinline__ void brick_origin(const SysView& v, uint32_t P, int* o, int* ext) {
    const uint32_t nb1 = v.nbrick[1], nb2 = v.nbrick[2];
    const uint32_t p[3] = {P / (nb1 * nb2), (P / nb2) % nb1, P % nb2};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        o[a] = (int)p[a] * PME_BRICK;
        ext[a] = min(PME_BRICK, (int)v.K[a] - o[a]);
    }
}

// An overflow site: its contributions go to the global fixed-point grid
// (float64 weights and products, the values the brick path adds), and the
// bricks they land in are flagged for their spread CTAs to fold in.
__device__ void spread_global(const SysView& v, const SiteRec& r) {
    int base[3];
    rec_base(r.base, base);
    double tx[4], ty[4], tz[4];
    bspline4d(r.w[0], tx);
    bspline4d(r.w[1], ty);
    bspline4d(r.w[2], tz);
    const int K0 = v.K[0], K1 = v.K[1], K2 = v.K[2];
    int iz[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) { int z = base[2] - 3 + c; iz[c] = z < 0 ? z + K2 : z; }
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        int x = base[0] - 3 + a; x = x < 0 ? x + K0 : x;
        const double qa = (double)r.q * tx[a];
#pragma unroll
        for (int bb = 0; bb < 4; ++bb) {
            int y = base[1] - 3 + bb; y = y < 0 ? y + K1 : y;
            const double qab = qa * ty[bb];
            long long* row = v.qgrid_fix + ((size_t)x * K1 + y) * K2;
#pragma unroll
            for (int c = 0; c < 4; ++c) fix_atomic_add(row + iz[c], fix_from_double(qab * tz[c]));
        }
    }
    // flag every brick that holds a stencil point: per axis the distinct
    // bricks of the 4 points (3 where the last brick is 1 or 2 points wide)
    int bl[3][4], nbl[3];
    for (int a = 0; a < 3; ++a) {
        nbl[a] = 0;
        for (int c = 0; c < 4; ++c) {
            int x = base[a] - 3 + c;
            if (x < 0) x += (int)v.K[a];
            const int q = x / PME_BRICK;
            bool seen = false;
            for (int t = 0; t < nbl[a]; ++t) seen = seen || bl[a][t] == q;
            if (!seen) bl[a][nbl[a]++] = q;
        }
    }
    for (int i = 0; i < nbl[0]; ++i)
        for (int j = 0; j < nbl[1]; ++j)
            for (int k = 0; k < nbl[2]; ++k)
                v.brick_ovf[((uint32_t)bl[0][i] * v.nbrick[1] + (uint32_t)bl[1][j]) * v.nbrick[2] + (uint32_t)bl[2][k]] =
                    1u;
}

// Bins the pass's charged sites by brick (records and site codes).  Atoms
// without charge get a zero reciprocal force on pass 0, as they have none.
// Neighbouring sites (cluster order) mostly share a brick: the lanes of a
// warp with the same brick take their slots with one atomic.
DYN_KERNEL(, k_bin_sites, (, int pass), (, pass)) {
    const BoxDev b = *v.box;
    const uint32_t nws = pass == 2 ? 0u : 3u * v.nw_cap;  // the molecule's own pass holds no water
    const uint32_t total = nws + v.na;
    const int lane = threadIdx.x & 31;
    const uint32_t wstride = bk.cnt * blockDim.x;
    for (uint32_t t0 = bk.idx * blockDim.x + (threadIdx.x & ~31u); t0 < total; t0 += wstride) {
        const uint32_t t = t0 + lane;
        bool has = false;
        float4 p = make_float4(0.f, 0.f, 0.f, 0.f);
        uint32_t sid = 0;
        if (t < total) {
            if (t < nws) {
                const uint32_t s = t / 3u, k = t % 3u;
                const uint32_t id = v.wid[s];
                if (id != INVALID_ID) {
                    p = v.wpos[4 * s + 1 + k];
                    sid = DYN_SITE_WATER | (3u * id + k);
                    has = true;
                }
            } else {
                const uint32_t a = t - nws;
                if (pass_has_atom(v, pass, a)) {
                    p = v.apos[a];
                    if (p.w != 0.f) {
                        sid = a;
                        has = true;
                    } else if (pass == 0) {
                        long long* c = v.arecip + 3 * (size_t)a;
                        c[0] = 0; c[1] = 0; c[2] = 0;
                    }
                }
            }
        }
        SiteRec r;
        uint32_t P = INVALID_ID;
        if (has) {
            r = make_rec(xyz(p), p.w, b, v.K);
            int base[3];
            rec_base(r.base, base);
            P = brick_index(v, base[0], base[1], base[2]);
        }
        const uint32_t peers = __match_any_sync(0xffffffffu, P);
        const int leader = __ffs(peers) - 1;
        uint32_t first = 0;
        if (has && lane == leader) first = atomicAdd(&v.brick_n[P], (uint32_t)__popc(peers));
        first = __shfl_sync(0xffffffffu, first, leader);
        if (!has) continue;
        const uint32_t slot = first + __popc(peers & ((1u << lane) - 1u));
        if (slot < v.brick_cap) {
            v.brick_site[(size_t)P * v.brick_cap + slot] = r;
            v.brick_sid[(size_t)P * v.brick_cap + slot] = sid;
        } else {
            const uint32_t o = atomicAdd(&v.sc->spme_ovf, 1u);  // < n_sites_max: one entry per site
            v.ovf_site[o] = r;
            v.ovf_sid[o] = sid;
            spread_global(v, r);
        }
    }
}

// Phase 1 of the spread: one CTA per brick, its own sites' whole stencils
// into an 11^3 tile (the brick and the 3 grid points below it in each
// dimension: a site with base b covers b-3 .. b, so every contribution
// lands in its own brick's tile, with no bounds checks and no neighbour
// reads).  A half-warp takes a site, a lane per (x, y) column of its
// stencil adding the column's 4 contributions (the per-site path's values:
// q tx, times ty, times tz, in FP64, to fixed point); the two halves of a
// warp take sites half the list apart.  Each int64 contribution f is added
// in shared memory as two native 32-bit atomics, f >> 18 and its low 18
// bits, whose sums give the int64 sum exactly (a tile point gets at most
// brick_cap <= 512 contributions of magnitude below 2^37); the tile is
// written out as int64.
constexpr int SPLIT = 18;
constexpr int HB3 = HB * HB * HB;

DYN_KERNEL(__launch_bounds__(SB_T), k_spread_brick, (, int pass), (, pass)) {
    __shared__ int acc_hi[HB3], acc_lo[HB3];
    __shared__ double wts[SB_T][12];   // tx[4], ty[4], tz[4] of each staged site
    __shared__ int4 sloc[SB_T];        // tile position of each staged site's stencil, (base - o) per axis
    __shared__ float sq[SB_T];
    const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
    const int half = lane >> 4, a = (lane >> 2) & 3, bb = lane & 3;
    for (uint32_t P = bk.idx; P < v.n_bricks; P += bk.cnt) {
        int o[3], ext[3];
        brick_origin(v, P, o, ext);
        for (int i = tid; i < HB3; i += SB_T) { acc_hi[i] = 0; acc_lo[i] = 0; }
        const uint32_t n = min(v.brick_n[P], v.brick_cap);
        for (uint32_t u0 = 0; u0 < n; u0 += SB_T) {
            if (u0 + tid < n) {
                const SiteRec r = v.brick_site[(size_t)P * v.brick_cap + u0 + tid];
                int base[3];
                rec_base(r.base, base);
                sloc[tid] = make_int4(base[0] - o[0], base[1] - o[1], base[2] - o[2], 0);
                sq[tid] = r.q;
                bspline4d(r.w[0], &wts[tid][0]);
                bspline4d(r.w[1], &wts[tid][4]);
                bspline4d(r.w[2], &wts[tid][8]);
            }
            __syncthreads();  // the staged sites (and, first, the zeroed tile)
            const uint32_t m = min((uint32_t)SB_T, n - u0), hn = (m + 1) / 2;
            for (uint32_t k0 = (uint32_t)wp; k0 < hn; k0 += SB_T / 32) {
                const uint32_t k = k0 + (half ? hn : 0u);
                if (k >= m) continue;
                const int4 lb = sloc[k];
                const double qab = ((double)sq[k] * wts[k][a]) * wts[k][4 + bb];
                const int row = ((lb.x + a) * HB + (lb.y + bb)) * HB + lb.z;
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const long long f = fix_from_double(qab * wts[k][8 + c]);
                    atomicAdd(&acc_hi[row + c], (int)(f >> SPLIT));
                    atomicAdd(&acc_lo[row + c], (int)(f & ((1ll << SPLIT) - 1)));
                }
            }
            __syncthreads();  // the staged sites are refilled by the next round
        }
        long long* tile = v.brick_tile + (size_t)P * HB3;
        for (int i = tid; i < HB3; i += SB_T) tile[i] = (long long)acc_hi[i] * (1ll << SPLIT) + (long long)acc_lo[i];
        __syncthreads();  // the tile is zeroed for the next brick
    }
}

// The (brick, tile offset) pairs whose tiles hold grid coordinate x of one
// axis: its own brick and the 1 or 2 bricks that start at most 3 points on
// (tile offset t of brick b is point o_b - 3 + t, periodic); with K < 11 a
// tile can hold a point twice.  Six fixed slots, (brick b0 + k, offset
// d + r K) for k < 3, r < 2; d[] = HB marks an empty slot.  Static indices
// only, so the slots stay in registers.
__device__ __forceinline__ void tile_holders(int x, int K, uint32_t nb, int (&hb)[6], int (&hd)[6]) {
    const int b0 = x / PME_BRICK;
    int bs[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) bs[k] = (int)(((uint32_t)b0 + (uint32_t)k) % nb);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const bool dup = (k >= 1 && bs[k] == bs[0]) || (k == 2 && bs[2] == bs[1]);
        const int d = ((x - bs[k] * PME_BRICK + 3) % K + K) % K;
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            hb[2 * k + r] = bs[k];
            hd[2 * k + r] = (!dup && d + r * K < HB) ? d + r * K : HB;
        }
    }
}

// The common case of tile_holders (every axis with K >= 11 and K mod 8 not
// 1 or 2, so no brick is narrower than 3 points and no tile wraps onto
// itself): the own brick (offset in [3, 11)) and the next brick, whose
// halo holds x when its offset d1 = x - (next origin) + 3 is >= 0.
__device__ __forceinline__ void tile_holders2(int x, int K, uint32_t nb, int& b0, int& d0, int& b1, int& d1) {
    b0 = x / PME_BRICK;
    d0 = x - b0 * PME_BRICK + 3;
    const bool last = b0 + 1 == (int)nb;
    b1 = last ? 0 : b0 + 1;
    d1 = x - (last ? K : (b0 + 1) * PME_BRICK) + 3;
}

__device__ __forceinline__ bool axis_simple(int K) { return K >= HB && (K % PME_BRICK == 0 || K % PME_BRICK >= 3); }

// Phase 2 for grids where every axis is simple: one CTA per brick, a thread
// per point; a point at local coordinate l of an axis is held by its own
// tile (offset l + 3) and, in the top 3 layers (l >= ext - 3), by the next
// brick's tile (offset l - ext + 3), exactly the entries phase 1 writes.
DYN_KERNEL(__launch_bounds__(SB_T), k_spread_merge_brick, (, int pass), (, pass)) {
    const int K[3] = {(int)v.K[0], (int)v.K[1], (int)v.K[2]};
    for (uint32_t P = bk.idx; P < v.n_bricks; P += bk.cnt) {
        int o[3], ext[3];
        brick_origin(v, P, o, ext);
        int bi[3][2];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const int pb = o[a] / PME_BRICK;
            bi[a][0] = pb;
            bi[a][1] = pb + 1 == (int)v.nbrick[a] ? 0 : pb + 1;
        }
        const bool fold = v.brick_ovf[P] != 0u;
        for (int i = threadIdx.x; i < BR3; i += SB_T) {
            const int l[3] = {i / (PME_BRICK * PME_BRICK), (i / PME_BRICK) % PME_BRICK, i % PME_BRICK};
            if (l[0] >= ext[0] || l[1] >= ext[1] || l[2] >= ext[2]) continue;
            int d[3][2];
#pragma unroll
            for (int a = 0; a < 3; ++a) { d[a][0] = l[a] + 3; d[a][1] = l[a] - ext[a] + 3; }
            long long sum = 0;
#pragma unroll
            for (int x = 0; x < 2; ++x) {
                if (d[0][x] < 0) continue;
#pragma unroll
                for (int y = 0; y < 2; ++y) {
                    if (d[1][y] < 0) continue;
                    const size_t bxy = ((size_t)bi[0][x] * v.nbrick[1] + bi[1][y]) * v.nbrick[2];
                    const int dxy = (d[0][x] * HB + d[1][y]) * HB;
#pragma unroll
                    for (int z = 0; z < 2; ++z)
                        if (d[2][z] >= 0) sum += v.brick_tile[(bxy + bi[2][z]) * HB3 + dxy + d[2][z]];
                }
            }
            const size_t gi = ((size_t)(o[0] + l[0]) * K[1] + (o[1] + l[1])) * K[2] + (o[2] + l[2]);
            if (fold) {
                // overflow sites' charge from the global fixed-point grid
                sum += v.qgrid_fix[gi];
                v.qgrid_fix[gi] = 0;
            }
            v.qgrid[gi] = (float)((double)sum * DYN_FIX_INV);
        }
    }
}

// Phase 2 for any grid: one thread per grid point, the sum of the tile
// entries that hold it (plus the overflow sites' charge where its brick is
// flagged), as float.
DYN_KERNEL(, k_spread_merge, (, int pass), (, pass)) {
    const int K0 = v.K[0], K1 = v.K[1], K2 = v.K[2];
    const uint32_t npts = (uint32_t)K0 * K1 * K2;
    const bool simple = axis_simple(K0) && axis_simple(K1) && axis_simple(K2);
    for (uint32_t p = bk.idx * blockDim.x + threadIdx.x; p < npts; p += bk.cnt * blockDim.x) {
        const int z = (int)(p % (uint32_t)K2), y = (int)((p / (uint32_t)K2) % (uint32_t)K1),
                  x = (int)(p / ((uint32_t)K1 * K2));
        if (simple) {
            int bx[2], dx[2], by[2], dy[2], bz[2], dz[2];
            tile_holders2(x, K0, v.nbrick[0], bx[0], dx[0], bx[1], dx[1]);
            tile_holders2(y, K1, v.nbrick[1], by[0], dy[0], by[1], dy[1]);
            tile_holders2(z, K2, v.nbrick[2], bz[0], dz[0], bz[1], dz[1]);
            long long sum = 0;
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                if (dx[i] < 0) continue;
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    if (dy[j] < 0) continue;
                    const size_t bxy = ((size_t)bx[i] * v.nbrick[1] + by[j]) * v.nbrick[2];
                    const int dxy = (dx[i] * HB + dy[j]) * HB;
#pragma unroll
                    for (int k = 0; k < 2; ++k)
                        if (dz[k] >= 0) sum += v.brick_tile[(bxy + bz[k]) * HB3 + dxy + dz[k]];
                }
            }
            if (v.brick_ovf[brick_index(v, x, y, z)]) {
                sum += v.qgrid_fix[p];
                v.qgrid_fix[p] = 0;
            }
            v.qgrid[p] = (float)((double)sum * DYN_FIX_INV);
            continue;
        }
        int bx[6], dx[6], by[6], dy[6], bz[6], dz[6];
        tile_holders(x, K0, v.nbrick[0], bx, dx);
        tile_holders(y, K1, v.nbrick[1], by, dy);
        tile_holders(z, K2, v.nbrick[2], bz, dz);
        long long sum = 0;
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            if (dx[i] >= HB) continue;
#pragma unroll
            for (int j = 0; j < 6; ++j) {
                if (dy[j] >= HB) continue;
                const size_t bxy = ((size_t)bx[i] * v.nbrick[1] + by[j]) * v.nbrick[2];
                const int dxy = (dx[i] * HB + dy[j]) * HB;
#pragma unroll
                for (int k = 0; k < 6; ++k)
                    if (dz[k] < HB) sum += v.brick_tile[(bxy + bz[k]) * HB3 + dxy + dz[k]];
            }
        }
        if (v.brick_ovf[brick_index(v, x, y, z)]) {
            // overflow sites' charge from the global fixed-point grid
            sum += v.qgrid_fix[p];
            v.qgrid_fix[p] = 0;
        }
        v.qgrid[p] = (float)((double)sum * DYN_FIX_INV);
    }
}

// -q q erf(alpha r)/r between two sites, float64 from the exact float64
// displacement (dx, dy, dz); returns the energy and the force on the first
__device__ __forceinline__ double excl_corr(double dx, double dy, double dz, double qq, double alpha,
                                           double3* f) {
    const double r2 = dx * dx + dy * dy + dz * dz;
    const double r = sqrt(r2);
    const double ar = alpha * r;
    const double er = erf(ar);
    const double du = qq * (er / r2 - 2.0 * alpha * 0.5641895835477563 * exp(-ar * ar) / r);
    const double s = -du / r;
    f->x = s * dx; f->y = s * dy; f->z = s * dz;
    return -qq * er / r;
}

// Influence function B(m) C(m) applied in place; energy and virial of the
// reciprocal sum (Essmann eq. 2.10 and the trace of the k-space virial).
DYN_KERNEL(, k_convolve, (), ()) {
    const BoxDev b = *v.box;
    const int K0 = v.K[0], K1 = v.K[1], K2 = v.K[2];
    const int K2h = K2 / 2 + 1;
    const uint32_t n = (uint32_t)K0 * K1 * K2h;
    const float inv_vol = b.inv_ext[0] * b.inv_ext[1] * b.inv_ext[2];
    const float pa2 = (float)(M_PI * M_PI) / (v.alpha * v.alpha);
    const float pref = inv_vol * (float)(1.0 / M_PI);
    double e = 0.0, w = 0.0;
    for (uint32_t i = bk.idx * blockDim.x + threadIdx.x; i < n; i += bk.cnt * blockDim.x) {
        const int kz = i % K2h;
        const int ky = (i / K2h) % K1;
        const int kx = i / (K2h * K1);
        const int mx = kx <= K0 / 2 ? kx : kx - K0;
        const int my = ky <= K1 / 2 ? ky : ky - K1;
        const float fx = mx * b.inv_ext[0], fy = my * b.inv_ext[1], fz = kz * b.inv_ext[2];
        const float m2 = fx * fx + fy * fy + fz * fz;
        float2 c = v.cgrid[i];
        float g = 0.f;
        if (m2 > 0.f) {
            g = v.bmod[0][kx] * v.bmod[1][ky] * v.bmod[2][kz] * pref * __expf(-pa2 * m2) / m2;
            const double mult = (kz == 0 || (K2 % 2 == 0 && kz == K2 / 2)) ? 1.0 : 2.0;
            const double em = 0.5 * mult * (double)g * ((double)c.x * c.x + (double)c.y * c.y);
            e += em;
            w += em * (1.0 - 2.0 * (double)pa2 * m2);
        }
        c.x *= g; c.y *= g;
        v.cgrid[i] = c;
    }
    double x[2] = {e, w};
    block_sum_d<2>(x);
    if (threadIdx.x == 0) {
        double* p = v.partials + ((size_t)REG_PME * v.max_blocks + bk.idx) * 4;
        p[0] = x[0]; p[1] = x[1]; p[2] = 0.0; p[3] = 0.0;
    }
}


// The gather of one site, grid values from at(a, bb, c) (stencil point
// base - 3 + (a, bb, c)): float B-splines of the float64 fractional
// coordinates and this order of fused multiply-adds, from shared memory or
// from the global grid alike.
template <typename G>
__device__ __forceinline__ float3 gather_rec(const SysView& v, const SiteRec& r, const BoxDev& b, G at) {
    float tx[4], ty[4], tz[4], dx[4], dy[4], dz[4];
    bspline4((float)r.w[0], tx, dx);
    bspline4((float)r.w[1], ty, dy);
    bspline4((float)r.w[2], tz, dz);
    float gx = 0.f, gy = 0.f, gz = 0.f;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
#pragma unroll
        for (int bb = 0; bb < 4; ++bb) {
            float sz = 0.f, sdz = 0.f;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const float ph = at(a, bb, c);
                sz = fmaf(tz[c], ph, sz);
                sdz = fmaf(dz[c], ph, sdz);
            }
            gx = fmaf(dx[a] * ty[bb], sz, gx);
            gy = fmaf(tx[a] * dy[bb], sz, gy);
            gz = fmaf(tx[a] * ty[bb], sdz, gz);
        }
    }
    const float q = r.q;
    return f3(-q * v.K[0] * b.inv_ext[0] * gx, -q * v.K[1] * b.inv_ext[1] * gy, -q * v.K[2] * b.inv_ext[2] * gz);
}

// A site's reciprocal force: atoms into the reciprocal cache (pass 0 stores,
// later passes add), water sites into the per-site scratch for
// k_gather_wfin.
__device__ __forceinline__ void gather_out(const SysView& v, uint32_t sid, float3 f, int pass) {
    if (sid & DYN_SITE_WATER) {
        float* o = v.wsite_f + 3 * (size_t)(sid & ~DYN_SITE_WATER);
        o[0] = f.x; o[1] = f.y; o[2] = f.z;
        return;
    }
    long long* c = v.arecip + 3 * (size_t)sid;
    if (pass == 0) {
        c[0] = fix_from_float(f.x); c[1] = fix_from_float(f.y); c[2] = fix_from_float(f.z);
    } else {
        c[0] += fix_from_float(f.x); c[1] += fix_from_float(f.y); c[2] += fix_from_float(f.z);
    }
}

// One CTA per brick: the brick and its 3-point halo staged once, its sites'
// stencils read from shared memory; the last OVF_BLOCKS CTAs take the
// overflow list from the global grid.  Each brick's count is cleared for
// the next pass.
DYN_KERNEL(__launch_bounds__(GB_T), k_gather_brick, (, int pass), (, pass)) {
    __shared__ float tile[HB * HB * HB];
    const BoxDev b = *v.box;
    const float wt = pass_weight(v, pass);
    const int tid = threadIdx.x;
    const int K[3] = {(int)v.K[0], (int)v.K[1], (int)v.K[2]};
    for (uint32_t P = bk.idx; P < v.n_bricks + OVF_BLOCKS; P += bk.cnt) {
        if (P >= v.n_bricks) {
            const uint32_t n = v.sc->spme_ovf;
            for (uint32_t t = (P - v.n_bricks) * GB_T + tid; t < n; t += OVF_BLOCKS * GB_T) {
                const SiteRec r = v.ovf_site[t];
                int base[3];
                rec_base(r.base, base);
                int ix[4], iy[4], iz[4];
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    ix[c] = base[0] - 3 + c; if (ix[c] < 0) ix[c] += K[0];
                    iy[c] = base[1] - 3 + c; if (iy[c] < 0) iy[c] += K[1];
                    iz[c] = base[2] - 3 + c; if (iz[c] < 0) iz[c] += K[2];
                }
                const float3 f = gather_rec(v, r, b, [&](int a, int bb, int c) {
                    return __ldg(v.qgrid + ((size_t)ix[a] * K[1] + iy[bb]) * K[2] + iz[c]);
                }) * wt;
                gather_out(v, v.ovf_sid[t], f, pass);
            }
            continue;
        }
        int o[3], ext[3];
        brick_origin(v, P, o, ext);
        // this thread's first site, loaded while the tile comes in
        const uint32_t n = min(v.brick_n[P], v.brick_cap);
        SiteRec r0;
        uint32_t sid0 = 0;
        if ((uint32_t)tid < n) {
            r0 = v.brick_site[(size_t)P * v.brick_cap + tid];
            sid0 = v.brick_sid[(size_t)P * v.brick_cap + tid];
        }
        constexpr int NT = (HB * HB * HB + GB_T - 1) / GB_T;
        float vals[NT];
#pragma unroll
        for (int k = 0; k < NT; ++k) {
            const int i = tid + k * GB_T;
            vals[k] = 0.f;
            if (i < HB * HB * HB) {
                int x = o[0] - 3 + i / (HB * HB), y = o[1] - 3 + (i / HB) % HB, z = o[2] - 3 + i % HB;
                x = x < 0 ? x + K[0] : (x >= K[0] ? x - K[0] : x);
                y = y < 0 ? y + K[1] : (y >= K[1] ? y - K[1] : y);
                z = z < 0 ? z + K[2] : (z >= K[2] ? z - K[2] : z);
                vals[k] = __ldg(v.qgrid + ((size_t)x * K[1] + y) * K[2] + z);
            }
        }
#pragma unroll
        for (int k = 0; k < NT; ++k)
            if (tid + k * GB_T < HB * HB * HB) tile[tid + k * GB_T] = vals[k];
        __syncthreads();
        for (uint32_t t = tid; t < n; t += GB_T) {
            const size_t e = (size_t)P * v.brick_cap + t;
            const SiteRec r = t == (uint32_t)tid ? r0 : v.brick_site[e];
            int base[3];
            rec_base(r.base, base);
            // stencil point a of the site is tile row (base - o) + a
            const int x0 = base[0] - o[0], y0 = base[1] - o[1], z0 = base[2] - o[2];
            const float3 f = gather_rec(v, r, b, [&](int a, int bb, int c) {
                return tile[((x0 + a) * HB + (y0 + bb)) * HB + z0 + c];
            }) * wt;
            gather_out(v, t == (uint32_t)tid ? sid0 : v.brick_sid[e], f, pass);
        }
        __syncthreads();  // every thread has read the count; the tile is refilled next
        if (tid == 0) { v.brick_n[P] = 0u; v.brick_ovf[P] = 0u; }
    }
}

// Water reciprocal forces by molecule, into the cache by original id: the
// sites' gathered forces in float64 plus, with Ewald corrections on, the
// intra-water exclusion corrections (H0-H1, H0-M, H1-M).  Pass 0 stores,
// later passes add.
DYN_KERNEL(, k_gather_wfin, (, int pass), (, pass)) {
    const bool corr = pass == 0 && (v.flags & DYN_FLAG_EWALD_CORRECTIONS);
    double e_c = 0.0, w_c = 0.0;
    for (uint32_t s = bk.idx * blockDim.x + threadIdx.x; s < v.nw_cap; s += bk.cnt * blockDim.x) {
        const uint32_t id = v.wid[s];
        if (id == INVALID_ID) continue;
        double3 fs[3];
        float3 ps[3];
        for (int k = 0; k < 3; ++k) {
            ps[k] = xyz(v.wpos[4 * s + 1 + k]);
            const float* f = v.wsite_f + 9 * (size_t)id + 3 * k;
            fs[k] = make_double3(f[0], f[1], f[2]);
        }
        if (corr) {
            const double q[3] = {OPC_Q_H, OPC_Q_H, OPC_Q_EP};
            const int pa[3] = {0, 0, 1}, pb[3] = {1, 2, 2};
            for (int k = 0; k < 3; ++k) {
                double3 f;
                const double dx = (double)ps[pa[k]].x - (double)ps[pb[k]].x;
                const double dy = (double)ps[pa[k]].y - (double)ps[pb[k]].y;
                const double dz = (double)ps[pa[k]].z - (double)ps[pb[k]].z;
                e_c += excl_corr(dx, dy, dz, q[pa[k]] * q[pb[k]], (double)v.alpha, &f);
                w_c += f.x * dx + f.y * dy + f.z * dz;
                fs[pa[k]].x += f.x; fs[pa[k]].y += f.y; fs[pa[k]].z += f.z;
                fs[pb[k]].x -= f.x; fs[pb[k]].y -= f.y; fs[pb[k]].z -= f.z;
            }
        }
        long long* c = v.wrecip + 9 * (size_t)id;
        for (int k = 0; k < 3; ++k) {
            const long long fx = fix_from_double(fs[k].x), fy = fix_from_double(fs[k].y),
                            fz = fix_from_double(fs[k].z);
            if (pass == 0) { c[3 * k + 0] = fx; c[3 * k + 1] = fy; c[3 * k + 2] = fz; }
            else { c[3 * k + 0] += fx; c[3 * k + 1] += fy; c[3 * k + 2] += fz; }
        }
    }
    if (pass != 0) return;  // the intra-water corrections belong to pass 0
    double x[2] = {e_c, w_c};
    block_sum_d<2>(x);
    if (threadIdx.x == 0) {
        double* p = v.partials + ((size_t)REG_CORR * v.max_blocks + bk.idx) * 4;
        p[0] = x[0]; p[1] = x[1]; p[2] = 0.0; p[3] = 0.0;
    }
}

// Atom corrections on SPME steps.  Reference bookkeeping: the 1-4 vacuum
// force correction (src/non_bonded.rs:763-790), applied to the step's forces
// only, its virial kept with the reciprocal virial.  Corrected mode: float64
// exclusion corrections for 1-2/1-3 pairs (full) and 1-4 pairs (1 - 1/1.2),
// into the reciprocal cache.
DYN_KERNEL(, k_corr_atoms, (), ()) {
    const BoxDev b = *v.box;
    const bool corr = v.flags & DYN_FLAG_EWALD_CORRECTIONS;
    double e_c = 0.0, w_c = 0.0;
    const uint32_t total = v.n14 + (corr ? v.nexcl : 0u);
    for (uint32_t k = bk.idx * blockDim.x + threadIdx.x; k < total; k += bk.cnt * blockDim.x) {
        uint2 p;
        double qq;
        double scale = 1.0;
        if (k < v.n14) { p = v.p14[k]; qq = v.p14_par[k].z; scale = 1.0 - 1.0 / 1.2; }
        else { p = v.excl[k - v.n14]; qq = v.excl_qq[k - v.n14]; }
        const float3 d = min_image_rint(xyz(v.apos[p.x]) - xyz(v.apos[p.y]), b);
        if (!corr) {
            // float32, as the reference: f_vac = dir qq / r^2, df = f_vac (1/1.2 - 1)
            const float r = sqrtf(dot3(d, d));
            if (fabsf(r) < 1e-6f) continue;
            const float3 dir = d * (1.0f / r);
            const float ir = 1.0f / r;
            const float3 df = dir * ((float)qq * ir * ir) * (0.833333333f - 1.0f);
            long long* fa = v.aforce + 3 * (size_t)p.x;
            long long* fb = v.aforce + 3 * (size_t)p.y;
            fix_atomic_add(fa + 0, fix_from_float(df.x)); fix_atomic_add(fa + 1, fix_from_float(df.y));
            fix_atomic_add(fa + 2, fix_from_float(df.z));
            fix_atomic_add(fb + 0, -fix_from_float(df.x)); fix_atomic_add(fb + 1, -fix_from_float(df.y));
            fix_atomic_add(fb + 2, -fix_from_float(df.z));
            w_c += (double)dot3(dir * r, df);
        } else {
            double3 f;
            // exact float64 displacement: positions are float32 and the
            // periodic shift is a whole number of box extents
            const float3 pa = xyz(v.apos[p.x]), pb = xyz(v.apos[p.y]);
            const float3 dr = pa - pb;
            const double sx = -(double)rintf(dr.x * b.inv_ext[0]) * (double)b.ext[0];
            const double sy = -(double)rintf(dr.y * b.inv_ext[1]) * (double)b.ext[1];
            const double sz = -(double)rintf(dr.z * b.inv_ext[2]) * (double)b.ext[2];
            const double dx = (double)pa.x - (double)pb.x + sx;
            const double dy = (double)pa.y - (double)pb.y + sy;
            const double dz = (double)pa.z - (double)pb.z + sz;
            const double qqe = (double)v.apos[p.x].w * (double)v.apos[p.y].w;
            e_c += excl_corr(dx, dy, dz, qqe * scale, (double)v.alpha, &f);
            w_c += f.x * dx + f.y * dy + f.z * dz;
            long long* fa = v.arecip + 3 * (size_t)p.x;
            long long* fb = v.arecip + 3 * (size_t)p.y;
            fix_atomic_add(fa + 0, fix_from_double(f.x)); fix_atomic_add(fa + 1, fix_from_double(f.y));
            fix_atomic_add(fa + 2, fix_from_double(f.z));
            fix_atomic_add(fb + 0, -fix_from_double(f.x)); fix_atomic_add(fb + 1, -fix_from_double(f.y));
            fix_atomic_add(fb + 2, -fix_from_double(f.z));
        }
    }
    double x[2] = {e_c, w_c};
    block_sum_d<2>(x);
    if (threadIdx.x == 0) {
        double* pp = v.partials + ((size_t)REG_CORR_A * v.max_blocks + bk.idx) * 4;
        pp[0] = x[0]; pp[1] = x[1]; pp[2] = 0.0; pp[3] = 0.0;
    }
}

// Energy and virial of one SPME pass (fixed-order sums), weighted into the
// evaluation's totals; with an alchemical molecule the cross term
// E_full - E_env - E_mol times dcoulomb_scale/dlambda goes to dH/dlambda.
DYN_KERNEL(, k_recip_pass, (, int pass), (, pass)) {
    double x[2] = {0.0, 0.0};
    for (uint32_t i = threadIdx.x; i < v.nb[REG_PME]; i += blockDim.x) {
        const double* p = v.partials + ((size_t)REG_PME * v.max_blocks + i) * 4;
        x[0] += p[0]; x[1] += p[1];
    }
    block_sum_d<2>(x);
    if (threadIdx.x != 0) return;
    Scalars* sc = v.sc;
    // the pass's overflow list is done with (k_bin_sites fills the next)
    sc->spme_ovf_max = max(sc->spme_ovf_max, sc->spme_ovf);
    sc->spme_ovf = 0u;
    const double w = (double)pass_weight(v, pass);
    const double dc = v.alch_on ? (double)v.alch_dcs : 0.0;
    if (pass == 0) {
        sc->recip_acc[0] = w * x[0];
        sc->recip_acc[1] = w * x[1];
        sc->recip_dh = dc * x[0];
    } else {
        sc->recip_acc[0] += w * x[0];
        sc->recip_acc[1] += w * x[1];
        sc->recip_dh -= dc * x[0];
    }
}

// The evaluation's reciprocal energy (with the self term), virial and
// corrections into the cache the steps between SPME evaluations reuse.
DYN_KERNEL(, k_recip_finalize, (), ()) {
    double x[4] = {0.0, 0.0, 0.0, 0.0};
    for (uint32_t i = threadIdx.x; i < v.nb[REG_CORR]; i += blockDim.x) {
        const double* p = v.partials + ((size_t)REG_CORR * v.max_blocks + i) * 4;
        x[2] += p[0]; x[3] += p[1];
    }
    for (uint32_t i = threadIdx.x; i < v.nb[REG_CORR_A]; i += blockDim.x) {
        const double* p = v.partials + ((size_t)REG_CORR_A * v.max_blocks + i) * 4;
        x[2] += p[0]; x[3] += p[1];
    }
    block_sum_d<4>(x);
    if (threadIdx.x == 0) {
        Scalars* sc = v.sc;
        sc->recip_cache[0] = sc->recip_acc[0] + v.e_self;
        sc->recip_cache[1] = sc->recip_acc[1];
        sc->recip_cache[2] = x[2];
        sc->recip_cache[3] = x[3];
        sc->recip_dh_cache = sc->recip_dh;
    }
}

inline int gblocks(const SysView& v, uint64_t n) {
    uint64_t bl = (n + GT - 1) / GT;
    if (bl < 1) bl = 1;
    return (int)(bl < v.max_blocks ? bl : v.max_blocks);
}

}  // namespace

namespace dyn {

int pme_blocks(const SysView& v) {
    return gblocks(v, (uint64_t)v.K[0] * v.K[1] * (v.K[2] / 2 + 1));
}
// blocks of k_gather_wfin (which writes the REG_CORR partials)
int gather_blocks(const SysView& v) { return v.nw ? gblocks(v, v.nw_cap) : 0; }

// The brick layout of the grid and the per-brick capacity (cap, or by
// default about twice the mean charged sites per brick plus 32, a multiple
// of 32: liquid densities vary far less), at most 512; the overflow list
// takes the rest.
void pme_bricks(SysView& v, uint32_t cap) {
    uint32_t n = 1;
    for (int a = 0; a < 3; ++a) {
        v.nbrick[a] = (v.K[a] + PME_BRICK - 1) / PME_BRICK;
        n *= v.nbrick[a];
    }
    v.n_bricks = n;
    v.n_sites_max = 3u * v.nw + v.na;
    const uint32_t mean = (v.n_sites_max + n - 1) / n;
    v.brick_cap = std::min(512u, cap ? cap : (2u * mean + 32u + 31u) / 32u * 32u);
}

int corr_blocks(const SysView& v) { return gblocks(v, (uint64_t)v.n14 + v.nexcl); }

int pme_init(SysView& v, cufftHandle* plan_f, cufftHandle* plan_b, cudaStream_t st) {
    const size_t n = (size_t)v.K[0] * v.K[1] * v.K[2];
    const size_t nc = (size_t)v.K[0] * v.K[1] * (v.K[2] / 2 + 1);
    DYN_CUDA(cudaMalloc(&v.qgrid_fix, n * sizeof(long long)));
    DYN_CUDA(cudaMemsetAsync(v.qgrid_fix, 0, n * sizeof(long long), st));
    DYN_CUDA(cudaMalloc(&v.qgrid, n * sizeof(float)));
    DYN_CUDA(cudaMalloc(&v.cgrid, nc * sizeof(float2)));
    for (int a = 0; a < 3; ++a) {
        // |b(m)|^2 = 1 / |sum_{k=0}^{2} M4(k+1) exp(2 pi i m k / K)|^2 (Essmann eq. 4.4)
        const int K = (int)v.K[a];
        std::vector<float> bm(K);
        const double mv[3] = {1.0 / 6.0, 4.0 / 6.0, 1.0 / 6.0};
        for (int m = 0; m < K; ++m) {
            double re = 0.0, im = 0.0;
            for (int k = 0; k < 3; ++k) {
                re += mv[k] * std::cos(2.0 * M_PI * m * k / K);
                im += mv[k] * std::sin(2.0 * M_PI * m * k / K);
            }
            bm[m] = (float)(1.0 / (re * re + im * im));
        }
        DYN_CUDA(cudaMalloc(&v.bmod[a], K * sizeof(float)));
        DYN_CUDA(cudaMemcpyAsync(v.bmod[a], bm.data(), K * sizeof(float), cudaMemcpyHostToDevice, st));
    }
    DYN_CUDA(cudaStreamSynchronize(st));
    if (cufftPlan3d(plan_f, v.K[0], v.K[1], v.K[2], CUFFT_R2C) != CUFFT_SUCCESS)
        return dyn::fail(DYN_ERR_CUDA, "cufftPlan3d R2C failed");
    if (cufftPlan3d(plan_b, v.K[0], v.K[1], v.K[2], CUFFT_C2R) != CUFFT_SUCCESS)
        return dyn::fail(DYN_ERR_CUDA, "cufftPlan3d C2R failed");
    if (cufftSetStream(*plan_f, st) != CUFFT_SUCCESS || cufftSetStream(*plan_b, st) != CUFFT_SUCCESS)
        return dyn::fail(DYN_ERR_CUDA, "cufftSetStream failed");
    return DYN_OK;
}

void pme_free(SysView& v, cufftHandle plan_f, cufftHandle plan_b) {
    if (plan_f) cufftDestroy(plan_f);
    if (plan_b) cufftDestroy(plan_b);
    cudaFree(v.qgrid_fix); cudaFree(v.qgrid); cudaFree(v.cgrid);
    for (int a = 0; a < 3; ++a) cudaFree(v.bmod[a]);
}

// Runs f(view, stream) for every system; a batch forks onto its FFT side
// streams (members round-robin) and joins back, so the members' small
// transforms run side by side.
template <typename F>
void each_fft(const Target& t, F f) {
    if (t.v) { f(*t.v, t.st); return; }
    if (batch_collecting(t.b)) return;
    const uint32_t n = batch_size(t.b);
    cudaStream_t* fs = nullptr;
    cudaEvent_t* fe = nullptr;
    const int nf = batch_fft_streams(t.b, &fs, &fe);
    if (nf <= 0 || n <= 1) {
        for (uint32_t i = 0; i < n; ++i) f(batch_view(t.b, i), t.st);
        return;
    }
    const int use = (int)std::min<uint32_t>((uint32_t)nf, n);
    cudaEventRecord(fe[nf], t.st);
    for (int k = 0; k < use; ++k) cudaStreamWaitEvent(fs[k], fe[nf], 0);
    for (uint32_t i = 0; i < n; ++i) f(batch_view(t.b, i), fs[i % (uint32_t)use]);
    for (int k = 0; k < use; ++k) {
        cudaEventRecord(fe[k], fs[k]);
        cudaStreamWaitEvent(t.st, fe[k], 0);
    }
}

// one SPME pass in three parts (the stage timer times them apart)
void launch_pme_spread(const Target& t, int pass) {
    auto on = [pass](const SysView& v) { return pass == 0 || v.alch_on != 0u; };
    t.launch(k_bin_sites, k_bin_sites_batch,
             [&](const SysView& v) { return on(v) ? gblocks(v, 3ull * v.nw_cap + v.na) : 0; }, GT, 0, pass);
    t.launch(k_spread_brick, k_spread_brick_batch,
             [&](const SysView& v) { return on(v) ? (int)std::min(v.n_bricks, v.max_blocks) : 0; }, SB_T, 0, pass);
    // phase 2: per brick where every axis is simple, per point otherwise
    auto simple = [](const SysView& v) {
        auto ax = [](uint32_t K) { return K >= (uint32_t)HB && (K % PME_BRICK == 0 || K % PME_BRICK >= 3); };
        return ax(v.K[0]) && ax(v.K[1]) && ax(v.K[2]);
    };
    t.launch(k_spread_merge_brick, k_spread_merge_brick_batch,
             [&](const SysView& v) { return on(v) && simple(v) ? (int)std::min(v.n_bricks, v.max_blocks) : 0; },
             SB_T, 0, pass);
    t.launch(k_spread_merge, k_spread_merge_batch,
             [&](const SysView& v) {
                 return on(v) && !simple(v) ? gblocks(v, (uint64_t)v.K[0] * v.K[1] * v.K[2]) : 0;
             },
             GT, 0, pass);
}

void launch_pme_transform(const Target& t, int pass) {
    auto on = [pass](const SysView& v) { return pass == 0 || v.alch_on != 0u; };
    each_fft(t, [on](const SysView& v, cudaStream_t s) {
        if (!on(v)) return;
        cufftSetStream(v.plan_f, s);
        cufftExecR2C(v.plan_f, v.qgrid, (cufftComplex*)v.cgrid);
    });
    t.launch(k_convolve, k_convolve_batch, [&](const SysView& v) { return on(v) ? (int)v.nb[REG_PME] : 0; }, GT, 0);
    each_fft(t, [on](const SysView& v, cudaStream_t s) {
        if (!on(v)) return;
        cufftSetStream(v.plan_b, s);
        cufftExecC2R(v.plan_b, (cufftComplex*)v.cgrid, v.qgrid);
    });
}

void launch_pme_gather(const Target& t, int pass) {
    auto on = [pass](const SysView& v) { return pass == 0 || v.alch_on != 0u; };
    t.launch(k_gather_brick, k_gather_brick_batch,
             [&](const SysView& v) { return on(v) ? (int)std::min(v.n_bricks + OVF_BLOCKS, v.max_blocks) : 0; },
             GB_T, 0, pass);
    // the molecule's own pass (2) holds no water
    t.launch(k_gather_wfin, k_gather_wfin_batch,
             [&](const SysView& v) { return on(v) && pass != 2 ? (int)v.nb[REG_CORR] : 0; }, GT, 0, pass);
    t.launch(k_recip_pass, k_recip_pass_batch, [&](const SysView& v) { return on(v) ? 1 : 0; }, 256, 0, pass);
}

void launch_pme(const Target& t) {
    // one pass, or three with an alchemical molecule in any system (systems
    // without one skip passes 1 and 2)
    const int npass = t.any([](const SysView& v) { return v.alch_on != 0u; }) ? 3 : 1;
    for (int pass = 0; pass < npass; ++pass) {
        launch_pme_spread(t, pass);
        launch_pme_transform(t, pass);
        launch_pme_gather(t, pass);
    }
}

void launch_corrections(const Target& t) {
    t.launch(k_corr_atoms, k_corr_atoms_batch, [](const SysView& v) { return (int)v.nb[REG_CORR_A]; }, GT, 0);
    t.launch(k_recip_finalize, k_recip_finalize_batch, [](const SysView&) { return 1; }, 256, 0);
}

}  // namespace dyn
