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

// Charge spreading with float64 weights and products, accumulated as 64-bit
// fixed point (exact, order-independent sums).
__device__ __forceinline__ void spread_one(const SysView& v, float3 p, float q, const BoxDev& b) {
    int base[3];
    double w[3];
    grid_coord(p, b, v.K, base, w);
    double tx[4], ty[4], tz[4];
    bspline4d(w[0], tx);
    bspline4d(w[1], ty);
    bspline4d(w[2], tz);
    const int K0 = v.K[0], K1 = v.K[1], K2 = v.K[2];
    int iz[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) { int z = base[2] - 3 + c; iz[c] = z < 0 ? z + K2 : z; }
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        int x = base[0] - 3 + a; x = x < 0 ? x + K0 : x;
        const double qa = (double)q * tx[a];
#pragma unroll
        for (int bb = 0; bb < 4; ++bb) {
            int y = base[1] - 3 + bb; y = y < 0 ? y + K1 : y;
            const double qab = qa * ty[bb];
            long long* row = v.qgrid_fix + ((size_t)x * K1 + y) * K2;
#pragma unroll
            for (int c = 0; c < 4; ++c) fix_atomic_add(row + iz[c], fix_from_double(qab * tz[c]));
        }
    }
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

// one thread per charged atom (the water sites go by group, below)
DYN_KERNEL(, k_spread, (, int pass), (, pass)) {
    const BoxDev b = *v.box;
    for (uint32_t t = bk.idx * blockDim.x + threadIdx.x; t < v.na; t += bk.cnt * blockDim.x) {
        const float4 p = v.apos[t];
        if (p.w != 0.f && pass_has_atom(v, pass, t)) spread_one(v, xyz(p), p.w, b);
    }
}

// ---------------------------------------------------------------------------
// Water sites by water group.  A CTA takes a 32-water group of the pair
// kernels (spatially compact): the order-4 stencils of its 96 charged sites
// fall in a small box of grid points, held in shared memory.  The spread
// adds every contribution there (the same int64 fixed-point values as one
// global atomic per contribution would add: integer sums in any order, so
// the grid is bit-identical) and then adds the box's nonzero points to the
// global grid, about half as many global atomics; the gather stages the
// box once with coalesced loads and reads the stencils from shared memory
// (the same float arithmetic in the same order as per site).  A group whose
// box exceeds the tile (scattered waters in a dilute system) takes the
// per-site path.
// ---------------------------------------------------------------------------
constexpr int SG_T = 128;               // threads per CTA
constexpr int SG_SITES = 3 * GRPW;      // charged sites of a group
constexpr int TILE_PTS = 4096;          // shared tile capacity (grid points)

struct GroupSites {
    int base[SG_SITES][3];              // stencil base of each site
    double w[SG_SITES][3];              // fractional grid coordinate
    float3 pos[SG_SITES];
    float q[SG_SITES];                  // 0: no site (padding slot)
    int lo[3], n[3];                    // tile origin (relative to ref) and size
    int ref[3];                         // base of the first site
    int use_tile;
};

// Fills the group's sites and its tile box (whole CTA; ends synchronised).
__device__ __forceinline__ void group_sites(const SysView& v, uint32_t g, const BoxDev& b, GroupSites& gs) {
    const int tid = threadIdx.x;
    if (tid < 3) { gs.lo[tid] = 1 << 30; gs.n[tid] = -(1 << 30); }
    for (int t = tid; t < SG_SITES; t += SG_T) {
        const uint32_t s = g * GRPW + t / 3;
        const bool ok = s < v.nw_cap && v.wid[s] != INVALID_ID;
        float4 p = make_float4(0.f, 0.f, 0.f, 0.f);
        if (ok) p = v.wpos[4 * s + 1 + t % 3];
        gs.pos[t] = xyz(p);
        gs.q[t] = ok ? p.w : 0.f;
        int bs[3];
        double ww[3];
        grid_coord(xyz(p), b, v.K, bs, ww);
        for (int a = 0; a < 3; ++a) { gs.base[t][a] = bs[a]; gs.w[t][a] = ww[a]; }
    }
    __syncthreads();
    if (tid == 0) {
        int f = 0;
        while (f < SG_SITES && gs.q[f] == 0.f) ++f;
        for (int a = 0; a < 3; ++a) gs.ref[a] = f < SG_SITES ? gs.base[f][a] : 0;
    }
    __syncthreads();
    for (int t = tid; t < SG_SITES; t += SG_T) {
        if (gs.q[t] == 0.f) continue;
        for (int a = 0; a < 3; ++a) {
            const int K = (int)v.K[a];
            int r = gs.base[t][a] - gs.ref[a];
            r -= K * (int)floorf((float)r / (float)K + 0.5f);  // nearest image, |r| <= K/2
            atomicMin(&gs.lo[a], r - 3);
            atomicMax(&gs.n[a], r);
        }
    }
    __syncthreads();
    if (tid == 0) {
        long long pts = 1;
        bool fits = true;
        for (int a = 0; a < 3; ++a) {
            gs.n[a] = gs.n[a] - gs.lo[a] + 1;
            fits = fits && gs.n[a] > 0 && gs.n[a] <= (int)v.K[a];
            pts *= gs.n[a] > 0 ? gs.n[a] : 0;
        }
        gs.use_tile = fits && pts > 0 && pts <= TILE_PTS;
    }
    __syncthreads();
}

// tile offset of a site's stencil point (a, bb, c) and the grid index of a tile point
__device__ __forceinline__ int rel_base(const SysView& v, const GroupSites& gs, int t, int a) {
    const int K = (int)v.K[a];
    int r = gs.base[t][a] - gs.ref[a];
    r -= K * (int)floorf((float)r / (float)K + 0.5f);
    return r - gs.lo[a];
}
__device__ __forceinline__ size_t tile_to_grid(const SysView& v, const GroupSites& gs, int idx) {
    const int z = idx % gs.n[2], y = (idx / gs.n[2]) % gs.n[1], x = idx / (gs.n[2] * gs.n[1]);
    int gi[3] = {x, y, z};
    for (int a = 0; a < 3; ++a) {
        const int K = (int)v.K[a];
        int u = gs.ref[a] + gs.lo[a] + gi[a];
        u %= K;
        if (u < 0) u += K;
        gi[a] = u;
    }
    return ((size_t)gi[0] * v.K[1] + gi[1]) * v.K[2] + gi[2];
}

DYN_KERNEL(__launch_bounds__(SG_T), k_spread_w, (, int pass), (, pass)) {
    if (pass == 2) return;  // the alchemical molecule's own pass holds no water
    __shared__ GroupSites gs;
    __shared__ unsigned long long tile[TILE_PTS];
    const BoxDev b = *v.box;
    const uint32_t ng = (v.sc->n_wclus + GRPW / WCL - 1) / (GRPW / WCL);
    const int tid = threadIdx.x;
    for (uint32_t g = bk.idx; g < ng; g += bk.cnt) {
        group_sites(v, g, b, gs);
        if (!gs.use_tile) {
            for (int t = tid; t < SG_SITES; t += SG_T)
                if (gs.q[t] != 0.f) spread_one(v, gs.pos[t], gs.q[t], b);
            __syncthreads();
            continue;
        }
        const int npts = gs.n[0] * gs.n[1] * gs.n[2];
        for (int i = tid; i < npts; i += SG_T) tile[i] = 0ull;
        __syncthreads();
        // one (site, x plane) per thread and round: 16 contributions each
        for (int u = tid; u < SG_SITES * 4; u += SG_T) {
            const int t = u >> 2, a = u & 3;
            if (gs.q[t] == 0.f) continue;
            double tx[4], ty[4], tz[4];
            bspline4d(gs.w[t][0], tx);
            bspline4d(gs.w[t][1], ty);
            bspline4d(gs.w[t][2], tz);
            const int x = rel_base(v, gs, t, 0) - 3 + a;
            const int y0 = rel_base(v, gs, t, 1) - 3, z0 = rel_base(v, gs, t, 2) - 3;
            const double qa = (double)gs.q[t] * tx[a];
#pragma unroll
            for (int bb = 0; bb < 4; ++bb) {
                const double qab = qa * ty[bb];
                const int row = (x * gs.n[1] + (y0 + bb)) * gs.n[2] + z0;
#pragma unroll
                for (int c = 0; c < 4; ++c)
                    atomicAdd(&tile[row + c], (unsigned long long)fix_from_double(qab * tz[c]));
            }
        }
        __syncthreads();
        for (int i = tid; i < npts; i += SG_T) {
            const long long q = (long long)tile[i];
            if (q != 0) fix_atomic_add(v.qgrid_fix + tile_to_grid(v, gs, i), q);
        }
        __syncthreads();
    }
}

DYN_KERNEL(, k_fix2real, (), ()) {
    const uint32_t n = v.K[0] * v.K[1] * v.K[2];
    for (uint32_t i = bk.idx * blockDim.x + threadIdx.x; i < n; i += bk.cnt * blockDim.x) {
        v.qgrid[i] = (float)((double)v.qgrid_fix[i] * DYN_FIX_INV);
        v.qgrid_fix[i] = 0;
    }
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

__device__ __forceinline__ float3 gather_one(const SysView& v, float3 p, float q, const BoxDev& b) {
    int base[3];
    double wd[3];
    grid_coord(p, b, v.K, base, wd);
    float tx[4], ty[4], tz[4], dx[4], dy[4], dz[4];
    bspline4((float)wd[0], tx, dx);
    bspline4((float)wd[1], ty, dy);
    bspline4((float)wd[2], tz, dz);
    const int K0 = v.K[0], K1 = v.K[1], K2 = v.K[2];
    int iz[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) { int z = base[2] - 3 + c; iz[c] = z < 0 ? z + K2 : z; }
    float gx = 0.f, gy = 0.f, gz = 0.f;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        int x = base[0] - 3 + a; x = x < 0 ? x + K0 : x;
#pragma unroll
        for (int bb = 0; bb < 4; ++bb) {
            int y = base[1] - 3 + bb; y = y < 0 ? y + K1 : y;
            const float* row = v.qgrid + ((size_t)x * K1 + y) * K2;
            float sz = 0.f, sdz = 0.f;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const float ph = __ldg(row + iz[c]);
                sz = fmaf(tz[c], ph, sz);
                sdz = fmaf(dz[c], ph, sdz);
            }
            gx = fmaf(dx[a] * ty[bb], sz, gx);
            gy = fmaf(tx[a] * dy[bb], sz, gy);
            gz = fmaf(tx[a] * ty[bb], sdz, gz);
        }
    }
    return f3(-q * K0 * b.inv_ext[0] * gx, -q * K1 * b.inv_ext[1] * gy, -q * K2 * b.inv_ext[2] * gz);
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

// Gather for the atoms: one thread per atom, writing the reciprocal cache.
// Pass 0 stores its (weighted) forces, later passes add theirs.
DYN_KERNEL(, k_gather, (, int pass), (, pass)) {
    const BoxDev b = *v.box;
    const float wt = pass_weight(v, pass);
    for (uint32_t t = bk.idx * blockDim.x + threadIdx.x; t < v.na; t += bk.cnt * blockDim.x) {
        if (!pass_has_atom(v, pass, t)) continue;
        const float4 p = v.apos[t];
        float3 f = f3(0.f, 0.f, 0.f);
        if (p.w != 0.f) f = gather_one(v, xyz(p), p.w, b) * wt;
        long long* c = v.arecip + 3 * (size_t)t;
        if (pass == 0) {
            c[0] = fix_from_float(f.x); c[1] = fix_from_float(f.y); c[2] = fix_from_float(f.z);
        } else {
            c[0] += fix_from_float(f.x); c[1] += fix_from_float(f.y); c[2] += fix_from_float(f.z);
        }
    }
}

// The gather of one site from a staged tile: gather_one's arithmetic, in its
// order, with the grid values read from shared memory.
__device__ __forceinline__ float3 gather_tile(const SysView& v, const GroupSites& gs, const float* tile, int t,
                                              const BoxDev& b) {
    float tx[4], ty[4], tz[4], dx[4], dy[4], dz[4];
    bspline4((float)gs.w[t][0], tx, dx);
    bspline4((float)gs.w[t][1], ty, dy);
    bspline4((float)gs.w[t][2], tz, dz);
    const int x0 = rel_base(v, gs, t, 0) - 3, y0 = rel_base(v, gs, t, 1) - 3, z0 = rel_base(v, gs, t, 2) - 3;
    float gx = 0.f, gy = 0.f, gz = 0.f;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
#pragma unroll
        for (int bb = 0; bb < 4; ++bb) {
            const float* row = tile + ((x0 + a) * gs.n[1] + (y0 + bb)) * gs.n[2] + z0;
            float sz = 0.f, sdz = 0.f;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const float ph = row[c];
                sz = fmaf(tz[c], ph, sz);
                sdz = fmaf(dz[c], ph, sdz);
            }
            gx = fmaf(dx[a] * ty[bb], sz, gx);
            gy = fmaf(tx[a] * dy[bb], sz, gy);
            gz = fmaf(tx[a] * ty[bb], sdz, gz);
        }
    }
    const float q = gs.q[t];
    return f3(-q * v.K[0] * b.inv_ext[0] * gx, -q * v.K[1] * b.inv_ext[1] * gy, -q * v.K[2] * b.inv_ext[2] * gz);
}

// Gather for the water sites by group (tile as for the spread), writing the
// reciprocal cache by original water id.  With Ewald corrections on, the
// intra-water exclusion corrections (H0-H1, H0-M, H1-M) are added here in
// float64.  Pass 0 stores its (weighted) forces, later passes add theirs.
DYN_KERNEL(__launch_bounds__(SG_T), k_gather_w, (, int pass), (, pass)) {
    __shared__ GroupSites gs;
    __shared__ float tile[TILE_PTS];
    __shared__ float3 fsite[SG_SITES];
    const BoxDev b = *v.box;
    const bool corr = pass == 0 && (v.flags & DYN_FLAG_EWALD_CORRECTIONS);
    const float wt = pass_weight(v, pass);
    const uint32_t ng = (v.sc->n_wclus + GRPW / WCL - 1) / (GRPW / WCL);
    const int tid = threadIdx.x;
    double e_c = 0.0, w_c = 0.0;
    for (uint32_t g = bk.idx; g < ng && pass != 2; g += bk.cnt) {
        group_sites(v, g, b, gs);
        if (gs.use_tile) {
            const int npts = gs.n[0] * gs.n[1] * gs.n[2];
            for (int i = tid; i < npts; i += SG_T) tile[i] = __ldg(v.qgrid + tile_to_grid(v, gs, i));
            __syncthreads();
        }
        for (int t = tid; t < SG_SITES; t += SG_T) {
            float3 f = f3(0.f, 0.f, 0.f);
            if (gs.q[t] != 0.f)
                f = (gs.use_tile ? gather_tile(v, gs, tile, t, b) : gather_one(v, gs.pos[t], gs.q[t], b)) * wt;
            fsite[t] = f;
        }
        __syncthreads();
        for (int w = tid; w < GRPW; w += SG_T) {
            const uint32_t s = g * GRPW + w;
            if (s >= v.nw_cap) continue;
            const uint32_t id = v.wid[s];
            if (id == INVALID_ID) continue;
            double3 fs[3];
            float3 ps[3];
            for (int k = 0; k < 3; ++k) {
                ps[k] = gs.pos[3 * w + k];
                const float3 f = fsite[3 * w + k];
                fs[k] = make_double3(f.x, f.y, f.z);
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
        __syncthreads();  // gs, the tile and fsite are refilled by the next group
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
// blocks of the water-group SPME kernels (k_gather_w writes REG_CORR partials)
int gather_blocks(const SysView& v) {
    return v.nw ? (int)std::min<uint32_t>(v.ngrp_cap, v.max_blocks) : 0;
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
    t.launch(k_spread, k_spread_batch, [&](const SysView& v) { return on(v) && v.na ? gblocks(v, v.na) : 0; },
             GT, 0, pass);
    t.launch(k_spread_w, k_spread_w_batch, [&](const SysView& v) { return on(v) ? gather_blocks(v) : 0; }, SG_T, 0,
             pass);
    t.launch(k_fix2real, k_fix2real_batch,
             [&](const SysView& v) { return on(v) ? gblocks(v, (uint64_t)v.K[0] * v.K[1] * v.K[2]) : 0; }, GT, 0);
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
    t.launch(k_gather, k_gather_batch, [&](const SysView& v) { return on(v) && v.na ? gblocks(v, v.na) : 0; }, GT, 0,
             pass);
    t.launch(k_gather_w, k_gather_w_batch, [&](const SysView& v) { return on(v) ? (int)v.nb[REG_CORR] : 0; }, SG_T,
             0, pass);
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
