// Bonded terms of the resident engine: harmonic bonds and angles and
// periodic (proper and improper) dihedrals, one thread per term, int64
// fixed-point atomics so the total is order independent.
//
// Forms follow src/bonded_forces.rs:11-178 (U = k (r - r0)^2,
// U = k (theta - theta0)^2, U = sum k (1 + cos(n phi - phase)) with phi the
// IUPAC dihedral) and the virials of src/bonded.rs:41-130.
#include "engine.cuh"

namespace {

constexpr int BT = 256;

__device__ __forceinline__ void addf(long long* f, uint32_t i, float3 v) {
    long long* p = f + 3 * (size_t)i;
    fix_atomic_add(p + 0, fix_from_float(v.x));
    fix_atomic_add(p + 1, fix_from_float(v.y));
    fix_atomic_add(p + 2, fix_from_float(v.z));
}

template <bool ENERGY>
__global__ void k_bonded(SysView v) {
    const BoxDev b = *v.box;
    double e_acc = 0.0, w_acc = 0.0;
    const uint32_t total = v.nbond + v.nangle + v.ndih;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        if (t < v.nbond) {
            const uint2 ij = v.bond[t];
            const float2 par = v.bond_par[t];  // k, r0
            const float3 d = min_image_rint(xyz(v.apos[ij.y]) - xyz(v.apos[ij.x]), b);
            const float r = sqrtf(dot3(d, d));
            const float dr = r - par.y;
            const float3 f0 = d * (2.0f * par.x * dr / fmaxf(r, 1e-8f));
            addf(v.aforce, ij.x, f0);
            addf(v.aforce, ij.y, f3(-f0.x, -f0.y, -f0.z));
            if (ENERGY) e_acc += (double)(par.x * dr * dr);
            w_acc += (double)dot3(d, f0);
        } else if (t < v.nbond + v.nangle) {
            const uint4 ijk = v.angle[t - v.nbond];
            const float2 par = v.angle_par[t - v.nbond];  // k, theta0
            const float3 p1 = xyz(v.apos[ijk.y]);
            const float3 v01 = min_image_rint(xyz(v.apos[ijk.x]) - p1, b);
            const float3 v21 = min_image_rint(xyz(v.apos[ijk.z]) - p1, b);
            const float l01s = dot3(v01, v01), l21s = dot3(v21, v21);
            if (l01s < 1e-8f || l21s < 1e-8f) continue;
            const float l01 = sqrtf(l01s), l21 = sqrtf(l21s);
            const float3 u01 = v01 * (1.0f / l01), u21 = v21 * (1.0f / l21);
            const float ct = fminf(1.0f, fmaxf(-1.0f, dot3(u01, u21)));
            const float th = acosf(ct);
            const float st = fmaxf(sqrtf(1.0f - ct * ct), 1e-8f);
            const float dth = th - par.y;
            const float de = 2.0f * par.x * dth;
            const float3 g0 = (u01 * ct - u21) * (1.0f / (l01 * st));
            const float3 g2 = (u21 * ct - u01) * (1.0f / (l21 * st));
            const float3 f0 = g0 * (-de), f2 = g2 * (-de);
            const float3 f1 = f3(-(f0.x + f2.x), -(f0.y + f2.y), -(f0.z + f2.z));
            addf(v.aforce, ijk.x, f0);
            addf(v.aforce, ijk.y, f1);
            addf(v.aforce, ijk.z, f2);
            if (ENERGY) e_acc += (double)(par.x * dth * dth);
            w_acc += (double)(dot3(v01, f0) + dot3(v21, f2));
        } else {
            const uint32_t k = t - v.nbond - v.nangle;
            const uint4 q = v.dih[k];
            const float4 par = v.dih_par[k];  // k, n, phase
            const float3 p0 = xyz(v.apos[q.x]);
            const float3 b1 = min_image_rint(xyz(v.apos[q.y]) - p0, b);
            const float3 b2 = min_image_rint(xyz(v.apos[q.z]) - xyz(v.apos[q.y]), b);
            const float3 b3 = min_image_rint(xyz(v.apos[q.w]) - xyz(v.apos[q.z]), b);
            const float3 n1 = cross3(b1, b2), n2 = cross3(b2, b3);
            const float n1s = dot3(n1, n1), n2s = dot3(n2, n2), b2s = dot3(b2, b2);
            const float b2n = sqrtf(b2s);
            if (n1s < 1e-6f || n2s < 1e-6f || b2n < 1e-6f) continue;
            const float x = dot3(n1, n2);
            const float y = dot3(cross3(n1, n2), b2) / b2n;
            const float phi = atan2f(y, x);
            float sn, cn;
            sincosf(par.y * phi - par.z, &sn, &cn);
            const float dv = -par.x * par.y * sn;  // dU/dphi
            const float3 g0 = n1 * (-b2n / n1s);
            const float3 g3 = n2 * (b2n / n2s);
            const float ta = dot3(b1, b2) / b2s, tb = dot3(b3, b2) / b2s;
            const float3 g1 = g0 * (-1.0f - ta) + g3 * tb;
            const float3 g2 = g3 * (-1.0f - tb) + g0 * ta;
            const float3 f0 = g0 * (-dv), f1 = g1 * (-dv), f2 = g2 * (-dv), f3v = g3 * (-dv);
            addf(v.aforce, q.x, f0);
            addf(v.aforce, q.y, f1);
            addf(v.aforce, q.z, f2);
            addf(v.aforce, q.w, f3v);
            if (ENERGY) e_acc += (double)(par.x * (1.0f + cn));
            // virial relative to atom 1 (src/bonded.rs:123-130)
            w_acc += (double)(dot3(f3(-b1.x, -b1.y, -b1.z), f0) + dot3(b2, f2) + dot3(b2 + b3, f3v));
        }
    }
    double xs[3] = {e_acc, 0.0, w_acc};
    block_sum_d<3>(xs);
    if (threadIdx.x == 0) {
        double* p = v.partials + ((size_t)REG_BOND * v.max_blocks + blockIdx.x) * 4;
        p[0] = xs[0]; p[1] = xs[1]; p[2] = xs[2]; p[3] = 0.0;
    }
}

}  // namespace

namespace dyn {

int bond_blocks(const SysView& v) {
    uint64_t n = (uint64_t)v.nbond + v.nangle + v.ndih;
    uint64_t bl = (n + BT - 1) / BT;
    if (bl < 1) bl = 1;
    return (int)(bl < v.max_blocks ? bl : v.max_blocks);
}

void launch_bonded(const SysView& v, cudaStream_t st, bool energy) {
    if (v.nbond + v.nangle + v.ndih == 0) return;
    if (energy) k_bonded<true><<<v.nb[REG_BOND], BT, 0, st>>>(v);
    else k_bonded<false><<<v.nb[REG_BOND], BT, 0, st>>>(v);
}

}  // namespace dyn
