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

// Exact float64 minimum-image displacement b - a of two float32 positions
// (the shift is a whole number of box extents), for the energies.
__device__ __forceinline__ double3 dd_min_image(float3 a, float3 bpos, const BoxDev& b) {
    const float3 d = bpos - a;
    double3 r;
    r.x = (double)bpos.x - (double)a.x - (double)rintf(d.x * b.inv_ext[0]) * (double)b.ext[0];
    r.y = (double)bpos.y - (double)a.y - (double)rintf(d.y * b.inv_ext[1]) * (double)b.ext[1];
    r.z = (double)bpos.z - (double)a.z - (double)rintf(d.z * b.inv_ext[2]) * (double)b.ext[2];
    return r;
}
__device__ __forceinline__ double ddot(double3 a, double3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ double3 dcross(double3 a, double3 b) {
    return make_double3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

DYN_KERNEL_T((bool ENERGY), (ENERGY), , k_bonded, (), ()) {
    const BoxDev b = *v.box;
    double e_acc = 0.0, w_acc = 0.0;
    const uint32_t total = v.nbond + v.nangle + v.ndih;
    for (uint32_t t = bk.idx * blockDim.x + threadIdx.x; t < total; t += bk.cnt * blockDim.x) {
        if (t < v.nbond) {
            const uint2 ij = v.bond[t];
            const float2 par = v.bond_par[t];  // k, r0
            const float3 d = min_image_rint(xyz(v.apos[ij.y]) - xyz(v.apos[ij.x]), b);
            const float r = sqrtf(dot3(d, d));
            const float dr = r - par.y;
            const float3 f0 = d * (2.0f * par.x * dr / fmaxf(r, 1e-8f));
            addf(v.aforce, ij.x, f0);
            addf(v.aforce, ij.y, f3(-f0.x, -f0.y, -f0.z));
            if (ENERGY) {
                const double3 e = dd_min_image(xyz(v.apos[ij.x]), xyz(v.apos[ij.y]), b);
                const double de = sqrt(ddot(e, e)) - (double)par.y;
                e_acc += (double)par.x * de * de;
            }
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
            if (ENERGY) {
                const double3 a0 = dd_min_image(p1, xyz(v.apos[ijk.x]), b);
                const double3 a2 = dd_min_image(p1, xyz(v.apos[ijk.z]), b);
                double c = ddot(a0, a2) / sqrt(ddot(a0, a0) * ddot(a2, a2));
                c = c > 1.0 ? 1.0 : (c < -1.0 ? -1.0 : c);
                const double dt = acos(c) - (double)par.y;
                e_acc += (double)par.x * dt * dt;
            }
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
            if (ENERGY) {
                const double3 c1 = dd_min_image(p0, xyz(v.apos[q.y]), b);
                const double3 c2 = dd_min_image(xyz(v.apos[q.y]), xyz(v.apos[q.z]), b);
                const double3 c3 = dd_min_image(xyz(v.apos[q.z]), xyz(v.apos[q.w]), b);
                const double3 m1 = dcross(c1, c2), m2 = dcross(c2, c3);
                const double xx = ddot(m1, m2);
                const double yy = ddot(dcross(m1, m2), c2) / sqrt(ddot(c2, c2));
                const double ph = atan2(yy, xx);
                e_acc += (double)par.x * (1.0 + cos((double)par.y * ph - (double)par.z));
            }
            // virial relative to atom 1 (src/bonded.rs:123-130)
            w_acc += (double)(dot3(f3(-b1.x, -b1.y, -b1.z), f0) + dot3(b2, f2) + dot3(b2 + b3, f3v));
        }
    }
    double xs[3] = {e_acc, 0.0, w_acc};
    block_sum_d<3>(xs);
    if (threadIdx.x == 0) {
        double* p = v.partials + ((size_t)REG_BOND * v.max_blocks + bk.idx) * 4;
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

void launch_bonded(const Target& t, bool energy) {
    auto g = [](const SysView& v) { return v.nbond + v.nangle + v.ndih ? (int)v.nb[REG_BOND] : 0; };
    if (energy) t.launch(k_bonded<true>, k_bonded_batch<true>, g, BT, 0);
    else t.launch(k_bonded<false>, k_bonded_batch<false>, g, BT, 0);
}

}  // namespace dyn
