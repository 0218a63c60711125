// Integrator kernels of the resident engine: rigid OPC water, solute atoms,
// Langevin OU noise, CSVR, C-rescale, COM removal, recentering, and the
// deterministic float64 reductions that feed the thermostat and barostat.
//
// The rigid-water update restates integrate_rigid_water
// (src/solvent/opc_settle.rs:107-198): COM translation plus a Rodrigues
// rotation with omega = I^-1 L, wrap of O, minimum-image H, M on the
// bisector.  Step orders follow MdState::step (src/integrate.rs:100-317):
//   Langevin-middle: kick dt/2, drift dt/2, OU(dt), drift dt/2, forces,
//                    kick dt/2;
//   velocity Verlet: kick dt/2, drift dt, forces, kick dt/2, CSVR.
// Every kernel processes one water slot or one atom per thread.
#include "engine.cuh"

namespace {

constexpr int IT = 256;

__device__ __forceinline__ float3 wrap_pos(float3 p, const BoxDev& b) {
    p.x -= floorf((p.x - b.lo[0]) * b.inv_ext[0]) * b.ext[0];
    p.y -= floorf((p.y - b.lo[1]) * b.inv_ext[1]) * b.ext[1];
    p.z -= floorf((p.z - b.lo[2]) * b.inv_ext[2]) * b.ext[2];
    return p;
}

__device__ __forceinline__ float3 rodrigues(float3 r, float3 w, float dt) {
    const float3 od = w * dt;
    const float th = sqrtf(dot3(od, od));
    if (th < 1e-12f) {
        const float3 wxr = cross3(od, r);
        return r + wxr + cross3(od, wxr) * 0.5f;
    }
    const float3 n = od * (1.0f / th);
    float s, c, sh, ch;
    sincosf(th, &s, &c);
    sincosf(0.5f * th, &sh, &ch);
    const float omc = 2.0f * sh * sh;  // 1 - cos(th) without cancellation
    return r * c + cross3(n, r) * s + n * (dot3(n, r) * omc);
}

// COM, COM-frame vectors and angular velocity omega = I^-1 L of one water
// (src/solvent/opc_settle.rs:108-153).
struct RigidFrame {
    float3 rcom, vcom, rO, rH0, rH1, uO, uH0, uH1, L, w;
};

__device__ __forceinline__ RigidFrame rigid_frame(float3 o, float3 h0, float3 h1, float3 vo, float3 vh0,
                                                  float3 vh1, const BoxDev& b) {
    const float mo = OPC_O_MASS, mh = OPC_H_MASS, mt = OPC_MASS_MOL;
    RigidFrame f;
    const float3 h0l = o + min_image_rint(h0 - o, b);
    const float3 h1l = o + min_image_rint(h1 - o, b);
    f.rcom = (o * mo + h0l * mh + h1l * mh) * (1.0f / mt);
    f.vcom = (vo * mo + vh0 * mh + vh1 * mh) * (1.0f / mt);
    f.rO = o - f.rcom; f.rH0 = h0l - f.rcom; f.rH1 = h1l - f.rcom;
    f.uO = vo - f.vcom; f.uH0 = vh0 - f.vcom; f.uH1 = vh1 - f.vcom;
    f.L = cross3(f.rO, f.uO) * mo + cross3(f.rH0, f.uH0) * mh + cross3(f.rH1, f.uH1) * mh;
    float ixx = 0.f, iyy = 0.f, izz = 0.f, ixy = 0.f, ixz = 0.f, iyz = 0.f;
    const float3 rs[3] = {f.rO, f.rH0, f.rH1};
    const float ms[3] = {mo, mh, mh};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float3 r = rs[k];
        const float m = ms[k];
        const float r2 = dot3(r, r);
        ixx += m * (r2 - r.x * r.x); iyy += m * (r2 - r.y * r.y); izz += m * (r2 - r.z * r.z);
        ixy += -m * r.x * r.y; ixz += -m * r.x * r.z; iyz += -m * r.y * r.z;
    }
    // solve_symmetric3 (src/solvent/opc_settle.rs:69-95)
    const float det = ixx * (iyy * izz - iyz * iyz) - ixy * (ixy * izz - iyz * ixz) +
                      ixz * (ixy * iyz - iyy * ixz);
    f.w = f3(0.f, 0.f, 0.f);
    if (fabsf(det) >= 1e-12f) {
        const float id = 1.0f / det;
        const float i00 = (iyy * izz - iyz * iyz) * id, i01 = (ixz * iyz - ixy * izz) * id;
        const float i02 = (ixy * iyz - ixz * iyy) * id, i11 = (ixx * izz - ixz * ixz) * id;
        const float i12 = (ixz * ixy - ixx * iyz) * id, i22 = (ixx * iyy - ixy * ixy) * id;
        const float3 L = f.L;
        f.w = f3(i00 * L.x + i01 * L.y + i02 * L.z, i01 * L.x + i11 * L.y + i12 * L.z,
                 i02 * L.x + i12 * L.y + i22 * L.z);
    }
    return f;
}

// Rigid drift of one water (src/solvent/opc_settle.rs:107-198).
__device__ void rigid_drift(float3& o, float3& h0, float3& h1, float3& vo, float3& vh0, float3& vh1,
                            float dt, const BoxDev& b) {
    const RigidFrame fr = rigid_frame(o, h0, h1, vo, vh0, vh1, b);
    const float3 rcom = fr.rcom, vcom = fr.vcom, rO = fr.rO, rH0 = fr.rH0, rH1 = fr.rH1, w = fr.w;
    const float3 delta = vcom * dt;
    const float3 rO2 = rodrigues(rO, w, dt), rH02 = rodrigues(rH0, w, dt), rH12 = rodrigues(rH1, w, dt);
    const float3 no = wrap_pos(rcom + delta + rO2, b);
    h0 = no + min_image_rint(rcom + delta + rH02 - no, b);
    h1 = no + min_image_rint(rcom + delta + rH12 - no, b);
    o = no;
    vo = vcom + cross3(w, rO2);
    vh0 = vcom + cross3(w, rH02);
    vh1 = vcom + cross3(w, rH12);
}

__device__ __forceinline__ float3 m_site(float3 o, float3 h0, float3 h1) {
    const float3 bis = (h0 - o) + (h1 - o);
    return o + bis * (OPC_O_EP_R * rsqrtf(dot3(bis, bis)));
}

__device__ __forceinline__ bool finite3(float3 a) {
    return isfinite(a.x) && isfinite(a.y) && isfinite(a.z);
}

// ---------------------------------------------------------------------------
// first half of the step
// ---------------------------------------------------------------------------
DYN_KERNEL(, k_water_first, (, float dt), (, dt)) {
    const BoxDev b = *v.box;
    const uint64_t step = v.sc->step;
    const bool lm = v.integrator == DYN_INTEGRATOR_LANGEVIN_MIDDLE;
    const float c = expf(-v.gamma * dt);
    const float num = KB_NATIVE * v.temperature * fmaxf(1.0f - c * c, 0.f);
    const float sg_o = sqrtf(num / OPC_O_MASS), sg_h = sqrtf(num / OPC_H_MASS);
    for (uint32_t s = bk.idx * blockDim.x + threadIdx.x; s < v.nw_cap; s += bk.cnt * blockDim.x) {
        const uint32_t id = v.wid[s];
        if (id == INVALID_ID) continue;
        float3 o = xyz(v.wpos[4 * s]), h0 = xyz(v.wpos[4 * s + 1]), h1 = xyz(v.wpos[4 * s + 2]);
        float3 vo = xyz(v.wvel[3 * s]), vh0 = xyz(v.wvel[3 * s + 1]), vh1 = xyz(v.wvel[3 * s + 2]);
        const float hk = 0.5f * dt;
        vo = vo + xyz(v.wacc[3 * s]) * hk;
        vh0 = vh0 + xyz(v.wacc[3 * s + 1]) * hk;
        vh1 = vh1 + xyz(v.wacc[3 * s + 2]) * hk;
        if (lm) {
            rigid_drift(o, h0, h1, vo, vh0, vh1, hk, b);
            const uint32_t pid = v.na + 3 * id;
            vo = vo * c + ou_normals(pid, step, v.seed) * sg_o;
            vh0 = vh0 * c + ou_normals(pid + 1, step, v.seed) * sg_h;
            vh1 = vh1 * c + ou_normals(pid + 2, step, v.seed) * sg_h;
            rigid_drift(o, h0, h1, vo, vh0, vh1, hk, b);
        } else {
            rigid_drift(o, h0, h1, vo, vh0, vh1, dt, b);
        }
        const float3 m = m_site(o, h0, h1);
        v.wpos[4 * s + 0] = make_float4(o.x, o.y, o.z, 0.f);
        v.wpos[4 * s + 1] = make_float4(h0.x, h0.y, h0.z, OPC_Q_H);
        v.wpos[4 * s + 2] = make_float4(h1.x, h1.y, h1.z, OPC_Q_H);
        v.wpos[4 * s + 3] = make_float4(m.x, m.y, m.z, OPC_Q_EP);
        v.wvel[3 * s + 0] = make_float4(vo.x, vo.y, vo.z, 0.f);
        v.wvel[3 * s + 1] = make_float4(vh0.x, vh0.y, vh0.z, 0.f);
        v.wvel[3 * s + 2] = make_float4(vh1.x, vh1.y, vh1.z, 0.f);
        if (!finite3(o)) v.sc->nonfinite = 1u;
    }
}

// ---------------------------------------------------------------------------
// constraint units: a heavy atom (slot 0) and the H constrained to it
// (slots 1..n-1), processed by one thread so the reference's sequential
// constraint loops run unchanged on each unit (src/bonded.rs:141-304)
// ---------------------------------------------------------------------------
struct Unit {
    int n;
    uint32_t id[UMAX];
    float3 x[UMAX], vel[UMAX];
    float m[UMAX], r02[UMAX];
    bool fixed[UMAX];
};

__device__ __forceinline__ void load_unit(const SysView& v, uint32_t u, Unit& U) {
    const uint32_t b = v.unit_off[u], e = v.unit_off[u + 1];
    U.n = (int)(e - b);
#pragma unroll
    for (int k = 0; k < UMAX; ++k) {
        if (k >= U.n) break;
        const uint32_t a = v.unit_idx[b + k];
        U.id[k] = a;
        U.x[k] = xyz(v.apos[a]);
        U.vel[k] = xyz(v.avel[a]);
        U.m[k] = v.amass[a];
        U.r02[k] = v.unit_r02[b + k];
        U.fixed[k] = v.astatic && v.astatic[a];
    }
}

// lincs_hydrogens (src/bonded.rs:218-284): order projection passes along the
// bond, then iter SHAKE-style passes; returns the constraint virial
// sum r_ij . f_i (native units) with f_i the heavy atom's displacement times
// m / dt^2 (the reference's estimate, :273-283)
__device__ __forceinline__ double constrain_unit(Unit& U, uint32_t order, uint32_t iter, float inv_dt2) {
    if (U.n < 2) return 0.0;
    const float3 x0 = U.x[0];
    for (uint32_t o = 0; o < order; ++o) {
#pragma unroll
        for (int k = 1; k < UMAX; ++k) {
            if (k >= U.n) break;
            const float3 d = U.x[k] - U.x[0];
            const float dl = fmaxf(sqrtf(dot3(d, d)), 1.1920929e-7f);
            const float3 bv = d * (1.0f / dl);
            const float im = 1.0f / U.m[0] + 1.0f / U.m[k];
            const float lam = (sqrtf(U.r02[k]) - dot3(bv, d)) / im;
            const float3 corr = bv * lam;
            if (!U.fixed[0]) U.x[0] = U.x[0] - corr * (1.0f / U.m[0]);
            if (!U.fixed[k]) U.x[k] = U.x[k] + corr * (1.0f / U.m[k]);
        }
    }
    for (uint32_t it = 0; it < iter; ++it) {
#pragma unroll
        for (int k = 1; k < UMAX; ++k) {
            if (k >= U.n) break;
            const float3 d = U.x[k] - U.x[0];
            const float d2 = dot3(d, d);
            const float im = 1.0f / U.m[0] + 1.0f / U.m[k];
            const float lam = (d2 - U.r02[k]) / (2.0f * im * fmaxf(d2, 1e-8f));
            const float3 corr = d * lam;
            if (!U.fixed[0]) U.x[0] = U.x[0] + corr * (1.0f / U.m[0]);
            if (!U.fixed[k]) U.x[k] = U.x[k] - corr * (1.0f / U.m[k]);
        }
    }
    const float3 fi = (U.x[0] - x0) * (U.m[0] * inv_dt2);
    double w = 0.0;
#pragma unroll
    for (int k = 1; k < UMAX; ++k)
        if (k < U.n) w += (double)dot3(U.x[k] - U.x[0], fi);
    return w;
}

// rattle_hydrogens (src/bonded.rs:288-304): remove the velocity component
// along each constrained bond
__device__ __forceinline__ void rattle_unit(Unit& U) {
#pragma unroll
    for (int k = 1; k < UMAX; ++k) {
        if (k >= U.n) break;
        const float3 r = U.x[k] - U.x[0];
        const float3 dv = U.vel[k] - U.vel[0];
        const float r2 = dot3(r, r);
        const float im = 1.0f / U.m[0] + 1.0f / U.m[k];
        const float lam = dot3(dv, r) / (im * fmaxf(r2, 1e-8f));
        const float3 corr = r * lam;
        U.vel[0] = U.vel[0] + corr * (1.0f / U.m[0]);
        U.vel[k] = U.vel[k] - corr * (1.0f / U.m[k]);
    }
}

// First half for non-water atoms, one constraint unit per thread:
// Langevin-middle kick dt/2 + drift dt/2, constrain + rattle, OU, rattle,
// drift dt/2, constrain (src/integrate.rs:100-160,478-511,566-587);
// velocity Verlet kick dt/2 + drift dt, constrain + rattle.  The constraint
// virial of the first projection (dt/2) is the step's (src/integrate.rs:105-165).
// RATTLE (Andersen, J. Comput. Phys. 52, 24 (1983)), used with
// DYN_FLAG_RATTLE_VELOCITIES.  Position stage: SHAKE iterations with the
// corrections along the bond vectors at the start of the drift (xr), which
// makes the map symplectic, until every |d|^2 is within 1e-6 of r0^2 (at
// most RATTLE_SWEEPS sweeps); the velocities then follow the displacement
// (v += dx / t_drift).  Velocity stage: the projection of rattle_unit,
// repeated so that the coupled bonds of a unit (CH3, NH3) all hold.
constexpr int RATTLE_SWEEPS = 32;

__device__ __forceinline__ double shake_unit(Unit& U, const float3 (&xr)[UMAX], float inv_dt2) {
    if (U.n < 2) return 0.0;
    const float3 x0 = U.x[0];
    for (int it = 0; it < RATTLE_SWEEPS; ++it) {
        bool done = true;
#pragma unroll
        for (int k = 1; k < UMAX; ++k) {
            if (k >= U.n) break;
            const float3 d = U.x[k] - U.x[0];
            const float diff = dot3(d, d) - U.r02[k];
            if (fabsf(diff) > 1e-6f * U.r02[k]) done = false;
            const float3 ro = xr[k] - xr[0];
            const float im = 1.0f / U.m[0] + 1.0f / U.m[k];
            const float g = diff / (2.0f * im * dot3(d, ro));
            const float3 corr = ro * g;
            if (!U.fixed[0]) U.x[0] = U.x[0] + corr * (1.0f / U.m[0]);
            if (!U.fixed[k]) U.x[k] = U.x[k] - corr * (1.0f / U.m[k]);
        }
        if (done) break;
    }
    const float3 fi = (U.x[0] - x0) * (U.m[0] * inv_dt2);
    double w = 0.0;
#pragma unroll
    for (int k = 1; k < UMAX; ++k)
        if (k < U.n) w += (double)dot3(U.x[k] - U.x[0], fi);
    return w;
}

__device__ __forceinline__ void follow_constraint(Unit& U, const float3 (&xu)[UMAX], float inv_t) {
#pragma unroll
    for (int k = 0; k < UMAX; ++k)
        if (k < U.n && !U.fixed[k]) U.vel[k] = U.vel[k] + (U.x[k] - xu[k]) * inv_t;
}

__device__ __forceinline__ void rattle_unit_converged(Unit& U) {
    if (U.n < 2) return;
    const int sweeps = U.n > 2 ? 8 : 1;  // one bond: the projection is exact
    for (int it = 0; it < sweeps; ++it) rattle_unit(U);
}

DYN_KERNEL(, k_atom_first, (, float dt), (, dt)) {
    const uint64_t step = v.sc->step;
    const bool lm = v.integrator == DYN_INTEGRATOR_LANGEVIN_MIDDLE;
    const bool rv = (v.flags & DYN_FLAG_RATTLE_VELOCITIES) != 0u;
    const float c = expf(-v.gamma * dt);
    const float num = KB_NATIVE * v.temperature * fmaxf(1.0f - c * c, 0.f);
    const float hk = 0.5f * dt;
    const float inv_dt2 = 1.0f / (hk * hk);
    const float t_drift = lm ? hk : dt;
    const float inv_td = 1.0f / t_drift, inv_hk = 1.0f / hk;
    double vir = 0.0;
    for (uint32_t u = bk.idx * blockDim.x + threadIdx.x; u < v.nunit; u += bk.cnt * blockDim.x) {
        Unit U;
        load_unit(v, u, U);
        float3 xr[UMAX], xu[UMAX];  // positions at the start of a drift, before its constraint pass
#pragma unroll
        for (int k = 0; k < UMAX; ++k) {
            if (k >= U.n) break;
            xr[k] = U.x[k];
            if (!U.fixed[k]) {
                U.vel[k] = U.vel[k] + xyz(v.aacc[U.id[k]]) * hk;
                U.x[k] = U.x[k] + U.vel[k] * t_drift;
            }
            xu[k] = U.x[k];
        }
        if (rv) {
            vir += shake_unit(U, xr, inv_dt2);
            follow_constraint(U, xu, inv_td);
        } else {
            vir += constrain_unit(U, v.lincs_order, v.lincs_iter, inv_dt2);
            rattle_unit(U);
        }
        if (lm) {
#pragma unroll
            for (int k = 0; k < UMAX; ++k) {
                if (k >= U.n) break;
                if (U.fixed[k]) continue;
                const float sg = sqrtf(num / U.m[k]);
                U.vel[k] = U.vel[k] * c + ou_normals(U.id[k], step, v.seed) * sg;
            }
            // the noise, projected onto the constraints
            if (rv) rattle_unit_converged(U);
            else rattle_unit(U);
#pragma unroll
            for (int k = 0; k < UMAX; ++k) {
                if (k >= U.n) break;
                xr[k] = U.x[k];
                if (!U.fixed[k]) U.x[k] = U.x[k] + U.vel[k] * hk;
                xu[k] = U.x[k];
            }
            if (rv) {
                shake_unit(U, xr, inv_dt2);
                follow_constraint(U, xu, inv_hk);
            } else {
                constrain_unit(U, v.lincs_order, v.lincs_iter, inv_dt2);
            }
        }
#pragma unroll
        for (int k = 0; k < UMAX; ++k) {
            if (k >= U.n) break;
            const uint32_t a = U.id[k];
            if (U.fixed[k]) continue;
            v.apos[a] = make_float4(U.x[k].x, U.x[k].y, U.x[k].z, v.apos[a].w);
            v.avel[a] = make_float4(U.vel[k].x, U.vel[k].y, U.vel[k].z, 0.f);
            if (!finite3(U.x[k])) v.sc->nonfinite = 1u;
        }
    }
    double x[1] = {vir};
    block_sum_d<1>(x);
    if (threadIdx.x == 0) {
        double* p = v.partials + ((size_t)REG_CONS * v.max_blocks + bk.idx) * 4;
        p[0] = x[0]; p[1] = 0.0; p[2] = 0.0; p[3] = 0.0;
    }
}

// ---------------------------------------------------------------------------
// second half: forces -> accelerations -> kick, KE partials
// ---------------------------------------------------------------------------
__device__ __forceinline__ float3 ldfix3(const long long* p) {
    return f3((float)((double)p[0] * DYN_FIX_INV), (float)((double)p[1] * DYN_FIX_INV),
              (float)((double)p[2] * DYN_FIX_INV));
}
__device__ __forceinline__ float3 ldfix3sum(const long long* p, const long long* q) {
    return f3((float)((double)(p[0] + q[0]) * DYN_FIX_INV), (float)((double)(p[1] + q[1]) * DYN_FIX_INV),
              (float)((double)(p[2] + q[2]) * DYN_FIX_INV));
}

// Besides the reference's KE (every site velocity after the kick,
// src/integrate.rs:561) this accumulates the rigid-body KE the next drift
// keeps (M v_com^2 + omega . L), and the intramolecular virial
// sum_s (r_s - R_com) . F_s, which turns the site virial into the molecular
// virial a rigid-water pressure needs.
DYN_KERNEL(, k_water_kick, (, float dt), (, dt)) {
    const BoxDev b = *v.box;
    double ke = 0.0, ket = 0.0, ker = 0.0, wi = 0.0;
    for (uint32_t s = bk.idx * blockDim.x + threadIdx.x; s < v.nw_cap; s += bk.cnt * blockDim.x) {
        const uint32_t id = v.wid[s];
        if (id == INVALID_ID) continue;
        const long long* f = v.wforce + (size_t)s * 12;
        const long long* r = v.wrecip + (size_t)id * 9;
        const float3 fo = ldfix3(f);
        const float3 fh0 = ldfix3sum(f + 3, r + 0);
        const float3 fh1 = ldfix3sum(f + 6, r + 3);
        const float3 fm = ldfix3sum(f + 9, r + 6);
        // project_ep_force (src/solvent/mod.rs:397-406)
        const float3 ao = (fo + fm * OPC_C_O) * (KCAL_TO_NATIVE / OPC_O_MASS);
        const float3 ah0 = (fh0 + fm * OPC_C_H) * (KCAL_TO_NATIVE / OPC_H_MASS);
        const float3 ah1 = (fh1 + fm * OPC_C_H) * (KCAL_TO_NATIVE / OPC_H_MASS);
        const float hk = 0.5f * dt;
        const float3 vo = xyz(v.wvel[3 * s]) + ao * hk;
        const float3 vh0 = xyz(v.wvel[3 * s + 1]) + ah0 * hk;
        const float3 vh1 = xyz(v.wvel[3 * s + 2]) + ah1 * hk;
        v.wacc[3 * s + 0] = make_float4(ao.x, ao.y, ao.z, 0.f);
        v.wacc[3 * s + 1] = make_float4(ah0.x, ah0.y, ah0.z, 0.f);
        v.wacc[3 * s + 2] = make_float4(ah1.x, ah1.y, ah1.z, 0.f);
        v.wvel[3 * s + 0] = make_float4(vo.x, vo.y, vo.z, 0.f);
        v.wvel[3 * s + 1] = make_float4(vh0.x, vh0.y, vh0.z, 0.f);
        v.wvel[3 * s + 2] = make_float4(vh1.x, vh1.y, vh1.z, 0.f);
        ke += (double)(OPC_O_MASS * dot3(vo, vo)) + (double)(OPC_H_MASS * dot3(vh0, vh0)) +
              (double)(OPC_H_MASS * dot3(vh1, vh1));
        const float3 po = xyz(v.wpos[4 * s]);
        const RigidFrame fr = rigid_frame(po, xyz(v.wpos[4 * s + 1]), xyz(v.wpos[4 * s + 2]), vo, vh0, vh1, b);
        ket += (double)(OPC_MASS_MOL * dot3(fr.vcom, fr.vcom));
        ker += (double)(OPC_MASS_MOL * dot3(fr.vcom, fr.vcom)) + (double)dot3(fr.w, fr.L);
        const float3 rm = po + min_image_rint(xyz(v.wpos[4 * s + 3]) - po, b) - fr.rcom;
        wi += (double)dot3(fr.rO, fo) + (double)dot3(fr.rH0, fh0) + (double)dot3(fr.rH1, fh1) +
              (double)dot3(rm, fm);
        if (!finite3(ao) || !finite3(ah0) || !finite3(ah1)) v.sc->nonfinite = 1u;
    }
    double x[4] = {ke, ket, ker, wi};
    block_sum_d<4>(x);
    if (threadIdx.x == 0) {
        double* p = v.partials + ((size_t)REG_KICK_W * v.max_blocks + bk.idx) * 4;
        p[0] = x[0]; p[1] = x[1]; p[2] = x[2]; p[3] = x[3];
    }
}

DYN_KERNEL(, k_atom_kick, (, float dt), (, dt)) {
    double ke = 0.0;
    for (uint32_t u = bk.idx * blockDim.x + threadIdx.x; u < v.nunit; u += bk.cnt * blockDim.x) {
        Unit U;
        load_unit(v, u, U);
#pragma unroll
        for (int k = 0; k < UMAX; ++k) {
            if (k >= U.n) break;
            if (U.fixed[k]) continue;
            const uint32_t a = U.id[k];
            const float3 f = ldfix3sum(v.aforce + 3 * (size_t)a, v.arecip + 3 * (size_t)a);
            // kick_and_calc_accel with the MAX_ACCEL clamp (src/integrate.rs:521-535)
            float3 acc = f * (KCAL_TO_NATIVE / U.m[k]);
            const float a2 = dot3(acc, acc);
            if (a2 > MAX_ACCEL * MAX_ACCEL) acc = acc * (MAX_ACCEL * rsqrtf(a2));
            U.vel[k] = U.vel[k] + acc * (0.5f * dt);
            v.aacc[a] = make_float4(acc.x, acc.y, acc.z, 0.f);
            if (!finite3(acc)) v.sc->nonfinite = 1u;
        }
        // src/integrate.rs:554-559
        if (v.flags & DYN_FLAG_RATTLE_VELOCITIES) rattle_unit_converged(U);
        else rattle_unit(U);
#pragma unroll
        for (int k = 0; k < UMAX; ++k) {
            if (k >= U.n) break;
            if (U.fixed[k]) continue;
            v.avel[U.id[k]] = make_float4(U.vel[k].x, U.vel[k].y, U.vel[k].z, 0.f);
            ke += (double)(U.m[k] * dot3(U.vel[k], U.vel[k]));
        }
    }
    double x[2] = {ke, ke};
    block_sum_d<2>(x);
    if (threadIdx.x == 0) {
        double* p = v.partials + ((size_t)REG_KICK_A * v.max_blocks + bk.idx) * 4;
        p[0] = x[0]; p[1] = x[1]; p[2] = x[0]; p[3] = 0.0;
    }
}

// ---------------------------------------------------------------------------
// finalize: fixed-order sums of all partials, pressure, temperature, CSVR
// and C-rescale scalars (single block)
// ---------------------------------------------------------------------------
__device__ double gamma_mt(double shape, uint64_t step, uint64_t seed) {
    // Marsaglia & Tsang (ACM TOMS 26, 2000); bounded attempts.
    const double d = shape - 1.0 / 3.0;
    const double c = 1.0 / sqrt(9.0 * d);
    for (uint32_t a = 0; a < 64; ++a) {
        const Philox4 r = philox4x32(a + 1, (uint32_t)step, DYN_STREAM_CSVR, (uint32_t)(step >> 32),
                                     (uint32_t)seed, (uint32_t)(seed >> 32));
        const double u1 = uniform24d(r.x[0]), u2 = uniform24d(r.x[1]);
        const double x = sqrt(-2.0 * log(u1)) * cos(2.0 * M_PI * u2);
        const double vv = (1.0 + c * x) * (1.0 + c * x) * (1.0 + c * x);
        if (vv <= 0.0) continue;
        const double u = uniform24d(r.x[2]);
        if (log(u) < 0.5 * x * x + d - d * vv + d * log(vv)) return d * vv;
    }
    return d;
}

DYN_KERNEL_T((bool ENERGY), (ENERGY), , k_finalize, (, float dt, bool thermo), (, dt, thermo)) {
    // one warp per region, all regions' partials in flight at once; each
    // region's sum has a fixed order
    __shared__ double rs[NREGION][4];
    // the thermostat's and barostat's random numbers depend only on the
    // step and the seed: two otherwise idle warps draw them while the
    // others reduce the partials
    __shared__ double rnd[4];  // CSVR normal, CSVR chi^2, exp(-dt/tau_t), barostat normal
    const bool csvr_on = thermo && v.integrator == DYN_INTEGRATOR_VERLET_VELOCITY &&
                         v.thermostat == DYN_THERMO_CSVR && v.tau_t > 0.f;
    const bool baro_on = thermo && v.barostat == DYN_BARO_CRESCALE && v.tau_p > 0.f;
    {
        const uint32_t wr = threadIdx.x >> 5;
        const uint32_t w_csvr = NREGION % (blockDim.x >> 5), w_baro = (NREGION + 1) % (blockDim.x >> 5);
        const uint64_t step = v.sc->step;
        if (csvr_on && wr == w_csvr && (threadIdx.x & 31) == 0) {
            const double dof = (double)(v.thermo_dof > 2 ? v.thermo_dof : 2);
            const Philox4 r = philox4x32(0u, (uint32_t)step, DYN_STREAM_CSVR, (uint32_t)(step >> 32),
                                         (uint32_t)v.seed, (uint32_t)(v.seed >> 32));
            rnd[0] = sqrt(-2.0 * log(uniform24d(r.x[0]))) * cos(2.0 * M_PI * uniform24d(r.x[1]));
            rnd[1] = 2.0 * gamma_mt(0.5 * (dof - 1.0), step, v.seed);
            rnd[2] = exp(-(double)dt / (double)v.tau_t);
        }
        if (baro_on && wr == w_baro && (threadIdx.x & 31) == 0) {
            const Philox4 r = philox4x32(0u, (uint32_t)step, DYN_STREAM_BARO, (uint32_t)(step >> 32),
                                         (uint32_t)v.seed, (uint32_t)(v.seed >> 32));
            rnd[3] = sqrt(-2.0 * log(uniform24d(r.x[0]))) * cos(2.0 * M_PI * uniform24d(r.x[1]));
        }
    }
    {
        const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
        for (int reg = w; reg < NREGION; reg += (int)(blockDim.x >> 5)) {
            double o[4] = {0.0, 0.0, 0.0, 0.0};
            const bool used = reg == REG_WW || reg == REG_KICK_W ||
                              (v.na && (reg == REG_SS || reg == REG_14 || reg == REG_BOND ||
                                        reg == REG_KICK_A || reg == REG_CONS || (v.nw && reg == REG_WS)));
            if (used) {
                const double4* p = reinterpret_cast<const double4*>(v.partials) + (size_t)reg * v.max_blocks;
                const uint32_t n = v.nb[reg];
                uint32_t i = lane;
                for (; i + 96 < n; i += 128) {
                    const double4 a = p[i], b = p[i + 32], c = p[i + 64], d = p[i + 96];
                    o[0] += a.x; o[1] += a.y; o[2] += a.z; o[3] += a.w;
                    o[0] += b.x; o[1] += b.y; o[2] += b.z; o[3] += b.w;
                    o[0] += c.x; o[1] += c.y; o[2] += c.z; o[3] += c.w;
                    o[0] += d.x; o[1] += d.y; o[2] += d.z; o[3] += d.w;
                }
                for (; i < n; i += 32) {
                    const double4 a = p[i];
                    o[0] += a.x; o[1] += a.y; o[2] += a.z; o[3] += a.w;
                }
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) o[k] = warp_sum_d(o[k]);
            if (lane == 0)
                for (int k = 0; k < 4; ++k) rs[reg][k] = o[k];
        }
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    const double* ww = rs[REG_WW];
    const double* ws = rs[REG_WS];
    const double* ss = rs[REG_SS];
    const double* p14 = rs[REG_14];
    const double* bo = rs[REG_BOND];
    const double* kw = rs[REG_KICK_W];
    const double* ka = rs[REG_KICK_A];
    const double* co = rs[REG_CONS];
    const double x[16] = {ww[0], ww[1], ww[2], ws[0] + ss[0], ws[1] + ss[1],
                          ws[2] + ss[2], p14[0], p14[2], bo[0], bo[2], kw[0] + ka[0],
                          kw[1] + ka[1], co[0], kw[2] + ka[2], kw[3], 0};
    Scalars* sc = v.sc;
    // every list (water-water half lists, atom cluster pairs) counts each
    // pair once
    if (ENERGY) {
        sc->acc[ACC_E_LJ_WW] = x[0];
        sc->acc[ACC_E_COUL_WW] = x[1];
        sc->acc[ACC_E_LJ_S] = x[3];
        sc->acc[ACC_E_COUL_S] = x[4];
        sc->acc[ACC_E_14] = x[6];
        sc->acc[ACC_E_BONDED] = x[8];
        // alchemical dH/dlambda: short-range cross pairs + SPME cross term
        sc->dh_dl = ws[3] + ss[3] + sc->recip_dh_cache;
    }
    sc->acc[ACC_VIR_SHORT] = x[2] + x[5] + x[7];
    sc->acc[ACC_VIR_14] = x[7];
    sc->acc[ACC_VIR_BONDED] = x[9];
    sc->acc[ACC_VIR_CONSTR] = x[12];
    sc->acc[ACC_E_RECIP] = sc->recip_cache[0];
    sc->acc[ACC_VIR_RECIP] = sc->recip_cache[1];
    sc->acc[ACC_E_CORR] = sc->recip_cache[2];
    sc->acc[ACC_VIR_CORR] = sc->recip_cache[3];
    const double to_kcal = 0.5 / (double)KCAL_TO_NATIVE;
    double ke = x[10] * to_kcal, ket = x[11] * to_kcal, ker = x[13] * to_kcal;
    const double w_intra = x[14];
    // CSVR (src/thermostat.rs:258-304) after the final kick of velocity Verlet
    sc->csvr_lambda = 1.0;
    if (csvr_on && ker > 1e-20) {
        const double dof = (double)(v.thermo_dof > 2 ? v.thermo_dof : 2);
        const double rn = rnd[0], chi = rnd[1], cc = rnd[2];
        const double ket_target = 0.5 * dof * GAS_CONST_R * (double)v.temperature;
        // the thermostat acts on the rigid-body KE (the degrees of freedom
        // that survive the next rigid drift), not the kicked site velocities
        double kp = ker * cc + ket_target * (1.0 - cc) * ((chi + rn * rn) / dof) +
                    2.0 * rn * sqrt(cc * (1.0 - cc) * ker * ket_target / dof);
        kp = kp > 1e-20 ? kp : 1e-20;
        const double lam = sqrt(kp / ker);
        sc->csvr_lambda = lam;
        ke *= lam * lam;
        ket *= lam * lam;
        ker *= lam * lam;
    }
    sc->acc[ACC_KE] = ke;
    sc->acc[ACC_KE_TRANS] = ket;
    sc->ke_rigid = ker;
    const BoxDev b = *v.box;
    const double vol = (double)b.ext[0] * b.ext[1] * b.ext[2];
    const double vir = sc->acc[ACC_VIR_SHORT] + sc->acc[ACC_VIR_RECIP] + sc->acc[ACC_VIR_CORR] +
                       sc->acc[ACC_VIR_BONDED] + sc->acc[ACC_VIR_CONSTR] / (double)KCAL_TO_NATIVE;
    // reference formula (src/barostat.rs:419-431): COM KE with the site virial
    sc->pressure_atomic = (2.0 * ket + vir) / (3.0 * vol) * BAR_PER_KCAL_MOL_A3;
    // molecular virial for the rigid waters: the barostat's pressure
    sc->pressure = (2.0 * ket + vir - w_intra) / (3.0 * vol) * BAR_PER_KCAL_MOL_A3;
    sc->temperature = v.thermo_dof ? 2.0 * ker / ((double)v.thermo_dof * GAS_CONST_R) : 0.0;
    // C-rescale (Bernetti & Bussi, J. Chem. Phys. 153, 114107 (2020))
    sc->baro_mu = 1.0;
    if (baro_on) {
        const double xi = rnd[3];
        const double kap = v.kappa, tau = v.tau_p;
        const double det = kap / tau * (sc->pressure - (double)v.p_target) * dt;
        const double sig = sqrt(2.0 * kap * KB_BAR_A3 * (double)v.temperature * dt / (tau * vol));
        double dl = det + sig * xi;
        dl = dl > 0.1 ? 0.1 : (dl < -0.1 ? -0.1 : dl);
        sc->baro_mu = exp(dl / 3.0);
    }
    if (ENERGY) {
        double pe;
        if (v.flags & DYN_FLAG_FULL_ENERGY)
            pe = sc->acc[ACC_E_LJ_WW] + sc->acc[ACC_E_COUL_WW] + sc->acc[ACC_E_LJ_S] +
                 sc->acc[ACC_E_COUL_S] + sc->acc[ACC_E_14] + sc->acc[ACC_E_RECIP] +
                 sc->acc[ACC_E_CORR] + sc->acc[ACC_E_BONDED];
        else
            pe = sc->acc[ACC_E_LJ_S] + sc->acc[ACC_E_COUL_S] + sc->acc[ACC_E_14] +
                 sc->acc[ACC_E_RECIP] + sc->acc[ACC_E_CORR] + sc->acc[ACC_E_BONDED];
        sc->pe = pe;
    }
    if (thermo) {
        // the step is complete; the periodic tasks that follow see its number
        const uint64_t next = sc->step + 1;
        unsigned int due = 0u;
        if ((v.flags & DYN_FLAG_COM_REMOVAL) && v.com_interval && next % v.com_interval == 0) due = 1u;
        if ((v.flags & DYN_FLAG_RECENTER) && v.recenter_interval && v.na && next % v.recenter_interval == 0)
            due = 1u;
        if ((v.flags & DYN_FLAG_RESET_ANGLE) && v.nw && next % 1000 == 0) due = 1u;
        if (v.snap_ratio && next % v.snap_ratio == 0) due = 1u;
        sc->step = next;
        sc->time_ps += (double)dt;
        if (v.use_cond && due) cudaGraphSetConditional(v.cond_periodic, 1u);
    }
}

// velocity scaling (CSVR) and C-rescale of positions / box
DYN_KERNEL(, k_scale, (), ()) {
    const double lam_d = v.sc->csvr_lambda, mu_d = v.sc->baro_mu;
    if (lam_d == 1.0 && mu_d == 1.0) return;
    const float lam = (float)lam_d, mu = (float)mu_d;
    const BoxDev b = *v.box;
    const float3 cen = f3(b.lo[0] + 0.5f * b.ext[0], b.lo[1] + 0.5f * b.ext[1], b.lo[2] + 0.5f * b.ext[2]);
    const float vs = lam / mu;  // C-rescale scales momenta by 1/mu
    const uint32_t tid = bk.idx * blockDim.x + threadIdx.x, stride = bk.cnt * blockDim.x;
    for (uint32_t s = tid; s < v.nw_cap; s += stride) {
        if (v.wid[s] == INVALID_ID) continue;
        for (int k = 0; k < 3; ++k) {
            float4 q = v.wvel[3 * s + k];
            q.x *= vs; q.y *= vs; q.z *= vs;
            v.wvel[3 * s + k] = q;
        }
        if (mu != 1.0f) {
            // rigid molecules: move the COM, keep the geometry
            const float3 o = xyz(v.wpos[4 * s]);
            const float3 h0 = o + min_image_rint(xyz(v.wpos[4 * s + 1]) - o, b);
            const float3 h1 = o + min_image_rint(xyz(v.wpos[4 * s + 2]) - o, b);
            const float3 com = (o * OPC_O_MASS + h0 * OPC_H_MASS + h1 * OPC_H_MASS) * (1.0f / OPC_MASS_MOL);
            const float3 sh = (com - cen) * (mu - 1.0f);
            for (int k = 0; k < 4; ++k) {
                float4 q = v.wpos[4 * s + k];
                q.x += sh.x; q.y += sh.y; q.z += sh.z;
                v.wpos[4 * s + k] = q;
            }
        }
    }
    for (uint32_t a = tid; a < v.na; a += stride) {
        if (v.astatic && v.astatic[a]) continue;
        float4 q = v.avel[a];
        q.x *= vs; q.y *= vs; q.z *= vs;
        v.avel[a] = q;
        if (mu != 1.0f) {
            float4 p = v.apos[a];
            p.x = cen.x + (p.x - cen.x) * mu; p.y = cen.y + (p.y - cen.y) * mu; p.z = cen.z + (p.z - cen.z) * mu;
            v.apos[a] = p;
        }
    }
    if (mu_d == 1.0) return;
    // the box itself is scaled (about its centre) by the last block to
    // finish, after every block has read the old one
    __syncthreads();
    if (threadIdx.x != 0) return;
    __threadfence();
    if (atomicAdd(&v.sc->ctr_scale, 1u) != bk.cnt - 1) return;
    BoxDev nb = b;
    for (int k = 0; k < 3; ++k) {
        const double c = (double)b.lo[k] + 0.5 * (double)b.ext[k];
        const double e = (double)b.ext[k] * mu_d;
        nb.lo[k] = (float)(c - 0.5 * e);
        nb.ext[k] = (float)e;
        nb.inv_ext[k] = (float)(1.0 / e);
    }
    *v.box = nb;
    v.sc->ctr_scale = 0u;
}

// COM motion removal (src/com_zero.rs:57-81) every com_interval steps
DYN_KERNEL(, k_com_reduce, (), ()) {
    const uint64_t next = v.sc->step;  // advanced by k_finalize
    const bool on = (v.flags & DYN_FLAG_COM_REMOVAL) && v.com_interval && (next % v.com_interval == 0);
    double x[4] = {0, 0, 0, 0};
    if (on) {
        for (uint32_t s = bk.idx * blockDim.x + threadIdx.x; s < v.nw_cap; s += bk.cnt * blockDim.x) {
            if (v.wid[s] == INVALID_ID) continue;
            const float3 p = xyz(v.wvel[3 * s]) * OPC_O_MASS + xyz(v.wvel[3 * s + 1]) * OPC_H_MASS +
                             xyz(v.wvel[3 * s + 2]) * OPC_H_MASS;
            x[0] += p.x; x[1] += p.y; x[2] += p.z; x[3] += OPC_MASS_MOL;
        }
        for (uint32_t a = bk.idx * blockDim.x + threadIdx.x; a < v.na; a += bk.cnt * blockDim.x) {
            if (v.astatic && v.astatic[a]) continue;
            const float3 p = xyz(v.avel[a]) * v.amass[a];
            x[0] += p.x; x[1] += p.y; x[2] += p.z; x[3] += v.amass[a];
        }
    }
    block_sum_d<4>(x);
    if (threadIdx.x == 0) {
        double* p = v.partials + ((size_t)REG_COM * v.max_blocks + bk.idx) * 4;
        p[0] = x[0]; p[1] = x[1]; p[2] = x[2]; p[3] = x[3];
    }
}

DYN_KERNEL(, k_com_apply, (), ()) {
    const uint64_t next = v.sc->step;  // advanced by k_finalize
    const bool on = (v.flags & DYN_FLAG_COM_REMOVAL) && v.com_interval && (next % v.com_interval == 0);
    if (!on) return;
    __shared__ float3 vc;
    if (threadIdx.x < 32) {
        double x[4] = {0, 0, 0, 0};
        for (uint32_t i = threadIdx.x; i < v.nb[REG_COM]; i += 32) {
            const double* p = v.partials + ((size_t)REG_COM * v.max_blocks + i) * 4;
            x[0] += p[0]; x[1] += p[1]; x[2] += p[2]; x[3] += p[3];
        }
        for (int k = 0; k < 4; ++k) x[k] = warp_sum_d(x[k]);
        if (threadIdx.x == 0) {
            vc = x[3] > 1e-6 ? f3((float)(x[0] / x[3]), (float)(x[1] / x[3]), (float)(x[2] / x[3]))
                             : f3(0.f, 0.f, 0.f);
        }
    }
    __syncthreads();
    const float3 c = vc;
    for (uint32_t s = bk.idx * blockDim.x + threadIdx.x; s < v.nw_cap; s += bk.cnt * blockDim.x) {
        if (v.wid[s] == INVALID_ID) continue;
        for (int k = 0; k < 3; ++k) {
            float4 q = v.wvel[3 * s + k];
            q.x -= c.x; q.y -= c.y; q.z -= c.z;
            v.wvel[3 * s + k] = q;
        }
    }
    for (uint32_t a = bk.idx * blockDim.x + threadIdx.x; a < v.na; a += bk.cnt * blockDim.x) {
        if (v.astatic && v.astatic[a]) continue;
        float4 q = v.avel[a];
        q.x -= c.x; q.y -= c.y; q.z -= c.z;
        v.avel[a] = q;
    }
}

// SimBox::recenter (src/barostat.rs:111-137) every recenter_interval steps
DYN_KERNEL(, k_recenter, (), ()) {
    const uint64_t next = v.sc->step;  // advanced by k_finalize
    const bool on = (v.flags & DYN_FLAG_RECENTER) && v.recenter_interval && v.na &&
                    (next % v.recenter_interval == 0);
    if (!on) return;
    double x[4] = {0, 0, 0, 0};
    for (uint32_t a = threadIdx.x; a < v.na; a += blockDim.x) {
        if (v.astatic && v.astatic[a]) continue;
        const float4 p = v.apos[a];
        x[0] += p.x; x[1] += p.y; x[2] += p.z; x[3] += 1.0;
    }
    block_sum_d<4>(x);
    if (threadIdx.x == 0 && x[3] > 0.0) {
        BoxDev b = *v.box;
        for (int k = 0; k < 3; ++k) b.lo[k] = (float)(x[k] / x[3]) - 0.5f * b.ext[k];
        *v.box = b;
    }
}

// reset_angle (src/solvent/opc_settle.rs:202-219) every 1000 steps
DYN_KERNEL(, k_reset_angle, (), ()) {
    const uint64_t next = v.sc->step;  // advanced by k_finalize
    if (!(v.flags & DYN_FLAG_RESET_ANGLE) || next % 1000 != 0) return;
    const BoxDev b = *v.box;
    for (uint32_t s = bk.idx * blockDim.x + threadIdx.x; s < v.nw_cap; s += bk.cnt * blockDim.x) {
        if (v.wid[s] == INVALID_ID) continue;
        const float3 o = xyz(v.wpos[4 * s]);
        const float3 h0 = o + min_image_rint(xyz(v.wpos[4 * s + 1]) - o, b);
        const float3 h1 = o + min_image_rint(xyz(v.wpos[4 * s + 2]) - o, b);
        float3 u = h0 + h1 - o * 2.0f;
        u = u * rsqrtf(dot3(u, u));
        float3 w = h0 - h1;
        w = w * rsqrtf(dot3(w, w));
        w = w - u * dot3(u, w);
        w = w * rsqrtf(dot3(w, w));
        float sh, ch;
        sincosf(0.5f * OPC_HOH_THETA, &sh, &ch);
        const float3 n0 = o + (u * ch + w * sh) * OPC_O_H_R;
        const float3 n1 = o + (u * ch - w * sh) * OPC_O_H_R;
        const float3 m = m_site(o, n0, n1);
        v.wpos[4 * s + 1] = make_float4(n0.x, n0.y, n0.z, OPC_Q_H);
        v.wpos[4 * s + 2] = make_float4(n1.x, n1.y, n1.z, OPC_Q_H);
        v.wpos[4 * s + 3] = make_float4(m.x, m.y, m.z, OPC_Q_EP);
    }
}


// ---------------------------------------------------------------------------
// snapshots (MdState::handle_snapshots, src/snapshot.rs:753-833): after a
// step whose number is a multiple of snap_ratio, the state goes into frame
// snap_count % snap_cap of the device ring
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool snapshot_due(const SysView& v) {
    return v.snap_ratio && v.sc->step % v.snap_ratio == 0;
}

DYN_KERNEL(, k_snapshot, (), ()) {
    if (!snapshot_due(v)) return;
    const uint64_t f = v.sc->snap_count % v.snap_cap;
    const size_t ns = (size_t)v.na + 3 * (size_t)v.nw;
    float* P = v.snap_pos + f * ns * 3;
    float* V = v.snap_vel ? v.snap_vel + f * ns * 3 : nullptr;
    float* F = v.snap_force ? v.snap_force + f * (size_t)v.na * 3 : nullptr;
    const BoxDev b = *v.box;
    const uint32_t tid = bk.idx * blockDim.x + threadIdx.x, stride = bk.cnt * blockDim.x;
    for (uint32_t a = tid; a < v.na; a += stride) {
        // atoms in the primary cell (Snapshot::new, src/snapshot.rs:158-161)
        const float3 p = xyz(v.apos[a]);
        float w[3] = {p.x, p.y, p.z};
        for (int k = 0; k < 3; ++k) w[k] -= floorf((w[k] - b.lo[k]) * b.inv_ext[k]) * b.ext[k];
        P[3 * (size_t)a + 0] = w[0]; P[3 * (size_t)a + 1] = w[1]; P[3 * (size_t)a + 2] = w[2];
        if (V) {
            const float4 q = v.avel[a];
            V[3 * (size_t)a + 0] = q.x; V[3 * (size_t)a + 1] = q.y; V[3 * (size_t)a + 2] = q.z;
        }
        if (F) {
            const long long* fa = v.aforce + 3 * (size_t)a;
            const long long* fr = v.arecip + 3 * (size_t)a;
            for (int k = 0; k < 3; ++k) F[3 * (size_t)a + k] = (float)((double)(fa[k] + fr[k]) * DYN_FIX_INV);
        }
    }
    for (uint32_t s = tid; s < v.nw_cap; s += stride) {
        const uint32_t id = v.wid[s];
        if (id == INVALID_ID) continue;
        const size_t o = 3 * ((size_t)v.na + 3 * (size_t)id);
        for (int k = 0; k < 3; ++k) {
            const float4 q = v.wpos[4 * s + k];
            P[o + 3 * k + 0] = q.x; P[o + 3 * k + 1] = q.y; P[o + 3 * k + 2] = q.z;
            if (V) {
                const float4 u = v.wvel[3 * s + k];
                V[o + 3 * k + 0] = u.x; V[o + 3 * k + 1] = u.y; V[o + 3 * k + 2] = u.z;
            }
        }
    }
}

// the frame's scalars, then the frame count (after k_snapshot has read it)
DYN_KERNEL(, k_snapshot_done, (), ()) {
    if (!snapshot_due(v) || bk.idx != 0 || threadIdx.x != 0) return;
    Scalars* sc = v.sc;
    const BoxDev b = *v.box;
    dyn_frame_t r;
    r.step = sc->step;
    r.time_ps = sc->time_ps;
    r.kinetic = sc->acc[ACC_KE];
    r.potential = sc->pe;
    r.potential_bonded = sc->acc[ACC_E_BONDED] + sc->acc[ACC_E_14];
    r.temperature = sc->temperature;
    r.pressure_bar = sc->pressure;
    double vol = 1.0;
    for (int k = 0; k < 3; ++k) {
        r.box_lo[k] = b.lo[k];
        r.box_hi[k] = (double)b.lo[k] + (double)b.ext[k];
        vol *= (double)b.ext[k];
    }
    r.volume = vol;
    r.density = v.total_mass / vol;
    r.dh_dl = sc->dh_dl;
    v.snap_frames[sc->snap_count % v.snap_cap] = r;
    sc->snap_count += 1ull;
}

inline int iblocks(const SysView& v, uint64_t n) {
    uint64_t bl = (n + IT - 1) / IT;
    if (bl < 1) bl = 1;
    return (int)(bl < v.max_blocks ? bl : v.max_blocks);
}

}  // namespace

namespace dyn {

int kick_blocks_w(const SysView& v) { return iblocks(v, v.nw_cap); }
int kick_blocks_a(const SysView& v) { return iblocks(v, v.nunit); }

void launch_first_half_water(const Target& t, float dt) {
    t.launch(k_water_first, k_water_first_batch, [](const SysView& v) { return v.nw ? iblocks(v, v.nw_cap) : 0; },
             IT, 0, dt);
}
void launch_first_half_atoms(const Target& t, float dt) {
    t.launch(k_atom_first, k_atom_first_batch, [](const SysView& v) { return v.na ? (int)v.nb[REG_CONS] : 0; },
             IT, 0, dt);
}
void launch_first_half(const Target& t, float dt) {
    launch_first_half_water(t, dt);
    launch_first_half_atoms(t, dt);
}

void launch_second_half_water(const Target& t, float dt) {
    t.launch(k_water_kick, k_water_kick_batch, [](const SysView& v) { return v.nw ? (int)v.nb[REG_KICK_W] : 0; },
             IT, 0, dt);
}
void launch_second_half_atoms(const Target& t, float dt) {
    t.launch(k_atom_kick, k_atom_kick_batch, [](const SysView& v) { return v.na ? (int)v.nb[REG_KICK_A] : 0; }, IT,
             0, dt);
}
void launch_second_half(const Target& t, float dt) {
    launch_second_half_water(t, dt);
    launch_second_half_atoms(t, dt);
}

void launch_finalize(const Target& t, float dt, bool energy, bool thermo) {
    auto one = [](const SysView&) { return 1; };
    // 16 warps: one per partial-sum region
    if (energy) t.launch(k_finalize<true>, k_finalize_batch<true>, one, 512, 0, dt, thermo);
    else t.launch(k_finalize<false>, k_finalize_batch<false>, one, 512, 0, dt, thermo);
    if (!thermo) return;
    t.launch(k_scale, k_scale_batch,
             [](const SysView& v) {
                 const bool scales =
                     (v.integrator == DYN_INTEGRATOR_VERLET_VELOCITY && v.thermostat == DYN_THERMO_CSVR) ||
                     v.barostat == DYN_BARO_CRESCALE;
                 return scales ? iblocks(v, (uint64_t)v.nw_cap + v.na) : 0;
             },
             IT, 0);
}

void launch_snapshot(const Target& t) {
    t.launch(k_snapshot, k_snapshot_batch,
             [](const SysView& v) { return v.snap_ratio ? iblocks(v, std::max<uint64_t>(v.na, v.nw_cap)) : 0; },
             IT, 0);
    t.launch(k_snapshot_done, k_snapshot_done_batch, [](const SysView& v) { return v.snap_ratio ? 1 : 0; }, 32, 0);
}

void launch_periodic(const Target& t) {
    auto com = [](const SysView& v) { return (v.flags & DYN_FLAG_COM_REMOVAL) ? (int)v.nb[REG_COM] : 0; };
    t.launch(k_com_reduce, k_com_reduce_batch, com, IT, 0);
    t.launch(k_com_apply, k_com_apply_batch, com, IT, 0);
    t.launch(k_recenter, k_recenter_batch,
             [](const SysView& v) { return ((v.flags & DYN_FLAG_RECENTER) && v.na) ? 1 : 0; }, 256, 0);
    t.launch(k_reset_angle, k_reset_angle_batch,
             [](const SysView& v) { return ((v.flags & DYN_FLAG_RESET_ANGLE) && v.nw) ? iblocks(v, v.nw_cap) : 0; },
             IT, 0);
    launch_snapshot(t);  // after the periodic tasks, as handle_snapshots
}

}  // namespace dyn
