// Steepest-descent energy minimization of the atoms on the device
// (MdState::minimize_energy, src/minimize_energy.rs:60-260).
//
// The reference's algorithm, kept alike: waters and static atoms stay put;
// reciprocal-space forces (and the corrections that come with them) are off
// (:96-99); every trial moves each atom by F * step / F_max, step =
// min(alpha * F_max, 0.2 A) (:160-190), then accepts when the potential
// energy did not rise (alpha * 1.2, at most 0.01; converged when the largest
// force is below the tolerance, :205-212) or reverts the move and halves
// alpha (stop below 1e-8, :214-237).
//
// B200 form: one trial is a fixed sequence of kernels with every decision
// taken on the device (Scalars.min_*), so K trials are one CUDA graph and
// the host only reads a done flag between graph launches.  The forces of
// the accepted geometry are kept (fsave) so a rejected trial restores them
// instead of evaluating them again.  Only the water-atom and atom-atom pair
// kernels run: the water-water forces do not move anything here.
#include <cmath>

#include "engine.cuh"
#include "sys_internal.cuh"

namespace {

constexpr float STEP_MAX = 0.2f;
constexpr float GROW = 1.2f;
constexpr float SHRINK = 0.5f;
constexpr float ALPHA_MIN = 1.0e-8f;
constexpr float ALPHA_MAX = 1.0e-2f;
constexpr int MT = 256;
constexpr int TRIALS_PER_GRAPH = 8;

__device__ __forceinline__ float3 force_of(const SysView& v, uint32_t a) {
    const long long* f = v.aforce + 3 * (size_t)a;
    return f3((float)((double)f[0] * DYN_FIX_INV), (float)((double)f[1] * DYN_FIX_INV),
              (float)((double)f[2] * DYN_FIX_INV));
}

__device__ __forceinline__ bool movable(const SysView& v, uint32_t a) {
    return !(v.astatic && v.astatic[a]);
}

__global__ void k_min_init(const __grid_constant__ SysView v) {
    Scalars* sc = v.sc;
    sc->min_alpha = 0.01f;  // src/minimize_energy.rs:121
    sc->min_alpha_try = 0.01f;
    sc->min_fmax_bits = 0u;
    sc->min_ctr = 0u;
    sc->min_accepted = 0u;
    sc->min_trials = 0u;
    sc->min_done = 0u;
    sc->min_action = 0u;
}

// Potential energy of the atom terms from the block partials (the
// reference's potential without the reciprocal part), one warp per region.
__device__ double min_energy(const SysView& v) {
    __shared__ double rs[4][2];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int regs[4] = {REG_WS, REG_SS, REG_14, REG_BOND};
    if (w < 4) {
        const int reg = regs[w];
        const bool used = v.na && (reg != REG_WS || v.nw);
        double o[2] = {0.0, 0.0};
        if (used) {
            const double4* p = reinterpret_cast<const double4*>(v.partials) + (size_t)reg * v.max_blocks;
            for (uint32_t i = lane; i < v.nb[reg]; i += 32) {
                const double4 a = p[i];
                o[0] += a.x; o[1] += a.y;
            }
        }
        o[0] = warp_sum_d(o[0]);
        o[1] = warp_sum_d(o[1]);
        if (lane == 0) { rs[w][0] = o[0]; rs[w][1] = o[1]; }
    }
    __syncthreads();
    // LJ + Coulomb of the atom lists (each pair once), 1-4 (energy in [0]),
    // bonded (energy in [0])
    return rs[0][0] + rs[0][1] + rs[1][0] + rs[1][1] + rs[2][0] + rs[3][0];
}

// Energy and saved forces of the starting geometry.
__global__ void k_min_start(const __grid_constant__ SysView v) {
    const double e = min_energy(v);
    if (threadIdx.x == 0) {
        v.sc->min_e_prev = e;
        v.sc->min_action = 1u;  // k_min_apply saves the forces
    }
}

// Largest force over the movable atoms; the last block sets this trial's
// step (or marks the minimization done when every force is zero).
__global__ void k_min_fmax(const __grid_constant__ SysView v) {
    Scalars* sc = v.sc;
    if (sc->min_done) return;
    float m = 0.f;
    for (uint32_t a = blockIdx.x * blockDim.x + threadIdx.x; a < v.na; a += gridDim.x * blockDim.x) {
        if (!movable(v, a)) continue;
        const float3 f = force_of(v, a);
        const float fm = sqrtf(dot3(f, f));
        if (isfinite(fm)) m = fmaxf(m, fm);
    }
    m = warp_max_f(m);
    if ((threadIdx.x & 31) == 0 && m > 0.f) atomicMax(&sc->min_fmax_bits, __float_as_uint(m));
    __threadfence();
    __syncthreads();
    if (threadIdx.x != 0) return;
    if (atomicAdd(&sc->min_ctr, 1u) != gridDim.x - 1) return;
    __threadfence();
    const float fmax = __uint_as_float(atomicExch(&sc->min_fmax_bits, 0u));
    sc->min_ctr = 0u;
    sc->min_fmax = fmax;
    if (fmax == 0.f) {
        sc->min_done = 1u;
        return;
    }
    sc->min_step = fminf(sc->min_alpha_try * fmax, STEP_MAX);
}

// x += F * step / F_max for the movable atoms with a finite, non-zero force.
__global__ void k_min_move(const __grid_constant__ SysView v, float4* __restrict__ moved) {
    const Scalars* sc = v.sc;
    if (sc->min_done) return;
    const float k = sc->min_step / sc->min_fmax;
    for (uint32_t a = blockIdx.x * blockDim.x + threadIdx.x; a < v.na; a += gridDim.x * blockDim.x) {
        float4 s = make_float4(0.f, 0.f, 0.f, 0.f);
        if (movable(v, a)) {
            const float3 f = force_of(v, a);
            const float fm = sqrtf(dot3(f, f));
            if (isfinite(fm) && fm != 0.f) {
                s = make_float4(f.x * k, f.y * k, f.z * k, 0.f);
                float4 p = v.apos[a];
                p.x += s.x; p.y += s.y; p.z += s.z;
                v.apos[a] = p;
            }
        }
        moved[a] = s;
    }
}

// Accept or reject the trial (single block).
__global__ void k_min_decide(const __grid_constant__ SysView v, float tol, uint32_t max_iters,
                             uint32_t max_trials) {
    Scalars* sc = v.sc;
    const bool was_done = sc->min_done != 0u;  // read by every thread before any write
    __syncthreads();
    if (was_done) {
        if (threadIdx.x == 0) sc->min_action = 0u;
        return;
    }
    const double e = min_energy(v);
    // largest force of the new geometry (convergence test on acceptance)
    float m = 0.f;
    for (uint32_t a = threadIdx.x; a < v.na; a += blockDim.x) {
        if (!movable(v, a)) continue;
        const float3 f = force_of(v, a);
        const float fm = sqrtf(dot3(f, f));
        if (isfinite(fm)) m = fmaxf(m, fm);
    }
    __shared__ float wm[MT / 32];
    m = warp_max_f(m);
    if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x != 0) return;
    for (int i = 1; i < (int)(blockDim.x >> 5); ++i) m = fmaxf(m, wm[i]);
    m = fmaxf(m, wm[0]);
    sc->min_trials += 1u;
    if (e <= sc->min_e_prev) {
        sc->min_e_prev = e;
        sc->min_alpha = fminf(sc->min_alpha_try * GROW, ALPHA_MAX);
        sc->min_alpha_try = sc->min_alpha;
        sc->min_accepted += 1u;
        sc->min_action = 1u;
        if (m <= tol) sc->min_done = 1u;
    } else {
        sc->min_action = 2u;
        sc->min_alpha_try *= SHRINK;
        if (sc->min_alpha_try < ALPHA_MIN) {
            sc->min_alpha = sc->min_alpha_try;
            sc->min_done = 1u;
        }
    }
    if (sc->min_accepted >= max_iters || sc->min_trials >= max_trials) sc->min_done = 1u;
}

// Accepted: keep these forces.  Rejected: move back and restore the forces
// of the accepted geometry.
__global__ void k_min_apply(const __grid_constant__ SysView v, const float4* __restrict__ moved,
                            long long* __restrict__ fsave) {
    const unsigned int act = v.sc->min_action;
    if (act == 0u) return;
    for (uint32_t a = blockIdx.x * blockDim.x + threadIdx.x; a < v.na; a += gridDim.x * blockDim.x) {
        long long* f = v.aforce + 3 * (size_t)a;
        long long* g = fsave + 3 * (size_t)a;
        if (act == 1u) {
            g[0] = f[0]; g[1] = f[1]; g[2] = f[2];
        } else {
            const float4 s = moved[a];
            float4 p = v.apos[a];
            p.x -= s.x; p.y -= s.y; p.z -= s.z;
            v.apos[a] = p;
            f[0] = g[0]; f[1] = g[1]; f[2] = g[2];
        }
    }
}

inline int mblocks(uint32_t n) {
    const uint32_t b = (n + MT - 1) / MT;
    return (int)std::max<uint32_t>(1u, std::min<uint32_t>(b, 148u * 4u));
}

// Atom forces and the atom energy partials at the current positions,
// without the reciprocal part.
void enqueue_atom_forces(const SysView& v, cudaStream_t st, bool check_list) {
    const Target T{&v, nullptr, st};
    if (check_list) dyn::launch_displacement_check(T);
    dyn::launch_rebuild(T, false);
    dyn::launch_gather_atoms(T);
    dyn::launch_pairs_ws(T, true);
    dyn::launch_pairs_atoms(T, true);
    dyn::launch_pair14(T, true);
    dyn::launch_bonded(T, true);
}

}  // namespace

extern "C" int dyn_sys_minimize(dyn_sys_t h, uint32_t max_iters, float tolerance, uint32_t* iters,
                                double* energy) {
    DYN_CHECK(h, DYN_ERR_INVALID, "dyn_sys_minimize: NULL handle");
    DYN_CHECK(tolerance >= 0.f && std::isfinite(tolerance), DYN_ERR_INVALID,
              "dyn_sys_minimize: tolerance must be finite and >= 0");
    DYN_CHECK(!h->batch_member, DYN_ERR_UNSUPPORTED, "dyn_sys_minimize: not for a batch member");
    if (iters) *iters = 0;
    SysView& v = h->v;
    cudaStream_t st = h->stream;
    if (v.na == 0 || max_iters == 0) {
        if (energy) *energy = 0.0;
        return DYN_OK;
    }
    // scratch: per-atom trial moves and the forces of the accepted geometry
    float4* moved = nullptr;
    long long* fsave = nullptr;
    DYN_CUDA(cudaMalloc(&moved, (size_t)v.na * sizeof(float4)));
    cudaError_t e = cudaMalloc(&fsave, (size_t)v.na * 3 * sizeof(long long));
    if (e != cudaSuccess) {
        cudaFree(moved);
        return dyn::cuda_fail(e, "cudaMalloc");
    }
    const uint64_t trials64 = (uint64_t)max_iters * 32u + 64u;
    const uint32_t max_trials = (uint32_t)std::min<uint64_t>(trials64, 0xFFFFFFF0ull);
    int rc = DYN_OK;
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    do {
        k_min_init<<<1, 1, 0, st>>>(v);
        enqueue_atom_forces(v, st, true);
        k_min_start<<<1, MT, 0, st>>>(v);
        k_min_apply<<<mblocks(v.na), MT, 0, st>>>(v, moved, fsave);
        // TRIALS_PER_GRAPH trials per graph launch
        if ((e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) {
            rc = dyn::cuda_fail(e, "cudaStreamBeginCapture");
            break;
        }
        for (int t = 0; t < TRIALS_PER_GRAPH; ++t) {
            k_min_fmax<<<mblocks(v.na), MT, 0, st>>>(v);
            k_min_move<<<mblocks(v.na), MT, 0, st>>>(v, moved);
            enqueue_atom_forces(v, st, true);
            k_min_decide<<<1, MT, 0, st>>>(v, tolerance, max_iters, max_trials);
            k_min_apply<<<mblocks(v.na), MT, 0, st>>>(v, moved, fsave);
        }
        e = cudaStreamEndCapture(st, &g);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e != cudaSuccess) { rc = dyn::cuda_fail(e, "capture of the minimizer trials"); break; }
        if ((e = cudaGraphInstantiate(&ge, g, 0)) != cudaSuccess) {
            rc = dyn::cuda_fail(e, "cudaGraphInstantiate");
            break;
        }
        // every launch either ends the minimization or advances the trial
        // count by TRIALS_PER_GRAPH, which is bounded by max_trials
        const uint64_t max_launches = max_trials / TRIALS_PER_GRAPH + 2;
        for (uint64_t k = 0; k < max_launches; ++k) {
            if ((e = cudaGraphLaunch(ge, st)) != cudaSuccess) { rc = dyn::cuda_fail(e, "cudaGraphLaunch"); break; }
            if ((rc = dyn::read_scalars(h)) != DYN_OK) break;
            if (h->h_sc->min_done) break;
        }
    } while (0);
    if (ge) cudaGraphExecDestroy(ge);
    if (g) cudaGraphDestroy(g);
    if (rc == DYN_OK) {
        if (iters) *iters = h->h_sc->min_accepted;
        if (energy) *energy = h->h_sc->min_e_prev;
        // full forces and accelerations at the minimized geometry, as after
        // dyn_sys_create
        rc = dyn::evaluate_forces(h);
    }
    cudaStreamSynchronize(st);
    cudaFree(moved);
    cudaFree(fsave);
    return rc;
}
