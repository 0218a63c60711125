// Internal to the library: the resident-system handle and the graph helpers
// that the single-system engine (system.cu) and the batch (batch.cu) share.
#pragma once

#include <vector>

#include "engine.cuh"

// Side streams and events that split a captured step into parallel graph
// branches (the atom half of the integrator, the atom-atom / 1-4 / bonded
// terms and SPME run beside the water work).
struct Branches {
    cudaStream_t side[2] = {nullptr, nullptr};
    cudaEvent_t ev[8] = {};
    int create();
    void destroy();
};

struct dyn_sys_s {
    cudaStream_t stream = nullptr;
    bool own_stream = false;       // created here because the caller passed NULL
    cudaStream_t aux = nullptr;    // captures the bodies of conditional graph nodes
    Branches br;
    SysView v{};
    dyn_config_t cfg{};
    cufftHandle plan_f = 0, plan_b = 0;
    cudaGraphExec_t graph[4] = {nullptr, nullptr, nullptr, nullptr};
    float graph_dt[4] = {0, 0, 0, 0};
    uint64_t host_step = 0;        // steps enqueued so far
    std::vector<void*> allocs;     // every device allocation, freed on destroy
    size_t bytes = 0;              // device memory held (allocations, PME grids, cuFFT work)
    Scalars* h_sc = nullptr;       // pinned mirror of the scalars
    bool batch_member = false;     // owned by a dyn_batch_t
    void* snap_mem = nullptr;      // snapshot ring (dyn_sys_snapshots)
    size_t snap_bytes = 0;
    uint64_t snap_read = 0;        // frames handed to the host so far
    cudaEvent_t window_ev = nullptr;  // bounds the steps one dyn_sys_step call queues
    bool window_armed = false;
    float* host_stage = nullptr;   // device staging of dyn_sys_step_host (in allocs)
    size_t host_stage_n = 0;       // floats
};

// Home-order host layout <-> the resident arrays.  Waters: (pos, vel) as
// [nw][3][3] floats (O, H0, H1) by original id; the virtual site M is
// placed from O, H0, H1.  Atoms: [na][3] floats by atom index.  One water
// slot (cluster order) or one atom per call.
__device__ __forceinline__ void water_in(const SysView& v, uint32_t s, const float* __restrict__ wp,
                                         const float* __restrict__ wv) {
    const uint32_t id = v.wid[s];
    if (id == INVALID_ID) return;
    if (wp) {
        const float* x = wp + 9 * (size_t)id;
        const float3 o = f3(x[0], x[1], x[2]), h0 = f3(x[3], x[4], x[5]), h1 = f3(x[6], x[7], x[8]);
        const float3 bis = (h0 - o) + (h1 - o);
        const float3 m = o + bis * (OPC_O_EP_R * rsqrtf(dot3(bis, bis)));
        v.wpos[4 * s + 0] = make_float4(o.x, o.y, o.z, 0.f);
        v.wpos[4 * s + 1] = make_float4(h0.x, h0.y, h0.z, OPC_Q_H);
        v.wpos[4 * s + 2] = make_float4(h1.x, h1.y, h1.z, OPC_Q_H);
        v.wpos[4 * s + 3] = make_float4(m.x, m.y, m.z, OPC_Q_EP);
    }
    if (wv) {
        const float* x = wv + 9 * (size_t)id;
        for (int k = 0; k < 3; ++k) v.wvel[3 * s + k] = make_float4(x[3 * k], x[3 * k + 1], x[3 * k + 2], 0.f);
    }
}

__device__ __forceinline__ void water_out(const SysView& v, uint32_t s, float* __restrict__ wp,
                                          float* __restrict__ wv) {
    const uint32_t id = v.wid[s];
    if (id == INVALID_ID) return;
    for (int k = 0; k < 3; ++k) {
        if (wp) {
            const float4 a = v.wpos[4 * s + k];
            float* o = wp + 9 * (size_t)id + 3 * k;
            o[0] = a.x; o[1] = a.y; o[2] = a.z;
        }
        if (wv) {
            const float4 b = v.wvel[3 * s + k];
            float* o = wv + 9 * (size_t)id + 3 * k;
            o[0] = b.x; o[1] = b.y; o[2] = b.z;
        }
    }
}

__device__ __forceinline__ void atom_in(const SysView& v, uint32_t a, const float* __restrict__ ap,
                                        const float* __restrict__ av) {
    if (ap) { float4 p = v.apos[a]; p.x = ap[3 * a]; p.y = ap[3 * a + 1]; p.z = ap[3 * a + 2]; v.apos[a] = p; }
    if (av) v.avel[a] = make_float4(av[3 * a], av[3 * a + 1], av[3 * a + 2], 0.f);
}

__device__ __forceinline__ void atom_out(const SysView& v, uint32_t a, float* __restrict__ ap,
                                         float* __restrict__ av) {
    const float4 p = v.apos[a], w = v.avel[a];
    if (ap) { ap[3 * a] = p.x; ap[3 * a + 1] = p.y; ap[3 * a + 2] = p.z; }
    if (av) { av[3 * a] = w.x; av[3 * a + 1] = w.y; av[3 * a + 2] = w.z; }
}

namespace dyn {

// Turns the device-side flags of h->h_sc (already on the host) into errors.
int check_scalars(dyn_sys_s* h);
// The energies of the last step from h->h_sc (already on the host).
void energies_of(dyn_sys_s* h, dyn_energies_t* e);
// The water-water kernel's CTAs per group (before any step graph exists).
void set_ww_split(dyn_sys_s* h, uint32_t split);
// Marks h as a batch member (before any step graph exists): no automatic
// water-water group split.  The chunk stays the one sized for three CTAs per
// SM although the kernel's batch form runs two (a chunk sized for two was
// slower on the batched workloads), so a member computes exactly what it
// computes alone.
void set_batch_member(dyn_sys_s* h);

// Inside an active capture on st: appends an IF node on hc after everything
// captured so far and starts capturing its body on aux.
int begin_if_body(cudaStream_t st, cudaStream_t aux, cudaGraphConditionalHandle hc, cudaGraph_t* body);
int end_if_body(cudaStream_t aux);
// Copies the scalars to the host and turns device-side flags into errors.
int read_scalars(dyn_sys_s* h);
// Kernel nodes of a graph (library kernels included).
int count_graph_kernels(cudaGraph_t g, uint32_t* n);
// Full forces, energies and accelerations at the current coordinates (list
// rebuilt), synchronous.
int evaluate_forces(dyn_sys_s* h);

// The parts of a step, enqueued on T's stream; with fork (only while a graph
// is being captured) the independent work goes to the side targets A and P
// (same systems, the side streams of br) as parallel branches that join
// back into T.  The launch order is the same either way, which a batch needs
// (it records its block maps in launch order).
//   first half:  water drift/thermostat on T | atom drift + constraints on A
//   forces:      water-water, water-atom on T | atom-atom, 1-4, bonded on A |
//                SPME and its corrections on P (spme steps)
//   second half: water kick on T | atom kick + RATTLE on A
int enqueue_first_half(const Target& T, const Target& A, const Branches& br, bool fork, float dt);
int enqueue_forces(const Target& T, const Target& A, const Target& P, const Branches& br, bool fork, bool spme,
                   bool energy);
int enqueue_second_half(const Target& T, const Target& A, const Branches& br, bool fork, float dt);

}  // namespace dyn
