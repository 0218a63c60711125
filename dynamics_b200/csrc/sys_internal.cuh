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
};

namespace dyn {

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
