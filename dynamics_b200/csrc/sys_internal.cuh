// Internal to the library: the resident-system handle and the graph helpers
// that the single-system engine (system.cu) and the batch (batch.cu) share.
#pragma once

#include <vector>

#include "engine.cuh"

struct dyn_sys_s {
    cudaStream_t stream = nullptr;
    bool own_stream = false;       // created here because the caller passed NULL
    cudaStream_t aux = nullptr;    // captures the bodies of conditional graph nodes
    SysView v{};
    dyn_config_t cfg{};
    cufftHandle plan_f = 0, plan_b = 0;
    cudaGraphExec_t graph[4] = {nullptr, nullptr, nullptr, nullptr};
    float graph_dt[4] = {0, 0, 0, 0};
    uint64_t host_step = 0;        // steps enqueued so far
    std::vector<void*> allocs;     // every device allocation, freed on destroy
    size_t bytes = 0;              // device memory held (allocations, PME grids, cuFFT work)
    Scalars* h_sc = nullptr;       // pinned mirror of the scalars
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

}  // namespace dyn
