// Batched form: many independent systems of uneven size advanced together.
//
// Every stage of a step is ONE launch for all member systems: the same
// kernel body as the single-system engine, in its NAME##_batch form, with a
// block map that gives each system the block range its single-system launch
// would have had (per-system offsets into one grid).  A step is one captured
// CUDA graph whose list rebuild and periodic tasks sit under IF nodes that
// any member can raise; each member's kernels still check its own flags, so
// a member's trajectory is bit-identical to running it alone.  cuFFT runs
// once per member on the batch stream (its plans are per grid size).
//
// The reference has no counterpart (it advances one MdState per call,
// src/integrate.rs:72); the batch is built from the same dyn_sys members, so
// dyn_sys_get_state / get_energies read any member's results.
#include <cmath>
#include <cstring>
#include <map>

#include "sys_internal.cuh"

struct BatchCtx {
    std::vector<SysView> views;                       // host copies of the members' views
    const SysView* d_views = nullptr;                 // device copy used by the graph being built
    bool collecting = false;                          // recording block maps, launching nothing
    std::map<std::vector<uint32_t>, BlockMap> maps;   // per-system block counts -> device map
    bool map_missing = false;
    bool map_too_large = false;
    uint32_t launches = 0;                            // batched launches recorded while collecting
    // the members' FFTs (one cuFFT plan per member) run over these streams
    // side by side instead of one after another on the batch stream
    static constexpr int N_FFT = 8;
    cudaStream_t fft_st[N_FFT] = {};
    cudaEvent_t fft_ev[N_FFT + 1] = {};
    int n_fft = 0;
};

int batch_fft_streams(BatchCtx* b, cudaStream_t** st, cudaEvent_t** ev) {
    *st = b->fft_st;
    *ev = b->fft_ev;
    return b->n_fft;
}

uint32_t batch_size(const BatchCtx* b) { return (uint32_t)b->views.size(); }
const SysView& batch_view(const BatchCtx* b, uint32_t i) { return b->views[i]; }
const SysView* batch_dviews(const BatchCtx* b) { return b->d_views; }
bool batch_collecting(const BatchCtx* b) { return b->collecting; }

BlockMap batch_map(BatchCtx* b, const std::vector<uint32_t>& blocks) {
    if (!b->collecting) {
        auto it = b->maps.find(blocks);
        if (it != b->maps.end()) return it->second;
        b->map_missing = true;
        return BlockMap{0, nullptr};
    }
    uint32_t total = 0;
    for (uint32_t x : blocks) total += x;
    if (total) ++b->launches;
    auto it2 = b->maps.find(blocks);
    if (it2 != b->maps.end()) return it2->second;
    total = 0;
    for (uint32_t x : blocks) {
        if (x > 0xFFFFu) b->map_too_large = true;
        total += x;
    }
    b->maps[blocks] = BlockMap{total, nullptr};
    return BlockMap{total, nullptr};
}

struct dyn_batch_s {
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaStream_t aux = nullptr;
    Branches br;
    std::vector<dyn_sys_t> members;
    BatchCtx ctx;
    SysView* d_views[4] = {nullptr, nullptr, nullptr, nullptr};  // one per graph variant
    std::vector<void*> map_allocs;
    cudaGraphExec_t graph[4] = {nullptr, nullptr, nullptr, nullptr};
    float graph_dt[4] = {0, 0, 0, 0};
    uint64_t host_step = 0;
    cudaEvent_t window_ev = nullptr;  // bounds the steps one dyn_batch_step call queues
    bool window_armed = false;
    uint32_t spme_interval = 1, energy_interval = 1;
    bool fixed_intervals = false;   // set by the first member
    uint32_t views_cap = 0;         // members the device view arrays hold
    // batch-wide host step (dyn_batch_step_host): the members' packed
    // states in one device area, their scalars gathered beside it
    struct HostIo {
        std::vector<unsigned long long> off;  // member offsets into the packed state (floats), n + 1
        std::vector<SysView> views;           // the views d_views holds
        float* d_state = nullptr;
        size_t cap_floats = 0;
        Scalars* d_sc = nullptr;
        Scalars* h_sc = nullptr;              // pinned
        SysView* d_views = nullptr;
        unsigned long long* d_off = nullptr;
        size_t cap_members = 0;
        float* h_buf = nullptr;               // pinned packed state (dyn_batch_host_buffer)
        size_t h_buf_floats = 0;
    } io;
};

namespace {

// Device copies of the block maps recorded by a collecting pass.
int upload_maps(dyn_batch_s* b) {
    if (b->ctx.map_too_large)
        return dyn::fail(DYN_ERR_UNSUPPORTED, "batch: a member needs more than 65535 blocks in one stage");
    for (auto& kv : b->ctx.maps) {
        if (kv.second.d_map || kv.second.total == 0) continue;
        std::vector<uint2> m;
        m.reserve(kv.second.total);
        const std::vector<uint32_t>& bl = kv.first;
        for (uint32_t i = 0; i < bl.size(); ++i)
            for (uint32_t j = 0; j < bl[i]; ++j) m.push_back(make_uint2(i, j | (bl[i] << 16)));
        uint2* d = nullptr;
        DYN_CUDA(cudaMalloc(&d, m.size() * sizeof(uint2)));
        b->map_allocs.push_back(d);
        DYN_CUDA(cudaMemcpy(d, m.data(), m.size() * sizeof(uint2), cudaMemcpyHostToDevice));
        kv.second.d_map = d;
    }
    return DYN_OK;
}

// The stages of one step, for all members at once (MdState::step,
// src/integrate.rs:100-473).  With cond, the rebuild and the periodic tasks
// go under IF nodes of the capture in progress.
int enqueue_batch_step(dyn_batch_s* b, float dt, bool spme, bool energy, bool cond,
                       cudaGraphConditionalHandle c_rebuild, cudaGraphConditionalHandle c_prune,
                       cudaGraphConditionalHandle c_periodic) {
    const Target T{nullptr, &b->ctx, b->stream}, TA{nullptr, &b->ctx, b->aux};
    const Target S0{nullptr, &b->ctx, b->br.side[0]}, S1{nullptr, &b->ctx, b->br.side[1]};
    cudaGraph_t body = nullptr;
    int rc = DYN_OK;
    // cond: capturing (parallel branches); otherwise a collecting pass
    if ((rc = dyn::enqueue_first_half(T, S0, b->br, cond, dt)) != DYN_OK) return rc;
    dyn::launch_displacement_check(T);
    if (cond && (rc = dyn::begin_if_body(b->stream, b->aux, c_rebuild, &body)) != DYN_OK) return rc;
    dyn::launch_rebuild(cond ? TA : T, false);
    if (cond && (rc = dyn::end_if_body(b->aux)) != DYN_OK) return rc;
    if (cond && (rc = dyn::begin_if_body(b->stream, b->aux, c_prune, &body)) != DYN_OK) return rc;
    dyn::launch_prune(cond ? TA : T, false);
    if (cond && (rc = dyn::end_if_body(b->aux)) != DYN_OK) return rc;
    dyn::launch_gather_atoms(T);
    if ((rc = dyn::enqueue_forces(T, S0, S1, b->br, cond, spme, energy)) != DYN_OK) return rc;
    if ((rc = dyn::enqueue_second_half(T, S0, b->br, cond, dt)) != DYN_OK) return rc;
    dyn::launch_finalize(T, dt, energy, true);
    if (cond && (rc = dyn::begin_if_body(b->stream, b->aux, c_periodic, &body)) != DYN_OK) return rc;
    dyn::launch_periodic(cond ? TA : T);
    if (cond && (rc = dyn::end_if_body(b->aux)) != DYN_OK) return rc;
    return DYN_OK;
}

// Records the block maps of a step variant (no launches) and uploads them.
int collect_maps(dyn_batch_s* b, float dt, bool spme, bool energy) {
    b->ctx.collecting = true;
    const int rc = enqueue_batch_step(b, dt, spme, energy, false, 0, 0, 0);
    b->ctx.collecting = false;
    if (rc) return rc;
    return upload_maps(b);
}

int capture_batch_step(dyn_batch_s* b, int g, float dt, bool spme, bool energy, cudaGraph_t* out) {
    *out = nullptr;
    DYN_CUDA(cudaStreamSynchronize(b->stream));  // d_views[g] may be read by work in flight
    b->ctx.views.clear();
    for (dyn_sys_t m : b->members) b->ctx.views.push_back(m->v);
    int rc = collect_maps(b, dt, spme, energy);
    if (rc) return rc;
    if (b->views_cap < b->members.size()) {
        // grow the per-variant view arrays (no graph that reads them is alive)
        for (int k = 0; k < 4; ++k) {
            if (b->graph[k]) { cudaGraphExecDestroy(b->graph[k]); b->graph[k] = nullptr; }
            if (b->d_views[k]) cudaFree(b->d_views[k]);
            b->d_views[k] = nullptr;
        }
        const uint32_t cap = std::max<uint32_t>(8u, (uint32_t)b->members.size() * 2);
        for (int k = 0; k < 4; ++k) DYN_CUDA(cudaMalloc(&b->d_views[k], cap * sizeof(SysView)));
        b->views_cap = cap;
    }
    b->ctx.d_views = b->d_views[g];
    b->ctx.map_missing = false;
    DYN_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    cudaGraphConditionalHandle hr = 0, hq = 0, hp = 0;
    {
        cudaStreamCaptureStatus cs;
        cudaGraph_t cg = nullptr;
        cudaError_t e = cudaStreamGetCaptureInfo(b->stream, &cs, nullptr, &cg, nullptr, nullptr);
        if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&hr, cg, 0, cudaGraphCondAssignDefault);
        if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&hq, cg, 0, cudaGraphCondAssignDefault);
        if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&hp, cg, 0, cudaGraphCondAssignDefault);
        if (e != cudaSuccess) rc = dyn::cuda_fail(e, "cudaGraphConditionalHandleCreate");
    }
    if (rc == DYN_OK) rc = enqueue_batch_step(b, dt, spme, energy, true, hr, hq, hp);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
    if (rc == DYN_OK && e != cudaSuccess) rc = dyn::cuda_fail(e, "cudaStreamEndCapture");
    if (rc == DYN_OK) {
        const cudaError_t le = cudaGetLastError();
        if (le != cudaSuccess) rc = dyn::cuda_fail(le, "kernel launch during capture");
    }
    if (rc == DYN_OK && b->ctx.map_missing) rc = dyn::fail(DYN_ERR_INVALID, "batch: block map missing");
    if (rc != DYN_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    // the graph's kernels read the views at run time: give them this
    // graph's conditional handles
    for (SysView& v : b->ctx.views) {
        v.cond_rebuild = hr;
        v.cond_prune = hq;
        v.cond_periodic = hp;
        v.use_cond = 1;
    }
    const cudaError_t ue = cudaMemcpy(b->d_views[g], b->ctx.views.data(), b->ctx.views.size() * sizeof(SysView),
                                      cudaMemcpyHostToDevice);
    if (ue != cudaSuccess) {
        cudaGraphDestroy(graph);
        return dyn::cuda_fail(ue, "batch views upload");
    }
    *out = graph;
    return DYN_OK;
}

}  // namespace

extern "C" int dyn_batch_destroy(dyn_batch_t b) {
    if (!b) return DYN_OK;
    if (b->stream) cudaStreamSynchronize(b->stream);
    for (int g = 0; g < 4; ++g) {
        if (b->graph[g]) cudaGraphExecDestroy(b->graph[g]);
        if (b->d_views[g]) cudaFree(b->d_views[g]);
    }
    for (void* p : b->map_allocs) cudaFree(p);
    for (dyn_sys_t m : b->members) dyn_sys_destroy(m);
    if (b->io.d_state) cudaFree(b->io.d_state);
    if (b->io.d_sc) cudaFree(b->io.d_sc);
    if (b->io.d_views) cudaFree(b->io.d_views);
    if (b->io.d_off) cudaFree(b->io.d_off);
    if (b->io.h_sc) cudaFreeHost(b->io.h_sc);
    if (b->io.h_buf) cudaFreeHost(b->io.h_buf);
    if (b->aux) cudaStreamDestroy(b->aux);
    if (b->window_ev) cudaEventDestroy(b->window_ev);
    b->br.destroy();
    for (int i = 0; i < BatchCtx::N_FFT; ++i)
        if (b->ctx.fft_st[i]) cudaStreamDestroy(b->ctx.fft_st[i]);
    for (int i = 0; i <= BatchCtx::N_FFT; ++i)
        if (b->ctx.fft_ev[i]) cudaEventDestroy(b->ctx.fft_ev[i]);
    if (b->own_stream) cudaStreamDestroy(b->stream);
    delete b;
    return DYN_OK;
}

extern "C" int dyn_batch_create(void* stream, uint32_t n, const dyn_config_t* cfgs,
                                const dyn_system_desc_t* systems, dyn_batch_t* out) {
    DYN_CHECK(out && (n == 0 || (cfgs && systems)), DYN_ERR_INVALID, "dyn_batch_create: NULL argument");
    *out = nullptr;
    for (uint32_t i = 1; i < n; ++i) {
        DYN_CHECK(std::max(1u, cfgs[i].spme_interval) == std::max(1u, cfgs[0].spme_interval) &&
                      std::max(1u, cfgs[i].energy_interval) == std::max(1u, cfgs[0].energy_interval),
                  DYN_ERR_INVALID, "dyn_batch_create: members must share spme_interval and energy_interval");
    }
    dyn_batch_s* b = new dyn_batch_s();
    b->stream = (cudaStream_t)stream;
    if (!b->stream) {
        const cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) { delete b; return dyn::cuda_fail(e, "cudaStreamCreateWithFlags"); }
        b->own_stream = true;
    }
    {
        const cudaError_t e = cudaStreamCreateWithFlags(&b->aux, cudaStreamNonBlocking);
        if (e != cudaSuccess) { dyn_batch_destroy(b); return dyn::cuda_fail(e, "cudaStreamCreateWithFlags"); }
        const int rc = b->br.create();
        if (rc != DYN_OK) { dyn_batch_destroy(b); return rc; }
        for (int i = 0; i < BatchCtx::N_FFT; ++i) {
            const cudaError_t e2 = cudaStreamCreateWithFlags(&b->ctx.fft_st[i], cudaStreamNonBlocking);
            if (e2 != cudaSuccess) { dyn_batch_destroy(b); return dyn::cuda_fail(e2, "cudaStreamCreateWithFlags"); }
        }
        for (int i = 0; i <= BatchCtx::N_FFT; ++i) {
            const cudaError_t e2 = cudaEventCreateWithFlags(&b->ctx.fft_ev[i], cudaEventDisableTiming);
            if (e2 != cudaSuccess) { dyn_batch_destroy(b); return dyn::cuda_fail(e2, "cudaEventCreateWithFlags"); }
        }
        b->ctx.n_fft = BatchCtx::N_FFT;
    }
    if (n > 0) {
        b->spme_interval = std::max(1u, cfgs[0].spme_interval);
        b->energy_interval = std::max(1u, cfgs[0].energy_interval);
        b->fixed_intervals = true;
    }
    for (uint32_t i = 0; i < n; ++i) {
        dyn_sys_t m = nullptr;
        const int rc = dyn_sys_create(b->stream, &cfgs[i], &systems[i], &m);
        if (rc == DYN_OK) dyn::set_batch_member(m);
        if (rc != DYN_OK) {
            const std::string msg = "dyn_batch_create: member " + std::to_string(i) + ": " + dyn_last_error();
            dyn_batch_destroy(b);
            return dyn::fail(rc, msg);
        }
        b->members.push_back(m);
    }
    *out = b;
    return DYN_OK;
}

extern "C" int dyn_batch_step(dyn_batch_t b, uint32_t n_steps, float dt) {
    DYN_CHECK(b, DYN_ERR_INVALID, "dyn_batch_step: NULL handle");
    DYN_CHECK(dt > 0.f && std::isfinite(dt), DYN_ERR_INVALID, "dyn_batch_step: dt must be > 0");
    if (b->members.empty()) return DYN_OK;
    for (uint32_t i = 0; i < n_steps; ++i) {
        const uint64_t s = b->host_step;
        const bool spme = (s % b->spme_interval) == 0;
        const bool energy = ((s + 1) % b->energy_interval) == 0;
        const int g = (spme ? 1 : 0) | (energy ? 2 : 0);
        if (!b->graph[g] || b->graph_dt[g] != dt) {
            if (b->graph[g]) { cudaGraphExecDestroy(b->graph[g]); b->graph[g] = nullptr; }
            cudaGraph_t graph = nullptr;
            const int rc = capture_batch_step(b, g, dt, spme, energy, &graph);
            if (rc != DYN_OK) return rc;
            const cudaError_t e = cudaGraphInstantiate(&b->graph[g], graph, 0);
            cudaGraphDestroy(graph);
            if (e != cudaSuccess) return dyn::cuda_fail(e, "cudaGraphInstantiate");
            b->graph_dt[g] = dt;
        }
        DYN_CUDA(cudaGraphLaunch(b->graph[g], b->stream));
        b->host_step += 1;
        for (dyn_sys_t m : b->members) m->host_step += 1;
        // at most about 2 x 512 steps queued at a time
        if ((i + 1) % 512 == 0 && i + 1 < n_steps) {
            if (!b->window_ev) DYN_CUDA(cudaEventCreateWithFlags(&b->window_ev, cudaEventDisableTiming));
            if (b->window_armed) DYN_CUDA(cudaEventSynchronize(b->window_ev));
            DYN_CUDA(cudaEventRecord(b->window_ev, b->stream));
            b->window_armed = true;
        }
    }
    b->window_armed = false;
    return DYN_OK;
}

extern "C" int dyn_batch_size(dyn_batch_t b, uint32_t* n) {
    DYN_CHECK(b && n, DYN_ERR_INVALID, "dyn_batch_size: NULL argument");
    *n = (uint32_t)b->members.size();
    return DYN_OK;
}

extern "C" int dyn_batch_member(dyn_batch_t b, uint32_t i, dyn_sys_t* out) {
    DYN_CHECK(b && out, DYN_ERR_INVALID, "dyn_batch_member: NULL argument");
    DYN_CHECK(i < b->members.size(), DYN_ERR_INVALID, "dyn_batch_member: index out of range");
    *out = b->members[i];
    return DYN_OK;
}

extern "C" int dyn_batch_sync(dyn_batch_t b) {
    DYN_CHECK(b, DYN_ERR_INVALID, "dyn_batch_sync: NULL handle");
    DYN_CUDA(cudaStreamSynchronize(b->stream));
    for (size_t i = 0; i < b->members.size(); ++i) {
        const int rc = dyn::read_scalars(b->members[i]);
        if (rc != DYN_OK) return dyn::fail(rc, "member " + std::to_string(i) + ": " + dyn_last_error());
    }
    return DYN_OK;
}

extern "C" int dyn_batch_launches(dyn_batch_t b, int spme, uint32_t* fixed, uint32_t* rebuild,
                                  uint32_t* periodic) {
    DYN_CHECK(b && fixed && rebuild && periodic, DYN_ERR_INVALID, "dyn_batch_launches: NULL argument");
    DYN_CUDA(cudaStreamSynchronize(b->stream));
    b->ctx.views.clear();
    for (dyn_sys_t m : b->members) b->ctx.views.push_back(m->v);
    const Target T{nullptr, &b->ctx, b->stream};
    // a collecting pass records one entry per batched launch and launches
    // nothing; cuFFT's per-member kernels are not counted
    auto count = [&](auto&& enqueue) {
        b->ctx.collecting = true;
        b->ctx.launches = 0;
        enqueue();
        b->ctx.collecting = false;
        return b->ctx.launches;
    };
    const uint32_t all = count([&] { enqueue_batch_step(b, 0.002f, spme != 0, true, false, 0, 0, 0); });
    *rebuild = count([&] {
        dyn::launch_rebuild(T, false);
        dyn::launch_prune(T, false);
    });
    *periodic = count([&] { dyn::launch_periodic(T); });
    *fixed = all - *rebuild - *periodic;
    return upload_maps(b);
}

namespace {

// After a membership change: the graphs and the block maps they reference
// describe the old member set.
void drop_graphs(dyn_batch_s* b) {
    for (int g = 0; g < 4; ++g)
        if (b->graph[g]) { cudaGraphExecDestroy(b->graph[g]); b->graph[g] = nullptr; }
    for (void* p : b->map_allocs) cudaFree(p);
    b->map_allocs.clear();
    b->ctx.maps.clear();
}

}  // namespace

extern "C" int dyn_batch_add(dyn_batch_t b, const dyn_config_t* cfg, const dyn_system_desc_t* system,
                             uint32_t* index) {
    DYN_CHECK(b && cfg && system, DYN_ERR_INVALID, "dyn_batch_add: NULL argument");
    if (b->fixed_intervals) {
        DYN_CHECK(std::max(1u, cfg->spme_interval) == b->spme_interval &&
                      std::max(1u, cfg->energy_interval) == b->energy_interval,
                  DYN_ERR_INVALID, "dyn_batch_add: members must share spme_interval and energy_interval");
    }
    // a member joins at a step where its SPME and energy schedule (counted
    // from its own step 0) matches the batch's
    DYN_CHECK(b->host_step % b->spme_interval == 0 && b->host_step % b->energy_interval == 0,
              DYN_ERR_INVALID, "dyn_batch_add: join only at a step that is a multiple of the SPME and "
              "energy intervals");
    DYN_CUDA(cudaStreamSynchronize(b->stream));
    dyn_sys_t m = nullptr;
    const int rc = dyn_sys_create(b->stream, cfg, system, &m);
    if (rc == DYN_OK) dyn::set_batch_member(m);
    if (rc != DYN_OK) return rc;
    if (!b->fixed_intervals) {
        b->spme_interval = std::max(1u, cfg->spme_interval);
        b->energy_interval = std::max(1u, cfg->energy_interval);
        b->fixed_intervals = true;
    }
    m->host_step = 0;
    drop_graphs(b);
    b->members.push_back(m);
    if (index) *index = (uint32_t)(b->members.size() - 1);
    return DYN_OK;
}

extern "C" int dyn_batch_remove(dyn_batch_t b, uint32_t i) {
    DYN_CHECK(b, DYN_ERR_INVALID, "dyn_batch_remove: NULL handle");
    DYN_CHECK(i < b->members.size(), DYN_ERR_INVALID, "dyn_batch_remove: index out of range");
    DYN_CUDA(cudaStreamSynchronize(b->stream));
    drop_graphs(b);
    dyn_sys_destroy(b->members[i]);
    b->members.erase(b->members.begin() + i);
    return DYN_OK;
}

extern "C" int dyn_batch_memory(dyn_batch_t b, uint64_t* bytes) {
    DYN_CHECK(b && bytes, DYN_ERR_INVALID, "dyn_batch_memory: NULL argument");
    uint64_t t = (uint64_t)b->views_cap * sizeof(SysView) * 4;
    for (dyn_sys_t m : b->members) t += m->bytes;
    for (auto& kv : b->ctx.maps) t += (uint64_t)kv.second.total * sizeof(uint2);
    *bytes = t;
    return DYN_OK;
}

// ---------------------------------------------------------------------------
// Batch-wide host step.  The packed host state holds, per member in order,
// atom_pos [na][3], atom_vel [na][3], water_pos [nw][3][3], water_vel
// [nw][3][3] (home order, as dyn_sys_step_host takes them); one copy moves
// all members' states each way and one launch scatters / gathers them
// (blockIdx.y = member).
// ---------------------------------------------------------------------------
namespace {

static_assert(sizeof(Scalars) % 8 == 0, "Scalars is copied as 8-byte words");

__global__ void k_batch_state_in(const SysView* __restrict__ vs, const unsigned long long* __restrict__ off,
                                 const float* __restrict__ stage) {
    const SysView& v = vs[blockIdx.y];
    const float* ap = stage + off[blockIdx.y];
    const float* av = ap + 3 * (size_t)v.na;
    const float* wp = av + 3 * (size_t)v.na;
    const float* wv = wp + 9 * (size_t)v.nw;
    const uint32_t n = v.nw_cap + v.na;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        if (t < v.nw_cap) water_in(v, t, wp, wv);
        else atom_in(v, t - v.nw_cap, ap, av);
    }
}

// stage == nullptr: the scalars only
__global__ void k_batch_state_out(const SysView* __restrict__ vs, const unsigned long long* __restrict__ off,
                                  float* __restrict__ stage, Scalars* __restrict__ sc) {
    const SysView& v = vs[blockIdx.y];
    if (blockIdx.x == 0) {
        const unsigned long long* src = reinterpret_cast<const unsigned long long*>(v.sc);
        unsigned long long* dst = reinterpret_cast<unsigned long long*>(sc + blockIdx.y);
        for (uint32_t k = threadIdx.x; k < sizeof(Scalars) / 8; k += blockDim.x) dst[k] = src[k];
    }
    if (!stage) return;
    float* ap = stage + off[blockIdx.y];
    float* av = ap + 3 * (size_t)v.na;
    float* wp = av + 3 * (size_t)v.na;
    float* wv = wp + 9 * (size_t)v.nw;
    const uint32_t n = v.nw_cap + v.na;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        if (t < v.nw_cap) water_out(v, t, wp, wv);
        else atom_out(v, t - v.nw_cap, ap, av);
    }
}

void host_layout(const dyn_batch_s* b, std::vector<unsigned long long>& off) {
    off.assign(b->members.size() + 1, 0ull);
    for (size_t i = 0; i < b->members.size(); ++i) {
        const SysView& v = b->members[i]->v;
        off[i + 1] = off[i] + 6ull * v.na + 18ull * v.nw;
    }
}

// Sizes the device areas for the current members and uploads their views
// and offsets when they changed (membership, or a member's arrays).
int ensure_io(dyn_batch_s* b) {
    auto& io = b->io;
    const size_t n = b->members.size();
    std::vector<unsigned long long> off;
    host_layout(b, off);
    if (off.back() > io.cap_floats) {
        if (io.d_state) cudaFree(io.d_state);
        io.d_state = nullptr;
        io.cap_floats = 0;
        DYN_CUDA(cudaMalloc(&io.d_state, off.back() * sizeof(float)));
        io.cap_floats = off.back();
    }
    if (n > io.cap_members) {
        if (io.d_sc) cudaFree(io.d_sc);
        if (io.d_views) cudaFree(io.d_views);
        if (io.d_off) cudaFree(io.d_off);
        if (io.h_sc) cudaFreeHost(io.h_sc);
        io.d_sc = nullptr; io.d_views = nullptr; io.d_off = nullptr; io.h_sc = nullptr;
        io.cap_members = 0;
        io.views.clear();
        const size_t cap = std::max<size_t>(8, 2 * n);
        DYN_CUDA(cudaMalloc(&io.d_sc, cap * sizeof(Scalars)));
        DYN_CUDA(cudaMalloc(&io.d_views, cap * sizeof(SysView)));
        DYN_CUDA(cudaMalloc(&io.d_off, (cap + 1) * sizeof(unsigned long long)));
        DYN_CUDA(cudaHostAlloc(&io.h_sc, cap * sizeof(Scalars), cudaHostAllocDefault));
        io.cap_members = cap;
    }
    bool same = io.views.size() == n && io.off == off;
    for (size_t i = 0; same && i < n; ++i)
        same = std::memcmp(&io.views[i], &b->members[i]->v, sizeof(SysView)) == 0;
    if (!same) {
        io.views.resize(n);
        for (size_t i = 0; i < n; ++i) io.views[i] = b->members[i]->v;
        io.off = off;
        DYN_CUDA(cudaMemcpyAsync(io.d_views, io.views.data(), n * sizeof(SysView), cudaMemcpyHostToDevice,
                                 b->stream));
        DYN_CUDA(cudaMemcpyAsync(io.d_off, io.off.data(), (n + 1) * sizeof(unsigned long long),
                                 cudaMemcpyHostToDevice, b->stream));
        DYN_CUDA(cudaStreamSynchronize(b->stream));  // the host vectors may change before the next call
    }
    return DYN_OK;
}

}  // namespace

extern "C" int dyn_batch_state_layout(dyn_batch_t b, uint64_t* offsets) {
    DYN_CHECK(b && offsets, DYN_ERR_INVALID, "dyn_batch_state_layout: NULL argument");
    std::vector<unsigned long long> off;
    host_layout(b, off);
    for (size_t i = 0; i < off.size(); ++i) offsets[i] = off[i];
    return DYN_OK;
}

extern "C" int dyn_batch_host_buffer(dyn_batch_t b, float** buf, uint64_t* n_floats) {
    DYN_CHECK(b && buf && n_floats, DYN_ERR_INVALID, "dyn_batch_host_buffer: NULL argument");
    std::vector<unsigned long long> off;
    host_layout(b, off);
    auto& io = b->io;
    if (off.back() > io.h_buf_floats || !io.h_buf) {
        DYN_CUDA(cudaStreamSynchronize(b->stream));
        if (io.h_buf) cudaFreeHost(io.h_buf);
        io.h_buf = nullptr;
        io.h_buf_floats = 0;
        const size_t nf = std::max<size_t>(off.back(), 1);
        const cudaError_t e = cudaHostAlloc(&io.h_buf, nf * sizeof(float), cudaHostAllocDefault);
        if (e != cudaSuccess) return dyn::fail(DYN_ERR_OOM, "dyn_batch_host_buffer: cudaHostAlloc failed");
        io.h_buf_floats = nf;
    }
    *buf = io.h_buf;
    *n_floats = off.back();
    return DYN_OK;
}

extern "C" int dyn_batch_step_host(dyn_batch_t b, uint32_t n_steps, float dt, const float* state_in,
                                   float* state_out, dyn_energies_t* energies) {
    DYN_CHECK(b, DYN_ERR_INVALID, "dyn_batch_step_host: NULL handle");
    DYN_CHECK(dt > 0.f && std::isfinite(dt), DYN_ERR_INVALID, "dyn_batch_step_host: dt must be > 0");
    if (b->members.empty()) return DYN_OK;
    int rc = ensure_io(b);
    if (rc != DYN_OK) return rc;
    auto& io = b->io;
    const uint32_t n = (uint32_t)b->members.size();
    DYN_CHECK(n <= 65535u, DYN_ERR_UNSUPPORTED, "dyn_batch_step_host: at most 65535 members");
    uint32_t most = 1;
    for (dyn_sys_t m : b->members) most = std::max(most, m->v.nw_cap + m->v.na);
    const dim3 grid(std::min(64u, (most + 255) / 256), n);
    const size_t bytes = io.off.back() * sizeof(float);
    if (state_in) {
        if (bytes) DYN_CUDA(cudaMemcpyAsync(io.d_state, state_in, bytes, cudaMemcpyHostToDevice, b->stream));
        k_batch_state_in<<<grid, 256, 0, b->stream>>>(io.d_views, io.d_off, io.d_state);
        DYN_CUDA(cudaGetLastError());
    }
    rc = dyn_batch_step(b, n_steps, dt);
    if (rc != DYN_OK) return rc;
    k_batch_state_out<<<grid, 256, 0, b->stream>>>(io.d_views, io.d_off, state_out ? io.d_state : nullptr, io.d_sc);
    DYN_CUDA(cudaGetLastError());
    if (state_out && bytes)
        DYN_CUDA(cudaMemcpyAsync(state_out, io.d_state, bytes, cudaMemcpyDeviceToHost, b->stream));
    DYN_CUDA(cudaMemcpyAsync(io.h_sc, io.d_sc, n * sizeof(Scalars), cudaMemcpyDeviceToHost, b->stream));
    DYN_CUDA(cudaStreamSynchronize(b->stream));
    for (uint32_t i = 0; i < n; ++i) {
        dyn_sys_t m = b->members[i];
        std::memcpy(m->h_sc, &io.h_sc[i], sizeof(Scalars));
        if (energies) dyn::energies_of(m, &energies[i]);
    }
    for (uint32_t i = 0; i < n; ++i) {
        const int e = dyn::check_scalars(b->members[i]);
        if (e != DYN_OK) return dyn::fail(e, "member " + std::to_string(i) + ": " + dyn_last_error());
    }
    return DYN_OK;
}
