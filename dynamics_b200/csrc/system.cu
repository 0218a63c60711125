// Layer 2 of the C ABI: the device-resident engine behind MdState::step
// (src/integrate.rs:72-473).  One handle owns one system's HBM state, its
// CUDA stream, two cuFFT plans and up to four captured CUDA graphs (step
// with/without SPME, with/without energies).  A step is entirely on the
// device; the host only picks which graph to launch.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "sys_internal.cuh"

using dyn::begin_if_body;
using dyn::count_graph_kernels;
using dyn::end_if_body;
using dyn::read_scalars;

namespace {

template <typename T>
int dev_alloc(dyn_sys_s* h, T** p, size_t n, bool zero = true) {
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
    if (e != cudaSuccess) return dyn::cuda_fail(e, "cudaMalloc");
    h->allocs.push_back((void*)*p);
    h->bytes += n * sizeof(T);
    if (zero) {
        e = cudaMemsetAsync(*p, 0, n * sizeof(T), h->stream);
        if (e != cudaSuccess) return dyn::cuda_fail(e, "cudaMemsetAsync");
    }
    return DYN_OK;
}

template <typename T>
int upload(dyn_sys_s* h, T* d, const T* src, size_t n) {
    if (n == 0 || src == nullptr) return DYN_OK;
    cudaError_t e = cudaMemcpyAsync(d, src, n * sizeof(T), cudaMemcpyHostToDevice, h->stream);
    if (e != cudaSuccess) return dyn::cuda_fail(e, "cudaMemcpyAsync H2D");
    return DYN_OK;
}

inline uint32_t round8(uint32_t x) { return (x + 7u) / 8u * 8u; }
inline uint32_t round_up(uint32_t x, uint32_t m) { return (x + m - 1u) / m * m; }

// Chebyshev interpolation of f(x) on x = xmax (s + 1) / 2, s in [-1, 1],
// at N Chebyshev nodes, converted to power-basis coefficients in s.
template <int N, typename F>
void cheb_poly(F f, double xmax, float* out) {
    const int n = N;
    double c[N];
    for (int k = 0; k < n; ++k) {
        double sum = 0.0;
        for (int j = 0; j < n; ++j) {
            const double th = M_PI * (j + 0.5) / n;
            sum += f(xmax * (std::cos(th) + 1.0) * 0.5) * std::cos(k * th);
        }
        c[k] = 2.0 / n * sum;
    }
    c[0] *= 0.5;
    double T[N][N] = {};
    T[0][0] = 1.0;
    if (n > 1) T[1][1] = 1.0;
    for (int k = 1; k + 1 < n; ++k)
        for (int m = 0; m < n; ++m)
            T[k + 1][m] = (m > 0 ? 2.0 * T[k][m - 1] : 0.0) - T[k - 1][m];
    for (int m = 0; m < n; ++m) {
        double p = 0.0;
        for (int k = 0; k < n; ++k) p += c[k] * T[k][m];
        out[m] = (float)p;
    }
}

// Water M site from O, H0, H1 on the host (src/solvent/mod.rs:411-422).
void host_m_site(const float* o, const float* h0, const float* h1, float* m) {
    double b[3];
    for (int k = 0; k < 3; ++k) b[k] = ((double)h0[k] - o[k]) + ((double)h1[k] - o[k]);
    const double n = std::sqrt(b[0] * b[0] + b[1] * b[1] + b[2] * b[2]);
    for (int k = 0; k < 3; ++k) m[k] = (float)(o[k] + b[k] / n * (double)OPC_O_EP_R);
}

// Waters per shared-memory chunk of the water-water kernel with ctas CTAs
// per SM (each CTA also needs 1 KB reserved plus < 5 KB static shared):
// per staged water its 4 site positions, its 12 int32 j sums and its slot,
// no more than the union capacity, and no more than cfg->ww_union_chunk
// when that is set.
uint32_t ww_chunk_for(const SysView& v, const dyn_config_t* cfg, int ctas) {
    int dev = 0, smem_sm = 0, smem_blk = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&smem_blk, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    size_t per_cta = smem_sm > 6144 * ctas ? (size_t)smem_sm / ctas - 6144 : 48 * 1024;
    per_cta = std::min<size_t>(per_cta, smem_blk > 0 ? (size_t)smem_blk : per_cta);
    const uint32_t fit =
        (uint32_t)((per_cta - 12 * sizeof(int)) / (4 * sizeof(float4) + 13 * sizeof(int))) / 32 * 32;
    uint32_t chunk = std::max<uint32_t>(32u, std::min<uint32_t>(fit, (v.cap_union + 31) / 32 * 32));
    if (cfg->ww_union_chunk) chunk = std::max<uint32_t>(32u, std::min<uint32_t>(chunk, cfg->ww_union_chunk / 32 * 32));
    return chunk;
}

void set_block_counts(SysView& v) {
    for (int r = 0; r < NREGION; ++r) v.nb[r] = 0;
    v.nb[REG_WW] = v.nw ? dyn::ww_tile_blocks(v) : 0;
    // the atom pair kernels write one partial per warp (4 per block)
    v.nb[REG_WS] = (v.nw && v.na) ? 4u * dyn::pair_blocks_ws(v) : 0;
    v.nb[REG_SW] = 0;
    v.nb[REG_SS] = v.na ? 4u * dyn::pair_blocks_ss(v) : 0;
    v.nb[REG_14] = v.n14 ? dyn::pair14_blocks(v) : 0;
    v.nb[REG_BOND] = (v.nbond + v.nangle + v.ndih) ? dyn::bond_blocks(v) : 0;
    v.nb[REG_KICK_W] = v.nw ? dyn::kick_blocks_w(v) : 0;
    v.nb[REG_KICK_A] = v.na ? dyn::kick_blocks_a(v) : 0;
    v.nb[REG_CONS] = v.na ? dyn::kick_blocks_a(v) : 0;  // written by the atoms' first half
    v.nb[REG_PME] = dyn::pme_blocks(v);
    v.nb[REG_CORR] = dyn::gather_blocks(v);
    v.nb[REG_CORR_A] = dyn::corr_blocks(v);
    v.nb[REG_COM] = dyn::kick_blocks_w(v) > dyn::kick_blocks_a(v) ? dyn::kick_blocks_w(v)
                                                                   : dyn::kick_blocks_a(v);
}

// Inside an active capture on st: appends an IF node on hc after everything
// captured so far (later work depends on it) and starts capturing its body
// on aux.
}  // namespace
namespace dyn {
int begin_if_body(cudaStream_t st, cudaStream_t aux, cudaGraphConditionalHandle hc, cudaGraph_t* body) {
    cudaStreamCaptureStatus cs;
    cudaGraph_t cg = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    DYN_CUDA(cudaStreamGetCaptureInfo(st, &cs, nullptr, &cg, &deps, &nd));
    cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
    cp.conditional.handle = hc;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    DYN_CUDA(cudaGraphAddNode(&node, cg, deps, nd, &cp));
    DYN_CUDA(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
    *body = cp.conditional.phGraph_out[0];
    DYN_CUDA(cudaStreamBeginCaptureToGraph(aux, *body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    return DYN_OK;
}
}  // namespace dyn
namespace {

}  // namespace
namespace dyn {
int end_if_body(cudaStream_t aux) {
    cudaGraph_t g = nullptr;
    DYN_CUDA(cudaStreamEndCapture(aux, &g));
    return DYN_OK;
}

// Work enqueued on `to` after this call depends on everything enqueued on
// `from` before it.
static int link_streams(cudaStream_t from, cudaStream_t to, cudaEvent_t e) {
    DYN_CUDA(cudaEventRecord(e, from));
    DYN_CUDA(cudaStreamWaitEvent(to, e, 0));
    return DYN_OK;
}

int enqueue_first_half(const Target& T, const Target& A, const Branches& br, bool fork, float dt) {
    int rc;
    if (fork && (rc = link_streams(T.st, A.st, br.ev[0])) != DYN_OK) return rc;
    launch_first_half_water(T, dt);
    launch_first_half_atoms(fork ? A : T, dt);
    if (fork && (rc = link_streams(A.st, T.st, br.ev[1])) != DYN_OK) return rc;
    return DYN_OK;
}

int enqueue_forces(const Target& T, const Target& A, const Target& P, const Branches& br, bool fork, bool spme,
                   bool energy) {
    int rc;
    if (fork && (rc = link_streams(T.st, A.st, br.ev[2])) != DYN_OK) return rc;
    if (fork && spme && (rc = link_streams(T.st, P.st, br.ev[3])) != DYN_OK) return rc;
    const Target& a = fork ? A : T;
    const Target& p = fork ? P : T;
    if (spme) {
        launch_pme(p);
        launch_corrections(p);
    }
    launch_pairs_atoms(a, energy);
    launch_pair14(a, energy);
    launch_bonded(a, energy);
    launch_pairs_water(T, energy);
    if (fork && (rc = link_streams(A.st, T.st, br.ev[4])) != DYN_OK) return rc;
    if (fork && spme && (rc = link_streams(P.st, T.st, br.ev[5])) != DYN_OK) return rc;
    return DYN_OK;
}

int enqueue_second_half(const Target& T, const Target& A, const Branches& br, bool fork, float dt) {
    int rc;
    if (fork && (rc = link_streams(T.st, A.st, br.ev[6])) != DYN_OK) return rc;
    launch_second_half_water(T, dt);
    launch_second_half_atoms(fork ? A : T, dt);
    if (fork && (rc = link_streams(A.st, T.st, br.ev[7])) != DYN_OK) return rc;
    return DYN_OK;
}
}  // namespace dyn

int Branches::create() {
    for (int i = 0; i < 2; ++i) DYN_CUDA(cudaStreamCreateWithFlags(&side[i], cudaStreamNonBlocking));
    for (int i = 0; i < 8; ++i) DYN_CUDA(cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming));
    return DYN_OK;
}

void Branches::destroy() {
    for (int i = 0; i < 2; ++i)
        if (side[i]) { cudaStreamDestroy(side[i]); side[i] = nullptr; }
    for (int i = 0; i < 8; ++i)
        if (ev[i]) { cudaEventDestroy(ev[i]); ev[i] = nullptr; }
}
namespace {

// Captures one step (MdState::step, src/integrate.rs:100-473) into a graph.
// The list rebuild and the periodic tasks (COM removal, recentering,
// reset_angle) sit under IF nodes that the displacement check and the step
// finalisation set on the device, so a step that needs neither launches none
// of their kernels.  body_rebuild / body_periodic receive the bodies (owned
// by *out).
int capture_step(dyn_sys_s* h, float dt, bool spme, bool energy, cudaGraph_t* out,
                 cudaGraph_t* body_rebuild = nullptr, cudaGraph_t* body_periodic = nullptr) {
    SysView& v = h->v;
    cudaStream_t st = h->stream;
    const Target T{&v, nullptr, st};
    const Target TA{&v, nullptr, h->aux};
    const Target S0{&v, nullptr, h->br.side[0]}, S1{&v, nullptr, h->br.side[1]};
    *out = nullptr;
    DYN_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int rc = DYN_OK;
    cudaGraph_t br = nullptr, bp = nullptr;
    do {
        cudaStreamCaptureStatus cs;
        cudaGraph_t cg = nullptr;
        cudaError_t e = cudaStreamGetCaptureInfo(st, &cs, nullptr, &cg, nullptr, nullptr);
        if (e == cudaSuccess)
            e = cudaGraphConditionalHandleCreate(&v.cond_rebuild, cg, 0, cudaGraphCondAssignDefault);
        if (e == cudaSuccess)
            e = cudaGraphConditionalHandleCreate(&v.cond_periodic, cg, 0, cudaGraphCondAssignDefault);
        if (e == cudaSuccess)
            e = cudaGraphConditionalHandleCreate(&v.cond_prune, cg, 0, cudaGraphCondAssignDefault);
        if (e != cudaSuccess) { rc = dyn::cuda_fail(e, "cudaGraphConditionalHandleCreate"); break; }
        v.use_cond = 1;
        if ((rc = dyn::enqueue_first_half(T, S0, h->br, true, dt)) != DYN_OK) break;
        dyn::launch_displacement_check(T);
        if ((rc = begin_if_body(st, h->aux, v.cond_rebuild, &br)) != DYN_OK) break;
        dyn::launch_rebuild(TA, false);
        if ((rc = end_if_body(h->aux)) != DYN_OK) break;
        cudaGraph_t bpr = nullptr;
        if ((rc = begin_if_body(st, h->aux, v.cond_prune, &bpr)) != DYN_OK) break;
        dyn::launch_prune(TA, false);
        if ((rc = end_if_body(h->aux)) != DYN_OK) break;
        dyn::launch_gather_atoms(T);
        if ((rc = dyn::enqueue_forces(T, S0, S1, h->br, true, spme, energy)) != DYN_OK) break;
        if ((rc = dyn::enqueue_second_half(T, S0, h->br, true, dt)) != DYN_OK) break;
        dyn::launch_finalize(T, dt, energy, true);
        if ((rc = begin_if_body(st, h->aux, v.cond_periodic, &bp)) != DYN_OK) break;
        dyn::launch_periodic(TA);
        if ((rc = end_if_body(h->aux)) != DYN_OK) break;
    } while (0);
    v.use_cond = 0;
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(st, &g);
    if (rc == DYN_OK && e != cudaSuccess) rc = dyn::cuda_fail(e, "cudaStreamEndCapture");
    if (rc == DYN_OK) {
        const cudaError_t le = cudaGetLastError();
        if (le != cudaSuccess) rc = dyn::cuda_fail(le, "kernel launch during capture");
    }
    if (rc != DYN_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    *out = g;
    if (body_rebuild) *body_rebuild = br;
    if (body_periodic) *body_periodic = bp;
    return DYN_OK;
}

// Forces at the current coordinates (no integration); dt = 0 kicks set the
// accelerations without changing velocities.
void enqueue_forces(dyn_sys_s* h, bool force_rebuild) {
    const SysView& v = h->v;
    cudaStream_t st = h->stream;
    const Target T{&v, nullptr, st};
    if (!force_rebuild) dyn::launch_displacement_check(T);
    dyn::launch_rebuild(T, force_rebuild);
    dyn::launch_prune(T, force_rebuild);
    dyn::launch_gather_atoms(T);
    dyn::launch_pairs(T, true);
    dyn::launch_pair14(T, true);
    dyn::launch_bonded(T, true);
    dyn::launch_pme(T);
    dyn::launch_corrections(T);
    dyn::launch_second_half(T, 0.0f);
    dyn::launch_finalize(T, 0.0f, true, false);
}

int evaluate_forces_now(dyn_sys_s* h) {
    enqueue_forces(h, true);
    return dyn::read_scalars(h);
}

}  // namespace
namespace dyn {
int read_scalars(dyn_sys_s* h) {
    DYN_CUDA(cudaMemcpyAsync(h->h_sc, h->v.sc, sizeof(Scalars), cudaMemcpyDeviceToHost, h->stream));
    DYN_CUDA(cudaStreamSynchronize(h->stream));
    return check_scalars(h);
}

int check_scalars(dyn_sys_s* h) {
    if (h->h_sc->overflow)
        return dyn::fail(DYN_ERR_UNSUPPORTED, "cluster list capacity exceeded (list length " +
                                                  std::to_string(h->h_sc->overflow) + ")");
    if (h->h_sc->nonfinite) return dyn::fail(DYN_ERR_NONFINITE, "non-finite coordinates or forces");
    if (h->h_sc->timeout) return dyn::fail(DYN_ERR_TIMEOUT, "a bounded device wait gave up");
    return DYN_OK;
}
}  // namespace dyn
namespace {

void fill_energies(dyn_sys_s* h, dyn_energies_t* e) {
    const Scalars& s = *h->h_sc;
    std::memset(e, 0, sizeof(*e));
    e->kinetic = s.acc[ACC_KE];
    e->kinetic_trans = s.acc[ACC_KE_TRANS];
    e->potential = s.pe;
    e->e_lj = s.acc[ACC_E_LJ_WW] + s.acc[ACC_E_LJ_S];
    e->e_coul_short = s.acc[ACC_E_COUL_WW] + s.acc[ACC_E_COUL_S];
    e->e_water_water_short = s.acc[ACC_E_LJ_WW] + s.acc[ACC_E_COUL_WW];
    e->e_recip = s.acc[ACC_E_RECIP];
    e->e_corrections = s.acc[ACC_E_CORR];
    e->e_bonded = s.acc[ACC_E_BONDED] + s.acc[ACC_E_14];
    e->virial_short = s.acc[ACC_VIR_SHORT];
    e->virial_recip = s.acc[ACC_VIR_RECIP] + s.acc[ACC_VIR_CORR];
    e->virial_bonded = s.acc[ACC_VIR_BONDED];
    e->virial_constraints = s.acc[ACC_VIR_CONSTR] / (double)KCAL_TO_NATIVE;
    e->virial = e->virial_short + e->virial_recip + e->virial_bonded + e->virial_constraints;
    e->pressure_bar = s.pressure;
    e->temperature = s.temperature;
    e->step = s.step;
    e->list_rebuilds = s.rebuilds;
    e->pairs_in_list = s.list_pairs;
    e->kinetic_rigid = s.ke_rigid;
    e->pressure_atomic_bar = s.pressure_atomic;
    e->list_union_max = s.union_max;
    e->dh_dl = s.dh_dl;
    e->list_prunes = s.prunes;
}

// staged_decoupling_schedule (src/alchemical.rs:77-96): Coulomb scaled
// 1 - 2 lambda over lambda < 0.5, then LJ soft-core lambda 2 lambda - 1
void set_alch_schedule(SysView& v, float lambda) {
    const float l = std::min(1.0f, std::max(0.0f, lambda));
    if (l < 0.5f) {
        v.alch_cs = 1.0f - 2.0f * l; v.alch_dcs = -2.0f;
        v.alch_ll = 0.0f; v.alch_dll = 0.0f;
    } else {
        v.alch_cs = 0.0f; v.alch_dcs = 0.0f;
        v.alch_ll = 2.0f * l - 1.0f; v.alch_dll = 2.0f;
    }
}

}  // namespace

extern "C" int dyn_sys_destroy(dyn_sys_t h) {
    if (!h) return DYN_OK;
    if (h->stream) cudaStreamSynchronize(h->stream); else cudaDeviceSynchronize();
    for (int g = 0; g < 4; ++g)
        if (h->graph[g]) cudaGraphExecDestroy(h->graph[g]);
    if (h->plan_f) cufftDestroy(h->plan_f);
    if (h->plan_b) cufftDestroy(h->plan_b);
    for (void* p : h->allocs) cudaFree(p);
    if (h->snap_mem) cudaFree(h->snap_mem);
    if (h->h_sc) cudaFreeHost(h->h_sc);
    if (h->own_stream) cudaStreamDestroy(h->stream);
    if (h->aux) cudaStreamDestroy(h->aux);
    if (h->window_ev) cudaEventDestroy(h->window_ev);
    h->br.destroy();
    delete h;
    return DYN_OK;
}

extern "C" int dyn_sys_create(void* stream, const dyn_config_t* cfg, const dyn_system_desc_t* d,
                              dyn_sys_t* out) {
    DYN_CHECK(cfg && d && out, DYN_ERR_INVALID, "dyn_sys_create: NULL argument");
    *out = nullptr;
    DYN_CHECK(d->n_atoms + d->n_water > 0, DYN_ERR_INVALID, "dyn_sys_create: empty system");
    DYN_CHECK(d->n_water == 0 || (d->water_pos && d->water_vel), DYN_ERR_INVALID,
              "dyn_sys_create: water arrays required");
    DYN_CHECK(d->n_atoms == 0 || (d->atom_pos && d->atom_vel && d->atom_mass && d->atom_q &&
                                  d->atom_sigma && d->atom_eps),
              DYN_ERR_INVALID, "dyn_sys_create: atom arrays required");
    float ext[3];
    for (int k = 0; k < 3; ++k) {
        ext[k] = cfg->box_hi[k] - cfg->box_lo[k];
        DYN_CHECK(ext[k] > 0.f, DYN_ERR_INVALID, "dyn_sys_create: box extent must be > 0");
    }
    const float rc = cfg->coulomb_cutoff, ljc = cfg->lj_cutoff > 0.f ? cfg->lj_cutoff : rc;
    DYN_CHECK(rc > 0.f && cfg->ewald_alpha > 0.f && cfg->list_buffer >= 0.f, DYN_ERR_INVALID,
              "dyn_sys_create: cutoff and alpha must be > 0, buffer >= 0");
    const float lmin = std::min(ext[0], std::min(ext[1], ext[2]));
    DYN_CHECK(std::max(rc, ljc) + 2.0f * OPC_SITE_REACH < 0.5f * lmin, DYN_ERR_INVALID,
              "dyn_sys_create: cutoff + 2 * 0.8725 A must be below half the smallest box edge");
    for (int k = 0; k < 3; ++k)
        DYN_CHECK(cfg->grid[k] >= 8 && cfg->grid[k] <= 1024, DYN_ERR_INVALID,
                  "dyn_sys_create: grid dimensions must be in [8, 1024]");
    DYN_CHECK(cfg->integrator <= 1 && cfg->thermostat <= 1 && cfg->barostat <= 1, DYN_ERR_INVALID,
              "dyn_sys_create: unknown integrator/thermostat/barostat");
    for (uint32_t i = 0; i < d->n_excl * 2; ++i)
        DYN_CHECK(d->excl[i] < d->n_atoms, DYN_ERR_INVALID, "dyn_sys_create: exclusion index out of range");
    for (uint32_t i = 0; i < d->n_pair14 * 2; ++i)
        DYN_CHECK(d->pair14[i] < d->n_atoms, DYN_ERR_INVALID, "dyn_sys_create: 1-4 index out of range");
    for (uint32_t i = 0; i < d->n_bonds * 2; ++i)
        DYN_CHECK(d->bonds[i] < d->n_atoms, DYN_ERR_INVALID, "dyn_sys_create: bond index out of range");
    for (uint32_t i = 0; i < d->n_angles * 3; ++i)
        DYN_CHECK(d->angles[i] < d->n_atoms, DYN_ERR_INVALID, "dyn_sys_create: angle index out of range");
    for (uint32_t i = 0; i < d->n_dihedrals * 4; ++i)
        DYN_CHECK(d->dihedrals[i] < d->n_atoms, DYN_ERR_INVALID, "dyn_sys_create: dihedral index out of range");
    for (uint32_t i = 0; i < d->n_atoms; ++i)
        DYN_CHECK(d->atom_mass[i] > 0.f || (d->atom_static && d->atom_static[i]), DYN_ERR_INVALID,
                  "dyn_sys_create: non-static atoms need mass > 0");
    // constraint units: each heavy atom with the H constrained to it
    std::vector<std::vector<uint32_t>> unit_h(d->n_atoms);
    std::vector<float> h_r02(d->n_atoms, 0.f);
    {
        std::vector<uint8_t> role(d->n_atoms, 0);  // 1 heavy end, 2 H end
        for (uint32_t c = 0; c < d->n_constraints; ++c) {
            DYN_CHECK(d->constraints && d->constraint_r0, DYN_ERR_INVALID, "dyn_sys_create: NULL constraint array");
            const uint32_t a = d->constraints[2 * c], b = d->constraints[2 * c + 1];
            DYN_CHECK(a < d->n_atoms && b < d->n_atoms && a != b, DYN_ERR_INVALID,
                      "dyn_sys_create: constraint index out of range");
            DYN_CHECK(d->constraint_r0[c] > 0.f, DYN_ERR_INVALID, "dyn_sys_create: constraint_r0 must be > 0");
            const uint32_t hv = d->atom_mass[a] >= d->atom_mass[b] ? a : b, hy = hv == a ? b : a;
            DYN_CHECK(role[hy] == 0 && role[hv] != 2, DYN_ERR_UNSUPPORTED,
                      "dyn_sys_create: constraints must be bonds from a heavy atom to its own hydrogens");
            role[hy] = 2;
            role[hv] = 1;
            unit_h[hv].push_back(hy);
            h_r02[hy] = d->constraint_r0[c] * d->constraint_r0[c];
            DYN_CHECK(unit_h[hv].size() < UMAX, DYN_ERR_UNSUPPORTED,
                      "dyn_sys_create: more than 4 hydrogens constrained to one atom");
        }
    }

    dyn_sys_s* h = new dyn_sys_s();
    h->stream = (cudaStream_t)stream;
    if (!h->stream) {
        // graphs cannot be captured on the legacy default stream
        cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) { delete h; return dyn::cuda_fail(e, "cudaStreamCreateWithFlags"); }
        h->own_stream = true;
    }
    {
        cudaError_t e = cudaStreamCreateWithFlags(&h->aux, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            if (h->own_stream) cudaStreamDestroy(h->stream);
            delete h;
            return dyn::cuda_fail(e, "cudaStreamCreateWithFlags");
        }
        const int rc = h->br.create();
        if (rc != DYN_OK) {
            dyn_sys_destroy(h);
            return rc;
        }
    }
    h->cfg = *cfg;
    SysView& v = h->v;
    int rc_ = DYN_OK;
#define TRY(x) do { if ((rc_ = (x)) != DYN_OK) { dyn_sys_destroy(h); return rc_; } } while (0)
#define TRYC(x) do { cudaError_t _e = (x); if (_e != cudaSuccess) { rc_ = dyn::cuda_fail(_e, #x); dyn_sys_destroy(h); return rc_; } } while (0)
    TRYC(cudaMallocHost((void**)&h->h_sc, sizeof(Scalars)));
    std::memset(h->h_sc, 0, sizeof(Scalars));

    v.nw = d->n_water;
    v.na = d->n_atoms;
    if (cfg->alch_end > cfg->alch_begin) {
        DYN_CHECK(cfg->alch_end <= d->n_atoms, DYN_ERR_INVALID, "dyn_sys_create: alchemical range beyond the atoms");
        DYN_CHECK(std::isfinite(cfg->alch_lambda), DYN_ERR_INVALID, "dyn_sys_create: alch_lambda not finite");
        v.alch_on = 1u;
        v.alch_lo = cfg->alch_begin;
        v.alch_hi = cfg->alch_end;
    }
    set_alch_schedule(v, cfg->alch_lambda);
    v.total_mass = (double)v.nw * (double)OPC_MASS_MOL;
    for (uint32_t a = 0; a < v.na && d->atom_mass; ++a) v.total_mass += (double)d->atom_mass[a];
    // parameters
    v.rc = rc; v.rc2 = rc * rc; v.ljc2 = ljc * ljc; v.alpha = cfg->ewald_alpha;
    v.buffer = cfg->list_buffer;
    v.r_ww = std::max(ljc, rc + 2.0f * OPC_SITE_REACH) + v.buffer;
    v.r_ws = std::max(ljc, rc + OPC_SITE_REACH) + v.buffer;
    v.r_ss = std::max(ljc, rc) + v.buffer;
    {
        const float rs = std::max(ljc, rc + OPC_SITE_REACH);
        v.r_ws_skip2 = rs * rs;
    }
    // pruned water-water lists (an inner buffer at most the outer one)
    v.prune_buf = std::min(cfg->prune_buffer > 0.f ? cfg->prune_buffer : 0.4f, v.buffer);
    v.r_in = std::max(ljc, rc + 2.0f * OPC_SITE_REACH) + v.prune_buf;
    v.flags = cfg->flags; v.seed = cfg->seed;
    v.temperature = cfg->temperature; v.gamma = cfg->langevin_gamma; v.tau_t = cfg->tau_temp;
    v.p_target = cfg->pressure_bar; v.tau_p = cfg->tau_pressure; v.kappa = cfg->compressibility;
    v.thermo_dof = cfg->thermo_dof;
    v.integrator = cfg->integrator; v.thermostat = cfg->thermostat; v.barostat = cfg->barostat;
    v.spme_interval = std::max(1u, cfg->spme_interval);
    v.com_interval = cfg->com_interval; v.recenter_interval = cfg->recenter_interval;
    for (int k = 0; k < 3; ++k) v.K[k] = cfg->grid[k];

    // column grid: edge close to that of a cube holding one 32-water group
    const double vol = (double)ext[0] * ext[1] * ext[2];
    const double dens = (double)std::max<uint32_t>(1u, v.nw + v.na / 3) / vol;
    const double edge = std::cbrt((double)GRPW / dens);
    v.ncx = std::max(1u, (uint32_t)std::floor(ext[0] / edge));
    v.ncy = std::max(1u, (uint32_t)std::floor(ext[1] / edge));
    v.ncol = v.ncx * v.ncy;
    // atoms (peptide density ~0.1 per A^3): columns about one 8-atom cube wide
    const double aedge = std::cbrt(8.0 / 0.1);
    v.ancx = std::min(1024u, std::max(1u, (uint32_t)std::floor(ext[0] / aedge)));
    v.ancy = std::min(1024u, std::max(1u, (uint32_t)std::floor(ext[1] / aedge)));
    v.ancol = v.ancx * v.ancy;
    // slots follow the column path without per-column padding; the tail is
    // padded to whole 32-water groups
    v.nw_cap = round_up(std::max(1u, v.nw), 2 * GRPW);
    v.nwclus_cap = v.nw_cap / WCL;
    // atoms without bonds (ions) take a cluster each, after the others
    std::vector<uint32_t> sparse_rank(std::max(1u, v.na), INVALID_ID);
    {
        std::vector<uint8_t> bonded(v.na, 0);
        for (uint32_t i = 0; i < 2 * d->n_bonds; ++i) bonded[d->bonds[i]] = 1;
        for (uint32_t i = 0; i < 2 * d->n_constraints; ++i) bonded[d->constraints[i]] = 1;
        uint32_t k = 0;
        for (uint32_t a = 0; a < v.na; ++a)
            if (!bonded[a]) sparse_rank[a] = k++;
        v.n_sparse = k;
    }
    v.na_cap = round8(v.na - v.n_sparse + 8) + ACL * v.n_sparse;
    v.naclus_cap = v.na_cap / ACL;
    v.max_blocks = 148 * 16;

    // list capacities from the cluster density, generous margin
    auto est = [&](double r, double cl_vol, uint32_t ncl) -> uint32_t {
        const double rad = r + 2.0 * 0.9 * std::cbrt(cl_vol);
        const double n = 4.0 / 3.0 * M_PI * rad * rad * rad / cl_vol;
        const uint32_t e = (uint32_t)(2.0 * n) + 32;
        return std::max(1u, std::min(e, ncl));
    };
    const double wcl_vol = v.nw ? vol / std::max(1.0, v.nw / 8.0) : vol;
    const double acl_vol = 8.0 / 0.1;  // clusters of a dense solute; ions are few
    // water-water: 32-water groups; candidate clusters within r_ww of the
    // group box; the union of needed waters; molecule lists within r_ww
    // (liquid density as the bound)
    // counts at liquid density or the system's, whichever is higher;
    // extents of groups and clusters at the lower of the two (a group drawn
    // from a dilute region spans more space, and may sit next to liquid)
    const double dl = std::max(0.0334, v.nw / vol);
    const double dx = std::max(1e-3, std::min(0.0334, v.nw / vol));
    v.ngrp_cap = v.nw_cap / GRPW;
    {
        const double r = v.r_ww;
        auto mink = [&](double a) {
            return a * a * a + 6.0 * a * a * r + 3.0 * M_PI * a * r * r + 4.0 / 3.0 * M_PI * r * r * r;
        };
        const double ag = 1.4 * std::cbrt(GRPW / dx), ac = 2.0 * std::cbrt(WCL / dx);
        v.cap_tile = std::min<uint32_t>((uint32_t)(2.0 * mink(ag + ac) * dl / WCL) + 16,
                                        std::max<uint32_t>(1u, v.nwclus_cap));
        // unions larger than the shared-memory chunk are processed in
        // several chunks, so this is only the list-build capacity
        v.cap_union = std::min<uint32_t>((uint32_t)(2.8 * mink(ag) * dl) + 64, 65534u);
        v.cap_union = std::min<uint32_t>(v.cap_union, v.nw_cap);
        // shared-memory chunk of the water-water kernel: three CTAs per SM
        v.union_chunk = ww_chunk_for(v, cfg, 3);
        v.cap_run = v.cap_union;  // a run per union water at worst
        // fewer water groups than SMs: several CTAs share each group's entries
        int dev = 0, n_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
        v.ww_split = v.ngrp_cap ? std::max<uint32_t>(1u, std::min<uint32_t>(8u, ((uint32_t)std::max(n_sm, 1) +
                                                                               v.ngrp_cap - 1) / v.ngrp_cap))
                                : 1u;
        if (cfg->ww_split) v.ww_split = std::min(8u, cfg->ww_split);
        const double nb = 4.0 / 3.0 * M_PI * r * r * r * dl;
        // half lists: about nb / 2 partners above a water's slot on average,
        // but the first waters of the slot order keep nearly all of theirs
        // (their periodic neighbours sit at the end of the order)
        v.cap_nb = std::min<uint32_t>((uint32_t)(1.5 * nb) + 32, 65535u);
    }
    DYN_CHECK((uint64_t)v.ngrp_cap * v.cap_union < (1ull << 32), DYN_ERR_UNSUPPORTED,
              "dyn_sys_create: too many waters in one system");
    // screened-Coulomb force: F = q q (r^-3 + g(r^2)) d for r < rc with
    // g(z) = 2 d/dz [erf(alpha sqrt z) / sqrt z], an entire function of z
    // fitted on [0, rc^2]; the r^-3 part is exact, so no cancellation-free
    // form of erfc is needed
    {
        const double a = v.alpha;
        auto g = [a](double z) {
            const double x2 = a * a * z;
            const double c = 2.0 * a / std::sqrt(M_PI);
            if (x2 < 0.25) {
                // h = c sum_n (-a^2 z)^n / (n! (2n+1)) (the series of
                // erf(x)/x), differentiated term by term in z
                double sum = 0.0, t = 1.0;  // t = (-a^2)^n / n!
                for (int n = 1; n < 20; ++n) {
                    t *= -a * a / n;
                    sum += t * n * std::pow(z, n - 1) / (2 * n + 1);
                }
                return 2.0 * c * sum;
            }
            const double r = std::sqrt(z), x = a * r;
            return (c * std::exp(-x * x) / r - std::erf(x) / z) / r;
        };
        cheb_poly<NPOLY_G>(g, (double)v.rc * (double)v.rc, v.poly_g);
        v.two_over_rc2 = (float)(2.0 / ((double)v.rc * (double)v.rc));
    }
    // mixed lists: every cluster while that stays small (sparse atoms such as
    // ions form clusters with wide bounding boxes), else the estimate
    auto cap_mixed = [&](double r, double vol_cl, uint32_t n_i, uint32_t n_j) -> uint32_t {
        if ((uint64_t)n_i * n_j <= (1ull << 24)) return std::max(1u, n_j);
        return est(r, vol_cl, n_j);
    };
    v.cap_ws = (v.nw && v.na) ? cap_mixed(v.r_ws, acl_vol, v.nwclus_cap, v.naclus_cap) : 1;
    v.cap_ss = v.na ? cap_mixed(v.r_ss, acl_vol, v.naclus_cap, v.naclus_cap) : 1;
    v.ch_mix = cfg->pair_item_entries ? std::min(32u, cfg->pair_item_entries) : 8u;
    v.ws_item_cap = v.nwclus_cap * ((v.cap_ws + v.ch_mix - 1) / v.ch_mix);
    v.ss_item_cap = v.naclus_cap * ((v.cap_ss + v.ch_mix - 1) / v.ch_mix);

    // ---- allocations ----
    TRY(dev_alloc(h, &v.wpos, 4 * (size_t)v.nw_cap));
    TRY(dev_alloc(h, &v.wvel, 3 * (size_t)v.nw_cap));
    TRY(dev_alloc(h, &v.wacc, 3 * (size_t)v.nw_cap));
    TRY(dev_alloc(h, &v.wid, v.nw_cap, false));
    TRYC(cudaMemsetAsync(v.wid, 0xFF, v.nw_cap * sizeof(uint32_t), h->stream));
    TRY(dev_alloc(h, &v.wforce, 12 * (size_t)v.nw_cap));
    TRY(dev_alloc(h, &v.wref, v.nw_cap));
    TRY(dev_alloc(h, &v.wtmp, 10 * (size_t)v.nw_cap));
    TRY(dev_alloc(h, &v.wtmp_id, v.nw_cap));
    TRY(dev_alloc(h, &v.wrecip, 9 * (size_t)std::max(1u, v.nw)));
    TRY(dev_alloc(h, &v.wnew, v.nw_cap));
    TRY(dev_alloc(h, &v.wkey, v.nw_cap));
    TRY(dev_alloc(h, &v.wcol, v.nw_cap));
    TRY(dev_alloc(h, &v.bucket, v.nw_cap));
    TRY(dev_alloc(h, &v.apos, std::max(1u, v.na)));
    TRY(dev_alloc(h, &v.avel, std::max(1u, v.na)));
    TRY(dev_alloc(h, &v.aacc, std::max(1u, v.na)));
    TRY(dev_alloc(h, &v.amass, std::max(1u, v.na)));
    TRY(dev_alloc(h, &v.alj, std::max(1u, v.na)));
    TRY(dev_alloc(h, &v.aforce, 3 * (size_t)std::max(1u, v.na)));
    TRY(dev_alloc(h, &v.arecip, 3 * (size_t)std::max(1u, v.na)));
    TRY(dev_alloc(h, &v.aref, std::max(1u, v.na)));
    TRY(dev_alloc(h, &v.asparse, std::max(1u, v.na), false));
    TRY(upload(h, v.asparse, sparse_rank.data(), v.na));
    TRY(dev_alloc(h, &v.spos, v.na_cap));
    TRY(dev_alloc(h, &v.slj, v.na_cap));
    TRY(dev_alloc(h, &v.sidx, v.na_cap, false));
    TRYC(cudaMemsetAsync(v.sidx, 0xFF, v.na_cap * sizeof(uint32_t), h->stream));
    TRY(dev_alloc(h, &v.aslot, std::max(1u, v.na)));
    TRY(dev_alloc(h, &v.akey, std::max(1u, v.na)));
    TRY(dev_alloc(h, &v.acol, std::max(1u, v.na)));
    TRY(dev_alloc(h, &v.abucket, std::max(1u, v.na)));
    TRY(dev_alloc(h, &v.col_count, v.ncol + 1));
    TRY(dev_alloc(h, &v.col_off, v.ncol + 1));
    TRY(dev_alloc(h, &v.col_fill, v.ncol + 1));
    TRY(dev_alloc(h, &v.col_boff, v.ncol + 1));
    TRY(dev_alloc(h, &v.acol_count, v.ancol + 1));
    TRY(dev_alloc(h, &v.acol_off, v.ancol + 1));
    TRY(dev_alloc(h, &v.acol_fill, v.ancol + 1));
    TRY(dev_alloc(h, &v.acol_boff, v.ancol + 1));
    TRY(dev_alloc(h, &v.wbb_c, v.nwclus_cap));
    TRY(dev_alloc(h, &v.wbb_h, v.nwclus_cap));
    TRY(dev_alloc(h, &v.abb_c, v.naclus_cap));
    TRY(dev_alloc(h, &v.abb_h, v.naclus_cap));
    TRY(dev_alloc(h, &v.gbb_c, v.ngrp_cap));
    TRY(dev_alloc(h, &v.gbb_h, v.ngrp_cap));
    TRY(dev_alloc(h, &v.tile_n, v.ngrp_cap));
    TRY(dev_alloc(h, &v.tile_j, (size_t)v.ngrp_cap * v.cap_tile));
    TRY(dev_alloc(h, &v.grp_nrun, v.ngrp_cap));
    TRY(dev_alloc(h, &v.grp_nloc, v.ngrp_cap));
    TRY(dev_alloc(h, &v.grp_run, (size_t)v.ngrp_cap * v.cap_run));
    TRY(dev_alloc(h, &v.cand_loc, (size_t)v.ngrp_cap * v.cap_tile * WCL));
    TRY(dev_alloc(h, &v.wnb_n, v.nw_cap));
    TRY(dev_alloc(h, &v.wnb, (size_t)v.nw_cap * v.cap_nb));
    TRY(dev_alloc(h, &v.winb_n, v.nw_cap));
    TRY(dev_alloc(h, &v.winb, (size_t)v.nw_cap * v.cap_nb));
    TRY(dev_alloc(h, &v.wprune, v.nw_cap));
    TRY(dev_alloc(h, &v.grp_uslot, (size_t)v.ngrp_cap * v.cap_union));
    TRY(dev_alloc(h, &v.ws_n, v.nwclus_cap));
    TRY(dev_alloc(h, &v.ws_j, (size_t)v.nwclus_cap * v.cap_ws));
    TRY(dev_alloc(h, &v.ws_item, std::max(1u, v.ws_item_cap)));
    TRY(dev_alloc(h, &v.ss_item, std::max(1u, v.ss_item_cap)));
    TRY(dev_alloc(h, &v.ss_n, v.naclus_cap));
    TRY(dev_alloc(h, &v.ss_j, (size_t)v.naclus_cap * v.cap_ss));
    TRY(dev_alloc(h, &v.ss_mask, (size_t)v.naclus_cap * v.cap_ss));
    TRY(dev_alloc(h, &v.box, 1));
    TRY(dev_alloc(h, &v.sc, 1));
    TRY(dev_alloc(h, &v.partials, (size_t)NREGION * v.max_blocks * 4));

    // ---- state upload ----
    if (v.nw) {
        std::vector<float4> wp(4 * (size_t)v.nw_cap, make_float4(0, 0, 0, 0));
        std::vector<float4> wv(3 * (size_t)v.nw_cap, make_float4(0, 0, 0, 0));
        std::vector<uint32_t> wid(v.nw_cap, INVALID_ID);
        const float q[4] = {0.f, OPC_Q_H, OPC_Q_H, OPC_Q_EP};
        for (uint32_t i = 0; i < v.nw; ++i) {
            const float* p = d->water_pos + 9 * (size_t)i;
            float m[3];
            host_m_site(p, p + 3, p + 6, m);
            for (int s = 0; s < 3; ++s) wp[4 * i + s] = make_float4(p[3 * s], p[3 * s + 1], p[3 * s + 2], q[s]);
            wp[4 * i + 3] = make_float4(m[0], m[1], m[2], q[3]);
            const float* w = d->water_vel + 9 * (size_t)i;
            for (int s = 0; s < 3; ++s) wv[3 * i + s] = make_float4(w[3 * s], w[3 * s + 1], w[3 * s + 2], 0.f);
            wid[i] = i;
        }
        TRY(upload(h, v.wpos, wp.data(), wp.size()));
        TRY(upload(h, v.wvel, wv.data(), wv.size()));
        TRY(upload(h, v.wid, wid.data(), wid.size()));
        TRYC(cudaStreamSynchronize(h->stream));
    }
    double qsum2 = (double)v.nw * (2.0 * (double)OPC_Q_H * OPC_Q_H + (double)OPC_Q_EP * OPC_Q_EP);
    if (v.na) {
        std::vector<float4> ap(v.na), av(v.na);
        std::vector<float2> lj(v.na);
        for (uint32_t i = 0; i < v.na; ++i) {
            ap[i] = make_float4(d->atom_pos[3 * i], d->atom_pos[3 * i + 1], d->atom_pos[3 * i + 2], d->atom_q[i]);
            av[i] = make_float4(d->atom_vel[3 * i], d->atom_vel[3 * i + 1], d->atom_vel[3 * i + 2], 0.f);
            lj[i] = make_float2(d->atom_sigma[i], d->atom_eps[i]);
            qsum2 += (double)d->atom_q[i] * d->atom_q[i];
        }
        TRY(upload(h, v.apos, ap.data(), v.na));
        TRY(upload(h, v.avel, av.data(), v.na));
        TRY(upload(h, v.amass, d->atom_mass, v.na));
        TRY(upload(h, v.alj, lj.data(), v.na));
        if (d->atom_static) {
            TRY(dev_alloc(h, &v.astatic, v.na));
            TRY(upload(h, v.astatic, d->atom_static, v.na));
        }
        // exclusion CSR (1-2, 1-3 and 1-4 partners; 1-4 pairs are evaluated
        // separately, scaled)
        std::vector<std::vector<uint32_t>> rows(v.na);
        for (uint32_t k = 0; k < d->n_excl; ++k) {
            rows[d->excl[2 * k]].push_back(d->excl[2 * k + 1]);
            rows[d->excl[2 * k + 1]].push_back(d->excl[2 * k]);
        }
        for (uint32_t k = 0; k < d->n_pair14; ++k) {
            rows[d->pair14[2 * k]].push_back(d->pair14[2 * k + 1]);
            rows[d->pair14[2 * k + 1]].push_back(d->pair14[2 * k]);
        }
        std::vector<uint32_t> off(v.na + 1, 0), idx;
        for (uint32_t i = 0; i < v.na; ++i) {
            std::sort(rows[i].begin(), rows[i].end());
            rows[i].erase(std::unique(rows[i].begin(), rows[i].end()), rows[i].end());
            off[i + 1] = off[i] + (uint32_t)rows[i].size();
            idx.insert(idx.end(), rows[i].begin(), rows[i].end());
        }
        TRY(dev_alloc(h, &v.ex_off, v.na + 1));
        TRY(dev_alloc(h, &v.ex_idx, std::max<size_t>(1, idx.size())));
        TRY(upload(h, v.ex_off, off.data(), off.size()));
        TRY(upload(h, v.ex_idx, idx.data(), idx.size()));
        // 1-4 and exclusion lists
        v.n14 = d->n_pair14;
        if (v.n14) {
            std::vector<uint2> p(v.n14);
            std::vector<float4> par(v.n14);
            for (uint32_t k = 0; k < v.n14; ++k) {
                const uint32_t i = d->pair14[2 * k], j = d->pair14[2 * k + 1];
                p[k] = make_uint2(i, j);
                par[k] = make_float4(0.5f * (d->atom_sigma[i] + d->atom_sigma[j]),
                                     std::sqrt(d->atom_eps[i] * d->atom_eps[j]), d->atom_q[i] * d->atom_q[j], 0.f);
            }
            TRY(dev_alloc(h, &v.p14, v.n14));
            TRY(dev_alloc(h, &v.p14_par, v.n14));
            TRY(upload(h, v.p14, p.data(), v.n14));
            TRY(upload(h, v.p14_par, par.data(), v.n14));
        }
        v.nexcl = d->n_excl;
        if (v.nexcl) {
            std::vector<uint2> p(v.nexcl);
            std::vector<float> qq(v.nexcl);
            for (uint32_t k = 0; k < v.nexcl; ++k) {
                p[k] = make_uint2(d->excl[2 * k], d->excl[2 * k + 1]);
                qq[k] = d->atom_q[d->excl[2 * k]] * d->atom_q[d->excl[2 * k + 1]];
            }
            TRY(dev_alloc(h, &v.excl, v.nexcl));
            TRY(dev_alloc(h, &v.excl_qq, v.nexcl));
            TRY(upload(h, v.excl, p.data(), v.nexcl));
            TRY(upload(h, v.excl_qq, qq.data(), v.nexcl));
        }
        // bonded terms
        v.nbond = d->n_bonds;
        if (v.nbond) {
            std::vector<uint2> p(v.nbond);
            std::vector<float2> par(v.nbond);
            for (uint32_t k = 0; k < v.nbond; ++k) {
                p[k] = make_uint2(d->bonds[2 * k], d->bonds[2 * k + 1]);
                par[k] = make_float2(d->bond_k[k], d->bond_r0[k]);
            }
            TRY(dev_alloc(h, &v.bond, v.nbond));
            TRY(dev_alloc(h, &v.bond_par, v.nbond));
            TRY(upload(h, v.bond, p.data(), v.nbond));
            TRY(upload(h, v.bond_par, par.data(), v.nbond));
        }
        v.nangle = d->n_angles;
        if (v.nangle) {
            std::vector<uint4> p(v.nangle);
            std::vector<float2> par(v.nangle);
            for (uint32_t k = 0; k < v.nangle; ++k) {
                p[k] = make_uint4(d->angles[3 * k], d->angles[3 * k + 1], d->angles[3 * k + 2], 0);
                par[k] = make_float2(d->angle_k[k], d->angle_theta0[k]);
            }
            TRY(dev_alloc(h, &v.angle, v.nangle));
            TRY(dev_alloc(h, &v.angle_par, v.nangle));
            TRY(upload(h, v.angle, p.data(), v.nangle));
            TRY(upload(h, v.angle_par, par.data(), v.nangle));
        }
        v.ndih = d->n_dihedrals;
        if (v.ndih) {
            std::vector<uint4> p(v.ndih);
            std::vector<float4> par(v.ndih);
            for (uint32_t k = 0; k < v.ndih; ++k) {
                p[k] = make_uint4(d->dihedrals[4 * k], d->dihedrals[4 * k + 1], d->dihedrals[4 * k + 2],
                                  d->dihedrals[4 * k + 3]);
                par[k] = make_float4(d->dihedral_k[k], d->dihedral_n[k], d->dihedral_phase[k], 0.f);
            }
            TRY(dev_alloc(h, &v.dih, v.ndih));
            TRY(dev_alloc(h, &v.dih_par, v.ndih));
            TRY(upload(h, v.dih, p.data(), v.ndih));
            TRY(upload(h, v.dih_par, par.data(), v.ndih));
        }
    }
    v.e_self = -(double)v.alpha / std::sqrt(M_PI) * qsum2;
    BoxDev bx{};
    for (int k = 0; k < 3; ++k) {
        bx.lo[k] = cfg->box_lo[k];
        bx.ext[k] = ext[k];
        bx.inv_ext[k] = (float)(1.0 / (double)ext[k]);
    }
    TRY(upload(h, v.box, &bx, 1));
    TRY(dyn::pme_init(v, &h->plan_f, &h->plan_b, h->stream));
    dyn::pme_bricks(v, cfg->spme_brick_cap);
    TRY(dev_alloc(h, &v.brick_n, v.n_bricks));
    TRY(dev_alloc(h, &v.brick_ovf, v.n_bricks));
    TRY(dev_alloc(h, &v.brick_tile, (size_t)v.n_bricks * 1331, false));  // 11^3 points per brick
    TRY(dev_alloc(h, &v.brick_site, (size_t)v.n_bricks * v.brick_cap, false));
    TRY(dev_alloc(h, &v.brick_sid, (size_t)v.n_bricks * v.brick_cap, false));
    TRY(dev_alloc(h, &v.ovf_site, v.n_sites_max, false));
    TRY(dev_alloc(h, &v.ovf_sid, v.n_sites_max, false));
    TRY(dev_alloc(h, &v.wsite_f, 9 * (size_t)v.nw));
    v.plan_f = (int)h->plan_f;
    v.plan_b = (int)h->plan_b;
    {
        const size_t ng = (size_t)v.K[0] * v.K[1] * v.K[2], nc = (size_t)v.K[0] * v.K[1] * (v.K[2] / 2 + 1);
        size_t wf = 0, wb = 0;
        cufftGetSize(h->plan_f, &wf);
        cufftGetSize(h->plan_b, &wb);
        h->bytes += ng * (sizeof(long long) + sizeof(float)) + nc * sizeof(float2) +
                    (v.K[0] + v.K[1] + v.K[2]) * sizeof(float) + wf + wb;
    }
    {
        // units in atom order; an H goes with its heavy atom
        std::vector<uint32_t> off(1, 0), idx;
        std::vector<float> r02;
        std::vector<uint8_t> is_h(d->n_atoms, 0);
        for (uint32_t a = 0; a < d->n_atoms; ++a)
            for (uint32_t hy : unit_h[a]) is_h[hy] = 1;
        for (uint32_t a = 0; a < d->n_atoms; ++a) {
            if (is_h[a]) continue;
            idx.push_back(a);
            r02.push_back(0.f);
            for (uint32_t hy : unit_h[a]) {
                idx.push_back(hy);
                r02.push_back(h_r02[hy]);
            }
            off.push_back((uint32_t)idx.size());
        }
        v.nunit = (uint32_t)off.size() - 1;
        v.ncons = d->n_constraints;
        v.lincs_order = cfg->lincs_order ? cfg->lincs_order : 4u;
        v.lincs_iter = cfg->lincs_iter ? cfg->lincs_iter : 1u;
        TRY(dev_alloc(h, &v.unit_off, off.size()));
        TRY(dev_alloc(h, &v.unit_idx, std::max<size_t>(1, idx.size())));
        TRY(dev_alloc(h, &v.unit_r02, std::max<size_t>(1, r02.size())));
        TRY(upload(h, v.unit_off, off.data(), off.size()));
        TRY(upload(h, v.unit_idx, idx.data(), idx.size()));
        TRY(upload(h, v.unit_r02, r02.data(), r02.size()));
        TRYC(cudaStreamSynchronize(h->stream));
    }
    h->allocs.push_back(v.qgrid_fix); h->allocs.push_back(v.qgrid); h->allocs.push_back(v.cgrid);
    for (int a = 0; a < 3; ++a) h->allocs.push_back(v.bmod[a]);
    set_block_counts(v);
    if (v.nw) TRY(dyn::pair_ww_setup(v));
    TRYC(cudaStreamSynchronize(h->stream));
    // prime: first list build and forces -> accelerations
    enqueue_forces(h, true);
    TRYC(cudaGetLastError());
    TRY(read_scalars(h));
#undef TRY
#undef TRYC
    *out = h;
    return DYN_OK;
}

// Launches a long dyn_sys_step call keeps in flight before it waits.
constexpr uint32_t STEP_WINDOW = 512;

extern "C" int dyn_sys_step(dyn_sys_t h, uint32_t n_steps, float dt) {
    DYN_CHECK(h, DYN_ERR_INVALID, "dyn_sys_step: NULL handle");
    DYN_CHECK(dt > 0.f && std::isfinite(dt), DYN_ERR_INVALID, "dyn_sys_step: dt must be > 0");
    const uint32_t e_int = std::max(1u, h->cfg.energy_interval);
    for (uint32_t i = 0; i < n_steps; ++i) {
        const uint64_t s = h->host_step;
        const bool spme = (s % h->v.spme_interval) == 0;
        const bool energy = ((s + 1) % e_int) == 0;
        const int g = (spme ? 1 : 0) | (energy ? 2 : 0);
        if (!h->graph[g] || h->graph_dt[g] != dt) {
            if (h->graph[g]) { cudaGraphExecDestroy(h->graph[g]); h->graph[g] = nullptr; }
            cudaGraph_t graph = nullptr;
            const int rc = capture_step(h, dt, spme, energy, &graph);
            if (rc != DYN_OK) return rc;
            cudaError_t e = cudaGraphInstantiate(&h->graph[g], graph, 0);
            cudaGraphDestroy(graph);
            if (e != cudaSuccess) return dyn::cuda_fail(e, "cudaGraphInstantiate");
            h->graph_dt[g] = dt;
        }
        DYN_CUDA(cudaGraphLaunch(h->graph[g], h->stream));
        h->host_step += 1;
        // at most about 2 x STEP_WINDOW steps queued at a time: every
        // STEP_WINDOW launches wait for the mark set STEP_WINDOW launches ago
        if ((i + 1) % STEP_WINDOW == 0 && i + 1 < n_steps) {
            if (!h->window_ev) DYN_CUDA(cudaEventCreateWithFlags(&h->window_ev, cudaEventDisableTiming));
            if (h->window_armed) DYN_CUDA(cudaEventSynchronize(h->window_ev));
            DYN_CUDA(cudaEventRecord(h->window_ev, h->stream));
            h->window_armed = true;
        }
    }
    h->window_armed = false;
    return DYN_OK;
}

extern "C" int dyn_sys_sync(dyn_sys_t h) {
    DYN_CHECK(h, DYN_ERR_INVALID, "dyn_sys_sync: NULL handle");
    DYN_CUDA(cudaStreamSynchronize(h->stream));
    return read_scalars(h);
}

extern "C" int dyn_sys_get_energies(dyn_sys_t h, dyn_energies_t* out) {
    DYN_CHECK(h && out, DYN_ERR_INVALID, "dyn_sys_get_energies: NULL argument");
    int rc = read_scalars(h);
    BoxDev bx;
    DYN_CUDA(cudaMemcpy(&bx, h->v.box, sizeof(BoxDev), cudaMemcpyDeviceToHost));
    fill_energies(h, out);
    for (int k = 0; k < 3; ++k) out->box[k] = bx.ext[k];
    return rc;
}

extern "C" int dyn_sys_forces(dyn_sys_t h, double* f_atoms, double* f_water, dyn_energies_t* energies) {
    DYN_CHECK(h, DYN_ERR_INVALID, "dyn_sys_forces: NULL handle");
    const SysView& v = h->v;
    enqueue_forces(h, false);
    DYN_CUDA(cudaGetLastError());
    int rc = read_scalars(h);
    if (rc) return rc;
    if (f_atoms && v.na) {
        std::vector<long long> a(3 * (size_t)v.na), r(3 * (size_t)v.na);
        DYN_CUDA(cudaMemcpy(a.data(), v.aforce, a.size() * 8, cudaMemcpyDeviceToHost));
        DYN_CUDA(cudaMemcpy(r.data(), v.arecip, r.size() * 8, cudaMemcpyDeviceToHost));
        for (size_t k = 0; k < a.size(); ++k) f_atoms[k] = (double)(a[k] + r[k]) * DYN_FIX_INV;
    }
    if (f_water && v.nw) {
        std::vector<long long> f(12 * (size_t)v.nw_cap), r(9 * (size_t)v.nw);
        std::vector<uint32_t> wid(v.nw_cap);
        DYN_CUDA(cudaMemcpy(f.data(), v.wforce, f.size() * 8, cudaMemcpyDeviceToHost));
        DYN_CUDA(cudaMemcpy(r.data(), v.wrecip, r.size() * 8, cudaMemcpyDeviceToHost));
        DYN_CUDA(cudaMemcpy(wid.data(), v.wid, wid.size() * 4, cudaMemcpyDeviceToHost));
        for (uint32_t s = 0; s < v.nw_cap; ++s) {
            const uint32_t id = wid[s];
            if (id == INVALID_ID) continue;
            // sites O, H0, H1, M; the cache holds H0, H1, M
            for (int c = 0; c < 12; ++c) {
                long long x = f[12 * (size_t)s + c];
                if (c >= 3) x += r[9 * (size_t)id + (c - 3)];
                f_water[12 * (size_t)id + c] = (double)x * DYN_FIX_INV;
            }
        }
    }
    if (energies) {
        BoxDev bx;
        DYN_CUDA(cudaMemcpy(&bx, v.box, sizeof(BoxDev), cudaMemcpyDeviceToHost));
        fill_energies(h, energies);
        for (int k = 0; k < 3; ++k) energies->box[k] = bx.ext[k];
    }
    return DYN_OK;
}

extern "C" int dyn_sys_get_state(dyn_sys_t h, float* atom_pos, float* atom_vel, float* water_pos,
                                 float* water_vel, float* water_m) {
    DYN_CHECK(h, DYN_ERR_INVALID, "dyn_sys_get_state: NULL handle");
    const SysView& v = h->v;
    DYN_CUDA(cudaStreamSynchronize(h->stream));
    if (v.na && (atom_pos || atom_vel)) {
        std::vector<float4> p(v.na), w(v.na);
        DYN_CUDA(cudaMemcpy(p.data(), v.apos, v.na * sizeof(float4), cudaMemcpyDeviceToHost));
        DYN_CUDA(cudaMemcpy(w.data(), v.avel, v.na * sizeof(float4), cudaMemcpyDeviceToHost));
        for (uint32_t i = 0; i < v.na; ++i) {
            if (atom_pos) { atom_pos[3 * i] = p[i].x; atom_pos[3 * i + 1] = p[i].y; atom_pos[3 * i + 2] = p[i].z; }
            if (atom_vel) { atom_vel[3 * i] = w[i].x; atom_vel[3 * i + 1] = w[i].y; atom_vel[3 * i + 2] = w[i].z; }
        }
    }
    if (v.nw && (water_pos || water_vel || water_m)) {
        std::vector<float4> p(4 * (size_t)v.nw_cap), w(3 * (size_t)v.nw_cap);
        std::vector<uint32_t> wid(v.nw_cap);
        DYN_CUDA(cudaMemcpy(p.data(), v.wpos, p.size() * sizeof(float4), cudaMemcpyDeviceToHost));
        DYN_CUDA(cudaMemcpy(w.data(), v.wvel, w.size() * sizeof(float4), cudaMemcpyDeviceToHost));
        DYN_CUDA(cudaMemcpy(wid.data(), v.wid, wid.size() * 4, cudaMemcpyDeviceToHost));
        for (uint32_t s = 0; s < v.nw_cap; ++s) {
            const uint32_t id = wid[s];
            if (id == INVALID_ID) continue;
            for (int k = 0; k < 3; ++k) {
                const float4 a = p[4 * (size_t)s + k], b = w[3 * (size_t)s + k];
                if (water_pos) { water_pos[9 * (size_t)id + 3 * k] = a.x; water_pos[9 * (size_t)id + 3 * k + 1] = a.y; water_pos[9 * (size_t)id + 3 * k + 2] = a.z; }
                if (water_vel) { water_vel[9 * (size_t)id + 3 * k] = b.x; water_vel[9 * (size_t)id + 3 * k + 1] = b.y; water_vel[9 * (size_t)id + 3 * k + 2] = b.z; }
            }
            if (water_m) {
                const float4 m = p[4 * (size_t)s + 3];
                water_m[3 * (size_t)id] = m.x; water_m[3 * (size_t)id + 1] = m.y; water_m[3 * (size_t)id + 2] = m.z;
            }
        }
    }
    return DYN_OK;
}

extern "C" int dyn_sys_set_state(dyn_sys_t h, const float* atom_pos, const float* atom_vel,
                                 const float* water_pos, const float* water_vel) {
    DYN_CHECK(h, DYN_ERR_INVALID, "dyn_sys_set_state: NULL handle");
    SysView& v = h->v;
    DYN_CUDA(cudaStreamSynchronize(h->stream));
    if (v.na && (atom_pos || atom_vel)) {
        std::vector<float4> p(v.na), w(v.na);
        DYN_CUDA(cudaMemcpy(p.data(), v.apos, v.na * sizeof(float4), cudaMemcpyDeviceToHost));
        DYN_CUDA(cudaMemcpy(w.data(), v.avel, v.na * sizeof(float4), cudaMemcpyDeviceToHost));
        for (uint32_t i = 0; i < v.na; ++i) {
            if (atom_pos) { p[i].x = atom_pos[3 * i]; p[i].y = atom_pos[3 * i + 1]; p[i].z = atom_pos[3 * i + 2]; }
            if (atom_vel) { w[i].x = atom_vel[3 * i]; w[i].y = atom_vel[3 * i + 1]; w[i].z = atom_vel[3 * i + 2]; }
        }
        DYN_CUDA(cudaMemcpy(v.apos, p.data(), v.na * sizeof(float4), cudaMemcpyHostToDevice));
        DYN_CUDA(cudaMemcpy(v.avel, w.data(), v.na * sizeof(float4), cudaMemcpyHostToDevice));
    }
    if (v.nw && (water_pos || water_vel)) {
        std::vector<float4> p(4 * (size_t)v.nw_cap), w(3 * (size_t)v.nw_cap);
        std::vector<uint32_t> wid(v.nw_cap);
        DYN_CUDA(cudaMemcpy(p.data(), v.wpos, p.size() * sizeof(float4), cudaMemcpyDeviceToHost));
        DYN_CUDA(cudaMemcpy(w.data(), v.wvel, w.size() * sizeof(float4), cudaMemcpyDeviceToHost));
        DYN_CUDA(cudaMemcpy(wid.data(), v.wid, wid.size() * 4, cudaMemcpyDeviceToHost));
        const float q[4] = {0.f, OPC_Q_H, OPC_Q_H, OPC_Q_EP};
        for (uint32_t s = 0; s < v.nw_cap; ++s) {
            const uint32_t id = wid[s];
            if (id == INVALID_ID) continue;
            if (water_pos) {
                const float* x = water_pos + 9 * (size_t)id;
                float m[3];
                host_m_site(x, x + 3, x + 6, m);
                for (int k = 0; k < 3; ++k) p[4 * (size_t)s + k] = make_float4(x[3 * k], x[3 * k + 1], x[3 * k + 2], q[k]);
                p[4 * (size_t)s + 3] = make_float4(m[0], m[1], m[2], q[3]);
            }
            if (water_vel) {
                const float* x = water_vel + 9 * (size_t)id;
                for (int k = 0; k < 3; ++k) w[3 * (size_t)s + k] = make_float4(x[3 * k], x[3 * k + 1], x[3 * k + 2], 0.f);
            }
        }
        DYN_CUDA(cudaMemcpy(v.wpos, p.data(), p.size() * sizeof(float4), cudaMemcpyHostToDevice));
        DYN_CUDA(cudaMemcpy(v.wvel, w.data(), w.size() * sizeof(float4), cudaMemcpyHostToDevice));
    }
    // new coordinates: rebuild lists and re-prime forces/accelerations
    enqueue_forces(h, true);
    DYN_CUDA(cudaGetLastError());
    return read_scalars(h);
}

// Home-order staging for the host-step path: water (pos, vel) as [nw*9]
// floats each; kernels scatter into / gather from the cluster-ordered slots.
__global__ void k_stage_in(SysView v, const float* __restrict__ wp, const float* __restrict__ wv) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < v.nw_cap; s += gridDim.x * blockDim.x)
        water_in(v, s, wp, wv);
}

__global__ void k_stage_out(SysView v, float* __restrict__ wp, float* __restrict__ wv) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < v.nw_cap; s += gridDim.x * blockDim.x)
        water_out(v, s, wp, wv);
}

__global__ void k_atoms_in(SysView v, const float* __restrict__ ap, const float* __restrict__ av) {
    for (uint32_t a = blockIdx.x * blockDim.x + threadIdx.x; a < v.na; a += gridDim.x * blockDim.x)
        atom_in(v, a, ap, av);
}

__global__ void k_atoms_out(SysView v, float* __restrict__ ap, float* __restrict__ av) {
    for (uint32_t a = blockIdx.x * blockDim.x + threadIdx.x; a < v.na; a += gridDim.x * blockDim.x)
        atom_out(v, a, ap, av);
}

namespace {

// The staging area of dyn_sys_step_host: [2 * (na*3 + nw*9)] floats,
// owned by the handle (freed with its other allocations).
int ensure_stage(dyn_sys_s* h) {
    const size_t need = 2 * (3 * (size_t)h->v.na) + 2 * (9 * (size_t)h->v.nw);
    if (h->host_stage && h->host_stage_n >= need) return DYN_OK;
    float* d = nullptr;
    DYN_CUDA(cudaMalloc(&d, std::max<size_t>(need, 1) * sizeof(float)));
    h->allocs.push_back(d);  // a smaller earlier area stays in allocs until destroy
    h->host_stage = d;
    h->host_stage_n = need;
    return DYN_OK;
}

}  // namespace
namespace dyn {
int count_graph_kernels(cudaGraph_t g, uint32_t* n) {
    size_t cnt = 0;
    DYN_CUDA(cudaGraphGetNodes(g, nullptr, &cnt));
    std::vector<cudaGraphNode_t> nodes(cnt);
    DYN_CUDA(cudaGraphGetNodes(g, nodes.data(), &cnt));
    uint32_t k = 0;
    for (auto nd : nodes) {
        cudaGraphNodeType t;
        DYN_CUDA(cudaGraphNodeGetType(nd, &t));
        if (t == cudaGraphNodeTypeKernel) ++k;
    }
    *n = k;
    return DYN_OK;
}
}  // namespace dyn
namespace {

}  // namespace

extern "C" int dyn_sys_step_host(dyn_sys_t h, uint32_t n_steps, float dt, const float* atom_pos_in,
                                 const float* atom_vel_in, const float* water_pos_in,
                                 const float* water_vel_in, float* atom_pos_out, float* atom_vel_out,
                                 float* water_pos_out, float* water_vel_out, dyn_energies_t* energies) {
    DYN_CHECK(h, DYN_ERR_INVALID, "dyn_sys_step_host: NULL handle");
    SysView& v = h->v;
    int rc = ensure_stage(h);
    if (rc) return rc;
    float* d_ap = h->host_stage;
    float* d_av = d_ap + 3 * (size_t)v.na;
    float* d_wp = d_av + 3 * (size_t)v.na;
    float* d_wv = d_wp + 9 * (size_t)v.nw;
    cudaStream_t st = h->stream;
    const int nbw = std::max(1u, std::min(v.max_blocks, (v.nw_cap + 255) / 256));
    const int nba = std::max(1u, std::min(v.max_blocks, (v.na + 255) / 256));
    if (v.na && (atom_pos_in || atom_vel_in)) {
        if (atom_pos_in) DYN_CUDA(cudaMemcpyAsync(d_ap, atom_pos_in, 12 * (size_t)v.na, cudaMemcpyHostToDevice, st));
        if (atom_vel_in) DYN_CUDA(cudaMemcpyAsync(d_av, atom_vel_in, 12 * (size_t)v.na, cudaMemcpyHostToDevice, st));
        k_atoms_in<<<nba, 256, 0, st>>>(v, atom_pos_in ? d_ap : nullptr, atom_vel_in ? d_av : nullptr);
    }
    if (v.nw && (water_pos_in || water_vel_in)) {
        if (water_pos_in) DYN_CUDA(cudaMemcpyAsync(d_wp, water_pos_in, 36 * (size_t)v.nw, cudaMemcpyHostToDevice, st));
        if (water_vel_in) DYN_CUDA(cudaMemcpyAsync(d_wv, water_vel_in, 36 * (size_t)v.nw, cudaMemcpyHostToDevice, st));
        k_stage_in<<<nbw, 256, 0, st>>>(v, water_pos_in ? d_wp : nullptr, water_vel_in ? d_wv : nullptr);
    }
    DYN_CUDA(cudaGetLastError());
    rc = dyn_sys_step(h, n_steps, dt);
    if (rc) return rc;
    if (v.na && (atom_pos_out || atom_vel_out)) {
        k_atoms_out<<<nba, 256, 0, st>>>(v, d_ap, d_av);
        if (atom_pos_out) DYN_CUDA(cudaMemcpyAsync(atom_pos_out, d_ap, 12 * (size_t)v.na, cudaMemcpyDeviceToHost, st));
        if (atom_vel_out) DYN_CUDA(cudaMemcpyAsync(atom_vel_out, d_av, 12 * (size_t)v.na, cudaMemcpyDeviceToHost, st));
    }
    if (v.nw && (water_pos_out || water_vel_out)) {
        k_stage_out<<<nbw, 256, 0, st>>>(v, d_wp, d_wv);
        if (water_pos_out) DYN_CUDA(cudaMemcpyAsync(water_pos_out, d_wp, 36 * (size_t)v.nw, cudaMemcpyDeviceToHost, st));
        if (water_vel_out) DYN_CUDA(cudaMemcpyAsync(water_vel_out, d_wv, 36 * (size_t)v.nw, cudaMemcpyDeviceToHost, st));
    }
    DYN_CUDA(cudaGetLastError());
    DYN_CUDA(cudaMemcpyAsync(h->h_sc, v.sc, sizeof(Scalars), cudaMemcpyDeviceToHost, st));
    DYN_CUDA(cudaStreamSynchronize(st));
    if (energies) {
        fill_energies(h, energies);
    }
    if (h->h_sc->nonfinite) return dyn::fail(DYN_ERR_NONFINITE, "non-finite coordinates or forces");
    if (h->h_sc->overflow) return dyn::fail(DYN_ERR_UNSUPPORTED, "cluster list capacity exceeded");
    return DYN_OK;
}

extern "C" int dyn_sys_stage_times(dyn_sys_t h, uint32_t n_steps, float dt, double* ms) {
    DYN_CHECK(h && ms, DYN_ERR_INVALID, "dyn_sys_stage_times: NULL argument");
    DYN_CHECK(dt > 0.f, DYN_ERR_INVALID, "dyn_sys_stage_times: dt must be > 0");
    const SysView& v = h->v;
    cudaStream_t st = h->stream;
    const Target T{&v, nullptr, st};
    // events: 0..6 bound the six stages; 7, 8 split the pair stage,
    // 9..11 the SPME stage
    constexpr int NE = 12;
    cudaEvent_t ev[NE];
    for (int i = 0; i < NE; ++i) DYN_CUDA(cudaEventCreate(&ev[i]));
    double acc[DYN_STAGES] = {};
    uint32_t n_spme = 0;
    const uint32_t e_int = std::max(1u, h->cfg.energy_interval);
    const bool alch = v.alch_on != 0u;
    auto el = [&](int a, int b) {
        float t = 0.f;
        cudaEventElapsedTime(&t, ev[a], ev[b]);
        return (double)t;
    };
    for (uint32_t i = 0; i < n_steps; ++i) {
        const uint64_t s = h->host_step;
        const bool spme = (s % v.spme_interval) == 0;
        const bool energy = ((s + 1) % e_int) == 0;
        cudaEventRecord(ev[0], st);
        dyn::launch_first_half(T, dt);
        cudaEventRecord(ev[1], st);
        dyn::launch_displacement_check(T);
        dyn::launch_rebuild(T, false);
        dyn::launch_prune(T, false);
        cudaEventRecord(ev[2], st);
        dyn::launch_gather_atoms(T);
        dyn::launch_pairs_ww(T, energy);
        cudaEventRecord(ev[7], st);
        dyn::launch_pairs_ws(T, energy);
        cudaEventRecord(ev[8], st);
        dyn::launch_pairs_atoms(T, energy);
        cudaEventRecord(ev[3], st);
        dyn::launch_pair14(T, energy);
        dyn::launch_bonded(T, energy);
        cudaEventRecord(ev[4], st);
        if (spme) {
            if (alch) {
                dyn::launch_pme(T);
            } else {
                dyn::launch_pme_spread(T, 0);
                cudaEventRecord(ev[9], st);
                dyn::launch_pme_transform(T, 0);
                cudaEventRecord(ev[10], st);
                dyn::launch_pme_gather(T, 0);
                cudaEventRecord(ev[11], st);
            }
            dyn::launch_corrections(T);
        }
        cudaEventRecord(ev[5], st);
        dyn::launch_second_half(T, dt);
        dyn::launch_finalize(T, dt, energy, true);
        dyn::launch_periodic(T);
        cudaEventRecord(ev[6], st);
        DYN_CUDA(cudaGetLastError());
        DYN_CUDA(cudaEventSynchronize(ev[6]));
        for (int k = 0; k < 6; ++k) acc[k] += el(k, k + 1);
        acc[6] += el(2, 7);   // includes the force zeroing and the atoms' cluster-order copy before it
        acc[7] += el(7, 8);
        acc[8] += el(8, 3);
        if (spme && !alch) {
            acc[9] += el(4, 9);
            acc[10] += el(9, 10);
            acc[11] += el(10, 11);
            acc[12] += el(11, 5);
        }
        n_spme += spme ? 1u : 0u;
        h->host_step += 1;
    }
    for (int i = 0; i < NE; ++i) cudaEventDestroy(ev[i]);
    for (int k = 0; k < DYN_STAGES; ++k) ms[k] = n_steps ? acc[k] / n_steps : 0.0;
    for (int k : {4, 9, 10, 11, 12}) ms[k] = n_spme ? acc[k] / n_spme : 0.0;
    return read_scalars(h);
}

// Kernel counts of a step's three parts, each captured on its own into a
// plain graph that is only inspected, never launched: the fixed part (with
// or without SPME; cuFFT's kernels excluded), the list rebuild and the
// periodic tasks.
int count_step_kernels(dyn_sys_s* h, bool spme, uint32_t* fixed, uint32_t* rebuild, uint32_t* periodic) {
    const SysView& v = h->v;
    cudaStream_t st = h->stream;
    const Target T{&v, nullptr, st};
    DYN_CUDA(cudaStreamSynchronize(st));
    auto count = [&](auto&& enqueue, uint32_t* n) -> int {
        cudaGraph_t g = nullptr;
        DYN_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        enqueue();
        const cudaError_t e = cudaStreamEndCapture(st, &g);
        if (e != cudaSuccess) return dyn::cuda_fail(e, "cudaStreamEndCapture");
        const int rc = count_graph_kernels(g, n);
        cudaGraphDestroy(g);
        return rc;
    };
    int rc = DYN_OK;
    if (fixed) {
        uint32_t total = 0, fft = 0;
        rc = count([&] {
            dyn::launch_first_half(T, 0.002f);
            dyn::launch_displacement_check(T);
            dyn::launch_gather_atoms(T);
            dyn::launch_pairs(T, true);
            dyn::launch_pair14(T, true);
            dyn::launch_bonded(T, true);
            if (spme) {
                dyn::launch_pme(T);
                dyn::launch_corrections(T);
            }
            dyn::launch_second_half(T, 0.002f);
            dyn::launch_finalize(T, 0.002f, true, true);
        }, &total);
        if (rc) return rc;
        if (spme) {
            rc = count([&] {
                cufftSetStream(h->plan_f, st);
                cufftSetStream(h->plan_b, st);
                cufftExecR2C(h->plan_f, h->v.qgrid, (cufftComplex*)h->v.cgrid);
                cufftExecC2R(h->plan_b, (cufftComplex*)h->v.cgrid, h->v.qgrid);
            }, &fft);
            if (rc) return rc;
        }
        *fixed = total - fft;
    }
    // a rebuild is always followed by a prune of the water-water lists (which
    // also runs alone, 2 kernels, when only the prune buffer is used up)
    if (rebuild && (rc = count([&] {
            dyn::launch_rebuild(T, false);
            dyn::launch_prune(T, false);
        }, rebuild))) return rc;
    if (periodic && (rc = count([&] { dyn::launch_periodic(T); }, periodic))) return rc;
    return DYN_OK;
}

extern "C" int dyn_sys_launches_per_step(dyn_sys_t h, int spme, uint32_t* out) {
    DYN_CHECK(h && out, DYN_ERR_INVALID, "dyn_sys_launches_per_step: NULL argument");
    return count_step_kernels(h, spme != 0, out, nullptr, nullptr);
}

extern "C" int dyn_sys_launches_conditional(dyn_sys_t h, uint32_t* rebuild, uint32_t* periodic) {
    DYN_CHECK(h && rebuild && periodic, DYN_ERR_INVALID, "dyn_sys_launches_conditional: NULL argument");
    return count_step_kernels(h, false, nullptr, rebuild, periodic);
}

extern "C" int dyn_sys_memory(dyn_sys_t h, uint64_t* bytes) {
    DYN_CHECK(h && bytes, DYN_ERR_INVALID, "dyn_sys_memory: NULL argument");
    *bytes = h->bytes + h->snap_bytes;
    return DYN_OK;
}

#define TRYC_ALLOC(ptr_, n_)                                       \
    do {                                                           \
        const int rc_a = dev_alloc(h, &(ptr_), (n_), true);        \
        if (rc_a != DYN_OK) return rc_a;                           \
    } while (0)

extern "C" int dyn_sys_set_lambda(dyn_sys_t h, float lambda) {
    DYN_CHECK(h, DYN_ERR_INVALID, "dyn_sys_set_lambda: NULL handle");
    DYN_CHECK(std::isfinite(lambda), DYN_ERR_INVALID, "dyn_sys_set_lambda: lambda not finite");
    DYN_CHECK(h->v.alch_on, DYN_ERR_INVALID, "dyn_sys_set_lambda: no alchemical molecule");
    DYN_CHECK(!h->batch_member, DYN_ERR_UNSUPPORTED, "dyn_sys_set_lambda: not for a batch member");
    DYN_CUDA(cudaStreamSynchronize(h->stream));
    for (int g = 0; g < 4; ++g)
        if (h->graph[g]) { cudaGraphExecDestroy(h->graph[g]); h->graph[g] = nullptr; }
    set_alch_schedule(h->v, lambda);
    h->cfg.alch_lambda = lambda;
    // the cached reciprocal forces belong to the old lambda
    return dyn::evaluate_forces(h);
}

extern "C" int dyn_sys_set_static(dyn_sys_t h, const uint8_t* atom_static, uint32_t thermo_dof) {
    DYN_CHECK(h, DYN_ERR_INVALID, "dyn_sys_set_static: NULL handle");
    DYN_CHECK(!h->batch_member, DYN_ERR_UNSUPPORTED, "dyn_sys_set_static: not for a batch member");
    SysView& v = h->v;
    DYN_CUDA(cudaStreamSynchronize(h->stream));
    if (v.na) {
        if (!v.astatic) {
            // the step graphs carry the view: capture them again
            for (int g = 0; g < 4; ++g)
                if (h->graph[g]) { cudaGraphExecDestroy(h->graph[g]); h->graph[g] = nullptr; }
            TRYC_ALLOC(v.astatic, v.na);
        }
        if (atom_static)
            DYN_CUDA(cudaMemcpyAsync(v.astatic, atom_static, v.na, cudaMemcpyHostToDevice, h->stream));
        else
            DYN_CUDA(cudaMemsetAsync(v.astatic, 0, v.na, h->stream));
    }
    if (thermo_dof && thermo_dof != v.thermo_dof) {
        for (int g = 0; g < 4; ++g)
            if (h->graph[g]) { cudaGraphExecDestroy(h->graph[g]); h->graph[g] = nullptr; }
        v.thermo_dof = thermo_dof;
        h->cfg.thermo_dof = thermo_dof;
    }
    // the cluster-pair masks leave out pairs of two static atoms
    const unsigned int one = 1u;
    DYN_CUDA(cudaMemcpyAsync(&v.sc->need_rebuild, &one, sizeof(one), cudaMemcpyHostToDevice, h->stream));
    DYN_CUDA(cudaStreamSynchronize(h->stream));
    return DYN_OK;
}

extern "C" int dyn_sys_snapshots(dyn_sys_t h, uint32_t ratio, uint32_t capacity, uint32_t fields) {
    DYN_CHECK(h, DYN_ERR_INVALID, "dyn_sys_snapshots: NULL handle");
    DYN_CHECK(!h->batch_member, DYN_ERR_UNSUPPORTED, "dyn_sys_snapshots: not for a batch member");
    DYN_CHECK(ratio == 0 || capacity > 0, DYN_ERR_INVALID, "dyn_sys_snapshots: capacity must be > 0");
    DYN_CHECK((fields & ~(DYN_SNAP_VELOCITIES | DYN_SNAP_FORCES)) == 0, DYN_ERR_INVALID,
              "dyn_sys_snapshots: unknown field bits");
    SysView& v = h->v;
    DYN_CUDA(cudaStreamSynchronize(h->stream));
    // the step graphs carry the view: capture them again with the new ring
    for (int g = 0; g < 4; ++g)
        if (h->graph[g]) { cudaGraphExecDestroy(h->graph[g]); h->graph[g] = nullptr; }
    if (h->snap_mem) { DYN_CUDA(cudaFree(h->snap_mem)); h->snap_mem = nullptr; }
    h->snap_bytes = 0;
    v.snap_ratio = 0; v.snap_cap = 0;
    v.snap_pos = v.snap_vel = v.snap_force = nullptr;
    v.snap_frames = nullptr;
    h->snap_read = 0;
    DYN_CUDA(cudaMemsetAsync(&v.sc->snap_count, 0, sizeof(v.sc->snap_count), h->stream));
    if (ratio == 0) return DYN_OK;
    const size_t ns = (size_t)v.na + 3 * (size_t)v.nw;
    const size_t pos_b = (size_t)capacity * ns * 3 * sizeof(float);
    const size_t vel_b = (fields & DYN_SNAP_VELOCITIES) ? pos_b : 0;
    const size_t frc_b = (fields & DYN_SNAP_FORCES) ? (size_t)capacity * v.na * 3 * sizeof(float) : 0;
    const size_t frm_b = (size_t)capacity * sizeof(dyn_frame_t);
    auto up = [](size_t x) { return (x + 255) / 256 * 256; };
    const size_t total = up(pos_b) + up(vel_b) + up(frc_b) + up(frm_b);
    void* mem = nullptr;
    const cudaError_t e = cudaMalloc(&mem, total);
    if (e != cudaSuccess) return dyn::cuda_fail(e, "cudaMalloc (snapshot ring)");
    h->snap_mem = mem;
    h->snap_bytes = total;
    char* p = (char*)mem;
    v.snap_pos = (float*)p; p += up(pos_b);
    if (vel_b) v.snap_vel = (float*)p;
    p += up(vel_b);
    if (frc_b) v.snap_force = (float*)p;
    p += up(frc_b);
    v.snap_frames = (dyn_frame_t*)p;
    v.snap_ratio = ratio;
    v.snap_cap = capacity;
    return DYN_OK;
}

extern "C" int dyn_sys_snapshots_read(dyn_sys_t h, uint32_t max_frames, float* pos, float* vel, float* force,
                                      dyn_frame_t* frames, uint32_t* n_read, uint64_t* n_lost) {
    DYN_CHECK(h && n_read, DYN_ERR_INVALID, "dyn_sys_snapshots_read: NULL argument");
    *n_read = 0;
    if (n_lost) *n_lost = 0;
    const SysView& v = h->v;
    if (!v.snap_ratio) return DYN_OK;
    DYN_CHECK(pos || max_frames == 0, DYN_ERR_INVALID, "dyn_sys_snapshots_read: NULL pos");
    DYN_CHECK(!vel || v.snap_vel, DYN_ERR_INVALID, "dyn_sys_snapshots_read: velocities are not recorded");
    DYN_CHECK(!force || v.snap_force, DYN_ERR_INVALID, "dyn_sys_snapshots_read: forces are not recorded");
    unsigned long long count = 0;
    DYN_CUDA(cudaMemcpyAsync(&count, &v.sc->snap_count, sizeof(count), cudaMemcpyDeviceToHost, h->stream));
    DYN_CUDA(cudaStreamSynchronize(h->stream));
    const uint64_t cap = v.snap_cap;
    const uint64_t first = std::max<uint64_t>(h->snap_read, count > cap ? count - cap : 0);
    if (n_lost) *n_lost = first - h->snap_read;
    const uint64_t n = std::min<uint64_t>(count - first, max_frames);
    const size_t ns = (size_t)v.na + 3 * (size_t)v.nw;
    const size_t fp = ns * 3, ff = (size_t)v.na * 3;
    // frames first .. first + n - 1 sit in at most two contiguous ranges of the ring
    for (uint64_t i = 0; i < n;) {
        const uint64_t slot = (first + i) % cap;
        const uint64_t run = std::min<uint64_t>(n - i, cap - slot);
        DYN_CUDA(cudaMemcpyAsync(pos + i * fp, v.snap_pos + slot * fp, run * fp * sizeof(float),
                                 cudaMemcpyDeviceToHost, h->stream));
        if (vel)
            DYN_CUDA(cudaMemcpyAsync(vel + i * fp, v.snap_vel + slot * fp, run * fp * sizeof(float),
                                     cudaMemcpyDeviceToHost, h->stream));
        if (force && ff)
            DYN_CUDA(cudaMemcpyAsync(force + i * ff, v.snap_force + slot * ff, run * ff * sizeof(float),
                                     cudaMemcpyDeviceToHost, h->stream));
        if (frames)
            DYN_CUDA(cudaMemcpyAsync(frames + i, v.snap_frames + slot, run * sizeof(dyn_frame_t),
                                     cudaMemcpyDeviceToHost, h->stream));
        i += run;
    }
    DYN_CUDA(cudaStreamSynchronize(h->stream));
    h->snap_read = first + n;
    *n_read = (uint32_t)n;
    return DYN_OK;
}

namespace dyn {
int evaluate_forces(dyn_sys_s* h) { return evaluate_forces_now(h); }
}  // namespace dyn

namespace dyn {
void energies_of(dyn_sys_s* h, dyn_energies_t* e) { fill_energies(h, e); }

void set_ww_split(dyn_sys_s* h, uint32_t split) {
    h->v.ww_split = std::max(1u, std::min(8u, split));
    set_block_counts(h->v);
}

void set_batch_member(dyn_sys_s* h) {
    h->batch_member = true;
    // the batch fills the GPU: no automatic group split
    if (h->cfg.ww_split == 0) h->v.ww_split = 1;
    set_block_counts(h->v);
}
}  // namespace dyn
