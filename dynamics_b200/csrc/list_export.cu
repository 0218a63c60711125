// Read-out of the resident engine's neighbour lists (dyn_sys_list_pairs).
//
// The pair kernels never see a flat pair list: water-water pairs come from
// per-water lists of indices into a water group's union of j-waters,
// water-atom and atom-atom pairs from cluster-pair lists (the latter with
// 64-bit interaction masks).  This expands the lists exactly as the kernels
// walk them into pairs of original indices (water ids in the order the
// system was created, atom indices), so that a test can check that every
// pair inside the cutoff is covered (src/neighbors.rs:102-281 holds every
// pair within cutoff + skin by construction; here the cluster geometry and
// the pruning decide it, so it is checked).  Host-side and synchronous; not
// for the step loop.
#include <cstring>
#include <vector>

#include "sys_internal.cuh"

namespace {

template <typename T>
int d2h(std::vector<T>& out, const T* src, size_t n) {
    out.resize(n);
    if (n) DYN_CUDA(cudaMemcpy(out.data(), src, n * sizeof(T), cudaMemcpyDeviceToHost));
    return DYN_OK;
}

#define TRY_D2H(out_, src_, n_)                          \
    do {                                                 \
        const int rc_ = d2h(out_, src_, (size_t)(n_));   \
        if (rc_ != DYN_OK) return rc_;                   \
    } while (0)

// water-water: the molecule pairs (i, j) the water-water kernel evaluates
int ww_pairs(const SysView& v, const Scalars& sc, std::vector<uint32_t>& out) {
    const uint32_t ng = (sc.n_wclus + GRPW / WCL - 1) / (GRPW / WCL);
    std::vector<uint32_t> wid, nloc, nrun, nb_n;
    std::vector<uint2> runs;
    std::vector<uint16_t> nb;
    TRY_D2H(wid, v.wid, v.nw_cap);
    TRY_D2H(nloc, v.grp_nloc, ng);
    TRY_D2H(nrun, v.grp_nrun, ng);
    TRY_D2H(runs, v.grp_run, (size_t)ng * v.cap_run);
    // the pruned lists: what the water-water kernel walks
    TRY_D2H(nb_n, v.winb_n, v.nw_cap);
    TRY_D2H(nb, v.winb, (size_t)v.nw_cap * v.cap_nb);
    std::vector<uint32_t> uni;
    for (uint32_t g = 0; g < ng; ++g) {
        // the group's union: union index -> slot, from its runs
        uni.assign(nloc[g], INVALID_ID);
        for (uint32_t t = 0; t < nrun[g]; ++t) {
            const uint2 r = runs[(size_t)g * v.cap_run + t];
            const uint32_t end = t + 1 < nrun[g] ? runs[(size_t)g * v.cap_run + t + 1].y : nloc[g];
            for (uint32_t u = r.y; u < end && u < nloc[g]; ++u) uni[u] = r.x + (u - r.y);
        }
        for (uint32_t il = 0; il < GRPW; ++il) {
            const uint32_t s = g * GRPW + il;
            if (s >= v.nw_cap || wid[s] == INVALID_ID) continue;
            for (uint32_t k = 0; k < nb_n[s]; ++k) {
                const uint32_t u = nb[(size_t)s * v.cap_nb + k];
                const uint32_t sj = u < uni.size() ? uni[u] : INVALID_ID;
                if (sj == INVALID_ID || sj >= v.nw_cap || wid[sj] == INVALID_ID) continue;
                out.push_back(wid[s]);
                out.push_back(wid[sj]);
            }
        }
    }
    return DYN_OK;
}

// water-atom: every (water, atom) of the water-cluster x atom-cluster pairs
int ws_pairs(const SysView& v, const Scalars& sc, std::vector<uint32_t>& out) {
    std::vector<uint32_t> wid, sidx, n, j;
    TRY_D2H(wid, v.wid, v.nw_cap);
    TRY_D2H(sidx, v.sidx, v.na_cap);
    TRY_D2H(n, v.ws_n, sc.n_wclus);
    TRY_D2H(j, v.ws_j, (size_t)sc.n_wclus * v.cap_ws);
    for (uint32_t ci = 0; ci < sc.n_wclus; ++ci)
        for (uint32_t k = 0; k < n[ci]; ++k) {
            const uint32_t cj = j[(size_t)ci * v.cap_ws + k];
            for (uint32_t ii = 0; ii < WCL; ++ii) {
                const uint32_t w = wid[ci * WCL + ii];
                if (w == INVALID_ID) continue;
                for (uint32_t jj = 0; jj < ACL; ++jj) {
                    const uint32_t a = sidx[(size_t)cj * ACL + jj];
                    if (a == INVALID_ID) continue;
                    out.push_back(w);
                    out.push_back(a);
                }
            }
        }
    return DYN_OK;
}

// atom-atom: the (i, j) pairs whose bit is set in a cluster pair's mask
int ss_pairs(const SysView& v, const Scalars& sc, std::vector<uint32_t>& out) {
    std::vector<uint32_t> sidx, n, j;
    std::vector<unsigned long long> m;
    TRY_D2H(sidx, v.sidx, v.na_cap);
    TRY_D2H(n, v.ss_n, sc.n_aclus);
    TRY_D2H(j, v.ss_j, (size_t)sc.n_aclus * v.cap_ss);
    TRY_D2H(m, v.ss_mask, (size_t)sc.n_aclus * v.cap_ss);
    for (uint32_t ci = 0; ci < sc.n_aclus; ++ci)
        for (uint32_t k = 0; k < n[ci]; ++k) {
            const size_t e = (size_t)ci * v.cap_ss + k;
            for (uint32_t b = 0; b < 64; ++b) {
                if (!((m[e] >> b) & 1ull)) continue;
                const uint32_t a = sidx[(size_t)ci * ACL + b / ACL], c = sidx[(size_t)j[e] * ACL + b % ACL];
                if (a == INVALID_ID || c == INVALID_ID) continue;
                out.push_back(a);
                out.push_back(c);
            }
        }
    return DYN_OK;
}

}  // namespace

extern "C" int dyn_sys_list_pairs(dyn_sys_t h, uint32_t kind, uint32_t* pairs, uint64_t capacity,
                                  uint64_t* n_pairs) {
    DYN_CHECK(h && n_pairs, DYN_ERR_INVALID, "dyn_sys_list_pairs: NULL argument");
    DYN_CHECK(kind <= 2, DYN_ERR_INVALID, "dyn_sys_list_pairs: kind must be 0, 1 or 2");
    DYN_CUDA(cudaStreamSynchronize(h->stream));
    Scalars sc;
    DYN_CUDA(cudaMemcpy(&sc, h->v.sc, sizeof(Scalars), cudaMemcpyDeviceToHost));
    const SysView& v = h->v;
    std::vector<uint32_t> out;
    int rc = DYN_OK;
    if (kind == 0 && v.nw) rc = ww_pairs(v, sc, out);
    else if (kind == 1 && v.nw && v.na) rc = ws_pairs(v, sc, out);
    else if (kind == 2 && v.na) rc = ss_pairs(v, sc, out);
    if (rc != DYN_OK) return rc;
    *n_pairs = out.size() / 2;
    if (!pairs) return DYN_OK;
    DYN_CHECK(capacity >= out.size() / 2, DYN_ERR_INVALID, "dyn_sys_list_pairs: capacity below the pair count");
    if (!out.empty()) std::memcpy(pairs, out.data(), out.size() * sizeof(uint32_t));
    return DYN_OK;
}
