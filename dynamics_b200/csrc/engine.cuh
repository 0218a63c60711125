// Internal layout of the device-resident engine (layer 2 of the C ABI).
//
// HBM layout of one system
// ------------------------
// Waters are stored in cluster order: the rebuild sorts molecules into
// columns of an xy grid, by z inside a column, and pads every column to a
// multiple of 8 so that each aligned group of 8 slots is a spatially
// compact cluster.  Per slot:
//   wpos  float4[4]  O, H0, H1, M positions (.w = site charge)
//   wvel  float4[3]  O, H0, H1 velocities
//   wacc  float4[3]  accelerations from the last kick
//   wid   uint32     original molecule index (INVALID_ID for padding)
// Forces are int64 fixed point (2^-32 kcal/mol/A): wforce[slot*12 + site*3].
// Non-water atoms stay in home order (their topology indexes them) and a
// cluster-ordered copy (spos/slj/sidx) is gathered for the pair kernels.
// Reciprocal-space forces are cached by original index (wid / atom index)
// so that they survive re-sorting between SPME evaluations.
#pragma once

#include <cufft.h>

#include <algorithm>
#include <vector>

#include "common.cuh"

#define WCL 8             // waters per cluster
#define GRPW 32           // waters per i-group of the water-water kernel (4 clusters)
#define NPOLY_G 14        // coefficients of the screened-Coulomb force polynomial (14: the virial within 1e-5 of float64)
#define UMAX 5            // atoms per constraint unit (a heavy atom and up to 4 H)
#define LPW 8             // lanes per i-water in the water-water kernel
#define ACL 8             // atoms per cluster
#define INVALID_ID 0xFFFFFFFFu
#define PME_BRICK 8       // edge of the SPME grid bricks (grid points)
#define DYN_SITE_WATER 0x80000000u  // site code flag: a water site (3 * id + site) rather than an atom
#define WW_JFIX_SHIFT 16  // j-side water-water sums: int32 fixed point, 2^-16 kcal/mol/A
#define NACC 16           // accumulator slots

enum Acc {
    ACC_E_LJ_WW = 0, ACC_E_COUL_WW, ACC_E_LJ_S, ACC_E_COUL_S, ACC_VIR_SHORT,
    ACC_E_BONDED, ACC_VIR_BONDED, ACC_KE, ACC_KE_TRANS, ACC_VIR_CONSTR,
    ACC_E_14, ACC_VIR_14, ACC_E_CORR, ACC_VIR_CORR, ACC_E_RECIP, ACC_VIR_RECIP
};

// Device-resident scalars of one system.
struct Scalars {
    unsigned long long step;      // completed steps
    unsigned long long rebuilds;
    unsigned int need_rebuild;    // set by the displacement check
    unsigned int n_wclus;         // current water cluster count
    unsigned int n_aclus;         // current atom cluster count
    unsigned int overflow;        // largest list length that did not fit (0 = ok)
    unsigned int nonfinite;       // set when a kernel saw NaN/Inf
    unsigned int max_disp2_bits;  // float bits, atomicMax over non-negative floats
    unsigned int timeout;         // a bounded device wait gave up
    unsigned int pad1;
    double acc[NACC];             // finalised accumulators of the last step
    double recip_cache[4];        // e_recip, vir_recip, e_corr, vir_corr of last SPME step
    double csvr_lambda;
    double baro_mu;
    double pressure, temperature;
    double pe;                    // potential energy of the last energy step
    double ke_rigid;              // rigid-body KE of the waters + atomic KE of atoms
    double pressure_atomic;       // the reference's site-virial pressure
    unsigned long long list_pairs;
    unsigned int ctr_disp;        // blocks done in k_disp_check (last one decides)
    unsigned int ctr_scale;       // blocks done in k_scale (last one scales the box)
    unsigned int union_max;       // largest group union of the last rebuild
    unsigned int a_sparse_base;   // first slot of the single-atom clusters
    unsigned int n_ws_items;      // work items of the water-atom pair kernel
    unsigned int n_ss_items;      // work items of the atom-atom pair kernel
    double time_ps;               // simulated time (sum of the steps' dt)
    unsigned long long snap_count;  // snapshot frames recorded
    // reciprocal energy / virial of the SPME passes of one evaluation, their
    // dH/dlambda (alchemical cross term), its cached value and the step's
    // total dH/dlambda
    double recip_acc[2];
    double recip_dh, recip_dh_cache, dh_dl;
    // steepest-descent minimizer (dyn_sys_minimize)
    double min_e_prev;            // energy of the last accepted geometry
    float min_alpha, min_alpha_try, min_fmax, min_step;
    unsigned int min_fmax_bits, min_ctr;
    unsigned int min_accepted, min_trials, min_done, min_action;
    // pruned water-water lists: set by the displacement check (or with a
    // rebuild), cleared when the prune has run
    unsigned int need_prune;
    unsigned int max_dprune_bits;  // float bits, as max_disp2_bits
    unsigned long long prunes;
    unsigned int spme_ovf;        // sites of this SPME pass beyond their brick's capacity
    unsigned int spme_ovf_max;    // largest spme_ovf seen
};

// One charged site of an SPME pass, binned by the grid brick of its stencil
// base: fractional grid coordinates, charge and base (x | y << 10 | z << 20).
struct SiteRec {
    double w[3];
    float q;
    uint32_t base;
};

// Partial-sum regions (each kernel family writes 4 doubles per block).
enum Region {
    REG_WW = 0, REG_WS, REG_SW, REG_SS, REG_14, REG_BOND, REG_KICK_W, REG_KICK_A,
    REG_CONS, REG_PME, REG_CORR, REG_CORR_A, REG_COM, NREGION
};

// Pointers and sizes passed by value to every kernel.
struct SysView {
    // waters (cluster order)
    uint32_t nw, nw_cap, nwclus_cap;
    float4* wpos; float4* wvel; float4* wacc; uint32_t* wid;
    long long* wforce;            // [nw_cap*12] O,H0,H1,M
    float4* wref;                 // O position at the last rebuild [nw_cap]
    float4* wtmp;                 // scratch for permutation [nw_cap*10]
    uint32_t* wtmp_id;
    long long* wrecip;            // [nw*9] recip + corrections on M, H0, H1 by original id (M,H0,H1)
    // atoms (home order)
    uint32_t na, na_cap, naclus_cap;
    float4* apos;                 // x, y, z, q
    float4* avel;                 // x, y, z, unused
    float4* aacc;
    float* amass;                 // 0 for static atoms' integration purposes handled by astatic
    float2* alj;                  // sigma, eps
    uint8_t* astatic;
    long long* aforce;            // [na*3]
    long long* arecip;            // [na*3]
    float4* aref;                 // position at the last rebuild
    // atom cluster copy
    float4* spos; float2* slj; uint32_t* sidx;   // [na_cap]
    uint32_t* aslot;              // home index -> cluster slot [na]
    // atoms without bonds (ions) get a cluster each: their rank among such
    // atoms, INVALID_ID for the others [na]
    uint32_t* asparse; uint32_t n_sparse;
    // exclusion CSR over home indices (1-2, 1-3 and 1-4 partners)
    uint32_t* ex_off; uint32_t* ex_idx;
    // columns
    uint32_t ncx, ncy, ncol;
    uint32_t ancx, ancy, ancol;   // a finer column grid for non-water atoms
    uint32_t* col_count; uint32_t* col_off; uint32_t* col_fill;   // [ncol(+1)]
    uint32_t* col_boff;                         // unpadded bucket offsets [ncol+1]
    uint32_t* acol_count; uint32_t* acol_off; uint32_t* acol_fill; uint32_t* acol_boff;
    uint32_t* wnew;                             // new slot of each old water slot
    float* wkey; float* akey;                   // z sort keys (fraction of the box)
    uint32_t* bucket; uint32_t* abucket;        // unsorted column members
    uint32_t* wcol; uint32_t* acol;             // column of each water / atom
    // cluster bounding boxes (center xyz, half extent xyz)
    float4* wbb_c; float4* wbb_h; float4* abb_c; float4* abb_h;
    // cluster lists (fixed capacity per i cluster): water cluster -> atom
    // clusters, atom cluster -> atom clusters (cj >= ci) with masks; work
    // items {i cluster, first entry} of ch_mix (1..32) list entries, in i order
    uint32_t cap_ws, cap_ss, ch_mix;
    uint32_t* ws_n; uint32_t* ws_j;
    uint32_t* ss_n; uint32_t* ss_j; unsigned long long* ss_mask;
    uint2* ws_item; uint2* ss_item;
    uint32_t ws_item_cap, ss_item_cap;
    // water-water: per 32-water i-group the candidate j-clusters (tile_j),
    // the union of the waters its members need, stored as runs of
    // consecutive slots (staged in shared memory by bulk copies), and per
    // i-water a list of indices into that union
    uint32_t ngrp_cap, cap_tile, cap_nb, cap_union, cap_run;
    uint32_t union_chunk;         // waters staged in shared memory at a time
    uint32_t ww_split;            // CTAs sharing one group's list entries (small systems)
    float4* gbb_c; float4* gbb_h;
    uint32_t* tile_n; uint32_t* tile_j;      // [ngrp_cap], [ngrp_cap*cap_tile]
    uint32_t* grp_nrun; uint32_t* grp_nloc;  // [ngrp_cap]
    uint2* grp_run;                          // [ngrp_cap*cap_run] (slot, union offset)
    uint16_t* cand_loc;                      // [ngrp_cap*cap_tile*8] rebuild scratch
    uint32_t* wnb_n; uint16_t* wnb;          // [nw_cap], [nw_cap*cap_nb]
    // the lists the water-water kernel walks: wnb pruned to molecule pairs
    // within r_in (k_ww_prune), re-pruned when a water has moved half of
    // r_in's buffer since the last prune (O positions then: wprune)
    uint32_t* winb_n; uint16_t* winb;        // [nw_cap], [nw_cap*cap_nb]
    float4* wprune;                          // [nw_cap]
    uint32_t* grp_uslot;                     // [ngrp_cap*cap_union] union index -> slot
    // The molecule lists are half lists (each water pair once, listed by
    // the lower slot).  The j-side forces a group's CTA computes are summed
    // in shared memory as int32 fixed point (2^-16 kcal/mol/A) per union
    // water and added to wforce with int64 atomics; contributions too large
    // for the int32 sums go to wforce directly.
    // 1-4 pairs, exclusions (pairs), bonded terms, constraints
    uint32_t n14; uint2* p14; float4* p14_par;     // sigma, eps, qq, unused
    uint32_t nexcl; uint2* excl; float* excl_qq;
    uint32_t nbond; uint2* bond; float2* bond_par;
    uint32_t nangle; uint4* angle; float2* angle_par;
    uint32_t ndih; uint4* dih; float4* dih_par;      // k, n, phase
    uint32_t ncons; uint2* cons; float* cons_r0;
    // atoms grouped for the constraints: unit u = atoms unit_idx[unit_off[u]
    // .. unit_off[u+1]), the heavy atom first, then its constrained H (with
    // r0^2 in unit_r02); unconstrained atoms are units of one
    uint32_t nunit; uint32_t* unit_off; uint32_t* unit_idx; float* unit_r02;
    uint32_t lincs_order, lincs_iter;
    // PME
    uint32_t K[3];
    long long* qgrid_fix;   // [K0*K1*K2] overflow charge (zero between passes)
    float* qgrid;           // real grid (cuFFT in/out)
    float2* cgrid;          // complex grid [K0*K1*(K2/2+1)]
    float* bmod[3];         // |b(m)|^2 per dimension
    // grid bricks of the spread and gather (PME_BRICK^3 points each): the
    // charged sites binned by their stencil base's brick, brick_cap per
    // brick, the rest in the overflow list
    uint32_t nbrick[3], n_bricks, brick_cap, n_sites_max;
    uint32_t* brick_n;      // [n_bricks] sites binned this pass (the gather zeroes it)
    uint32_t* brick_ovf;    // [n_bricks] 1: overflow charge for this brick waits in qgrid_fix
    long long* brick_tile;  // [n_bricks][11^3] each brick's spread tile (the brick and 3 points below)
    SiteRec* brick_site;    // [n_bricks * brick_cap]
    uint32_t* brick_sid;    // site codes (atom index, or DYN_SITE_WATER | 3 * water id + site)
    SiteRec* ovf_site;      // [n_sites_max]
    uint32_t* ovf_sid;
    float* wsite_f;         // [nw*9] reciprocal force on H0, H1, M by water id, before corrections
    // box and scalars
    BoxDev* box;
    Scalars* sc;
    double* partials;       // [NREGION][max_blocks][4]
    uint32_t max_blocks;
    // parameters
    float rc, rc2, ljc2, alpha, buffer;
    float r_ww, r_ws, r_ss;     // list radii
    float r_ws_skip2;           // (cutoff + O-H reach)^2: water-atom entries beyond it are skipped
    float r_in, prune_buf;      // pruned water-water radius and its buffer
    uint32_t flags;
    uint64_t seed;
    float temperature, gamma, tau_t, p_target, tau_p, kappa;
    uint32_t thermo_dof;
    uint32_t integrator, thermostat, barostat;
    uint32_t spme_interval, com_interval, recenter_interval;
    // snapshot ring (dyn_sys_snapshots): every snap_ratio steps one frame of
    // snap_cap; positions / velocities [n_atoms + 3 n_water][3], forces
    // [n_atoms][3] (NULL = not recorded)
    uint32_t snap_ratio, snap_cap;
    float* snap_pos; float* snap_vel; float* snap_force;
    dyn_frame_t* snap_frames;
    double total_mass;            // amu, for the frame density
    // alchemical decoupling of atoms [alch_lo, alch_hi) on the staged
    // schedule: Coulomb scale and its lambda derivative, soft-core LJ
    // lambda and its lambda derivative
    uint32_t alch_on, alch_lo, alch_hi;
    float alch_cs, alch_dcs, alch_ll, alch_dll;
    double e_self;          // Ewald self energy -alpha/sqrt(pi) sum q^2
    // screened-Coulomb force q q (r^-3 + g(r^2)) d: g as a polynomial in
    // t = 2 r^2 / rc^2 - 1 (Chebyshev interpolation, power basis, Horner in
    // float32)
    float poly_g[NPOLY_G];
    float two_over_rc2;
    // IF-node handles of the captured step graph: the displacement check
    // sets cond_rebuild, the step finalisation sets cond_periodic; only
    // kernels captured for a graph (use_cond != 0) set them
    cudaGraphConditionalHandle cond_rebuild, cond_periodic, cond_prune;
    uint32_t use_cond;
    uint32_t nb[NREGION];   // blocks each region's kernel is launched with
    int plan_f, plan_b;     // cuFFT plans (host-side handles, used by launch code only)
};

// ---------------------------------------------------------------------------
// One kernel body, two launch forms.  Every step kernel is written once as
// the body of NAME##_B::run(v, bk, ...), where bk is the block's index and
// the block count within its system.  NAME is the single-system kernel (the
// SysView in parameter space); NAME##_batch runs the same body for many
// systems in one launch: block b works on system bm[b].x as its local block
// bm[b].y & 0xFFFF of bm[b].y >> 16, reading that system's SysView from
// global memory.  The block ranges are laid out by Target::launch below.
// ---------------------------------------------------------------------------
struct Blk { uint32_t idx, cnt; };

// Programmatic dependent launch: every step kernel is launched allowed to
// overlap its launch with the end of the kernel before it on the stream; it
// waits here until that kernel has completed and its writes are visible.
// No kernel triggers its dependents early: blocks of the next kernel parked
// on SMs while the current one runs cost more than the launch they hide
// (measured on the step graphs).
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

#define DYN_UNPAREN(...) __VA_ARGS__

#define DYN_KERNEL(LB, NAME, PARAMS, ARGS)                                                          \
    struct NAME##_B {                                                                                \
        static __device__ __forceinline__ void run(const SysView& v, Blk bk DYN_UNPAREN PARAMS);     \
    };                                                                                               \
    __global__ void LB NAME(const __grid_constant__ SysView v DYN_UNPAREN PARAMS) {                  \
        pdl_enter();                                                                                 \
        NAME##_B::run(v, Blk{blockIdx.x, gridDim.x} DYN_UNPAREN ARGS);                               \
    }                                                                                                \
    __global__ void LB NAME##_batch(const SysView* __restrict__ vs,                                  \
                                    const uint2* __restrict__ bm DYN_UNPAREN PARAMS) {               \
        pdl_enter();                                                                                 \
        const uint2 m = bm[blockIdx.x];                                                              \
        NAME##_B::run(vs[m.x], Blk{m.y & 0xFFFFu, m.y >> 16} DYN_UNPAREN ARGS);                      \
    }                                                                                                \
    __device__ __forceinline__ void NAME##_B::run(const SysView& v, Blk bk DYN_UNPAREN PARAMS)

// DYN_KERNEL for a template (TDECL its parameters, TARGS their names), with
// launch bounds LBB of their own for NAME##_batch, which reads its SysView
// from global memory and so holds more registers; DYN_KERNEL_T gives both
// forms the same bounds.
#define DYN_KERNEL_T2(TDECL, TARGS, LB, LBB, NAME, PARAMS, ARGS)                                    \
    template <DYN_UNPAREN TDECL>                                                                     \
    struct NAME##_B {                                                                                \
        static __device__ __forceinline__ void run(const SysView& v, Blk bk DYN_UNPAREN PARAMS);     \
    };                                                                                               \
    template <DYN_UNPAREN TDECL>                                                                     \
    __global__ void LB NAME(const __grid_constant__ SysView v DYN_UNPAREN PARAMS) {                  \
        pdl_enter();                                                                                 \
        NAME##_B<DYN_UNPAREN TARGS>::run(v, Blk{blockIdx.x, gridDim.x} DYN_UNPAREN ARGS);            \
    }                                                                                                \
    template <DYN_UNPAREN TDECL>                                                                     \
    __global__ void LBB NAME##_batch(const SysView* __restrict__ vs,                                 \
                                     const uint2* __restrict__ bm DYN_UNPAREN PARAMS) {              \
        pdl_enter();                                                                                 \
        const uint2 m = bm[blockIdx.x];                                                              \
        NAME##_B<DYN_UNPAREN TARGS>::run(vs[m.x], Blk{m.y & 0xFFFFu, m.y >> 16} DYN_UNPAREN ARGS);   \
    }                                                                                                \
    template <DYN_UNPAREN TDECL>                                                                     \
    __device__ __forceinline__ void NAME##_B<DYN_UNPAREN TARGS>::run(const SysView& v,               \
                                                                     Blk bk DYN_UNPAREN PARAMS)

#define DYN_KERNEL_T(TDECL, TARGS, LB, NAME, PARAMS, ARGS) DYN_KERNEL_T2(TDECL, TARGS, LB, LB, NAME, PARAMS, ARGS)

// ---------------------------------------------------------------------------
// Launch target: one system, or every system of a batch.  The launch code
// of each stage is written once against a Target; grid(v) gives the blocks
// one system needs (0 = skip it).  For a batch, the per-system ranges are
// concatenated into one block map and the NAME##_batch kernel runs them all.
// ---------------------------------------------------------------------------
struct BatchCtx;
struct BlockMap { uint32_t total; const uint2* d_map; };
uint32_t batch_size(const BatchCtx* b);
const SysView& batch_view(const BatchCtx* b, uint32_t i);
const SysView* batch_dviews(const BatchCtx* b);
bool batch_collecting(const BatchCtx* b);
BlockMap batch_map(BatchCtx* b, const std::vector<uint32_t>& blocks);
// Side streams (and fork/join events: ev[0..n) join, ev[n] forks) over
// which a batch spreads its members' cuFFT executions; n = 0 for none.
int batch_fft_streams(BatchCtx* b, cudaStream_t** st, cudaEvent_t** ev);

struct Target {
    const SysView* v = nullptr;   // single system
    BatchCtx* b = nullptr;        // batch (v == nullptr)
    cudaStream_t st = nullptr;

    template <typename K, typename... A>
    static void launch_pdl(K k, int grid, int threads, size_t smem, cudaStream_t s, A... a) {
        cudaLaunchConfig_t c = {};
        c.gridDim = dim3((unsigned)grid);
        c.blockDim = dim3((unsigned)threads);
        c.dynamicSmemBytes = smem;
        c.stream = s;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[0].val.programmaticStreamSerializationAllowed = 1;
        c.attrs = at;
        c.numAttrs = 1;
        cudaLaunchKernelEx(&c, k, a...);
    }

    template <typename KP, typename KB, typename G, typename... A>
    void launch(KP kp, KB kb, G grid, int threads, size_t smem, A... a) const {
        if (v) {
            const int g = grid(*v);
            if (g > 0) launch_pdl(kp, g, threads, smem, st, *v, a...);
            return;
        }
        const uint32_t n = batch_size(b);
        std::vector<uint32_t> bl(n);
        for (uint32_t i = 0; i < n; ++i) {
            const int g = grid(batch_view(b, i));
            bl[i] = g > 0 ? (uint32_t)g : 0u;
        }
        const BlockMap m = batch_map(b, bl);
        if (m.total && !batch_collecting(b))
            launch_pdl(kb, (int)m.total, threads, smem, st, batch_dviews(b), m.d_map, a...);
    }
    // host-side work per system (library calls such as cuFFT); skipped
    // while a batch only collects its block maps
    template <typename F>
    void each(F f) const {
        if (v) { f(*v); return; }
        if (batch_collecting(b)) return;
        for (uint32_t i = 0; i < batch_size(b); ++i) f(batch_view(b, i));
    }
    template <typename F>
    size_t max_over(F f) const {
        if (v) return f(*v);
        size_t m = 0;
        for (uint32_t i = 0; i < batch_size(b); ++i) m = std::max<size_t>(m, f(batch_view(b, i)));
        return m;
    }
    bool any(bool (*pred)(const SysView&)) const {
        if (v) return pred(*v);
        for (uint32_t i = 0; i < batch_size(b); ++i)
            if (pred(batch_view(b, i))) return true;
        return false;
    }
};

// ---------------------------------------------------------------------------
// launch wrappers (defined in the .cu files)
// ---------------------------------------------------------------------------
namespace dyn {

// nblist.cu
void launch_displacement_check(const Target& t);
void launch_rebuild(const Target& t, bool force);
// prunes the water-water lists if the displacement check (or a rebuild) asked
// for it, or with force
void launch_prune(const Target& t, bool force);
void launch_gather_atoms(const Target& t);

// pair.cu
void launch_pairs(const Target& t, bool energy);
// the two independent parts of launch_pairs: water-water then water-atom
// (the latter adds to the water forces the former stores), and atom-atom
void launch_pairs_water(const Target& t, bool energy);
void launch_pairs_atoms(const Target& t, bool energy);
// the parts of launch_pairs_water, in order: water-water, its j-side
// gather, water-atom
void launch_pairs_ww(const Target& t, bool energy);
void launch_pairs_ws(const Target& t, bool energy);
void launch_pair14(const Target& t, bool energy);
int pair_ww_setup(const SysView& v);
int ww_tile_blocks(const SysView& v);
size_t ww_tile_smem(const SysView& v);
int pair_blocks_ss(const SysView& v);
int pair_blocks_ws(const SysView& v);
int pair14_blocks(const SysView& v);

// pme.cu
int pme_init(SysView& v, cufftHandle* plan_f, cufftHandle* plan_b, cudaStream_t st);
void pme_free(SysView& v, cufftHandle plan_f, cufftHandle plan_b);
void launch_pme(const Target& t);
// the parts of one SPME pass (launch_pme runs them for every pass)
void launch_pme_spread(const Target& t, int pass);
void launch_pme_transform(const Target& t, int pass);
void launch_pme_gather(const Target& t, int pass);
void launch_corrections(const Target& t);
int pme_blocks(const SysView& v);
int gather_blocks(const SysView& v);
// brick layout and capacity of the spread / gather (nbrick, n_bricks, brick_cap, n_sites_max)
void pme_bricks(SysView& v, uint32_t cap);
int corr_blocks(const SysView& v);

// integrate.cu
void launch_first_half(const Target& t, float dt);
void launch_second_half(const Target& t, float dt);
// their water and atom parts, which touch disjoint data
void launch_first_half_water(const Target& t, float dt);
void launch_first_half_atoms(const Target& t, float dt);
void launch_second_half_water(const Target& t, float dt);
void launch_second_half_atoms(const Target& t, float dt);
void launch_finalize(const Target& t, float dt, bool energy, bool thermo);
void launch_periodic(const Target& t);
void launch_bonded(const Target& t, bool energy);
int kick_blocks_w(const SysView& v);
int kick_blocks_a(const SysView& v);
int bond_blocks(const SysView& v);

}  // namespace dyn
