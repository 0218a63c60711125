/*
 * dynb200 -- B200-native (sm_100a) nonbonded force and integration engine
 * for the molecular-dynamics library David-OConnor/dynamics (crate
 * `dynamics` 0.2.2).  This header is the whole drop-in boundary: a plain
 * C ABI (opaque handles, pointers and sizes, int status codes) that a Rust
 * `extern "C"` block, ctypes or C++ can bind.
 *
 * Two layers:
 *
 *  1. dyn_nb_*  -- one-to-one replacement of src/gpu_interface.rs.  The
 *     caller keeps the simulation state on the host, exactly like the
 *     reference's MdState, and asks the GPU for the short-range forces of a
 *     flat pair list each step.  dyn_nb_build_pairs additionally replaces
 *     build_all_neighbors + setup_pairs (src/neighbors.rs:102-156,
 *     src/non_bonded.rs:541-677) with a GPU cell-list build whose pair set is
 *     bit-identical to the reference's brute-force lists.
 *
 *  2. dyn_sys_*  -- the native, device-resident engine behind
 *     MdState::step (src/integrate.rs:72): positions, velocities, neighbour
 *     cluster lists and PME grids stay in HBM; one call advances n steps.
 *
 * Conventions (both layers):
 *  - Every call returns DYN_OK (0) or a negative DYN_ERR_* code and never
 *    aborts the process.  dyn_last_error() returns a message for the last
 *    failure on the calling thread.
 *  - Handles are opaque.  One handle = one CUDA stream; a handle is not
 *    thread-safe, distinct handles may be used from distinct threads.
 *  - Caller-owned host buffers are only read/written during the call.
 *    Device memory is owned by the library and released by *_destroy.
 *  - Units: Angstrom, ps, amu, kcal/mol.  Charges are pre-scaled by
 *    18.2223 = sqrt(332.0522) as in the reference (src/non_bonded.rs:58-63).
 *  - Streams are passed as `void*` holding a cudaStream_t.  For dyn_nb_*
 *    NULL means the legacy default stream; dyn_sys_create with NULL creates
 *    a non-blocking stream of its own (a captured CUDA graph cannot be
 *    launched on the legacy stream).
 */
#ifndef DYNB200_H
#define DYNB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DYN_OK 0
#define DYN_ERR_INVALID (-1)    /* bad argument, size or call order        */
#define DYN_ERR_CUDA (-2)       /* a CUDA runtime / cuFFT call failed      */
#define DYN_ERR_OOM (-3)        /* device or pinned allocation failed      */
#define DYN_ERR_NONFINITE (-5)  /* NaN/Inf detected in coordinates/forces  */
#define DYN_ERR_TIMEOUT (-6)    /* a bounded device wait gave up           */
#define DYN_ERR_UNSUPPORTED (-7)/* feature not available for this system  */

/* ------------------------------------------------------------------ */
/* errors / version                                                    */
/* ------------------------------------------------------------------ */

/* Message describing the last failed call on this thread ("" if none). */
const char* dyn_last_error(void);
/* Library version, e.g. 1 */
int dyn_version(void);
/* Number of CUDA devices visible; 0 without a GPU (never fails). */
int dyn_device_count(void);
/* Measured FP32 FMA throughput of the current device in TFLOP/s (best of 5
 * launches of an FMA-chain kernel over all SMs); the roofline denominator
 * for the FP32 pair kernels. */
int dyn_probe_fp32_peak(void* stream, double* tflops);

/* ------------------------------------------------------------------ */
/* Layer 1: gpu_interface.rs replacement                              */
/* ------------------------------------------------------------------ */

typedef struct dyn_nb_s* dyn_nb_t;

/* Override bits, mirroring MdOverrides (src/lib.rs:590-607) as the pair
 * kernel honours them (src/cuda/cuda.cu:229-230). */
#define DYN_OVR_COULOMB_DISABLED 1u
#define DYN_OVR_LJ_DISABLED 2u

/* Pair flag bits for dyn_nb_set_pairs' packed flags array; one byte per
 * pair replaces the reference's four bool arrays (scale_14s, calc_ljs,
 * calc_coulombs, symmetric; src/gpu_interface.rs:233-237). */
#define DYN_PAIR_SCALE14 1u
#define DYN_PAIR_LJ 2u
#define DYN_PAIR_COULOMB 4u
#define DYN_PAIR_SYMMETRIC 8u
/* The pair crosses the alchemical molecule's boundary (the reference's
 * alch_interactions array, src/gpu_interface.rs:238,267-338): soft-core LJ
 * and scaled Coulomb on the staged decoupling schedule in
 * dyn_nb_forces_alch.  dyn_nb_forces_static ignores it (full coupling). */
#define DYN_PAIR_ALCH 16u

/* Body codes, one byte per pair end: 0 = non-water atom, 1..4 = water site
 * O, M, H0, H1 (the reference's atom_types_* + water_types_* arrays,
 * src/gpu_interface.rs:269-279, WaterSite src/solvent/mod.rs:256-261). */
#define DYN_BODY_ATOM 0u
#define DYN_BODY_W_O 1u
#define DYN_BODY_W_M 2u
#define DYN_BODY_W_H0 3u
#define DYN_BODY_W_H1 4u

/* Replaces ForcesPositsGpu::new (src/gpu_interface.rs:123-214): device and
 * pinned buffers for n_dyn atoms and n_water 4-site waters.
 * lj_cutoff <= 0 reproduces the reference CUDA kernel (no LJ cutoff,
 * src/cuda/cuda.cu:277-279); lj_cutoff > 0 reproduces the CPU path
 * (LJ only for r <= lj_cutoff, src/non_bonded.rs:1001). */
int dyn_nb_create(void* stream, uint32_t n_dyn, uint32_t n_water, float cutoff_ewald,
                  float alpha_ewald, float lj_cutoff, dyn_nb_t* out);
/* n_dyn and n_water must each be below 2^27. */

/* Replaces PerNeighborGpu::new (src/gpu_interface.rs:243-410): uploads the
 * flat pair list.  tgt/src index the atom array (body 0) or the water
 * molecule (bodies 1..4).  body_tgt/body_src: DYN_BODY_* per pair.
 * flags: DYN_PAIR_* per pair.  The library re-packs these into its own
 * 20-byte-per-pair layout. */
int dyn_nb_set_pairs(dyn_nb_t h, uint64_t n_pairs, const uint32_t* tgt, const uint32_t* src,
                     const float* sigma, const float* eps, const float* q_tgt,
                     const float* q_src, const uint8_t* body_tgt, const uint8_t* body_src,
                     const uint8_t* flags);

/* Replaces build_all_neighbors + setup_pairs + PerNeighborGpu::new
 * (src/neighbors.rs:102-156, src/non_bonded.rs:541-677,
 * src/gpu_interface.rs:243-410) on the GPU.  Builds the three Verlet lists
 * with |min_image(d)|^2 < (cutoff+skin)^2 in the reference's float32
 * arithmetic (bit-identical pair set; water uses wrapped O positions), then
 * the flat pair list in the reference's canonical order, and installs it as
 * if by dyn_nb_set_pairs.
 *   atom_*: n_dyn entries (positions [n_dyn*3]); is_static/bonded_only may be
 *           NULL (all false).
 *   excl / pair14: (i, j) index pairs, i < j, for 1-2/1-3 exclusions and
 *           1-4 scaled pairs (src/prep.rs:114-143).
 *   box_lo/box_hi: SimBox bounds (src/barostat.rs:56-61).
 * n_pairs_out receives the flat pair count. */
int dyn_nb_build_pairs(dyn_nb_t h, const float* pos_dyn, const float* pos_w_o,
                       const float* atom_q, const float* atom_sigma, const float* atom_eps,
                       const uint8_t* is_static, const uint8_t* bonded_only,
                       uint64_t n_excl, const uint32_t* excl, uint64_t n_pair14,
                       const uint32_t* pair14, const float box_lo[3], const float box_hi[3],
                       float skin, uint64_t* n_pairs_out);

/* Copies the installed flat pair list back to the host (arrays of n_pairs
 * entries, any of them may be NULL).  Used to check the pair set. */
int dyn_nb_get_pairs(dyn_nb_t h, uint64_t n_pairs, uint32_t* tgt, uint32_t* src, float* sigma,
                     float* eps, float* q_tgt, float* q_src, uint8_t* body_tgt,
                     uint8_t* body_src, uint8_t* flags);

/* Replaces force_nonbonded_gpu (src/gpu_interface.rs:463-632): uploads the
 * positions (float [3*n] per array, as the reference's five position
 * arrays), evaluates the installed pair list and returns forces on the
 * target/source of every pair (float64 [3*n] arrays), the virial sum and
 * the potential energy with the reference's conventions (energy only for
 * pairs whose target is a non-water atom).  Forces are accumulated as
 * 64-bit fixed point on the device, so repeated calls are bit-identical.
 * cell_extent: SimBox extent (bounds_high - bounds_low). */
int dyn_nb_forces(dyn_nb_t h, const float* pos_dyn, const float* pos_w_o, const float* pos_w_m,
                  const float* pos_w_h0, const float* pos_w_h1, const float cell_extent[3],
                  uint32_t override_bits, double* f_dyn, double* f_w_o, double* f_w_m,
                  double* f_w_h0, double* f_w_h1, double* virial, double* energy);

/* force_nonbonded_gpu with its lambda_alch argument (src/gpu_interface.rs:
 * 463-632, kernel src/cuda/cuda.cu:367-566).  When any installed pair
 * carries DYN_PAIR_ALCH, those pairs take Beutler soft-core LJ (alpha 0.5,
 * power 1, soft-core sigma >= 3 A) at the schedule's LJ lambda and
 * short-range Coulomb times the schedule's scale (staged schedule: Coulomb
 * off over lambda 0..0.5, LJ decoupled over 0.5..1, lambda clamped to
 * [0, 1]), and *dh_dl receives the sum of their dH/dlambda.  With no
 * alchemical pair installed this is dyn_nb_forces and *dh_dl = 0.
 * dyn_nb_forces is this call with lambda_alch = 0 and no dh_dl. */
int dyn_nb_forces_alch(dyn_nb_t h, const float* pos_dyn, const float* pos_w_o,
                       const float* pos_w_m, const float* pos_w_h0, const float* pos_w_h1,
                       const float cell_extent[3], uint32_t override_bits, double lambda_alch,
                       double* f_dyn, double* f_w_o, double* f_w_m, double* f_w_h0,
                       double* f_w_h1, double* virial, double* energy, double* dh_dl);

/* Sets DYN_PAIR_ALCH on the installed pairs as setup_pairs does for the
 * alchemical molecule (src/non_bonded.rs:581-612) when that molecule is the
 * atoms [atom_begin, atom_end): atom-atom pairs with exactly one end in the
 * range and atom-water pairs whose atom is in it.  Clears it on every other
 * pair; an empty range clears all.  n_marked (may be NULL) receives the
 * number of marked pairs. */
int dyn_nb_mark_alch(dyn_nb_t h, uint32_t atom_begin, uint32_t atom_end, uint64_t* n_marked);

/* Releases everything dyn_nb_create allocated. */
int dyn_nb_destroy(dyn_nb_t h);

/* Largest n_dyn + 4*n_water that dyn_nb_forces_static accepts. */
#define DYN_NB_STATIC_MAX_SITES 131072u

/* No counterpart in the reference.  The pair-force evaluation of
 * dyn_nb_forces for callers that must not allocate device memory (a host
 * framework that owns every device buffer through its own pool, or code
 * running where a cudaMalloc could block or fail): no handle, every array
 * is a DEVICE pointer owned by the caller, and the call allocates nothing
 * (no cudaMalloc / cudaFree / allocating library routine).
 *   Inputs: positions as in dyn_nb_forces (float [3*n] per body); the flat
 *   pair list in the unpacked form of dyn_nb_set_pairs (n_pairs entries per
 *   array); cutoff_ewald, alpha_ewald and lj_cutoff as in dyn_nb_create.
 *   Outputs: float64 [3*n] forces per body as in dyn_nb_forces, and
 *   scalars[3] = {virial, energy, pairs skipped because of a body code > 4
 *   or an index out of range}.
 * Its scratch (64-bit fixed-point accumulators, block partials) is a
 * fixed-size static device array sized for DYN_NB_STATIC_MAX_SITES sites,
 * about 3 MiB, held on every device that loads the library until exit; a
 * larger system is rejected with DYN_ERR_INVALID.  Every call on a device
 * shares it: calls whose work overlaps on one device (unordered streams)
 * race and give wrong results.  Each call clears what it uses first.  The
 * call is asynchronous on `stream`.  The first call on each device sets it
 * up with that device current: it looks up the scratch's address and loads
 * this entry point's kernels, which is when the CUDA driver (lazy module
 * loading, the default since CUDA 12.2) places the scratch in device memory;
 * so make that first call before reserving the rest of the device and
 * before any stream capture.  Not valid after cudaDeviceReset in the same
 * process (the cached address belongs to the destroyed context). */
int dyn_nb_forces_static(void* stream, uint32_t n_dyn, uint32_t n_water, const float* pos_dyn,
                         const float* pos_w_o, const float* pos_w_m, const float* pos_w_h0,
                         const float* pos_w_h1, uint64_t n_pairs, const uint32_t* tgt,
                         const uint32_t* src, const float* sigma, const float* eps,
                         const float* q_tgt, const float* q_src, const uint8_t* body_tgt,
                         const uint8_t* body_src, const uint8_t* flags,
                         const float cell_extent[3], float cutoff_ewald, float alpha_ewald,
                         float lj_cutoff, uint32_t override_bits, double* f_dyn, double* f_w_o,
                         double* f_w_m, double* f_w_h0, double* f_w_h1, double* scalars);

/* ------------------------------------------------------------------ */
/* Layer 2: device-resident engine (MdState::step)                    */
/* ------------------------------------------------------------------ */

typedef struct dyn_sys_s* dyn_sys_t;

/* Integrator (src/integrate.rs:32-44). */
#define DYN_INTEGRATOR_LANGEVIN_MIDDLE 0u
#define DYN_INTEGRATOR_VERLET_VELOCITY 1u

/* Thermostat for the velocity-Verlet integrator (src/thermostat.rs:258). */
#define DYN_THERMO_NONE 0u
#define DYN_THERMO_CSVR 1u

/* Barostat (src/barostat.rs:300-413). */
#define DYN_BARO_NONE 0u
#define DYN_BARO_CRESCALE 1u

/* dyn_config_t.flags */
/* Add the Ewald exclusion corrections (intra-water, 1-2/1-3 and 1-4 pairs)
 * in float64.  Off = the reference's bookkeeping (no correction, plus its
 * 1-4 vacuum force correction, src/non_bonded.rs:763-790). */
#define DYN_FLAG_EWALD_CORRECTIONS 1u
/* Count water-water short-range energy in the potential energy (the
 * reference omits it, src/non_bonded.rs:335-342). */
#define DYN_FLAG_FULL_ENERGY 2u
/* Remove linear COM motion every com_interval steps (src/com_zero.rs:57). */
#define DYN_FLAG_COM_REMOVAL 4u
/* Recenter the box on the solute every recenter_interval steps
 * (src/barostat.rs:111-137, src/integrate.rs:439-443). */
#define DYN_FLAG_RECENTER 8u
/* Re-establish the water geometry every 1000 steps
 * (src/solvent/opc_settle.rs:202-219, src/integrate.rs:445-449). */
#define DYN_FLAG_RESET_ANGLE 16u
/* RATTLE for the bond-to-hydrogen constraints: SHAKE iterations along the
 * bond vectors at the start of each drift, velocities corrected by the
 * constraint displacement, velocity projection iterated for coupled bonds:
 * a symplectic, energy-conserving constrained integrator.  Off = the
 * reference's lincs_hydrogens + rattle_hydrogens (src/bonded.rs:218-304,
 * src/integrate.rs:498-507), which corrects positions along the current
 * bond vectors and leaves the velocities to one projection; that map is not
 * symplectic and drains energy at a rate proportional to dt. */
#define DYN_FLAG_RATTLE_VELOCITIES 32u

typedef struct {
    float box_lo[3];
    float box_hi[3];
    float coulomb_cutoff;   /* MdConfig.coulomb_cutoff (src/config.rs:100)  */
    float lj_cutoff;        /* MdConfig.lj_cutoff                           */
    float list_buffer;      /* Verlet buffer of the cluster lists (A)       */
    float ewald_alpha;      /* MdConfig.spme_alpha                          */
    uint32_t grid[3];       /* SPME grid; spline order is 4                 */
    uint32_t integrator;    /* DYN_INTEGRATOR_*                             */
    uint32_t thermostat;    /* DYN_THERMO_* (velocity Verlet only)          */
    uint32_t barostat;      /* DYN_BARO_*                                   */
    float temperature;      /* K                                            */
    float langevin_gamma;   /* 1/ps                                         */
    float tau_temp;         /* ps (CSVR)                                    */
    float pressure_bar;     /* C-rescale target                             */
    float tau_pressure;     /* ps                                           */
    float compressibility;  /* 1/bar                                        */
    uint32_t spme_interval; /* recompute SPME every n steps (reference: 2)  */
    uint32_t com_interval;  /* reference: 100                               */
    uint32_t recenter_interval; /* reference: 30                            */
    uint32_t energy_interval;   /* energies every n steps (1 = every step)  */
    uint32_t flags;         /* DYN_FLAG_*                                   */
    uint32_t thermo_dof;    /* degrees of freedom (src/thermostat.rs:220)   */
    uint64_t seed;          /* Philox key for all stochastic terms          */
    uint32_t ww_union_chunk;/* waters per shared-memory chunk of the
                             * water-water kernel; 0 = the largest that lets
                             * three CTAs share an SM (a tuning knob: it changes
                             * how float sums are grouped, so results only
                             * at rounding level)                           */
    uint32_t lincs_order;   /* bond-to-H constraints: projection passes of
                             * HydrogenConstraint::Linear (src/prep.rs:55-78);
                             * 0 = 4 (the reference default)                */
    uint32_t lincs_iter;    /* SHAKE-style correction passes; 0 = 1         */
    float prune_buffer;     /* water-water lists are pruned to molecule pairs
                             * within cutoff + 2 x O-H reach + this (A)
                             * whenever a water has moved half of it since
                             * the last prune; 0 = 0.4 A; >= list_buffer:
                             * pruned only at list rebuilds (a tuning knob:
                             * results change only at rounding level)       */
    /* Alchemical decoupling of the atoms [alch_begin, alch_end) (one
     * molecule, StateAlchemical, src/alchemical.rs:98-121): pairs between
     * them and the rest use soft-core LJ and scaled Coulomb, SPME is
     * evaluated three times and mixed, and dH/dlambda is reported, on the
     * reference's staged schedule (staged_decoupling_schedule,
     * src/alchemical.rs:77-96: Coulomb off over lambda 0..0.5, LJ soft-core
     * decoupled over 0.5..1).  alch_end <= alch_begin: off. */
    uint32_t alch_begin;
    uint32_t alch_end;
    float alch_lambda;      /* 0 = fully coupled, 1 = decoupled             */
    uint32_t spme_brick_cap; /* charged sites per 8^3 SPME grid brick before
                             * the overflow path (global atomics, per-site
                             * gather) takes them; 0 = about twice the mean.
                             * Results do not depend on it (integer sums). */
    uint32_t pair_item_entries; /* list entries per work item of the
                             * water-atom and atom-atom pair kernels (1..32);
                             * 0 = 8.  A tuning knob: results change only at
                             * rounding level.                              */
    uint32_t ww_split;      /* CTAs that share one 32-water group's list
                             * entries in the water-water kernel (1..8);
                             * 0 = automatic: more than 1 only for a system
                             * stepped alone with fewer groups than the GPU
                             * has SMs; batch members get 1.  A tuning knob:
                             * results change only at rounding level.       */
} dyn_config_t;

typedef struct {
    /* non-water atoms (solute + ions), home order */
    uint32_t n_atoms;
    const float* atom_pos;     /* [n_atoms*3] */
    const float* atom_vel;     /* [n_atoms*3] */
    const float* atom_mass;    /* [n_atoms]   */
    const float* atom_q;       /* [n_atoms]   */
    const float* atom_sigma;   /* [n_atoms]   */
    const float* atom_eps;     /* [n_atoms]   */
    const uint8_t* atom_static;/* [n_atoms] or NULL */
    /* rigid OPC waters: O, H0, H1 per molecule */
    uint32_t n_water;
    const float* water_pos;    /* [n_water*9] */
    const float* water_vel;    /* [n_water*9] */
    /* topology (atom indices) */
    uint32_t n_excl;   const uint32_t* excl;     /* [n_excl*2] 1-2, 1-3  */
    uint32_t n_pair14; const uint32_t* pair14;   /* [n_pair14*2]         */
    uint32_t n_bonds;  const uint32_t* bonds;    /* [n_bonds*2]          */
    const float* bond_k; const float* bond_r0;
    uint32_t n_angles; const uint32_t* angles;   /* [n_angles*3]         */
    const float* angle_k; const float* angle_theta0;
    uint32_t n_dihedrals; const uint32_t* dihedrals; /* [n*4], one row per term */
    const float* dihedral_k; const float* dihedral_n; const float* dihedral_phase;
    /* bonds to hydrogen held at constraint_r0 (src/bonded.rs:141-304): each
     * pair is (heavy atom, H) in either order; every H in at most one pair,
     * at most 4 H per heavy atom, no H as the heavy end of another pair */
    uint32_t n_constraints; const uint32_t* constraints; /* [n*2] */
    const float* constraint_r0;
} dyn_system_desc_t;

typedef struct {
    double kinetic;         /* kcal/mol, all sites but M                   */
    double kinetic_trans;   /* solute + water COM KE                       */
    double potential;       /* per the reference or full convention        */
    double e_lj;            /* short-range LJ                              */
    double e_coul_short;    /* erfc real-space Coulomb                     */
    double e_water_water_short; /* with DYN_FLAG_FULL_ENERGY only (else 0)  */
    double e_recip;         /* SPME incl. self term                        */
    double e_corrections;   /* exclusion corrections (corrected mode)     */
    double e_bonded;
    double virial;          /* total virial, kcal/mol                      */
    double virial_short, virial_recip, virial_bonded, virial_constraints;
    double pressure_bar;
    double temperature;
    double box[3];
    uint64_t step;
    uint64_t list_rebuilds;
    uint64_t pairs_in_list;   /* molecule/atom pair slots in the cluster lists */
    double kinetic_rigid;     /* KE of the rigid-body motion of the waters (what the
                               * next rigid drift keeps) + atomic KE of the atoms;
                               * temperature and CSVR use this */
    double pressure_atomic_bar; /* the reference's formula: COM KE with the site
                               * virial (src/barostat.rs:419-431); pressure_bar
                               * uses the molecular virial of the rigid waters */
    uint64_t list_union_max;  /* largest set of j-waters one 32-water group
                               * needed at the last list build */
    double dh_dl;             /* alchemical dH/dlambda, kcal/mol (short-range
                               * cross pairs + SPME cross term), energy steps */
    uint64_t list_prunes;     /* prunes of the water-water lists so far (every
                               * rebuild is followed by one) */
} dyn_energies_t;

/* Creates a resident system (replaces MdState::new's device setup,
 * src/lib.rs:1072-1099, and owns everything MdState::step touches). */
int dyn_sys_create(void* stream, const dyn_config_t* cfg, const dyn_system_desc_t* sys,
                   dyn_sys_t* out);

/* Advances n_steps steps of length dt (ps): MdState::step
 * (src/integrate.rs:72-473) with the configured integrator, fully on the
 * device.  Asynchronous on the handle's stream. */
int dyn_sys_step(dyn_sys_t h, uint32_t n_steps, float dt);

/* One force evaluation at the current coordinates, as
 * reset_f_acc_pe_virial + apply_all_forces (src/lib.rs:1220-1348); writes
 * forces (float64, home order): f_atoms [n_atoms*3], f_water [n_water*12]
 * with sites O, H0, H1, M.  Either pointer may be NULL.  Synchronous. */
int dyn_sys_forces(dyn_sys_t h, double* f_atoms, double* f_water, dyn_energies_t* energies);

/* Current state in home order (any pointer may be NULL).  water_pos and
 * water_vel are [n_water*9] (O, H0, H1); water_m [n_water*3].  Synchronous. */
int dyn_sys_get_state(dyn_sys_t h, float* atom_pos, float* atom_vel, float* water_pos,
                      float* water_vel, float* water_m);

/* Overwrites positions and velocities (home order, NULL = keep). */
int dyn_sys_set_state(dyn_sys_t h, const float* atom_pos, const float* atom_vel,
                      const float* water_pos, const float* water_vel);

/* Energies of the last step that computed them (synchronous). */
int dyn_sys_get_energies(dyn_sys_t h, dyn_energies_t* out);

/* Blocks until the handle's stream is idle; returns DYN_ERR_NONFINITE if the
 * device flagged non-finite coordinates since the last call. */
int dyn_sys_sync(dyn_sys_t h);

int dyn_sys_destroy(dyn_sys_t h);

/* Device memory the system holds (its arrays, PME grids, cuFFT work areas). */
int dyn_sys_memory(dyn_sys_t h, uint64_t* bytes);

/* Drop-in step with the state on the host, as the reference's MdState keeps
 * it (src/integrate.rs:72, README "state lives on the host"): copies the
 * given positions/velocities (home order, NULL = keep the resident ones) to
 * the device, advances n_steps, then copies positions, velocities and
 * energies back (NULL outputs are skipped).  Synchronous.  Host buffers
 * should be page-locked for full copy bandwidth. */
int dyn_sys_step_host(dyn_sys_t h, uint32_t n_steps, float dt, const float* atom_pos_in,
                      const float* atom_vel_in, const float* water_pos_in,
                      const float* water_vel_in, float* atom_pos_out, float* atom_vel_out,
                      float* water_pos_out, float* water_vel_out, dyn_energies_t* energies);

/* Stage timing, the device counterpart of the reference's per-component
 * timers (ComputationTimeSums, src/util.rs:111-180): runs n_steps steps
 * without graphs, with CUDA events between stages on the handle's stream,
 * and writes the mean milliseconds per step of each stage into
 * ms[DYN_STAGES]: [0] first half (kick/drift/thermostat), [1] displacement
 * check, list rebuild and prune, [2] short-range pair kernels, [3] 1-4 and
 * bonded terms, [4] SPME (mean over the steps that ran it), [5] kick,
 * reductions, thermostat/barostat and periodic tasks; the pair stage split
 * into [6] water-water (with the force zeroing and the atoms'
 * cluster-order copy before it), [7] water-atom, [8] atom-atom; the SPME
 * stage (per SPME step, without an alchemical molecule) into [9] spread,
 * [10] FFTs and convolution, [11] gather, [12] corrections. */
#define DYN_STAGES 13
int dyn_sys_stage_times(dyn_sys_t h, uint32_t n_steps, float dt, double* ms);

/* Number of this library's kernels one step launches (library kernels such
 * as cuFFT's are not counted), for the step with SPME (spme != 0) or
 * without, when the step neither rebuilds the lists nor runs a periodic task
 * (COM removal, recentering, reset_angle). */
int dyn_sys_launches_per_step(dyn_sys_t h, int spme, uint32_t* out);

/* Kernels a step adds when it rebuilds the lists (*rebuild, including the
 * prune of the water-water lists that follows every rebuild; a step that
 * only prunes adds 2) and when a periodic task is due (*periodic); in the
 * captured step graph these sit under conditional nodes that the device
 * sets. */
int dyn_sys_launches_conditional(dyn_sys_t h, uint32_t* rebuild, uint32_t* periodic);

/* The pairs the resident engine's pair kernels evaluate at this moment, as
 * written by the last list build or prune: kind 0 water-water molecule pairs
 * (water i, water j; original water indices), kind 1 water-atom (water,
 * atom), kind 2 atom-atom (atom i, atom j).  pairs[2k], pairs[2k+1] form one
 * pair; *n_pairs receives the count (pairs = NULL: count only).  Replaces
 * the reference's inspectable neighbour lists (NeighborsNb,
 * src/neighbors.rs:25-53) for checking that every pair inside the cutoff is
 * covered.  Synchronous; for tests and diagnostics, not the step loop. */
int dyn_sys_list_pairs(dyn_sys_t h, uint32_t kind, uint32_t* pairs, uint64_t capacity, uint64_t* n_pairs);

/* Moves an alchemical system to another lambda (a new window of the
 * thermodynamic integration, set_alchemical_window, src/alchemical.rs). */
int dyn_sys_set_lambda(dyn_sys_t h, float lambda);

/* Replaces the atoms' static flags (1 = held fixed; NULL = none) and the
 * thermostat degrees of freedom (0 = keep), between steps, e.g. to freeze
 * the solute while the solvent relaxes around it (MdState::md_on_solute_only,
 * src/solvent/init.rs:773-805, with mark_solute_static_for_init_relaxation
 * and restore_static_state, :745-762).  The next step rebuilds the lists
 * (pairs of two static atoms are skipped). */
int dyn_sys_set_static(dyn_sys_t h, const uint8_t* atom_static, uint32_t thermo_dof);

/* Steepest-descent energy minimization of the atoms
 * (MdState::minimize_energy, src/minimize_energy.rs:60-260), the
 * reference's algorithm: waters and static atoms fixed, reciprocal-space
 * forces off, each trial moving every atom by F * step / F_max with step =
 * min(alpha F_max, 0.2 A); a trial that does not raise the potential energy
 * is accepted (alpha * 1.2, at most 0.01), one that does is reverted (alpha
 * / 2; stop below 1e-8).  Stops after max_iters accepted steps or when the
 * largest force is at most tolerance (kcal/mol/A; the reference's default
 * is 23.9005).  All decisions are taken on the device; the host only reads
 * a done flag every few trials.  Velocities are kept; forces and
 * accelerations are evaluated again (with the reciprocal part) at the end.
 * *iters (may be NULL): accepted steps; *energy (may be NULL): potential
 * energy of the atom terms without the reciprocal part, kcal/mol.
 * Synchronous; not for a batch member. */
int dyn_sys_minimize(dyn_sys_t h, uint32_t max_iters, float tolerance, uint32_t* iters, double* energy);

/* ------------------------------------------------------------------ */
/* Device-resident snapshots (trajectory output)                      */
/* ------------------------------------------------------------------ */

/* dyn_sys_snapshots fields */
#define DYN_SNAP_VELOCITIES 1u  /* velocities, same layout as positions      */
#define DYN_SNAP_FORCES 2u      /* total force on each atom (float32)        */

/* One recorded frame's scalars (Snapshot / SnapshotEnergyData,
 * src/snapshot.rs:59-220).  Energies are those of the last step that
 * computed them (every energy_interval steps). */
typedef struct {
    uint64_t step;
    double time_ps;
    double kinetic;           /* kcal/mol, as dyn_energies_t.kinetic        */
    double potential;         /* kcal/mol                                   */
    double potential_bonded;  /* kcal/mol (bonded + 1-4)                    */
    double temperature;       /* K                                          */
    double pressure_bar;
    double box_lo[3], box_hi[3];
    double volume;            /* A^3                                        */
    double density;           /* amu / A^3 (src/snapshot.rs:206-211)        */
    double dh_dl;             /* alchemical dH/dlambda, kcal/mol            */
} dyn_frame_t;

/* Device side of MdState::handle_snapshots (src/snapshot.rs:753-833):
 * after every step whose number is a multiple of ratio, after the periodic
 * tasks as in the reference (src/integrate.rs:408-466), the step graph
 * copies the state into a ring of capacity frames in device memory, with
 * no host synchronisation.  A frame holds the positions of every site in
 * home order -- the atoms wrapped into the box, then O, H0, H1 of each
 * water (the reference's DCD layout, src/snapshot.rs:293-313) -- as float
 * [n_sites * 3] with n_sites = n_atoms + 3 * n_water, optionally the
 * velocities (same layout) and the atoms' total forces [n_atoms * 3], and a
 * dyn_frame_t.  ratio = 0 turns recording off and frees the ring.  Resets
 * the ring; not for a batch member. */
int dyn_sys_snapshots(dyn_sys_t h, uint32_t ratio, uint32_t capacity, uint32_t fields);

/* Copies the frames recorded since the last read, oldest first, at most
 * max_frames, into host buffers (pos [n * n_sites * 3]; vel likewise or
 * NULL; force [n * n_atoms * 3] or NULL; frames [n] or NULL), after the
 * work queued on the handle's stream.  *n_read receives the frames copied,
 * *n_lost (may be NULL) the frames overwritten in the ring before they
 * were read.  Host buffers should be page-locked for full bandwidth. */
int dyn_sys_snapshots_read(dyn_sys_t h, uint32_t max_frames, float* pos, float* vel, float* force,
                           dyn_frame_t* frames, uint32_t* n_read, uint64_t* n_lost);

/* ------------------------------------------------------------------ */
/* Batched form: many independent systems, one launch per stage      */
/* ------------------------------------------------------------------ */

typedef struct dyn_batch_s* dyn_batch_t;

/* Creates n resident systems (cfgs[i], systems[i], as dyn_sys_create) that
 * are advanced together: every stage of a step is one kernel launch for all
 * members, with per-member block ranges, and a step is one captured CUDA
 * graph.  Members must share spme_interval and energy_interval; sizes,
 * boxes, grids and integrators may differ.  No counterpart in the reference
 * (it advances one MdState per call, src/integrate.rs:72). */
int dyn_batch_create(void* stream, uint32_t n, const dyn_config_t* cfgs,
                     const dyn_system_desc_t* systems, dyn_batch_t* out);

/* Advances every member n_steps steps of length dt (asynchronous). */
int dyn_batch_step(dyn_batch_t b, uint32_t n_steps, float dt);

/* Number of members. */
int dyn_batch_size(dyn_batch_t b, uint32_t* n);

/* Handle of member i for dyn_sys_get_state / get_energies / set_state /
 * forces / step.  Owned by the batch: do not destroy it. */
int dyn_batch_member(dyn_batch_t b, uint32_t i, dyn_sys_t* out);

/* Waits for the batch stream; returns the first member's device-side error
 * (DYN_ERR_NONFINITE, DYN_ERR_TIMEOUT, capacity overflow), if any. */
int dyn_batch_sync(dyn_batch_t b);

/* Batched kernel launches of one step (spme != 0: a step with SPME):
 * *fixed every step, *rebuild more on a step that rebuilds any member's
 * lists, *periodic more on a step with a periodic task.  cuFFT's kernels
 * (one R2C and one C2R per member on SPME steps) are not counted. */
int dyn_batch_launches(dyn_batch_t b, int spme, uint32_t* fixed, uint32_t* rebuild,
                       uint32_t* periodic);

/* Continuous batching: adds a member (as dyn_sys_create, on the batch
 * stream) between steps; *index receives its position.  A member joins only
 * at a batch step that is a multiple of the SPME and energy intervals, so
 * that its schedule, counted from its own step 0, is the one it would have
 * alone.  n = 0 in dyn_batch_create makes an empty batch to add to. */
int dyn_batch_add(dyn_batch_t b, const dyn_config_t* cfg, const dyn_system_desc_t* system,
                  uint32_t* index);

/* Removes (and destroys) member i between steps; later members move down by
 * one index. */
int dyn_batch_remove(dyn_batch_t b, uint32_t i);

/* Layout of a batch's packed host state: member i's block starts at
 * offsets[i] floats and holds atom_pos [na][3], atom_vel [na][3],
 * water_pos [nw][3][3] and water_vel [nw][3][3] (home order, the arrays
 * dyn_sys_step_host takes); offsets[n] is the total.  offsets holds n + 1
 * entries.  The layout changes with dyn_batch_add / dyn_batch_remove. */
int dyn_batch_state_layout(dyn_batch_t b, uint64_t* offsets);

/* A page-locked host area of the packed size, owned by the batch (freed by
 * dyn_batch_destroy; reallocated, and the old pointer invalid, when a later
 * call finds the batch has grown).  *n_floats receives the packed size. */
int dyn_batch_host_buffer(dyn_batch_t b, float** buf, uint64_t* n_floats);

/* Batch-wide drop-in step with the states on the host (dyn_sys_step_host
 * for every member at once): one host->device copy of the packed state
 * (state_in; NULL keeps the resident states), one launch that scatters it
 * to the members, n_steps batch steps, one launch that gathers positions,
 * velocities and every member's scalars, one device->host copy into
 * state_out (NULL skips it) and one of the scalars; energies[i] receives
 * member i's energies (NULL skips them).  state_in may equal state_out.
 * Synchronous; returns the first member's device-side error, if any.
 * Host buffers should be page-locked (dyn_batch_host_buffer) for full copy
 * bandwidth.  No counterpart in the reference (src/integrate.rs:72 steps
 * one MdState whose state lives on the host). */
int dyn_batch_step_host(dyn_batch_t b, uint32_t n_steps, float dt, const float* state_in,
                        float* state_out, dyn_energies_t* energies);

/* Device memory the batch holds (members, block maps, views), in bytes. */
int dyn_batch_memory(dyn_batch_t b, uint64_t* bytes);

/* Releases the batch and all its members. */
int dyn_batch_destroy(dyn_batch_t b);

#ifdef __cplusplus
}
#endif

#endif /* DYNB200_H */
