/*
 * alma_b200.h — C ABI of the B200-native ALMA nonbonded-energy / MC-ΔE engine.
 *
 * Plain pointers and sizes only.  Every device pointer is caller-allocated
 * device memory; every call is asynchronous on the given CUDA stream
 * (passed as void*, a cudaStream_t) unless its comment says otherwise.
 * Every entry point returns 0 on success or a negative ALMA_E* code;
 * alma_last_error() returns a thread-local message for the last failure.
 *
 * Reference interfaces replaced (noira-913/Protein-Structure-Analysis):
 *   src/physics_engine.cpp      — CPU engine, module `protein_physics`
 *   src/physics_engine_cuda.cu  — CUDA engine, module `protein_physics_cuda`
 * The reference binds these through pybind11 (physics_engine.cpp:3692-3888,
 * physics_engine_cuda.cu:1287-1396); the Python package protein_physics_b200
 * re-exposes the same Python surface over this ABI.
 *
 * Batched layout: a batch holds `nsys` independent systems (chains or
 * replicas) concatenated atom-wise; atom_off[nsys+1] gives each system's
 * first atom.  All atom indices in topology / neighbor arrays are global
 * (batch) indices.  A single chain is a batch with nsys = 1.
 */
#ifndef ALMA_B200_H
#define ALMA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ALMA_ABI_VERSION 1

enum {
    ALMA_OK = 0,
    ALMA_EINVAL = -1,    /* bad argument (null pointer, size, index)       */
    ALMA_ECUDA = -2,     /* CUDA runtime error                             */
    ALMA_ECAPACITY = -3, /* caller buffer too small (see the call's doc)   */
    ALMA_EDEVICE = -4,   /* device-side status flag set (see alma_status)  */
    ALMA_ENODEV = -5     /* no usable sm_100 device                        */
};

/* Precision of the pair arithmetic.  Accumulations (Born-radius integral,
 * energies, ΔE) and the Metropolis test are FP64 in both modes; pair
 * distances and the 12 Å / 14 Å cutoff tests are always FP64. */
enum { ALMA_PREC_MIXED = 0, ALMA_PREC_FP64 = 1 };

/* Device status word bits (AlmaBatch.status): sticky error flags. */
enum {
    ALMA_ST_NL_OVERFLOW = 1,    /* neighbor list exceeded its capacity       */
    ALMA_ST_CELL_OVERFLOW = 2,  /* cell grid exceeded its capacity           */
    ALMA_ST_BAD_INDEX = 4,      /* topology index out of range               */
    ALMA_ST_NONFINITE = 8,      /* non-finite coordinate or energy seen      */
    ALMA_ST_SPEC_ABORT = 16     /* a team of a speculative MC round waited   */
                                /* past its limit; the chain state of that   */
                                /* launch was not written                    */
};

/* Energy-model constants (physics_engine.cpp:181-196).  Passed by value;
 * alma_params_reference() fills the reference preset. */
typedef struct {
    double coulomb, eps_water, eps_prot, kappa;
    double gamma_sa, beta_sa, probe_r;
    double pair_cut2;          /* 12 Å squared: pair terms use r² <= this   */
    double nl_rcut2;           /* 14 Å squared: list membership r² < this   */
    double half_skin2;         /* drift² that triggers a rebuild            */
    double hard_scale, hard_cap, hard_frac;
    double k_ss, r0_ss;
} AlmaParams;

/* A batch of systems resident on the device (all pointers device memory). */
typedef struct {
    int32_t nsys;
    int32_t natoms;
    const int32_t *atom_off; /* [nsys+1]                                    */
    double *xyz;             /* [natoms*4] FP64 x,y,z,(unused)              */
    const float *prm;        /* [natoms*4] charge, R*, epsilon, (unused)    */
    const double *prm64;     /* [natoms*4] charge, R*, epsilon, (unused)    */
    double *born;            /* [natoms] effective Born radii               */
    uint32_t *status;        /* [1] sticky ALMA_ST_* flags                  */
    double *sasa;            /* [natoms] optional (NULL: none): per-atom    */
                             /* SASA term gamma*max(0, sa_i) of the current */
                             /* coordinates.  alma_energy fills it for the  */
                             /* systems it evaluates; the move / MC kernels */
                             /* read it instead of recomputing the old SASA */
                             /* and keep it current on commit.  Pass NULL   */
                             /* after changing coordinates any other way.   */
} AlmaBatch;

/* Flat topology of the batch (physics_engine.cpp:3746-3841 exports). */
typedef struct {
    const int64_t *excl_ptr;  /* [natoms+1] 1-2/1-3/SS exclusions, j > i    */
    const int32_t *excl_cols;
    int32_t nrb;              /* rotatable bonds, all systems               */
    const int32_t *rb_off;    /* [nsys+1]                                   */
    const int32_t *rb_ij;     /* [nrb*2] axis atoms                         */
    const int32_t *rb_kind;   /* [nrb] 0 phi, 1 psi, 2 sidechain, 3 fixed   */
    const double *rb_scale;   /* [nrb] lever-arm scale                      */
    const int64_t *side_ptr;  /* [nrb+1] j-side: explicit atoms, sorted     */
    const int32_t *side_idx;
    const int32_t *side_lo;   /* [nrb] j-side: plus the atom range [lo, hi) */
    const int32_t *side_hi;
    int32_t ndih;
    const int32_t *dih_off;   /* [nsys+1]                                   */
    const int32_t *dih_abcd;  /* [ndih*4]                                   */
    const int32_t *term_off;  /* [ndih+1]                                   */
    const double *term_v2;
    const int32_t *term_n;
    const double *term_gamma;
    int32_t nss;
    const int32_t *ss_off;    /* [nsys+1]                                   */
    const int32_t *ss_ij;     /* [nss*2]                                    */
    int32_t ncp;
    const int32_t *cp_off;    /* [nsys+1] crankshaft pairs                  */
    const int32_t *cp;        /* [ncp*2] (phi rot bond, psi rot bond)        */
    int32_t ncsp;
    const int32_t *csp_off;   /* [nsys+1] concerted sidechain pairs         */
    const int32_t *csp;       /* [ncsp*2]                                   */
    const uint32_t *excl_win; /* optional [4*natoms] exclusion windows from */
                              /* alma_excl_window (the list build then tests */
                              /* one bit per pair instead of searching the  */
                              /* CSR rows); NULL: CSR search                 */
} AlmaTopo;

/* Exclusion window of every atom from the CSR exclusions (excl_ptr,
 * excl_cols: rows of j > i, global atom indices): win[4*i .. 4*i+3] is a
 * 128-bit mask whose bit d + 64 is set when atoms i and i + d are excluded
 * (0 < |d| < 64); bit 64 (d = 0) is set when atom i has an exclusion
 * partner outside the window, which the CSR rows then decide; bit 0 is
 * unused.
 * Fills win (device, 16 bytes per atom) on `stream`.  Exclusions depend on
 * the topology only: build once, point AlmaTopo.excl_win at it.  Replaces
 * the per-pair search of BondTopology::is_excluded (physics_engine.cpp:
 * 1700-1705) in the list build; the exclusion flags are the same. */
int alma_excl_window(const int64_t *excl_ptr, const int32_t *excl_cols, int32_t natoms, uint32_t *win,
                     void *stream);

/* Neighbor list: for every atom a full row (all j != i with r² < 14²) and
 * a half row (j > i), both in the reference's cell-scan order
 * (NeighborList::build, physics_engine.cpp:293-342).  Row i occupies
 * cols[ptr[i] .. ptr[i]+len[i]).  Each system owns the region
 * [base[s], base[s+1]) of the column arrays, so one system can be rebuilt
 * without touching the others.  Column entries carry the exclusion flag in
 * bit 31 (atom index = entry & 0x7fffffff).  Optional short rows (sfull,
 * shalf; set sfull_cols = NULL to skip them) are the order-preserving
 * sub-rows of the pairs within SASA reach plus the skin at build time
 * (r < R*_i + R*_j + 2 probe + skin): while every atom stays within half the
 * skin of its build position no other pair can come within SASA reach, so
 * the move kernels walk these instead.  need[4*s + k] receives the entry
 * counts (k: full, half, short full, short half) of system s at its last
 * build; when a count exceeds its region, the rows of that system are
 * incomplete and ALMA_ST_NL_OVERFLOW is raised (regrow the regions from
 * need[] and build again).  Rows lie in their system's region in no
 * particular order: read them through ptr/len. */
typedef struct {
    int64_t *full_ptr;        /* [natoms] */
    int32_t *full_len;        /* [natoms] */
    uint32_t *full_cols;      /* [full_base[nsys]] */
    const int64_t *full_base; /* [nsys+1] */
    int64_t *half_ptr;        /* [natoms] */
    int32_t *half_len;        /* [natoms] */
    uint32_t *half_cols;      /* [half_base[nsys]] */
    const int64_t *half_base; /* [nsys+1] */
    double *ref_xyz;          /* [natoms*4] positions at the last build     */
    int64_t *need;            /* [nsys*4]                                   */
    int64_t *sfull_ptr;       /* [natoms] short rows (optional)             */
    int32_t *sfull_len;
    uint32_t *sfull_cols;
    const int64_t *sfull_base;
    int64_t *shalf_ptr;
    int32_t *shalf_len;
    uint32_t *shalf_cols;
    const int64_t *shalf_base;
    int32_t *full_span;       /* [natoms*2] optional (NULL: not kept): the
                               * smallest and largest atom index in each full
                               * row at the last build (INT32_MAX, -1 for an
                               * empty row).  A moved atom whose span lies in
                               * its side's atom range has no neighbour that
                               * stays behind, so the move kernels skip its
                               * cross-pair and SASA-mark scans. */
} AlmaNL;

/* ---- library ------------------------------------------------------------ */
int alma_abi_version(void);
const char *alma_last_error(void);
/* Kernel launches the library has issued since load (all threads). */
long long alma_launch_count(void);
/* Reference preset (P1: 0.6 sigma smooth capped hard core, gamma 0.00542). */
void alma_params_reference(AlmaParams *p);
/* Bytes of device workspace alma_nl_build needs for a batch. */
size_t alma_nl_workspace_bytes(int32_t nsys, int32_t natoms, int64_t max_cells);

/* ---- host topology helper ------------------------------------------------ */
/* j_side for each bond (bi, bj): atoms reached by a DFS from bj that never
 * enters bi, listed in DFS visiting order (BondTopology::j_side,
 * physics_engine.cpp:1731-1745).  Host memory.  side_ptr[nb+1]; returns
 * ALMA_ECAPACITY when cap < total (side_ptr still filled). */
int alma_topo_sides(int32_t n, const int64_t *adj_ptr, const int32_t *adj_idx, int32_t nb,
                    const int32_t *bonds, int64_t *side_ptr, int32_t *side_idx, int64_t cap);
/* The same sets in the engine's compact form: the longest run of
 * consecutive atom indices [lo[b], hi[b]) plus the other atoms, sorted, in
 * (ex_ptr[nb+1], ex_idx); count[b] = set size.  ALMA_ECAPACITY when
 * ex_cap < total explicit atoms (ex_ptr still filled). */
int alma_topo_sides_compact(int32_t n, const int64_t *adj_ptr, const int32_t *adj_idx, int32_t nb,
                            const int32_t *bonds, int32_t *lo, int32_t *hi, int64_t *count,
                            int64_t *ex_ptr, int32_t *ex_idx, int64_t ex_cap);

/* ---- device kernels ------------------------------------------------------ */
/* Neighbor list for every system of the batch (replaces
 * NeighborList::build, physics_engine.cpp:293-342).  p: probe radius and
 * skin of the short rows (NULL: reference preset).  sys_mask: device
 * uint8[nsys]; only systems with a nonzero entry are rebuilt (NULL: all).
 * workspace: device scratch of alma_nl_workspace_bytes(nsys, natoms,
 * max_cells) bytes. */
int alma_nl_build(const AlmaBatch *b, const AlmaTopo *t, AlmaNL *nl, const AlmaParams *p,
                  const uint8_t *sys_mask, void *workspace, int64_t max_cells, void *stream);

/* Effective Born radii over the full rows (replaces born_radii,
 * physics_engine.cpp:2024-2039, and born_sum/born_finalize kernels,
 * physics_engine_cuda.cu:537-578).  Writes b->born for the systems with a
 * nonzero sys_mask entry (device uint8[nsys]; NULL: all). */
int alma_born_radii(const AlmaBatch *b, const AlmaNL *nl, const AlmaParams *p, int prec,
                    const uint8_t *sys_mask, void *stream);

/* Per-system energy terms (replaces total_e / calculate_potential,
 * physics_engine.cpp:2205-2248, and pair_energy_kernel,
 * physics_engine_cuda.cu:587-617).  terms: device double[nsys*5] =
 * {sasa, dihedral, disulfide, pair sum, total} per system.  t may be NULL
 * (no exclusions / dihedrals / disulfides).  sys_mask as above (terms of
 * other systems are left untouched).  atom_e: device double[natoms*2]
 * scratch (per-atom pair and SASA contributions). */
int alma_energy(const AlmaBatch *b, const AlmaTopo *t, const AlmaNL *nl, const AlmaParams *p,
                int prec, const uint8_t *sys_mask, double *atom_e, double *terms, void *stream);

/* Analytic gradient of the total energy (the backward of alma_energy; the
 * reference has no gradient: this is the derivative of total_e,
 * physics_engine.cpp:2205-2234, through born_radii :2024-2039, pair_e
 * :2148-2164, sasa_nonpolar :2068-2083, dihedral_e :1912-1921 and ss_e
 * :1965-1974).  grad: device double[natoms*4], dE/dx per atom (x, y, z, 0)
 * in kcal/mol/Å.  b->born must hold the radii of the current coordinates
 * (alma_born_radii or alma_energy) and nl a list valid for them; the HCT
 * derivatives are recomputed, not stored.  Deterministic: every sum has a
 * fixed order (pair and Born parts gathered over full rows, SASA and bonded
 * parts added as 64-bit fixed point, 2^-32 kcal/mol/Å).  workspace:
 * alma_forces_workspace_bytes(natoms) device bytes.  sys_mask as above. */
size_t alma_forces_workspace_bytes(int32_t natoms);
int alma_forces(const AlmaBatch *b, const AlmaTopo *t, const AlmaNL *nl, const AlmaParams *p, int prec,
                const uint8_t *sys_mask, void *workspace, double *grad, void *stream);

/* ---- torsion space: gradient, all-bond moves, gradient-guided sampling ----
 * The reference moves one or two torsions per proposal (rodrigues,
 * physics_engine.cpp:1848-1862); these entry points have no reference
 * counterpart: they are the torsion-space side of the analytic gradient
 * (descent minimisation, Langevin / MALA proposals). */

/* Nesting of the rotatable bonds' j-sides, local indices per system (each
 * system's rows start at its own bond / atom offset).  Built on the host by
 * alma_torsion_tree, uploaded by the caller. */
typedef struct {
    const int32_t *rb_parent; /* [nrb] innermost bond whose j-side holds this bond's axis atom i, -1 none */
    const int32_t *atom_rb;   /* [natoms] innermost bond whose j-side holds the atom, -1 none             */
} AlmaTorsionTree;

/* Host: the tree of one system from its j-sides (local atom indices:
 * side_ptr [nrb+1] / side_idx explicit atoms, [side_lo, side_hi) range).
 * ALMA_EINVAL when the j-sides are not nested (a ring in the bond graph). */
int alma_torsion_tree(int32_t natoms, int32_t nrb, const int32_t *rb_ij, const int64_t *side_ptr,
                      const int32_t *side_idx, const int32_t *side_lo, const int32_t *side_hi, int32_t *rb_parent,
                      int32_t *atom_rb);
size_t alma_torsion_workspace_bytes(int32_t natoms, int32_t nsys, int32_t nrb);
/* gtheta[k] = dE/dθ_k = u_k · Σ_{m in j-side k} (x_m - x_i) × grad_m for every
 * rotatable bond (grad: device double[natoms*4], e.g. from alma_forces). */
int alma_torsion_grad(const AlmaBatch *b, const AlmaTopo *t, const double *grad, const uint8_t *sys_mask,
                      void *workspace, double *gtheta, void *stream);
/* Turns every rotatable bond k by delta[k] radians at once (the same
 * structure as the reference's moves applied one after another with axes
 * from the updated coordinates).  Coordinates change in place; Born radii
 * and neighbor list are the caller's to refresh. */
int alma_torsion_apply(const AlmaBatch *b, const AlmaTopo *t, const AlmaTorsionTree *tree, const double *delta,
                       const uint8_t *sys_mask, void *workspace, void *stream);

/* Per-system state of the Langevin (MALA) torsion sampler (64 bytes). */
typedef struct {
    double energy;            /* energy of the current state (kcal/mol)     */
    double beta;              /* 1/T, T in kcal/mol                         */
    double scale;             /* multiplies every bond's sigma (adapted)    */
    double log_alpha;         /* log acceptance ratio of the last proposal  */
    int64_t step;             /* proposals made (the RNG counter)           */
    int64_t n_proposed, n_accepted;
    int32_t acc_win, tot_win; /* adaptation window                          */
} AlmaMalaState;

typedef struct {
    uint64_t seed;            /* Philox key                                  */
    double drift_clip;        /* drift clipped to ±drift_clip·σ per bond     */
    int32_t tune_freq;        /* proposals per adaptation window, 0 = off    */
    int32_t pad;
    double target_lo, target_hi;  /* acceptance band of the window           */
    double scale_up, scale_down;  /* scale factors outside the band          */
    double scale_min, scale_max;
} AlmaMalaConfig;

/* delta[k] = clip(-½ σ_k² β ∇_θE_k, ±drift_clip σ_k) + σ_k ξ_k with
 * σ_k = state.scale × sigma[k], ξ ~ N(0,1) (Philox, keyed by seed, system,
 * state.step, bond); sigma[k] <= 0 keeps bond k fixed.  The truncated drift
 * keeps clash gradients from throwing proposals away. */
int alma_mala_propose(const AlmaTopo *t, int32_t nsys, const double *gtheta, const double *sigma,
                      const AlmaMalaConfig *cfg, const AlmaMalaState *states, const uint8_t *sys_mask,
                      double *delta, void *stream);
/* Metropolis–Hastings test of the proposal (energy terms_new[5s+4],
 * torsion gradients before / after): accept[s], state energy / counters,
 * then the scale adaptation. */
int alma_mala_accept(const AlmaTopo *t, int32_t nsys, const double *delta, const double *g_old, const double *g_new,
                     const double *sigma, const double *terms_new, const AlmaMalaConfig *cfg,
                     const uint8_t *sys_mask, AlmaMalaState *states, uint8_t *accept, void *stream);
/* Rejected systems: xyz, born <- saved copies.  Accepted: g_cur <- g_new
 * (both may be NULL). */
int alma_mala_select(AlmaBatch *b, const AlmaTopo *t, const uint8_t *accept, const uint8_t *sys_mask,
                     const double *xyz_old, const double *born_old, const double *g_new, double *g_cur,
                     void *stream);

/* Ensemble metrics of snapshots resident on the device (replaces
 * compute_mean_dist_matrix and compute_contact_freq_matrix,
 * analysis_ext.cpp:85-170).  coords: device double[n_snaps*n_ca*3];
 * out: device double[n_ca*n_ca], the mean distance (or the fraction of
 * snapshots with distance < cutoff) of every residue pair, 0 on the
 * diagonal.  Each cell sums its snapshots in order. */
int alma_mean_dist_matrix(const double *coords, int32_t n_snaps, int32_t n_ca, double *out, void *stream);
int alma_contact_freq_matrix(const double *coords, int32_t n_snaps, int32_t n_ca, double cutoff, double *out,
                             void *stream);

/* Device scratch for the move / MC kernels: alma_move_scratch_bytes(natoms)
 * bytes, zeroed once by alma_move_scratch_init; every call leaves it zeroed.
 * Calls that share a scratch buffer must not overlap on the GPU. */
size_t alma_move_scratch_bytes(int32_t natoms);
int alma_move_scratch_init(void *scratch, int32_t natoms, void *stream);
/* Cumulative work of the move / MC kernels per system (host out[8*nsys]):
 * out[4s..4s+3] = {pair-term evaluations, hct evaluations, SASA neighbour
 * visits, moved atoms}; out[4*nsys + 4s ..] = SM cycles spent in the four
 * ΔE phases (copy+rotate, Born+marks, pairs+SASA, reduction).
 * Synchronises the stream. */
int alma_move_counters(const void *scratch, int32_t natoms, int32_t nsys, unsigned long long *out,
                       void *stream);

/* ΔE of one proposal per system, replayed for a given move (the ΔE core of
 * try_torsion / try_crankshaft / the concerted sidechain move,
 * physics_engine.cpp:2328-2501, :2798-2878; cross_pair_energy_kernel,
 * physics_engine_cuda.cu:629-661).  move_kind[s]: 0 torsion (move_a =
 * rot-bond index within system s), 1 crankshaft (move_a = crank-pair
 * index), 2 concerted sidechain (move_a = pair index), -1 none.
 * move_delta[2*s+0..1]: angle(s) in radians (the second is used by kind 2).
 * Outputs per system: dE[s], dterms[4*s..] = {Δcross, Δsasa, Δdih, Δss};
 * NaN for a degenerate proposal (empty side, zero-length axis).  When
 * apply != 0 the proposal is committed (coordinates and Born radii of the
 * moved atoms), as an accepted Metropolis step would.  Device arrays. */
int alma_move_dE(const AlmaBatch *b, const AlmaTopo *t, const AlmaNL *nl, const AlmaParams *p,
                 int prec, void *scratch, const int32_t *move_kind, const int32_t *move_a,
                 const double *move_delta, int apply, double *dE, double *dterms, void *stream);

/* alma_move_dE without caller scratch — no counterpart in the reference.
 *
 * For callers that cannot allocate device memory themselves: hosts whose
 * own allocator already owns the GPU's memory and forbids other
 * allocations, and latency-critical sampling loops that cannot pay for
 * cudaMalloc's implicit device-wide synchronisation.  Such callers still
 * pass their own input and output buffers; only the scratch moves into the
 * library.
 *
 * Same arguments and results as alma_move_dE, minus `scratch`.  The
 * scratch is a static area built into the library of
 * ALMA_NOALLOC_SCRATCH_BYTES (5 MiB), which every GPU that loads the
 * library holds until the process exits; batches up to
 * ALMA_NOALLOC_MAX_ATOMS atoms fit, larger ones are rejected with
 * ALMA_EINVAL and a message.  No call allocates or frees device memory.
 * The first call on each device looks up the area's device address (with
 * that device current); make that first call before any stream capture.
 * The address is cached per device under the context it was looked up in;
 * a call under another context (after cudaDeviceReset re-created the
 * primary context) looks it up again.  A rejected call (bad size, null
 * buffer) returns before touching the area.
 * All calls on a device share the one area: calls whose kernels overlap on
 * the GPU (two streams, two host threads) race and corrupt each other's
 * results — serialise them.  Each call clears the part it uses before
 * running. */
#define ALMA_NOALLOC_SCRATCH_BYTES (5u << 20)
#define ALMA_NOALLOC_MAX_ATOMS 16384
size_t alma_move_noalloc_capacity_bytes(void);
int alma_move_dE_noalloc(const AlmaBatch *b, const AlmaTopo *t, const AlmaNL *nl, const AlmaParams *p,
                         int prec, const int32_t *move_kind, const int32_t *move_a,
                         const double *move_delta, int apply, double *dE, double *dterms, void *stream);

/* ---- device Monte Carlo ------------------------------------------------- */
/* Proposal policy (the MC loop of generate_ensemble / run_landscape_*,
 * physics_engine.cpp:2273-2543, :2557-3270). */
typedef struct {
    uint64_t seed;            /* Philox key; every run reproducible from it  */
    int32_t policy;           /* 0 generate_ensemble, 1 landscape, 2 torsion */
    int32_t tune_freq;        /* 200; 0 disables the cur_max adaptation      */
    double target_lo, target_hi;  /* 0.28, 0.52                              */
    double scale_up, scale_down;  /* 1.06, 0.94                              */
    double angle_max, angle_min;  /* 0.5, 0.004 rad                          */
    double sidechain_mult;    /* 2.5                                         */
    double crank_prob;        /* 0.25                                        */
    double concerted_prob;    /* 0.15 (policy 1)                             */
    double fixed_delta;       /* > 0: angles ~ U(-fixed_delta, fixed_delta)  */
    const int32_t *moveset_off;   /* optional [nsys+1] device: torsion moves */
    const int32_t *moveset;       /* drawn from these local rot-bond indices */
    int32_t threads_per_system;   /* CTA size 256 or 512; 0 = by batch size  */
    int32_t cluster_size;         /* CTAs per system (1,2,4,8,16; 0 = 1): a  */
                                  /* thread-block cluster shares a proposal  */
    int32_t spec_teams;           /* teams (clusters) per system, 0/1 = one: */
                                  /* K > 1 evaluates the next K proposals at */
                                  /* once against the committed state and    */
                                  /* commits the first accepted one — the    */
                                  /* same chain, up to K proposals per round */
                                  /* (scratch: alma_mc_scratch_bytes)        */
    int32_t pad;
    void *rebuild_ws;             /* optional device workspace of             */
                                  /* alma_mc_rebuild_bytes(natoms, nsys): a   */
                                  /* chain that drifts rebuilds its neighbor  */
                                  /* list, Born radii and energy inside the   */
                                  /* persistent kernel (one team); NULL: it   */
                                  /* stops for the host rebuild                */
    const int32_t *sys_order;     /* optional [nsys] device permutation: the  */
                                  /* order in which systems take CTAs (the   */
                                  /* hardware starts CTAs in index order, so */
                                  /* largest-first packs uneven chains onto  */
                                  /* the SMs with the shortest tail); NULL:  */
                                  /* system s on CTA s.  Results do not      */
                                  /* depend on it.                           */
    int32_t launch_systems;       /* > 0 (needs sys_order): only the first   */
                                  /* launch_systems entries of sys_order get */
                                  /* CTAs; the other systems do not advance  */
                                  /* in this launch.  0: every system.  Lets */
                                  /* the last chains of a run take wider     */
                                  /* clusters and more teams                 */
    int32_t pad2;
} AlmaMCConfig;

/* Per-system chain state, device memory, one per system (72 bytes). */
typedef struct {
    double cur_max;           /* adaptive max angle (rad)                    */
    double energy;            /* running energy: last full evaluation + ΣΔE  */
    double temperature;       /* kcal/mol                                    */
    int64_t step;             /* proposals drawn (the RNG counter)           */
    int64_t n_proposed, n_accepted, n_rebuild;
    int32_t acc_win, tot_win; /* adaptation window                           */
    int32_t need_rebuild;     /* set when an accepted move drifted > skin/2  */
    int32_t parity;           /* scratch double-buffer selector (internal)   */
} AlmaChainState;

/* Workspace bytes of the in-kernel rebuild (AlmaMCConfig.rebuild_ws). */
size_t alma_mc_rebuild_bytes(int32_t natoms, int32_t nsys);
/* Scratch bytes of alma_mc_run for spec_teams = teams (zeroed once before
 * first use; teams <= 1: alma_move_scratch_bytes(natoms)). */
size_t alma_mc_scratch_bytes(int32_t natoms, int32_t nsys, int32_t teams);
/* Runs proposals on every system until its state.step reaches step_limit
 * or it needs a neighbor-list rebuild (one CTA per system, no host sync).
 * The caller then rebuilds flagged systems (alma_nl_build + alma_born_radii
 * + alma_energy with their mask), calls alma_mc_after_rebuild, and calls
 * again.  Scratch as for alma_move_dE. */
int alma_mc_run(const AlmaBatch *b, const AlmaTopo *t, const AlmaNL *nl, const AlmaParams *p, int prec,
                void *scratch, const AlmaMCConfig *cfg, AlmaChainState *states, int64_t step_limit,
                void *stream);
/* Self-test of the speculative rounds' bounded cross-team wait: one CTA
 * waits at a barrier that nothing else reaches; after its poll limit (about
 * a second) it raises ALMA_ST_SPEC_ABORT in *status, writes 1 to *aborted
 * and returns.  round_buf: alma_spec_round_bytes() bytes of device memory. */
size_t alma_spec_round_bytes(void);
int alma_spec_wait_selftest(void *round_buf, uint32_t *status, int32_t *aborted, void *stream);

/* state.energy <- terms[5*s+4], need_rebuild <- 0 for masked systems. */
int alma_mc_after_rebuild(AlmaChainState *states, const double *terms, const uint8_t *sys_mask,
                          int32_t nsys, void *stream);

/* Replica exchange between temperature neighbours (parallel tempering; the
 * reference swaps landscape-segment states between Python threads,
 * gui_main.py:1960-2013).  Every replica is a system of the batch;
 * sys_of_temp[t] (device, a permutation) names the system at temperature
 * slot t, slots in ascending temperature.  Round r tries the pairs
 * (t, t+1), t ≡ r mod 2: swap with probability
 * min(1, exp((1/T_a - 1/T_b)(E_a - E_b))), E = terms[5s+4] (fresh energies),
 * T from mc_states.  A swap exchanges the systems' temperatures, cur_max and
 * adaptation windows (and MALA beta / scale when mala_states is not NULL).
 * attempts / accepts: device counters per slot pair [nsys].  nsys <= 2048. */
int alma_replica_exchange(int32_t nsys, const double *terms, AlmaChainState *mc_states, AlmaMalaState *mala_states,
                          int32_t *sys_of_temp, uint64_t seed, int64_t round, unsigned long long *attempts,
                          unsigned long long *accepts, void *stream);

/* Size in bytes of each ABI struct, for bindings that mirror them (ctypes,
 * cgo, JNA) to check their layout against the library's: which = 0
 * AlmaParams, 1 AlmaBatch, 2 AlmaTopo, 3 AlmaNL, 4 AlmaMCConfig,
 * 5 AlmaChainState, 6 AlmaTorsionTree, 7 AlmaMalaState, 8 AlmaMalaConfig;
 * 0 for any other value.  No counterpart in the reference (its binding is
 * pybind11, which checks types at compile time). */
size_t alma_struct_size(int32_t which);

#ifdef __cplusplus
}
#endif
#endif /* ALMA_B200_H */
