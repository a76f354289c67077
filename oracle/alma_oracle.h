/* TEST INFRASTRUCTURE — the oracle, a plain-C FP64 restatement of the
 * reference ALMA nonbonded-energy path (noira-913/Protein-Structure-Analysis,
 * src/physics_engine.cpp).  Only the test suite, the smoke check and the
 * CPU-baseline leg of bench.py load it, and only as a checker / baseline;
 * the product never links it.
 *
 * Parity pin: tests/test_oracle_golden.py checks every function here
 * against golden vectors produced by the reference engine itself
 * (oracle/_ref, built from the reference sources by oracle/Makefile;
 * generator: tests/golden/make_golden.py).
 *
 * Conventions: coordinates are xyz[3*i+k] (FP64, Å); neighbor lists are
 * CSR (row_ptr[n+1], cols[]) holding, for row i, the j > i of the
 * reference's cell-scan order.
 */
#ifndef ALMA_ORACLE_H
#define ALMA_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Flat topology, as the reference's BondTopology exports it
 * (physics_engine.cpp:3746-3841): exclusion CSR (excl[i] = sorted j > i),
 * dihedral records (a,b,c,d) with CSR Fourier terms, disulfide pairs. */
typedef struct {
    int n;
    const int64_t *excl_ptr;   /* n+1 */
    const int32_t *excl_cols;
    int ndih;
    const int32_t *dih_abcd;   /* 4*ndih */
    const int32_t *term_off;   /* ndih+1 */
    const double *term_v2;
    const int32_t *term_n;
    const double *term_gamma;
    int nss;
    const int32_t *ss;         /* 2*nss, i < j */
} or_topo;

/* Neighbor list (physics_engine.cpp:293-342).  Returns the pair count, or
 * -count when cap is too small (row_ptr is still filled). */
int64_t or_nl_build(int n, const double *xyz, int64_t *row_ptr, int32_t *cols, int64_t cap);

/* Max-drift test against the positions at the last build (:345-351). */
int or_needs_rebuild(int n, const double *xyz, const double *ref_xyz);

/* HCT pair integral (:2007-2011). */
double or_hct(double r, double r2, double ri, double rj);

/* Born radii, symmetric over the half list (:2024-2039). */
void or_born_radii(int n, const double *xyz, const double *radius, const int64_t *row_ptr,
                   const int32_t *cols, double *a);

/* Half-list Born radius of one atom (:2043-2051). */
void or_update_born(int idx, const double *xyz, const double *radius, const int64_t *row_ptr,
                    const int32_t *cols, double *a);

/* SASA nonpolar term, order dependent (:2068-2083).  sa_out may be NULL;
 * otherwise receives each atom's clamped area max(0, sa). */
double or_sasa(int n, const double *xyz, const double *radius, const int64_t *row_ptr,
               const int32_t *cols, double *sa_out);

/* Pair energy DH + GB + LJ + capped hard core (:2148-2164); p = {x,y,z,q,R*,eps}. */
double or_pair_e(const double *pi, const double *pj, double ai, double aj);

int or_is_excluded(const or_topo *t, int i, int j);                      /* :1700-1705 */
double or_dihedral_angle(const double *xyz, int a, int b, int c, int d); /* :1871-1887 */
double or_dihedral_e(const double *xyz, const or_topo *t);               /* :1912-1921 */
double or_ss_e(const double *xyz, const or_topo *t);                     /* :1965-1974 */

/* Total energy (:2205-2234).  t may be NULL (calculate_potential without
 * topology).  terms[5] = {sasa, dihedral, disulfide, pair sum, total}. */
double or_energy(int n, const double *xyz, const double *q, const double *radius,
                 const double *eps, const int64_t *row_ptr, const int32_t *cols,
                 const double *a, const or_topo *t, double *terms);

/* calculate_potential (:2242-2248): NL build + Born radii + total energy. */
double or_calculate_potential(int n, const double *xyz, const double *q, const double *radius,
                              const double *eps, const or_topo *t, double *terms);

/* One proposal's ΔE (try_torsion :2328-2399, try_crankshaft :2407-2501,
 * concerted sidechain :2798-2878).  The move is `nrot` rigid rotations
 * applied in order; rotation k turns atoms rot_idx[rot_ptr[k]..rot_ptr[k+1])
 * by rot_delta[k] about the axis from atom rot_axis[2k] to rot_axis[2k+1],
 * the axis taken from the coordinates current at that point.  group[n]:
 * 0 = fixed, g > 0 = moving group g; a pair is a cross pair when the groups
 * differ (the reference's in_side / side_group test).  Born radii of every
 * moved atom are refreshed by the half-list update (P4 semantics).
 * xyz and a are the state before the move and are not modified; the
 * proposed coordinates / radii go to new_xyz / new_a (may be NULL).
 * terms[4] = {Δcross, Δsasa, Δdihedral, Δdisulfide}.  Returns ΔE, or NaN
 * for a degenerate proposal (zero-length axis). */
double or_move_dE(int n, const double *xyz, const double *q, const double *radius,
                  const double *eps, const int64_t *row_ptr, const int32_t *cols,
                  const double *a, const or_topo *t, int nrot, const int32_t *rot_axis,
                  const double *rot_delta, const int64_t *rot_ptr, const int32_t *rot_idx,
                  const int8_t *group, double *terms, double *new_xyz, double *new_a);

/* ---- Monte Carlo driver ------------------------------------------------------
 * Restates the proposal loop of generate_ensemble / run_landscape_*
 * (physics_engine.cpp:2273-2543, :2557-2921) with the move draws taken
 * from Philox4x32-10 (counter = step, key = seed and system) instead of
 * mt19937, so a run is reproducible and comparable draw for draw with the
 * device engine's alma_mc_run.  Layout of the state matches AlmaChainState. */
typedef struct {
    double cur_max, energy, temperature;
    int64_t step, n_proposed, n_accepted, n_rebuild;
    int32_t acc_win, tot_win, need_rebuild, pad;
} or_mc_state;

typedef struct {
    uint64_t seed;
    int policy, tune_freq;
    double target_lo, target_hi, scale_up, scale_down, angle_max, angle_min;
    double sidechain_mult, crank_prob, concerted_prob, fixed_delta;
    int nset;              /* > 0: torsion moves drawn from moveset[0..nset) */
    const int32_t *moveset;
} or_mc_cfg;

typedef struct {
    int n;
    double *xyz;           /* [3n], updated in place */
    const double *q, *radius, *eps;
    double *born;          /* [n], updated in place */
    const or_topo *topo;
    int nrb;
    const int32_t *rb_ij, *rb_kind;
    const double *rb_scale;
    const int64_t *side_ptr;   /* [nrb+1] full j-sides, sorted */
    const int32_t *side_idx;
    int ncp;
    const int32_t *cp;         /* [2 ncp] (phi, psi) rot-bond indices */
    int ncsp;
    const int32_t *csp;        /* [2 ncsp] */
    int sys_index;             /* the system number used in the RNG key */
} or_mc_sys;

/* Advances the chain to step_limit.  Builds the neighbor list, Born radii
 * and energy on entry (as a chain starts, :2288-2292) and again whenever
 * the drift flag is set at the start of a step (:2506-2510). */
void or_mc_run(or_mc_sys *sys, const or_mc_cfg *cfg, or_mc_state *st, int64_t step_limit);

/* Philox4x32-10 block (out[4]). */
void or_philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1, uint32_t *out);

/* Rodrigues rotation of one point (:1848-1862). */
void or_rodrigues(double *p, const double *o, const double *u, double c, double s);

#ifdef __cplusplus
}
#endif
#endif
