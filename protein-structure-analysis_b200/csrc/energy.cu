// Full-structure energy on the device: HCT Born radii, the ordered SASA
// term, the nonbonded pair sum, dihedral and disulfide terms, and a
// deterministic per-system reduction.
//
//   born   : warp per atom over its full row (every j with r² < 14²), FP64
//            accumulation of hct(i<-j) — the same set the reference's
//            symmetric half-list loop adds into sum[i] (physics_engine.cpp
//            :2024-2039), without float atomics.
//   pairs  : warp per atom over its half row, in one pass that also walks
//            the row in order for SASA (:2068-2083 — order dependent, so the
//            32 lanes compute the caps of 32 consecutive entries and the
//            recurrence sa -= min(0.85 sa, cap) is applied lane by lane),
//            and evaluates pair_e (:2148-2164) for non-excluded entries with
//            r² <= 12² (:2223-2232).
//   reduce : one CTA per system — pair and SASA sums in a fixed order, plus
//            the dihedral (:1912-1921) and disulfide (:1965-1974) terms.
#include "energy_core.cuh"

namespace alma {

template <typename R>
__global__ void born_kernel(int natoms, const int32_t *__restrict__ atom_off, int nsys, const uint8_t *__restrict__ mask,
                            const double *__restrict__ xyz, const float *__restrict__ prm,
                            const double *__restrict__ prm64, const int64_t *__restrict__ full_ptr,
                            const int32_t *__restrict__ full_len, const uint32_t *__restrict__ full_cols,
                            double *__restrict__ born) {
    const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= natoms) return;
    if (mask && !mask[sys_of_atom(atom_off, nsys, i)]) return;
    born_atom<R>(i, lane, xyz, prm, prm64, full_ptr, full_len, full_cols, born);
}

// Warp per atom: pair energy and SASA of row i.  atom_e[2*i] = pair sum of
// row i, atom_e[2*i+1] = gamma * max(0, sa_i).  Held to 64 registers (four
// 256-thread blocks per SM): the row gathers are latency bound and need the
// resident warps.
template <typename R>
__global__ void __launch_bounds__(256, 4) pair_sasa_kernel(DevParams P, int natoms, const int32_t *__restrict__ atom_off, int nsys,
                                 const uint8_t *__restrict__ mask, const double *__restrict__ xyz,
                                 const float *__restrict__ prm,
                                 const double *__restrict__ prm64, const double *__restrict__ born,
                                 const int64_t *__restrict__ half_ptr, const int32_t *__restrict__ half_len,
                                 const uint32_t *__restrict__ half_cols, int use_excl, double *__restrict__ atom_e,
                                 double *__restrict__ sasa_out) {
    const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= natoms) return;
    if (mask && !mask[sys_of_atom(atom_off, nsys, i)]) return;
    pair_sasa_atom<R>(P, i, lane, xyz, prm, prm64, born, half_ptr, half_len, half_cols, use_excl, atom_e, sasa_out);
}

// One CTA per system.
__global__ void energy_reduce_kernel(DevParams P, const int32_t *__restrict__ atom_off, const double *__restrict__ xyz,
                                     const double *__restrict__ atom_e, AlmaTopo t, int has_topo,
                                     const uint8_t *__restrict__ mask, double *__restrict__ terms) {
    __shared__ double sm[32];
    const int s = blockIdx.x;
    if (mask && !mask[s]) return;
    const int a0 = atom_off[s], a1 = atom_off[s + 1];
    double ep = 0.0, es = 0.0, ed = 0.0, ess = 0.0;
    for (int i = a0 + threadIdx.x; i < a1; i += blockDim.x) {
        ep += atom_e[2 * (size_t)i];
        es += atom_e[2 * (size_t)i + 1];
    }
    if (has_topo) {
        for (int r = t.dih_off[s] + threadIdx.x; r < t.dih_off[s + 1]; r += blockDim.x)
            ed += dih_record_energy(xyz, t, r);
        for (int k = t.ss_off[s] + threadIdx.x; k < t.ss_off[s + 1]; k += blockDim.x) {
            const double dr = sqrt(dist2(xyz, t.ss_ij[2 * k], t.ss_ij[2 * k + 1])) - P.r0_ss;
            ess += P.k_ss * dr * dr;
        }
    }
    ep = block_sum(ep, sm);
    es = block_sum(es, sm);
    ed = block_sum(ed, sm);
    ess = block_sum(ess, sm);
    if (threadIdx.x == 0) {
        const double sasa = (a1 > a0) ? P.beta_sa + es : 0.0;
        double *o = terms + 5 * (size_t)s;
        o[0] = sasa;
        o[1] = ed;
        o[2] = ess;
        o[3] = ep;
        o[4] = sasa + ed + ess + ep;
    }
}

}  // namespace alma

using namespace alma;

static int check_batch(const AlmaBatch *b, const char *who) {
    if (!b || b->nsys <= 0 || b->natoms < 0 || !b->atom_off || !b->xyz || !b->prm || !b->prm64 || !b->born)
        return alma_set_error(ALMA_EINVAL, "%s: bad batch", who);
    return ALMA_OK;
}

extern "C" int alma_born_radii(const AlmaBatch *b, const AlmaNL *nl, const AlmaParams *p, int prec,
                               const uint8_t *sys_mask, void *stream) {
    int rc = check_batch(b, "alma_born_radii");
    if (rc) return rc;
    if (!nl || !nl->full_ptr || !nl->full_cols || !p) return alma_set_error(ALMA_EINVAL, "alma_born_radii: null");
    if (b->natoms == 0) return ALMA_OK;
    cudaStream_t st = (cudaStream_t)stream;
    const int wpb = 8, nb = (b->natoms + wpb - 1) / wpb;
    if (prec == ALMA_PREC_FP64)
        born_kernel<double><<<nb, wpb * 32, 0, st>>>(b->natoms, b->atom_off, b->nsys, sys_mask, b->xyz, b->prm, b->prm64, nl->full_ptr, nl->full_len, nl->full_cols, b->born);
    else
        born_kernel<float><<<nb, wpb * 32, 0, st>>>(b->natoms, b->atom_off, b->nsys, sys_mask, b->xyz, b->prm, b->prm64, nl->full_ptr, nl->full_len, nl->full_cols, b->born);
    ALMA_LAUNCH_CHECK("alma_born_radii");
    return ALMA_OK;
}

extern "C" int alma_energy(const AlmaBatch *b, const AlmaTopo *t, const AlmaNL *nl, const AlmaParams *p, int prec,
                           const uint8_t *sys_mask, double *atom_e, double *terms, void *stream) {
    int rc = check_batch(b, "alma_energy");
    if (rc) return rc;
    if (!nl || !nl->half_ptr || !nl->half_cols || !p || !atom_e || !terms)
        return alma_set_error(ALMA_EINVAL, "alma_energy: null argument");
    cudaStream_t st = (cudaStream_t)stream;
    const DevParams P = make_dev_params(*p);
    if (b->natoms > 0) {
        const int wpb = 8, nb = (b->natoms + wpb - 1) / wpb;
        const int use_excl = t != nullptr;
        if (prec == ALMA_PREC_FP64)
            pair_sasa_kernel<double><<<nb, wpb * 32, 0, st>>>(P, b->natoms, b->atom_off, b->nsys, sys_mask, b->xyz, b->prm, b->prm64, b->born,
                                                              nl->half_ptr, nl->half_len, nl->half_cols, use_excl, atom_e, b->sasa);
        else
            pair_sasa_kernel<float><<<nb, wpb * 32, 0, st>>>(P, b->natoms, b->atom_off, b->nsys, sys_mask, b->xyz, b->prm, b->prm64, b->born,
                                                             nl->half_ptr, nl->half_len, nl->half_cols, use_excl, atom_e, b->sasa);
    }
    AlmaTopo tt;
    if (t) tt = *t;
    else memset(&tt, 0, sizeof(tt));
    energy_reduce_kernel<<<b->nsys, 256, 0, st>>>(P, b->atom_off, b->xyz, atom_e, tt, t != nullptr, sys_mask, terms);
    ALMA_LAUNCH_CHECK_N("alma_energy", b->natoms > 0 ? 2 : 1);
    return ALMA_OK;
}
