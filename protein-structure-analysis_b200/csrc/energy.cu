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
#include "alma_common.cuh"

namespace alma {

// (charge, R*, epsilon) in precision R.
template <typename R>
__device__ __forceinline__ void load_prm(const float *prm, const double *prm64, int i, R &q, R &rad, R &eps) {
    if constexpr (sizeof(R) == 4) {
        const float4 p = *reinterpret_cast<const float4 *>(prm + 4 * (size_t)i);
        q = p.x; rad = p.y; eps = p.z;
    } else {
        const double4 p = *reinterpret_cast<const double4 *>(prm64 + 4 * (size_t)i);
        q = p.x; rad = p.y; eps = p.z;
    }
}

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
    R qi, ri, ei;
    load_prm<R>(prm, prm64, i, qi, ri, ei);
    const double4 pi = ld_xyz(xyz, i);
    double sum = 0.0;
    for (int64_t k = full_ptr[i] + lane; k < full_ptr[i] + full_len[i]; k += 32) {
        const int j = (int)(full_cols[k] & ALMA_IDX_MASK);
        R qj, rj, ej;
        load_prm<R>(prm, prm64, j, qj, rj, ej);
        const double r2d = d2_of(pi, ld_xyz(xyz, j));
        const R r2 = (R)r2d;
        sum += (double)hct_term<R>(m_sqrt(r2), r2, ri, rj);
    }
    sum = warp_sum(sum);
    if (lane == 0) {
        const double r64 = prm64[4 * (size_t)i + 1];
        const double inv = 1.0 / r64 - 0.5 * sum;
        born[i] = 1.0 / fmax(inv, 2.0);
    }
}

// Warp per atom: pair energy and SASA of row i.  atom_e[2*i] = pair sum of
// row i, atom_e[2*i+1] = gamma * max(0, sa_i).
template <typename R>
__global__ void pair_sasa_kernel(DevParams P, int natoms, const int32_t *__restrict__ atom_off, int nsys,
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
    R qi, ri, ei;
    load_prm<R>(prm, prm64, i, qi, ri, ei);
    const R ai = (R)born[i];
    const double4 pi = ld_xyz(xyz, i);
    const double rsi = prm64[4 * (size_t)i + 1] + P.probe_r;
    const double cap_scale = 2.0 * 3.14159265358979323846 * rsi * rsi;
    double sa = 4.0 * 3.14159265358979323846 * rsi * rsi;
    double e = 0.0;
    const int64_t beg = half_ptr[i], end = half_ptr[i] + half_len[i];
    for (int64_t k0 = beg; k0 < end; k0 += 32) {
        const int64_t k = k0 + lane;
        double cap = 0.0;
        bool hit = false;
        if (k < end) {
            const uint32_t ent = half_cols[k];
            const int j = (int)(ent & ALMA_IDX_MASK);
            const double r2d = d2_of(pi, ld_xyz(xyz, j));
            const double rsj = prm64[4 * (size_t)j + 1] + P.probe_r;
            const double r = sqrt(r2d), dc = rsi + rsj;
            if (r < dc) {
                hit = true;
                cap = cap_scale * ((dc - r) / (2.0 * rsi));
            }
            if (!(use_excl && (ent & ALMA_EXCL_BIT)) && r2d <= P.pair_cut2) {
                R qj, rj, ej;
                load_prm<R>(prm, prm64, j, qj, rj, ej);
                e += (double)pair_energy<R>(P, (R)r2d, qi * qj, ri + rj, ei * ej, ai, (R)born[j]);
            }
        }
        unsigned m = __ballot_sync(0xffffffffu, hit);
        while (m) {  // the order-dependent recurrence, entry by entry
            const int l = __ffs(m) - 1;
            m &= m - 1;
            const double c = __shfl_sync(0xffffffffu, cap, l);
            sa -= fmin(sa * 0.85, c);
        }
    }
    e = warp_sum(e);
    if (lane == 0) {
        atom_e[2 * (size_t)i] = e;
        atom_e[2 * (size_t)i + 1] = P.gamma_sa * fmax(0.0, sa);
        if (sasa_out) sasa_out[i] = atom_e[2 * (size_t)i + 1];
    }
}

__device__ __forceinline__ double dihedral_angle(const double *xyz, int a, int b, int c, int d) {
    const double4 A = ld_xyz(xyz, a), B = ld_xyz(xyz, b), C = ld_xyz(xyz, c), D = ld_xyz(xyz, d);
    const double b1x = A.x - B.x, b1y = A.y - B.y, b1z = A.z - B.z;
    const double b2x = C.x - B.x, b2y = C.y - B.y, b2z = C.z - B.z;
    const double b3x = D.x - C.x, b3y = D.y - C.y, b3z = D.z - C.z;
    const double n1x = b1y * b2z - b1z * b2y, n1y = b1z * b2x - b1x * b2z, n1z = b1x * b2y - b1y * b2x;
    const double n2x = b2y * b3z - b2z * b3y, n2y = b2z * b3x - b2x * b3z, n2z = b2x * b3y - b2y * b3x;
    const double m1x = n1y * b2z - n1z * b2y, m1y = n1z * b2x - n1x * b2z, m1z = n1x * b2y - n1y * b2x;
    return atan2(m1x * n2x + m1y * n2y + m1z * n2z, n1x * n2x + n1y * n2y + n1z * n2z);
}

__device__ __forceinline__ double dih_record_energy(const double *xyz, const AlmaTopo &t, int r) {
    const int4 q = *reinterpret_cast<const int4 *>(t.dih_abcd + 4 * (size_t)r);
    const double phi = dihedral_angle(xyz, q.x, q.y, q.z, q.w);
    double E = 0.0;
    for (int k = t.term_off[r]; k < t.term_off[r + 1]; ++k)
        E += t.term_v2[k] * (1.0 + cos((double)t.term_n[k] * phi - t.term_gamma[k]));
    return E;
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
