// Per-atom cores of the energy evaluation (Born radius of one atom, pair
// energy and SASA of one half row, dihedral records), shared by the
// stand-alone kernels (energy.cu) and the rebuild inside the persistent MC
// kernel (mc.cu).
#pragma once
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

// HCT Born radius of atom i over its full row (one warp; FP64 sum).
template <typename R>
__device__ __forceinline__ void born_atom(int i, int lane, const double *__restrict__ xyz, const float *__restrict__ prm,
                                          const double *__restrict__ prm64, const int64_t *__restrict__ full_ptr,
                                          const int32_t *__restrict__ full_len, const uint32_t *__restrict__ full_cols,
                                          double *__restrict__ born) {
    R qi, ri, ei;
    load_prm<R>(prm, prm64, i, qi, ri, ei);
    const double4 pi = ld_xyz(xyz, i);
    double sum = 0.0;
    const int64_t end = full_ptr[i] + full_len[i];
    int64_t k = full_ptr[i] + lane;
    uint32_t nxt = k < end ? full_cols[k] : 0u;  // the next entry is fetched while this one is evaluated
    for (; k < end; k += 32) {
        const int j = (int)(nxt & ALMA_IDX_MASK);
        if (k + 32 < end) nxt = full_cols[k + 32];
        R qj, rj, ej;
        load_prm<R>(prm, prm64, j, qj, rj, ej);
        const double r2d = d2_of(pi, ld_xyz(xyz, j));
        const R r2 = (R)r2d;
        sum += (double)hct_term<R>(f_sqrt(r2), r2, ri, rj);
    }
    sum = warp_sum(sum);
    if (lane == 0) {
        const double r64 = prm64[4 * (size_t)i + 1];
        const double inv = 1.0 / r64 - 0.5 * sum;
        born[i] = 1.0 / fmax(inv, 2.0);
    }
}

// Pair energy and SASA of atom i's half row (one warp): atom_e[2i] = pair
// sum of the row, atom_e[2i+1] = gamma * max(0, sa_i), also into sasa_out[i]
// when given.
template <typename R>
__device__ __forceinline__ void pair_sasa_atom(const DevParams &P, int i, int lane, const double *__restrict__ xyz,
                                               const float *__restrict__ prm, const double *__restrict__ prm64,
                                               const double *__restrict__ born, const int64_t *__restrict__ half_ptr,
                                               const int32_t *__restrict__ half_len,
                                               const uint32_t *__restrict__ half_cols, int use_excl,
                                               double *__restrict__ atom_e, double *__restrict__ sasa_out) {
    R qi, ri, ei;
    load_prm<R>(prm, prm64, i, qi, ri, ei);
    const R ai = (R)born[i];
    const double4 pi = ld_xyz(xyz, i);
    const double ri64 = prm64[4 * (size_t)i + 1], ei64 = prm64[4 * (size_t)i + 2];
    const double rsi = ri64 + P.probe_r;
    const double cap_scale = 2.0 * 3.14159265358979323846 * rsi * rsi;
    double sa = 4.0 * 3.14159265358979323846 * rsi * rsi;
    double e = 0.0;
    const int64_t beg = half_ptr[i], end = half_ptr[i] + half_len[i];
    // the next chunk's entry is fetched while this one is evaluated, and all
    // of an entry's gathers are issued together (one dependent round trip
    // per chunk; the 12-14 Å entries load parameters they do not use)
    uint32_t nxt = beg + lane < end ? half_cols[beg + lane] : 0u;
    for (int64_t k0 = beg; k0 < end; k0 += 32) {
        const int64_t k = k0 + lane;
        double cap = 0.0;
        bool hit = false;
        if (k < end) {
            const uint32_t ent = nxt;
            if (k + 32 < end) nxt = half_cols[k + 32];
            const int j = (int)(ent & ALMA_IDX_MASK);
            const double4 pj = ld_xyz(xyz, j);
            const double rj64 = prm64[4 * (size_t)j + 1];
            R qj, rj, ej;
            load_prm<R>(prm, prm64, j, qj, rj, ej);
            const R aj = (R)born[j];
            const double r2d = d2_of(pi, pj);
            const double rsj = rj64 + P.probe_r;
            const double r = sqrt(r2d), dc = rsi + rsj;
            if (r < dc) {
                hit = true;
                cap = cap_scale * ((dc - r) / (2.0 * rsi));
            }
            if (!(use_excl && (ent & ALMA_EXCL_BIT)) && r2d <= P.pair_cut2) {
                // FP64 sigma from the radii already loaded; the FP64 epsilon
                // product only for a contact inside sigma (steep LJ)
                const double sig64 = ri64 + rj64;
                const double eps64 = r2d < sig64 * sig64 ? ei64 * prm64[4 * (size_t)j + 2] : 0.0;
                e += (double)pair_energy<R>(P, r2d, qi * qj, ri + rj, ei * ej, ai, aj, sig64, eps64);
            }
        }
        sa = sasa_chunk(sa, __ballot_sync(0xffffffffu, hit), cap, lane);  // in row order
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

}  // namespace alma
