// Analytic gradient dE/dx of the full energy (the backward of alma_energy).
//
// E = Σ_pairs e(r_ij, a_i a_j) + E_SASA + E_dihedral + E_SS with the Born
// radii a_i = 1/max(1/rho_i - ½ Σ_j hct(r_ij; rho_i, rho_j), 2) (born_radii,
// physics_engine.cpp:2024-2039).  Four kernels:
//
//   pair   warp per atom over its FULL row: the direct pair force of every
//          non-excluded partner within 12 Å, gathered (each pair is seen
//          from both ends, so no atomics), and dE/da_i = Σ_j ∂e/∂(a_i a_j)·a_j;
//          zeroes the atom's fixed-point slots;
//   sasa   warp per atom over its HALF row: the SASA recurrence
//          sa <- sa - min(0.85 sa, cap_k) (:2068-2083) is run twice — once to
//          count the entries that took the 0.85·sa branch, once to give each
//          entry that took the cap branch its adjoint γ·π·R*·0.15^(number of
//          later 0.85 entries); the pair force goes to both atoms through
//          64-bit fixed-point atomics (integer adds: order independent);
//   bonded thread per dihedral record / disulfide, fixed-point atomics.  The
//          reference angle is atan2(|b2| sinφ, cosφ) (its m1 = n1 × b2 is not
//          normalised, :1871-1887), and the gradient is that of this angle;
//   born   warp per atom over its FULL row: the chain rule through the
//          recomputed HCT integrals, Σ_j (c_i hct'(r; rho_i, rho_j) +
//          c_j hct'(r; rho_j, rho_i)) (x_i - x_j)/r with c_k = dE/da_k · a_k²/2
//          (0 where the radius is clamped), plus the pair and fixed-point
//          parts: the final gradient.
//
// Precision R: the pair and HCT derivative arithmetic (float in mixed mode;
// LJ and hard core inside sigma in FP64, as in the ΔE path), accumulation
// in FP64.  Every sum has a fixed order, so the gradient is deterministic.
#include "alma_common.cuh"

namespace alma {

constexpr double FIX_SCALE = 4294967296.0;  // 2^32: resolution 2.3e-10, range ±2.1e9
constexpr double FIX_INV = 1.0 / 4294967296.0;

__device__ __forceinline__ void fix_add(unsigned long long *slot, double v) {
    atomicAdd(slot, (unsigned long long)__double2ll_rn(v * FIX_SCALE));
}

template <typename R>
__device__ __forceinline__ void load_prm_g(const float *prm, const double *prm64, int i, R &q, R &rad, R &eps) {
    if constexpr (sizeof(R) == 4) {
        const float4 p = *reinterpret_cast<const float4 *>(prm + 4 * (size_t)i);
        q = p.x; rad = p.y; eps = p.z;
    } else {
        const double4 p = *reinterpret_cast<const double4 *>(prm64 + 4 * (size_t)i);
        q = p.x; rad = p.y; eps = p.z;
    }
}

// (dE/dr)/r of one pair and ∂E/∂(a_i a_j), pair_e (:2148-2164):
//   DH  K qq e^{-κr}/r            -> -e_dh (1/r + κ) / r
//   GB  C qq / f, f² = r² + A D, D = e^{-r²/4A}
//       -> -e_gb (2 - D/2) / (2 f²),   ∂/∂A = -e_gb D (1 + r²/4A) / (2 f²)
//   LJ  4√εε (s¹² - s⁶), s = σ/r  -> 4√εε (6 s⁶ - 12 s¹²) / r²
//   hard min(H x², cap), x = (rc/r)¹² - 1 -> -24 H x (rc/r)¹² / r² below the cap
template <typename R>
__device__ __forceinline__ void pair_grad(const DevParams &P, double r2d, R qp, R sig, R eps_prod, R ai, R aj,
                                          double sig64, double eps64, double &fr, double &dEdA) {
    const R r2 = (R)r2d;
    R f_dh, f_gb;
    if constexpr (sizeof(R) == 4) {  // the fast FP32 forms of pair_energy (same error budget)
        const float rinv = rsqrtf(r2), r = r2 * rinv;
        const float kap = (float)P.kappa;
        const float edh = (float)P.coulomb_over_epsw * qp * rinv * __expf(-kap * r);
        f_dh = -edh * (rinv + kap) * rinv;
        const float A = ai * aj;
        const float r2_4A = 0.25f * __fdividef(r2, A);
        const float D = __expf(-r2_4A);
        const float f2 = r2 + A * D;
        const float rf2 = __fdividef(1.0f, f2);
        const float egb = (float)P.gb_coef * qp * rsqrtf(f2);
        f_gb = -egb * (2.0f - 0.5f * D) * 0.5f * rf2;
        dEdA = (double)(-egb * D * (1.0f + r2_4A) * 0.5f * rf2);
    } else {
        const R r = m_sqrt(r2);
        const R kap = (R)P.kappa;
        const R edh = (R)P.coulomb_over_epsw * qp / r * m_exp(-kap * r);
        f_dh = -edh * ((R)1 / r + kap) / r;
        const R A = ai * aj;
        const R D = m_exp(-r2 / ((R)4 * A));
        const R f2 = r2 + A * D;
        const R egb = (R)P.gb_coef * qp / m_sqrt(f2);
        f_gb = -egb * ((R)2 - (R)0.5 * D) / ((R)2 * f2);
        dEdA = (double)(-egb * D * ((R)1 + r2 / ((R)4 * A)) / ((R)2 * f2));
    }
    double f_lj;
    const double sig2 = sig64 * sig64;
    if (r2d < sig2) {  // steep: FP64 with FP64 sigma / epsilon
        const double s2 = sig2 / r2d, s6 = s2 * s2 * s2;
        f_lj = 4.0 * sqrt(eps64) * (6.0 * s6 - 12.0 * s6 * s6) / r2d;
        const double rc = sig64 * P.hard_frac, rc2 = rc * rc;
        if (r2d < rc2) {
            const double t2 = rc2 / r2d, t6 = t2 * t2 * t2, t12 = t6 * t6, x = t12 - 1.0;
            if (P.hard_scale * x * x < P.hard_cap) f_lj += -24.0 * P.hard_scale * x * t12 / r2d;
        }
    } else {
        const R s2 = (R)(sig2 / r2d);
        const R s6 = s2 * s2 * s2;
        if constexpr (sizeof(R) == 4)
            f_lj = (double)(4.0f * f_sqrt(eps_prod) * (6.0f * s6 - 12.0f * s6 * s6) * __fdividef(1.0f, r2));
        else
            f_lj = (double)((R)4 * m_sqrt(eps_prod) * ((R)6 * s6 - (R)12 * s6 * s6) / r2);
    }
    fr = (double)f_dh + (double)f_gb + f_lj;
}

// d/dr of hct(r; ri, rj) = 1/L - 1/U + P ln(L/U) / (4 ri² r²),
// L = max(|r - rj|, ri), U = r + rj, P = r² - rj² + ri² (:2007-2011).
template <typename R>
__device__ __forceinline__ R hct_deriv(R r, R r2, R ri, R rj) {
    const R U = r + rj;
    if (ri >= U) return (R)0;
    if constexpr (sizeof(R) == 4) {  // fast reciprocals, logf kept (see hct_term)
        const float d = fabsf(r - rj);
        float L, Lp;
        if (d > ri) {
            L = d;
            Lp = r > rj ? 1.0f : -1.0f;
        } else {
            L = ri;
            Lp = 0.0f;
        }
        const float rL = __fdividef(1.0f, L), rU = __fdividef(1.0f, U), rr = __fdividef(1.0f, r);
        const float Pp = r2 - rj * rj + ri * ri;
        const float Q = logf(L * rU);
        const float rden = __fdividef(0.25f, ri * ri * r2);
        const float T = Pp * Q * rden;
        const float dT = (2.0f * r * Q + Pp * (Lp * rL - rU)) * rden - 2.0f * T * rr;
        return -Lp * rL * rL + rU * rU + dT;
    }
    const R d = m_abs(r - rj);
    R L, Lp;
    if (d > ri) {
        L = d;
        Lp = r > rj ? (R)1 : (R)-1;
    } else {
        L = ri;
        Lp = (R)0;
    }
    const R Pp = r2 - rj * rj + ri * ri;
    const R Q = m_log(L / U);
    const R den = (R)4 * ri * ri * r2;
    const R T = Pp * Q / den;
    const R dT = ((R)2 * r * Q + Pp * (Lp / L - (R)1 / U)) / den - (R)2 * T / r;
    return -Lp / (L * L) + (R)1 / (U * U) + dT;
}

// Warp per atom, 256 threads, 4 blocks per SM (64 registers): the row
// gathers are latency bound and the occupancy pays.
template <typename R>
__global__ void __launch_bounds__(256, 4) grad_pair_kernel(DevParams P, int natoms, const int32_t *__restrict__ atom_off, int nsys,
                                 const uint8_t *__restrict__ mask, const double *__restrict__ xyz,
                                 const float *__restrict__ prm, const double *__restrict__ prm64,
                                 const double *__restrict__ born, const int64_t *__restrict__ full_ptr,
                                 const int32_t *__restrict__ full_len, const uint32_t *__restrict__ full_cols,
                                 int use_excl, double *__restrict__ grad, double *__restrict__ dEda,
                                 unsigned long long *__restrict__ fix) {
    const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= natoms) return;
    if (mask && !mask[sys_of_atom(atom_off, nsys, i)]) return;
    R qi, ri, ei;
    load_prm_g<R>(prm, prm64, i, qi, ri, ei);
    const double4 pi = ld_xyz(xyz, i);
    const double4 p64i = *reinterpret_cast<const double4 *>(prm64 + 4 * (size_t)i);
    const R ai = (R)born[i];
    double gx = 0.0, gy = 0.0, gz = 0.0, da = 0.0;
    const int64_t beg = full_ptr[i], end = beg + full_len[i];
    // the next entry is fetched while this one is evaluated, and an entry's
    // gathers are issued together (one dependent round trip per entry)
    uint32_t nxt = beg + lane < end ? full_cols[beg + lane] : 0u;
    for (int64_t k = beg + lane; k < end; k += 32) {
        const uint32_t ent = nxt;
        if (k + 32 < end) nxt = full_cols[k + 32];
        if (use_excl && (ent & ALMA_EXCL_BIT)) continue;
        const int j = (int)(ent & ALMA_IDX_MASK);
        const double4 pj = ld_xyz(xyz, j);
        R qj, rj, ej;
        load_prm_g<R>(prm, prm64, j, qj, rj, ej);
        const double rj64 = prm64[4 * (size_t)j + 1], ej64 = prm64[4 * (size_t)j + 2];
        const double bj = born[j];
        const double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
        const double r2 = dx * dx + dy * dy + dz * dz;
        if (r2 > P.pair_cut2) continue;
        double fr, dEdA;
        pair_grad<R>(P, r2, qi * qj, ri + rj, ei * ej, ai, (R)bj, p64i.y + rj64, p64i.z * ej64, fr, dEdA);
        gx += fr * dx;
        gy += fr * dy;
        gz += fr * dz;
        da += dEdA * bj;
    }
    gx = warp_sum(gx);
    gy = warp_sum(gy);
    gz = warp_sum(gz);
    da = warp_sum(da);
    if (lane == 0) {
        *reinterpret_cast<double4 *>(grad + 4 * (size_t)i) = make_double4(gx, gy, gz, 0.0);
        dEda[i] = da;
        fix[3 * (size_t)i] = fix[3 * (size_t)i + 1] = fix[3 * (size_t)i + 2] = 0ull;
    }
}

// SASA adjoints over the ordered half row (FP64, as the forward).
__global__ void __launch_bounds__(256, 4) grad_sasa_kernel(DevParams P, int natoms, const int32_t *__restrict__ atom_off, int nsys,
                                 const uint8_t *__restrict__ mask, const double *__restrict__ xyz,
                                 const double *__restrict__ prm64, const int64_t *__restrict__ half_ptr,
                                 const int32_t *__restrict__ half_len, const uint32_t *__restrict__ half_cols,
                                 unsigned long long *__restrict__ fix) {
    const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= natoms) return;
    if (mask && !mask[sys_of_atom(atom_off, nsys, i)]) return;
    const double4 pi = ld_xyz(xyz, i);
    const double rsi = prm64[4 * (size_t)i + 1] + P.probe_r;
    const double cap_scale = 2.0 * 3.14159265358979323846 * rsi * rsi;
    const double sa0 = 4.0 * 3.14159265358979323846 * rsi * rsi;
    const int64_t beg = half_ptr[i], end = beg + half_len[i];
    // pass 1: final sa and the number of 0.85-branch entries
    double sa = sa0;
    int n_frac = 0;
    for (int64_t k0 = beg; k0 < end; k0 += 32) {
        const int64_t k = k0 + lane;
        double cap = 0.0;
        bool hit = false;
        if (k < end) {
            const int j = (int)(half_cols[k] & ALMA_IDX_MASK);
            const double r = sqrt(d2_of(pi, ld_xyz(xyz, j)));
            const double dc = rsi + prm64[4 * (size_t)j + 1] + P.probe_r;
            if (r < dc) {
                hit = true;
                cap = cap_scale * ((dc - r) / (2.0 * rsi));
            }
        }
        const unsigned m = __ballot_sync(0xffffffffu, hit);
        const int n = __popc(m);
        const double packed = sasa_pack(m, cap, lane);
        for (int q = 0; q < n; ++q) {  // row order; the shuffles do not wait for sa
            const double c = __shfl_sync(0xffffffffu, packed, q);
            if (c <= sa * 0.85) {
                sa -= c;
            } else {
                sa -= sa * 0.85;
                ++n_frac;
            }
        }
    }
    if (!(sa > 0.0)) return;  // max(0, sa) is flat here
    // pass 2: the same recurrence; adjoint of each cap-branch entry
    const double base = P.gamma_sa * 3.14159265358979323846 * rsi;  // -dE/dcap * dcap/dr
    double gx = 0.0, gy = 0.0, gz = 0.0;
    sa = sa0;
    int seen = 0;
    for (int64_t k0 = beg; k0 < end; k0 += 32) {
        const int64_t k = k0 + lane;
        double cap = 0.0, dx = 0.0, dy = 0.0, dz = 0.0, r = 1.0;
        bool hit = false;
        int j = 0;
        if (k < end) {
            j = (int)(half_cols[k] & ALMA_IDX_MASK);
            const double4 pj = ld_xyz(xyz, j);
            dx = pi.x - pj.x;
            dy = pi.y - pj.y;
            dz = pi.z - pj.z;
            r = sqrt(dx * dx + dy * dy + dz * dz);
            const double dc = rsi + prm64[4 * (size_t)j + 1] + P.probe_r;
            if (r < dc) {
                hit = true;
                cap = cap_scale * ((dc - r) / (2.0 * rsi));
            }
        }
        // the recurrence over the packed hits: packed lane q holds the q-th
        // hit; its cap-branch adjoint goes back to the hit's own lane
        const unsigned m = __ballot_sync(0xffffffffu, hit);
        const int n = __popc(m);
        const double packed = sasa_pack(m, cap, lane);
        double pcoef = 0.0;
        for (int q = 0; q < n; ++q) {
            const double c = __shfl_sync(0xffffffffu, packed, q);
            if (c <= sa * 0.85) {
                sa -= c;
                if (lane == q) pcoef = base * pow(0.15, (double)(n_frac - seen));
            } else {
                sa -= sa * 0.85;
                ++seen;
            }
        }
        const double coef = __shfl_sync(0xffffffffu, pcoef, __popc(m & ((1u << lane) - 1u)));
        if (hit && coef != 0.0) {
            const double s = coef / r;
            gx += s * dx;
            gy += s * dy;
            gz += s * dz;
            fix_add(&fix[3 * (size_t)j], -s * dx);
            fix_add(&fix[3 * (size_t)j + 1], -s * dy);
            fix_add(&fix[3 * (size_t)j + 2], -s * dz);
        }
    }
    gx = warp_sum(gx);
    gy = warp_sum(gy);
    gz = warp_sum(gz);
    if (lane == 0) {
        fix_add(&fix[3 * (size_t)i], gx);
        fix_add(&fix[3 * (size_t)i + 1], gy);
        fix_add(&fix[3 * (size_t)i + 2], gz);
    }
}

__device__ __forceinline__ double3 sub3(double4 a, double4 b) { return make_double3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ double3 cross3(double3 a, double3 b) {
    return make_double3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double dot3(double3 a, double3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

__device__ __forceinline__ void fix_add3(unsigned long long *fix, int i, double s, double3 v) {
    fix_add(&fix[3 * (size_t)i], s * v.x);
    fix_add(&fix[3 * (size_t)i + 1], s * v.y);
    fix_add(&fix[3 * (size_t)i + 2], s * v.z);
}

// Dihedral records and disulfide springs, one thread each.
__global__ void grad_bonded_kernel(DevParams P, const int32_t *__restrict__ atom_off, int nsys,
                                   const uint8_t *__restrict__ mask, const double *__restrict__ xyz, AlmaTopo t,
                                   int ndih, int nss, unsigned long long *__restrict__ fix) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < ndih) {
        const int4 q = *reinterpret_cast<const int4 *>(t.dih_abcd + 4 * (size_t)r);
        if (mask && !mask[sys_of_atom(atom_off, nsys, q.x)]) return;
        const double4 A = ld_xyz(xyz, q.x), B = ld_xyz(xyz, q.y), Cc = ld_xyz(xyz, q.z), D = ld_xyz(xyz, q.w);
        const double3 b1 = sub3(A, B), b2 = sub3(Cc, B), b3 = sub3(D, Cc);
        const double3 n1 = cross3(b1, b2), n2 = cross3(b2, b3), m1 = cross3(n1, b2);
        const double x = dot3(n1, n2), y = dot3(m1, n2);
        const double phi = atan2(y, x);
        double dEdphi = 0.0;
        for (int k = t.term_off[r]; k < t.term_off[r + 1]; ++k) {
            const double n = (double)t.term_n[k];
            dEdphi -= t.term_v2[k] * n * sin(n * phi - t.term_gamma[k]);
        }
        // gradient of the true dihedral (Blondel & Karplus, J. Comput. Chem.
        // 17:1132, 1996) with F = a-b, G = b-c, H = d-c, then the map
        // phi_ref = atan2(L sin phi, cos phi), L = |b2|.
        const double3 F = b1, G = make_double3(-b2.x, -b2.y, -b2.z), H = b3;
        const double3 Av = cross3(F, G), Bv = cross3(H, G);
        const double A2 = dot3(Av, Av), B2 = dot3(Bv, Bv), Gn = sqrt(dot3(G, G));
        const double FG = dot3(F, G), HG = dot3(H, G);
        const double NN = dot3(n1, n1) * dot3(n2, n2);
        const double den = (x * x + y * y) / NN;  // cos^2 + L^2 sin^2
        const double sc = (y / Gn) * x / NN;       // sin cos
        const double sA = dEdphi * Gn / den, sB = dEdphi / den;
        // d(phi_ref) = (L d(phi) + sin cos dL) / den, d(phi) = -(BK terms)
        const double ka = Gn / A2, kb = Gn / B2, kfa = FG / (A2 * Gn), khb = HG / (B2 * Gn);
        fix_add3(fix, q.x, sA, make_double3(ka * Av.x, ka * Av.y, ka * Av.z));
        fix_add3(fix, q.w, -sA, make_double3(kb * Bv.x, kb * Bv.y, kb * Bv.z));
        const double3 gb = make_double3(ka * Av.x + kfa * Av.x - khb * Bv.x, ka * Av.y + kfa * Av.y - khb * Bv.y,
                                        ka * Av.z + kfa * Av.z - khb * Bv.z);
        const double3 gc = make_double3(-kfa * Av.x + khb * Bv.x - kb * Bv.x, -kfa * Av.y + khb * Bv.y - kb * Bv.y,
                                        -kfa * Av.z + khb * Bv.z - kb * Bv.z);
        const double3 u2 = make_double3(b2.x / Gn, b2.y / Gn, b2.z / Gn);  // dL/dc = b2/L = -dL/db
        fix_add3(fix, q.y, -sA, gb);
        fix_add3(fix, q.y, -sB * sc, u2);
        fix_add3(fix, q.z, -sA, gc);
        fix_add3(fix, q.z, sB * sc, u2);
        return;
    }
    const int k = r - ndih;
    if (k < nss) {
        const int i = t.ss_ij[2 * k], j = t.ss_ij[2 * k + 1];
        if (mask && !mask[sys_of_atom(atom_off, nsys, i)]) return;
        const double3 d = sub3(ld_xyz(xyz, i), ld_xyz(xyz, j));
        const double rr = sqrt(dot3(d, d));
        const double s = 2.0 * P.k_ss * (rr - P.r0_ss) / rr;
        fix_add3(fix, i, s, d);
        fix_add3(fix, j, -s, d);
    }
}

// Born-radius chain rule plus the final sum into grad.
template <typename R>
__global__ void grad_born_kernel(int natoms, const int32_t *__restrict__ atom_off, int nsys,
                                 const uint8_t *__restrict__ mask, const double *__restrict__ xyz,
                                 const float *__restrict__ prm, const double *__restrict__ prm64,
                                 const double *__restrict__ born, const int64_t *__restrict__ full_ptr,
                                 const int32_t *__restrict__ full_len, const uint32_t *__restrict__ full_cols,
                                 const double *__restrict__ dEda, const unsigned long long *__restrict__ fix,
                                 double *__restrict__ grad) {
    const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= natoms) return;
    if (mask && !mask[sys_of_atom(atom_off, nsys, i)]) return;
    R qi, ri, ei;
    load_prm_g<R>(prm, prm64, i, qi, ri, ei);
    const double4 pi = ld_xyz(xyz, i);
    const double ai = born[i];
    const double ci = ai < 0.5 ? 0.5 * dEda[i] * ai * ai : 0.0;
    double gx = 0.0, gy = 0.0, gz = 0.0;
    const int64_t beg = full_ptr[i], end = beg + full_len[i];
    uint32_t nxt = beg + lane < end ? full_cols[beg + lane] : 0u;  // next entry in flight
    for (int64_t k = beg + lane; k < end; k += 32) {
        const int j = (int)(nxt & ALMA_IDX_MASK);
        if (k + 32 < end) nxt = full_cols[k + 32];
        // every gather of the entry issued together (one round trip)
        const double aj = born[j], dj = dEda[j];
        R qj, rj, ej;
        load_prm_g<R>(prm, prm64, j, qj, rj, ej);
        const double4 pj = ld_xyz(xyz, j);
        const double cj = aj < 0.5 ? 0.5 * dj * aj * aj : 0.0;
        if (ci == 0.0 && cj == 0.0) continue;
        const double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
        const R r2 = (R)(dx * dx + dy * dy + dz * dz);
        const R r = f_sqrt(r2);
        const double s = (ci * (double)hct_deriv<R>(r, r2, ri, rj) + cj * (double)hct_deriv<R>(r, r2, rj, ri)) /
                         (double)r;
        gx += s * dx;
        gy += s * dy;
        gz += s * dz;
    }
    gx = warp_sum(gx);
    gy = warp_sum(gy);
    gz = warp_sum(gz);
    if (lane == 0) {
        double4 g = *reinterpret_cast<const double4 *>(grad + 4 * (size_t)i);
        g.x += gx + (double)(long long)fix[3 * (size_t)i] * FIX_INV;
        g.y += gy + (double)(long long)fix[3 * (size_t)i + 1] * FIX_INV;
        g.z += gz + (double)(long long)fix[3 * (size_t)i + 2] * FIX_INV;
        g.w = 0.0;
        *reinterpret_cast<double4 *>(grad + 4 * (size_t)i) = g;
    }
}

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace alma

using namespace alma;

extern "C" size_t alma_forces_workspace_bytes(int32_t natoms) {
    const size_t n = natoms > 0 ? (size_t)natoms : 1;
    return align256(sizeof(double) * n) + align256(sizeof(unsigned long long) * 3 * n);
}

extern "C" int alma_forces(const AlmaBatch *b, const AlmaTopo *t, const AlmaNL *nl, const AlmaParams *p,
                           int precision, const uint8_t *sys_mask, void *workspace, double *grad, void *stream) {
    if (!b || !nl || !p || !grad || !workspace || b->nsys <= 0 || b->natoms < 0)
        return alma_set_error(ALMA_EINVAL, "alma_forces: bad arguments");
    if (!b->atom_off || !b->xyz || !b->prm || !b->prm64 || !b->born || !nl->full_ptr || !nl->full_len ||
        !nl->full_cols || !nl->half_ptr || !nl->half_len || !nl->half_cols)
        return alma_set_error(ALMA_EINVAL, "alma_forces: null buffer");
    if (precision != ALMA_PREC_MIXED && precision != ALMA_PREC_FP64)
        return alma_set_error(ALMA_EINVAL, "alma_forces: precision must be ALMA_PREC_MIXED or ALMA_PREC_FP64");
    if (b->natoms == 0) return ALMA_OK;
    cudaStream_t st = (cudaStream_t)stream;
    const DevParams P = make_dev_params(*p);
    char *ws = (char *)workspace;
    double *dEda = (double *)ws;
    unsigned long long *fix = (unsigned long long *)(ws + align256(sizeof(double) * (size_t)b->natoms));
    const int wpb = 8;
    const int nb = (b->natoms + wpb - 1) / wpb;
    const int use_excl = t != nullptr;
    if (precision == ALMA_PREC_FP64)
        grad_pair_kernel<double><<<nb, wpb * 32, 0, st>>>(P, b->natoms, b->atom_off, b->nsys, sys_mask, b->xyz, b->prm,
                                                          b->prm64, b->born, nl->full_ptr, nl->full_len,
                                                          nl->full_cols, use_excl, grad, dEda, fix);
    else
        grad_pair_kernel<float><<<nb, wpb * 32, 0, st>>>(P, b->natoms, b->atom_off, b->nsys, sys_mask, b->xyz, b->prm,
                                                         b->prm64, b->born, nl->full_ptr, nl->full_len,
                                                         nl->full_cols, use_excl, grad, dEda, fix);
    grad_sasa_kernel<<<nb, wpb * 32, 0, st>>>(P, b->natoms, b->atom_off, b->nsys, sys_mask, b->xyz, b->prm64,
                                              nl->half_ptr, nl->half_len, nl->half_cols, fix);
    int nlaunch = 3;
    if (t && (t->ndih > 0 || t->nss > 0)) {
        const int n = t->ndih + t->nss;
        grad_bonded_kernel<<<(n + 255) / 256, 256, 0, st>>>(P, b->atom_off, b->nsys, sys_mask, b->xyz, *t, t->ndih,
                                                            t->nss, fix);
        ++nlaunch;
    }
    if (precision == ALMA_PREC_FP64)
        grad_born_kernel<double><<<nb, wpb * 32, 0, st>>>(b->natoms, b->atom_off, b->nsys, sys_mask, b->xyz, b->prm,
                                                          b->prm64, b->born, nl->full_ptr, nl->full_len,
                                                          nl->full_cols, dEda, fix, grad);
    else
        grad_born_kernel<float><<<nb, wpb * 32, 0, st>>>(b->natoms, b->atom_off, b->nsys, sys_mask, b->xyz, b->prm,
                                                         b->prm64, b->born, nl->full_ptr, nl->full_len,
                                                         nl->full_cols, dEda, fix, grad);
    ALMA_LAUNCH_CHECK_N("alma_forces", nlaunch);
    return ALMA_OK;
}
