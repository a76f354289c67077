// Shared device code of the ALMA B200 engine: constants, pair arithmetic,
// the Philox counter RNG, warp/block reductions, error plumbing.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "alma_b200.h"

#define ALMA_WARP 32
#define ALMA_EXCL_BIT 0x80000000u
#define ALMA_IDX_MASK 0x7fffffffu

// ---------------------------------------------------------------------------
// host-side error state (alma_host.cpp)
// ---------------------------------------------------------------------------
int alma_set_error(int code, const char *fmt, ...);
int alma_cuda_error(cudaError_t e, const char *what);

#define ALMA_CUDA_TRY(expr)                                        \
    do {                                                           \
        cudaError_t _e = (expr);                                   \
        if (_e != cudaSuccess) return alma_cuda_error(_e, #expr);  \
    } while (0)

// Kernel launches issued by the library (alma_launch_count); every launch
// site is followed by ALMA_LAUNCH_CHECK(what, number of kernels launched).
void alma_count_launches(int n);

#define ALMA_LAUNCH_CHECK_N(what, n)                                   \
    do {                                                               \
        cudaError_t _e = cudaGetLastError();                           \
        if (_e != cudaSuccess) return alma_cuda_error(_e, what);       \
        alma_count_launches(n);                                        \
    } while (0)
#define ALMA_LAUNCH_CHECK(what) ALMA_LAUNCH_CHECK_N(what, 1)

// ---------------------------------------------------------------------------
// energy model (physics_engine.cpp:181-196, :2007-2011, :2148-2164)
// ---------------------------------------------------------------------------
struct DevParams {
    double coulomb_over_epsw;  // COULOMB / EPS_WATER
    double kappa;
    double gb_coef;            // -0.5 (1/eps_prot - 1/eps_water) COULOMB
    double gamma_sa, beta_sa, probe_r;
    double pair_cut2, nl_rcut2, half_skin2;
    double hard_scale, hard_cap, hard_frac;
    double k_ss, r0_ss;
};

inline DevParams make_dev_params(const AlmaParams &p) {
    DevParams d;
    d.coulomb_over_epsw = p.coulomb / p.eps_water;
    d.kappa = p.kappa;
    d.gb_coef = -0.5 * (1.0 / p.eps_prot - 1.0 / p.eps_water) * p.coulomb;
    d.gamma_sa = p.gamma_sa;
    d.beta_sa = p.beta_sa;
    d.probe_r = p.probe_r;
    d.pair_cut2 = p.pair_cut2;
    d.nl_rcut2 = p.nl_rcut2;
    d.half_skin2 = p.half_skin2;
    d.hard_scale = p.hard_scale;
    d.hard_cap = p.hard_cap;
    d.hard_frac = p.hard_frac;
    d.k_ss = p.k_ss;
    d.r0_ss = p.r0_ss;
    return d;
}

// Math shims so the pair code is written once for float and double.  The
// float versions are CUDA's accurate single-precision functions (no
// fast-math intrinsics); division and sqrt are IEEE-rounded.
__device__ __forceinline__ float m_exp(float x) { return expf(x); }
__device__ __forceinline__ double m_exp(double x) { return exp(x); }
__device__ __forceinline__ float m_log(float x) { return logf(x); }
__device__ __forceinline__ double m_log(double x) { return log(x); }
__device__ __forceinline__ float m_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double m_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float m_abs(float x) { return fabsf(x); }
__device__ __forceinline__ double m_abs(double x) { return fabs(x); }

// Fast FP32 forms for the pair passes (the FP64 passes keep the exact
// forms).  Error budget per call, relative: rsqrtf <= 2 ulp; __fdividef
// <= 2 ulp (denominators here are far inside [2^-126, 2^126]); __expf
// 2 + floor(1.16 |x|) ulp — 3 ulp for the Debye-Hückel factor (kappa r <=
// 1.51 inside the cutoff) and for the GB factor wherever it is not
// negligible against r^2.  Logarithms stay logf (the HCT log of L/U near 1
// needs its relative accuracy) and so do expm1f / log1pf of the ΔE
// differences.  Summed over ~10^6 pairs these stay well inside the 1e-6
// relative bar on the total energy and the 1e-4 kcal/mol bar on ΔE.
__device__ __forceinline__ float f_sqrt(float x) { return x > 0.0f ? x * rsqrtf(x) : 0.0f; }
__device__ __forceinline__ double f_sqrt(double x) { return sqrt(x); }

// One nonbonded pair: Debye-Hückel + GB + LJ 12-6 + smooth capped hard core.
// r2d is the FP64 squared distance; q = qi*qj product; the caller has
// already applied the exclusion and 12 Å tests.  FP32: the fast forms
// above, and LJ + hard core in FP64 with the FP64 sigma / epsilon product
// (sig64, eps64) inside sigma (the steep terms: a clash's r^-12 would
// amplify the FP32 rounding of sigma twelvefold).
template <typename R>
__device__ __forceinline__ R pair_energy(const DevParams &P, double r2d, R qp, R sig, R eps_prod,
                                         R ai, R aj, double sig64, double eps64) {
    if constexpr (sizeof(R) == 4) {
        const float r2 = (float)r2d;
        const float rinv = rsqrtf(r2), r = r2 * rinv;
        const float edh = (float)P.coulomb_over_epsw * qp * rinv * __expf(-(float)P.kappa * r);
        const float aa = ai * aj;
        const float f2 = r2 + aa * __expf(-0.25f * __fdividef(r2, aa));
        const float egb = (float)P.gb_coef * qp * rsqrtf(f2);
        const double sig2 = sig64 * sig64;
        if (r2d < sig2) {
            const double s2 = sig2 / r2d, s6 = s2 * s2 * s2;
            double lj = 4.0 * sqrt(eps64) * (s6 * s6 - s6);
            const double rc = sig64 * P.hard_frac, rc2 = rc * rc;
            if (r2d < rc2) {
                const double t2 = rc2 / r2d, t6 = t2 * t2 * t2, x = t6 * t6 - 1.0;
                lj += fmin(P.hard_scale * x * x, P.hard_cap);
            }
            return (float)((double)(edh + egb) + lj);
        }
        const float sr = sig * rinv, s2 = sr * sr, s6 = s2 * s2 * s2;
        return edh + egb + 4.0f * f_sqrt(eps_prod) * (s6 * s6 - s6);
    }
    const R r2 = (R)r2d;
    const R r = m_sqrt(r2);
    const R edh = (R)P.coulomb_over_epsw * qp / r * m_exp(-(R)P.kappa * r);
    const R aa = ai * aj;
    const R fgb = m_sqrt(r2 + aa * m_exp(-r2 / ((R)4 * aa)));
    const R egb = (R)P.gb_coef * qp / fgb;
    const R eps = m_sqrt(eps_prod);
    const R sr = sig / r;
    const R s2 = sr * sr;
    const R s6 = s2 * s2 * s2;
    R E = edh + egb + (R)4 * eps * (s6 * s6 - s6);
    const R r_cut = sig * (R)P.hard_frac;
    if (r < r_cut) {
        const R t = r_cut / r;
        const R t2 = t * t;
        const R t6 = t2 * t2 * t2;
        const R x = t6 * t6 - (R)1;
        const R h = (R)P.hard_scale * x * x;
        E += h < (R)P.hard_cap ? h : (R)P.hard_cap;
    }
    return E;
}

__device__ __forceinline__ float m_expm1(float x) { return expm1f(x); }
__device__ __forceinline__ double m_expm1(double x) { return expm1(x); }
__device__ __forceinline__ float m_log1p(float x) { return log1pf(x); }
__device__ __forceinline__ double m_log1p(double x) { return log1p(x); }

// LJ 12-6 + capped hard core of one pair (r2 in FP64).  Inside sigma the
// terms grow steeply and are evaluated in FP64 with FP64 sigma and
// epsilon (sig64 = R*_i + R*_j, eps64 = eps_i eps_j); outside, in
// precision R.
template <typename R>
__device__ __forceinline__ double lj_hard(const DevParams &P, double r2, R sig, R eps_prod, double sig64,
                                          double eps64) {
    const double sig2 = sig64 * sig64;
    if (r2 < sig2) {
        const double s2 = sig2 / r2, s6 = s2 * s2 * s2;
        double E = 4.0 * sqrt(eps64) * (s6 * s6 - s6);
        const double rc = sig64 * P.hard_frac, rc2 = rc * rc;
        if (r2 < rc2) {
            const double t2 = rc2 / r2, t6 = t2 * t2 * t2, x = t6 * t6 - 1.0;
            E += fmin(P.hard_scale * x * x, P.hard_cap);
        }
        return E;
    }
    const R s2 = (R)(sig2 / r2);
    const R s6 = s2 * s2 * s2;
    return (double)((R)4 * m_sqrt(eps_prod) * (s6 * s6 - s6));
}

// Change of one pair's energy between two geometries (old: r2o, Born
// product aao; new: r2n, aan), both inside the pair cutoff.  Written as a
// difference so the rounding error scales with the change, not with the
// pair energy: r2n - r2o comes from FP64 coordinates,
//   DH: K qq g(ro) expm1(-kappa dr - log1p(dr/ro)),  g(r) = exp(-kappa r)/r
//   GB: C qq (fo^2 - fn^2) / (fo fn (fo + fn)),  f^2 = r^2 + aa exp(-r^2/4aa)
// LJ and the hard core are differenced directly (FP64 inside sigma).
template <typename R>
__device__ __forceinline__ double pair_delta(const DevParams &P, double r2o, double r2n, R qp, R sig, R eps_prod,
                                             R aao, R aan, double sig64, double eps64) {
    if constexpr (sizeof(R) == 4) {
        const double d2 = r2n - r2o;
        const float ro2 = (float)r2o, rn2 = (float)r2n;
        const float rio = rsqrtf(ro2), rin = rsqrtf(rn2);
        const float ro = ro2 * rio, rn = rn2 * rin;
        const float dr = __fdividef((float)d2, ro + rn);
        const float kap = (float)P.kappa;
        const float gdo = (float)P.coulomb_over_epsw * qp * rio * __expf(-kap * ro);
        const float ddh = gdo * expm1f(-kap * dr - log1pf(dr * rio));
        const float xo = aao * __expf(-0.25f * __fdividef(ro2, aao));
        const float xn = aan * __expf(-0.25f * __fdividef(rn2, aan));
        const float fo2 = ro2 + xo, fn2 = rn2 + xn;
        const float fo = fo2 * rsqrtf(fo2), fn = fn2 * rsqrtf(fn2);
        const float num = (float)(-d2) + (xo - xn);
        const float dgb = (float)P.gb_coef * qp * __fdividef(num, fo * fn * (fo + fn));
        return (double)ddh + (double)dgb +
               (lj_hard<float>(P, r2n, sig, eps_prod, sig64, eps64) - lj_hard<float>(P, r2o, sig, eps_prod, sig64, eps64));
    }
    const double d2 = r2n - r2o;
    const R ro2 = (R)r2o, rn2 = (R)r2n;
    const R ro = m_sqrt(ro2), rn = m_sqrt(rn2);
    const R dr = (R)d2 / (ro + rn);
    const R kap = (R)P.kappa;
    const R gdo = (R)P.coulomb_over_epsw * qp / ro * m_exp(-kap * ro);
    const R ddh = gdo * m_expm1(-kap * dr - m_log1p(dr / ro));
    const R xo = aao * m_exp(-ro2 / ((R)4 * aao)), xn = aan * m_exp(-rn2 / ((R)4 * aan));
    const R fo = m_sqrt(ro2 + xo), fn = m_sqrt(rn2 + xn);
    const R num = (R)(-d2) + (xo - xn);
    const R dgb = (R)P.gb_coef * qp * num / (fo * fn * (fo + fn));
    return (double)ddh + (double)dgb +
           (lj_hard<R>(P, r2n, sig, eps_prod, sig64, eps64) - lj_hard<R>(P, r2o, sig, eps_prod, sig64, eps64));
}

// HCT descreening integral of atom j (radius rj) on atom i (radius ri).
template <typename R>
__device__ __forceinline__ R hct_term(R r, R r2, R ri, R rj) {
    if constexpr (sizeof(R) == 4) {
        const float d = fabsf(r - rj);
        const float L = d > ri ? d : ri;
        const float U = r + rj;
        if (ri >= U) return 0.0f;
        const float rU = __fdividef(1.0f, U);
        return __fdividef(1.0f, L) - rU +
               (r2 - rj * rj + ri * ri) * __fdividef(0.25f, r2 * ri * ri) * logf(L * rU);
    }
    const R d = m_abs(r - rj);
    const R L = d > ri ? d : ri;
    const R U = r + rj;
    if (ri >= U) return (R)0;
    return (R)1 / L - (R)1 / U + (r2 - rj * rj + ri * ri) / ((R)2 * r * ri * ri) * m_log(L / U) * (R)0.5 / r;
}

__device__ __forceinline__ double dist2(const double *xyz, int i, int j) {
    const double4 a = *reinterpret_cast<const double4 *>(xyz + 4 * (size_t)i);
    const double4 b = *reinterpret_cast<const double4 *>(xyz + 4 * (size_t)j);
    const double dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
    return dx * dx + dy * dy + dz * dz;
}

__device__ __forceinline__ double4 ld_xyz(const double *xyz, int i) {
    return *reinterpret_cast<const double4 *>(xyz + 4 * (size_t)i);
}

__device__ __forceinline__ double d2_of(double4 a, double4 b) {
    const double dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
    return dx * dx + dy * dy + dz * dz;
}

// ---------------------------------------------------------------------------
// reductions (fixed order: deterministic for a given launch shape)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// ---------------------------------------------------------------------------
// SASA cap recurrence (physics_engine.cpp:2068-2083) over a 32-entry chunk
// of a row: sa -= min(0.85 sa, c_l) for every lane l set in `hits`, in lane
// (= row) order.  The hit values are first packed into lanes 0..n-1 (one
// shuffle from the position of each lane's set bit), then read back by
// index in groups of four: those shuffles do not depend on sa, so they
// issue ahead of the dependent FP64 chain instead of one round trip per
// entry.  The arithmetic and its order are those of the entry-by-entry
// loop, so the result is the same to the bit.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double sasa_pack(unsigned hits, double c, int lane) {
    const int src = lane < __popc(hits) ? (int)__fns(hits, 0, lane + 1) : lane;
    return __shfl_sync(0xffffffffu, c, src);
}

__device__ __forceinline__ double sasa_step(double sa, double c) { return sa - fmin(sa * 0.85, c); }

__device__ __forceinline__ double sasa_chunk(double sa, unsigned hits, double c, int lane) {
    const int n = __popc(hits);
    if (n == 0) return sa;
    const double packed = sasa_pack(hits, c, lane);
    int k = 0;
    for (; k + 4 <= n; k += 4) {
        const double c0 = __shfl_sync(0xffffffffu, packed, k), c1 = __shfl_sync(0xffffffffu, packed, k + 1);
        const double c2 = __shfl_sync(0xffffffffu, packed, k + 2), c3 = __shfl_sync(0xffffffffu, packed, k + 3);
        sa = sasa_step(sasa_step(sasa_step(sasa_step(sa, c0), c1), c2), c3);
    }
    for (; k < n; ++k) sa = sasa_step(sa, __shfl_sync(0xffffffffu, packed, k));
    return sa;
}

// Two independent recurrences (old and new geometry) over the same chunk,
// interleaved.
__device__ __forceinline__ void sasa_chunk2(double &sa_a, unsigned hits_a, double c_a, double &sa_b,
                                            unsigned hits_b, double c_b, int lane) {
    const int na = __popc(hits_a), nb = __popc(hits_b);
    const double pa = sasa_pack(hits_a, c_a, lane), pb = sasa_pack(hits_b, c_b, lane);
    const int n = na < nb ? na : nb;
    int k = 0;
    for (; k + 2 <= n; k += 2) {
        const double a0 = __shfl_sync(0xffffffffu, pa, k), a1 = __shfl_sync(0xffffffffu, pa, k + 1);
        const double b0 = __shfl_sync(0xffffffffu, pb, k), b1 = __shfl_sync(0xffffffffu, pb, k + 1);
        sa_a = sasa_step(sasa_step(sa_a, a0), a1);
        sa_b = sasa_step(sasa_step(sa_b, b0), b1);
    }
    for (int q = k; q < na; ++q) sa_a = sasa_step(sa_a, __shfl_sync(0xffffffffu, pa, q));
    for (int q = k; q < nb; ++q) sa_b = sasa_step(sa_b, __shfl_sync(0xffffffffu, pb, q));
}

// Block-wide sum; every thread gets the result.  smem: >= 32 doubles.
__device__ __forceinline__ double block_sum(double v, double *smem) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) smem[wid] = v;
    __syncthreads();
    double t = (threadIdx.x < (unsigned)nw) ? smem[threadIdx.x] : 0.0;
    if (wid == 0) t = warp_sum(t);
    if (threadIdx.x == 0) smem[0] = t;
    __syncthreads();
    t = smem[0];
    __syncthreads();
    return t;
}

// ---------------------------------------------------------------------------
// Philox4x32-10 counter-based RNG (Salmon, Moraes, Dror, Shaw, "Parallel
// random numbers: as easy as 1, 2, 3", SC'11).  Written from the published
// round function; the oracle's MC driver carries the same restatement.
// ---------------------------------------------------------------------------
struct Philox4 {
    uint32_t v[4];
};

__host__ __device__ __forceinline__ void philox_mulhilo(uint32_t a, uint32_t b, uint32_t &hi, uint32_t &lo) {
    const uint64_t p = (uint64_t)a * (uint64_t)b;
    hi = (uint32_t)(p >> 32);
    lo = (uint32_t)p;
}

__host__ __device__ __forceinline__ Philox4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                                           uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0, lo0, hi1, lo1;
        philox_mulhilo(M0, c0, hi0, lo0);
        philox_mulhilo(M1, c2, hi1, lo1);
        const uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += W0; k1 += W1;
    }
    Philox4 o;
    o.v[0] = c0; o.v[1] = c1; o.v[2] = c2; o.v[3] = c3;
    return o;
}

// 53-bit uniform double in [0, 1) from two 32-bit words.
__host__ __device__ __forceinline__ double u01_from(uint32_t a, uint32_t b) {
    return (double)(((uint64_t)(a >> 5) << 26) | (uint64_t)(b >> 6)) * (1.0 / 9007199254740992.0);
}

// System of global atom i: binary search in atom_off[nsys+1].
__device__ __forceinline__ int sys_of_atom(const int32_t *atom_off, int nsys, int i) {
    int lo = 0, hi = nsys - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (atom_off[mid] <= i) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ void set_status(uint32_t *status, uint32_t bit) {
    if (status) atomicOr(status, bit);
}
