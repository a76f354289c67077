/* TEST INFRASTRUCTURE — the oracle (see alma_oracle.h).
 *
 * A plain-C FP64 restatement of the reference ALMA nonbonded path.  Every
 * function cites the reference lines (src/physics_engine.cpp) whose
 * arithmetic it follows; expression order is kept so the strict build
 * (-fno-fast-math -ffp-contract=off) differs from the reference's
 * -ffast-math build only by last-bit rounding.  Sequential by design: this
 * is the checker, never the thing measured or shipped.
 */
#include "alma_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* Physical constants, physics_engine.cpp:181-196. */
#define COULOMB 332.0636
#define EPS_WATER 78.5
#define EPS_PROT 1.0
#define KAPPA 0.1257
#define GAMMA_SA 0.00542
#define BETA_SA 0.92
#define PROBE_R 1.4
#define NL_CUTOFF 12.0
#define NL_SKIN 2.0
#define NL_RCUT2 ((NL_CUTOFF + NL_SKIN) * (NL_CUTOFF + NL_SKIN))
#define PAIR_CUT2 (NL_CUTOFF * NL_CUTOFF)
#define HALF_SKIN2 ((NL_SKIN * 0.5) * (NL_SKIN * 0.5))
#define HARD_SCALE 1.0e4
#define HARD_CAP 5.0e3
#define HARD_CUTOFF_FRAC 0.6
#define GB_COEF (-0.5 * (1.0 / EPS_PROT - 1.0 / EPS_WATER) * COULOMB)
#define K_SS 600.0  /* :1948 */
#define R0_SS 2.044 /* :1950 */
#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

static inline double dmax(double a, double b) { return a > b ? a : b; }
static inline double dmin(double a, double b) { return a < b ? a : b; }
static inline int imax(int a, int b) { return a > b ? a : b; }
static inline int imin(int a, int b) { return a < b ? a : b; }

static inline double d2(const double *xyz, int i, int j) {
    double dx = xyz[3 * i] - xyz[3 * j], dy = xyz[3 * i + 1] - xyz[3 * j + 1],
           dz = xyz[3 * i + 2] - xyz[3 * j + 2];
    return dx * dx + dy * dy + dz * dz;
}

/* ---- neighbor list: cell list, 27-cell scan (:293-342) ------------------- */
int64_t or_nl_build(int n, const double *xyz, int64_t *row_ptr, int32_t *cols, int64_t cap) {
    row_ptr[0] = 0;
    if (n <= 1) {
        for (int i = 0; i < n; ++i) row_ptr[i + 1] = 0;
        return 0;
    }
    double xlo = xyz[0], xhi = xyz[0], ylo = xyz[1], yhi = xyz[1], zlo = xyz[2], zhi = xyz[2];
    for (int i = 0; i < n; ++i) {
        xlo = dmin(xlo, xyz[3 * i]); xhi = dmax(xhi, xyz[3 * i]);
        ylo = dmin(ylo, xyz[3 * i + 1]); yhi = dmax(yhi, xyz[3 * i + 1]);
        zlo = dmin(zlo, xyz[3 * i + 2]); zhi = dmax(zhi, xyz[3 * i + 2]);
    }
    const double cs = sqrt(NL_RCUT2) + 1e-6;
    const double mg = cs;
    xlo -= mg; ylo -= mg; zlo -= mg;
    double lx = xhi - xlo + 2.0 * mg, ly = yhi - ylo + 2.0 * mg, lz = zhi - zlo + 2.0 * mg;
    int nx = imax(1, (int)ceil(lx / cs));
    int ny = imax(1, (int)ceil(ly / cs));
    int nz = imax(1, (int)ceil(lz / cs));
    size_t ncell = (size_t)nx * (size_t)ny * (size_t)nz;
    int *cx = malloc(sizeof(int) * (size_t)n), *cy = malloc(sizeof(int) * (size_t)n),
        *cz = malloc(sizeof(int) * (size_t)n);
    int64_t *cstart = calloc(ncell + 1, sizeof(int64_t));
    int32_t *cell_atoms = malloc(sizeof(int32_t) * (size_t)n);
    int64_t *fill = malloc(sizeof(int64_t) * ncell);
    for (int i = 0; i < n; ++i) {
        cx[i] = imin(nx - 1, imax(0, (int)floor((xyz[3 * i] - xlo) / cs)));
        cy[i] = imin(ny - 1, imax(0, (int)floor((xyz[3 * i + 1] - ylo) / cs)));
        cz[i] = imin(nz - 1, imax(0, (int)floor((xyz[3 * i + 2] - zlo) / cs)));
        cstart[(size_t)cx[i] + (size_t)nx * ((size_t)cy[i] + (size_t)ny * (size_t)cz[i]) + 1]++;
    }
    for (size_t c = 0; c < ncell; ++c) cstart[c + 1] += cstart[c];
    memcpy(fill, cstart, sizeof(int64_t) * ncell);
    for (int i = 0; i < n; ++i) /* atoms ascend within a cell, as push_back does */
        cell_atoms[fill[(size_t)cx[i] + (size_t)nx * ((size_t)cy[i] + (size_t)ny * (size_t)cz[i])]++] = i;
    int64_t k = 0;
    for (int i = 0; i < n; ++i) {
        for (int dz = -1; dz <= 1; ++dz) {
            int cz2 = cz[i] + dz;
            if (cz2 < 0 || cz2 >= nz) continue;
            for (int dy = -1; dy <= 1; ++dy) {
                int cy2 = cy[i] + dy;
                if (cy2 < 0 || cy2 >= ny) continue;
                for (int dx = -1; dx <= 1; ++dx) {
                    int cx2 = cx[i] + dx;
                    if (cx2 < 0 || cx2 >= nx) continue;
                    size_t c = (size_t)cx2 + (size_t)nx * ((size_t)cy2 + (size_t)ny * (size_t)cz2);
                    for (int64_t q = cstart[c]; q < cstart[c + 1]; ++q) {
                        int j = cell_atoms[q];
                        if (j <= i) continue;
                        if (d2(xyz, i, j) < NL_RCUT2) {
                            if (k < cap) cols[k] = j;
                            ++k;
                        }
                    }
                }
            }
        }
        row_ptr[i + 1] = k;
    }
    free(cx); free(cy); free(cz); free(cstart); free(cell_atoms); free(fill);
    return k <= cap ? k : -k;
}

int or_needs_rebuild(int n, const double *xyz, const double *ref_xyz) {
    for (int i = 0; i < n; ++i) {
        double dx = xyz[3 * i] - ref_xyz[3 * i], dy = xyz[3 * i + 1] - ref_xyz[3 * i + 1],
               dz = xyz[3 * i + 2] - ref_xyz[3 * i + 2];
        if (dx * dx + dy * dy + dz * dz > HALF_SKIN2) return 1;
    }
    return 0;
}

/* ---- HCT integral and Born radii (:2007-2051) ----------------------------- */
double or_hct(double r, double r2, double ri, double rj) {
    double L = dmax(fabs(r - rj), ri), U = r + rj;
    if (ri >= U) return 0.0;
    return 1.0 / L - 1.0 / U + (r2 - rj * rj + ri * ri) / (2.0 * r * ri * ri) * log(L / U) * 0.5 / r;
}

void or_born_radii(int n, const double *xyz, const double *radius, const int64_t *row_ptr,
                   const int32_t *cols, double *a) {
    double *sum = calloc((size_t)n, sizeof(double));
    for (int i = 0; i < n; ++i)
        for (int64_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) {
            int j = cols[k];
            double r2 = d2(xyz, i, j), r = sqrt(r2);
            sum[i] += or_hct(r, r2, radius[i], radius[j]);
            sum[j] += or_hct(r, r2, radius[j], radius[i]);
        }
    for (int i = 0; i < n; ++i) {
        double inv = 1.0 / radius[i] - 0.5 * sum[i];
        a[i] = 1.0 / dmax(inv, 2.0);
    }
    free(sum);
}

void or_update_born(int idx, const double *xyz, const double *radius, const int64_t *row_ptr,
                    const int32_t *cols, double *a) {
    double ri = radius[idx], sum = 0.0;
    for (int64_t k = row_ptr[idx]; k < row_ptr[idx + 1]; ++k) {
        int j = cols[k];
        double r2 = d2(xyz, idx, j), r = sqrt(r2);
        sum += or_hct(r, r2, ri, radius[j]);
    }
    a[idx] = 1.0 / dmax(1.0 / ri - 0.5 * sum, 2.0);
}

/* ---- SASA nonpolar (:2068-2083) ------------------------------------------ */
double or_sasa(int n, const double *xyz, const double *radius, const int64_t *row_ptr,
               const int32_t *cols, double *sa_out) {
    double E = BETA_SA;
    for (int i = 0; i < n; ++i) {
        double ri = radius[i] + PROBE_R, sa = 4.0 * M_PI * ri * ri;
        for (int64_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) {
            int j = cols[k];
            double rj = radius[j] + PROBE_R;
            double r = sqrt(d2(xyz, i, j)), dc = ri + rj;
            if (r >= dc) continue;
            double h = (dc - r) / (2.0 * ri);
            sa -= dmin(sa * 0.85, 2.0 * M_PI * ri * ri * h);
        }
        if (sa_out) sa_out[i] = dmax(0.0, sa);
        E += GAMMA_SA * dmax(0.0, sa);
    }
    return E;
}

/* ---- pair energy (:2148-2164) --------------------------------------------- */
double or_pair_e(const double *pi, const double *pj, double ai, double aj) {
    double dx = pi[0] - pj[0], dy = pi[1] - pj[1], dz = pi[2] - pj[2];
    double r2 = dx * dx + dy * dy + dz * dz, r = sqrt(r2), sig = pi[4] + pj[4];
    double qp = pi[3] * pj[3];
    double edh = (COULOMB * qp) / (EPS_WATER * r) * exp(-KAPPA * r);
    double fgb = sqrt(r2 + ai * aj * exp(-r2 / (4.0 * ai * aj)));
    double egb = GB_COEF * qp / fgb;
    double eps = sqrt(pi[5] * pj[5]), s6 = pow(sig / r, 6);
    double elj = 4.0 * eps * (s6 * s6 - s6);
    double E = edh + egb + elj;
    double r_cut = sig * HARD_CUTOFF_FRAC;
    if (r < r_cut) {
        double x = pow(r_cut / r, 12.0) - 1.0;
        E += dmin(HARD_SCALE * x * x, HARD_CAP);
    }
    return E;
}

/* ---- topology-dependent terms ---------------------------------------------- */
int or_is_excluded(const or_topo *t, int i, int j) { /* :1700-1705, binary search */
    if (!t || i < 0 || j < 0 || i >= t->n || j >= t->n) return 0;
    if (i > j) { int s = i; i = j; j = s; }
    int64_t lo = t->excl_ptr[i], hi = t->excl_ptr[i + 1];
    while (lo < hi) {
        int64_t mid = lo + (hi - lo) / 2;
        if (t->excl_cols[mid] < j) lo = mid + 1;
        else hi = mid;
    }
    return lo < t->excl_ptr[i + 1] && t->excl_cols[lo] == j;
}

double or_dihedral_angle(const double *p, int a, int b, int c, int d) { /* :1871-1887 */
    double b1x = p[3 * a] - p[3 * b], b1y = p[3 * a + 1] - p[3 * b + 1], b1z = p[3 * a + 2] - p[3 * b + 2];
    double b2x = p[3 * c] - p[3 * b], b2y = p[3 * c + 1] - p[3 * b + 1], b2z = p[3 * c + 2] - p[3 * b + 2];
    double b3x = p[3 * d] - p[3 * c], b3y = p[3 * d + 1] - p[3 * c + 1], b3z = p[3 * d + 2] - p[3 * c + 2];
    double n1x = b1y * b2z - b1z * b2y, n1y = b1z * b2x - b1x * b2z, n1z = b1x * b2y - b1y * b2x;
    double n2x = b2y * b3z - b2z * b3y, n2y = b2z * b3x - b2x * b3z, n2z = b2x * b3y - b2y * b3x;
    double m1x = n1y * b2z - n1z * b2y, m1y = n1z * b2x - n1x * b2z, m1z = n1x * b2y - n1y * b2x;
    double x = n1x * n2x + n1y * n2y + n1z * n2z;
    double y = m1x * n2x + m1y * n2y + m1z * n2z;
    return atan2(y, x);
}

static double dih_record_e(const double *xyz, const or_topo *t, int r) {
    const int32_t *q = t->dih_abcd + 4 * r;
    double phi = or_dihedral_angle(xyz, q[0], q[1], q[2], q[3]);
    double E = 0.0;
    for (int k = t->term_off[r]; k < t->term_off[r + 1]; ++k)
        E += t->term_v2[k] * (1.0 + cos((double)t->term_n[k] * phi - t->term_gamma[k]));
    return E;
}

double or_dihedral_e(const double *xyz, const or_topo *t) { /* :1912-1921 */
    double E = 0.0;
    for (int r = 0; r < t->ndih; ++r) E += dih_record_e(xyz, t, r);
    return E;
}

/* :1893-1910, boundary records only (some atoms moving, some fixed). */
static double dihedral_e_boundary(const double *xyz, const or_topo *t, const int8_t *group) {
    double E = 0.0;
    for (int r = 0; r < t->ndih; ++r) {
        const int32_t *q = t->dih_abcd + 4 * r;
        int s_a = group[q[0]] != 0, s_b = group[q[1]] != 0, s_c = group[q[2]] != 0, s_d = group[q[3]] != 0;
        int any_side = s_a || s_b || s_c || s_d;
        int any_fixed = !s_a || !s_b || !s_c || !s_d;
        if (!any_side || !any_fixed) continue;
        E += dih_record_e(xyz, t, r);
    }
    return E;
}

double or_ss_e(const double *xyz, const or_topo *t) { /* :1965-1974 */
    double E = 0.0;
    for (int k = 0; k < t->nss; ++k) {
        double dr = sqrt(d2(xyz, t->ss[2 * k], t->ss[2 * k + 1])) - R0_SS;
        E += K_SS * dr * dr;
    }
    return E;
}

static double ss_e_side(const double *xyz, const or_topo *t, const int8_t *group) { /* :1981-1994 */
    double E = 0.0;
    for (int k = 0; k < t->nss; ++k) {
        int i = t->ss[2 * k], j = t->ss[2 * k + 1];
        if (group[i] == 0 && group[j] == 0) continue;
        double dr = sqrt(d2(xyz, i, j)) - R0_SS;
        E += K_SS * dr * dr;
    }
    return E;
}

static void particle(double *p, const double *xyz, const double *q, const double *radius,
                     const double *eps, int i) {
    p[0] = xyz[3 * i]; p[1] = xyz[3 * i + 1]; p[2] = xyz[3 * i + 2];
    p[3] = q[i]; p[4] = radius[i]; p[5] = eps[i];
}

/* ---- total energy (:2205-2234) --------------------------------------------- */
double or_energy(int n, const double *xyz, const double *q, const double *radius,
                 const double *eps, const int64_t *row_ptr, const int32_t *cols,
                 const double *a, const or_topo *t, double *terms) {
    double sasa = or_sasa(n, xyz, radius, row_ptr, cols, NULL);
    double dih = (t && t->ndih > 0) ? or_dihedral_e(xyz, t) : 0.0;
    double ss = (t && t->nss > 0) ? or_ss_e(xyz, t) : 0.0;
    double pairs = 0.0, pi[6], pj[6];
    for (int i = 0; i < n; ++i)
        for (int64_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) {
            int j = cols[k];
            if (t && or_is_excluded(t, i, j)) continue;
            if (d2(xyz, i, j) > PAIR_CUT2) continue;
            particle(pi, xyz, q, radius, eps, i);
            particle(pj, xyz, q, radius, eps, j);
            pairs += or_pair_e(pi, pj, a[i], a[j]);
        }
    double total = sasa + dih + ss + pairs;
    if (terms) {
        terms[0] = sasa; terms[1] = dih; terms[2] = ss; terms[3] = pairs; terms[4] = total;
    }
    return total;
}

double or_calculate_potential(int n, const double *xyz, const double *q, const double *radius,
                              const double *eps, const or_topo *t, double *terms) {
    if (n <= 0) {
        if (terms) memset(terms, 0, 5 * sizeof(double));
        return 0.0;
    }
    int64_t *row_ptr = malloc(sizeof(int64_t) * (size_t)(n + 1));
    int64_t cap = 64 * (int64_t)n + 64;
    int32_t *cols = malloc(sizeof(int32_t) * (size_t)cap);
    int64_t m = or_nl_build(n, xyz, row_ptr, cols, cap);
    if (m < 0) {
        free(cols);
        cap = -m;
        cols = malloc(sizeof(int32_t) * (size_t)cap);
        or_nl_build(n, xyz, row_ptr, cols, cap);
    }
    double *a = malloc(sizeof(double) * (size_t)n);
    or_born_radii(n, xyz, radius, row_ptr, cols, a);
    double E = or_energy(n, xyz, q, radius, eps, row_ptr, cols, a, t, terms);
    free(a); free(cols); free(row_ptr);
    return E;
}

/* ---- one proposal's ΔE ------------------------------------------------------ */
void or_rodrigues(double *p, const double *o, const double *u, double c, double s) { /* :1848-1862 */
    double vx = p[0] - o[0], vy = p[1] - o[1], vz = p[2] - o[2];
    double dot = u[0] * vx + u[1] * vy + u[2] * vz;
    double cx = u[1] * vz - u[2] * vy;
    double cy = u[2] * vx - u[0] * vz;
    double cz = u[0] * vy - u[1] * vx;
    double k = 1.0 - c;
    p[0] = o[0] + vx * c + cx * s + u[0] * dot * k;
    p[1] = o[1] + vy * c + cy * s + u[1] * dot * k;
    p[2] = o[2] + vz * c + cz * s + u[2] * dot * k;
}

/* The cross_e lambda (:2312-2323) with the side_group generalisation of the
 * concerted-sidechain move (:2782-2796). */
static double cross_e(int n, const double *xyz, const double *q, const double *radius,
                      const double *eps, const int64_t *row_ptr, const int32_t *cols,
                      const double *a, const or_topo *t, const int8_t *group) {
    double E = 0.0, pi[6], pj[6];
    for (int i = 0; i < n; ++i)
        for (int64_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) {
            int j = cols[k];
            if (group[i] == group[j]) continue;
            if (t && or_is_excluded(t, i, j)) continue;
            if (d2(xyz, i, j) > PAIR_CUT2) continue;
            particle(pi, xyz, q, radius, eps, i);
            particle(pj, xyz, q, radius, eps, j);
            E += or_pair_e(pi, pj, a[i], a[j]);
        }
    return E;
}

double or_move_dE(int n, const double *xyz, const double *q, const double *radius,
                  const double *eps, const int64_t *row_ptr, const int32_t *cols,
                  const double *a, const or_topo *t, int nrot, const int32_t *rot_axis,
                  const double *rot_delta, const int64_t *rot_ptr, const int32_t *rot_idx,
                  const int8_t *group, double *terms, double *new_xyz, double *new_a) {
    double *st = malloc(sizeof(double) * 3 * (size_t)n);
    double *aa = malloc(sizeof(double) * (size_t)n);
    memcpy(st, xyz, sizeof(double) * 3 * (size_t)n);
    memcpy(aa, a, sizeof(double) * (size_t)n);
    double before[4], after[4];
    before[0] = cross_e(n, st, q, radius, eps, row_ptr, cols, aa, t, group);
    before[1] = or_sasa(n, st, radius, row_ptr, cols, NULL);
    before[2] = t ? dihedral_e_boundary(st, t, group) : 0.0;
    before[3] = (t && t->nss > 0) ? ss_e_side(st, t, group) : 0.0;
    double result = 0.0;
    for (int r = 0; r < nrot; ++r) {
        int ai = rot_axis[2 * r], aj = rot_axis[2 * r + 1];
        double o[3] = {st[3 * ai], st[3 * ai + 1], st[3 * ai + 2]};
        double u[3] = {st[3 * aj] - o[0], st[3 * aj + 1] - o[1], st[3 * aj + 2] - o[2]};
        double l = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
        if (l < 1e-10) { result = NAN; goto done; }
        u[0] /= l; u[1] /= l; u[2] /= l;
        double c = cos(rot_delta[r]), s = sin(rot_delta[r]);
        for (int64_t k = rot_ptr[r]; k < rot_ptr[r + 1]; ++k) or_rodrigues(st + 3 * rot_idx[k], o, u, c, s);
    }
    for (int i = 0; i < n; ++i)
        if (group[i] != 0) or_update_born(i, st, radius, row_ptr, cols, aa);
    after[0] = cross_e(n, st, q, radius, eps, row_ptr, cols, aa, t, group);
    after[1] = or_sasa(n, st, radius, row_ptr, cols, NULL);
    after[2] = t ? dihedral_e_boundary(st, t, group) : 0.0;
    after[3] = (t && t->nss > 0) ? ss_e_side(st, t, group) : 0.0;
    result = (after[0] - before[0]) + (after[1] - before[1]) + (after[2] - before[2]) + (after[3] - before[3]);
    if (terms)
        for (int k = 0; k < 4; ++k) terms[k] = after[k] - before[k];
    if (new_xyz) memcpy(new_xyz, st, sizeof(double) * 3 * (size_t)n);
    if (new_a) memcpy(new_a, aa, sizeof(double) * (size_t)n);
done:
    free(st); free(aa);
    return result;
}


/* ---- Monte Carlo driver (see alma_oracle.h) ----------------------------------- */
/* Philox4x32-10: Salmon, Moraes, Dror, Shaw, SC'11. */
void or_philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1, uint32_t *out) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)M0 * c0, p1 = (uint64_t)M1 * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0, hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += W0; k1 += W1;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static double u01(uint32_t a, uint32_t b) {
    return (double)(((uint64_t)(a >> 5) << 26) | (uint64_t)(b >> 6)) * (1.0 / 9007199254740992.0);
}

static int pick_index(double u, int n) {
    int k = (int)(u * (double)n);
    return k < n ? k : n - 1;
}

typedef struct {
    int64_t *row_ptr;
    int32_t *cols;
    int64_t cap;
    double *ref;
} mc_nl;

static void mc_rebuild(or_mc_sys *S, mc_nl *nl, or_mc_state *st) {
    int64_t m = or_nl_build(S->n, S->xyz, nl->row_ptr, nl->cols, nl->cap);
    if (m < 0) {
        free(nl->cols);
        nl->cap = -m + 1024;
        nl->cols = malloc(sizeof(int32_t) * (size_t)nl->cap);
        or_nl_build(S->n, S->xyz, nl->row_ptr, nl->cols, nl->cap);
    }
    memcpy(nl->ref, S->xyz, sizeof(double) * 3 * (size_t)S->n);
    or_born_radii(S->n, S->xyz, S->radius, nl->row_ptr, nl->cols, S->born);
    st->energy = or_energy(S->n, S->xyz, S->q, S->radius, S->eps, nl->row_ptr, nl->cols, S->born, S->topo, NULL);
}

void or_mc_run(or_mc_sys *S, const or_mc_cfg *cfg, or_mc_state *st, int64_t step_limit) {
    const int n = S->n;
    mc_nl nl;
    nl.row_ptr = malloc(sizeof(int64_t) * (size_t)(n + 1));
    nl.cap = 256 * (int64_t)n + 64;
    nl.cols = malloc(sizeof(int32_t) * (size_t)nl.cap);
    nl.ref = malloc(sizeof(double) * 3 * (size_t)n);
    mc_rebuild(S, &nl, st); /* every call starts from a fresh list, as a chain does */
    int8_t *group = calloc((size_t)n, 1);
    double *new_xyz = malloc(sizeof(double) * 3 * (size_t)n);
    double *new_born = malloc(sizeof(double) * (size_t)n);
    int32_t axis[4];
    double dl[2];
    int64_t rptr[3];
    int32_t *ridx = malloc(sizeof(int32_t) * 2 * (size_t)n + 8);
    const uint32_t k0 = (uint32_t)cfg->seed ^ (0x9E3779B9u * (uint32_t)(S->sys_index + 1)),
                   k1 = (uint32_t)(cfg->seed >> 32);
    while (st->step < step_limit) {
        if (st->need_rebuild) {
            mc_rebuild(S, &nl, st);
            st->need_rebuild = 0;
            st->n_rebuild++;
        }
        const uint64_t sp = (uint64_t)st->step;
        uint32_t w0[4], w1[4], w2[4];
        or_philox((uint32_t)sp, (uint32_t)(sp >> 32), (uint32_t)S->sys_index, 0u, k0, k1, w0);
        or_philox((uint32_t)sp, (uint32_t)(sp >> 32), (uint32_t)S->sys_index, 1u, k0, k1, w1);
        or_philox((uint32_t)sp, (uint32_t)(sp >> 32), (uint32_t)S->sys_index, 2u, k0, k1, w2);
        const double u[6] = {u01(w0[0], w0[1]), u01(w0[2], w0[3]), u01(w1[0], w1[1]),
                             u01(w1[2], w1[3]), u01(w2[0], w2[1]), u01(w2[2], w2[3])};
        int conc = 0, crank = 0, kind = -1, nrot = 0;
        dl[0] = dl[1] = 0.0;
        if (cfg->policy == 1) {
            conc = S->ncsp > 0 && u[0] < cfg->concerted_prob;
            crank = !conc && S->ncp > 0 && u[4] < cfg->crank_prob;
        } else if (cfg->policy == 0) {
            crank = S->ncp > 0 && u[0] < cfg->crank_prob;
        }
        int ka = -1, kb = -1;
        if (conc) {
            kind = 2;
            const int p = pick_index(u[1], S->ncsp);
            ka = S->csp[2 * p];
            kb = S->csp[2 * p + 1];
            const double da = st->cur_max * cfg->sidechain_mult * S->rb_scale[ka];
            const double db = st->cur_max * cfg->sidechain_mult * S->rb_scale[kb];
            dl[0] = -da + 2.0 * da * u[2];
            dl[1] = -db + 2.0 * db * u[5];
        } else if (crank) {
            kind = 1;
            const int p = pick_index(u[1], S->ncp);
            ka = S->cp[2 * p];
            kb = S->cp[2 * p + 1];
            dl[0] = -st->cur_max + 2.0 * st->cur_max * u[2];
        } else {
            const int nset = cfg->nset > 0 ? cfg->nset : S->nrb;
            if (nset > 0) {
                kind = 0;
                const int q = pick_index(u[1], nset);
                ka = cfg->nset > 0 ? cfg->moveset[q] : q;
                const int bk = S->rb_kind[ka];
                double base = (bk == 0 || bk == 1) ? st->cur_max : st->cur_max * cfg->sidechain_mult;
                base *= S->rb_scale[ka];
                dl[0] = -base + 2.0 * base * u[2];
            }
        }
        if (cfg->fixed_delta > 0.0) {
            dl[0] = cfg->fixed_delta * (2.0 * u[2] - 1.0);
            dl[1] = cfg->fixed_delta * (2.0 * u[5] - 1.0);
        }
        if (kind < 0) { st->step++; continue; }
        /* rotations and groups */
        int64_t pos = 0;
        rptr[0] = 0;
        const int32_t *sa = S->side_idx + S->side_ptr[ka];
        const int64_t na = S->side_ptr[ka + 1] - S->side_ptr[ka];
        double rdelta[2];
        if (kind == 0) {
            axis[0] = S->rb_ij[2 * ka]; axis[1] = S->rb_ij[2 * ka + 1];
            rdelta[0] = dl[0];
            for (int64_t k = 0; k < na; ++k) { ridx[pos++] = sa[k]; group[sa[k]] = 1; }
            rptr[1] = pos;
            nrot = 1;
        } else {
            const int32_t *sb = S->side_idx + S->side_ptr[kb];
            const int64_t nb = S->side_ptr[kb + 1] - S->side_ptr[kb];
            axis[0] = S->rb_ij[2 * ka]; axis[1] = S->rb_ij[2 * ka + 1];
            axis[2] = S->rb_ij[2 * kb]; axis[3] = S->rb_ij[2 * kb + 1];
            rdelta[0] = dl[0];
            rdelta[1] = kind == 1 ? -dl[0] : dl[1];
            for (int64_t k = 0; k < na; ++k) { ridx[pos++] = sa[k]; group[sa[k]] = 1; }
            rptr[1] = pos;
            for (int64_t k = 0; k < nb; ++k) { ridx[pos++] = sb[k]; if (kind == 2) group[sb[k]] = 2; }
            rptr[2] = pos;
            nrot = 2;
            if (na == 0 || nb == 0) { memset(group, 0, (size_t)n); st->step++; continue; }
        }
        if (na == 0) { memset(group, 0, (size_t)n); st->step++; continue; }
        double terms[4];
        const double dE = or_move_dE(n, S->xyz, S->q, S->radius, S->eps, nl.row_ptr, nl.cols, S->born, S->topo, nrot,
                                     axis, rdelta, rptr, ridx, group, terms, new_xyz, new_born);
        if (dE != dE) { /* degenerate axis */
            memset(group, 0, (size_t)n);
            st->step++;
            continue;
        }
        const int acc = (dE < 0.0) || (u[3] < exp(-dE / st->temperature));
        int drift = 0;
        if (acc) {
            for (int i = 0; i < n; ++i)
                if (group[i]) {
                    S->xyz[3 * i] = new_xyz[3 * i];
                    S->xyz[3 * i + 1] = new_xyz[3 * i + 1];
                    S->xyz[3 * i + 2] = new_xyz[3 * i + 2];
                    S->born[i] = new_born[i];
                    double dx = S->xyz[3 * i] - nl.ref[3 * i], dy = S->xyz[3 * i + 1] - nl.ref[3 * i + 1],
                           dz = S->xyz[3 * i + 2] - nl.ref[3 * i + 2];
                    if (dx * dx + dy * dy + dz * dz > HALF_SKIN2) drift = 1;
                }
            st->energy += dE;
            st->n_accepted++;
            if (drift) st->need_rebuild = 1;
        }
        memset(group, 0, (size_t)n);
        st->n_proposed++;
        st->acc_win += acc;
        if (cfg->tune_freq > 0 && ++st->tot_win == cfg->tune_freq) {
            const double rate = (double)st->acc_win / (double)cfg->tune_freq;
            if (rate > cfg->target_hi) st->cur_max = dmin(cfg->angle_max, st->cur_max * cfg->scale_up);
            else if (rate < cfg->target_lo) st->cur_max = dmax(cfg->angle_min, st->cur_max * cfg->scale_down);
            st->acc_win = 0;
            st->tot_win = 0;
        }
        st->step++;
    }
    free(group); free(new_xyz); free(new_born); free(ridx);
    free(nl.row_ptr); free(nl.cols); free(nl.ref);
}
