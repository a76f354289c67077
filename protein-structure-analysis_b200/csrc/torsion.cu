// Torsion-space kinematics and the gradient-guided (MALA) torsion sampler.
//
// The sampler's coordinates are the rotatable-bond torsions: rotating bond
// k by θ turns its j-side about the axis x_i -> x_j (the reference's move,
// rodrigues physics_engine.cpp:1848-1862).  On a tree the j-sides are
// nested or disjoint (AlmaTorsionTree), which gives
//
//   gradient  dE/dθ_k = u_k · Σ_{m in side k} (x_m - x_i) × ∇_m E, from one
//             prefix sum per system over atoms of ((x_m - c) × ∇_m E, ∇_m E)
//             (a j-side is a range plus a few explicit atoms);
//   apply     all bonds at once: with every axis taken from the current
//             coordinates, turning the innermost bonds first equals the
//             reference's one-after-the-other moves with updated axes, so
//             atom m moves by T_k = A_root ∘ ... ∘ A_parent ∘ A_k, k = the
//             innermost bond holding m.  T is built per bond by pointer
//             jumping (log2(depth) rounds) inside one CTA per system;
//   MALA      θ' = θ + clip(-½ σ² β ∇_θE, ±c σ) + σ ξ per bond (σ_k =
//             state scale × step × lever scale), accepted with the
//             Metropolis–Hastings ratio of the Langevin proposal densities;
//             Philox draws keyed by (seed, system, step, bond).
#include <algorithm>

#include "alma_common.cuh"

namespace alma {

struct Affine {
    double m[12];  // row-major 3x3 rotation, then translation
};

__device__ __forceinline__ Affine affine_compose(const Affine &A, const Affine &B) {  // A ∘ B
    Affine C;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
#pragma unroll
        for (int c = 0; c < 3; ++c)
            C.m[3 * r + c] = A.m[3 * r] * B.m[c] + A.m[3 * r + 1] * B.m[3 + c] + A.m[3 * r + 2] * B.m[6 + c];
        C.m[9 + r] = A.m[3 * r] * B.m[9] + A.m[3 * r + 1] * B.m[10] + A.m[3 * r + 2] * B.m[11] + A.m[9 + r];
    }
    return C;
}

__device__ __forceinline__ void affine_load(Affine &A, const double *p) {
#pragma unroll
    for (int q = 0; q < 12; ++q) A.m[q] = p[q];
}

__device__ __forceinline__ void affine_store(const Affine &A, double *p) {
#pragma unroll
    for (int q = 0; q < 12; ++q) p[q] = A.m[q];
}

// Rotation by angle d about the unit axis through o along (pj - pi).
__device__ __forceinline__ Affine bond_rotation(double4 pi, double4 pj, double d) {
    Affine A;
    double ux = pj.x - pi.x, uy = pj.y - pi.y, uz = pj.z - pi.z;
    const double l = sqrt(ux * ux + uy * uy + uz * uz);
    if (d == 0.0 || l < 1e-10) {
        for (int q = 0; q < 12; ++q) A.m[q] = 0.0;
        A.m[0] = A.m[4] = A.m[8] = 1.0;
        return A;
    }
    ux /= l; uy /= l; uz /= l;
    const double c = cos(d), s = sin(d), k = 1.0 - c;
    A.m[0] = c + ux * ux * k;      A.m[1] = ux * uy * k - uz * s; A.m[2] = ux * uz * k + uy * s;
    A.m[3] = uy * ux * k + uz * s; A.m[4] = c + uy * uy * k;      A.m[5] = uy * uz * k - ux * s;
    A.m[6] = uz * ux * k - uy * s; A.m[7] = uz * uy * k + ux * s; A.m[8] = c + uz * uz * k;
    A.m[9] = pi.x - (A.m[0] * pi.x + A.m[1] * pi.y + A.m[2] * pi.z);
    A.m[10] = pi.y - (A.m[3] * pi.x + A.m[4] * pi.y + A.m[5] * pi.z);
    A.m[11] = pi.z - (A.m[6] * pi.x + A.m[7] * pi.y + A.m[8] * pi.z);
    return A;
}

constexpr int TORSION_THREADS = 1024;

// One CTA per system: T_k for every bond of the system into Tout.
__global__ void __launch_bounds__(TORSION_THREADS)
torsion_compose_kernel(const double *__restrict__ xyz, AlmaTopo t, const int32_t *__restrict__ rb_parent,
                       const double *__restrict__ delta, const uint8_t *__restrict__ mask, int nrb_total,
                       double *__restrict__ Tbuf, int32_t *__restrict__ Pbuf) {
    const int s = blockIdx.x;
    if (mask && !mask[s]) return;
    const int r0 = t.rb_off[s], nr = t.rb_off[s + 1] - r0;
    double *T[2] = {Tbuf + 12 * (size_t)r0, Tbuf + 12 * ((size_t)nrb_total + r0)};
    int32_t *Pp[2] = {Pbuf + r0, Pbuf + nrb_total + r0};
    for (int k = threadIdx.x; k < nr; k += blockDim.x) {
        const int g = r0 + k;
        const Affine A = bond_rotation(ld_xyz(xyz, t.rb_ij[2 * g]), ld_xyz(xyz, t.rb_ij[2 * g + 1]), delta[g]);
        affine_store(A, T[0] + 12 * (size_t)k);
        Pp[0][k] = rb_parent[g];
    }
    int cur = 0;
    for (int round = 0; round < 32; ++round) {
        bool any = false;
        __syncthreads();
        for (int k = threadIdx.x; k < nr; k += blockDim.x) {
            const int p = Pp[cur][k];
            Affine Tk;
            affine_load(Tk, T[cur] + 12 * (size_t)k);
            if (p >= 0) {
                Affine Tp;
                affine_load(Tp, T[cur] + 12 * (size_t)p);
                Tk = affine_compose(Tp, Tk);
                Pp[cur ^ 1][k] = Pp[cur][p];
                any = true;
            } else {
                Pp[cur ^ 1][k] = -1;
            }
            affine_store(Tk, T[cur ^ 1] + 12 * (size_t)k);
        }
        cur ^= 1;
        if (!__syncthreads_or(any)) break;
    }
    if (cur == 1) {  // the result lives in buffer 0
        __syncthreads();
        for (int q = threadIdx.x; q < 12 * nr; q += blockDim.x) T[0][q] = T[1][q];
    }
}

__global__ void torsion_move_atoms_kernel(int natoms, int nsys, const int32_t *__restrict__ atom_off,
                                          const int32_t *__restrict__ rb_off, const int32_t *__restrict__ atom_rb,
                                          const uint8_t *__restrict__ mask, const double *__restrict__ Tbuf,
                                          double *__restrict__ xyz) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= natoms) return;
    const int k = atom_rb[m];
    if (k < 0) return;
    const int s = sys_of_atom(atom_off, nsys, m);
    if (mask && !mask[s]) return;
    Affine T;
    affine_load(T, Tbuf + 12 * ((size_t)rb_off[s] + k));
    double4 p = ld_xyz(xyz, m);
    const double x = p.x, y = p.y, z = p.z;
    p.x = T.m[0] * x + T.m[1] * y + T.m[2] * z + T.m[9];
    p.y = T.m[3] * x + T.m[4] * y + T.m[5] * z + T.m[10];
    p.z = T.m[6] * x + T.m[7] * y + T.m[8] * z + T.m[11];
    *reinterpret_cast<double4 *>(xyz + 4 * (size_t)m) = p;
}

struct V6 {
    double v[6];
};

__device__ __forceinline__ V6 v6_add(const V6 &a, const V6 &b) {
    V6 c;
#pragma unroll
    for (int q = 0; q < 6; ++q) c.v[q] = a.v[q] + b.v[q];
    return c;
}

// Inclusive block scan of V6 (blockDim.x multiple of 32, <= 1024).
__device__ __forceinline__ V6 block_scan6(V6 x, V6 *sm, V6 &total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        V6 y;
#pragma unroll
        for (int q = 0; q < 6; ++q) y.v[q] = __shfl_up_sync(0xffffffffu, x.v[q], o);
        if (lane >= o) x = v6_add(x, y);
    }
    if (lane == 31) sm[wid] = x;
    __syncthreads();
    if (wid == 0) {
        V6 w;
#pragma unroll
        for (int q = 0; q < 6; ++q) w.v[q] = lane < nw ? sm[lane].v[q] : 0.0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            V6 y;
#pragma unroll
            for (int q = 0; q < 6; ++q) y.v[q] = __shfl_up_sync(0xffffffffu, w.v[q], o);
            if (lane >= o) w = v6_add(w, y);
        }
        sm[lane] = w;  // inclusive warp-total prefix
    }
    __syncthreads();
    if (wid > 0) x = v6_add(x, sm[wid - 1]);
    total = sm[nw - 1];
    __syncthreads();
    return x;
}

// One CTA per system: prefix sums of ((x_m - c) × g_m, g_m), then the
// torsion derivative of every bond.
__global__ void __launch_bounds__(TORSION_THREADS)
torsion_grad_kernel(const int32_t *__restrict__ atom_off, const double *__restrict__ xyz,
                    const double *__restrict__ grad, AlmaTopo t, const uint8_t *__restrict__ mask,
                    double *__restrict__ P, double *__restrict__ gtheta) {
    __shared__ V6 sm[32];
    const int s = blockIdx.x;
    if (mask && !mask[s]) return;
    const int a0 = atom_off[s], a1 = atom_off[s + 1];
    if (a1 <= a0) return;
    double *Ps = P + 6 * ((size_t)a0 + s);  // [a1 - a0 + 1] exclusive prefixes
    const double4 c = ld_xyz(xyz, a0);
    V6 carry;
    for (int q = 0; q < 6; ++q) carry.v[q] = 0.0;
    for (int base = a0; base < a1; base += blockDim.x) {
        const int m = base + threadIdx.x;
        V6 x;
        if (m < a1) {
            const double4 p = ld_xyz(xyz, m), g = ld_xyz(grad, m);
            const double rx = p.x - c.x, ry = p.y - c.y, rz = p.z - c.z;
            x.v[0] = ry * g.z - rz * g.y;
            x.v[1] = rz * g.x - rx * g.z;
            x.v[2] = rx * g.y - ry * g.x;
            x.v[3] = g.x; x.v[4] = g.y; x.v[5] = g.z;
        } else {
            for (int q = 0; q < 6; ++q) x.v[q] = 0.0;
        }
        V6 tot;
        const V6 inc = block_scan6(x, sm, tot);
        if (m < a1)
            for (int q = 0; q < 6; ++q) Ps[6 * (size_t)(m - a0) + q] = carry.v[q] + inc.v[q] - x.v[q];
        carry = v6_add(carry, tot);
    }
    if (threadIdx.x == 0)
        for (int q = 0; q < 6; ++q) Ps[6 * (size_t)(a1 - a0) + q] = carry.v[q];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    for (int k = t.rb_off[s] + (threadIdx.x >> 5); k < t.rb_off[s + 1]; k += blockDim.x >> 5) {
        V6 S;
        for (int q = 0; q < 6; ++q) S.v[q] = 0.0;
        for (int64_t e = t.side_ptr[k] + lane; e < t.side_ptr[k + 1]; e += 32) {
            const int m = t.side_idx[e];
            const double4 p = ld_xyz(xyz, m), g = ld_xyz(grad, m);
            const double rx = p.x - c.x, ry = p.y - c.y, rz = p.z - c.z;
            S.v[0] += ry * g.z - rz * g.y;
            S.v[1] += rz * g.x - rx * g.z;
            S.v[2] += rx * g.y - ry * g.x;
            S.v[3] += g.x; S.v[4] += g.y; S.v[5] += g.z;
        }
        for (int q = 0; q < 6; ++q) S.v[q] = warp_sum(S.v[q]);
        if (lane == 0) {
            const int lo = t.side_lo[k], hi = t.side_hi[k];
            if (hi > lo)
                for (int q = 0; q < 6; ++q)
                    S.v[q] += Ps[6 * (size_t)(hi - a0) + q] - Ps[6 * (size_t)(lo - a0) + q];
            const double4 pi = ld_xyz(xyz, t.rb_ij[2 * k]), pj = ld_xyz(xyz, t.rb_ij[2 * k + 1]);
            double ux = pj.x - pi.x, uy = pj.y - pi.y, uz = pj.z - pi.z;
            const double l = sqrt(ux * ux + uy * uy + uz * uz);
            double gk = 0.0;
            if (l >= 1e-10) {
                ux /= l; uy /= l; uz /= l;
                const double ox = pi.x - c.x, oy = pi.y - c.y, oz = pi.z - c.z;
                // Σ (x - o) × g = Σ (x - c) × g - (o - c) × Σ g
                const double tx = S.v[0] - (oy * S.v[5] - oz * S.v[4]);
                const double ty = S.v[1] - (oz * S.v[3] - ox * S.v[5]);
                const double tz = S.v[2] - (ox * S.v[4] - oy * S.v[3]);
                gk = ux * tx + uy * ty + uz * tz;
            }
            gtheta[k] = gk;
        }
    }
}

// ---- MALA ------------------------------------------------------------------
__device__ __forceinline__ int sys_of_bond(const int32_t *rb_off, int nsys, int k) {
    return sys_of_atom(rb_off, nsys, k);  // same search over the [nsys+1] offsets
}

__device__ __forceinline__ void mala_key(uint64_t seed, int s, uint32_t &k0, uint32_t &k1) {
    k0 = (uint32_t)seed ^ (0x85EBCA6Bu * (uint32_t)(s + 1));
    k1 = (uint32_t)(seed >> 32) ^ 0x27D4EB2Fu;
}

// Truncated Langevin drift of bond k (MALTA: Roberts & Tweedie, Bernoulli
// 2:341, 1996): -½ σ² β g clipped to ±clip·σ.  Steep clashes give
// gradients of 1e3-1e6 kcal/mol/rad whose untruncated drift would throw
// the proposal far away; any deterministic drift keeps detailed balance as
// long as the same function enters the forward and reverse densities.
__device__ __forceinline__ double mala_drift(double sg, double beta, double g, double clip) {
    const double mu = -0.5 * sg * sg * beta * g, lim = clip * sg;
    return fmin(fmax(mu, -lim), lim);
}

__global__ void mala_propose_kernel(int nrb, int nsys, const int32_t *__restrict__ rb_off,
                                    const double *__restrict__ gtheta, const double *__restrict__ sigma,
                                    const AlmaMalaState *__restrict__ st, AlmaMalaConfig cfg,
                                    const uint8_t *__restrict__ mask, double *__restrict__ delta) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nrb) return;
    const int s = sys_of_bond(rb_off, nsys, k);
    if (mask && !mask[s]) return;
    const double sg = sigma[k] * st[s].scale;
    if (!(sg > 0.0)) {
        delta[k] = 0.0;
        return;
    }
    const int kl = k - rb_off[s];
    const uint64_t step = (uint64_t)st[s].step;
    uint32_t k0, k1;
    mala_key(cfg.seed, s, k0, k1);
    const Philox4 r = philox4x32_10((uint32_t)step, (uint32_t)(step >> 32), (uint32_t)s,
                                    0x40000000u + ((uint32_t)kl >> 1), k0, k1);
    // Box–Muller: two normals per draw, bond parity picks one
    const double u1 = 1.0 - u01_from(r.v[0], r.v[1]), u2 = u01_from(r.v[2], r.v[3]);
    const double rad = sqrt(-2.0 * log(u1));
    const double xi = (kl & 1) ? rad * sin(6.283185307179586 * u2) : rad * cos(6.283185307179586 * u2);
    delta[k] = mala_drift(sg, st[s].beta, gtheta[k], cfg.drift_clip) + sg * xi;
}

// One CTA per system: Metropolis–Hastings test of the Langevin proposal,
// then the step-scale adaptation window.
__global__ void mala_accept_kernel(int nsys, const int32_t *__restrict__ rb_off, const double *__restrict__ delta,
                                   const double *__restrict__ g_old, const double *__restrict__ g_new,
                                   const double *__restrict__ sigma, const double *__restrict__ terms_new,
                                   AlmaMalaConfig cfg, const uint8_t *__restrict__ mask,
                                   AlmaMalaState *__restrict__ st, uint8_t *__restrict__ accept) {
    __shared__ double sm[32];
    const int s = blockIdx.x;
    if (mask && !mask[s]) return;
    const double beta = st[s].beta, scale = st[s].scale;
    double fwd = 0.0, rev = 0.0;
    for (int k = rb_off[s] + threadIdx.x; k < rb_off[s + 1]; k += blockDim.x) {
        const double sg = sigma[k] * scale;
        if (!(sg > 0.0)) continue;
        const double rf = delta[k] - mala_drift(sg, beta, g_old[k], cfg.drift_clip);
        const double rr = -delta[k] - mala_drift(sg, beta, g_new[k], cfg.drift_clip);
        fwd += rf * rf / (2.0 * sg * sg);
        rev += rr * rr / (2.0 * sg * sg);
    }
    fwd = block_sum(fwd, sm);
    rev = block_sum(rev, sm);
    if (threadIdx.x == 0) {
        AlmaMalaState S = st[s];
        const double En = terms_new[5 * (size_t)s + 4];
        const double log_alpha = -beta * (En - S.energy) - rev + fwd;
        uint32_t k0, k1;
        mala_key(cfg.seed, s, k0, k1);
        const Philox4 r = philox4x32_10((uint32_t)S.step, (uint32_t)(S.step >> 32), (uint32_t)s, 0x3FFFFFFFu, k0, k1);
        const double u = u01_from(r.v[0], r.v[1]);
        const int acc = isfinite(En) && isfinite(log_alpha) && (log_alpha >= 0.0 || log(u) < log_alpha);
        accept[s] = (uint8_t)acc;
        S.log_alpha = log_alpha;
        S.n_proposed++;
        if (acc) {
            S.energy = En;
            S.n_accepted++;
        }
        S.acc_win += acc;
        if (cfg.tune_freq > 0 && ++S.tot_win == cfg.tune_freq) {
            const double rate = (double)S.acc_win / (double)cfg.tune_freq;
            if (rate > cfg.target_hi) S.scale = fmin(cfg.scale_max, S.scale * cfg.scale_up);
            else if (rate < cfg.target_lo) S.scale = fmax(cfg.scale_min, S.scale * cfg.scale_down);
            S.acc_win = 0;
            S.tot_win = 0;
        }
        S.step++;
        st[s] = S;
    }
}

// Rejected systems take back their saved coordinates and Born radii;
// accepted systems take the proposal's torsion gradient.
__global__ void mala_select_kernel(int natoms, int nrb, int nsys, const int32_t *__restrict__ atom_off,
                                   const int32_t *__restrict__ rb_off, const uint8_t *__restrict__ accept,
                                   const uint8_t *__restrict__ mask, const double *__restrict__ xyz_old,
                                   const double *__restrict__ born_old, double *__restrict__ xyz,
                                   double *__restrict__ born, const double *__restrict__ g_new,
                                   double *__restrict__ g_cur) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < natoms) {
        const int s = sys_of_atom(atom_off, nsys, q);
        if ((!mask || mask[s]) && !accept[s]) {
            *reinterpret_cast<double4 *>(xyz + 4 * (size_t)q) = ld_xyz(xyz_old, q);
            born[q] = born_old[q];
        }
    }
    if (q < nrb && g_new && g_cur) {
        const int s = sys_of_bond(rb_off, nsys, q);
        if ((!mask || mask[s]) && accept[s]) g_cur[q] = g_new[q];
    }
}

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace alma

using namespace alma;

extern "C" size_t alma_torsion_workspace_bytes(int32_t natoms, int32_t nsys, int32_t nrb) {
    const size_t n = natoms > 0 ? (size_t)natoms : 0, S = nsys > 0 ? (size_t)nsys : 0, r = nrb > 0 ? (size_t)nrb : 0;
    const size_t compose = align256(sizeof(double) * 24 * r) + align256(sizeof(int32_t) * 2 * r);
    const size_t prefix = align256(sizeof(double) * 6 * (n + S));
    return std::max(compose, prefix) + 256;
}

static int torsion_args(const AlmaBatch *b, const AlmaTopo *t, const char *who) {
    if (!b || !t || b->nsys <= 0 || b->natoms < 0 || !b->atom_off || !b->xyz)
        return alma_set_error(ALMA_EINVAL, "%s: bad arguments", who);
    if (t->nrb > 0 && (!t->rb_off || !t->rb_ij || !t->side_ptr || !t->side_lo || !t->side_hi))
        return alma_set_error(ALMA_EINVAL, "%s: topology without rotatable-bond arrays", who);
    if (!t->rb_off) return alma_set_error(ALMA_EINVAL, "%s: topology without rb_off", who);
    return ALMA_OK;
}

extern "C" int alma_torsion_grad(const AlmaBatch *b, const AlmaTopo *t, const double *grad, const uint8_t *sys_mask,
                                 void *workspace, double *gtheta, void *stream) {
    int rc = torsion_args(b, t, "alma_torsion_grad");
    if (rc) return rc;
    if (!grad || !gtheta || !workspace) return alma_set_error(ALMA_EINVAL, "alma_torsion_grad: null buffer");
    if (b->natoms == 0 || t->nrb == 0) return ALMA_OK;
    torsion_grad_kernel<<<b->nsys, TORSION_THREADS, 0, (cudaStream_t)stream>>>(
        b->atom_off, b->xyz, grad, *t, sys_mask, (double *)workspace, gtheta);
    ALMA_LAUNCH_CHECK("alma_torsion_grad");
    return ALMA_OK;
}

extern "C" int alma_torsion_apply(const AlmaBatch *b, const AlmaTopo *t, const AlmaTorsionTree *tree,
                                  const double *delta, const uint8_t *sys_mask, void *workspace, void *stream) {
    int rc = torsion_args(b, t, "alma_torsion_apply");
    if (rc) return rc;
    if (!tree || !tree->rb_parent || !tree->atom_rb || !delta || !workspace)
        return alma_set_error(ALMA_EINVAL, "alma_torsion_apply: null buffer");
    if (b->natoms == 0 || t->nrb == 0) return ALMA_OK;
    cudaStream_t st = (cudaStream_t)stream;
    double *Tbuf = (double *)workspace;
    int32_t *Pbuf = (int32_t *)((char *)workspace + align256(sizeof(double) * 24 * (size_t)t->nrb));
    torsion_compose_kernel<<<b->nsys, TORSION_THREADS, 0, st>>>(b->xyz, *t, tree->rb_parent, delta, sys_mask, t->nrb,
                                                                Tbuf, Pbuf);
    torsion_move_atoms_kernel<<<(b->natoms + 255) / 256, 256, 0, st>>>(b->natoms, b->nsys, b->atom_off, t->rb_off,
                                                                       tree->atom_rb, sys_mask, Tbuf, b->xyz);
    ALMA_LAUNCH_CHECK_N("alma_torsion_apply", 2);
    return ALMA_OK;
}

extern "C" int alma_mala_propose(const AlmaTopo *t, int32_t nsys, const double *gtheta, const double *sigma,
                                 const AlmaMalaConfig *cfg, const AlmaMalaState *states, const uint8_t *sys_mask,
                                 double *delta, void *stream) {
    if (!t || nsys <= 0 || !t->rb_off || !gtheta || !sigma || !cfg || !states || !delta)
        return alma_set_error(ALMA_EINVAL, "alma_mala_propose: bad arguments");
    if (t->nrb == 0) return ALMA_OK;
    mala_propose_kernel<<<(t->nrb + 255) / 256, 256, 0, (cudaStream_t)stream>>>(t->nrb, nsys, t->rb_off, gtheta,
                                                                                sigma, states, *cfg, sys_mask, delta);
    ALMA_LAUNCH_CHECK("alma_mala_propose");
    return ALMA_OK;
}

extern "C" int alma_mala_accept(const AlmaTopo *t, int32_t nsys, const double *delta, const double *g_old,
                                const double *g_new, const double *sigma, const double *terms_new,
                                const AlmaMalaConfig *cfg, const uint8_t *sys_mask, AlmaMalaState *states,
                                uint8_t *accept, void *stream) {
    if (!t || nsys <= 0 || !t->rb_off || !delta || !g_old || !g_new || !sigma || !terms_new || !cfg || !states ||
        !accept)
        return alma_set_error(ALMA_EINVAL, "alma_mala_accept: bad arguments");
    mala_accept_kernel<<<nsys, 256, 0, (cudaStream_t)stream>>>(nsys, t->rb_off, delta, g_old, g_new, sigma, terms_new,
                                                               *cfg, sys_mask, states, accept);
    ALMA_LAUNCH_CHECK("alma_mala_accept");
    return ALMA_OK;
}

extern "C" int alma_mala_select(AlmaBatch *b, const AlmaTopo *t, const uint8_t *accept, const uint8_t *sys_mask,
                                const double *xyz_old, const double *born_old, const double *g_new, double *g_cur,
                                void *stream) {
    if (!b || !t || !t->rb_off || !accept || !xyz_old || !born_old || !b->xyz || !b->born)
        return alma_set_error(ALMA_EINVAL, "alma_mala_select: bad arguments");
    const int n = std::max(b->natoms, t->nrb);
    if (n == 0) return ALMA_OK;
    mala_select_kernel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(b->natoms, t->nrb, b->nsys, b->atom_off,
                                                                          t->rb_off, accept, sys_mask, xyz_old,
                                                                          born_old, b->xyz, b->born, g_new, g_cur);
    ALMA_LAUNCH_CHECK("alma_mala_select");
    return ALMA_OK;
}
