// ΔE of one torsion-space proposal, evaluated by one CTA for one system.
//
// Semantics follow the reference proposal core (try_torsion,
// physics_engine.cpp:2328-2399; try_crankshaft :2407-2501; concerted
// sidechain move :2798-2878):
//   ΔE = Δ(cross-pair sum) + Δ(SASA of the whole structure)
//      + Δ(boundary dihedral records) + Δ(disulfide pairs touching a moved atom)
// where cross pairs are neighbor-list pairs whose atoms are in different
// move groups (0 = fixed), not excluded, with r² <= 12² (:2312-2323), the
// "after" sum uses the moved atoms' half-list Born radii (update_born
// :2043-2051) and the fixed atoms' unchanged radii.
//
// Work is proportional to the move, not to the structure:
//   * cross pairs come from the moved atoms' full rows only, old and new
//     geometry evaluated in the same pass (each fixed partner once, pairs
//     between two moving groups once, from the lower index);
//   * SASA is recomputed only for atoms whose half row holds an atom of a
//     different group (moved atoms, plus fixed atoms that list a moved atom)
//     — every other atom's SASA is unchanged bit for bit;
//   * dihedral records are tested for a mixed group pattern;
//   * a moved atom whose full row lies inside its side's atom range (the
//     row's index span, kept by the list build) has no partner that stays
//     behind: it skips the cross-pair and SASA-mark scans, and its new Born
//     radius (which no cross pair reads) is computed only when the move is
//     accepted — a move of half the chain scans only the rows at the cut.
// Per-atom contributions land in dE_atom[2*i] (cross) / dE_atom[2*i+1]
// (SASA) and are summed in atom order, so the result is deterministic.
#pragma once
#include <cooperative_groups.h>

#include "alma_common.cuh"

namespace alma {

namespace cg = cooperative_groups;

// The threads that evaluate one system's proposal: one CTA (CL = 1) or a
// thread-block cluster of CL CTAs on CL SMs.  Work is strided over all the
// team's threads / warps; phase barriers are CTA or cluster barriers (the
// latter order global-memory writes across the cluster's CTAs).
template <int CL>
struct Team {
    int rank;
    __device__ Team() { rank = CL > 1 ? (int)cg::this_cluster().block_rank() : 0; }
    __device__ __forceinline__ int gtid() const { return rank * (int)blockDim.x + (int)threadIdx.x; }
    __device__ __forceinline__ int gthreads() const { return CL * (int)blockDim.x; }
    __device__ __forceinline__ int gwarp() const { return rank * ((int)blockDim.x >> 5) + ((int)threadIdx.x >> 5); }
    __device__ __forceinline__ int gwarps() const { return CL * ((int)blockDim.x >> 5); }
    __device__ __forceinline__ void sync() const {
        if constexpr (CL > 1) cg::this_cluster().sync();
        else __syncthreads();
    }
};

// Team-wide sums of K doubles; every thread of every CTA gets the same
// totals.  One block reduction for all K values (warp trees, then warp 0
// over the warp totals), then the CTA partials combined in rank order
// through distributed shared memory.  smem: >= 32*K doubles; part:
// __shared__ double[K] per CTA, double-buffered by the caller (proposal
// parity) — no barrier follows the remote reads: the next write to the same
// buffer is two proposals later, behind several team barriers, and every
// caller passes a team barrier before it exits.
template <int CL, int K>
__device__ __forceinline__ void team_sum(const Team<CL> &T, double (&v)[K], double *smem, double *part) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (int)(blockDim.x >> 5);
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = warp_sum(v[k]);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < K; ++k) smem[32 * k + wid] = v[k];
    __syncthreads();
    if (wid == 0) {
        double t[K];
#pragma unroll
        for (int k = 0; k < K; ++k) t[k] = warp_sum(lane < nw ? smem[32 * k + lane] : 0.0);
        if (lane == 0)
#pragma unroll
            for (int k = 0; k < K; ++k) part[k] = t[k];
    }
    if constexpr (CL > 1) {
        T.sync();
        cg::cluster_group cl = cg::this_cluster();
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] = 0.0;
        for (int r = 0; r < CL; ++r) {
            const double *pr = cl.map_shared_rank(part, r);
#pragma unroll
            for (int k = 0; k < K; ++k) v[k] += pr[k];
        }
    } else {
        __syncthreads();
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] = part[k];
    }
}

constexpr int MOVE_THREADS = 512;

// A cross pair that passed the filters (different groups, not excluded,
// within the cutoff before or after): packed per warp so the pair
// arithmetic runs with every lane busy.
struct CrossCand {
    double r2o, r2n;
    int j, gj;
};
constexpr int CROSS_BUF = 64;  // per warp: < 32 waiting + one batch of 32
constexpr int MAX_ROT = 2;
constexpr int MAX_WPR = 4;  // segments (tasks) per moved-atom row, at most

// Global scratch for the move kernels; every array is all-zero between
// proposals (each proposal clears what it set).
struct MoveScratch {
    int8_t *group;      // [natoms] move group for the cross-pair sum (0 fixed)
    int8_t *body;       // [natoms] rigid body for the SASA reach test: equals
                        // group, except the psi side of a crankshaft (2),
                        // which turns twice and so moves against the rest of
                        // its group
    int *mark;          // [natoms] SASA recompute flags (first marker appends
                        // the atom to `affected`)
    double *xyz_new;    // [natoms*4]
    double *born_new;   // [natoms]
    double *dE_atom;    // [natoms*2] SASA of affected atoms: new term [2i],
                        // change [2i+1]
    double *hct_part;   // [natoms*MAX_WPR] per-segment hct sums of moved atoms
    double *cross_part; // [natoms*MAX_WPR] per-segment cross-pair ΔE of moved atoms
    int32_t *affected;  // [natoms] atoms whose SASA is recomputed (per-system
                        // region), appended during the marking pass
    int32_t *edge;      // [natoms] moved atoms with a neighbour outside their
                        // rigid body (per-system region), appended in P1
    unsigned long long *ctr;  // [4*nsys] cumulative work counters: pair terms,
                              // hct terms, SASA neighbour visits, moved atoms
    unsigned long long *phase;  // [4*nsys] cumulative SM cycles of rank 0 in
                                // the four phases of move_eval (+ finish)
    int *queue;               // [QUEUE_PER_SYS*nsys] per proposal parity
                              // (QUEUE_PER_PARITY ints): [0] = next P3 task,
                              // [1] = edge atoms, [2] = a trial atom is
                              // beyond half the skin, [3] = affected atoms,
                              // [4] = next P2 task (others reserved)
    int *drift;               // [2*nsys] drift flags, two proposals
};

constexpr int QUEUE_PER_PARITY = 8;
constexpr int QUEUE_PER_SYS = 2 * QUEUE_PER_PARITY;

// Next task index of a dynamically scheduled phase for the calling warp
// (lane 0 draws from the team's counter; every lane gets it).
__device__ __forceinline__ int64_t draw_task(int *counter, int lane) {
    int v = 0;
    if (lane == 0) v = atomicAdd(counter, 1);
    return __shfl_sync(0xffffffffu, v, 0);
}

// A j-side: sorted explicit atoms side_idx[eb, ee) plus the range [lo, hi).
struct SideRef {
    int64_t eb, ee;
    int32_t lo, hi;
};

__device__ __forceinline__ SideRef side_ref(const AlmaTopo &t, int k) {
    SideRef S;
    S.eb = t.side_ptr[k];
    S.ee = t.side_ptr[k + 1];
    S.lo = t.side_lo[k];
    S.hi = t.side_hi[k];
    return S;
}

__device__ __forceinline__ int64_t side_count(const SideRef &S) { return (S.ee - S.eb) + (int64_t)(S.hi - S.lo); }

__device__ __forceinline__ int side_atom(const SideRef &S, const int32_t *side_idx, int64_t k) {
    const int64_t ne = S.ee - S.eb;
    return k < ne ? side_idx[S.eb + k] : S.lo + (int)(k - ne);
}

__device__ __forceinline__ bool contains_sorted(const int32_t *a, int64_t beg, int64_t end, int v) {
    int64_t lo = beg, hi = end;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (a[mid] < v) lo = mid + 1;
        else hi = mid;
    }
    return lo < end && a[lo] == v;
}

__device__ __forceinline__ bool side_has(const SideRef &S, const int32_t *side_idx, int v) {
    return (v >= S.lo && v < S.hi) || contains_sorted(side_idx, S.eb, S.ee, v);
}

struct Rot {
    double o[3], u[3], c, s;
    SideRef side;  // rotated atoms
};

struct MoveDesc {
    int kind;            // -1 none
    int nrot;
    Rot rot[MAX_ROT];
    int nmem;            // member lists (define move groups 1..nmem)
    SideRef mem[2];
    int degenerate;      // 1: zero-length axis / empty side (no proposal)
};

// Rodrigues rotation about unit axis u anchored at o (physics_engine.cpp:1848-1862).
__device__ __forceinline__ void rodrigues(double &px, double &py, double &pz, const Rot &R) {
    const double vx = px - R.o[0], vy = py - R.o[1], vz = pz - R.o[2];
    const double dot = R.u[0] * vx + R.u[1] * vy + R.u[2] * vz;
    const double cx = R.u[1] * vz - R.u[2] * vy;
    const double cy = R.u[2] * vx - R.u[0] * vz;
    const double cz = R.u[0] * vy - R.u[1] * vx;
    const double k = 1.0 - R.c;
    px = R.o[0] + vx * R.c + cx * R.s + R.u[0] * dot * k;
    py = R.o[1] + vy * R.c + cy * R.s + R.u[1] * dot * k;
    pz = R.o[2] + vz * R.c + cz * R.s + R.u[2] * dot * k;
}

// Axis from atom ai to aj at the given positions; false when degenerate.
__device__ __forceinline__ bool make_axis(Rot &R, double4 pi, double4 pj, double delta) {
    R.o[0] = pi.x; R.o[1] = pi.y; R.o[2] = pi.z;
    double ux = pj.x - pi.x, uy = pj.y - pi.y, uz = pj.z - pi.z;
    const double l = sqrt(ux * ux + uy * uy + uz * uz);
    if (l < 1e-10) return false;
    ux /= l; uy /= l; uz /= l;
    R.u[0] = ux; R.u[1] = uy; R.u[2] = uz;
    R.c = cos(delta);
    R.s = sin(delta);
    return true;
}

// Thread 0 only: decode (kind, a, delta) of system s into a MoveDesc.
// kind 0 torsion (a = rot-bond index local to s), 1 crankshaft (crank-pair
// index), 2 concerted sidechain pair (pair index; delta[0], delta[1]).
__device__ inline void decode_move(MoveDesc &M, const AlmaTopo &t, const double *xyz, int s, int kind, int a,
                                   const double *delta) {
    M.kind = kind;
    M.nrot = 0;
    M.nmem = 0;
    M.degenerate = 1;
    if (kind == 0) {
        const int k = t.rb_off[s] + a;
        M.mem[0] = side_ref(t, k);
        M.nmem = 1;
        if (side_count(M.mem[0]) == 0) return;
        Rot &R = M.rot[0];
        if (!make_axis(R, ld_xyz(xyz, t.rb_ij[2 * k]), ld_xyz(xyz, t.rb_ij[2 * k + 1]), delta[0])) return;
        R.side = M.mem[0];
        M.nrot = 1;
        M.degenerate = 0;
    } else if (kind == 1) {
        const int cpi = t.cp_off[s] + a;
        const int kphi = t.rb_off[s] + t.cp[2 * cpi], kpsi = t.rb_off[s] + t.cp[2 * cpi + 1];
        M.mem[0] = side_ref(t, kphi);
        M.nmem = 1;
        const SideRef psi = side_ref(t, kpsi);
        if (side_count(M.mem[0]) == 0 || side_count(psi) == 0) return;
        Rot &R1 = M.rot[0];
        if (!make_axis(R1, ld_xyz(xyz, t.rb_ij[2 * kphi]), ld_xyz(xyz, t.rb_ij[2 * kphi + 1]), delta[0])) return;
        R1.side = M.mem[0];
        // psi axis from the post-phi positions of its two atoms (:2447-2452)
        const int bi = t.rb_ij[2 * kpsi], bj = t.rb_ij[2 * kpsi + 1];
        double4 pb4 = ld_xyz(xyz, bi), pj4 = ld_xyz(xyz, bj);
        if (side_has(R1.side, t.side_idx, bi)) rodrigues(pb4.x, pb4.y, pb4.z, R1);
        if (side_has(R1.side, t.side_idx, bj)) rodrigues(pj4.x, pj4.y, pj4.z, R1);
        Rot &R2 = M.rot[1];
        if (!make_axis(R2, pb4, pj4, 0.0)) return;
        R2.c = R1.c;   // cos(-d) = cos(d)
        R2.s = -R1.s;  // the reference passes (cosD, -sinD)
        R2.side = psi;
        M.nrot = 2;
        M.degenerate = 0;
    } else if (kind == 2) {
        const int pi = t.csp_off[s] + a;
        const int ka = t.rb_off[s] + t.csp[2 * pi], kb = t.rb_off[s] + t.csp[2 * pi + 1];
        M.mem[0] = side_ref(t, ka);
        M.mem[1] = side_ref(t, kb);
        M.nmem = 2;
        if (side_count(M.mem[0]) == 0 || side_count(M.mem[1]) == 0) return;
        for (int r = 0; r < 2; ++r) {
            const int k = r == 0 ? ka : kb;
            Rot &R = M.rot[r];
            if (!make_axis(R, ld_xyz(xyz, t.rb_ij[2 * k]), ld_xyz(xyz, t.rb_ij[2 * k + 1]), delta[r])) return;
            R.side = M.mem[r];
        }
        M.nrot = 2;
        M.degenerate = 0;
    }
}

template <typename R>
__device__ __forceinline__ void prm_of(const float *prm, const double *prm64, int i, R &q, R &rad, R &eps) {
    if constexpr (sizeof(R) == 4) {
        const float4 p = *reinterpret_cast<const float4 *>(prm + 4 * (size_t)i);
        q = p.x; rad = p.y; eps = p.z;
    } else {
        const double4 p = *reinterpret_cast<const double4 *>(prm64 + 4 * (size_t)i);
        q = p.x; rad = p.y; eps = p.z;
    }
}

struct MoveResult {
    double dE, dcross, dsasa, ddih, dss;
};

__device__ __forceinline__ double4 pos_new(const double *xyz, const double *xyz_new, const int8_t *group, int j) {
    return group[j] ? ld_xyz(xyz_new, j) : ld_xyz(xyz, j);
}

// The same, with the three loads issued together (one dependent L2 round
// trip instead of two; the row scans are latency bound).  xyz_new of an
// atom that does not move holds a stale value that is not used.
__device__ __forceinline__ double4 pos_new_eager(const double *xyz, const double *xyz_new, const int8_t *group,
                                                 int j) {
    const int8_t g = group[j];
    const double4 a = ld_xyz(xyz, j), n = ld_xyz(xyz_new, j);
    return g ? n : a;
}

__device__ __forceinline__ double dih_angle4(double4 A, double4 B, double4 C, double4 D) {
    const double b1x = A.x - B.x, b1y = A.y - B.y, b1z = A.z - B.z;
    const double b2x = C.x - B.x, b2y = C.y - B.y, b2z = C.z - B.z;
    const double b3x = D.x - C.x, b3y = D.y - C.y, b3z = D.z - C.z;
    const double n1x = b1y * b2z - b1z * b2y, n1y = b1z * b2x - b1x * b2z, n1z = b1x * b2y - b1y * b2x;
    const double n2x = b2y * b3z - b2z * b3y, n2y = b2z * b3x - b2x * b3z, n2z = b2x * b3y - b2y * b3x;
    const double m1x = n1y * b2z - n1z * b2y, m1y = n1z * b2x - n1x * b2z, m1z = n1x * b2y - n1y * b2x;
    return atan2(m1x * n2x + m1y * n2y + m1z * n2z, n1x * n2x + n1y * n2y + n1z * n2z);
}

struct MoveCtx {
    DevParams P;
    AlmaBatch b;
    AlmaTopo t;
    AlmaNL nl;
    MoveScratch w;
};

// True when every atom of system s is within half the skin of its position
// at the last list build (the condition under which the lists are valid and
// the short rows may stand in for the full ones).  Every thread of the CTA
// gets the result; the CTA scans the whole system, so every CTA of a team
// computes the same answer.
__device__ __forceinline__ bool system_within_skin(const MoveCtx &C, int s) {
    bool far = false;
    if (C.nl.ref_xyz) {
        const int a0 = C.b.atom_off[s], a1 = C.b.atom_off[s + 1];
        for (int i = a0 + (int)threadIdx.x; i < a1 && !far; i += (int)blockDim.x)
            far = d2_of(ld_xyz(C.b.xyz, i), ld_xyz(C.nl.ref_xyz, i)) > C.P.half_skin2;
    }
    return !__syncthreads_or(far) && C.nl.ref_xyz != nullptr;
}

// Number of member atoms and the k-th one (concatenated member lists).
__device__ __forceinline__ int64_t n_members(const MoveDesc &M) {
    int64_t n = 0;
    for (int g = 0; g < M.nmem; ++g) n += side_count(M.mem[g]);
    return n;
}

__device__ __forceinline__ int member(const MoveDesc &M, const int32_t *side_idx, int64_t k, int &g) {
    for (g = 0; g < M.nmem - 1; ++g) {
        const int64_t len = side_count(M.mem[g]);
        if (k < len) break;
        k -= len;
    }
    return side_atom(M.mem[g], side_idx, k);
}

// True when every neighbour in member m's full row lies in the atom range
// of m's own rigid body, read from the row's index span: then the row holds
// no cross pair (all partners move with m) and no pair whose distance
// changes (no SASA mark), so the cross-pair and marking scans of m add
// nothing and are skipped.  A torsion's body is its j-side range; a
// crankshaft's psi-side atoms (body 2) need their span inside both sides'
// ranges; the phi-only atoms of a crankshaft and the members of a concerted
// pair (two groups) always scan.  Atoms of a side's explicit list are not in
// its range, so a row that reaches one scans too.
// Moves of fewer members scan every row: the skip would save little and
// its edge-list reads sit on the phase's critical path.
constexpr int INNER_MIN_MEMBERS = 128;

// body < 0: not known to the caller (looked up for a crankshaft).
__device__ __forceinline__ bool inner_member(const MoveCtx &C, const MoveDesc &M, int m, int body = -1) {
    if (C.nl.full_span == nullptr || M.kind == 2 || n_members(M) < INNER_MIN_MEMBERS) return false;
    const int2 sp = *reinterpret_cast<const int2 *>(C.nl.full_span + 2 * (size_t)m);
    const SideRef &A = M.mem[0];
    if (sp.x < A.lo || sp.y >= A.hi) return false;
    if (M.kind == 0) return true;
    const SideRef &B = M.rot[1].side;
    if (sp.x < B.lo || sp.y >= B.hi) return false;
    return body < 0 ? side_has(B, C.t.side_idx, m) : body == 2;
}

// Whole-CTA evaluation of a decoded, non-degenerate proposal of system s.
// smem_d: >= 128 doubles; s_nAff: shared counter.  Leaves group/xyz_new/
// born_new set for the members (the caller commits or discards, then calls
// move_clear).
// New half-list Born radius of moved atom m from its segment sums
// (update_born, physics_engine.cpp:2043-2051), segments summed in order.
__device__ __forceinline__ double born_new_of(const MoveScratch &w, const double *prm64, int m, int wpr) {
    double sum = 0.0;
    for (int sg = 0; sg < wpr; ++sg) sum += w.hct_part[(size_t)m * MAX_WPR + sg];
    return 1.0 / fmax(1.0 / prm64[4 * (size_t)m + 1] - 0.5 * sum, 2.0);
}

// SASA change of affected atom k of system s: the ordered recurrence over
// its half row (or short half row) at the new geometry, minus the old term
// — read from b.sasa when the batch carries the current per-atom terms,
// else recomputed at the old geometry in the same pass (the two
// recurrences are independent and interleaved).  The new term goes to
// dE_atom[2i] for the commit, the change to dE_atom[2i+1].  One warp.
__device__ __forceinline__ void sasa_row(const MoveCtx &C, int s, int k, bool short_rows, double pi2, double pi4,
                                         int lane, unsigned long long &nsasa) {
    const AlmaBatch &b = C.b;
    const MoveScratch &w = C.w;
    const int a0 = b.atom_off[s];
    const int i = w.affected[a0 + k];
    const bool moved = w.group[i] != 0;
    const bool cached = b.sasa != nullptr;
    const double4 pio = ld_xyz(b.xyz, i), pin = moved ? ld_xyz(w.xyz_new, i) : pio;
    const double rsi = b.prm64[4 * (size_t)i + 1] + C.P.probe_r;
    const double cs = pi2 * rsi * rsi;
    double sao = pi4 * rsi * rsi, san = sao;
    const uint32_t *rc = short_rows ? C.nl.shalf_cols : C.nl.half_cols;
    const int64_t beg = short_rows ? C.nl.shalf_ptr[i] : C.nl.half_ptr[i];
    const int64_t end = beg + (short_rows ? C.nl.shalf_len[i] : C.nl.half_len[i]);
    uint32_t nxt = beg + lane < end ? rc[beg + lane] : 0u;
    for (int64_t e0 = beg; e0 < end; e0 += 32) {
        const int64_t e = e0 + lane;
        double co = 0.0, cn = 0.0;
        bool ho = false, hn = false;
        if (e < end) {
            const int j = (int)(nxt & ALMA_IDX_MASK);
            if (e + 32 < end) nxt = rc[e + 32];  // next entry in flight
            const double rsj = b.prm64[4 * (size_t)j + 1] + C.P.probe_r;
            const double dc = rsi + rsj;
            const double4 pjn = pos_new_eager(b.xyz, w.xyz_new, w.group, j);
            const double4 pjo = ld_xyz(b.xyz, j);
            if (!cached) {
                const double ro = sqrt(d2_of(pio, pjo));
                if (ro < dc) { ho = true; co = cs * ((dc - ro) / (2.0 * rsi)); }
            }
            const double rn = sqrt(d2_of(pin, pjn));
            if (rn < dc) { hn = true; cn = cs * ((dc - rn) / (2.0 * rsi)); }
        }
        const unsigned mo = __ballot_sync(0xffffffffu, ho), mn = __ballot_sync(0xffffffffu, hn);
        if (cached)  // independent recurrences, in row order (interleaved when both run)
            san = sasa_chunk(san, mn, cn, lane);
        else
            sasa_chunk2(sao, mo, co, san, mn, cn, lane);
    }
    if (lane == 0) {
        const double tn = C.P.gamma_sa * fmax(0.0, san);
        const double to = cached ? b.sasa[i] : C.P.gamma_sa * fmax(0.0, sao);
        w.dE_atom[2 * (size_t)i] = tn;
        w.dE_atom[2 * (size_t)i + 1] = tn - to;
    }
    nsasa += (cached ? 1ull : 2ull) * (unsigned long long)(end - beg);
}

// Whole-team evaluation of a decoded, non-degenerate proposal of system s.
// parity alternates between consecutive proposals (double-buffered queue
// counters, CTA partials and drift flag).  Leaves group/body/xyz_new/
// born_new set for the members; move_finish commits or discards.
//
// Members are strided over the team's threads (P1, P4); row tasks (P2, P3)
// are drawn from per-team counters.  Team barriers: (1) after the moved
// coordinates and the edge list, (2) after the edge members' Born radii and
// the SASA marks (the marking pass also builds the affected-atom list),
// (3) after the cross-pair and SASA slots, (4) the CTA-partials exchange of
// team_sum.
//
// rows_ok: every committed atom of system s is within half the skin of its
// position at the last list build.  Then, when every trial position is too,
// the SASA reach tests walk the short rows (the pairs within SASA reach plus
// the skin at build time, in row order): no pair outside them can come
// within reach, and the SASA recurrence only consumes pairs within reach, so
// the result is the same bit for bit.
template <typename R, int CL>
__device__ MoveResult move_eval(const MoveCtx &C, const MoveDesc &M, int s, double *smem_d, double *part,
                                CrossCand *cq, int parity, bool rows_ok, const Team<CL> &T) {
    const AlmaBatch &b = C.b;
    const AlmaTopo &t = C.t;
    const MoveScratch &w = C.w;
    const int tid = T.gtid(), nthr = T.gthreads();
    const int lane = threadIdx.x & 31;
    const int a0 = b.atom_off[s], a1 = b.atom_off[s + 1];
    const int64_t nm = n_members(M);
    int *q = w.queue + QUEUE_PER_SYS * s + QUEUE_PER_PARITY * parity;  // this proposal's queue counters
    const bool timer = tid == 0;
    long long t0 = timer ? clock64() : 0;
    rows_ok = rows_ok && C.nl.sfull_cols != nullptr && C.nl.ref_xyz != nullptr;

    // P1: move groups, rigid bodies and the proposed coordinates — every
    // rotation applied in order (the crankshaft's second rotation turns its
    // psi side again, taking the axis from the post-phi positions).
    // Members whose rows reach outside their body go to the edge list (one
    // atomic per warp); only these scan rows for cross pairs and SASA marks.
    for (int64_t k0 = tid - lane; k0 < nm; k0 += nthr) {
        const int64_t k = k0 + lane;
        bool edge = false;
        int m = 0;
        if (k < nm) {
            int g;
            m = member(M, t.side_idx, k, g);
            double4 p = ld_xyz(b.xyz, m);
            int body = g + 1;
            if (M.kind == 2) {
                rodrigues(p.x, p.y, p.z, M.rot[g]);
            } else {
                rodrigues(p.x, p.y, p.z, M.rot[0]);
                if (M.kind == 1 && side_has(M.rot[1].side, t.side_idx, m)) {
                    rodrigues(p.x, p.y, p.z, M.rot[1]);
                    body = 2;
                }
            }
            w.group[m] = (int8_t)(g + 1);
            w.body[m] = (int8_t)body;
            *reinterpret_cast<double4 *>(w.xyz_new + 4 * (size_t)m) = p;
            if (rows_ok && d2_of(p, ld_xyz(C.nl.ref_xyz, m)) > C.P.half_skin2) q[2] = 1;
            edge = !inner_member(C, M, m, body);
        }
        const unsigned em = __ballot_sync(0xffffffffu, edge);
        if (em) {
            int base = 0;
            if (lane == 0) base = atomicAdd(&q[1], __popc(em));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (edge) w.edge[a0 + base + __popc(em & ((1u << lane) - 1u))] = m;
        }
    }
    T.sync();
    const int64_t ne = q[1];
    const bool by_edge = ne < nm;  // else every member scans: take them in member order
    const bool short_rows = rows_ok && q[2] == 0;
    if (timer) {
        const long long t1 = clock64();
        atomicAdd(&w.phase[4 * s + 0], (unsigned long long)(t1 - t0));
        t0 = t1;
    }
    // The other parity's counters and drift flag belong to the previous
    // proposal, whose last readers finished before the barrier above: clear
    // them for the next proposal.
    if (tid == 0) {
        int *qn = w.queue + QUEUE_PER_SYS * s + QUEUE_PER_PARITY * (parity ^ 1);
        for (int k = 0; k < QUEUE_PER_PARITY; ++k) qn[k] = 0;
        w.drift[2 * s + (parity ^ 1)] = 0;
    }

    // P2: half-list Born radii of the edge members at the new geometry
    // (update_born semantics) and SASA marks.  SASA reach: atoms i < j interact when j is
    // in i's half row and r < R*_i + R*_j + 2 probe; a pair whose distance
    // changes (rigid bodies differ) and is within reach before or after the
    // move changes the SASA of its lower atom only: mark that atom.
    // Two task sets — Born segments of the edge rows, then mark segments —
    // drawn by the team's warps from a shared counter as each finishes a
    // task (the row lengths vary, so a fixed striding leaves warps idle while
    // others work through long rows); rows are cut into up to MAX_WPR
    // segments so that there are about two tasks per warp.
    // Only edge members take part in cross pairs, so only their new radii
    // enter ΔE; the other members' radii are computed by the commit.
    const int nw = T.gwarps();
    int wph = 1;
    while (wph < MAX_WPR && 2 * ne * wph < 2 * (int64_t)nw) wph *= 2;
    const int64_t nhct = ne * wph;
    int nx = 0;
    for (int64_t it = draw_task(q + 4, lane); it < 2 * nhct; it = __shfl_sync(0xffffffffu, nx, 0)) {
        if (lane == 0) nx = atomicAdd(q + 4, 1);  // the next draw, in flight during this task
        const bool marking = it >= nhct;
        const int64_t i2 = marking ? it - nhct : it;
        const int64_t k = i2 / wph;
        const int seg = (int)(i2 % wph);
        int g;
        const int m = by_edge ? w.edge[a0 + k] : member(M, t.side_idx, k, g);
        const double4 pm = ld_xyz(w.xyz_new, m);
        if (!marking) {
        R qm, rm, em;
        prm_of<R>(b.prm, b.prm64, m, qm, rm, em);
        double sum = 0.0;
        const int64_t hb = C.nl.half_ptr[m], he = hb + C.nl.half_len[m];
        // the next entry of the row is fetched while this one is evaluated
        const int64_t stp = 32 * wph;
        int64_t e = hb + 32 * seg + lane;
        uint32_t nxt = e < he ? C.nl.half_cols[e] : 0u;
        for (; e < he; e += stp) {
            const int j = (int)(nxt & ALMA_IDX_MASK);
            if (e + stp < he) nxt = C.nl.half_cols[e + stp];
            R qj, rj, ej;
            prm_of<R>(b.prm, b.prm64, j, qj, rj, ej);
            const double r2d = d2_of(pm, pos_new_eager(b.xyz, w.xyz_new, w.group, j));
            const R r2 = (R)r2d;
            sum += (double)hct_term<R>(f_sqrt(r2), r2, rm, rj);
        }
        sum = warp_sum(sum);
        if (lane == 0) {
            w.hct_part[(size_t)m * MAX_WPR + seg] = sum;
            if (seg == 0) atomicAdd(&w.ctr[4 * s + 1], (unsigned long long)C.nl.half_len[m]);
        }
        continue;
        }
        const double4 pmo = ld_xyz(b.xyz, m);
        const double rsm = b.prm64[4 * (size_t)m + 1] + C.P.probe_r;
        const int bm = w.body[m];
        const uint32_t *rc = short_rows ? C.nl.sfull_cols : C.nl.full_cols;
        const int64_t fb = short_rows ? C.nl.sfull_ptr[m] : C.nl.full_ptr[m];
        const int64_t fe = fb + (short_rows ? C.nl.sfull_len[m] : C.nl.full_len[m]);
        const int64_t stp = 32 * wph;
        int64_t e = fb + 32 * seg + lane;
        uint32_t nxt = e < fe ? rc[e] : 0u;
        for (; e < fe; e += stp) {
            const int j = (int)(nxt & ALMA_IDX_MASK);
            if (e + stp < fe) nxt = rc[e + stp];
            // every load of the entry at once; most partners share m's body
            const int bj = w.body[j];
            const int8_t gj = w.group[j];
            const double rj = b.prm64[4 * (size_t)j + 1];
            const double4 pjo = ld_xyz(b.xyz, j), pjx = ld_xyz(w.xyz_new, j);
            if (bj == bm) continue;
            const double dc = rsm + rj + C.P.probe_r, dc2 = dc * dc;
            const double4 pjn = gj ? pjx : pjo;
            if (d2_of(pmo, pjo) < dc2 || d2_of(pm, pjn) < dc2) {
                const int a = j < m ? j : m;
                if (atomicExch(&w.mark[a], 1) == 0) w.affected[a0 + atomicAdd(&q[3], 1)] = a;
            }
        }
    }
    T.sync();
    if (timer) {
        const long long t1 = clock64();
        atomicAdd(&w.phase[4 * s + 1], (unsigned long long)(t1 - t0));
        t0 = t1;
    }

    // P3: cross pairs from the members' full rows (old and new geometry in
    // one pass), then SASA of the affected atoms (old and new, in row
    // order); boundary dihedrals and disulfides strided over threads.
    // One task space: cross-pair segments first (every warp gets one when
    // the rows allow), then the affected atoms' SASA, which wraps round onto
    // the warps: a short SASA row after a half row beats a full row.
    // Drawn from the team's counter like P2: the SASA rows first (each an
    // ordered recurrence, the longest tasks), then the cross-pair segments.
    const int naff = q[3];
    int wpc = 1;
    while (wpc < MAX_WPR && ne * wpc + naff < 2 * (int64_t)nw) wpc *= 2;
    const int64_t ncross = ne * wpc;
    const double pi4 = 4.0 * 3.14159265358979323846, pi2 = 2.0 * 3.14159265358979323846;
    unsigned long long nsasa = 0;
    for (int64_t it = draw_task(q + 0, lane); it < ncross + naff; it = __shfl_sync(0xffffffffu, nx, 0)) {
        if (lane == 0) nx = atomicAdd(q + 0, 1);  // the next draw, in flight during this task
        if (it < naff) {
            sasa_row(C, s, (int)it, short_rows, pi2, pi4, lane, nsasa);
            continue;
        }
        const int64_t k = (it - naff) / wpc;
        const int seg = (int)((it - naff) % wpc);
        int g;
        const int m = by_edge ? w.edge[a0 + k] : member(M, t.side_idx, k, g);
        const int gm = by_edge ? (int)w.group[m] : g + 1;
        const double4 pmo = ld_xyz(b.xyz, m), pmn = ld_xyz(w.xyz_new, m);
        R qm, rm, em;
        prm_of<R>(b.prm, b.prm64, m, qm, rm, em);
        const double bn = born_new_of(w, b.prm64, m, wph);
        if (seg == 0 && lane == 0) w.born_new[m] = bn;
        const R amo = (R)b.born[m], amn = (R)bn;
        const double rm64 = b.prm64[4 * (size_t)m + 1], em64 = b.prm64[4 * (size_t)m + 2];
        double acc = 0.0;
        int npair = 0;
        const int64_t fb = C.nl.full_ptr[m], fe = fb + C.nl.full_len[m];
        // Pass 1 walks the row with loads and distance tests only and packs
        // the pairs within the cutoff into the warp's buffer (about one entry
        // in eight); the pair arithmetic then runs on full batches of 32.
        CrossCand *buf = cq + (threadIdx.x >> 5) * CROSS_BUF;
        auto evaluate = [&](int cnt) {
            if (lane >= cnt) return;
            const CrossCand c = buf[lane];
            const int j = c.j, gj = c.gj;
            const double r2o = c.r2o, r2n = c.r2n;
            const bool ino = r2o <= C.P.pair_cut2, inn = r2n <= C.P.pair_cut2;
            npair += (int)ino + (int)inn;
            R qj, rj, ej;
            prm_of<R>(b.prm, b.prm64, j, qj, rj, ej);
            const R qp = qm * qj, sig = rm + rj, ep = em * ej;
            const R ajo = (R)b.born[j];
            const R ajn = gj ? (R)born_new_of(w, b.prm64, j, wph) : ajo;
            // FP64 sigma/epsilon only for contacts inside sigma (steep LJ)
            double sig64 = (double)sig, eps64 = (double)ep;
            if (fmin(ino ? r2o : r2n, inn ? r2n : r2o) < 1.0001 * sig64 * sig64) {
                const double4 pj64 = *reinterpret_cast<const double4 *>(b.prm64 + 4 * (size_t)j);
                sig64 = rm64 + pj64.y;
                eps64 = em64 * pj64.z;
            }
            if (ino && inn) {
                acc += pair_delta<R>(C.P, r2o, r2n, qp, sig, ep, amo * ajo, amn * ajn, sig64, eps64);
            } else if (ino) {
                acc -= (double)pair_energy<R>(C.P, r2o, qp, sig, ep, amo, ajo, sig64, eps64);
            } else {
                acc += (double)pair_energy<R>(C.P, r2n, qp, sig, ep, amn, ajn, sig64, eps64);
            }
        };
        const unsigned below = (1u << lane) - 1u;
        int nq = 0;
        const int64_t stp = 32 * wpc;
        uint32_t nxt = fb + 32 * seg + lane < fe ? C.nl.full_cols[fb + 32 * seg + lane] : 0u;
        for (int64_t e0 = fb + 32 * seg; e0 < fe; e0 += stp) {
            const int64_t e = e0 + lane;
            bool pass = false;
            CrossCand c;
            if (e < fe) {
                const uint32_t ent = nxt;
                if (e + stp < fe) nxt = C.nl.full_cols[e + stp];  // next entry in flight
                if (!(ent & ALMA_EXCL_BIT)) {
                    c.j = (int)(ent & ALMA_IDX_MASK);
                    c.gj = w.group[c.j];
                    const double4 pjo = ld_xyz(b.xyz, c.j);  // with the group load
                    if (!(c.gj == gm || (c.gj != 0 && c.j < m))) {
                        const double4 pjn = c.gj ? ld_xyz(w.xyz_new, c.j) : pjo;
                        c.r2o = d2_of(pmo, pjo);
                        c.r2n = d2_of(pmn, pjn);
                        pass = c.r2o <= C.P.pair_cut2 || c.r2n <= C.P.pair_cut2;
                    }
                }
            }
            const unsigned msk = __ballot_sync(0xffffffffu, pass);
            if (pass) buf[nq + __popc(msk & below)] = c;
            nq += __popc(msk);
            __syncwarp();
            if (nq >= 32) {
                evaluate(32);
                __syncwarp();
                if (lane < nq - 32) buf[lane] = buf[32 + lane];
                nq -= 32;
                __syncwarp();
            }
        }
        if (nq > 0) evaluate(nq);
        __syncwarp();  // the buffer is free for this warp's next task
        acc = warp_sum(acc);
        npair = __reduce_add_sync(0xffffffffu, npair);
        if (lane == 0) {
            w.cross_part[(size_t)m * MAX_WPR + seg] = acc;
            atomicAdd(&w.ctr[4 * s + 0], (unsigned long long)npair);
        }
    }
    if (lane == 0 && nsasa) atomicAdd(&w.ctr[4 * s + 2], nsasa);
    double ddih = 0.0, dss = 0.0;
    for (int r = t.dih_off[s] + tid; r < t.dih_off[s + 1]; r += nthr) {
        const int4 qd = *reinterpret_cast<const int4 *>(t.dih_abcd + 4 * (size_t)r);
        const int sa = w.group[qd.x] != 0, sb = w.group[qd.y] != 0, sc = w.group[qd.z] != 0, sd = w.group[qd.w] != 0;
        if (!(sa || sb || sc || sd) || (sa && sb && sc && sd)) continue;
        const double po = dih_angle4(ld_xyz(b.xyz, qd.x), ld_xyz(b.xyz, qd.y), ld_xyz(b.xyz, qd.z), ld_xyz(b.xyz, qd.w));
        const double pn = dih_angle4(pos_new(b.xyz, w.xyz_new, w.group, qd.x), pos_new(b.xyz, w.xyz_new, w.group, qd.y),
                                     pos_new(b.xyz, w.xyz_new, w.group, qd.z), pos_new(b.xyz, w.xyz_new, w.group, qd.w));
        double eo = 0.0, en = 0.0;
        for (int k = t.term_off[r]; k < t.term_off[r + 1]; ++k) {
            const double n = (double)t.term_n[k];
            eo += t.term_v2[k] * (1.0 + cos(n * po - t.term_gamma[k]));
            en += t.term_v2[k] * (1.0 + cos(n * pn - t.term_gamma[k]));
        }
        ddih += en - eo;
    }
    for (int k = t.ss_off[s] + tid; k < t.ss_off[s + 1]; k += nthr) {
        const int i = t.ss_ij[2 * k], j = t.ss_ij[2 * k + 1];
        if (w.group[i] == 0 && w.group[j] == 0) continue;
        const double dro = sqrt(d2_of(ld_xyz(b.xyz, i), ld_xyz(b.xyz, j))) - C.P.r0_ss;
        const double drn = sqrt(d2_of(pos_new(b.xyz, w.xyz_new, w.group, i), pos_new(b.xyz, w.xyz_new, w.group, j))) - C.P.r0_ss;
        dss += C.P.k_ss * drn * drn - C.P.k_ss * dro * dro;
    }
    if (tid == 0) atomicAdd(&w.ctr[4 * s + 3], (unsigned long long)nm);
    T.sync();
    if (timer) {
        const long long t1 = clock64();
        atomicAdd(&w.phase[4 * s + 2], (unsigned long long)(t1 - t0));
        t0 = t1;
    }

    // P4: deterministic sums — per-atom slots in member / atom order (edge
    // members only: the others have no cross pair), then the CTA partials in
    // rank order.
    double c = 0.0, sa = 0.0;
    for (int64_t k = tid; k < nm; k += nthr) {
        int g;
        const int m = member(M, t.side_idx, k, g);
        if (by_edge && inner_member(C, M, m, w.body[m])) continue;
        for (int sg = 0; sg < wpc; ++sg) c += w.cross_part[(size_t)m * MAX_WPR + sg];
    }
    for (int i = a0 + tid; i < a1; i += nthr) sa += w.dE_atom[2 * (size_t)i + 1];
    double v[4] = {c, sa, ddih, dss};
    team_sum<CL, 4>(T, v, smem_d, part + 4 * parity);
    if (timer) atomicAdd(&w.phase[4 * s + 3], (unsigned long long)(clock64() - t0));
    MoveResult res;
    res.dcross = v[0];
    res.dsasa = v[1];
    res.ddih = v[2];
    res.dss = v[3];
    res.dE = res.dcross + res.dsasa + res.ddih + res.dss;
    return res;
}

// Commit (accept != 0) the members' proposal and clear all scratch; flags a
// committed atom that drifted more than half the skin from its position at
// the last list build in w.drift[2s + parity] (read after the caller's
// next team barrier).
//
// An accepted move also gives its non-edge members their half-list Born
// radii at the new geometry (update_born, physics_engine.cpp:2043-2051):
// one warp per such member, whose half row holds members only, so every
// position comes from xyz_new and nothing the commit writes is read.
template <typename R, int CL>
__device__ inline void move_finish(const MoveCtx &C, const MoveDesc &M, int s, int accept, int parity,
                                   const Team<CL> &T) {
    const MoveScratch &w = C.w;
    const int tid = T.gtid(), nthr = T.gthreads();
    const int a0 = C.b.atom_off[s];
    const int64_t nm = n_members(M);
    if (accept && C.nl.full_span != nullptr && M.kind != 2 && nm >= INNER_MIN_MEMBERS) {
        const int lane = threadIdx.x & 31, wid = T.gwarp(), nw = T.gwarps();
        unsigned long long nh = 0;
        for (int64_t k = wid; k < nm; k += nw) {
            int g;
            const int m = member(M, C.t.side_idx, k, g);
            if (!inner_member(C, M, m)) continue;
            R qm, rm, em;
            prm_of<R>(C.b.prm, C.b.prm64, m, qm, rm, em);
            const double4 pm = ld_xyz(w.xyz_new, m);
            const int64_t hb = C.nl.half_ptr[m], he = hb + C.nl.half_len[m];
            double sum = 0.0;
            for (int64_t e = hb + lane; e < he; e += 32) {
                const int j = (int)(C.nl.half_cols[e] & ALMA_IDX_MASK);
                R qj, rj, ej;
                prm_of<R>(C.b.prm, C.b.prm64, j, qj, rj, ej);
                const R r2 = (R)d2_of(pm, ld_xyz(w.xyz_new, j));
                sum += (double)hct_term<R>(f_sqrt(r2), r2, rm, rj);
            }
            sum = warp_sum(sum);
            if (lane == 0) C.b.born[m] = 1.0 / fmax(1.0 / C.b.prm64[4 * (size_t)m + 1] - 0.5 * sum, 2.0);
            nh += (unsigned long long)(he - hb);
        }
        if (lane == 0 && nh) atomicAdd(&w.ctr[4 * s + 1], nh);
    }
    int drift = 0;
    for (int64_t k = tid; k < nm; k += nthr) {
        int g;
        const int m = member(M, C.t.side_idx, k, g);
        if (accept) {
            const double4 p = ld_xyz(w.xyz_new, m);
            *reinterpret_cast<double4 *>(C.b.xyz + 4 * (size_t)m) = p;
            if (!inner_member(C, M, m, w.body[m])) C.b.born[m] = w.born_new[m];
            if (C.nl.ref_xyz && d2_of(p, ld_xyz(C.nl.ref_xyz, m)) > C.P.half_skin2) drift = 1;
        }
        w.group[m] = 0;
        w.body[m] = 0;
    }
    const int naff = w.queue[QUEUE_PER_SYS * s + QUEUE_PER_PARITY * parity + 3];
    for (int k = tid; k < naff; k += nthr) {
        const int i = w.affected[a0 + k];
        if (accept && C.b.sasa) C.b.sasa[i] = w.dE_atom[2 * (size_t)i];  // the committed atoms' SASA terms
        w.mark[i] = 0;
        w.dE_atom[2 * (size_t)i] = 0.0;
        w.dE_atom[2 * (size_t)i + 1] = 0.0;
    }
    if (__any_sync(0xffffffffu, drift) && (threadIdx.x & 31) == 0) atomicOr(&w.drift[2 * s + parity], 1);
}

}  // namespace alma
