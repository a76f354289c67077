// Device Monte Carlo: one CTA per system runs proposals back to back.
//
// Per proposal (the generate_ensemble / run_landscape_* step,
// physics_engine.cpp:2504-2528, :2880-2921):
//   draw   Philox4x32-10 keyed by (seed, system), counter = step: move type,
//          move index, angle(s), Metropolis uniform — reproducible from the
//          seed (the reference's mt19937 seeded from random_device is not);
//   move   policy 0 = generate_ensemble: crankshaft with p 0.25 when pairs
//          exist, else torsion; policy 1 = landscape: concerted sidechain
//          pair with p 0.15, else crankshaft with p 0.25, else torsion;
//          policy 2 = torsion only.  Torsion step = cur_max (backbone) or
//          sidechain_mult * cur_max, times the lever scale
//          (:2340-2346); crankshaft step cur_max (:2441); concerted steps
//          2.5 cur_max * scale (:2818-2821); fixed_delta > 0 replaces all
//          of that by U(-fixed_delta, fixed_delta);
//   ΔE     move_eval (move.cuh);
//   test   accept when dE < 0 or u < exp(-dE / T), FP64 (:2387);
//   commit moved coordinates + half-list Born radii, else discard;
//   tune   every tune_freq proposals that moved: rate > target_hi ->
//          cur_max *= scale_up (<= angle_max); rate < target_lo -> *=
//          scale_down (>= angle_min) (:2515-2526);
//   drift  an accepted move that takes any moved atom more than the half
//          skin from its position at the last list build flags the system
//          for a rebuild (NeighborList::needs_rebuild, :345-351); the CTA
//          stops at the start of its next step, the host rebuilds the
//          list, the Born radii and the energy for flagged systems only
//          (alma_mc_after_rebuild) and relaunches.  A launch that finds
//          any atom of a system already beyond the half skin (coordinates
//          changed since the list was built) flags it before its first
//          proposal, as the reference's check at the top of every step
//          would.
#include "alma_block_scan.cuh"
#include "energy_core.cuh"
#include "move.cuh"
#include "nl_core.cuh"

namespace alma {

// Device workspace of the in-kernel rebuild (per system: a cell region of
// REB_CELLS_PER_ATOM cells per atom + REB_CELLS_PAD; per atom: cell, slot,
// four row counts, two energy slots).  A chain whose grid is sparser
// (an extended chain in a large box: the per-cell passes of one team would
// cost more than the whole-GPU host build) stops for the host rebuild.
constexpr int REB_CELLS_PER_ATOM = 2;
constexpr int REB_CELLS_PAD = 256;

struct RebuildWS {
    int32_t *ccount;     // [cells] counts, then fill counters
    int64_t *cstart;     // [cells] absolute starts in cell_atoms
    int32_t *cell_of;    // [natoms]
    int32_t *cell_atoms; // [natoms]
    int32_t *cnt;        // [4*natoms] row counts (kind-major); kind 0 doubles as sort scratch
    double *atom_e;      // [2*natoms]
    int32_t *flag;       // [nsys] rows fit their regions
};

struct MCConfigDev {
    uint64_t seed;
    int policy, tune_freq;
    double target_lo, target_hi, scale_up, scale_down, angle_max, angle_min;
    double sidechain_mult, crank_prob, concerted_prob, fixed_delta;
    const int32_t *moveset_off, *moveset;
    const int32_t *sys_order;  // CTA (team) -> system, or nullptr: identity
    RebuildWS rw;         // rw.ccount == nullptr: no in-kernel rebuild
    double reach_pad;     // short-row reach padding of the list build
};

__device__ __forceinline__ int pick(double u, int n) {
    int k = (int)(u * (double)n);
    return k < n ? k : n - 1;
}

// One proposal of system s at RNG counter `step` (thread 0): the Philox
// draws u[0..5], the move (kind, index, angles) under the policy and the
// chain's cur_max, decoded into M.  Returns 1 when the proposal moves atoms
// (0: no move in the set, or a degenerate move — only the step counts).
__device__ int draw_proposal(const MoveCtx &C, const MCConfigDev &cfg, const AlmaChainState &S, int s, uint64_t step,
                             int nrb, int ncp, int ncsp, int nset, MoveDesc &M, double *u) {
    const uint64_t st = step;
    const uint32_t k0 = (uint32_t)cfg.seed ^ (0x9E3779B9u * (uint32_t)(s + 1)), k1 = (uint32_t)(cfg.seed >> 32);
    const Philox4 r0 = philox4x32_10((uint32_t)st, (uint32_t)(st >> 32), (uint32_t)s, 0u, k0, k1);
    const Philox4 r1 = philox4x32_10((uint32_t)st, (uint32_t)(st >> 32), (uint32_t)s, 1u, k0, k1);
    const Philox4 r2 = philox4x32_10((uint32_t)st, (uint32_t)(st >> 32), (uint32_t)s, 2u, k0, k1);
    u[0] = u01_from(r0.v[0], r0.v[1]);
    u[1] = u01_from(r0.v[2], r0.v[3]);
    u[2] = u01_from(r1.v[0], r1.v[1]);
    u[3] = u01_from(r1.v[2], r1.v[3]);
    u[4] = u01_from(r2.v[0], r2.v[1]);
    u[5] = u01_from(r2.v[2], r2.v[3]);
    int kind = 0, idx = 0;
    double delta[2] = {0.0, 0.0};
    bool conc = false, crank = false;
    if (cfg.policy == 1) {
        conc = ncsp > 0 && u[0] < cfg.concerted_prob;
        crank = !conc && ncp > 0 && u[4] < cfg.crank_prob;
    } else if (cfg.policy == 0) {
        crank = ncp > 0 && u[0] < cfg.crank_prob;
    }
    if (conc) {
        kind = 2;
        idx = pick(u[1], ncsp);
        const int pi = C.t.csp_off[s] + idx;
        const double sa = C.t.rb_scale[C.t.rb_off[s] + C.t.csp[2 * pi]];
        const double sb = C.t.rb_scale[C.t.rb_off[s] + C.t.csp[2 * pi + 1]];
        const double da = S.cur_max * cfg.sidechain_mult * sa, db = S.cur_max * cfg.sidechain_mult * sb;
        delta[0] = -da + 2.0 * da * u[2];
        delta[1] = -db + 2.0 * db * u[5];
    } else if (crank) {
        kind = 1;
        idx = pick(u[1], ncp);
        delta[0] = -S.cur_max + 2.0 * S.cur_max * u[2];
    } else if (nset > 0) {
        kind = 0;
        const int q = pick(u[1], nset);
        idx = cfg.moveset_off ? cfg.moveset[cfg.moveset_off[s] + q] : q;
        const int k = C.t.rb_off[s] + idx;
        const int bk = C.t.rb_kind[k];
        double base = (bk == 0 || bk == 1) ? S.cur_max : S.cur_max * cfg.sidechain_mult;
        base *= C.t.rb_scale[k];
        delta[0] = -base + 2.0 * base * u[2];
    } else {
        kind = -1;
    }
    if (cfg.fixed_delta > 0.0) {
        delta[0] = cfg.fixed_delta * (2.0 * u[2] - 1.0);
        delta[1] = cfg.fixed_delta * (2.0 * u[5] - 1.0);
    }
    if (kind >= 0) decode_move(M, C.t, C.b.xyz, s, kind, idx, delta);
    else M.degenerate = 1;
    return !M.degenerate;
}

// Team-wide min (lo) and max (hi) of three coordinates.  rsm: >= 192
// doubles of shared memory; rpart: __shared__ double[6] per CTA.
template <int CL>
__device__ void team_minmax3(const Team<CL> &T, double (&lo)[3], double (&hi)[3], double *rsm, double *rpart) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (int)(blockDim.x >> 5);
    for (int d = 0; d < 3; ++d) {
        double a = lo[d], b = hi[d];
        for (int o = 16; o > 0; o >>= 1) {
            a = fmin(a, __shfl_xor_sync(0xffffffffu, a, o));
            b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
        }
        if (lane == 0) {
            rsm[32 * d + wid] = a;
            rsm[32 * (3 + d) + wid] = b;
        }
    }
    __syncthreads();
    if (wid == 0) {
        for (int d = 0; d < 3; ++d) {
            double a = lane < nw ? rsm[32 * d + lane] : 1e300, b = lane < nw ? rsm[32 * (3 + d) + lane] : -1e300;
            for (int o = 16; o > 0; o >>= 1) {
                a = fmin(a, __shfl_xor_sync(0xffffffffu, a, o));
                b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
            }
            if (lane == 0) {
                rpart[d] = a;
                rpart[3 + d] = b;
            }
        }
    }
    if constexpr (CL > 1) {
        T.sync();
        cg::cluster_group cl = cg::this_cluster();
        for (int d = 0; d < 3; ++d) {
            lo[d] = 1e300;
            hi[d] = -1e300;
        }
        for (int r = 0; r < CL; ++r) {
            const double *pr = cl.map_shared_rank(rpart, r);
            for (int d = 0; d < 3; ++d) {
                lo[d] = fmin(lo[d], pr[d]);
                hi[d] = fmax(hi[d], pr[3 + d]);
            }
        }
        T.sync();  // rpart is read before anyone writes it again
    } else {
        __syncthreads();
        for (int d = 0; d < 3; ++d) {
            lo[d] = rpart[d];
            hi[d] = rpart[3 + d];
        }
        __syncthreads();
    }
}

// Neighbor list, Born radii and energy of system s rebuilt by its own team
// inside the persistent kernel (the host path: alma_nl_build + alma_born_radii
// + alma_energy for the system).  The same per-atom row, Born and pair/SASA
// code as those entry points, so the rows come out identical, order
// included.  Returns false, leaving the list untouched where it matters,
// when the cell grid or the rows do not fit: the chain then stops for a
// host rebuild, which grows the regions.  E: the fresh total energy.
template <typename R, int CL>
__device__ bool team_rebuild(const MoveCtx &C, const MCConfigDev &cfg, int s, const Team<CL> &T, double *sm,
                             double *rsm, double *rpart, int64_t *ssm, double &E) {
    const RebuildWS &ws = cfg.rw;
    const AlmaBatch &b = C.b;
    const AlmaNL &nl = C.nl;
    const int a0 = b.atom_off[s], a1 = b.atom_off[s + 1], n = a1 - a0;
    const int tid = T.gtid(), nthr = T.gthreads(), wid = T.gwarp(), nw = T.gwarps(), lane = threadIdx.x & 31;
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int i = a0 + tid; i < a1; i += nthr) {
        const double4 p = ld_xyz(b.xyz, i);
        lo[0] = fmin(lo[0], p.x); hi[0] = fmax(hi[0], p.x);
        lo[1] = fmin(lo[1], p.y); hi[1] = fmax(hi[1], p.y);
        lo[2] = fmin(lo[2], p.z); hi[2] = fmax(hi[2], p.z);
    }
    team_minmax3<CL>(T, lo, hi, rsm, rpart);
    SysGrid g = grid_from_box(lo, hi, C.P.nl_rcut2, n);
    if (g.ncell > (int64_t)REB_CELLS_PER_ATOM * n + REB_CELLS_PAD) return false;  // same answer in every thread
    g.cell_off = (int64_t)REB_CELLS_PER_ATOM * a0 + (int64_t)(REB_CELLS_PAD + 1) * s;
    int32_t *cnt_c = ws.ccount + g.cell_off;
    int64_t *start = ws.cstart + g.cell_off;
    const int NA = b.natoms;
    for (int64_t c = tid; c < g.ncell; c += nthr) cnt_c[c] = 0;
    T.sync();
    for (int i = a0 + tid; i < a1; i += nthr) {
        const int c = cell_of_point(g, ld_xyz(b.xyz, i));
        ws.cell_of[i] = c;
        atomicAdd(&cnt_c[c], 1);
    }
    T.sync();
    if (T.rank == 0) {  // cell starts; the counts become fill counters
        int64_t carry = a0;
        for (int64_t b0 = 0; b0 < g.ncell; b0 += blockDim.x) {
            const int64_t c = b0 + threadIdx.x;
            const int64_t v = c < g.ncell ? cnt_c[c] : 0;
            int64_t ex;
            const int64_t tot = block_exclusive_scan(v, ex, ssm);
            if (c < g.ncell) {
                start[c] = carry + ex;
                cnt_c[c] = 0;
            }
            carry += tot;
        }
        if (threadIdx.x == 0) start[g.ncell] = carry;
    }
    T.sync();
    for (int i = a0 + tid; i < a1; i += nthr) {
        const int c = ws.cell_of[i];
        ws.cell_atoms[start[c] + atomicAdd(&cnt_c[c], 1)] = i;
    }
    T.sync();
    // ascending atoms in every cell: cells holding two or more atoms are
    // listed (at most n/2 of them), then rank-sorted one warp per cell
    int32_t *tmp = ws.cnt;                      // kind-0 counts: free until the count pass
    int32_t *multi = ws.cnt + (size_t)NA + a0;  // kind-1 counts: the list of cells to sort
    int *nmulti = reinterpret_cast<int *>(ws.flag + s);
    if (tid == 0) *nmulti = 0;
    T.sync();
    for (int64_t c = tid; c < g.ncell; c += nthr)
        if (start[c + 1] - start[c] > 1) multi[atomicAdd(nmulti, 1)] = (int32_t)c;
    T.sync();
    const int nm = __ldcg(nmulti);
    for (int q = wid; q < nm; q += nw) {
        const int64_t c = multi[q];
        const int64_t b0 = start[c];
        const int m = (int)(start[c + 1] - b0);
        for (int k = lane; k < m; k += 32) {
            const int v = ws.cell_atoms[b0 + k];
            int rank = 0;
            for (int q2 = 0; q2 < m; ++q2) rank += ws.cell_atoms[b0 + q2] < v;
            tmp[b0 + rank] = v;
        }
        __syncwarp();
        for (int k = lane; k < m; k += 32) ws.cell_atoms[b0 + k] = tmp[b0 + k];
        __syncwarp();
    }
    T.sync();
    const double rcut2 = C.P.nl_rcut2;
    const int64_t *ep = C.t.excl_ptr;
    const int32_t *ec = C.t.excl_cols;
    for (int i = a0 + wid; i < a1; i += nw) {
        int nf, nh, nsf, nsh;
        nl_row_atom<0>(i, lane, g, b.xyz, rcut2, ws.cell_of, ws.cstart, ws.cell_atoms, b.prm64, cfg.reach_pad, ep, ec,
                       C.t.excl_win, nl, nf, nh, nsf, nsh);
        if (lane == 0) {
            ws.cnt[i] = nf;
            ws.cnt[(size_t)NA + i] = nh;
            ws.cnt[2 * (size_t)NA + i] = nsf;
            ws.cnt[3 * (size_t)NA + i] = nsh;
        }
    }
    T.sync();
    if (T.rank == 0) {  // row pointers inside the system's regions
        const int nkind = nl.sfull_cols ? 4 : 2;
        int fits = 1;
        for (int kind = 0; kind < nkind; ++kind) {
            const int32_t *cnt = ws.cnt + (size_t)kind * NA;
            int64_t *ptr = kind == 0 ? nl.full_ptr : kind == 1 ? nl.half_ptr : kind == 2 ? nl.sfull_ptr : nl.shalf_ptr;
            int32_t *len = kind == 0 ? nl.full_len : kind == 1 ? nl.half_len : kind == 2 ? nl.sfull_len : nl.shalf_len;
            const int64_t *basev = kind == 0 ? nl.full_base : kind == 1 ? nl.half_base : kind == 2 ? nl.sfull_base
                                                                                                    : nl.shalf_base;
            const int64_t base = basev[s], cap = basev[s + 1] - base;
            int64_t carry = 0;
            for (int i0 = a0; i0 < a1; i0 += blockDim.x) {
                const int i = i0 + threadIdx.x;
                const int64_t v = i < a1 ? cnt[i] : 0;
                int64_t ex;
                const int64_t tot = block_exclusive_scan(v, ex, ssm);
                if (i < a1) {
                    ptr[i] = base + carry + ex;
                    len[i] = (int32_t)v;
                }
                carry += tot;
            }
            if (threadIdx.x == 0) nl.need[4 * s + kind] = carry;
            if (carry > cap) fits = 0;
        }
        if (threadIdx.x == 0) ws.flag[s] = fits;
    }
    T.sync();
    if (!__ldcg(&ws.flag[s])) return false;
    for (int i = a0 + wid; i < a1; i += nw) {
        int nf, nh, nsf, nsh;
        nl_row_atom<1>(i, lane, g, b.xyz, rcut2, ws.cell_of, ws.cstart, ws.cell_atoms, b.prm64, cfg.reach_pad, ep, ec,
                       C.t.excl_win, nl, nf, nh, nsf, nsh);
    }
    T.sync();
    for (int i = a0 + wid; i < a1; i += nw)
        born_atom<R>(i, lane, b.xyz, b.prm, b.prm64, nl.full_ptr, nl.full_len, nl.full_cols, b.born);
    T.sync();
    for (int i = a0 + wid; i < a1; i += nw)
        pair_sasa_atom<R>(C.P, i, lane, b.xyz, b.prm, b.prm64, b.born, nl.half_ptr, nl.half_len, nl.half_cols,
                          ep != nullptr, ws.atom_e, b.sasa);
    T.sync();
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    for (int i = a0 + tid; i < a1; i += nthr) {
        v[0] += ws.atom_e[2 * (size_t)i];
        v[1] += ws.atom_e[2 * (size_t)i + 1];
    }
    if (C.t.dih_off)
        for (int r = C.t.dih_off[s] + tid; r < C.t.dih_off[s + 1]; r += nthr) v[2] += dih_record_energy(b.xyz, C.t, r);
    if (C.t.ss_off)
        for (int k = C.t.ss_off[s] + tid; k < C.t.ss_off[s + 1]; k += nthr) {
            const double dr = sqrt(dist2(b.xyz, C.t.ss_ij[2 * k], C.t.ss_ij[2 * k + 1])) - C.P.r0_ss;
            v[3] += C.P.k_ss * dr * dr;
        }
    team_sum<CL, 4>(T, v, sm, rpart);
    T.sync();  // the partials are read before anyone writes them again
    const double sasa = n > 0 ? C.P.beta_sa + v[1] : 0.0;
    E = sasa + v[2] + v[3] + v[0];
    return true;
}

// One system per CTA (CL = 1) or per cluster of CL CTAs.  Every CTA of a
// cluster keeps its own copy of the chain state and makes the same draws
// and decisions (the ΔE totals are bit-identical in every CTA); rank 0
// writes the state back.
template <typename R, int NT, int CL>
__global__ void __launch_bounds__(NT, 512 / NT) mc_kernel(MoveCtx C, MCConfigDev cfg,
                                                          AlmaChainState *__restrict__ states, int64_t step_limit) {
    __shared__ MoveDesc M;
    __shared__ double sm[128];
    __shared__ double part[8];
    __shared__ CrossCand cq[(NT / 32) * CROSS_BUF];
    __shared__ AlmaChainState S;
    __shared__ double u[6];
    __shared__ int did_move, accept;
    __shared__ double rsm[192], rpart[8];
    __shared__ int64_t ssm[33];
    const Team<CL> T;
    const int s = cfg.sys_order ? cfg.sys_order[blockIdx.x / CL] : (int)(blockIdx.x / CL);
    if (threadIdx.x == 0) S = states[s];
    __syncthreads();
    bool rows_ok = system_within_skin(C, s);
    if (threadIdx.x == 0 && !rows_ok && C.nl.ref_xyz && S.step < step_limit) S.need_rebuild = 1;
    __syncthreads();
    const int nrb = C.t.rb_off[s + 1] - C.t.rb_off[s];
    const int ncp = C.t.cp_off[s + 1] - C.t.cp_off[s];
    const int ncsp = C.t.csp_off[s + 1] - C.t.csp_off[s];
    const int nset = cfg.moveset_off ? cfg.moveset_off[s + 1] - cfg.moveset_off[s] : nrb;
    while (S.step < step_limit) {
        if (S.need_rebuild) {  // drifted: rebuild this chain in place, or stop for the host
            double E = 0.0;
            if (!cfg.rw.ccount || !C.nl.ref_xyz || !team_rebuild<R, CL>(C, cfg, s, T, sm, rsm, rpart, ssm, E)) break;
            if (threadIdx.x == 0) {
                S.energy = E;
                S.n_rebuild++;
                S.need_rebuild = 0;
            }
            rows_ok = true;
            __syncthreads();
            continue;
        }
        if (threadIdx.x == 0) did_move = draw_proposal(C, cfg, S, s, (uint64_t)S.step, nrb, ncp, ncsp, nset, M, u);
        __syncthreads();
        if (!did_move) {
            if (threadIdx.x == 0) S.step++;
            __syncthreads();
            continue;
        }
        const int parity = S.parity & 1;
        const MoveResult r = move_eval<R, CL>(C, M, s, sm, part, cq, parity, rows_ok, T);
        if (threadIdx.x == 0) accept = (r.dE < 0.0) || (u[3] < exp(-r.dE / S.temperature));
        __syncthreads();
        const int acc = accept;
        move_finish<R, CL>(C, M, s, acc, parity, T);
        // commits and the drift flag visible to every CTA before the state
        // update and the next proposal's coordinate reads
        T.sync();
        const int drift = C.w.drift[2 * s + parity];
        if (threadIdx.x == 0) {
            S.parity ^= 1;
            S.n_proposed++;
            if (acc) {
                S.n_accepted++;
                S.energy += r.dE;
                if (drift) S.need_rebuild = 1;
            }
            S.acc_win += acc;
            if (cfg.tune_freq > 0 && ++S.tot_win == cfg.tune_freq) {
                const double rate = (double)S.acc_win / (double)cfg.tune_freq;
                if (rate > cfg.target_hi) S.cur_max = fmin(cfg.angle_max, S.cur_max * cfg.scale_up);
                else if (rate < cfg.target_lo) S.cur_max = fmax(cfg.angle_min, S.cur_max * cfg.scale_down);
                S.acc_win = 0;
                S.tot_win = 0;
            }
            S.step++;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0 && T.rank == 0) states[s] = S;
}

template <typename R, int NT, int CL>
static cudaError_t launch_mc(const MoveCtx &C, const MCConfigDev &d, AlmaChainState *states, int64_t step_limit,
                             int nsys, cudaStream_t st) {
    if constexpr (CL == 1) {
        mc_kernel<R, NT, 1><<<nsys, NT, 0, st>>>(C, d, states, step_limit);
        return cudaGetLastError();
    } else {
        auto kfn = mc_kernel<R, NT, CL>;
        if (CL > 8) {
            cudaError_t e = cudaFuncSetAttribute(kfn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
            if (e != cudaSuccess) return e;
        }
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)(nsys * CL), 1, 1);
        cfg.blockDim = dim3(NT, 1, 1);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = CL;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int max_clusters = 0;
        cudaError_t e = cudaOccupancyMaxActiveClusters(&max_clusters, kfn, &cfg);
        if (e != cudaSuccess) return e;
        if (max_clusters < 1) return cudaErrorInvalidConfiguration;  // cluster does not fit a GPC
        return cudaLaunchKernelEx(&cfg, kfn, C, d, states, step_limit);
    }
}

// ---- speculative rounds: K teams per system ---------------------------------
//
// A single chain fills 16 of 148 SMs, and most proposals are rejected; a
// rejected proposal leaves the state as it was.  So K teams (clusters) of a
// system evaluate the proposals of steps S.step + 0 .. S.step + K-1 at once,
// all against the committed state, each in its own scratch; the first one
// accepted is committed and the ones after it are dropped (their steps are
// drawn again in the next round).  Every proposal uses the counter-keyed
// draws of its own step, and a round never crosses a cur_max adaptation
// boundary, so the chain is exactly the sequential kernel's.
//
// Teams meet twice per round (results, then the commit) at a barrier on a
// per-system counter in global memory.  The counter is reset by the host
// before the launch; a team that waits longer than SPEC_SPIN_LIMIT polls
// (about a second) raises the abort flag and ALMA_ST_SPEC_ABORT, and every
// team leaves its loop without writing the chain state.  The host launches
// only when every cluster of the grid can be resident at once.
constexpr int SPEC_MAX_TEAMS = 8;
constexpr long long SPEC_SPIN_LIMIT = 1ll << 22;

struct SpecSlot {
    double dE;
    int32_t flags;  // 1 proposal, 2 moves atoms, 4 accepted, 8 commit drifted
    int32_t pad;
};

struct SpecRound {
    unsigned int bar;
    unsigned int abort;
    int32_t pad[2];
    SpecSlot slot[2][SPEC_MAX_TEAMS];
};

__device__ __forceinline__ MoveScratch scratch_at(const MoveScratch &w, size_t off) {
    MoveScratch t = w;
    auto sh = [off](auto *p) { return reinterpret_cast<decltype(p)>(reinterpret_cast<char *>(p) + off); };
    t.group = sh(w.group);
    t.body = sh(w.body);
    t.mark = sh(w.mark);
    t.xyz_new = sh(w.xyz_new);
    t.born_new = sh(w.born_new);
    t.dE_atom = sh(w.dE_atom);
    t.hct_part = sh(w.hct_part);
    t.cross_part = sh(w.cross_part);
    t.affected = sh(w.affected);
    t.edge = sh(w.edge);
    t.queue = sh(w.queue);
    t.drift = sh(w.drift);
    return t;  // work counters and phase timers stay shared (team 0's)
}

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int *p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Cross-team barrier of one system; returns nonzero when the round aborts.
template <int CL>
__device__ __forceinline__ int spec_barrier(const Team<CL> &T, SpecRound *Rd, unsigned int target, int *abort_sh,
                                            uint32_t *status) {
    if (T.rank == 0 && threadIdx.x == 0) {
        __threadfence();
        atomicAdd(&Rd->bar, 1u);
        int ab = 0;
        long long it = 0;
        while ((int)(ld_acquire(&Rd->bar) - target) < 0) {
            if (*(volatile unsigned int *)&Rd->abort) {
                ab = 1;
                break;
            }
            __nanosleep(64);
            if (++it > SPEC_SPIN_LIMIT) {
                atomicExch(&Rd->abort, 1u);
                set_status(status, ALMA_ST_SPEC_ABORT);
                ab = 1;
                break;
            }
        }
        *abort_sh = ab;
    }
    T.sync();
    int ab;
    if constexpr (CL > 1) ab = *cg::this_cluster().map_shared_rank(abort_sh, 0);
    else ab = *abort_sh;
    __threadfence();  // the other teams' results and commit, seen by every thread
    return ab;
}

// One CTA alone at a barrier of two: its wait runs out (the timeout path of
// spec_barrier, exercised without a second team that never arrives).
__global__ void spec_wait_selftest_kernel(SpecRound *Rd, uint32_t *status, int32_t *aborted) {
    __shared__ int abort_sh;
    const Team<1> T;
    const int ab = spec_barrier<1>(T, Rd, 2u, &abort_sh, status);
    if (threadIdx.x == 0) *aborted = ab;
}

template <typename R, int NT, int CL>
__global__ void __launch_bounds__(NT, 512 / NT)
mc_spec_kernel(MoveCtx C, MCConfigDev cfg, AlmaChainState *__restrict__ states, int64_t step_limit, int teams,
               size_t team_stride, SpecRound *__restrict__ rounds) {
    __shared__ MoveDesc M;
    __shared__ double sm[128];
    __shared__ double part[8];
    __shared__ CrossCand cq[(NT / 32) * CROSS_BUF];
    __shared__ AlmaChainState S;
    __shared__ double u[6];
    __shared__ int did_move, acc_sh, a_sh, abort_sh;
    const Team<CL> T;
    const int grp = blockIdx.x / CL;
    const int s = cfg.sys_order ? cfg.sys_order[grp / teams] : grp / teams, q = grp % teams;
    MoveCtx Cq = C;
    Cq.w = scratch_at(C.w, (size_t)q * team_stride);
    SpecRound *Rd = rounds + s;
    if (threadIdx.x == 0) {
        S = states[s];
        if (T.rank == 0) {
            for (int k = 0; k < QUEUE_PER_SYS; ++k) Cq.w.queue[QUEUE_PER_SYS * s + k] = 0;  // this team's queues, both parities
            Cq.w.drift[2 * s] = Cq.w.drift[2 * s + 1] = 0;
        }
    }
    __syncthreads();
    const bool rows_ok = system_within_skin(Cq, s);
    if (threadIdx.x == 0 && !rows_ok && C.nl.ref_xyz && S.step < step_limit) S.need_rebuild = 1;
    T.sync();
    const int nrb = C.t.rb_off[s + 1] - C.t.rb_off[s];
    const int ncp = C.t.cp_off[s + 1] - C.t.cp_off[s];
    const int ncsp = C.t.csp_off[s + 1] - C.t.csp_off[s];
    const int nset = cfg.moveset_off ? cfg.moveset_off[s + 1] - cfg.moveset_off[s] : nrb;
    int parity = 0, aborted = 0;
    unsigned int nbar = 0;
    for (int round = 0; S.step < step_limit && !S.need_rebuild; ++round) {
        // round size: within the step limit, no cur_max adaptation inside
        int64_t keff = teams;
        if (cfg.tune_freq > 0) keff = min(keff, (int64_t)(cfg.tune_freq - S.tot_win));
        keff = min(keff, step_limit - S.step);
        const int rp = round & 1;
        if (threadIdx.x == 0)
            did_move = q < keff ? draw_proposal(Cq, cfg, S, s, (uint64_t)(S.step + q), nrb, ncp, ncsp, nset, M, u) : 0;
        __syncthreads();
        double dE = 0.0;
        int acc = 0;
        if (did_move) {
            const MoveResult r = move_eval<R, CL>(Cq, M, s, sm, part, cq, parity, rows_ok, T);
            if (threadIdx.x == 0) acc_sh = (r.dE < 0.0) || (u[3] < exp(-r.dE / S.temperature));
            __syncthreads();
            acc = acc_sh;
            dE = r.dE;
        }
        if (T.rank == 0 && threadIdx.x == 0) {
            Rd->slot[rp][q].dE = dE;
            Rd->slot[rp][q].flags = (q < keff ? 1 : 0) | (did_move ? 2 : 0) | (acc ? 4 : 0);
        }
        nbar += (unsigned int)teams;
        if (spec_barrier<CL>(T, Rd, nbar, &abort_sh, C.b.status)) {
            aborted = 1;
            break;
        }
        if (threadIdx.x == 0) {
            int a = -1;
            for (int i = 0; i < keff; ++i)
                if (__ldcg(&Rd->slot[rp][i].flags) & 4) {
                    a = i;
                    break;
                }
            a_sh = a;
        }
        __syncthreads();
        const int a = a_sh;
        if (did_move) {
            move_finish<R, CL>(Cq, M, s, q == a, parity, T);
            T.sync();  // the commit and its drift flag, within the team
            if (q == a && T.rank == 0 && threadIdx.x == 0 && Cq.w.drift[2 * s + parity])
                Rd->slot[rp][q].flags |= 8;
            parity ^= 1;
        }
        nbar += (unsigned int)teams;
        if (spec_barrier<CL>(T, Rd, nbar, &abort_sh, C.b.status)) {
            aborted = 1;
            break;
        }
        if (threadIdx.x == 0) {  // the sequential kernel's bookkeeping, step by step
            const int consumed = a >= 0 ? a + 1 : (int)keff;
            for (int i = 0; i < consumed; ++i) {
                const int f = __ldcg(&Rd->slot[rp][i].flags);
                if (f & 2) {
                    const int ai = i == a;
                    S.n_proposed++;
                    if (ai) {
                        S.n_accepted++;
                        S.energy += __ldcg(&Rd->slot[rp][i].dE);
                        if (f & 8) S.need_rebuild = 1;
                    }
                    S.acc_win += ai;
                    if (cfg.tune_freq > 0 && ++S.tot_win == cfg.tune_freq) {
                        const double rate = (double)S.acc_win / (double)cfg.tune_freq;
                        if (rate > cfg.target_hi) S.cur_max = fmin(cfg.angle_max, S.cur_max * cfg.scale_up);
                        else if (rate < cfg.target_lo) S.cur_max = fmax(cfg.angle_min, S.cur_max * cfg.scale_down);
                        S.acc_win = 0;
                        S.tot_win = 0;
                    }
                }
                S.step++;
            }
        }
        __syncthreads();
    }
    // no CTA leaves while another of its cluster may still read its shared
    // memory (the abort word of the last barrier)
    T.sync();
    // team 0 writes the state; its scratch parity is the clean one for a
    // following one-team launch
    if (threadIdx.x == 0 && T.rank == 0 && q == 0 && !aborted) {
        S.parity = parity;
        states[s] = S;
    }
}

template <typename R, int NT, int CL>
static cudaError_t launch_mc_spec(const MoveCtx &C, const MCConfigDev &d, AlmaChainState *states, int64_t step_limit,
                                  int nsys, int teams, size_t team_stride, SpecRound *rounds, cudaStream_t st,
                                  bool *fits) {
    auto kfn = mc_spec_kernel<R, NT, CL>;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(nsys * teams * CL), 1, 1);
    cfg.blockDim = dim3(NT, 1, 1);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = CL;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (CL > 8) {
        cudaError_t e = cudaFuncSetAttribute(kfn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return e;
    }
    int max_clusters = 0;
    cudaError_t e = cudaOccupancyMaxActiveClusters(&max_clusters, kfn, &cfg);
    if (e != cudaSuccess) return e;
    // every team of every system must be resident at once (they wait on
    // one another); otherwise decline
    *fits = max_clusters >= nsys * teams;
    if (!*fits) return cudaSuccess;
    return cudaLaunchKernelEx(&cfg, kfn, C, d, states, step_limit, teams, team_stride, rounds);
}

// After a rebuild of the flagged systems: energy <- fresh total, flag
// cleared, rebuild counted.
__global__ void mc_after_rebuild_kernel(AlmaChainState *__restrict__ states, const double *__restrict__ terms,
                                        const uint8_t *__restrict__ mask, int nsys) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsys || (mask && !mask[s])) return;
    states[s].energy = terms[5 * (size_t)s + 4];
    if (states[s].need_rebuild) states[s].n_rebuild++;
    states[s].need_rebuild = 0;
}

}  // namespace alma

using namespace alma;

static size_t align_up256(size_t x) { return (x + 255) & ~(size_t)255; }

static size_t rebuild_bytes(int32_t natoms, int32_t nsys, RebuildWS *ws, void *base) {
    const size_t n = natoms > 0 ? (size_t)natoms : 1, S = nsys > 0 ? (size_t)nsys : 1;
    const size_t cells = (size_t)REB_CELLS_PER_ATOM * n + (size_t)(REB_CELLS_PAD + 1) * S;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        char *q = base ? (char *)base + off : nullptr;
        off += align_up256(bytes);
        return q;
    };
    RebuildWS t;
    t.ccount = (int32_t *)take(sizeof(int32_t) * cells);
    t.cstart = (int64_t *)take(sizeof(int64_t) * cells);
    t.cell_of = (int32_t *)take(sizeof(int32_t) * n);
    t.cell_atoms = (int32_t *)take(sizeof(int32_t) * n);
    t.cnt = (int32_t *)take(sizeof(int32_t) * 4 * n);
    t.atom_e = (double *)take(sizeof(double) * 2 * n);
    t.flag = (int32_t *)take(sizeof(int32_t) * S);
    if (ws) *ws = t;
    return off;
}

static RebuildWS carve_rebuild(void *base, int32_t natoms, int32_t nsys) {
    RebuildWS t = {};
    if (base) rebuild_bytes(natoms, nsys, &t, base);
    return t;
}

extern "C" size_t alma_spec_round_bytes(void) { return sizeof(SpecRound); }

extern "C" int alma_spec_wait_selftest(void *round_buf, uint32_t *status, int32_t *aborted, void *stream) {
    if (!round_buf || !status || !aborted) return alma_set_error(ALMA_EINVAL, "alma_spec_wait_selftest: null buffer");
    cudaStream_t st = (cudaStream_t)stream;
    ALMA_CUDA_TRY(cudaMemsetAsync(round_buf, 0, sizeof(SpecRound), st));
    spec_wait_selftest_kernel<<<1, 64, 0, st>>>((SpecRound *)round_buf, status, aborted);
    ALMA_LAUNCH_CHECK("alma_spec_wait_selftest");
    return ALMA_OK;
}

extern "C" size_t alma_mc_rebuild_bytes(int32_t natoms, int32_t nsys) {
    return rebuild_bytes(natoms, nsys, nullptr, nullptr);
}

int alma_check_move_args(const AlmaBatch *b, const AlmaTopo *t, const AlmaNL *nl, const AlmaParams *p,
                         void *scratch, const char *who);
MoveCtx alma_make_move_ctx(const AlmaBatch *b, const AlmaTopo *t, const AlmaNL *nl, const AlmaParams *p,
                           void *scratch);

extern "C" int alma_mc_run(const AlmaBatch *b, const AlmaTopo *t, const AlmaNL *nl, const AlmaParams *p, int prec,
                           void *scratch, const AlmaMCConfig *cfg, AlmaChainState *states, int64_t step_limit,
                           void *stream) {
    int rc = alma_check_move_args(b, t, nl, p, scratch, "alma_mc_run");
    if (rc) return rc;
    if (!cfg || !states) return alma_set_error(ALMA_EINVAL, "alma_mc_run: null config/states");
    if (cfg->policy < 0 || cfg->policy > 2) return alma_set_error(ALMA_EINVAL, "alma_mc_run: bad policy");
    // systems that get CTAs in this launch: the first nl_sys entries of sys_order
    if (cfg->launch_systems < 0 || cfg->launch_systems > b->nsys || (cfg->launch_systems > 0 && !cfg->sys_order))
        return alma_set_error(ALMA_EINVAL, "alma_mc_run: launch_systems must be 0..nsys, and > 0 needs sys_order");
    const int nl_sys = cfg->launch_systems > 0 ? cfg->launch_systems : b->nsys;
    const MoveCtx C = alma_make_move_ctx(b, t, nl, p, scratch);
    MCConfigDev d;
    d.seed = cfg->seed;
    d.policy = cfg->policy;
    d.tune_freq = cfg->tune_freq;
    d.target_lo = cfg->target_lo;
    d.target_hi = cfg->target_hi;
    d.scale_up = cfg->scale_up;
    d.scale_down = cfg->scale_down;
    d.angle_max = cfg->angle_max;
    d.angle_min = cfg->angle_min;
    d.sidechain_mult = cfg->sidechain_mult;
    d.crank_prob = cfg->crank_prob;
    d.concerted_prob = cfg->concerted_prob;
    d.fixed_delta = cfg->fixed_delta;
    d.moveset_off = cfg->moveset_off;
    d.moveset = cfg->moveset;
    d.sys_order = cfg->sys_order;
    d.reach_pad = 2.0 * p->probe_r + 2.0 * sqrt(p->half_skin2) + 1e-6;  // as alma_nl_build
    d.rw = carve_rebuild(cfg->rebuild_ws, b->natoms, b->nsys);
    cudaStream_t st = (cudaStream_t)stream;
    // Threads per system: 512 when the batch fits one CTA per SM, else 256
    // (two CTAs per SM), so every chain of a persistent launch is resident.
    // cluster_size CTAs cooperate on each system (1, 2, 4, 8 or 16).
    int nt = cfg->threads_per_system;
    if (nt == 0) {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        nt = nl_sys <= sms ? 512 : 256;
    }
    const int cl = cfg->cluster_size <= 0 ? 1 : cfg->cluster_size;
    if (nt != 256 && nt != 512) return alma_set_error(ALMA_EINVAL, "alma_mc_run: threads_per_system must be 0, 256 or 512");
    if (cl != 1 && cl != 2 && cl != 4 && cl != 8 && cl != 16)
        return alma_set_error(ALMA_EINVAL, "alma_mc_run: cluster_size must be 1, 2, 4, 8 or 16");
    const int teams = cfg->spec_teams <= 1 ? 1 : cfg->spec_teams;
    if (teams > SPEC_MAX_TEAMS) return alma_set_error(ALMA_EINVAL, "alma_mc_run: spec_teams must be <= %d", SPEC_MAX_TEAMS);
    cudaError_t e = cudaSuccess;
    if (teams > 1) {
        const size_t stride = align_up256(alma_move_scratch_bytes(b->natoms));
        SpecRound *rounds = (SpecRound *)((char *)scratch + (size_t)teams * stride);
        ALMA_CUDA_TRY(cudaMemsetAsync(rounds, 0, sizeof(SpecRound) * (size_t)b->nsys, st));
        bool fits = true;
#define ALMA_SPEC_CASE(R, NT)                                                                                   \
    switch (cl) {                                                                                               \
        case 1: e = launch_mc_spec<R, NT, 1>(C, d, states, step_limit, nl_sys, teams, stride, rounds, st, &fits); break;   \
        case 2: e = launch_mc_spec<R, NT, 2>(C, d, states, step_limit, nl_sys, teams, stride, rounds, st, &fits); break;   \
        case 4: e = launch_mc_spec<R, NT, 4>(C, d, states, step_limit, nl_sys, teams, stride, rounds, st, &fits); break;   \
        case 8: e = launch_mc_spec<R, NT, 8>(C, d, states, step_limit, nl_sys, teams, stride, rounds, st, &fits); break;   \
        default: e = launch_mc_spec<R, NT, 16>(C, d, states, step_limit, nl_sys, teams, stride, rounds, st, &fits); break; \
    }
        if (prec == ALMA_PREC_FP64) {
            if (nt == 512) { ALMA_SPEC_CASE(double, 512) } else { ALMA_SPEC_CASE(double, 256) }
        } else {
            if (nt == 512) { ALMA_SPEC_CASE(float, 512) } else { ALMA_SPEC_CASE(float, 256) }
        }
#undef ALMA_SPEC_CASE
        if (e != cudaSuccess) return alma_cuda_error(e, "alma_mc_run launch");
        if (!fits)
            return alma_set_error(ALMA_EINVAL, "alma_mc_run: %d systems x %d teams x %d CTAs cannot all be resident",
                                  nl_sys, teams, cl);
        ALMA_LAUNCH_CHECK("alma_mc_run");
        // In a scratch sized for more teams, the round buffers of a K-team
        // launch lie over the start of team K's move scratch, whose flags
        // must read zero between proposals: leave them zeroed, so a later
        // launch with more teams finds team K clean.
        ALMA_CUDA_TRY(cudaMemsetAsync(rounds, 0, sizeof(SpecRound) * (size_t)b->nsys, st));
        return ALMA_OK;
    }
#define ALMA_MC_CASE(R, NT)                                                              \
    switch (cl) {                                                                        \
        case 1: e = launch_mc<R, NT, 1>(C, d, states, step_limit, nl_sys, st); break;   \
        case 2: e = launch_mc<R, NT, 2>(C, d, states, step_limit, nl_sys, st); break;   \
        case 4: e = launch_mc<R, NT, 4>(C, d, states, step_limit, nl_sys, st); break;   \
        case 8: e = launch_mc<R, NT, 8>(C, d, states, step_limit, nl_sys, st); break;   \
        default: e = launch_mc<R, NT, 16>(C, d, states, step_limit, nl_sys, st); break; \
    }
    if (prec == ALMA_PREC_FP64) {
        if (nt == 512) { ALMA_MC_CASE(double, 512) } else { ALMA_MC_CASE(double, 256) }
    } else {
        if (nt == 512) { ALMA_MC_CASE(float, 512) } else { ALMA_MC_CASE(float, 256) }
    }
#undef ALMA_MC_CASE
    if (e != cudaSuccess) return alma_cuda_error(e, "alma_mc_run launch");
    ALMA_LAUNCH_CHECK("alma_mc_run");
    return ALMA_OK;
}

extern "C" size_t alma_mc_scratch_bytes(int32_t natoms, int32_t nsys, int32_t teams) {
    if (teams <= 1) return alma_move_scratch_bytes(natoms);
    return (size_t)teams * align_up256(alma_move_scratch_bytes(natoms)) +
           align_up256(sizeof(SpecRound) * (size_t)(nsys > 0 ? nsys : 1));
}

extern "C" int alma_mc_after_rebuild(AlmaChainState *states, const double *terms, const uint8_t *sys_mask,
                                     int32_t nsys, void *stream) {
    if (!states || !terms || nsys <= 0) return alma_set_error(ALMA_EINVAL, "alma_mc_after_rebuild: bad arguments");
    mc_after_rebuild_kernel<<<(nsys + 127) / 128, 128, 0, (cudaStream_t)stream>>>(states, terms, sys_mask, nsys);
    ALMA_LAUNCH_CHECK("alma_mc_after_rebuild");
    return ALMA_OK;
}
