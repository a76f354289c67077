// Host-side pieces of the C ABI: error state, parameter presets, and the
// topology j-side walk.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <atomic>
#include <vector>

#include "alma_b200.h"

namespace {
thread_local char g_err[512] = "";
std::atomic<long long> g_launches{0};
}

void alma_count_launches(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

int alma_set_error(int code, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

int alma_cuda_error(cudaError_t e, const char *what) {
    return alma_set_error(ALMA_ECUDA, "%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
}

extern "C" {

int alma_abi_version(void) { return ALMA_ABI_VERSION; }

const char *alma_last_error(void) { return g_err; }

long long alma_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

// Reference preset: physics_engine.cpp:181-196 (hard core 0.6 sigma, smooth
// and capped at 5000, gamma_SA 0.00542, kappa 0.1257) and the disulfide
// restraint constants at :1948-1950.
void alma_params_reference(AlmaParams *p) {
    p->coulomb = 332.0636;
    p->eps_water = 78.5;
    p->eps_prot = 1.0;
    p->kappa = 0.1257;
    p->gamma_sa = 0.00542;
    p->beta_sa = 0.92;
    p->probe_r = 1.4;
    p->pair_cut2 = 12.0 * 12.0;
    p->nl_rcut2 = (12.0 + 2.0) * (12.0 + 2.0);
    p->half_skin2 = (2.0 * 0.5) * (2.0 * 0.5);
    p->hard_scale = 1.0e4;
    p->hard_cap = 5.0e3;
    p->hard_frac = 0.6;
    p->k_ss = 600.0;
    p->r0_ss = 2.044;
}

// DFS from bj that never enters bi; stack order as BondTopology::j_side
// (physics_engine.cpp:1731-1745): pop the top, skip if visited, record,
// push all neighbours in adjacency order.
int alma_topo_sides(int32_t n, const int64_t *adj_ptr, const int32_t *adj_idx, int32_t nb,
                    const int32_t *bonds, int64_t *side_ptr, int32_t *side_idx, int64_t cap) {
    if (n < 0 || nb < 0 || !adj_ptr || (nb > 0 && (!bonds || !side_ptr)))
        return alma_set_error(ALMA_EINVAL, "alma_topo_sides: bad arguments");
    std::vector<uint32_t> stamp((size_t)n, 0u);
    std::vector<int32_t> stk;
    stk.reserve(64);
    int64_t k = 0;
    side_ptr[0] = 0;
    for (int32_t b = 0; b < nb; ++b) {
        const int32_t bi = bonds[2 * b], bj = bonds[2 * b + 1];
        const uint32_t mark = (uint32_t)b + 1u;
        if (bi < 0 || bi >= n || bj < 0 || bj >= n) {
            side_ptr[b + 1] = k;
            continue;
        }
        stamp[(size_t)bi] = mark;
        stk.clear();
        stk.push_back(bj);
        while (!stk.empty()) {
            int32_t cur = stk.back();
            stk.pop_back();
            if (stamp[(size_t)cur] == mark) continue;
            stamp[(size_t)cur] = mark;
            if (k < cap && side_idx) side_idx[k] = cur;
            ++k;
            for (int64_t e = adj_ptr[cur]; e < adj_ptr[cur + 1]; ++e) stk.push_back(adj_idx[e]);
        }
        side_ptr[b + 1] = k;
    }
    if (k > cap) return alma_set_error(ALMA_ECAPACITY, "alma_topo_sides: need %lld entries", (long long)k);
    return ALMA_OK;
}

// Same walk, compact output: each side as its longest run of consecutive
// atom indices [lo, hi) plus the remaining atoms, sorted, in the CSR
// (ex_ptr, ex_idx).  count[b] = side size.  For residue-ordered chains a
// backbone side is a handful of explicit atoms plus one long range.
int alma_topo_sides_compact(int32_t n, const int64_t *adj_ptr, const int32_t *adj_idx, int32_t nb,
                            const int32_t *bonds, int32_t *lo_out, int32_t *hi_out, int64_t *count,
                            int64_t *ex_ptr, int32_t *ex_idx, int64_t ex_cap) {
    if (n < 0 || nb < 0 || !adj_ptr || (nb > 0 && (!bonds || !lo_out || !hi_out || !count || !ex_ptr)))
        return alma_set_error(ALMA_EINVAL, "alma_topo_sides_compact: bad arguments");
    // The side's atoms are marked in `stamp` by the walk; its sorted order,
    // its longest run of consecutive indices and the remainder all come
    // from one scan of the marks over [min, max] (no sort: for a residue-
    // ordered chain that span is the side itself).
    std::vector<uint32_t> stamp((size_t)n, 0u);
    std::vector<int32_t> stk;
    int64_t k = 0;
    ex_ptr[0] = 0;
    for (int32_t b = 0; b < nb; ++b) {
        const int32_t bi = bonds[2 * b], bj = bonds[2 * b + 1];
        const uint32_t mark = (uint32_t)b + 1u;
        int64_t cnt = 0;
        int32_t mn = n, mx = -1;
        if (bi >= 0 && bi < n && bj >= 0 && bj < n) {
            stamp[(size_t)bi] = mark;
            stk.clear();
            stk.push_back(bj);
            while (!stk.empty()) {
                int32_t cur = stk.back();
                stk.pop_back();
                if (stamp[(size_t)cur] == mark) continue;
                stamp[(size_t)cur] = mark;
                ++cnt;
                mn = std::min(mn, cur);
                mx = std::max(mx, cur);
                for (int64_t e = adj_ptr[cur]; e < adj_ptr[cur + 1]; ++e) stk.push_back(adj_idx[e]);
            }
            // the axis atom i carries the mark too but is not on the side
            stamp[(size_t)bi] = 0u;
        }
        // longest run of consecutive marked indices (first one on ties)
        int32_t best_lo = 0, best_len = 0;
        for (int32_t a = mn; a <= mx;) {
            if (stamp[(size_t)a] != mark) { ++a; continue; }
            int32_t e = a + 1;
            while (e <= mx && stamp[(size_t)e] == mark) ++e;
            if (e - a > best_len) { best_len = e - a; best_lo = a; }
            a = e;
        }
        count[b] = cnt;
        if (best_len >= 2) {
            lo_out[b] = best_lo;
            hi_out[b] = best_lo + best_len;
        } else {
            lo_out[b] = hi_out[b] = 0;
            best_len = 0;
        }
        for (int32_t a = mn; a <= mx; ++a) {
            if (stamp[(size_t)a] != mark) continue;
            if (best_len && a >= best_lo && a < best_lo + best_len) continue;
            if (k < ex_cap && ex_idx) ex_idx[k] = a;
            ++k;
        }
        ex_ptr[b + 1] = k;
    }
    if (k > ex_cap) return alma_set_error(ALMA_ECAPACITY, "alma_topo_sides_compact: need %lld entries", (long long)k);
    return ALMA_OK;
}

// Nesting of the rotatable bonds' j-sides (one system, local indices).  On
// a tree every two j-sides are nested or disjoint: atom_rb[m] = the bond
// with the smallest side that holds atom m, rb_parent[k] = atom_rb[i_k]
// (a side that holds the axis atom i_k holds all of side k).  Sides are
// assigned in decreasing size, so the smallest one wins; the check
// Σ_k |side_k| = Σ_m depth(m) rejects sides that overlap without nesting
// (a ring, e.g. a disulfide, inside the bond graph).
int alma_torsion_tree(int32_t natoms, int32_t nrb, const int32_t *rb_ij, const int64_t *side_ptr,
                      const int32_t *side_idx, const int32_t *side_lo, const int32_t *side_hi, int32_t *rb_parent,
                      int32_t *atom_rb) {
    if (natoms < 0 || nrb < 0 || (natoms > 0 && !atom_rb) ||
        (nrb > 0 && (!rb_ij || !side_ptr || !side_lo || !side_hi || !rb_parent)))
        return alma_set_error(ALMA_EINVAL, "alma_torsion_tree: bad arguments");
    std::vector<int64_t> size((size_t)nrb);
    for (int32_t k = 0; k < nrb; ++k)
        size[(size_t)k] = (side_ptr[k + 1] - side_ptr[k]) + std::max(0, side_hi[k] - side_lo[k]);
    std::vector<int32_t> order((size_t)nrb);
    for (int32_t k = 0; k < nrb; ++k) order[(size_t)k] = k;
    std::stable_sort(order.begin(), order.end(),
                     [&](int32_t a, int32_t b) { return size[(size_t)a] > size[(size_t)b]; });
    for (int32_t m = 0; m < natoms; ++m) atom_rb[m] = -1;
    int64_t total = 0;
    for (int32_t k : order) {
        for (int32_t m = side_lo[k]; m < side_hi[k]; ++m) {
            if (m < 0 || m >= natoms) return alma_set_error(ALMA_EINVAL, "alma_torsion_tree: side atom out of range");
            atom_rb[m] = k;
        }
        for (int64_t e = side_ptr[k]; e < side_ptr[k + 1]; ++e) {
            const int32_t m = side_idx[e];
            if (m < 0 || m >= natoms) return alma_set_error(ALMA_EINVAL, "alma_torsion_tree: side atom out of range");
            atom_rb[m] = k;
        }
        total += size[(size_t)k];
    }
    for (int32_t k = 0; k < nrb; ++k) {
        const int32_t i = rb_ij[2 * k];
        if (i < 0 || i >= natoms) return alma_set_error(ALMA_EINVAL, "alma_torsion_tree: axis atom out of range");
        rb_parent[k] = atom_rb[i];
        if (rb_parent[k] == k || (rb_parent[k] >= 0 && size[(size_t)rb_parent[k]] <= size[(size_t)k]))
            return alma_set_error(ALMA_EINVAL, "alma_torsion_tree: j-sides are not nested (ring in the bond graph)");
    }
    std::vector<int64_t> depth((size_t)nrb, -1);
    int64_t sum = 0;
    for (int32_t m = 0; m < natoms; ++m) {
        int32_t k = atom_rb[m];
        if (k < 0) continue;
        if (depth[(size_t)k] < 0) {  // walk up to a known depth (sizes strictly grow: no cycle)
            std::vector<int32_t> path;
            int32_t c = k;
            while (c >= 0 && depth[(size_t)c] < 0) {
                path.push_back(c);
                c = rb_parent[c];
            }
            int64_t d = c >= 0 ? depth[(size_t)c] : 0;
            for (size_t q = path.size(); q-- > 0;) depth[(size_t)path[q]] = ++d;
        }
        sum += depth[(size_t)k];
    }
    if (sum != total)
        return alma_set_error(ALMA_EINVAL, "alma_torsion_tree: j-sides are not nested (ring in the bond graph)");
    return ALMA_OK;
}

}  // extern "C"

extern "C" size_t alma_struct_size(int32_t which) {
    switch (which) {
        case 0: return sizeof(AlmaParams);
        case 1: return sizeof(AlmaBatch);
        case 2: return sizeof(AlmaTopo);
        case 3: return sizeof(AlmaNL);
        case 4: return sizeof(AlmaMCConfig);
        case 5: return sizeof(AlmaChainState);
        case 6: return sizeof(AlmaTorsionTree);
        case 7: return sizeof(AlmaMalaState);
        case 8: return sizeof(AlmaMalaConfig);
        default: return 0;
    }
}
