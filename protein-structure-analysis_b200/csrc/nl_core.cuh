// Per-atom core of the neighbor-list build, shared by the stand-alone
// build (nl.cu) and the rebuild inside the persistent MC kernel (mc.cu), so
// both produce the same rows in the same order.
#pragma once
#include "alma_common.cuh"

namespace alma {

struct SysGrid {
    double xlo, ylo, zlo, cs;
    int32_t nx, ny, nz;
    float margin2;     // FP32 prefilter margin on r² (Å²), see fp32_margin2
    int64_t cell_off;  // first global cell of this system
    int64_t ncell;
};

// Margin on r² within which an FP32 distance test (coordinates relative to
// the grid origin, so |x| <= the grid's extent E) cannot decide a 14 Å or
// SASA-reach cutoff and the FP64 test runs.  Each coordinate carries at
// most E 2^-24 of rounding, a difference twice that plus its own rounding,
// so near a cutoff r <= 14 Å the squared distance is off by at most
// 2 (2 E 2^-24) sqrt(3) 14 plus a few ulps of 196; the margin takes 16x
// that (0.05 Å² at E = 1,000 Å) and never less than 0.01 Å².
__device__ __forceinline__ float fp32_margin2(double extent) {
    const double d = 2.0 * extent * 5.9604644775390625e-8 + 1e-6;
    return (float)fmax(0.01, 16.0 * (2.0 * d * 1.7320508075688772 * 14.0 + 3.0e-5));
}

// Grid of one system from its bounding box (physics_engine.cpp:299-316):
// cells of 14 Å + 1e-6, the box padded by one cell on every side.
__device__ __forceinline__ SysGrid grid_from_box(const double lo[3], const double hi[3], double nl_rcut2, int natoms) {
    SysGrid g;
    g.cs = sqrt(nl_rcut2) + 1e-6;
    const double mg = g.cs;
    g.xlo = lo[0] - mg; g.ylo = lo[1] - mg; g.zlo = lo[2] - mg;
    const double lx = hi[0] - g.xlo + 2.0 * mg, ly = hi[1] - g.ylo + 2.0 * mg, lz = hi[2] - g.zlo + 2.0 * mg;
    g.nx = max(1, (int)ceil(lx / g.cs));
    g.ny = max(1, (int)ceil(ly / g.cs));
    g.nz = max(1, (int)ceil(lz / g.cs));
    if (natoms <= 0) { g.nx = g.ny = g.nz = 1; }
    g.margin2 = fp32_margin2(fmax(g.nx, fmax(g.ny, g.nz)) * g.cs);
    g.ncell = (int64_t)g.nx * g.ny * g.nz;
    g.cell_off = 0;
    return g;
}

__device__ __forceinline__ int cell_of_point(const SysGrid &g, double4 p) {
    const int cx = min(g.nx - 1, max(0, (int)floor((p.x - g.xlo) / g.cs)));
    const int cy = min(g.ny - 1, max(0, (int)floor((p.y - g.ylo) / g.cs)));
    const int cz = min(g.nz - 1, max(0, (int)floor((p.z - g.zlo) / g.cs)));
    return cx + g.nx * (cy + g.ny * cz);
}

__device__ __forceinline__ bool excluded(const int64_t *__restrict__ excl_ptr, const int32_t *__restrict__ excl_cols,
                                         int i, int j) {
    if (!excl_ptr) return false;
    int lo_i = i < j ? i : j, hi_j = i < j ? j : i;
    int64_t lo = excl_ptr[lo_i], hi = excl_ptr[lo_i + 1];
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (excl_cols[mid] < hi_j) lo = mid + 1;
        else hi = mid;
    }
    return lo < excl_ptr[lo_i + 1] && excl_cols[lo] == hi_j;
}

// Exclusion window (alma_excl_window): bit d + 64 of atom i's 128-bit word
// marks i and i + d as excluded, |d| < 64; bit 64 (d = 0, never a pair)
// marks an exclusion partner outside the window (bit 0 stays unused).  Bonded exclusions
// lie within a few residues, so nearly every pair is decided by one bit of
// a word the warp loaded once; only atoms with a far partner (disulfides)
// search their CSR row for pairs outside the window.
constexpr int EXCL_WIN = 64;

__device__ __forceinline__ uint4 excl_window_of(const uint32_t *__restrict__ win, int i) {
    return win ? __ldg(reinterpret_cast<const uint4 *>(win) + i) : make_uint4(0u, 0u, 0u, 0u);
}

__device__ __forceinline__ bool excluded_w(const uint32_t *win, uint4 w, const int64_t *__restrict__ excl_ptr,
                                           const int32_t *__restrict__ excl_cols, int i, int j) {
    if (!win) return excluded(excl_ptr, excl_cols, i, j);
    const int d = j - i;
    if (d > -EXCL_WIN && d < EXCL_WIN) {
        const unsigned b = (unsigned)(d + EXCL_WIN);
        const uint32_t word = b < 64u ? (b < 32u ? w.x : w.y) : (b < 96u ? w.z : w.w);
        return (word >> (b & 31u)) & 1u;
    }
    return (w.z & 1u) && excluded(excl_ptr, excl_cols, i, j);
}

// The rows of atom i, one warp (27 cells in (dz, dy, dx) order, ascending
// atoms per cell, ballot-compacted).  PASS 0 counts (full, half, short full,
// short half); PASS 1 writes the rows at the list's pointers and ref_xyz.
// cell_start[g.cell_off + c] are absolute positions in cell_atoms.
template <int PASS>
__device__ __forceinline__ void nl_row_atom(int i, int lane, const SysGrid &g, const double *__restrict__ xyz,
                                            double rcut2, const int32_t *__restrict__ cell_of,
                                            const int64_t *__restrict__ cell_start,
                                            const int32_t *__restrict__ cell_atoms, const double *__restrict__ prm64,
                                            double reach_pad, const int64_t *__restrict__ excl_ptr,
                                            const int32_t *__restrict__ excl_cols, const uint32_t *excl_win,
                                            const AlmaNL &nl, int &nfull, int &nhalf, int &nsfull, int &nshalf) {
    const int c = cell_of[i];
    const uint4 ew = excl_window_of(excl_win, i);
    const int cx = c % g.nx, cy = (c / g.nx) % g.ny, cz = c / (g.nx * g.ny);
    const double4 pi = ld_xyz(xyz, i);
    const bool shorts = nl.sfull_cols != nullptr;
    const double ri_pad = shorts ? prm64[4 * (size_t)i + 1] + reach_pad : 0.0;
    int64_t fo = 0, ho = 0, sfo = 0, sho = 0;
    if (PASS == 1) {
        fo = nl.full_ptr[i];
        ho = nl.half_ptr[i];
        if (shorts) {
            sfo = nl.sfull_ptr[i];
            sho = nl.shalf_ptr[i];
        }
        if (lane == 0) *reinterpret_cast<double4 *>(nl.ref_xyz + 4 * (size_t)i) = pi;
    }
    nfull = nhalf = nsfull = nshalf = 0;
    int jmin = 0x7fffffff, jmax = -1;  // index span of the full row (PASS 1)
    for (int dz = -1; dz <= 1; ++dz) {
        const int cz2 = cz + dz;
        if (cz2 < 0 || cz2 >= g.nz) continue;
        for (int dy = -1; dy <= 1; ++dy) {
            const int cy2 = cy + dy;
            if (cy2 < 0 || cy2 >= g.ny) continue;
            for (int dx = -1; dx <= 1; ++dx) {
                const int cx2 = cx + dx;
                if (cx2 < 0 || cx2 >= g.nx) continue;
                const int64_t cell = g.cell_off + cx2 + (int64_t)g.nx * (cy2 + (int64_t)g.ny * cz2);
                const int64_t beg = cell_start[cell], end = cell_start[cell + 1];
                for (int64_t k0 = beg; k0 < end; k0 += 32) {
                    const int64_t k = k0 + lane;
                    int j = -1;
                    bool in = false, sh = false;
                    if (k < end) {
                        j = cell_atoms[k];
                        const double r2 = d2_of(pi, ld_xyz(xyz, j));
                        in = (j != i) && r2 < rcut2;
                        if (in && shorts) {
                            const double reach = ri_pad + prm64[4 * (size_t)j + 1];
                            sh = r2 < reach * reach;
                        }
                    }
                    const unsigned mf = __ballot_sync(0xffffffffu, in);
                    const unsigned mh = __ballot_sync(0xffffffffu, in && j > i);
                    const unsigned msf = __ballot_sync(0xffffffffu, sh);
                    const unsigned msh = __ballot_sync(0xffffffffu, sh && j > i);
                    if (PASS == 1 && in) {
                        jmin = min(jmin, j);
                        jmax = max(jmax, j);
                        const unsigned lt = (1u << lane) - 1u;
                        const uint32_t e =
                            (uint32_t)j | (excluded_w(excl_win, ew, excl_ptr, excl_cols, i, j) ? ALMA_EXCL_BIT : 0u);
                        nl.full_cols[fo + nfull + __popc(mf & lt)] = e;
                        if (j > i) nl.half_cols[ho + nhalf + __popc(mh & lt)] = e;
                        if (sh) {
                            nl.sfull_cols[sfo + nsfull + __popc(msf & lt)] = e;
                            if (j > i) nl.shalf_cols[sho + nshalf + __popc(msh & lt)] = e;
                        }
                    }
                    nfull += __popc(mf);
                    nhalf += __popc(mh);
                    nsfull += __popc(msf);
                    nshalf += __popc(msh);
                }
            }
        }
    }
    if (PASS == 1 && nl.full_span != nullptr) {
        jmin = __reduce_min_sync(0xffffffffu, jmin);
        jmax = __reduce_max_sync(0xffffffffu, jmax);
        if (lane == 0) {
            nl.full_span[2 * (size_t)i] = jmin;
            nl.full_span[2 * (size_t)i + 1] = jmax;
        }
    }
}

}  // namespace alma
