// Neighbor-list build on the device.
//
// Reproduces NeighborList::build (physics_engine.cpp:293-342) bit-exactly,
// including row order: a 14 Å+1e-6 cubic cell grid over the system's
// bounding box padded by one cell, atoms binned by floor((x-lo)/cs), and
// each row listing the atoms of the 27 neighbour cells in (dz, dy, dx)
// order, ascending atom index inside a cell, keeping r² < 14² (FP64).
// The half row keeps j > i (the reference's nb[i]); the full row keeps every
// j != i (used by Born radii and the move kernels, where the order is
// irrelevant).  Each entry carries the 1-2/1-3/SS exclusion flag in bit 31.
//
// Pipeline (all stream-ordered, no host sync):
//   grid   : one CTA per system — FP64 bounding box, cell-grid shape
//   offsets: one CTA — per-system cell offsets, capacity check
//   bin    : atom -> cell, cell histogram
//   scan   : cell starts
//   scatter: atoms into cells, then a per-cell rank sort (ascending index)
//   cellpos: FP32 positions (relative to the grid origin) and R* in cell
//            order, so the row scan streams its candidates coalesced
//   rows   : warp per atom — one scan stages the row in shared memory,
//            takes space from the system's cursors, writes the four rows
//            ballot-compacted in scan order
//   final  : per system — entry counts, overflow flag
// Every stage honours an optional per-system mask, so systems can be
// rebuilt independently (the MC driver rebuilds only chains that drifted).
#include <cstdio>

#include "alma_common.cuh"
#include "alma_scan.cuh"
#include "nl_core.cuh"

namespace alma {

struct NLWork {
    SysGrid *grid;        // [nsys]
    int32_t *cell_of;     // [natoms] local cell index
    int32_t *cell_count;  // [max_cells]
    int32_t *cell_fill;   // [max_cells]
    int64_t *cell_start;  // [max_cells+1]
    int32_t *cell_atoms;  // [natoms]
    float4 *cell_pos;     // [natoms] per cell slot: FP32 position relative to the grid origin, R*
    int32_t *sort_spill;  // [natoms] rank-sort space for oversized cells
    int64_t *tile_sums;   // scan scratch
    int64_t *total_cells; // [1]
    int32_t *ok;          // [1] 1 when the grid fit
    int32_t *sys_ok;      // [nsys] 1 when the system's rows fit its region
    int64_t *cursor;      // [4*nsys] next free entry of each row kind in the system's region
};

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

static size_t carve(NLWork *w, char *base, int32_t nsys, int32_t natoms, int64_t max_cells) {
    size_t off = 0;
    auto take = [&](size_t bytes) {
        char *p = base ? base + off : nullptr;
        off += align256(bytes);
        return p;
    };
    const int64_t big = (max_cells + 1 > (int64_t)natoms + 1) ? max_cells + 1 : (int64_t)natoms + 1;
    const int64_t ntiles = scan_num_tiles(big) + 1;
    NLWork t;
    t.grid = (SysGrid *)take(sizeof(SysGrid) * (size_t)(nsys > 0 ? nsys : 1));
    t.cell_of = (int32_t *)take(sizeof(int32_t) * (size_t)natoms);
    t.cell_count = (int32_t *)take(sizeof(int32_t) * (size_t)max_cells);
    t.cell_fill = (int32_t *)take(sizeof(int32_t) * (size_t)max_cells);
    t.cell_start = (int64_t *)take(sizeof(int64_t) * (size_t)(max_cells + 1));
    t.cell_atoms = (int32_t *)take(sizeof(int32_t) * (size_t)natoms);
    t.cell_pos = (float4 *)take(sizeof(float4) * (size_t)natoms);
    t.sort_spill = (int32_t *)take(sizeof(int32_t) * (size_t)natoms);
    t.tile_sums = (int64_t *)take(sizeof(int64_t) * (size_t)ntiles);
    t.total_cells = (int64_t *)take(sizeof(int64_t));
    t.ok = (int32_t *)take(sizeof(int32_t));
    t.sys_ok = (int32_t *)take(sizeof(int32_t) * (size_t)(nsys > 0 ? nsys : 1));
    t.cursor = (int64_t *)take(sizeof(int64_t) * 4 * (size_t)(nsys > 0 ? nsys : 1));
    if (w) *w = t;
    return off;
}

// One CTA per system: bounding box and grid shape (physics_engine.cpp:299-316).
// A system outside the mask gets a 1x1x1 grid that no atom uses.
__global__ void nl_grid_kernel(const int32_t *__restrict__ atom_off, const uint8_t *__restrict__ mask,
                               const double *__restrict__ xyz, double nl_rcut2, SysGrid *__restrict__ grid) {
    __shared__ double red[6][32];
    const int s = blockIdx.x;
    const int a0 = atom_off[s], a1 = (mask && !mask[s]) ? atom_off[s] : atom_off[s + 1];
    double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
    for (int i = a0 + threadIdx.x; i < a1; i += blockDim.x) {
        const double4 p = ld_xyz(xyz, i);
        mn[0] = fmin(mn[0], p.x); mx[0] = fmax(mx[0], p.x);
        mn[1] = fmin(mn[1], p.y); mx[1] = fmax(mx[1], p.y);
        mn[2] = fmin(mn[2], p.z); mx[2] = fmax(mx[2], p.z);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int d = 0; d < 3; ++d) {
        double a = mn[d], b = mx[d];
        for (int o = 16; o > 0; o >>= 1) {
            a = fmin(a, __shfl_xor_sync(0xffffffffu, a, o));
            b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
        }
        if (lane == 0) { red[d][wid] = a; red[3 + d][wid] = b; }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nw = blockDim.x >> 5;
        double lo[3], hi[3];
        for (int d = 0; d < 3; ++d) {
            lo[d] = red[d][0]; hi[d] = red[3 + d][0];
            for (int w = 1; w < nw; ++w) { lo[d] = fmin(lo[d], red[d][w]); hi[d] = fmax(hi[d], red[3 + d][w]); }
        }
        SysGrid g = grid_from_box(lo, hi, nl_rcut2, a1 - a0);
        grid[s] = g;
    }
}

__global__ void nl_offsets_kernel(int nsys, SysGrid *__restrict__ grid, int64_t max_cells,
                                  int64_t *__restrict__ total_cells, int32_t *__restrict__ ok,
                                  uint32_t *__restrict__ status) {
    if (threadIdx.x != 0) return;
    int64_t acc = 0;
    for (int s = 0; s < nsys; ++s) {
        grid[s].cell_off = acc;
        acc += grid[s].ncell;
    }
    *total_cells = acc;
    const int fits = acc <= max_cells;
    *ok = fits;
    if (!fits) set_status(status, ALMA_ST_CELL_OVERFLOW);
}

__global__ void nl_bin_kernel(const int32_t *__restrict__ atom_off, int nsys, int natoms,
                              const uint8_t *__restrict__ mask, const double *__restrict__ xyz,
                              const SysGrid *__restrict__ grid, const int32_t *__restrict__ ok,
                              int32_t *__restrict__ cell_of, int32_t *__restrict__ cell_count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= natoms || !*ok) return;
    const int s = sys_of_atom(atom_off, nsys, i);
    if (mask && !mask[s]) return;
    const SysGrid g = grid[s];
    const int c = cell_of_point(g, ld_xyz(xyz, i));
    cell_of[i] = c;
    atomicAdd(&cell_count[g.cell_off + c], 1);
}

__global__ void nl_scatter_kernel(const int32_t *__restrict__ atom_off, int nsys, int natoms,
                                  const uint8_t *__restrict__ mask, const SysGrid *__restrict__ grid,
                                  const int32_t *__restrict__ ok, const int32_t *__restrict__ cell_of,
                                  const int64_t *__restrict__ cell_start, int32_t *__restrict__ cell_fill,
                                  int32_t *__restrict__ cell_atoms) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= natoms || !*ok) return;
    const int s = sys_of_atom(atom_off, nsys, i);
    if (mask && !mask[s]) return;
    const int64_t c = grid[s].cell_off + cell_of[i];
    const int slot = atomicAdd(&cell_fill[c], 1);
    cell_atoms[cell_start[c] + slot] = i;
}

// Sorts every cell's atom list ascending (the reference pushes atoms in
// index order).  Rank sort: each element's position is the number of
// smaller elements (indices are distinct).
constexpr int SORT_SMEM = 2048;
__global__ void nl_cellsort_kernel(const int64_t *__restrict__ total_cells, const int32_t *__restrict__ ok,
                                   const int64_t *__restrict__ cell_start, int32_t *__restrict__ cell_atoms,
                                   int32_t *__restrict__ spill) {
    __shared__ int32_t buf[SORT_SMEM];
    if (!*ok) return;
    const int64_t nc = *total_cells;
    for (int64_t c = blockIdx.x; c < nc; c += gridDim.x) {
        const int64_t b = cell_start[c];
        const int m = (int)(cell_start[c + 1] - b);
        if (m <= 1) continue;
        int32_t *src = cell_atoms + b;
        if (m <= SORT_SMEM) {
            for (int k = threadIdx.x; k < m; k += blockDim.x) buf[k] = src[k];
            __syncthreads();
            for (int k = threadIdx.x; k < m; k += blockDim.x) {
                const int32_t v = buf[k];
                int rank = 0;
                for (int q = 0; q < m; ++q) rank += buf[q] < v;
                src[rank] = v;
            }
            __syncthreads();
        } else {
            // Oversized cell: rank in global memory through the spill buffer
            // (same positions as cell_atoms), then copy back.
            int32_t *tmp = spill + b;
            for (int k = threadIdx.x; k < m; k += blockDim.x) {
                const int32_t v = src[k];
                int rank = 0;
                for (int q = 0; q < m; ++q) rank += src[q] < v;
                tmp[rank] = v;
            }
            __syncthreads();
            for (int k = threadIdx.x; k < m; k += blockDim.x) src[k] = tmp[k];
            __syncthreads();
        }
    }
}

// Cell-ordered copy of the candidates' positions for the row scan: slot k
// of cell_atoms gets its atom's position relative to its system's grid
// origin in FP32 and its R* (the SASA-reach radius).  The 27-cell scan then
// reads each 32-candidate chunk as one coalesced 512-byte load instead of
// 32 scattered FP64 gathers; FP64 decides only inside the margin.
__global__ void nl_cellpos_kernel(const int32_t *__restrict__ atom_off, int nsys, int natoms,
                                  const int64_t *__restrict__ total_cells, const int32_t *__restrict__ ok,
                                  const int64_t *__restrict__ cell_start, const int32_t *__restrict__ cell_atoms,
                                  const SysGrid *__restrict__ grid, const double *__restrict__ xyz,
                                  const double *__restrict__ prm64, float4 *__restrict__ cell_pos) {
    if (!*ok) return;
    const int64_t used = cell_start[*total_cells];
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < used && k < natoms;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int j = cell_atoms[k];
        const SysGrid g = grid[sys_of_atom(atom_off, nsys, j)];
        const double4 p = ld_xyz(xyz, j);
        cell_pos[k] = make_float4((float)(p.x - g.xlo), (float)(p.y - g.ylo), (float)(p.z - g.zlo),
                                  prm64 ? (float)prm64[4 * (size_t)j + 1] : 0.0f);
    }
}

// Entries of one row staged per warp in shared memory by the one-pass
// build (48 KB per 8-warp block); a longer row is scanned a second time.
constexpr int NL_STAGE = 1536;
constexpr uint32_t NL_SHORT_BIT = 0x40000000u;  // staging only: the pair is within SASA reach

// One-pass build, warp per atom: the 27-cell scan stages the row (exclusion
// flag in bit 31, SASA-reach flag in bit 30) in shared memory in scan
// order, lane 0 then takes space for the four rows from the system's
// cursors (one atomic per row kind), and the warp writes the full row, the
// half row (j > i) and the short rows from the staged entries — the same
// rows, in the same order, as counting and filling in two scans.  Rows sit
// in their system's region in the order the warps reach the cursors; every
// reader goes through ptr/len.  A row that would overflow its region is not
// written (nl_finalize_kernel raises the overflow); a row longer than the
// stage is written by a second scan straight into its space.
__global__ void __launch_bounds__(256, 4)
nl_rows_onepass_kernel(const int32_t *__restrict__ atom_off, int nsys, int natoms, const uint8_t *__restrict__ mask,
                       const double *__restrict__ xyz, double rcut2, const SysGrid *__restrict__ grid,
                       const int32_t *__restrict__ ok, const int32_t *__restrict__ cell_of,
                       const int64_t *__restrict__ cell_start, const int32_t *__restrict__ cell_atoms,
                       const float4 *__restrict__ cell_pos, const double *__restrict__ prm64, double reach_pad,
                       const int64_t *__restrict__ excl_ptr, const int32_t *__restrict__ excl_cols,
                       const uint32_t *__restrict__ excl_win, AlmaNL nl, int64_t *__restrict__ cursor) {
    extern __shared__ uint32_t nl_stage_smem[];
    const int warps_per_block = blockDim.x >> 5;
    const int i = blockIdx.x * warps_per_block + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= natoms || !*ok) return;
    const int s = sys_of_atom(atom_off, nsys, i);
    if (mask && !mask[s]) return;
    const SysGrid g = grid[s];
    uint32_t *stage = nl_stage_smem + (threadIdx.x >> 5) * NL_STAGE;
    const bool shorts = nl.sfull_cols != nullptr;
    const int c = cell_of[i];
    const int cx = c % g.nx, cy = (c / g.nx) % g.ny, cz = c / (g.nx * g.ny);
    const double4 pi = ld_xyz(xyz, i);
    const double ri_pad = shorts ? prm64[4 * (size_t)i + 1] + reach_pad : 0.0;
    const uint4 ew = excl_window_of(excl_win, i);
    // the FP32 frame of the cell copy; r² within margin2 of a cutoff is
    // decided in FP64, so the rows are those of the FP64 test bit for bit
    const float pfx = (float)(pi.x - g.xlo), pfy = (float)(pi.y - g.ylo), pfz = (float)(pi.z - g.zlo);
    const float m2 = g.margin2, cut_lo = (float)rcut2 - m2, cut_hi = (float)rcut2 + m2;
    const float rpad_f = (float)ri_pad;
    int nfull = 0, nhalf = 0, nsfull = 0, nshalf = 0;
    int jmin = 0x7fffffff, jmax = -1;
    const unsigned lt = (1u << lane) - 1u;
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
                        const float4 q = cell_pos[k];
                        const float dx = q.x - pfx, dy = q.y - pfy, dz = q.z - pfz;
                        const float r2f = dx * dx + dy * dy + dz * dz;
                        if (r2f < cut_hi && j != i) {
                            double r2 = -1.0;  // FP64 r², computed only when a test needs it
                            if (r2f > cut_lo) {
                                r2 = d2_of(pi, ld_xyz(xyz, j));
                                in = r2 < rcut2;
                            } else {
                                in = true;
                            }
                            if (in && shorts) {
                                const float rf = rpad_f + q.w, rf2 = rf * rf;
                                if (r2f < rf2 - m2) {
                                    sh = true;
                                } else if (r2f <= rf2 + m2) {
                                    if (r2 < 0.0) r2 = d2_of(pi, ld_xyz(xyz, j));
                                    const double reach = ri_pad + prm64[4 * (size_t)j + 1];
                                    sh = r2 < reach * reach;
                                }
                            }
                        }
                    }
                    const unsigned mf = __ballot_sync(0xffffffffu, in);
                    const int at = nfull + __popc(mf & lt);
                    if (in) {
                        jmin = min(jmin, j);
                        jmax = max(jmax, j);
                        if (at < NL_STAGE)
                            stage[at] = (uint32_t)j |
                                        (excluded_w(excl_win, ew, excl_ptr, excl_cols, i, j) ? ALMA_EXCL_BIT : 0u) |
                                        (sh ? NL_SHORT_BIT : 0u);
                    }
                    // the other row kinds are counted from the stage after the
                    // scan; only entries past its end (a rare long row) here
                    if (nfull + __popc(mf) > NL_STAGE) {
                        const bool over = in && at >= NL_STAGE;
                        nhalf += __popc(__ballot_sync(0xffffffffu, over && j > i));
                        nsfull += __popc(__ballot_sync(0xffffffffu, over && sh));
                        nshalf += __popc(__ballot_sync(0xffffffffu, over && sh && j > i));
                    }
                    nfull += __popc(mf);
                }
            }
        }
    }
    __syncwarp();
    for (int t0 = 0; t0 < min(nfull, NL_STAGE); t0 += 32) {  // half / short counts of the staged entries
        const int t = t0 + lane;
        const uint32_t st = t < min(nfull, NL_STAGE) ? stage[t] : 0u;
        const bool v = t < min(nfull, NL_STAGE);
        const bool hf = v && (int)(st & ALMA_IDX_MASK & ~NL_SHORT_BIT) > i, sh = v && (st & NL_SHORT_BIT);
        nhalf += __popc(__ballot_sync(0xffffffffu, hf));
        nsfull += __popc(__ballot_sync(0xffffffffu, sh));
        nshalf += __popc(__ballot_sync(0xffffffffu, hf && sh));
    }
    // space in the system's regions (relative offsets; -1: does not fit)
    int64_t off[4] = {0, 0, 0, 0};
    const int nkind = shorts ? 4 : 2;
    if (lane == 0) {
        const int n[4] = {nfull, nhalf, nsfull, nshalf};
        const int64_t *basev[4] = {nl.full_base, nl.half_base, nl.sfull_base, nl.shalf_base};
        for (int kd = 0; kd < nkind; ++kd) {
            const int64_t o = atomicAdd(reinterpret_cast<unsigned long long *>(cursor + 4 * s + kd),
                                        (unsigned long long)n[kd]);
            off[kd] = o + n[kd] <= basev[kd][s + 1] - basev[kd][s] ? basev[kd][s] + o : -1;
        }
    }
    for (int kd = 0; kd < 4; ++kd) off[kd] = __shfl_sync(0xffffffffu, off[kd], 0);
    bool fits = true;
    for (int kd = 0; kd < nkind; ++kd) fits = fits && off[kd] >= 0;
    if (!fits) return;  // the system overflows: nl_finalize_kernel flags it
    if (lane == 0) {
        nl.full_ptr[i] = off[0];
        nl.full_len[i] = nfull;
        nl.half_ptr[i] = off[1];
        nl.half_len[i] = nhalf;
        if (shorts) {
            nl.sfull_ptr[i] = off[2];
            nl.sfull_len[i] = nsfull;
            nl.shalf_ptr[i] = off[3];
            nl.shalf_len[i] = nshalf;
        }
    }
    if (nfull > NL_STAGE) {  // too long to stage: scan again, writing at the pointers just set
        __syncwarp();
        int a, bb, cc, dd;
        nl_row_atom<1>(i, lane, g, xyz, rcut2, cell_of, cell_start, cell_atoms, prm64, reach_pad, excl_ptr, excl_cols,
                       excl_win, nl, a, bb, cc, dd);
        return;
    }
    __syncwarp();
    if (lane == 0) *reinterpret_cast<double4 *>(nl.ref_xyz + 4 * (size_t)i) = pi;
    int wf = 0, wh = 0, wsf = 0, wsh = 0;
    for (int t0 = 0; t0 < nfull; t0 += 32) {
        const int t = t0 + lane;
        const bool v = t < nfull;
        const uint32_t st = v ? stage[t] : 0u;
        const uint32_t e = st & ~NL_SHORT_BIT;
        const int j = (int)(st & ALMA_IDX_MASK & ~NL_SHORT_BIT);
        const bool hf = v && j > i, sh = v && (st & NL_SHORT_BIT);
        const unsigned mh = __ballot_sync(0xffffffffu, hf);
        const unsigned msf = __ballot_sync(0xffffffffu, sh);
        const unsigned msh = __ballot_sync(0xffffffffu, sh && hf);
        if (v) nl.full_cols[off[0] + t] = e;
        if (hf) nl.half_cols[off[1] + wh + __popc(mh & lt)] = e;
        if (sh) {
            nl.sfull_cols[off[2] + wsf + __popc(msf & lt)] = e;
            if (hf) nl.shalf_cols[off[3] + wsh + __popc(msh & lt)] = e;
        }
        wf += 32;
        wh += __popc(mh);
        wsf += __popc(msf);
        wsh += __popc(msh);
    }
    (void)wf;
    if (nl.full_span != nullptr) {
        jmin = __reduce_min_sync(0xffffffffu, jmin);
        jmax = __reduce_max_sync(0xffffffffu, jmax);
        if (lane == 0) {
            nl.full_span[2 * (size_t)i] = jmin;
            nl.full_span[2 * (size_t)i + 1] = jmax;
        }
    }
}

// Per system after the one-pass build: entry counts into need[], overflow
// into the status word.
__global__ void nl_finalize_kernel(int nsys, const uint8_t *__restrict__ mask, const int32_t *__restrict__ ok,
                                   const int64_t *__restrict__ cursor, AlmaNL nl, uint32_t *__restrict__ status) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsys || !*ok || (mask && !mask[s])) return;
    const int nkind = nl.sfull_cols ? 4 : 2;
    const int64_t *basev[4] = {nl.full_base, nl.half_base, nl.sfull_base, nl.shalf_base};
    bool fits = true;
    for (int kd = 0; kd < nkind; ++kd) {
        const int64_t n = cursor[4 * s + kd];
        nl.need[4 * s + kd] = n;
        fits = fits && n <= basev[kd][s + 1] - basev[kd][s];
    }
    if (!fits) set_status(status, ALMA_ST_NL_OVERFLOW);
}

// Exclusion windows (alma_excl_window): thread per atom over its CSR row
// (partners j > i); each pair sets its bit in both atoms' windows, or the
// far flag (bit 64) of both when j - i >= EXCL_WIN.
__global__ void excl_window_kernel(const int64_t *__restrict__ excl_ptr, const int32_t *__restrict__ excl_cols,
                                   int natoms, uint32_t *__restrict__ win) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= natoms) return;
    for (int64_t k = excl_ptr[i]; k < excl_ptr[i + 1]; ++k) {
        const int j = excl_cols[k];
        if (j < 0 || j >= natoms || j == i) continue;
        const int d = j - i;
        if (d > -EXCL_WIN && d < EXCL_WIN) {
            const unsigned bi = (unsigned)(d + EXCL_WIN), bj = (unsigned)(EXCL_WIN - d);
            atomicOr(&win[4 * (size_t)i + (bi >> 5)], 1u << (bi & 31u));
            atomicOr(&win[4 * (size_t)j + (bj >> 5)], 1u << (bj & 31u));
        } else {
            atomicOr(&win[4 * (size_t)i + 2], 1u);
            atomicOr(&win[4 * (size_t)j + 2], 1u);
        }
    }
}

}  // namespace alma

using namespace alma;

extern "C" int alma_excl_window(const int64_t *excl_ptr, const int32_t *excl_cols, int32_t natoms, uint32_t *win,
                                void *stream) {
    if (natoms < 0 || (natoms > 0 && (!excl_ptr || !excl_cols || !win)))
        return alma_set_error(ALMA_EINVAL, "alma_excl_window: bad arguments");
    if (natoms == 0) return ALMA_OK;
    cudaStream_t st = (cudaStream_t)stream;
    ALMA_CUDA_TRY(cudaMemsetAsync(win, 0, sizeof(uint32_t) * 4 * (size_t)natoms, st));
    excl_window_kernel<<<(natoms + 255) / 256, 256, 0, st>>>(excl_ptr, excl_cols, natoms, win);
    ALMA_LAUNCH_CHECK("alma_excl_window");
    return ALMA_OK;
}

extern "C" size_t alma_nl_workspace_bytes(int32_t nsys, int32_t natoms, int64_t max_cells) {
    return carve(nullptr, nullptr, nsys, natoms, max_cells);
}

extern "C" int alma_nl_build(const AlmaBatch *b, const AlmaTopo *t, AlmaNL *nl, const AlmaParams *p,
                             const uint8_t *sys_mask, void *workspace, int64_t max_cells, void *stream) {
    if (!b || !nl || !workspace || b->nsys <= 0 || b->natoms < 0 || max_cells <= 0)
        return alma_set_error(ALMA_EINVAL, "alma_nl_build: bad arguments");
    if (b->natoms >= (1 << 30))  // the build stages a flag in bit 30 of each entry
        return alma_set_error(ALMA_EINVAL, "alma_nl_build: at most 2^30 - 1 atoms");
    if (!nl->full_ptr || !nl->full_len || !nl->half_ptr || !nl->half_len || !nl->full_base || !nl->half_base ||
        !nl->ref_xyz || !nl->need || !b->xyz || !b->atom_off)
        return alma_set_error(ALMA_EINVAL, "alma_nl_build: null buffer");
    if (nl->sfull_cols && (!nl->sfull_ptr || !nl->sfull_len || !nl->sfull_base || !nl->shalf_ptr || !nl->shalf_len ||
                           !nl->shalf_cols || !nl->shalf_base || !b->prm64))
        return alma_set_error(ALMA_EINVAL, "alma_nl_build: incomplete short rows");
    AlmaParams pref;
    if (!p) {
        alma_params_reference(&pref);
        p = &pref;
    }
    // SASA reach R*_i + R*_j + 2 probe, plus the skin (both atoms may each
    // drift half the skin before a rebuild).
    // A 1e-6 A margin keeps rounding at the boundary on the safe side.
    const double reach_pad = 2.0 * p->probe_r + 2.0 * sqrt(p->half_skin2) + 1e-6;
    cudaStream_t st = (cudaStream_t)stream;
    const int nsys = b->nsys, natoms = b->natoms;
    NLWork w;
    carve(&w, (char *)workspace, nsys, natoms, max_cells);
    if (natoms == 0) return ALMA_OK;
    ALMA_CUDA_TRY(cudaMemsetAsync(w.cell_count, 0, sizeof(int32_t) * (size_t)max_cells, st));
    ALMA_CUDA_TRY(cudaMemsetAsync(w.cell_fill, 0, sizeof(int32_t) * (size_t)max_cells, st));
    const double rcut2 = (12.0 + 2.0) * (12.0 + 2.0);
    nl_grid_kernel<<<nsys, 256, 0, st>>>(b->atom_off, sys_mask, b->xyz, rcut2, w.grid);
    nl_offsets_kernel<<<1, 32, 0, st>>>(nsys, w.grid, max_cells, w.total_cells, w.ok, b->status);
    const int tb = 256, nb = (natoms + tb - 1) / tb;
    nl_bin_kernel<<<nb, tb, 0, st>>>(b->atom_off, nsys, natoms, sys_mask, b->xyz, w.grid, w.ok, w.cell_of,
                                     w.cell_count);
    exclusive_scan<int32_t>(w.cell_count, w.cell_start, max_cells, w.tile_sums, st);
    nl_scatter_kernel<<<nb, tb, 0, st>>>(b->atom_off, nsys, natoms, sys_mask, w.grid, w.ok, w.cell_of, w.cell_start,
                                         w.cell_fill, w.cell_atoms);
    // oversized cells (> SORT_SMEM atoms) sort through the spill space
    nl_cellsort_kernel<<<1184, 256, 0, st>>>(w.total_cells, w.ok, w.cell_start, w.cell_atoms, w.sort_spill);
    nl_cellpos_kernel<<<nb, tb, 0, st>>>(b->atom_off, nsys, natoms, w.total_cells, w.ok, w.cell_start, w.cell_atoms,
                                         w.grid, b->xyz, b->prm64, w.cell_pos);
    const int wpb = 8, rb = (natoms + wpb - 1) / wpb;
    const int64_t *ep = t ? t->excl_ptr : nullptr;
    const int32_t *ec = t ? t->excl_cols : nullptr;
    const uint32_t *ew = t && t->excl_ptr ? t->excl_win : nullptr;
    ALMA_CUDA_TRY(cudaMemsetAsync(w.cursor, 0, sizeof(int64_t) * 4 * (size_t)nsys, st));
    nl_rows_onepass_kernel<<<rb, wpb * 32, sizeof(uint32_t) * NL_STAGE * wpb, st>>>(
        b->atom_off, nsys, natoms, sys_mask, b->xyz, rcut2, w.grid, w.ok, w.cell_of, w.cell_start, w.cell_atoms,
        w.cell_pos, b->prm64, reach_pad, ep, ec, ew, *nl, w.cursor);
    nl_finalize_kernel<<<(nsys + 255) / 256, 256, 0, st>>>(nsys, sys_mask, w.ok, w.cursor, *nl, b->status);
    ALMA_LAUNCH_CHECK_N("alma_nl_build", 11);
    return ALMA_OK;
}
