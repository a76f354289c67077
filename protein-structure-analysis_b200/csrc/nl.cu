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
//   count  : warp per atom — row lengths
//   rowscan: one CTA per system — row pointers inside the system's region
//   fill   : warp per atom — rows, ballot-compacted in scan order
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
    int32_t *full_cnt;    // [natoms]
    int32_t *half_cnt;    // [natoms]
    int32_t *sfull_cnt;   // [natoms]
    int32_t *shalf_cnt;   // [natoms]
    int64_t *tile_sums;   // scan scratch
    int64_t *total_cells; // [1]
    int32_t *ok;          // [1] 1 when the grid fit
    int32_t *sys_ok;      // [nsys] 1 when the system's rows fit its region
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
    t.full_cnt = (int32_t *)take(sizeof(int32_t) * (size_t)natoms);
    t.half_cnt = (int32_t *)take(sizeof(int32_t) * (size_t)natoms);
    t.sfull_cnt = (int32_t *)take(sizeof(int32_t) * (size_t)natoms);
    t.shalf_cnt = (int32_t *)take(sizeof(int32_t) * (size_t)natoms);
    t.tile_sums = (int64_t *)take(sizeof(int64_t) * (size_t)ntiles);
    t.total_cells = (int64_t *)take(sizeof(int64_t));
    t.ok = (int32_t *)take(sizeof(int32_t));
    t.sys_ok = (int32_t *)take(sizeof(int32_t) * (size_t)(nsys > 0 ? nsys : 1));
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

// One CTA per system: row pointers inside the system's region, overflow
// check, for the four row kinds (full, half, short full, short half; the
// short ones only when the list carries them).
__global__ void nl_rowscan_kernel(const int32_t *__restrict__ atom_off, const uint8_t *__restrict__ mask,
                                  const int32_t *__restrict__ full_cnt, const int32_t *__restrict__ half_cnt,
                                  const int32_t *__restrict__ sfull_cnt, const int32_t *__restrict__ shalf_cnt,
                                  AlmaNL nl, int32_t *__restrict__ sys_ok, uint32_t *__restrict__ status) {
    __shared__ int64_t sm[33];
    const int s = blockIdx.x;
    if (mask && !mask[s]) return;
    const int a0 = atom_off[s], a1 = atom_off[s + 1];
    const int nkind = nl.sfull_cols ? 4 : 2;
    int fits = 1;
    for (int kind = 0; kind < nkind; ++kind) {
        const int32_t *cnt = kind == 0 ? full_cnt : kind == 1 ? half_cnt : kind == 2 ? sfull_cnt : shalf_cnt;
        int64_t *ptr = kind == 0 ? nl.full_ptr : kind == 1 ? nl.half_ptr : kind == 2 ? nl.sfull_ptr : nl.shalf_ptr;
        int32_t *len = kind == 0 ? nl.full_len : kind == 1 ? nl.half_len : kind == 2 ? nl.sfull_len : nl.shalf_len;
        const int64_t *basev = kind == 0 ? nl.full_base : kind == 1 ? nl.half_base : kind == 2 ? nl.sfull_base
                                                                                                : nl.shalf_base;
        const int64_t base = basev[s], cap = basev[s + 1] - base;
        int64_t carry = 0;
        for (int b0 = a0; b0 < a1; b0 += blockDim.x) {
            const int i = b0 + threadIdx.x;
            const int64_t v = i < a1 ? cnt[i] : 0;
            int64_t ex;
            const int64_t tot = block_exclusive_scan(v, ex, sm);
            if (i < a1) {
                ptr[i] = base + carry + ex;
                len[i] = (int32_t)v;
            }
            carry += tot;
        }
        if (threadIdx.x == 0) {
            nl.need[4 * s + kind] = carry;
            if (carry > cap) fits = 0;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        sys_ok[s] = fits;
        if (!fits) set_status(status, ALMA_ST_NL_OVERFLOW);
    }
}

// Warp per atom.  PASS 0 counts, PASS 1 writes.  256 threads, 4 blocks per
// SM (at most 64 registers: the scan is latency bound, occupancy pays).
template <int PASS>
__global__ void __launch_bounds__(256, 4) nl_rows_kernel(const int32_t *__restrict__ atom_off, int nsys, int natoms, const uint8_t *__restrict__ mask,
                               const double *__restrict__ xyz, double rcut2, const SysGrid *__restrict__ grid,
                               const int32_t *__restrict__ ok, const int32_t *__restrict__ cell_of,
                               const int64_t *__restrict__ cell_start, const int32_t *__restrict__ cell_atoms,
                               int32_t *__restrict__ full_cnt, int32_t *__restrict__ half_cnt,
                               int32_t *__restrict__ sfull_cnt, int32_t *__restrict__ shalf_cnt,
                               const double *__restrict__ prm64, double reach_pad,
                               const int64_t *__restrict__ excl_ptr, const int32_t *__restrict__ excl_cols,
                               AlmaNL nl, const int32_t *__restrict__ sys_ok) {
    const int warps_per_block = blockDim.x >> 5;
    const int i = blockIdx.x * warps_per_block + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= natoms || !*ok) return;
    const int s = sys_of_atom(atom_off, nsys, i);
    if (mask && !mask[s]) return;
    if (PASS == 1 && !sys_ok[s]) return;
    const SysGrid g = grid[s];
    int nfull, nhalf, nsfull, nshalf;
    nl_row_atom<PASS>(i, lane, g, xyz, rcut2, cell_of, cell_start, cell_atoms, prm64, reach_pad, excl_ptr, excl_cols,
                      nl, nfull, nhalf, nsfull, nshalf);
    if (PASS == 0 && lane == 0) {
        full_cnt[i] = nfull;
        half_cnt[i] = nhalf;
        sfull_cnt[i] = nsfull;
        shalf_cnt[i] = nshalf;
    }
}

}  // namespace alma

using namespace alma;

extern "C" size_t alma_nl_workspace_bytes(int32_t nsys, int32_t natoms, int64_t max_cells) {
    return carve(nullptr, nullptr, nsys, natoms, max_cells);
}

extern "C" int alma_nl_build(const AlmaBatch *b, const AlmaTopo *t, AlmaNL *nl, const AlmaParams *p,
                             const uint8_t *sys_mask, void *workspace, int64_t max_cells, void *stream) {
    if (!b || !nl || !workspace || b->nsys <= 0 || b->natoms < 0 || max_cells <= 0)
        return alma_set_error(ALMA_EINVAL, "alma_nl_build: bad arguments");
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
    // Oversized cells (> SORT_SMEM atoms) sort through half_cnt as spill
    // space: it holds natoms ints and is only written later by the count pass.
    nl_cellsort_kernel<<<1184, 256, 0, st>>>(w.total_cells, w.ok, w.cell_start, w.cell_atoms, w.half_cnt);
    const int wpb = 8, rb = (natoms + wpb - 1) / wpb;
    const int64_t *ep = t ? t->excl_ptr : nullptr;
    const int32_t *ec = t ? t->excl_cols : nullptr;
    nl_rows_kernel<0><<<rb, wpb * 32, 0, st>>>(b->atom_off, nsys, natoms, sys_mask, b->xyz, rcut2, w.grid, w.ok,
                                               w.cell_of, w.cell_start, w.cell_atoms, w.full_cnt, w.half_cnt,
                                               w.sfull_cnt, w.shalf_cnt, b->prm64, reach_pad, ep, ec, *nl, w.sys_ok);
    nl_rowscan_kernel<<<nsys, 1024, 0, st>>>(b->atom_off, sys_mask, w.full_cnt, w.half_cnt, w.sfull_cnt, w.shalf_cnt,
                                             *nl, w.sys_ok, b->status);
    nl_rows_kernel<1><<<rb, wpb * 32, 0, st>>>(b->atom_off, nsys, natoms, sys_mask, b->xyz, rcut2, w.grid, w.ok,
                                               w.cell_of, w.cell_start, w.cell_atoms, w.full_cnt, w.half_cnt,
                                               w.sfull_cnt, w.shalf_cnt, b->prm64, reach_pad, ep, ec, *nl, w.sys_ok);
    ALMA_LAUNCH_CHECK_N("alma_nl_build", 11);
    return ALMA_OK;
}
