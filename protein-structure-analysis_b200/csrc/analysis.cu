// Ensemble metrics over snapshots resident on the device: the mean Cα-Cα
// distance matrix and the contact-frequency matrix (compute_mean_dist_matrix
// and compute_contact_freq_matrix, analysis_ext.cpp:85-170; callers
// gui_main.py:1075-1200).  coords: [n_snaps, n_ca, 3] FP64.
//
// 32x32 tiles of the (i, j) matrix, one thread per cell of the upper
// triangle (the lower one is its mirror); each snapshot's coordinates of
// the tile's rows and columns are staged in shared memory.  Every cell sums
// its snapshots in order, as the reference's outer loop does, then scales
// by 1/n_snaps.
#include "alma_common.cuh"

namespace alma {

constexpr int AN_TILE = 32;

template <bool CONTACT>
__global__ void __launch_bounds__(AN_TILE * 8)
ensemble_matrix_kernel(const double *__restrict__ coords, int n_snaps, int n_ca, double cutoff2,
                       double *__restrict__ out) {
    __shared__ double ci[AN_TILE][3], cj[AN_TILE][3];
    const int ti = blockIdx.y, tj = blockIdx.x;
    if (tj < ti) return;  // upper triangle of tiles
    const int i0 = ti * AN_TILE, j0 = tj * AN_TILE;
    const int tx = threadIdx.x & (AN_TILE - 1), ty = threadIdx.x / AN_TILE;  // 32 x 8 threads
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int s = 0; s < n_snaps; ++s) {
        const double *snap = coords + (size_t)s * n_ca * 3;
        __syncthreads();
        for (int q = threadIdx.x; q < AN_TILE * 3; q += blockDim.x) {
            const int a = q / 3, d = q % 3;
            ci[a][d] = i0 + a < n_ca ? snap[(size_t)(i0 + a) * 3 + d] : 0.0;
            cj[a][d] = j0 + a < n_ca ? snap[(size_t)(j0 + a) * 3 + d] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int a = ty + 8 * r;
            const double dx = ci[a][0] - cj[tx][0], dy = ci[a][1] - cj[tx][1], dz = ci[a][2] - cj[tx][2];
            const double d2 = dx * dx + dy * dy + dz * dz;
            if (CONTACT) acc[r] += d2 < cutoff2 ? 1.0 : 0.0;
            else acc[r] += sqrt(d2);
        }
    }
    const double inv = n_snaps > 0 ? 1.0 / (double)n_snaps : 0.0;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int i = i0 + ty + 8 * r, j = j0 + tx;
        if (i >= n_ca || j >= n_ca) continue;
        if (j > i) {
            out[(size_t)i * n_ca + j] = acc[r] * inv;
            out[(size_t)j * n_ca + i] = acc[r] * inv;
        } else if (j == i) {
            out[(size_t)i * n_ca + i] = 0.0;
        }
    }
}

template <bool CONTACT>
static int ensemble_matrix(const double *coords, int32_t n_snaps, int32_t n_ca, double cutoff, double *out,
                           void *stream, const char *who) {
    if (n_snaps < 0 || n_ca < 0 || (n_ca > 0 && (!coords && n_snaps > 0)) || (n_ca > 0 && !out))
        return alma_set_error(ALMA_EINVAL, "%s: bad arguments", who);
    if (n_ca == 0) return ALMA_OK;
    const int nt = (n_ca + AN_TILE - 1) / AN_TILE;
    if (nt > 65535) return alma_set_error(ALMA_EINVAL, "%s: n_ca too large", who);
    ensemble_matrix_kernel<CONTACT><<<dim3(nt, nt), AN_TILE * 8, 0, (cudaStream_t)stream>>>(
        coords, n_snaps, n_ca, cutoff * cutoff, out);
    ALMA_LAUNCH_CHECK(who);
    return ALMA_OK;
}

}  // namespace alma

using namespace alma;

extern "C" int alma_mean_dist_matrix(const double *coords, int32_t n_snaps, int32_t n_ca, double *out, void *stream) {
    return ensemble_matrix<false>(coords, n_snaps, n_ca, 0.0, out, stream, "alma_mean_dist_matrix");
}

extern "C" int alma_contact_freq_matrix(const double *coords, int32_t n_snaps, int32_t n_ca, double cutoff,
                                        double *out, void *stream) {
    return ensemble_matrix<true>(coords, n_snaps, n_ca, cutoff, out, stream, "alma_contact_freq_matrix");
}
