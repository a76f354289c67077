// Move ΔE entry points: one given proposal per system, one CTA per system.
#include <cuda.h>

#include <mutex>

#include "move.cuh"

namespace alma {

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

static size_t carve_scratch(MoveScratch *w, char *base, int32_t natoms) {
    size_t off = 0;
    auto take = [&](size_t bytes) {
        char *p = base ? base + off : nullptr;
        off += align256(bytes);
        return p;
    };
    MoveScratch t;
    t.group = (int8_t *)take((size_t)natoms);
    t.body = (int8_t *)take((size_t)natoms);
    t.mark = (int *)take(sizeof(int) * (size_t)natoms);
    t.xyz_new = (double *)take(sizeof(double) * 4 * (size_t)natoms);
    t.born_new = (double *)take(sizeof(double) * (size_t)natoms);
    t.dE_atom = (double *)take(sizeof(double) * 2 * (size_t)natoms);
    t.affected = (int32_t *)take(sizeof(int32_t) * (size_t)natoms);
    t.edge = (int32_t *)take(sizeof(int32_t) * (size_t)natoms);
    t.hct_part = (double *)take(sizeof(double) * MAX_WPR * (size_t)natoms);
    t.cross_part = (double *)take(sizeof(double) * MAX_WPR * (size_t)natoms);
    t.ctr = (unsigned long long *)take(sizeof(unsigned long long) * 4 * (size_t)(natoms + 1));
    t.phase = (unsigned long long *)take(sizeof(unsigned long long) * 4 * (size_t)(natoms + 1));
    t.queue = (int *)take(sizeof(int) * QUEUE_PER_SYS * (size_t)(natoms + 1));
    t.drift = (int *)take(sizeof(int) * 2 * (size_t)(natoms + 1));
    if (w) *w = t;
    return off;
}

template <typename R>
__global__ void __launch_bounds__(MOVE_THREADS) move_dE_kernel(MoveCtx C, const int32_t *__restrict__ kind,
                                                               const int32_t *__restrict__ a,
                                                               const double *__restrict__ delta, int apply,
                                                               double *__restrict__ dE, double *__restrict__ dterms) {
    __shared__ MoveDesc M;
    __shared__ double sm[128];
    __shared__ double part[8];
    __shared__ CrossCand cq[(MOVE_THREADS / 32) * CROSS_BUF];
    const Team<1> T;
    const int s = blockIdx.x;
    const int k = kind[s];
    if (threadIdx.x == 0) {
        for (int q = 0; q < QUEUE_PER_SYS; ++q) C.w.queue[QUEUE_PER_SYS * s + q] = 0;  // fresh queues: parity 0
        C.w.drift[2 * s] = C.w.drift[2 * s + 1] = 0;
        if (k >= 0) decode_move(M, C.t, C.b.xyz, s, k, a[s], delta + 2 * (size_t)s);
        else M.degenerate = 1;
    }
    __syncthreads();
    if (M.degenerate) {
        if (threadIdx.x == 0) {
            const double nan = __longlong_as_double(0x7ff8000000000000ll);
            dE[s] = nan;
            for (int q = 0; q < 4; ++q) dterms[4 * (size_t)s + q] = nan;
        }
        return;
    }
    const bool rows_ok = system_within_skin(C, s);
    const MoveResult r = move_eval<R, 1>(C, M, s, sm, part, cq, 0, rows_ok, T);
    if (threadIdx.x == 0) {
        dE[s] = r.dE;
        dterms[4 * (size_t)s + 0] = r.dcross;
        dterms[4 * (size_t)s + 1] = r.dsasa;
        dterms[4 * (size_t)s + 2] = r.ddih;
        dterms[4 * (size_t)s + 3] = r.dss;
    }
    move_finish<R, 1>(C, M, s, apply, 0, T);
}

}  // namespace alma

using namespace alma;

extern "C" size_t alma_move_scratch_bytes(int32_t natoms) { return carve_scratch(nullptr, nullptr, natoms); }

// Cumulative work counters of the move kernels, per system: {pair-term
// evaluations, hct evaluations, SASA neighbour visits, moved atoms}, then
// (out[4*nsys ..]) the SM cycles rank 0 spent in the four ΔE phases.
extern "C" int alma_move_counters(const void *scratch, int32_t natoms, int32_t nsys, unsigned long long *out,
                                  void *stream) {
    if (!scratch || !out || nsys <= 0 || nsys > natoms + 1)
        return alma_set_error(ALMA_EINVAL, "alma_move_counters: bad arguments");
    MoveScratch w;
    carve_scratch(&w, (char *)scratch, natoms);
    ALMA_CUDA_TRY(cudaMemcpyAsync(out, w.ctr, sizeof(unsigned long long) * 4 * (size_t)nsys, cudaMemcpyDeviceToHost,
                                  (cudaStream_t)stream));
    ALMA_CUDA_TRY(cudaMemcpyAsync(out + 4 * (size_t)nsys, w.phase, sizeof(unsigned long long) * 4 * (size_t)nsys,
                                  cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    ALMA_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
    return ALMA_OK;
}

extern "C" int alma_move_scratch_init(void *scratch, int32_t natoms, void *stream) {
    if (!scratch || natoms < 0) return alma_set_error(ALMA_EINVAL, "alma_move_scratch_init: bad arguments");
    ALMA_CUDA_TRY(cudaMemsetAsync(scratch, 0, carve_scratch(nullptr, nullptr, natoms), (cudaStream_t)stream));
    return ALMA_OK;
}

int alma_check_move_args(const AlmaBatch *b, const AlmaTopo *t, const AlmaNL *nl, const AlmaParams *p,
                         void *scratch, const char *who) {
    if (!b || !t || !nl || !p || !scratch || b->nsys <= 0 || !b->atom_off || !b->xyz || !b->prm || !b->prm64 ||
        !b->born)
        return alma_set_error(ALMA_EINVAL, "%s: null argument", who);
    if (b->nsys > b->natoms + 1) return alma_set_error(ALMA_EINVAL, "%s: more systems than atoms", who);
    if (!nl->full_ptr || !nl->full_len || !nl->full_cols || !nl->half_ptr || !nl->half_len || !nl->half_cols)
        return alma_set_error(ALMA_EINVAL, "%s: neighbor list not set", who);
    if (!t->rb_off || !t->side_ptr || !t->dih_off || !t->ss_off || !t->cp_off || !t->csp_off)
        return alma_set_error(ALMA_EINVAL, "%s: topology offsets not set", who);
    return ALMA_OK;
}

MoveCtx alma_make_move_ctx(const AlmaBatch *b, const AlmaTopo *t, const AlmaNL *nl, const AlmaParams *p,
                           void *scratch) {
    MoveCtx C;
    C.P = make_dev_params(*p);
    C.b = *b;
    C.t = *t;
    C.nl = *nl;
    carve_scratch(&C.w, (char *)scratch, b->natoms);
    return C;
}

extern "C" int alma_move_dE(const AlmaBatch *b, const AlmaTopo *t, const AlmaNL *nl, const AlmaParams *p, int prec,
                            void *scratch, const int32_t *move_kind, const int32_t *move_a, const double *move_delta,
                            int apply, double *dE, double *dterms, void *stream) {
    int rc = alma_check_move_args(b, t, nl, p, scratch, "alma_move_dE");
    if (rc) return rc;
    if (!move_kind || !move_a || !move_delta || !dE || !dterms)
        return alma_set_error(ALMA_EINVAL, "alma_move_dE: null move buffer");
    const MoveCtx C = alma_make_move_ctx(b, t, nl, p, scratch);
    cudaStream_t st = (cudaStream_t)stream;
    if (prec == ALMA_PREC_FP64)
        move_dE_kernel<double><<<b->nsys, MOVE_THREADS, 0, st>>>(C, move_kind, move_a, move_delta, apply, dE, dterms);
    else
        move_dE_kernel<float><<<b->nsys, MOVE_THREADS, 0, st>>>(C, move_kind, move_a, move_delta, apply, dE, dterms);
    ALMA_LAUNCH_CHECK("alma_move_dE");
    return ALMA_OK;
}

// ---------------------------------------------------------------------------
// alma_move_dE_noalloc: the same ΔE evaluation for callers that cannot
// allocate device memory.  Its scratch is this file-scope array, which every
// GPU that loads the library holds until the process exits.
// ---------------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_move_scratch[ALMA_NOALLOC_SCRATCH_BYTES];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
void *g_scratch_ptr[kMaxDevices] = {};
unsigned long long g_scratch_ctx[kMaxDevices] = {};  // context the address was looked up under

typedef CUresult (*CtxGetCurrentFn)(CUcontext *);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long *);

// Unique ID of the calling thread's current context (0 when it cannot be
// read).  A device reset or a re-created primary context gets a new ID,
// and with it a new module load: the cached address is then stale.
unsigned long long current_ctx_id() {
    static CtxGetCurrentFn get_cur = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q;
        void *f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_cur = (CtxGetCurrentFn)f;
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = (CtxGetIdFn)f;
    });
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (!get_cur || !get_id || get_cur(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}
}  // namespace

// Device address of g_move_scratch on the current device.  In host code the
// array's name is only a host-side handle, so the address is looked up with
// the device current, on the first call on that device and again whenever
// the current context is not the one it was looked up under (after a
// device reset the module, and the array with it, is loaded anew).
static int noalloc_scratch(void **out) {
    int dev = 0;
    ALMA_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return alma_set_error(ALMA_EINVAL, "alma_move_dE_noalloc: device %d", dev);
    const unsigned long long ctx = current_ctx_id();  // 0 before the runtime has made a context current
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_ptr[dev] || ctx == 0 || ctx != g_scratch_ctx[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_move_scratch);
        if (e != cudaSuccess) return alma_cuda_error(e, "alma_move_dE_noalloc: cudaGetSymbolAddress");
        g_scratch_ptr[dev] = p;
        g_scratch_ctx[dev] = current_ctx_id();  // the lookup made the device's context current
    }
    *out = g_scratch_ptr[dev];
    return ALMA_OK;
}

extern "C" size_t alma_move_noalloc_capacity_bytes(void) { return (size_t)ALMA_NOALLOC_SCRATCH_BYTES; }

extern "C" int alma_move_dE_noalloc(const AlmaBatch *b, const AlmaTopo *t, const AlmaNL *nl, const AlmaParams *p,
                                    int prec, const int32_t *move_kind, const int32_t *move_a,
                                    const double *move_delta, int apply, double *dE, double *dterms, void *stream) {
    if (!b || b->natoms < 0) return alma_set_error(ALMA_EINVAL, "alma_move_dE_noalloc: null batch");
    const size_t need = carve_scratch(nullptr, nullptr, b->natoms);
    if (b->natoms > ALMA_NOALLOC_MAX_ATOMS || need > (size_t)ALMA_NOALLOC_SCRATCH_BYTES)
        return alma_set_error(ALMA_EINVAL,
                              "alma_move_dE_noalloc: batch of %d atoms exceeds the built-in scratch area "
                              "(%d atoms, %zu bytes); use alma_move_dE with caller scratch",
                              b->natoms, ALMA_NOALLOC_MAX_ATOMS, (size_t)ALMA_NOALLOC_SCRATCH_BYTES);
    void *scratch = nullptr;
    int rc = noalloc_scratch(&scratch);  // looks the address up; touches nothing on the device
    if (rc) return rc;
    // Validate everything before the clear: a rejected call leaves the shared
    // area untouched (another call's kernel may still be using it).
    rc = alma_check_move_args(b, t, nl, p, scratch, "alma_move_dE_noalloc");
    if (rc) return rc;
    if (!move_kind || !move_a || !move_delta || !dE || !dterms)
        return alma_set_error(ALMA_EINVAL, "alma_move_dE_noalloc: null move buffer");
    // The area keeps whatever the previous call left: start from zero.
    ALMA_CUDA_TRY(cudaMemsetAsync(scratch, 0, need, (cudaStream_t)stream));
    return alma_move_dE(b, t, nl, p, prec, scratch, move_kind, move_a, move_delta, apply, dE, dterms, stream);
}
