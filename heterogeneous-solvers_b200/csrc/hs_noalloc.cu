// hs_noalloc.cu — symmetric block matvec that performs no device allocation.
//
// hs_symv_block grows a per-context scratch buffer with cudaMalloc the first
// time a rectangle needs more partial-sum space than it holds.  Some callers
// cannot let a library allocate: applications whose device memory is owned by
// their own allocator (a caching allocator that has already reserved the free
// memory, so a raw cudaMalloc can fail), and latency-critical loops in which the
// device-wide synchronisation that cudaMalloc/cudaFree imply is not acceptable.
// hs_symv_block_noalloc serves them: it runs the same two kernels as
// hs_symv_block, but its partial sums live in the fixed array below, which is
// part of the library image and is never allocated or freed at run time.
//
// Rules of use (also stated in include/hs_b200.h):
//  * The array holds HS_SYMV_NOALLOC_MAX_DOUBLES doubles (16 MiB) on every GPU
//    that loads the library, until the process exits.  A call whose partials
//    (blockCount_i * blockCount_j * matrixBlockSize doubles) do not fit is
//    rejected with HS_ERR_INVALID_ARG before anything is launched.
//  * All calls on a device share the one array.  Calls whose kernels may run at
//    the same time on that device (different streams, or different host
//    threads) race on it; order such calls on one stream.
//  * Nothing in the array needs to start at zero: every partial slot the
//    second kernel reads is written by the first kernel of the same call, so
//    the contents a previous call left behind are never used.
//  * The array's device address is looked up once per device (and again after
//    the device's primary context was reset, e.g. by cudaDeviceReset), by the
//    first call made there, with that device current; make that first call
//    before any stream capture begins.  Devices 0..63 are supported.
//  * In reference-order mode (hs_ctx_set_reference_order) the call runs the
//    reference-order kernel of hs_symv_block, which needs no scratch at all: the
//    two entry points give the same bits in either mode.
#include <cudaTypedefs.h>

#include <mutex>

#include "hs_internal.cuh"

namespace {

// the partial-sum scratch of hs_symv_block_noalloc (HS_SYMV_NOALLOC_MAX_DOUBLES doubles)
static __device__ __align__(256) double g_symv_noalloc_scratch[HS_SYMV_NOALLOC_MAX_DOUBLES];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
struct ScratchAddr {
    CUcontext owner = nullptr;  // the context the address belongs to
    double* ptr = nullptr;
};
ScratchAddr g_scratch_addr[kMaxDevices];
PFN_cuCtxGetCurrent_v4000 g_ctx_current = nullptr;

// set-up, once per device context, with `device` current: the host-side symbol is
// only a stand-in, the kernels need the array's device address
hs_status scratch_address(int device, double** out) {
    if (device < 0 || device >= kMaxDevices) {
        hs::set_error("hs_symv_block_noalloc: device index out of range (devices 0..63 are supported)");
        return HS_ERR_INVALID_ARG;
    }
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_ctx_current) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        const cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q);
        if (e != cudaSuccess) return hs::cuda_fail(e, "cudaGetDriverEntryPoint(cuCtxGetCurrent)");
        if (q != cudaDriverEntryPointSuccess || !fn) {
            hs::set_error("hs_symv_block_noalloc: cuCtxGetCurrent is not available from the driver");
            return HS_ERR_UNSUPPORTED;
        }
        g_ctx_current = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(fn);
    }
    CUcontext cur = nullptr;
    if (g_ctx_current(&cur) != CUDA_SUCCESS || !cur) {
        hs::set_error("hs_symv_block_noalloc: no current CUDA context");
        return HS_ERR_CUDA;
    }
    ScratchAddr& a = g_scratch_addr[device];
    if (!a.ptr || a.owner != cur) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_symv_noalloc_scratch);
        if (e != cudaSuccess) return hs::cuda_fail(e, "cudaGetSymbolAddress(g_symv_noalloc_scratch)");
        a.ptr = static_cast<double*>(p);
        a.owner = cur;
    }
    *out = a.ptr;
    return HS_OK;
}

}  // namespace

extern "C" hs_status hs_symv_block_noalloc(hs_ctx ctx, const double* A, const double* b, double* result,
                                           int blockStart_i, int blockStart_j, int blockCount_i, int blockCount_j,
                                           int blockCountXY, int reset) {
    hs_status st = hs::require_ctx(ctx, "hs_symv_block_noalloc");
    if (st != HS_OK) return st;
    if (!A || !b || !result) {
        hs::set_error("hs_symv_block_noalloc: null pointer");
        return HS_ERR_INVALID_ARG;
    }
    if (blockCountXY != ctx->nb) {
        hs::set_error("hs_symv_block_noalloc: blockCountXY does not match the context's N / matrixBlockSize");
        return HS_ERR_INVALID_ARG;
    }
    if (blockStart_i < 0 || blockCount_i < 0 || blockStart_i + blockCount_i > ctx->nb || blockStart_j < 0 ||
        blockCount_j < 0 || blockStart_j + blockCount_j > ctx->nb) {
        hs::set_error("hs_symv_block_noalloc: blocks out of range");
        return HS_ERR_INVALID_ARG;
    }
    if (ctx->ref_chunks > 0)  // the reference-order kernel of hs_symv_block uses no scratch
        return hs::launch_symv_refseq(ctx, A, b, result, blockStart_i, blockStart_j, blockCount_i, blockCount_j,
                                      reset, ctx->stream);
    const long long need = (long long)blockCount_i * blockCount_j * ctx->bsz;
    if (need > (long long)HS_SYMV_NOALLOC_MAX_DOUBLES) {
        hs::set_error("hs_symv_block_noalloc: this rectangle needs " + std::to_string(need) +
                      " doubles of partial sums; the static scratch holds " +
                      std::to_string((long long)HS_SYMV_NOALLOC_MAX_DOUBLES) +
                      " (use hs_symv_block, which allocates, for larger rectangles)");
        return HS_ERR_INVALID_ARG;
    }
    double* P = nullptr;
    st = scratch_address(ctx->device, &P);
    if (st != HS_OK) return st;
    return hs::launch_symv_partials_at(ctx, A, b, result, blockStart_i, blockStart_j, blockCount_i, blockCount_j,
                                       reset, P, ctx->stream);
}
