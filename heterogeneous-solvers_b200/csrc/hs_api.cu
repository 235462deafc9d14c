// hs_api.cu — the C ABI: context management, error reporting, argument
// validation and the operator-level entry points of include/hs_b200.h.
#include <cstdio>
#include <cstring>
#include <string>

#include "hs_internal.cuh"

namespace hs {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

hs_status cuda_fail(cudaError_t e, const char* what) {
    cudaGetLastError();  // clear a non-sticky error so that later calls do not inherit it
    set_error(std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
    return e == cudaErrorMemoryAllocation ? HS_ERR_OOM : HS_ERR_CUDA;
}

hs_status require_ctx(hs_ctx ctx, const char* fn) {
    if (!ctx) {
        set_error(std::string(fn) + ": null context");
        return HS_ERR_INVALID_ARG;
    }
    if (ctx->bsz <= 0 && std::strcmp(fn, "hs_ctx_set_problem") != 0) {
        set_error(std::string(fn) + ": call hs_ctx_set_problem first");
        return HS_ERR_INVALID_ARG;
    }
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    return HS_OK;
}

hs_status ensure_scratch(hs_ctx ctx, size_t bytes) {
    if (ctx->scratch_bytes >= bytes) return HS_OK;
    size_t want = bytes + bytes / 8;
    if (want < 1024 * 1024) want = 1024 * 1024;
    HS_CUDA(cudaStreamSynchronize(ctx->stream));
    if (ctx->side) HS_CUDA(cudaStreamSynchronize(ctx->side));
    if (ctx->side_hi) HS_CUDA(cudaStreamSynchronize(ctx->side_hi));
    if (ctx->scratch) HS_CUDA(cudaFree(ctx->scratch));
    ctx->scratch = nullptr;
    ctx->scratch_bytes = 0;
    HS_CUDA(cudaMalloc(&ctx->scratch, want));
    ctx->scratch_bytes = want;
    return HS_OK;
}

hs_status ensure_work(hs_ctx ctx, size_t bytes) {
    if (ctx->work_bytes >= bytes) return HS_OK;
    HS_CUDA(cudaStreamSynchronize(ctx->stream));
    if (ctx->work) HS_CUDA(cudaFree(ctx->work));
    ctx->work = nullptr;
    ctx->work_bytes = 0;
    HS_CUDA(cudaMalloc(&ctx->work, bytes));
    ctx->work_bytes = bytes;
    return HS_OK;
}

hs_status ensure_mixed(hs_ctx ctx, size_t bytes) {
    if (ctx->mixed_bytes >= bytes) return HS_OK;
    HS_CUDA(cudaStreamSynchronize(ctx->stream));
    if (ctx->mixed) HS_CUDA(cudaFree(ctx->mixed));
    ctx->mixed = nullptr;
    ctx->mixed_bytes = 0;
    HS_CUDA(cudaMalloc(&ctx->mixed, bytes));
    ctx->mixed_bytes = bytes;
    return HS_OK;
}

hs_status ensure_gp(hs_ctx ctx, size_t bytes) {
    if (ctx->gpws_bytes >= bytes) return HS_OK;
    HS_CUDA(cudaStreamSynchronize(ctx->stream));
    if (ctx->gpws) HS_CUDA(cudaFree(ctx->gpws));
    ctx->gpws = nullptr;
    ctx->gpws_bytes = 0;
    HS_CUDA(cudaMalloc(&ctx->gpws, bytes));
    ctx->gpws_bytes = bytes;
    return HS_OK;
}

hs_status ensure_hostws(hs_ctx ctx, size_t bytes) {
    if (ctx->hostws_bytes >= bytes) return HS_OK;
    HS_CUDA(cudaStreamSynchronize(ctx->stream));
    if (ctx->hostws) HS_CUDA(cudaFree(ctx->hostws));
    ctx->hostws = nullptr;
    ctx->hostws_bytes = 0;
    HS_CUDA(cudaMalloc(&ctx->hostws, bytes));
    ctx->hostws_bytes = bytes;
    return HS_OK;
}

hs_status ensure_solvews(hs_ctx ctx, size_t bytes) {
    if (ctx->solvews_bytes >= bytes) return HS_OK;
    HS_CUDA(cudaStreamSynchronize(ctx->stream));
    if (ctx->solvews) HS_CUDA(cudaFree(ctx->solvews));
    ctx->solvews = nullptr;
    ctx->solvews_bytes = 0;
    HS_CUDA(cudaMalloc(&ctx->solvews, bytes));
    ctx->solvews_bytes = bytes;
    return HS_OK;
}

__global__ void set_i64_kernel(long long* p, long long v) { *p = v; }

void set_i64_dev(long long* p, long long v, cudaStream_t s) { set_i64_kernel<<<1, 1, 0, s>>>(p, v); }

static cudaEvent_t pool_get(hs_ctx ctx) {
    if (!ctx->prof_pool.empty()) {
        cudaEvent_t e = ctx->prof_pool.back();
        ctx->prof_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

void prof_begin(hs_ctx ctx, cudaStream_t s, int kernel) {
    if (!ctx->profiling) return;
    hs_ctx_s::ProfRec r{kernel, pool_get(ctx), pool_get(ctx), 0.0, 0.0};
    cudaEventRecord(r.start, s);
    ctx->prof_pending.push_back(r);
}

void prof_end(hs_ctx ctx, cudaStream_t s, int kernel, double flops, double bytes) {
    if (!ctx->profiling) return;
    for (auto it = ctx->prof_pending.rbegin(); it != ctx->prof_pending.rend(); ++it) {
        if (it->kernel == kernel && it->flops == 0.0 && it->bytes == 0.0) {
            cudaEventRecord(it->stop, s);
            it->flops = flops > 0 ? flops : -1.0;  // marks the pair closed
            it->bytes = bytes;
            return;
        }
    }
}

static hs_status prof_collect(hs_ctx ctx) {
    if (ctx->prof_pending.empty()) return HS_OK;
    HS_CUDA(cudaDeviceSynchronize());
    for (auto& r : ctx->prof_pending) {
        float ms = 0.f;
        if (r.flops != 0.0 && cudaEventElapsedTime(&ms, r.start, r.stop) == cudaSuccess) {
            auto& t = ctx->prof_total[r.kernel];
            t.launches += 1;
            t.ms += ms;
            t.flops += r.flops > 0 ? r.flops : 0.0;
            t.bytes += r.bytes;
        }
        ctx->prof_pool.push_back(r.start);
        ctx->prof_pool.push_back(r.stop);
    }
    ctx->prof_pending.clear();
    return HS_OK;
}

}  // namespace hs

using namespace hs;

#define HS_API_BEGIN(fn)                         \
    {                                            \
        hs_status st_ = require_ctx(ctx, fn);    \
        if (st_ != HS_OK) return st_;            \
    }

#define HS_ARG(cond, msg)                                   \
    do {                                                    \
        if (!(cond)) {                                      \
            set_error(std::string(__func__) + ": " + (msg)); \
            return HS_ERR_INVALID_ARG;                      \
        }                                                   \
    } while (0)

extern "C" {

int hs_abi_version(void) { return HS_B200_ABI_VERSION; }

const char* hs_last_error(void) { return g_last_error.c_str(); }

const char* hs_status_string(hs_status s) {
    switch (s) {
        case HS_OK: return "HS_OK";
        case HS_ERR_INVALID_ARG: return "HS_ERR_INVALID_ARG";
        case HS_ERR_OOM: return "HS_ERR_OOM";
        case HS_ERR_NOT_SPD: return "HS_ERR_NOT_SPD";
        case HS_ERR_NO_CONVERGENCE: return "HS_ERR_NO_CONVERGENCE";
        case HS_ERR_REFINEMENT_STALLED: return "HS_ERR_REFINEMENT_STALLED";
        case HS_ERR_CUDA: return "HS_ERR_CUDA";
        case HS_ERR_TIMEOUT: return "HS_ERR_TIMEOUT";
        case HS_ERR_UNSUPPORTED: return "HS_ERR_UNSUPPORTED";
    }
    return "HS_ERR_UNKNOWN";
}

int64_t hs_packed_matrix_size(int64_t N, int bsz) {
    if (N <= 0 || bsz <= 0) return 0;
    const int64_t nb = (N + bsz - 1) / bsz;
    return nb * (nb + 1) / 2 * (int64_t)bsz * bsz;
}

int64_t hs_padded_vector_size(int64_t N, int bsz) {
    if (N <= 0 || bsz <= 0) return 0;
    return (N + bsz - 1) / bsz * (int64_t)bsz;
}

hs_status hs_ctx_create(int device, void* stream, hs_ctx* out) {
    if (!out) {
        set_error("hs_ctx_create: null output");
        return HS_ERR_INVALID_ARG;
    }
    *out = nullptr;
    int count = 0;
    HS_CUDA(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count) {
        set_error("hs_ctx_create: no CUDA device " + std::to_string(device));
        return HS_ERR_INVALID_ARG;
    }
    HS_CUDA(cudaSetDevice(device));
    hs_ctx ctx = new hs_ctx_s();
    ctx->device = device;
    cudaDeviceProp prop;
    HS_CUDA(cudaGetDeviceProperties(&prop, device));
    ctx->num_sms = prop.multiProcessorCount;
    ctx->stream = static_cast<cudaStream_t>(stream);  // NULL: the CUDA default stream
    HS_CUDA(cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking));
    {
        int least = 0, greatest = 0;
        HS_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        HS_CUDA(cudaStreamCreateWithPriority(&ctx->side_hi, cudaStreamNonBlocking, greatest));
    }
    HS_CUDA(cudaEventCreateWithFlags(&ctx->ev_a, cudaEventDisableTiming));
    HS_CUDA(cudaEventCreateWithFlags(&ctx->ev_b, cudaEventDisableTiming));
    HS_CUDA(cudaMalloc(&ctx->d_info, 2 * sizeof(long long)));
    HS_CUDA(cudaMallocHost(&ctx->h_pinned, 64 * sizeof(double)));
    set_i64_kernel<<<1, 1, 0, ctx->stream>>>(ctx->d_info, INT64_MAX);
    HS_CUDA(cudaGetLastError());
    HS_CUDA(cudaStreamSynchronize(ctx->stream));
    *out = ctx;
    return HS_OK;
}

hs_status hs_ctx_destroy(hs_ctx ctx) {
    if (!ctx) return HS_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->side) {
        cudaStreamSynchronize(ctx->side);
        cudaStreamDestroy(ctx->side);
    }
    if (ctx->side_hi) {
        cudaStreamSynchronize(ctx->side_hi);
        cudaStreamDestroy(ctx->side_hi);
    }
    if (ctx->ev_a) cudaEventDestroy(ctx->ev_a);
    if (ctx->ev_b) cudaEventDestroy(ctx->ev_b);
    for (auto& r : ctx->prof_pending) {
        cudaEventDestroy(r.start);
        cudaEventDestroy(r.stop);
    }
    for (auto e : ctx->prof_pool) cudaEventDestroy(e);
    if (ctx->scratch) cudaFree(ctx->scratch);
    if (ctx->work) cudaFree(ctx->work);
    if (ctx->mixed) cudaFree(ctx->mixed);
    if (ctx->gpws) cudaFree(ctx->gpws);
    if (ctx->hostws) cudaFree(ctx->hostws);
    if (ctx->solvews) cudaFree(ctx->solvews);
    if (ctx->d_info) cudaFree(ctx->d_info);
    if (ctx->h_pinned) cudaFreeHost(ctx->h_pinned);
    delete ctx;
    return HS_OK;
}

hs_status hs_ctx_release_buffers(hs_ctx ctx) {
    if (!ctx) {
        set_error("hs_ctx_release_buffers: null context");
        return HS_ERR_INVALID_ARG;
    }
    HS_CUDA(cudaSetDevice(ctx->device));
    HS_CUDA(cudaStreamSynchronize(ctx->stream));
    if (ctx->side) HS_CUDA(cudaStreamSynchronize(ctx->side));
    if (ctx->side_hi) HS_CUDA(cudaStreamSynchronize(ctx->side_hi));
    if (ctx->scratch) HS_CUDA(cudaFree(ctx->scratch));
    if (ctx->work) HS_CUDA(cudaFree(ctx->work));
    if (ctx->mixed) HS_CUDA(cudaFree(ctx->mixed));
    if (ctx->gpws) HS_CUDA(cudaFree(ctx->gpws));
    if (ctx->hostws) HS_CUDA(cudaFree(ctx->hostws));
    if (ctx->solvews) HS_CUDA(cudaFree(ctx->solvews));
    ctx->scratch = ctx->work = ctx->mixed = ctx->gpws = ctx->hostws = ctx->solvews = nullptr;
    ctx->scratch_bytes = ctx->work_bytes = ctx->mixed_bytes = ctx->gpws_bytes = ctx->hostws_bytes = 0;
    ctx->solvews_bytes = 0;
    return HS_OK;
}

hs_status hs_ctx_set_stream(hs_ctx ctx, void* stream) {
    if (!ctx) {
        set_error("hs_ctx_set_stream: null context");
        return HS_ERR_INVALID_ARG;
    }
    HS_CUDA(cudaSetDevice(ctx->device));
    HS_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->stream = static_cast<cudaStream_t>(stream);  // NULL: the CUDA default stream
    return HS_OK;
}

hs_status hs_ctx_set_problem(hs_ctx ctx, int64_t N, int bsz) {
    HS_API_BEGIN("hs_ctx_set_problem");
    HS_ARG(N > 0, "N must be positive");
    HS_ARG(bsz > 0 && bsz <= 1024, "matrixBlockSize must be in [1, 1024]");
    const int64_t nb = (N + bsz - 1) / bsz;
    HS_ARG(nb < (1 << 20), "too many block rows");
    ctx->N = N;
    ctx->bsz = bsz;
    ctx->nb = (int)nb;
    return HS_OK;
}

hs_status hs_sync(hs_ctx ctx) {
    if (!ctx) {
        set_error("hs_sync: null context");
        return HS_ERR_INVALID_ARG;
    }
    HS_CUDA(cudaSetDevice(ctx->device));
    HS_CUDA(cudaStreamSynchronize(ctx->stream));
    return HS_OK;
}

hs_status hs_ctx_set_profiling(hs_ctx ctx, int enable) {
    if (!ctx) {
        set_error("hs_ctx_set_profiling: null context");
        return HS_ERR_INVALID_ARG;
    }
    ctx->profiling = enable != 0;
    return HS_OK;
}

hs_status hs_ctx_read_profile(hs_ctx ctx, int kernel, hs_kernel_profile* out) {
    if (!ctx || !out || kernel < 0 || kernel >= HS_KERNEL_COUNT) {
        set_error("hs_ctx_read_profile: bad arguments");
        return HS_ERR_INVALID_ARG;
    }
    HS_CUDA(cudaSetDevice(ctx->device));
    hs_status st = prof_collect(ctx);
    if (st != HS_OK) return st;
    *out = ctx->prof_total[kernel];
    return HS_OK;
}

hs_status hs_ctx_reset_profile(hs_ctx ctx) {
    if (!ctx) {
        set_error("hs_ctx_reset_profile: null context");
        return HS_ERR_INVALID_ARG;
    }
    HS_CUDA(cudaSetDevice(ctx->device));
    hs_status st = prof_collect(ctx);
    if (st != HS_OK) return st;
    for (auto& t : ctx->prof_total) t = hs_kernel_profile{};
    return HS_OK;
}

int64_t hs_ctx_launch_count(hs_ctx ctx) { return ctx ? ctx->launches : -1; }

hs_status hs_ctx_set_reference_order(hs_ctx ctx, int cpu_chunks) {
    if (!ctx || cpu_chunks < 0 || cpu_chunks > 4096) {
        set_error("hs_ctx_set_reference_order: chunks must be in [0, 4096]");
        return HS_ERR_INVALID_ARG;
    }
    ctx->ref_chunks = cpu_chunks;
    return HS_OK;
}

hs_status hs_ctx_set_mixed_accumulation(hs_ctx ctx, int panels) {
    if (!ctx || (panels != 1 && panels != 2 && panels != 4)) {
        set_error("hs_ctx_set_mixed_accumulation: panels must be 1, 2 or 4");
        return HS_ERR_INVALID_ARG;
    }
    ctx->mixed_acc_panels = panels;
    return HS_OK;
}

hs_status hs_ctx_set_mixed_lookahead(hs_ctx ctx, int side_sms, int min_rows) {
    if (!ctx || side_sms < 0 || side_sms > ctx->num_sms / 2 || min_rows < 0) {
        set_error("hs_ctx_set_mixed_lookahead: side_sms must be in [0, SMs / 2] and min_rows >= 0");
        return HS_ERR_INVALID_ARG;
    }
    ctx->mixed_side_sms = side_sms;
    ctx->mixed_min_rows = min_rows;
    return HS_OK;
}

hs_status hs_ctx_take_info(hs_ctx ctx, int64_t* info) {
    HS_API_BEGIN("hs_ctx_take_info");
    long long v = 0;
    HS_CUDA(cudaMemcpyAsync(&v, ctx->d_info, sizeof(long long), cudaMemcpyDeviceToHost, ctx->stream));
    HS_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->launches += 1;
    set_i64_kernel<<<1, 1, 0, ctx->stream>>>(ctx->d_info, INT64_MAX);
    HS_CHECK_LAUNCH("reset info");
    if (info) *info = (v == INT64_MAX) ? -1 : (int64_t)v;
    return HS_OK;
}

hs_status hs_selftest_bounded_wait(hs_ctx ctx, int64_t timeout_ns) {
    HS_API_BEGIN("hs_selftest_bounded_wait");
    HS_ARG(timeout_ns >= 1000000 && timeout_ns <= 2000000000LL, "timeout_ns must be in [1e6, 2e9]");
    return launch_bounded_wait_selftest(ctx, timeout_ns);
}

// ---------------------------------------------------------------- operators
hs_status hs_potrf_block(hs_ctx ctx, double* A, int blockID, int blockRow) {
    HS_API_BEGIN("hs_potrf_block");
    const int64_t T = total_blocks(ctx->nb);
    HS_ARG(A != nullptr, "null matrix");
    HS_ARG(blockID >= 0 && blockID < T, "blockID out of range");
    HS_ARG(blockRow >= 0 && blockRow < ctx->nb, "blockRow out of range");
    return launch_potrf(ctx, A, blockID, blockRow, ctx->stream);
}

hs_status hs_trsm_panel(hs_ctx ctx, double* A, int blockID, int blockRow, int blockStart, int blockCount) {
    HS_API_BEGIN("hs_trsm_panel");
    const int64_t T = total_blocks(ctx->nb);
    HS_ARG(A != nullptr, "null matrix");
    HS_ARG(blockID >= 0 && blockID < T, "blockID out of range");
    HS_ARG(blockRow >= 0 && blockRow < ctx->nb, "blockRow out of range");
    HS_ARG(blockCount >= 0, "negative blockCount");
    HS_ARG(blockCount == 0 || (blockStart > blockRow && blockStart + blockCount <= ctx->nb),
           "blocks must lie below the diagonal block and inside the matrix");
    HS_ARG(blockCount == 0 || (int64_t)blockID + (blockStart - blockRow) + blockCount <= T, "blocks outside storage");
    return launch_trsm(ctx, A, blockID, blockRow, blockStart, blockCount, ctx->stream);
}

hs_status hs_syrk_diag(hs_ctx ctx, double* A, int blockID, int blockRow, int blockStart, int blockCount,
                       int blockCountXY) {
    HS_API_BEGIN("hs_syrk_diag");
    HS_ARG(A != nullptr, "null matrix");
    HS_ARG(blockCountXY == ctx->nb, "blockCountXY does not match the context's N / matrixBlockSize");
    HS_ARG(blockID >= 0 && blockID < total_blocks(ctx->nb), "blockID out of range");
    HS_ARG(blockRow >= 0 && blockRow < ctx->nb, "blockRow out of range");
    HS_ARG(blockCount >= 0, "negative blockCount");
    HS_ARG(blockCount == 0 || (blockStart > blockRow && blockStart + blockCount <= ctx->nb),
           "diagonal blocks must lie below blockRow and inside the matrix");
    return launch_update(ctx, A, blockID, blockRow, blockStart, blockCount, 0, 0, ctx->stream);
}

hs_status hs_gemm_trailing(hs_ctx ctx, double* A, int blockID, int blockRow, int blockStart, int blockCount,
                           int blockCountXY) {
    HS_API_BEGIN("hs_gemm_trailing");
    HS_ARG(A != nullptr, "null matrix");
    HS_ARG(blockCountXY == ctx->nb, "blockCountXY does not match the context's N / matrixBlockSize");
    HS_ARG(blockID >= 0 && blockID < total_blocks(ctx->nb), "blockID out of range");
    HS_ARG(blockRow >= 0 && blockRow < ctx->nb, "blockRow out of range");
    HS_ARG(blockCount >= 0, "negative blockCount");
    HS_ARG(blockCount == 0 || (blockStart >= blockRow + 2 && blockStart + blockCount <= ctx->nb),
           "rows must lie in [blockRow+2, blockCountXY)");
    return launch_update(ctx, A, blockID, blockRow, 0, 0, blockStart, blockCount, ctx->stream);
}

hs_status hs_symv_block(hs_ctx ctx, const double* A, const double* b, double* result, int bi0, int bj0, int nbi,
                        int nbj, int blockCountXY, int reset) {
    HS_API_BEGIN("hs_symv_block");
    HS_ARG(A && b && result, "null pointer");
    HS_ARG(blockCountXY == ctx->nb, "blockCountXY does not match the context's N / matrixBlockSize");
    HS_ARG(bi0 >= 0 && nbi >= 0 && bi0 + nbi <= ctx->nb, "row blocks out of range");
    HS_ARG(bj0 >= 0 && nbj >= 0 && bj0 + nbj <= ctx->nb, "column blocks out of range");
    if (ctx->ref_chunks > 0) return launch_symv_refseq(ctx, A, b, result, bi0, bj0, nbi, nbj, reset, ctx->stream);
    return launch_symv(ctx, A, b, result, bi0, bj0, nbi, nbj, reset, nullptr, nullptr, ctx->stream);
}

hs_status hs_trsv_block(hs_ctx ctx, const double* A, double* b, int blockRow, int blockID, int transposed) {
    HS_API_BEGIN("hs_trsv_block");
    HS_ARG(A && b, "null pointer");
    HS_ARG(blockRow >= 0 && blockRow < ctx->nb, "blockRow out of range");
    HS_ARG(blockID >= 0 && blockID < total_blocks(ctx->nb), "blockID out of range");
    return launch_trsv(ctx, A, b, blockRow, blockID, transposed, ctx->stream);
}

hs_status hs_column_update(hs_ctx ctx, const double* A, double* b, int blockStart, int blockCount, int blockRow,
                           int blockID, int blockCountXY, int transposed) {
    HS_API_BEGIN("hs_column_update");
    HS_ARG(A && b, "null pointer");
    HS_ARG(blockCountXY == ctx->nb, "blockCountXY does not match the context's N / matrixBlockSize");
    HS_ARG(blockRow >= 0 && blockRow < ctx->nb, "blockRow out of range");
    HS_ARG(blockCount >= 0 && blockStart >= 0 && blockStart + blockCount <= ctx->nb, "blocks out of range");
    if (!transposed) {
        HS_ARG(blockCount == 0 || blockStart > blockRow, "forward update needs blocks below blockRow");
        HS_ARG(blockCount == 0 || (int64_t)blockID + (blockStart - blockRow) + blockCount <= total_blocks(ctx->nb),
               "blocks outside storage");
    } else {
        HS_ARG(blockCount == 0 || blockStart + blockCount <= blockRow, "transposed update needs blocks left of blockRow");
    }
    return launch_column_update(ctx, A, b, blockStart, blockCount, blockRow, blockID, transposed, ctx->stream);
}

static hs_status vec_common(hs_ctx ctx, int op, const double* x, const double* y, double alpha, double* out,
                            int bi0, int nbi, const char* fn) {
    HS_API_BEGIN(fn);
    if (!x || !out || (op != 0 && !y)) {
        set_error(std::string(fn) + ": null pointer");
        return HS_ERR_INVALID_ARG;
    }
    if (bi0 < 0 || nbi < 0 || bi0 + nbi > ctx->nb) {
        set_error(std::string(fn) + ": blocks out of range");
        return HS_ERR_INVALID_ARG;
    }
    return launch_vec(ctx, op, x, y, alpha, out, (int64_t)bi0 * ctx->bsz, (int64_t)nbi * ctx->bsz, ctx->stream);
}

hs_status hs_scale_block(hs_ctx ctx, const double* x, double alpha, double* result, int bi0, int nbi) {
    return vec_common(ctx, 0, x, nullptr, alpha, result, bi0, nbi, "hs_scale_block");
}
hs_status hs_add_block(hs_ctx ctx, const double* x, const double* y, double* result, int bi0, int nbi) {
    return vec_common(ctx, 1, x, y, 0.0, result, bi0, nbi, "hs_add_block");
}
hs_status hs_sub_block(hs_ctx ctx, const double* x, const double* y, double* result, int bi0, int nbi) {
    return vec_common(ctx, 2, x, y, 0.0, result, bi0, nbi, "hs_sub_block");
}
hs_status hs_axpy_block(hs_ctx ctx, const double* x, double alpha, const double* y, double* result, int bi0,
                        int nbi) {
    return vec_common(ctx, 3, x, y, alpha, result, bi0, nbi, "hs_axpy_block");
}

hs_status hs_dot_block(hs_ctx ctx, const double* x, const double* y, double* result, int bi0, int nbi) {
    HS_API_BEGIN("hs_dot_block");
    HS_ARG(x && y && result, "null pointer");
    HS_ARG(bi0 >= 0 && nbi >= 0 && bi0 + nbi <= ctx->nb, "blocks out of range");
    if (ctx->ref_chunks > 0)
        return launch_dot_refseq(ctx, x, y, result, (int64_t)bi0 * ctx->bsz, (int64_t)nbi * ctx->bsz,
                                 ctx->ref_chunks, ctx->stream);
    return launch_dot(ctx, x, y, result, (int64_t)bi0 * ctx->bsz, (int64_t)nbi * ctx->bsz, ctx->stream);
}

}  // extern "C"
