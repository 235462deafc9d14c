// k_vector.cu — vector operations, deterministic dot product, symmetric block
// matvec, single-block triangular solve and block-column update.
//
// Reference kernels replaced (paths relative to the reference root):
//   VectorOperations.cpp:6-82     scale/add/sub/scaleAndAdd
//   VectorOperations.cpp:84-185   scalarProduct + sumFinalScalarProduct
//   MatrixVectorOperations.cpp:8-280    matrixVectorBlock{,_GPU,_CPU}
//   MatrixVectorOperations.cpp:282-335  triangularSolveBlockVector
//   MatrixVectorOperations.cpp:337-377  matrixVectorColumnUpdate
//
// The symmetric matvec streams every stored block of the touched sub-rectangle
// exactly once and applies it both as A_ij (row part, for output block row i)
// and as A_ij^T (column part, for output block row j).  Each part lands in its
// own slot of a partial buffer indexed by the sub-rectangle position, and a
// second kernel sums the slots of an output block row in a fixed order, so the
// result is bitwise reproducible without atomics.
#include "hs_internal.cuh"
#include "hs_mixed.cuh"

namespace hs {
namespace {

constexpr int kThreads = 256;

// ------------------------------------------------------------------ elementwise
template <int OP>
__global__ void vec_kernel(const double* __restrict__ x, const double* __restrict__ y, double alpha,
                           double* __restrict__ out, int64_t first, int64_t len) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < len; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = first + t;
        double v;
        if (OP == 0) v = x[i] * alpha;          // scaleVectorBlock          VectorOperations.cpp:19
        else if (OP == 1) v = x[i] + y[i];      // addVectorBlock            :39
        else if (OP == 2) v = x[i] - y[i];      // subVectorBlock            :58
        else v = x[i] + y[i] * alpha;           // scaleAndAddVectorBlock    :78
        out[i] = v;
    }
}

// reference-order forms: no contraction, the reference's operand order
template <int OP>
__global__ void vec_kernel_ref(const double* __restrict__ x, const double* __restrict__ y, double alpha,
                               double* __restrict__ out, int64_t first, int64_t len) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < len; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = first + t;
        double v;
        if (OP == 0) v = __dmul_rn(x[i], alpha);
        else if (OP == 1) v = __dadd_rn(x[i], y[i]);
        else if (OP == 2) v = __dsub_rn(x[i], y[i]);
        else v = __dadd_rn(x[i], __dmul_rn(y[i], alpha));
        out[i] = v;
    }
}

// ------------------------------------------------------------------ dot
constexpr int kDotBlocks = 512;

// VectorOperations.cpp:187-238: ceil(len/chunks) elements per chunk summed
// from zero, then the chunk sums in order; one thread per chunk
__global__ void dot_refseq_chunks(const double* __restrict__ x, const double* __restrict__ y, int64_t first,
                                  int64_t len, int chunks, double* __restrict__ part) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= chunks) return;
    const int64_t per = (len + chunks - 1) / chunks;
    const int64_t s = (int64_t)c * per + first;
    const int64_t e = (s + per < first + len) ? s + per : first + len;
    double v = 0.0;
    for (int64_t i = s; i < e; ++i) v = __dadd_rn(v, __dmul_rn(x[i], y[i]));
    part[c] = v;
}

__global__ void dot_refseq_final(const double* __restrict__ part, int chunks, double* __restrict__ out) {
    double v = 0.0;
    for (int c = 0; c < chunks; ++c) v = __dadd_rn(v, part[c]);
    *out = v;
}

__device__ __forceinline__ double block_reduce_sum(double v, double* sh) {
    // fixed-order tree: warp butterfly, then the 8 warp sums in order
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += sh[i];
    return s;  // valid in thread 0
}

__global__ void dot_stage1(const double* __restrict__ x, const double* __restrict__ y, int64_t first, int64_t len,
                           double* __restrict__ partial) {
    __shared__ double sh[32];
    double v = 0.0;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < len; t += (int64_t)gridDim.x * blockDim.x)
        v += x[first + t] * y[first + t];
    const double s = block_reduce_sum(v, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

__global__ void dot_stage2(const double* __restrict__ partial, int n, double* __restrict__ out) {
    __shared__ double sh[32];
    double v = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) v += partial[i];
    const double s = block_reduce_sum(v, sh);
    if (threadIdx.x == 0) out[0] = s;
}

// ------------------------------------------------------------------ block apply
// One CTA applies one bsz x bsz block M (row major) to a vector:
//   rowOut[r] = sum_c M[r][c] * xc[c]      (row part)
//   colOut[c] = sum_r M[r][c] * xr[r]      (column part)
// Fast path for bsz in {128, 256}: 8 warps own bsz/8 consecutive rows each,
// lane l owns bsz/32 consecutive columns loaded with 16-byte streaming loads.
// CPL consecutive elements of one row as doubles, 16-byte streaming loads
template <int CPL>
__device__ __forceinline__ void load_row(const double* p, double (&a)[CPL]) {
#pragma unroll
    for (int j = 0; j < CPL / 2; ++j) {
        const double2 v = __ldcs(reinterpret_cast<const double2*>(p) + j);
        a[2 * j] = v.x;
        a[2 * j + 1] = v.y;
    }
}
template <int CPL>
__device__ __forceinline__ void load_row(const float* p, double (&a)[CPL]) {
#pragma unroll
    for (int j = 0; j < CPL / 4; ++j) {
        const float4 v = __ldcs(reinterpret_cast<const float4*>(p) + j);
        a[4 * j] = v.x;
        a[4 * j + 1] = v.y;
        a[4 * j + 2] = v.z;
        a[4 * j + 3] = v.w;
    }
}

template <int BSZ, typename T = double>
struct BlockApply {
    static constexpr int CPL = BSZ / 32;  // columns per lane
    static constexpr int RPW = BSZ / 8;   // rows per warp

    // sums a per-lane vector s[RPW] across the warp so that lane l ends with
    // the total for row (l % RPW); fixed butterfly order
    __device__ static __forceinline__ double reduce_rows(double (&s)[RPW], int lane) {
        if (RPW == 16) {
#pragma unroll
            for (int i = 0; i < RPW; ++i) s[i] += __shfl_xor_sync(0xffffffffu, s[i], 16);
        }
#pragma unroll
        for (int step = RPW / 2; step >= 1; step >>= 1) {
            const bool upper = (lane & step) != 0;
#pragma unroll
            for (int i = 0; i < step; ++i) {
                const double send = upper ? s[i] : s[i + step];
                const double keep = upper ? s[i + step] : s[i];
                s[i] = keep + __shfl_xor_sync(0xffffffffu, send, step);
            }
        }
        return s[0];
    }

    // mode bit 1: row part, bit 2: column part.  colOut / rowOut get "=" semantics.
    __device__ static void run(const T* __restrict__ M, const double* __restrict__ xc,
                               const double* __restrict__ xr, double* __restrict__ rowOut,
                               double* __restrict__ colOut, int mode, double* smem /* 8*BSZ */) {
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const int r0 = warp * RPW;
        const int c0 = lane * CPL;
        double xcv[CPL], z[CPL], s[RPW];
#pragma unroll
        for (int j = 0; j < CPL; ++j) {
            xcv[j] = (mode & 1) ? xc[c0 + j] : 0.0;
            z[j] = 0.0;
        }
        const double xrl = ((mode & 2) && lane < RPW) ? xr[r0 + lane] : 0.0;
#pragma unroll
        for (int rr = 0; rr < RPW; ++rr) {
            double a[CPL];
            load_row<CPL>(M + (size_t)(r0 + rr) * BSZ + c0, a);
            double acc = 0.0;
#pragma unroll
            for (int j = 0; j < CPL; ++j) acc = fma(a[j], xcv[j], acc);
            s[rr] = acc;
            const double xv = __shfl_sync(0xffffffffu, xrl, rr);
#pragma unroll
            for (int j = 0; j < CPL; ++j) z[j] = fma(a[j], xv, z[j]);
        }
        if (mode & 1) {
            const double rs = reduce_rows(s, lane);
            if (lane < RPW) rowOut[r0 + lane] = rs;
        }
        if (mode & 2) {
#pragma unroll
            for (int j = 0; j < CPL; ++j) smem[warp * BSZ + c0 + j] = z[j];
            __syncthreads();
            for (int c = threadIdx.x; c < BSZ; c += blockDim.x) {
                double v = 0.0;
#pragma unroll
                for (int w = 0; w < 8; ++w) v += smem[w * BSZ + c];
                colOut[c] = v;
            }
        }
    }
};

// generic path for any bsz: thread per row (row part), thread per column (column part)
__device__ void block_apply_generic(const double* __restrict__ M, int bsz, const double* __restrict__ xc,
                                    const double* __restrict__ xr, double* __restrict__ rowOut,
                                    double* __restrict__ colOut, int mode) {
    if (mode & 1)
        for (int r = threadIdx.x; r < bsz; r += blockDim.x) {
            double v = 0.0;
            for (int c = 0; c < bsz; ++c) v += M[(size_t)r * bsz + c] * xc[c];
            rowOut[r] = v;
        }
    if (mode & 2)
        for (int c = threadIdx.x; c < bsz; c += blockDim.x) {
            double v = 0.0;
            for (int r = 0; r < bsz; ++r) v += M[(size_t)r * bsz + c] * xr[r];
            colOut[c] = v;
        }
}

template <int BSZ>
__device__ __forceinline__ void block_apply(const double* M, int bsz, const double* xc, const double* xr,
                                            double* rowOut, double* colOut, int mode, double* smem) {
    if constexpr (BSZ > 0) BlockApply<BSZ>::run(M, xc, xr, rowOut, colOut, mode, smem);
    else block_apply_generic(M, bsz, xc, xr, rowOut, colOut, mode);
}

// ------------------------------------------------------------------ SYMV phase 1
// grid: one CTA per sub-rectangle position (I, J); the CTA owning the stored
// block computes every part of it the rectangle needs.
template <int BSZ>
__global__ void __launch_bounds__(kThreads, 2) symv_partials(const double* __restrict__ A, const double* __restrict__ b,
                                                          double* __restrict__ P, int bsz, int nb, int bi0,
                                                          int bj0, int nbi, int nbj) {
    __shared__ double smem[(BSZ > 0 ? 8 * BSZ : 1)];
    const int64_t pos = blockIdx.x;
    const int I = bi0 + (int)(pos / nbj);
    const int J = bj0 + (int)(pos % nbj);
    const auto inRect = [&](int i, int j) { return i >= bi0 && i < bi0 + nbi && j >= bj0 && j < bj0 + nbj; };
    const size_t bb = (size_t)bsz * bsz;
    if (J <= I) {
        // stored block (I, J): row part for (I, J); column part for (J, I) if also requested
        const double* M = A + (size_t)block_id(I, J, nb) * bb;
        int mode = 1;
        if (I != J && inRect(J, I)) mode |= 2;
        double* rowOut = P + ((size_t)(I - bi0) * nbj + (J - bj0)) * bsz;
        double* colOut = (mode & 2) ? P + ((size_t)(J - bi0) * nbj + (I - bj0)) * bsz : nullptr;
        block_apply<BSZ>(M, bsz, b + (size_t)J * bsz, b + (size_t)I * bsz, rowOut, colOut, mode, smem);
    } else if (!inRect(J, I)) {
        // stored block (J, I) seen only transposed: column part for (I, J)
        const double* M = A + (size_t)block_id(J, I, nb) * bb;
        double* colOut = P + ((size_t)(I - bi0) * nbj + (J - bj0)) * bsz;
        block_apply<BSZ>(M, bsz, nullptr, b + (size_t)J * bsz, nullptr, colOut, 2, smem);
    }
}

// ------------------------------------------------------------------ SYMV phase 2
// result[i] = (reset ? 0 : result[i]) + sum_J P[I][J][r] (J ascending); optional
// fused per-CTA partial of result . w
__global__ void __launch_bounds__(kThreads) symv_reduce(const double* __restrict__ P, double* __restrict__ result,
                                                        int bsz, int bi0, int nbi, int nbj, int reset,
                                                        const double* __restrict__ w, double* __restrict__ wpart) {
    __shared__ double sh[32];
    const int64_t rows = (int64_t)nbi * bsz;
    double prod = 0.0;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < rows; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t I = t / bsz;
        const int r = (int)(t % bsz);
        const int64_t i = (int64_t)bi0 * bsz + t;
        double v = reset ? 0.0 : result[i];
        const double* p = P + (size_t)I * nbj * bsz + r;
        for (int J = 0; J < nbj; ++J) v += p[(size_t)J * bsz];
        result[i] = v;
        if (w) prod += v * w[i];
    }
    if (w) {
        const double s = block_reduce_sum(prod, sh);
        if (threadIdx.x == 0) wpart[blockIdx.x] = s;
    }
}

// reference-order SYMV (MatrixVectorOperations.cpp:194-280): one thread per
// row, one running sum over the stored blocks j <= i row-wise and then the
// blocks j > i column-wise, products and sums rounded separately
__global__ void symv_refseq_kernel(const double* __restrict__ A, const double* __restrict__ b,
                                   double* __restrict__ result, int bsz, int nb, int bi0, int bj0, int nbi, int nbj,
                                   int reset) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= (int64_t)nbi * bsz) return;
    const int64_t i = t + (int64_t)bi0 * bsz;
    const int iIn = (int)(i % bsz);
    const int bi = (int)(i / bsz);
    const size_t bb = (size_t)bsz * bsz;
    double v = 0.0;
    if (!reset) v = __dadd_rn(v, result[i]);
    int bj = bj0;
    const int last = bj0 + nbj - 1;
    for (; bj <= (bi < last ? bi : last); ++bj) {
        const double* row = A + (size_t)block_id(bi, bj, nb) * bb + (size_t)iIn * bsz;
        const double* bv = b + (size_t)bj * bsz;
        for (int j = 0; j < bsz; ++j) v = __dadd_rn(v, __dmul_rn(row[j], bv[j]));
    }
    for (; bj < bj0 + nbj; ++bj) {
        const double* blk = A + (size_t)block_id(bj, bi, nb) * bb;
        const double* bv = b + (size_t)bj * bsz;
        for (int j = 0; j < bsz; ++j) v = __dadd_rn(v, __dmul_rn(blk[(size_t)j * bsz + iIn], bv[j]));
    }
    result[i] = v;
}

// ------------------------------------------------------------------ column update
template <int BSZ>
__global__ void __launch_bounds__(kThreads) column_update_kernel(const double* __restrict__ A, double* __restrict__ b,
                                                                 int bsz, int nb, int blockStart, int blockRow,
                                                                 int64_t blockID, int transposed) {
    __shared__ double smem[(BSZ > 0 ? 8 * BSZ : 1)];
    __shared__ double out[(BSZ > 0 ? BSZ : 1024)];
    const int g = blockIdx.x;
    const size_t bb = (size_t)bsz * bsz;
    const double* b0 = b + (size_t)blockRow * bsz;
    double* bi = b + (size_t)(blockStart + g) * bsz;
    if (!transposed) {
        const double* M = A + (size_t)(blockID + (blockStart - blockRow + g)) * bb;
        block_apply<BSZ>(M, bsz, b0, nullptr, out, nullptr, 1, smem);
    } else {
        const double* M = A + (size_t)block_id(blockRow, blockStart + g, nb) * bb;
        block_apply<BSZ>(M, bsz, nullptr, b0, nullptr, out, 2, smem);
    }
    __syncthreads();
    for (int r = threadIdx.x; r < bsz; r += blockDim.x) bi[r] -= out[r];
}

// block-column update reading FP32 blocks (mixed-precision solves), FP64 sums
template <int BSZ>
__global__ void __launch_bounds__(kThreads) column_update_f32_kernel(const float* __restrict__ A,
                                                                     double* __restrict__ b, int nb, int blockStart,
                                                                     int blockRow, int64_t blockID, int transposed) {
    __shared__ double smem[8 * BSZ];
    __shared__ double out[BSZ];
    const int g = blockIdx.x;
    const size_t bb = (size_t)BSZ * BSZ;
    const double* b0 = b + (size_t)blockRow * BSZ;
    double* bi = b + (size_t)(blockStart + g) * BSZ;
    if (!transposed) {
        const float* M = A + (size_t)(blockID + (blockStart - blockRow + g)) * bb;
        BlockApply<BSZ, float>::run(M, b0, nullptr, out, nullptr, 1, smem);
    } else {
        const float* M = A + (size_t)block_id(blockRow, blockStart + g, nb) * bb;
        BlockApply<BSZ, float>::run(M, nullptr, b0, nullptr, out, 2, smem);
    }
    __syncthreads();
    for (int r = threadIdx.x; r < BSZ; r += blockDim.x) bi[r] -= out[r];
}

// Whole sweep in one launch.  CTA c owns block rows i = c, c + P, ... (P = grid)
// and keeps their running right-hand sides in shared memory.  Forward (t = L^-1 b):
// row i takes L_ij out_j off for j = 0 .. i-1 in that order, then its owner solves
// out_i = Y_i^T t_i and publishes it; backward (L^-T) mirrors this with the
// transposed blocks L_ji^T and descending columns.  Each row is reduced by one CTA
// in column order, so the sums follow a fixed order.  Publication: the owner
// stores out_i, fences, and sets flags[i] = epoch; readers wait for that value
// (bounded: on timeout *err = 2 and the CTA stops) and read out_j past L1.
// Needs all CTAs resident at once (cooperative launch).
constexpr uint64_t kSweepWaitNs = 2000000000ull;

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint64_t sweep_clock_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Self-test of the bounded device-side wait every spin in the library uses: one
// thread waits on *flag, which nothing sets, the way a sweep waits on a row's flag
// (acquire loads against a deadline on the global timer), and records the expiry
// in *err instead of waiting on.
__global__ void bounded_wait_kernel(const unsigned* __restrict__ flag, unsigned long long timeout_ns,
                                    int* __restrict__ err) {
    const uint64_t deadline = sweep_clock_ns() + timeout_ns;
    while (ld_acquire_u32(flag) == 0u) {
        if (sweep_clock_ns() > deadline) {
            atomicExch(err, 1);
            return;
        }
    }
}

// hint: bring `bytes` (a multiple of 16) at p (16-byte aligned) into L2
__device__ __forceinline__ void sweep_prefetch_l2(const void* p, uint32_t bytes) {
    const char* b = static_cast<const char*>(p);
    for (uint32_t off = 0; off < bytes; off += 65536u) {
        const uint32_t n = bytes - off < 65536u ? bytes - off : 65536u;
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(b + off), "r"(n) : "memory");
    }
}
// The bulk of a sweep's block products streams past L2 (evict-first loads) while
// most CTAs work at once, so a row's last two block products — the one with the
// block next to the diagonal, once the previous row is published, then the one
// with its inverse diagonal block — run on the chain at a CTA's share of a busy
// HBM.  Their blocks are hinted into L2 when the owner applies the column
// kSweepAhead before the diagonal, so the chain reads them from L2.
constexpr int kSweepAhead = 4;

template <int BSZ, typename T>
__global__ void __launch_bounds__(kThreads) mixed_sweep_whole_kernel(const T* __restrict__ A,
                                                                     const T* __restrict__ Y,
                                                                     const double* __restrict__ in,
                                                                     double* __restrict__ out, int nb, int forward,
                                                                     unsigned epoch, unsigned* __restrict__ flags,
                                                                     int* __restrict__ err) {
    extern __shared__ double ssm[];
    const int P = gridDim.x, c = blockIdx.x, tid = threadIdx.x;
    const int nown = (nb - c + P - 1) / P;  // rows c + P q, q < nown
    double* smem = ssm;                     // 8 BSZ: BlockApply
    double* xs = smem + 8 * BSZ;            // the published block of out
    double* tmp = xs + BSZ;                 // one block product
    double* wk = tmp + BSZ;                 // nown rows of running right-hand side
    __shared__ int s_stop;
    const size_t bb = (size_t)BSZ * BSZ;
    for (int q = 0; q < nown; ++q)
        for (int r = tid; r < BSZ; r += blockDim.x) wk[q * BSZ + r] = in[(size_t)(c + P * q) * BSZ + r];
    if (tid == 0) s_stop = 0;
    __syncthreads();

    // the owner's diagonal solve of row i (running right-hand side in wk row q)
    auto solve = [&](int i, int q) {
        const T* Yi = Y + (size_t)i * bb;
        if (forward)
            BlockApply<BSZ, T>::run(Yi, nullptr, wk + q * BSZ, nullptr, out + (size_t)i * BSZ, 2, smem);
        else
            BlockApply<BSZ, T>::run(Yi, wk + q * BSZ, nullptr, out + (size_t)i * BSZ, nullptr, 1, smem);
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            st_release_u32(flags + i, epoch);
        }
    };
    // wk row q -= (block (r, cc) or its transpose) xs
    auto update = [&](int r, int cc, int q) {
        const T* M = A + (size_t)block_id(r, cc, nb) * bb;
        if (forward)
            BlockApply<BSZ, T>::run(M, xs, nullptr, tmp, nullptr, 1, smem);
        else
            BlockApply<BSZ, T>::run(M, nullptr, xs, nullptr, tmp, 2, smem);
        __syncthreads();
        for (int e = tid; e < BSZ; e += blockDim.x) wk[q * BSZ + e] -= tmp[e];
        __syncthreads();
    };

    // Greedy order: act on the CTA's smallest open row (forward; largest backward)
    // that can progress: apply its next column once published, or solve it once
    // every column is in.  Columns are published in order, so `known` (the last
    // column seen published) settles most checks without a load.
    int* nextc = reinterpret_cast<int*>(wk + nown * BSZ);  // per owned row: next column to apply
    __shared__ int s_pick, s_col, s_known, s_xs;
    if (tid == 0) {
        for (int q = 0; q < nown; ++q) nextc[q] = forward ? 0 : nb - 1;
        s_known = 0;  // columns seen published (forward: 0 .. known-1; backward: nb-known .. nb-1)
        s_xs = -1;
    }
    __syncthreads();
    int solved = 0;
    while (solved < nown) {
        if (tid == 0) {
            int pick = -1, col = -1;
            for (;;) {
                bool open = false;
                for (int qq = 0; qq < nown; ++qq) {
                    const int q = forward ? qq : nown - 1 - qq;
                    const int i = c + P * q;
                    const int jn = nextc[q];
                    if (jn < 0) continue;  // solved
                    open = true;
                    if (jn == i) {  // every column applied
                        pick = q;
                        col = -2;
                        break;
                    }
                    if (forward ? (jn < s_known) : (jn > nb - 1 - s_known)) {
                        pick = q;
                        col = jn;
                        break;
                    }
                }
                if (pick >= 0 || !open) break;
                // nothing to do: wait (bounded) for the next column in publication order
                const int jw = forward ? s_known : nb - 1 - s_known;
                const uint64_t deadline = sweep_clock_ns() + kSweepWaitNs;
                while (ld_acquire_u32(flags + jw) != epoch) {
                    if (sweep_clock_ns() > deadline || *reinterpret_cast<volatile int*>(err) != 0) {
                        atomicExch(err, 2);
                        s_stop = 1;
                        break;
                    }
                }
                if (s_stop) break;
                ++s_known;
            }
            s_pick = pick;
            s_col = col;
            if (pick >= 0 && col >= 0) {
                // row i's chain blocks: link block (i, i-1) forward, (i+1, i) backward
                // (both exist: a row takes column picks only when it has a link), and Y_i
                const int i = c + P * pick;
                const int first = forward ? (i > kSweepAhead ? i - kSweepAhead : 0)
                                          : (i + kSweepAhead < nb - 1 ? i + kSweepAhead : nb - 1);
                if (col == first) {
                    const int lr = forward ? i : i + 1, lc = lr - 1;
                    sweep_prefetch_l2(A + (size_t)block_id(lr, lc, nb) * bb, (uint32_t)(bb * sizeof(T)));
                    sweep_prefetch_l2(Y + (size_t)i * bb, (uint32_t)(bb * sizeof(T)));
                }
            }
        }
        __syncthreads();
        if (s_stop || s_pick < 0) break;
        const int q = s_pick, i = c + P * q, j = s_col;
        if (j == -2) {
            solve(i, q);
            if (tid == 0) nextc[q] = -1;
            ++solved;
            __syncthreads();
            continue;
        }
        if (s_xs != j) {
            for (int e = tid; e < BSZ; e += blockDim.x) xs[e] = __ldcg(out + (size_t)j * BSZ + e);
            __syncthreads();
            if (tid == 0) s_xs = j;
        }
        if (forward) update(i, j, q);
        else update(j, i, q);
        if (tid == 0) nextc[q] = forward ? j + 1 : j - 1;
        __syncthreads();
    }
}

// ------------------------------------------------------------------ TRSV
// Blocked substitution on one diagonal block: 32-row chunks, warp 0 solves the
// chunk's triangle (column oriented, as the reference), all warps then apply
// the chunk to the remaining rows.  Entries with global index >= N are neither
// written nor used (MatrixVectorOperations.cpp:303-330).
constexpr int kCh = 32;

__global__ void __launch_bounds__(kThreads) trsv_kernel(const double* __restrict__ A, double* __restrict__ b,
                                                        int bsz, int64_t N, int blockRow, int64_t blockID,
                                                        int transposed, double* __restrict__ vbuf /* unused */) {
    extern __shared__ double sh[];
    double* v = sh;                 // bsz entries of b
    double* T = sh + bsz;           // kCh x (kCh+1) triangle
    const double* L = A + (size_t)blockID * bsz * bsz;
    double* bb = b + (size_t)blockRow * bsz;
    const int64_t base = (int64_t)blockRow * bsz;
    const int valid = (N - base) < (int64_t)bsz ? (int)(N - base) : bsz;  // rows < N in this block
    for (int i = threadIdx.x; i < bsz; i += blockDim.x) v[i] = bb[i];
    __syncthreads();
    const int nch = (bsz + kCh - 1) / kCh;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int cc = 0; cc < nch; ++cc) {
        const int c = transposed ? nch - 1 - cc : cc;
        const int k0 = c * kCh;
        const int kn = min(kCh, bsz - k0);
        // stage the chunk triangle: T[i][k] = L[k0+i][k0+k] (lower) or L[k0+k][k0+i] (upper view)
        for (int e = threadIdx.x; e < kn * kn; e += blockDim.x) {
            const int i = e / kn, k = e % kn;
            T[i * (kCh + 1) + k] = transposed ? L[(size_t)(k0 + k) * bsz + (k0 + i)] : L[(size_t)(k0 + i) * bsz + (k0 + k)];
        }
        __syncthreads();
        if (warp == 0) {
            double x = lane < kn ? v[k0 + lane] : 0.0;
            for (int s = 0; s < kn; ++s) {
                const int k = transposed ? kn - 1 - s : s;
                const double diag = T[k * (kCh + 1) + k];
                const double bk = __shfl_sync(0xffffffffu, x, k) / diag;
                if (k0 + k < valid) {
                    if (lane == k) x = bk;
                    const bool below = transposed ? (lane < k) : (lane > k && lane < kn);
                    if (below) x = x - T[lane * (kCh + 1) + k] * bk;
                }
            }
            if (lane < kn && k0 + lane < valid) v[k0 + lane] = x;
        }
        __syncthreads();
        // apply the solved chunk to the rows not yet solved
        const int lo = transposed ? 0 : k0 + kn;
        const int hi = transposed ? k0 : bsz;
        for (int r = lo + (int)threadIdx.x; r < hi; r += blockDim.x) {
            if (r >= valid) continue;
            double acc = v[r];
            for (int k = 0; k < kn; ++k) {
                const int kk = transposed ? kn - 1 - k : k;
                if (k0 + kk >= valid) continue;
                const double lv = transposed ? L[(size_t)(k0 + kk) * bsz + r] : L[(size_t)r * bsz + (k0 + kk)];
                acc = acc - lv * v[k0 + kk];
            }
            v[r] = acc;
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < valid; i += blockDim.x) bb[i] = v[i];
}

int dot_blocks(int64_t len) {
    int64_t g = (len + 2047) / 2048;
    if (g < 1) g = 1;
    if (g > kDotBlocks) g = kDotBlocks;
    return (int)g;
}

}  // namespace

hs_status launch_dot(hs_ctx ctx, const double* x, const double* y, double* result, int64_t first, int64_t len,
                     cudaStream_t s) {
    hs_status st = ensure_scratch(ctx, kSmallScratch);
    if (st != HS_OK) return st;
    double* partial = static_cast<double*>(ctx->scratch);
    const int g = dot_blocks(len);
    prof_begin(ctx, s, HS_KERNEL_VECTOR);
    ctx->launches += 2;
    dot_stage1<<<g, kThreads, 0, s>>>(x, y, first, len, partial);
    dot_stage2<<<1, kThreads, 0, s>>>(partial, g, result);
    HS_CHECK_LAUNCH("dot");
    prof_end(ctx, s, HS_KERNEL_VECTOR, 2.0 * len, 16.0 * len);
    return HS_OK;
}

hs_status launch_symv_refseq(hs_ctx ctx, const double* A, const double* b, double* result, int bi0, int bj0,
                             int nbi, int nbj, int reset, cudaStream_t s) {
    const int64_t rows = (int64_t)nbi * ctx->bsz;
    if (rows <= 0) return HS_OK;
    ctx->launches += 1;
    symv_refseq_kernel<<<(unsigned)((rows + 127) / 128), 128, 0, s>>>(A, b, result, ctx->bsz, ctx->nb, bi0, bj0, nbi,
                                                                     nbj, reset);
    HS_CHECK_LAUNCH("symv_refseq");
    return HS_OK;
}

hs_status launch_dot_refseq(hs_ctx ctx, const double* x, const double* y, double* result, int64_t first,
                            int64_t len, int chunks, cudaStream_t s) {
    hs_status st = ensure_scratch(ctx, kSmallScratch);
    if (st != HS_OK) return st;
    HS_REQUIRE(chunks <= kMaxPartials, "too many chunks");
    double* part = static_cast<double*>(ctx->scratch);
    ctx->launches += 2;
    dot_refseq_chunks<<<(chunks + 127) / 128, 128, 0, s>>>(x, y, first, len, chunks, part);
    dot_refseq_final<<<1, 1, 0, s>>>(part, chunks, result);
    HS_CHECK_LAUNCH("dot_refseq");
    return HS_OK;
}

hs_status launch_symv(hs_ctx ctx, const double* A, const double* b, double* result, int bi0, int bj0, int nbi,
                      int nbj, int reset, double* dot_with, double* dot_out, cudaStream_t s) {
    if (nbi <= 0) return HS_OK;
    const int bsz = ctx->bsz;
    const size_t pbytes = (size_t)nbi * (size_t)(nbj > 0 ? nbj : 1) * bsz * sizeof(double);
    hs_status st = ensure_scratch(ctx, kSmallScratch + pbytes);
    if (st != HS_OK) return st;
    double* small = static_cast<double*>(ctx->scratch);
    double* P = reinterpret_cast<double*>(static_cast<char*>(ctx->scratch) + kSmallScratch);
    // algorithmic bytes: every stored block the rectangle touches, read once, plus the
    // vectors; positions (I, J), J > I, whose mirror (J, I) is also in the rectangle
    // reuse that block: c(c-1)/2 of them, c = the overlap of the row and column ranges
    const int64_t ov_lo = bi0 > bj0 ? bi0 : bj0, ov_hi = (bi0 + nbi < bj0 + nbj) ? bi0 + nbi : bj0 + nbj;
    const int64_t c_ov = ov_hi > ov_lo ? ov_hi - ov_lo : 0;
    const int64_t stored = (int64_t)nbi * nbj - c_ov * (c_ov - 1) / 2;
    const double bb = (double)bsz * bsz;
    prof_begin(ctx, s, HS_KERNEL_SYMV);
    if (nbj > 0) {
        ctx->launches += 1;
        // one CTA per rectangle position (I, J), row-major; positions whose block is
        // handled through its mirror exit at once.  Measured faster than one CTA per
        // stored block in storage order (5.2 vs 4.95 TB/s at N=131072).
        const int64_t grid = (int64_t)nbi * nbj;
        if (bsz == 256)
            symv_partials<256><<<(unsigned)grid, kThreads, 0, s>>>(A, b, P, bsz, ctx->nb, bi0, bj0, nbi, nbj);
        else if (bsz == 128)
            symv_partials<128><<<(unsigned)grid, kThreads, 0, s>>>(A, b, P, bsz, ctx->nb, bi0, bj0, nbi, nbj);
        else
            symv_partials<0><<<(unsigned)grid, kThreads, 0, s>>>(A, b, P, bsz, ctx->nb, bi0, bj0, nbi, nbj);
        HS_CHECK_LAUNCH("symv_partials");
    }
    const int64_t rows = (int64_t)nbi * bsz;
    int64_t rg64 = (rows + kThreads - 1) / kThreads;
    if (rg64 > kMaxPartials) rg64 = kMaxPartials;
    const unsigned rg = (unsigned)rg64;
    double* wpart = small;
    ctx->launches += dot_with ? 2 : 1;
    symv_reduce<<<rg, kThreads, 0, s>>>(P, result, bsz, bi0, nbi, nbj, reset, dot_with, wpart);
    if (dot_with) dot_stage2<<<1, kThreads, 0, s>>>(wpart, (int)rg, dot_out);
    HS_CHECK_LAUNCH("symv_reduce");
    prof_end(ctx, s, HS_KERNEL_SYMV, 2.0 * (double)nbi * nbj * bb,
             (double)stored * bb * 8.0 + 8.0 * ((double)nbj * bsz + 2.0 * nbi * bsz));
    return HS_OK;
}

// the two matvec kernels with a caller-provided partial-sum buffer P of at
// least nbi * nbj * bsz doubles; allocates nothing (hs_symv_block_noalloc)
hs_status launch_symv_partials_at(hs_ctx ctx, const double* A, const double* b, double* result, int bi0, int bj0,
                                  int nbi, int nbj, int reset, double* P, cudaStream_t s) {
    if (nbi <= 0) return HS_OK;
    const int bsz = ctx->bsz;
    if (nbj > 0) {
        const int64_t grid = (int64_t)nbi * nbj;
        ctx->launches += 1;
        if (bsz == 256)
            symv_partials<256><<<(unsigned)grid, kThreads, 0, s>>>(A, b, P, bsz, ctx->nb, bi0, bj0, nbi, nbj);
        else if (bsz == 128)
            symv_partials<128><<<(unsigned)grid, kThreads, 0, s>>>(A, b, P, bsz, ctx->nb, bi0, bj0, nbi, nbj);
        else
            symv_partials<0><<<(unsigned)grid, kThreads, 0, s>>>(A, b, P, bsz, ctx->nb, bi0, bj0, nbi, nbj);
        HS_CHECK_LAUNCH("symv_partials");
    }
    const int64_t rows = (int64_t)nbi * bsz;
    int64_t rg64 = (rows + kThreads - 1) / kThreads;
    if (rg64 > kMaxPartials) rg64 = kMaxPartials;
    ctx->launches += 1;
    symv_reduce<<<(unsigned)rg64, kThreads, 0, s>>>(P, result, bsz, bi0, nbi, nbj, reset, nullptr, nullptr);
    HS_CHECK_LAUNCH("symv_reduce");
    return HS_OK;
}

hs_status launch_column_update(hs_ctx ctx, const double* A, double* b, int blockStart, int blockCount, int blockRow,
                               int blockID, int transposed, cudaStream_t s) {
    if (blockCount <= 0) return HS_OK;
    const int bsz = ctx->bsz;
    HS_REQUIRE(bsz <= 1024, "matrixBlockSize > 1024 is not supported by the column update");
    prof_begin(ctx, s, HS_KERNEL_COLUPD);
    ctx->launches += 1;
    if (bsz == 256)
        column_update_kernel<256><<<blockCount, kThreads, 0, s>>>(A, b, bsz, ctx->nb, blockStart, blockRow, blockID,
                                                                  transposed);
    else if (bsz == 128)
        column_update_kernel<128><<<blockCount, kThreads, 0, s>>>(A, b, bsz, ctx->nb, blockStart, blockRow, blockID,
                                                                  transposed);
    else
        column_update_kernel<0><<<blockCount, kThreads, 0, s>>>(A, b, bsz, ctx->nb, blockStart, blockRow, blockID,
                                                                transposed);
    HS_CHECK_LAUNCH("column_update");
    prof_end(ctx, s, HS_KERNEL_COLUPD, 2.0 * blockCount * (double)bsz * bsz,
             (double)blockCount * bsz * bsz * 8.0 + 24.0 * blockCount * bsz);
    return HS_OK;
}

hs_status launch_bounded_wait_selftest(hs_ctx ctx, int64_t timeout_ns) {
    hs_status st = ensure_scratch(ctx, kSmallScratch);
    if (st != HS_OK) return st;
    char* base = static_cast<char*>(ctx->scratch);
    unsigned* flag = reinterpret_cast<unsigned*>(base);
    int* err = reinterpret_cast<int*>(base + 256);
    cudaStream_t s = ctx->stream;
    HS_CUDA(cudaMemsetAsync(base, 0, 512, s));
    ctx->launches += 1;
    bounded_wait_kernel<<<1, 1, 0, s>>>(flag, (unsigned long long)timeout_ns, err);
    HS_CHECK_LAUNCH("bounded_wait");
    int e = 0;
    HS_CUDA(cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, s));
    HS_CUDA(cudaStreamSynchronize(s));
    if (e) {
        set_error("hs_selftest_bounded_wait: the device-side wait ran out and returned an error status "
                  "(expected: nothing sets its flag)");
        return HS_ERR_TIMEOUT;
    }
    return HS_OK;
}

namespace {

template <typename T>
hs_status launch_sweep_whole(hs_ctx ctx, const T* A, const T* Y, const double* in, double* out, int forward,
                             unsigned epoch, unsigned* flags, int* err, cudaStream_t s) {
    const int bsz = ctx->bsz, nb = ctx->nb;
    HS_REQUIRE(bsz == 128 || bsz == 256, "the whole-sweep solve supports matrixBlockSize 128 or 256");
    int per_sm = 0;
    const void* fn = bsz == 256 ? (const void*)mixed_sweep_whole_kernel<256, T>
                                : (const void*)mixed_sweep_whole_kernel<128, T>;
    // rows per CTA for the grid used (at least one row each); shared memory for them
    auto smem_for = [&](int grid) {
        const int nown = (nb + grid - 1) / grid;
        return (size_t)(10 + nown) * bsz * sizeof(double) + (size_t)nown * sizeof(int);
    };
    int grid = nb < 2 * ctx->num_sms ? nb : 2 * ctx->num_sms;
    HS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kThreads, smem_for(grid)));
    if (grid > per_sm * ctx->num_sms) grid = per_sm * ctx->num_sms;
    HS_REQUIRE(grid >= 1, "the whole-sweep solve does not fit on the device");
    const size_t smem = smem_for(grid);
    HS_REQUIRE(smem <= 200 * 1024, "matrix too large for the single-launch sweep");
    if (smem > 48 * 1024) HS_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    void* args[] = {(void*)&A, (void*)&Y, (void*)&in, (void*)&out, (void*)&nb, (void*)&forward,
                    (void*)&epoch, (void*)&flags, (void*)&err};
    prof_begin(ctx, s, HS_KERNEL_COLUPD);
    ctx->launches += 1;
    HS_CUDA(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kThreads), args, smem, s));
    const double Tb = (double)nb * (nb - 1) / 2.0;
    prof_end(ctx, s, HS_KERNEL_COLUPD, 2.0 * (Tb + nb) * bsz * bsz, (Tb + nb) * sizeof(T) * bsz * bsz);
    return HS_OK;
}

}  // namespace

hs_status launch_mixed_sweep_whole(hs_ctx ctx, const float* A32, const float* Y, const double* in, double* out,
                                   int forward, unsigned epoch, unsigned* flags, int* err, cudaStream_t s) {
    return launch_sweep_whole<float>(ctx, A32, Y, in, out, forward, epoch, flags, err, s);
}

hs_status launch_sweep_whole_f64(hs_ctx ctx, const double* L, const double* Y, const double* in, double* out,
                                 int forward, unsigned epoch, unsigned* flags, int* err, cudaStream_t s) {
    return launch_sweep_whole<double>(ctx, L, Y, in, out, forward, epoch, flags, err, s);
}

hs_status launch_column_update_f32(hs_ctx ctx, const float* A32, double* b, int blockStart, int blockCount,
                                   int blockRow, int blockID, int transposed, cudaStream_t s) {
    if (blockCount <= 0) return HS_OK;
    const int bsz = ctx->bsz;
    HS_REQUIRE(bsz == 128 || bsz == 256, "FP32 column update supports matrixBlockSize 128 or 256");
    prof_begin(ctx, s, HS_KERNEL_COLUPD);
    ctx->launches += 1;
    if (bsz == 256)
        column_update_f32_kernel<256><<<blockCount, kThreads, 0, s>>>(A32, b, ctx->nb, blockStart, blockRow, blockID,
                                                                     transposed);
    else
        column_update_f32_kernel<128><<<blockCount, kThreads, 0, s>>>(A32, b, ctx->nb, blockStart, blockRow, blockID,
                                                                     transposed);
    HS_CHECK_LAUNCH("column_update_f32");
    prof_end(ctx, s, HS_KERNEL_COLUPD, 2.0 * blockCount * (double)bsz * bsz,
             (double)blockCount * bsz * bsz * 4.0 + 24.0 * blockCount * bsz);
    return HS_OK;
}

hs_status launch_trsv(hs_ctx ctx, const double* A, double* b, int blockRow, int blockID, int transposed,
                      cudaStream_t s) {
    const int bsz = ctx->bsz;
    const size_t smem = (size_t)(bsz + kCh * (kCh + 1)) * sizeof(double);
    HS_REQUIRE(smem <= 200 * 1024, "matrixBlockSize too large for the block triangular solve");
    if (smem > 48 * 1024) HS_CUDA(cudaFuncSetAttribute(trsv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                       (int)smem));
    prof_begin(ctx, s, HS_KERNEL_TRSV);
    ctx->launches += 1;
    trsv_kernel<<<1, kThreads, smem, s>>>(A, b, bsz, ctx->N, blockRow, blockID, transposed, nullptr);
    HS_CHECK_LAUNCH("trsv");
    prof_end(ctx, s, HS_KERNEL_TRSV, (double)bsz * bsz, (double)bsz * bsz * 4.0 + 16.0 * bsz);
    return HS_OK;
}

hs_status launch_vec(hs_ctx ctx, int op, const double* x, const double* y, double alpha, double* out,
                     int64_t first, int64_t len, cudaStream_t s) {
    if (len <= 0) return HS_OK;
    int64_t g = (len + kThreads - 1) / kThreads;
    if (g > 8 * (int64_t)ctx->num_sms) g = 8 * (int64_t)ctx->num_sms;
    ctx->launches += 1;
    if (ctx->ref_chunks > 0) {
        switch (op) {
            case 0: vec_kernel_ref<0><<<(unsigned)g, kThreads, 0, s>>>(x, y, alpha, out, first, len); break;
            case 1: vec_kernel_ref<1><<<(unsigned)g, kThreads, 0, s>>>(x, y, alpha, out, first, len); break;
            case 2: vec_kernel_ref<2><<<(unsigned)g, kThreads, 0, s>>>(x, y, alpha, out, first, len); break;
            default: vec_kernel_ref<3><<<(unsigned)g, kThreads, 0, s>>>(x, y, alpha, out, first, len); break;
        }
        HS_CHECK_LAUNCH("vector op");
        return HS_OK;
    }
    switch (op) {
        case 0: vec_kernel<0><<<(unsigned)g, kThreads, 0, s>>>(x, y, alpha, out, first, len); break;
        case 1: vec_kernel<1><<<(unsigned)g, kThreads, 0, s>>>(x, y, alpha, out, first, len); break;
        case 2: vec_kernel<2><<<(unsigned)g, kThreads, 0, s>>>(x, y, alpha, out, first, len); break;
        default: vec_kernel<3><<<(unsigned)g, kThreads, 0, s>>>(x, y, alpha, out, first, len); break;
    }
    HS_CHECK_LAUNCH("vector op");
    return HS_OK;
}

}  // namespace hs
