// k_factor.cu — kernels of the blocked right-looking Cholesky in FP64:
// diagonal-block POTRF, panel TRSM and the SYRK/GEMM trailing update.
//
// Reference kernels replaced (paths relative to the reference root):
//   MatrixOperations.cpp:7-191          cholesky / cholesky_GPU / cholesky_optimizedGPU
//   MatrixMatrixOperations.cpp:5-144    triangularSolve{,_optimizedGPU,_optimizedCPU}
//   MatrixMatrixOperations.cpp:146-361  symmetricMatrixMatrixDiagonal{,...}
//   MatrixMatrixOperations.cpp:364-906  matrixMatrixStep{,...}
//
// The trailing update is the only O(N^3) part.  For bsz a multiple of 128 it
// runs on the FP64 tensor pipe (DMMA, mma.sync m8n8k4 f64): 128x128 output
// tiles per CTA, K streamed in 16-wide slabs through a 4-stage cp.async ring in
// shared memory, accumulators held in registers and initialised with -C so the
// result is C - sum_k a_ik b_jk accumulated in k order.  Other block sizes use
// a scalar fallback with the reference's accumulation order.
#include "hs_internal.cuh"
#include "hs_mixed.cuh"

namespace hs {
namespace {

// ------------------------------------------------------------------ POTRF
// In-shared-memory POTRF of an n x n (n <= 128) sub-block with leading
// dimension ld: the reference's column-by-column right-looking order
// (MatrixOperations.cpp:23-57), rows >= valid untouched, strict upper triangle
// of valid rows zeroed.  A pivot that is not > 0 on a valid row records its
// global row in *info.
__global__ void __launch_bounds__(512) potrf_smem_kernel(double* __restrict__ Ablk, int ld, int n, int valid,
                                                         long long* __restrict__ info, long long row_base) {
    extern __shared__ double S[];
    const int sld = n + 1;
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int i = e / n, j = e % n;
        S[i * sld + j] = Ablk[(size_t)i * ld + j];
    }
    __syncthreads();
    for (int k = 0; k < n; ++k) {
        const double piv = S[k * sld + k];
        const double s = sqrt(piv);
        if (threadIdx.x == 0 && k < valid && !(piv > 0.0)) atomicMin(info, row_base + k);
        for (int i = k + 1 + (int)threadIdx.x; i < valid; i += blockDim.x) S[i * sld + k] = S[i * sld + k] / s;
        __syncthreads();
        if (threadIdx.x == 0) S[k * sld + k] = s;
        // lower trailing part: j in (k, n), i in [j, valid); one warp per column,
        // lanes over rows (no index divisions, no idle lanes above the diagonal)
        {
            const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
            for (int j = k + 1 + warp; j < valid; j += nw) {
                const double sjk = S[j * sld + k];
                for (int i = j + lane; i < valid; i += 32) S[i * sld + j] = S[i * sld + j] - S[i * sld + k] * sjk;
            }
        }
        __syncthreads();
    }
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int i = e / n, j = e % n;
        if (i >= valid) continue;
        Ablk[(size_t)i * ld + j] = (j > i) ? 0.0 : S[i * sld + j];
    }
    // the reference also writes a_kk = sqrt(a_kk) on padding rows (MatrixOperations.cpp:38-40)
    for (int k = valid + (int)threadIdx.x; k < n; k += blockDim.x) Ablk[(size_t)k * ld + k] = S[k * sld + k];
}

// global-memory fallback (bsz > 256): one CTA, same order as the reference
__global__ void __launch_bounds__(1024) potrf_global_kernel(double* __restrict__ B, int n, int valid,
                                                            long long* __restrict__ info, long long row_base) {
    for (int k = 0; k < n; ++k) {
        const double piv = B[(size_t)k * n + k];
        const double s = sqrt(piv);
        if (threadIdx.x == 0 && k < valid && !(piv > 0.0)) atomicMin(info, row_base + k);
        __syncthreads();
        for (int i = k + 1 + (int)threadIdx.x; i < valid; i += blockDim.x) B[(size_t)i * n + k] /= s;
        __syncthreads();
        if (threadIdx.x == 0) B[(size_t)k * n + k] = s;
        const int m = n - k - 1;
        for (int64_t e = threadIdx.x; e < (int64_t)m * m; e += blockDim.x) {
            const int j = k + 1 + (int)(e / m);
            const int i = k + 1 + (int)(e % m);
            if (i >= j && i < valid) B[(size_t)i * n + j] -= B[(size_t)i * n + k] * B[(size_t)j * n + k];
        }
        __syncthreads();
    }
    for (int64_t e = threadIdx.x; e < (int64_t)n * n; e += blockDim.x) {
        const int i = (int)(e / n), j = (int)(e % n);
        if (i < valid && j > i) B[e] = 0.0;
    }
}

__global__ void zero_tile_kernel(double* __restrict__ P, int ld, int rows, int cols) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < rows * cols; e += gridDim.x * blockDim.x)
        P[(size_t)(e / cols) * ld + (e % cols)] = 0.0;
}

// ------------------------------------------------------------------ TRSM
// B <- B L^-T for slabs of up to 64 rows: each CTA keeps its slab in shared
// memory and walks the columns in 32-wide chunks: solve the chunk against the
// chunk's diagonal triangle (column order, divisions as the reference's CPU
// kernel, MatrixMatrixOperations.cpp:125-139), then subtract the chunk's
// contribution from the columns to its right, accumulating in k order.
constexpr int kTrsmRows = 64;
constexpr int kTrsmCh = 32;

struct TrsmArgs {
    const double* L;   // triangle (lower), leading dimension ldL
    int ldL;
    int n;             // triangle size = columns of B
    double* A;         // base for B items
    int ldB;
    int64_t item0;     // panel mode: first B block id; sub mode: ignored
    int slabs;         // slabs per B item
    int rows_last;     // rows in each item (bsz or sub-block rows)
    int64_t block_elems;  // panel mode: stride between B blocks (elements); 0: single item at A
    int l_diag_nb;        // > 0: item q solves against its own triangle, the diagonal block q of the
                          // packed matrix at L with this many block columns (L = its base)
    int slab_rows;        // rows of B a CTA solves (0: kTrsmRows); fewer rows, more CTAs an item
};

__global__ void __launch_bounds__(256) trsm_kernel(TrsmArgs a) {
    extern __shared__ double sm[];
    const int n = a.n;
    const int bld = n + 1;
    double* Bs = sm;                                  // kTrsmRows x (n+1)
    double* Tc = Bs + kTrsmRows * bld;                // kTrsmCh x (kTrsmCh+1)
    double* Lp = Tc + kTrsmCh * (kTrsmCh + 1);        // n x (kTrsmCh+1)
    const int item = blockIdx.x / a.slabs;
    const int slab = blockIdx.x % a.slabs;
    const double* Lt = a.l_diag_nb > 0 ? a.L + (size_t)column_start(item, a.l_diag_nb) * n * n : a.L;
    const int sr = a.slab_rows > 0 ? a.slab_rows : kTrsmRows;
    double* B = a.A + (a.block_elems ? (size_t)(a.item0 + item) * a.block_elems : 0) + (size_t)slab * sr * a.ldB;
    const int rows = min(sr, a.rows_last - slab * sr);
    for (int e = threadIdx.x; e < rows * n; e += blockDim.x) {
        const int r = e / n, c = e % n;
        Bs[r * bld + c] = B[(size_t)r * a.ldB + c];
    }
    const int nch = (n + kTrsmCh - 1) / kTrsmCh;
    for (int ch = 0; ch < nch; ++ch) {
        const int k0 = ch * kTrsmCh;
        const int kn = min(kTrsmCh, n - k0);
        const int rest = n - (k0 + kn);
        __syncthreads();
        for (int e = threadIdx.x; e < kn * kn; e += blockDim.x) {
            const int i = e / kn, k = e % kn;
            Tc[i * (kTrsmCh + 1) + k] = Lt[(size_t)(k0 + i) * a.ldL + (k0 + k)];
        }
        for (int e = threadIdx.x; e < rest * kn; e += blockDim.x) {
            const int i = e / kn, k = e % kn;
            Lp[i * (kTrsmCh + 1) + k] = Lt[(size_t)(k0 + kn + i) * a.ldL + (k0 + k)];
        }
        __syncthreads();
        // chunk solve: one thread per row (rows are independent)
        for (int r = threadIdx.x; r < rows; r += blockDim.x) {
            double* row = Bs + r * bld + k0;
            for (int k = 0; k < kn; ++k) {
                const double bk = row[k] / Tc[k * (kTrsmCh + 1) + k];
                row[k] = bk;
                for (int i = k + 1; i < kn; ++i) row[i] = row[i] - Tc[i * (kTrsmCh + 1) + k] * bk;
            }
        }
        __syncthreads();
        // trailing columns: b_rc -= sum_k b_rk * L[c][k], k ascending
        for (int e = threadIdx.x; e < rows * rest; e += blockDim.x) {
            const int r = e / rest, c = e % rest;
            double v = Bs[r * bld + k0 + kn + c];
            const double* bk = Bs + r * bld + k0;
            const double* lc = Lp + c * (kTrsmCh + 1);
            for (int k = 0; k < kn; ++k) v = v - lc[k] * bk[k];
            Bs[r * bld + k0 + kn + c] = v;
        }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < rows * n; e += blockDim.x) {
        const int r = e / n, c = e % n;
        B[(size_t)r * a.ldB + c] = Bs[r * bld + c];
    }
}

size_t trsm_smem(int n) {
    return (size_t)(kTrsmRows * (n + 1) + kTrsmCh * (kTrsmCh + 1) + n * (kTrsmCh + 1)) * sizeof(double);
}

// ------------------------------------------------------------------ DMMA tile
constexpr int BM = 128, BN = 128, BK = 16, STAGES = 4, SPAD = 20;
constexpr int kTileSmem = 2 * STAGES * BM * SPAD * (int)sizeof(double);  // 160 KB


__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// C (128 x 128, ldc) -= A (128 x K, lda) * B (128 x K, ldb)^T; `lower`: only
// entries with row >= col are written (diagonal tile of a diagonal block).
__device__ __forceinline__ void dmma_tile(double* __restrict__ C, int64_t ldc, const double* __restrict__ Ag,
                                          int64_t lda, const double* __restrict__ Bg, int64_t ldb, int K,
                                          bool lower, double* smem) {
    double* As = smem;                         // [STAGES][BM][SPAD]
    double* Bs = smem + STAGES * BM * SPAD;    // [STAGES][BN][SPAD]
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int wm = warp >> 2, wn = warp & 3;
    const int g = lane >> 2, t = lane & 3;

    double acc[8][4][2];
#pragma unroll
    for (int mi = 0; mi < 8; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) {
            const int r = wm * 64 + mi * 8 + g;
            const int c = wn * 32 + ni * 8 + 2 * t;
            const double2 v = *reinterpret_cast<const double2*>(C + (size_t)r * ldc + c);
            acc[mi][ni][0] = -v.x;
            acc[mi][ni][1] = -v.y;
        }

    const int ktiles = K / BK;
    auto load_stage = [&](int stage, int kt) {
        const int kc = kt * BK;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int e = tid + 256 * q;
            const int row = e >> 3, ch = e & 7;
            cp_async16(As + (stage * BM + row) * SPAD + ch * 2, Ag + (size_t)row * lda + kc + ch * 2);
            cp_async16(Bs + (stage * BN + row) * SPAD + ch * 2, Bg + (size_t)row * ldb + kc + ch * 2);
        }
    };
#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
        if (s < ktiles) load_stage(s, s);
        cp_async_commit();
    }
    for (int kt = 0; kt < ktiles; ++kt) {
        cp_async_wait<STAGES - 2>();
        __syncthreads();
        {
            const int nk = kt + STAGES - 1;
            if (nk < ktiles) load_stage(nk % STAGES, nk);
            cp_async_commit();
        }
        const double* as = As + (kt % STAGES) * BM * SPAD + (wm * 64 + g) * SPAD + t;
        const double* bs = Bs + (kt % STAGES) * BN * SPAD + (wn * 32 + g) * SPAD + t;
#pragma unroll
        for (int kk = 0; kk < BK / 4; ++kk) {
            double a[8], b[4];
#pragma unroll
            for (int mi = 0; mi < 8; ++mi) a[mi] = as[mi * 8 * SPAD + kk * 4];
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) b[ni] = bs[ni * 8 * SPAD + kk * 4];
#pragma unroll
            for (int mi = 0; mi < 8; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni) dmma884(acc[mi][ni], a[mi], b[ni]);
        }
    }
    cp_async_wait<0>();
    __syncthreads();  // the ring is reused by the CTA's next tile
#pragma unroll
    for (int mi = 0; mi < 8; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) {
            const int r = wm * 64 + mi * 8 + g;
            const int c = wn * 32 + ni * 8 + 2 * t;
            double* p = C + (size_t)r * ldc + c;
            if (!lower || c + 1 <= r) {
                *reinterpret_cast<double2*>(p) = make_double2(-acc[mi][ni][0], -acc[mi][ni][1]);
            } else if (c <= r) {
                p[0] = -acc[mi][ni][0];
            }
        }
}

// ------------------------------------------------------ templated DMMA tiles
// A CTA computes a TM x TN output tile with (TM/WM) x (TN/WN) warps of WM x WN
// (m8n8k4 sub-tiles), K streamed in 16-wide slabs through an ST-stage cp.async
// ring with rows padded to SPAD doubles (row stride 40 banks: the eight rows a
// fragment load touches fall in distinct bank groups).
template <int TM, int TN, int WM, int WN, int ST>
struct DTile {
    static constexpr int kWarpsN = TN / WN;
    static constexpr int kThreads = 32 * (TM / WM) * (TN / WN);
    static constexpr int kMi = WM / 8, kNi = WN / 8;
    static constexpr int kSmem = ST * (TM + TN) * SPAD * (int)sizeof(double);
    static constexpr int kChunks = (TM + TN) * (BK / 2);  // 16-byte copies a stage
    static_assert(kChunks % kThreads == 0, "copies must split evenly over the threads");
    static_assert((TM * (BK / 2)) % 32 == 0, "A and B copies must not share a warp");
};

// PRODUCT = false: C (TM x TN, ldc) <- C - A (TM x K, lda) B (TN x K, ldb)^T,
//   accumulated from -C in k order; with `lower`, entry (r, c) is written only
//   if c + shift <= r (a tile that crosses the diagonal of a diagonal block).
// PRODUCT = true: C <- A B^T with B lower triangular by rows (B[c][k] = 0 for
//   k > c): a warp skips the K slabs past its last column.  C may be A itself:
//   every load of A completes before the first store.
template <int TM, int TN, int WM, int WN, int ST, bool PRODUCT>
__device__ __forceinline__ void dmma_tile_t(double* C, int64_t ldc, const double* Ag, int64_t lda,
                                            const double* __restrict__ Bg, int64_t ldb, int K, bool lower, int shift,
                                            double* smem) {
    using D = DTile<TM, TN, WM, WN, ST>;
    double* As = smem;                   // [ST][TM][SPAD]
    double* Bs = smem + ST * TM * SPAD;  // [ST][TN][SPAD]
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int wm = warp / D::kWarpsN, wn = warp % D::kWarpsN;
    const int g = lane >> 2, t = lane & 3;

    double acc[D::kMi][D::kNi][2];
#pragma unroll
    for (int mi = 0; mi < D::kMi; ++mi)
#pragma unroll
        for (int ni = 0; ni < D::kNi; ++ni) {
            if (PRODUCT) {
                acc[mi][ni][0] = acc[mi][ni][1] = 0.0;
            } else {
                const int r = wm * WM + mi * 8 + g;
                const int c = wn * WN + ni * 8 + 2 * t;
                const double2 v = *reinterpret_cast<const double2*>(C + (size_t)r * ldc + c);
                acc[mi][ni][0] = -v.x;
                acc[mi][ni][1] = -v.y;
            }
        }

    const int ktiles = K / BK;
    // PRODUCT: rows wn*WN .. wn*WN+WN-1 of B vanish past column wn*WN+WN-1
    const int kt_warp = PRODUCT ? min(ktiles, (wn * WN + WN + BK - 1) / BK) : ktiles;
    auto load_stage = [&](int stage, int kt) {
        const int kc = kt * BK;
#pragma unroll
        for (int q = 0; q < D::kChunks / D::kThreads; ++q) {
            const int e = tid + D::kThreads * q;
            const int row = e >> 3, ch = e & 7;
            if (row < TM)
                cp_async16(As + (stage * TM + row) * SPAD + ch * 2, Ag + (size_t)row * lda + kc + ch * 2);
            else
                cp_async16(Bs + (stage * TN + row - TM) * SPAD + ch * 2, Bg + (size_t)(row - TM) * ldb + kc + ch * 2);
        }
    };
#pragma unroll
    for (int s = 0; s < ST - 1; ++s) {
        if (s < ktiles) load_stage(s, s);
        cp_async_commit();
    }
    for (int kt = 0; kt < ktiles; ++kt) {
        cp_async_wait<ST - 2>();
        __syncthreads();
        {
            const int nk = kt + ST - 1;
            if (nk < ktiles) load_stage(nk % ST, nk);
            cp_async_commit();
        }
        if (kt < kt_warp) {
            const double* as = As + (kt % ST) * TM * SPAD + (wm * WM + g) * SPAD + t;
            const double* bs = Bs + (kt % ST) * TN * SPAD + (wn * WN + g) * SPAD + t;
#pragma unroll
            for (int kk = 0; kk < BK / 4; ++kk) {
                double a[D::kMi], b[D::kNi];
#pragma unroll
                for (int mi = 0; mi < D::kMi; ++mi) a[mi] = as[mi * 8 * SPAD + kk * 4];
#pragma unroll
                for (int ni = 0; ni < D::kNi; ++ni) b[ni] = bs[ni * 8 * SPAD + kk * 4];
#pragma unroll
                for (int mi = 0; mi < D::kMi; ++mi)
#pragma unroll
                    for (int ni = 0; ni < D::kNi; ++ni) dmma884(acc[mi][ni], a[mi], b[ni]);
            }
        }
    }
    cp_async_wait<0>();
    __syncthreads();  // every load of A has landed before C (possibly A) is written
#pragma unroll
    for (int mi = 0; mi < D::kMi; ++mi)
#pragma unroll
        for (int ni = 0; ni < D::kNi; ++ni) {
            const int r = wm * WM + mi * 8 + g;
            const int c = wn * WN + ni * 8 + 2 * t;
            const double v0 = PRODUCT ? acc[mi][ni][0] : -acc[mi][ni][0];
            const double v1 = PRODUCT ? acc[mi][ni][1] : -acc[mi][ni][1];
            double* p = C + (size_t)r * ldc + c;
            if (!lower || c + 1 + shift <= r) {
                *reinterpret_cast<double2*>(p) = make_double2(v0, v1);
            } else if (c + shift <= r) {
                p[0] = v0;
            }
        }
}

// Trailing update, two CTAs an SM: 128 x 64 tiles, 8 warps of 32 x 32, 3 stages.
// Each CTA's C preload and store overlap the other CTA's tensor work.
constexpr int kUTM = 128, kUTN = 64, kUWM = 32, kUWN = 32, kUST = 3;
using UTile = DTile<kUTM, kUTN, kUWM, kUWN, kUST>;

// Work list of a trailing update.  Column mode (the factor driver): the pairs
// (r, c) of the columns c in [colStart, colEnd), c <= r < nb, column by column.
// Row mode (the operator entry points, MatrixMatrixOperations.cpp:146-906): GEMM
// pairs (r, c), r in [gemmStart, gemmStart+gemmCount), blockRow < c < r, then
// SYRK diagonal blocks j in [syrkStart, syrkStart+syrkCount).
struct UpdateArgs {
    double* A;
    int64_t blockID;  // diagonal block of column blockRow (the panel's column)
    int blockRow, nb, bsz;
    int rowMode;
    int colStart, colEnd;            // column mode
    int64_t gemmPairs, pairBase;     // row mode
    int syrkStart;
    int tilesM, tilesN;
    int64_t totalPairs;
};

__device__ __forceinline__ void decode_pair(const UpdateArgs& a, int64_t pair, int* r, int* c) {
    if (a.rowMode) {
        if (pair < a.gemmPairs) {
            const int64_t tt = pair + a.pairBase;
            const int u = tri_root(tt);
            *r = a.blockRow + 1 + (u + 1);
            *c = a.blockRow + 1 + (int)(tt - (int64_t)u * (u + 1) / 2);
        } else {
            *r = *c = a.syrkStart + (int)(pair - a.gemmPairs);
        }
        return;
    }
    // column c holds nb - c pairs: the largest c with offset(c) <= pair
    auto offset = [&](int cc) -> int64_t {
        return (int64_t)(cc - a.colStart) * a.nb - ((int64_t)cc * (cc - 1) - (int64_t)a.colStart * (a.colStart - 1)) / 2;
    };
    int lo = a.colStart, hi = a.colEnd - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (offset(mid) <= pair) lo = mid; else hi = mid - 1;
    }
    *c = lo;
    *r = lo + (int)(pair - offset(lo));
}

__global__ void __launch_bounds__(UTile::kThreads, 2) update_dmma_kernel(UpdateArgs a) {
    extern __shared__ __align__(16) double smem[];
    const int tpb = a.tilesM * a.tilesN;
    const int64_t pair = blockIdx.x / tpb;
    const int tile = (int)(blockIdx.x % tpb);
    int r, c;
    decode_pair(a, pair, &r, &c);
    const int ti = tile / a.tilesN, tj = tile % a.tilesN;
    const int shift = tj * kUTN - ti * kUTM;  // tile column offset minus row offset inside the block
    const bool diag = r == c;
    if (diag && shift > kUTM - 1) return;      // entirely above the diagonal
    const bool lower = diag && shift + kUTN - 1 > 0;
    const size_t bb = (size_t)a.bsz * a.bsz;
    double* C = a.A + (size_t)block_id(r, c, a.nb) * bb + (size_t)ti * kUTM * a.bsz + (size_t)tj * kUTN;
    const double* Ag = a.A + (size_t)(a.blockID + (r - a.blockRow)) * bb + (size_t)ti * kUTM * a.bsz;
    const double* Bg = a.A + (size_t)(a.blockID + (c - a.blockRow)) * bb + (size_t)tj * kUTN * a.bsz;
    dmma_tile_t<kUTM, kUTN, kUWM, kUWN, kUST, false>(C, a.bsz, Ag, a.bsz, Bg, a.bsz, a.bsz, lower, shift, smem);
}

// Panel TRSM as a tensor-core product: B <- B X^T with X = L_kk^-1 (row major,
// lower triangular), in place; one CTA per 64 rows of a panel block.
template <int BSZ>
struct TrsmTile {
    using T = DTile<64, BSZ, 32, BSZ / 4, 3>;
};

template <int BSZ>
__global__ void __launch_bounds__(256, 1) trsm_dmma_kernel(double* A, int64_t firstBlock, const double* __restrict__ X) {
    extern __shared__ __align__(16) double smem[];
    constexpr int kSlabs = BSZ / 64;
    const int64_t item = blockIdx.x / kSlabs;
    const int slab = blockIdx.x % kSlabs;
    double* B = A + (size_t)(firstBlock + item) * BSZ * BSZ + (size_t)slab * 64 * BSZ;
    dmma_tile_t<64, BSZ, 32, BSZ / 4, 3, true>(B, BSZ, B, BSZ, X, BSZ, BSZ, false, 0, smem);
}

__global__ void identity_block_kernel(double* __restrict__ Y, int n) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n * n; e += gridDim.x * blockDim.x)
        Y[e] = (e / n == e % n) ? 1.0 : 0.0;
}

// X = Y^T for one n x n block (32 x 32 tiles through shared memory)
__global__ void transpose_block_kernel(const double* __restrict__ Y, double* __restrict__ X, int n) {
    __shared__ double tile[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int i = threadIdx.y; i < 32; i += blockDim.y) tile[i][threadIdx.x] = Y[(size_t)(by + i) * n + bx + threadIdx.x];
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y) X[(size_t)(bx + i) * n + by + threadIdx.x] = tile[threadIdx.x][i];
}

// single-tile form used inside the blocked POTRF of a 256 block
__global__ void __launch_bounds__(256, 1) tile_update_kernel(double* C, int ldc, const double* Ag, const double* Bg,
                                                             int ld, int K, int lower) {
    extern __shared__ __align__(16) double smem[];
    dmma_tile(C, ldc, Ag, ld, Bg, ld, K, lower != 0, smem);
}

// scalar fallback (any bsz): one thread per output element; SYRK follows
// MatrixMatrixOperations.cpp:346-355 (value -= c_ik c_jk in k order), GEMM
// follows :893-900 (sum from zero, subtracted once)
__global__ void update_scalar_kernel(UpdateArgs a) {
    const int64_t bb = (int64_t)a.bsz * a.bsz;
    const int64_t pair = blockIdx.y + (int64_t)blockIdx.z * 65535;
    if (pair >= a.totalPairs) return;
    int r, c;
    decode_pair(a, pair, &r, &c);
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= bb) return;
    const int i = (int)(e / a.bsz), j = (int)(e % a.bsz);
    double* C = a.A + block_id(r, c, a.nb) * bb;
    const double* Rk = a.A + (a.blockID + (r - a.blockRow)) * bb;
    const double* Ck = a.A + (a.blockID + (c - a.blockRow)) * bb;
    if (r == c) {
        if (i < j) return;
        double v = C[(size_t)i * a.bsz + j];
        for (int k = 0; k < a.bsz; ++k) v = v - Rk[(size_t)i * a.bsz + k] * Rk[(size_t)j * a.bsz + k];
        C[(size_t)i * a.bsz + j] = v;
    } else {
        double v = 0.0;
        for (int k = 0; k < a.bsz; ++k) v += Rk[(size_t)i * a.bsz + k] * Ck[(size_t)j * a.bsz + k];
        C[(size_t)i * a.bsz + j] -= v;
    }
}

bool attrs_done[64] = {};
hs_status set_attrs() {
    int dev = 0;
    HS_CUDA(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && attrs_done[dev]) return HS_OK;
    HS_CUDA(cudaFuncSetAttribute(update_dmma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, UTile::kSmem));
    HS_CUDA(cudaFuncSetAttribute(trsm_dmma_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 TrsmTile<128>::T::kSmem));
    HS_CUDA(cudaFuncSetAttribute(trsm_dmma_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 TrsmTile<256>::T::kSmem));
    HS_CUDA(cudaFuncSetAttribute(tile_update_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kTileSmem));
    HS_CUDA(cudaFuncSetAttribute(trsm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)trsm_smem(256)));
    HS_CUDA(cudaFuncSetAttribute(potrf_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(128 * 129 * sizeof(double))));
    if (dev >= 0 && dev < 64) attrs_done[dev] = true;
    return HS_OK;
}

hs_status launch_trsm_args(hs_ctx ctx, const TrsmArgs& ta, int items, cudaStream_t s) {
    ctx->launches += 1;
    HS_REQUIRE(ta.n <= 256, "TRSM supports triangles up to 256");
    const size_t smem = trsm_smem(ta.n);
    trsm_kernel<<<items * ta.slabs, 256, smem, s>>>(ta);
    HS_CHECK_LAUNCH("trsm");
    return HS_OK;
}

hs_status potrf_small(hs_ctx ctx, double* blk, int ld, int n, int valid, long long row_base, cudaStream_t s) {
    const size_t smem = (size_t)n * (n + 1) * sizeof(double);
    ctx->launches += 1;
    potrf_smem_kernel<<<1, 512, smem, s>>>(blk, ld, n, valid, ctx->d_info, row_base);
    HS_CHECK_LAUNCH("potrf");
    return HS_OK;
}

}  // namespace

static hs_status potrf_impl(hs_ctx ctx, double* A, int blockID, int blockRow, cudaStream_t s) {
    hs_status st = set_attrs();
    if (st != HS_OK) return st;
    const int bsz = ctx->bsz;
    double* blk = A + (size_t)blockID * bsz * bsz;
    const long long row_base = (long long)blockRow * bsz;
    const int64_t rem = ctx->N - row_base;
    const int valid = rem <= 0 ? 0 : (rem < bsz ? (int)rem : bsz);
    if (bsz <= 128) return potrf_small(ctx, blk, bsz, bsz, valid, row_base, s);
    if (bsz == 256) {
        // [A11 . ; A21 A22] with 128 x 128 quadrants: POTRF(A11), A21 <- A21 L11^-T,
        // A22 -= A21 A21^T (lower, DMMA tile), POTRF(A22), zero the upper-right quadrant
        const int n1 = 128, n2 = 128;
        st = potrf_small(ctx, blk, bsz, n1, min(valid, n1), row_base, s);
        if (st != HS_OK) return st;
        double* A21 = blk + (size_t)n1 * bsz;
        double* A22 = A21 + n1;
        if (valid > n1) {
            TrsmArgs ta{blk, bsz, n1, A21, bsz, 0, n2 / kTrsmRows, n2, 0};
            st = launch_trsm_args(ctx, ta, 1, s);
            if (st != HS_OK) return st;
            ctx->launches += 1;
            tile_update_kernel<<<1, 256, kTileSmem, s>>>(A22, bsz, A21, A21, bsz, n1, 1);
            HS_CHECK_LAUNCH("potrf syrk");
            st = potrf_small(ctx, A22, bsz, n2, valid - n1, row_base + n1, s);
        } else {
            // rows >= 128 are padding; the reference still writes sqrt(0) on their diagonal
            st = potrf_small(ctx, A22, bsz, n2, 0, row_base + n1, s);
        }
        if (st != HS_OK) return st;
        ctx->launches += 1;
        zero_tile_kernel<<<16, 256, 0, s>>>(blk + n1, bsz, min(valid, n1), n2);
        HS_CHECK_LAUNCH("potrf zero");
        return HS_OK;
    }
    ctx->launches += 1;
    potrf_global_kernel<<<1, 1024, 0, s>>>(blk, bsz, valid, ctx->d_info, row_base);
    HS_CHECK_LAUNCH("potrf");
    return HS_OK;
}

hs_status launch_potrf(hs_ctx ctx, double* A, int blockID, int blockRow, cudaStream_t s) {
    const double n = ctx->bsz;
    prof_begin(ctx, s, HS_KERNEL_POTRF);
    hs_status st = potrf_impl(ctx, A, blockID, blockRow, s);
    prof_end(ctx, s, HS_KERNEL_POTRF, n * n * n / 3.0, 2.0 * n * n * 8.0);
    return st;
}

hs_status launch_diag_inverse(hs_ctx ctx, const double* Lkk, double* Y, double* X, cudaStream_t s) {
    // Y = I L^-T by the substitution kernel, X = Y^T = L^-1 (row major, lower triangular:
    // every entry above the diagonal of Y comes out exactly zero)
    const int n = ctx->bsz;
    ctx->launches += 1;
    identity_block_kernel<<<64, 256, 0, s>>>(Y, n);
    HS_CHECK_LAUNCH("identity");
    // one block on the critical path of the factor: 16 rows of Y a CTA (16 CTAs for
    // bsz 256) instead of 64, the trailing products of a chunk spread 4x wider
    constexpr int kRows = 16;
    TrsmArgs ta{Lkk, n, n, Y, n, 0, (n + kRows - 1) / kRows, n, (int64_t)n * n, 0, kRows};
    hs_status st = launch_trsm_args(ctx, ta, 1, s);
    if (st != HS_OK) return st;
    ctx->launches += 1;
    transpose_block_kernel<<<dim3(n / 32, n / 32), dim3(32, 8), 0, s>>>(Y, X, n);
    HS_CHECK_LAUNCH("transpose");
    return HS_OK;
}

__global__ void identity_blocks_kernel(double* __restrict__ Y, int n, int64_t blocks) {
    const int64_t total = (int64_t)n * n * blocks;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t w = e % ((int64_t)n * n);
        Y[e] = (w / n == w % n) ? 1.0 : 0.0;
    }
}

// P = the last diagonal block with a unit diagonal on its padding rows (valid < n)
__global__ void pad_unit_block_kernel(const double* __restrict__ D, double* __restrict__ P, int n, int valid) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n * n; e += gridDim.x * blockDim.x) {
        const int i = e / n, j = e % n;
        P[e] = (i < valid && j < valid) ? D[e] : (i == j ? 1.0 : 0.0);
    }
}

hs_status launch_diag_inverses(hs_ctx ctx, const double* L, double* Y, double* pad, cudaStream_t s) {
    // Y_k = L_kk^-T for every diagonal block: the substitution kernel on identity blocks,
    // every item against its own triangle; the last block, when it has padding rows,
    // against a copy with a unit diagonal there (its padding rows are never used)
    hs_status st = set_attrs();
    if (st != HS_OK) return st;
    const int n = ctx->bsz, nb = ctx->nb;
    const int64_t bb = (int64_t)n * n;
    const int valid = (int)(ctx->N - (int64_t)(nb - 1) * n);
    ctx->launches += 1;
    identity_blocks_kernel<<<4 * ctx->num_sms, 256, 0, s>>>(Y, n, nb);
    HS_CHECK_LAUNCH("identity blocks");
    const int full = valid < n ? nb - 1 : nb;
    if (full > 0) {
        TrsmArgs ta{L, n, n, Y, n, 0, (n + kTrsmRows - 1) / kTrsmRows, n, bb, nb};
        if ((st = launch_trsm_args(ctx, ta, full, s)) != HS_OK) return st;
    }
    if (full < nb) {
        ctx->launches += 1;
        pad_unit_block_kernel<<<64, 256, 0, s>>>(L + (size_t)column_start(nb - 1, nb) * bb, pad, n, valid);
        HS_CHECK_LAUNCH("pad block");
        TrsmArgs ta{pad, n, n, Y + (size_t)(nb - 1) * bb, n, 0, (n + kTrsmRows - 1) / kTrsmRows, n, bb, 0};
        if ((st = launch_trsm_args(ctx, ta, 1, s)) != HS_OK) return st;
    }
    return HS_OK;
}

hs_status launch_trsm_dmma(hs_ctx ctx, double* A, int64_t firstBlock, int blockCount, const double* X,
                           cudaStream_t s) {
    if (blockCount <= 0) return HS_OK;
    hs_status st = set_attrs();
    if (st != HS_OK) return st;
    const int bsz = ctx->bsz;
    HS_REQUIRE(bsz == 128 || bsz == 256, "the tensor-core TRSM needs matrixBlockSize 128 or 256");
    const double n = bsz;
    prof_begin(ctx, s, HS_KERNEL_TRSM);
    ctx->launches += 1;
    const unsigned grid = (unsigned)((int64_t)blockCount * (bsz / 64));
    if (bsz == 256)
        trsm_dmma_kernel<256><<<grid, 256, TrsmTile<256>::T::kSmem, s>>>(A, firstBlock, X);
    else
        trsm_dmma_kernel<128><<<grid, 256, TrsmTile<128>::T::kSmem, s>>>(A, firstBlock, X);
    HS_CHECK_LAUNCH("trsm_dmma");
    // algorithmic work: the triangular solve's n^3 flops a block
    prof_end(ctx, s, HS_KERNEL_TRSM, blockCount * n * n * n, (2.0 * blockCount + 1.0) * n * n * 8.0);
    return HS_OK;
}

hs_status launch_trsm(hs_ctx ctx, double* A, int blockID, int blockRow, int blockStart, int blockCount,
                      cudaStream_t s) {
    if (blockCount <= 0) return HS_OK;
    hs_status st = set_attrs();
    if (st != HS_OK) return st;
    const int bsz = ctx->bsz;
    HS_REQUIRE(bsz <= 256, "TRSM supports matrixBlockSize up to 256");
    const size_t bb = (size_t)bsz * bsz;
    if (bsz == 128 || bsz == 256) {
        // on the FP64 tensor pipe: X = L_kk^-1 once, then B <- B X^T block by block
        st = ensure_scratch(ctx, kSmallScratch + 2 * bb * sizeof(double));
        if (st != HS_OK) return st;
        double* Y = reinterpret_cast<double*>(static_cast<char*>(ctx->scratch) + kSmallScratch);
        double* X = Y + bb;
        st = launch_diag_inverse(ctx, A + (size_t)blockID * bb, Y, X, s);
        if (st != HS_OK) return st;
        return launch_trsm_dmma(ctx, A, (int64_t)blockID + (blockStart - blockRow), blockCount, X, s);
    }
    TrsmArgs ta{A + (size_t)blockID * bb, bsz, bsz, A, bsz, (int64_t)blockID + (blockStart - blockRow),
                (bsz + kTrsmRows - 1) / kTrsmRows, bsz, (int64_t)bb};
    const double n = bsz;
    prof_begin(ctx, s, HS_KERNEL_TRSM);
    st = launch_trsm_args(ctx, ta, blockCount, s);
    prof_end(ctx, s, HS_KERNEL_TRSM, blockCount * n * n * n, (2.0 * blockCount + 1.0) * n * n * 8.0);
    return st;
}

hs_status launch_trsm_on(hs_ctx ctx, const double* L, int n, double* B, int items, cudaStream_t s) {
    hs_status st = set_attrs();
    if (st != HS_OK) return st;
    TrsmArgs ta{L, n, n, B, n, 0, (n + kTrsmRows - 1) / kTrsmRows, n, (int64_t)n * n};
    return launch_trsm_args(ctx, ta, items, s);
}

namespace {

// launches the update of `a` (totalPairs set) with its algorithmic flops / bytes
hs_status run_update(hs_ctx ctx, UpdateArgs& a, double flops, double bytes, cudaStream_t s) {
    if (a.totalPairs <= 0) return HS_OK;
    const bool dmma = ctx->bsz % kUTM == 0;
    a.tilesM = dmma ? ctx->bsz / kUTM : 1;
    a.tilesN = dmma ? ctx->bsz / kUTN : 1;
    const int64_t grid = a.totalPairs * a.tilesM * a.tilesN;
    HS_REQUIRE(grid < (1LL << 31), "trailing update too large for one launch");
    prof_begin(ctx, s, HS_KERNEL_UPDATE);
    ctx->launches += 1;
    if (dmma) {
        update_dmma_kernel<<<(unsigned)grid, UTile::kThreads, UTile::kSmem, s>>>(a);
        HS_CHECK_LAUNCH("update_dmma");
    } else {
        const int64_t bb = (int64_t)ctx->bsz * ctx->bsz;
        const int64_t total = a.totalPairs;
        dim3 g((unsigned)((bb + 255) / 256), (unsigned)(total < 65535 ? total : 65535),
               (unsigned)((total + 65534) / 65535));
        update_scalar_kernel<<<g, 256, 0, s>>>(a);
        HS_CHECK_LAUNCH("update_scalar");
    }
    prof_end(ctx, s, HS_KERNEL_UPDATE, flops, bytes);
    return HS_OK;
}

}  // namespace

hs_status launch_update(hs_ctx ctx, double* A, int blockID, int blockRow, int syrkStart, int syrkCount,
                        int gemmStart, int gemmCount, cudaStream_t s) {
    hs_status st = set_attrs();
    if (st != HS_OK) return st;
    UpdateArgs a{};
    a.A = A;
    a.blockID = blockID;
    a.blockRow = blockRow;
    a.nb = ctx->nb;
    a.bsz = ctx->bsz;
    a.rowMode = 1;
    int64_t pairs = 0;
    if (gemmCount > 0) {
        // rows r' = r - blockRow - 1 in [g0, g0 + gemmCount) own r' pairs each
        const int64_t g0 = gemmStart - blockRow - 1;
        const int64_t g1 = g0 + gemmCount;
        a.pairBase = g0 * (g0 - 1) / 2;
        pairs = g1 * (g1 - 1) / 2 - a.pairBase;
    }
    a.gemmPairs = pairs;
    a.syrkStart = syrkStart;
    const int64_t syrkN = syrkCount > 0 ? syrkCount : 0;
    a.totalPairs = pairs + syrkN;
    // algorithmic work: 2 bsz^3 per GEMM pair, bsz^2 (bsz + 1) per SYRK block;
    // bytes: read + write of every output block plus the panel column once
    const double n = ctx->bsz;
    const double flops = (double)pairs * 2.0 * n * n * n + (double)syrkN * n * n * (n + 1.0);
    const int64_t panel = (gemmCount > 0 ? gemmCount + 1 : 0) > syrkN ? (gemmCount + 1) : syrkN;
    const double bytes = ((double)pairs * 2.0 + (double)syrkN * 2.0 + (double)panel) * n * n * 8.0;
    return run_update(ctx, a, flops, bytes, s);
}

hs_status launch_update_cols(hs_ctx ctx, double* A, int blockID, int blockRow, int colStart, int colEnd,
                             cudaStream_t s) {
    hs_status st = set_attrs();
    if (st != HS_OK) return st;
    const int nb = ctx->nb;
    HS_REQUIRE(blockRow < colStart && colStart <= colEnd && colEnd <= nb, "columns outside the trailing matrix");
    UpdateArgs a{};
    a.A = A;
    a.blockID = blockID;
    a.blockRow = blockRow;
    a.nb = nb;
    a.bsz = ctx->bsz;
    a.rowMode = 0;
    a.colStart = colStart;
    a.colEnd = colEnd;
    int64_t pairs = 0;
    for (int c = colStart; c < colEnd; ++c) pairs += nb - c;
    a.totalPairs = pairs;
    const double n = ctx->bsz;
    const int64_t syrkN = colEnd - colStart;
    const double flops = (double)(pairs - syrkN) * 2.0 * n * n * n + (double)syrkN * n * n * (n + 1.0);
    const double bytes = ((double)pairs * 2.0 + (double)(nb - colStart)) * n * n * 8.0;
    return run_update(ctx, a, flops, bytes, s);
}

}  // namespace hs
