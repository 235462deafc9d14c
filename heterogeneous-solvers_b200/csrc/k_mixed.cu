// k_mixed.cu — mixed-precision blocked Cholesky: FP32 factor whose panel TRSM
// and SYRK/GEMM trailing updates run on the 5th-generation tensor cores
// (tcgen05, kind::tf32) as 3xTF32 split products with FP32 accumulation in
// TMEM, while every diagonal-block POTRF runs in FP64.
//
// No reference counterpart (the reference factors in FP64 or FP32 only,
// src/utility/Configuration.hpp:14-19); the block structure is the reference's
// right-looking algorithm (src/solver/cholesky/Cholesky.cpp:446-471).
//
// Split products: an FP32 operand a is read by the tensor core as TF32
// (its top 19 bits), a_hi; a_lo = a - a_hi is exact in FP32 and kept in a
// second buffer.  a*b ~ a_hi*b_hi + a_hi*b_lo + a_lo*b_hi: three MMAs per
// k-step, accumulated in FP32, relative error ~2^-21 instead of TF32's 2^-11.
// The trailing update can instead take 16-bit splits of the factored panel on
// tcgen05 kind::f16 at twice the rate: BF16 (hi = bf16(a), lo = bf16(a - hi),
// ~2^-16) or FP16 of the panel scaled by a power of two s (hi = fp16(s a),
// lo = fp16(s a - hi), ~2^-22), the accumulator being multiplied by s^-2.
//
// Panel TRSM kernel (one 128 x bsz output tile per CTA, 4 warps):
//   thread 0   TMA producer: A_hi, A_lo (128 x 32 FP32) and B_hi, B_lo
//              (rows 32 kc .. bsz-1 x 32 FP32 of K slab kc: B = L_kk^-1 is lower
//              triangular) per K slab, 128-byte swizzle, 2-stage ring
//   thread 32  MMA issuer: 3 x 4 tcgen05.mma (K = 8 each, N = bsz - 32 kc) per
//              slab, commit to the stage's "empty" barrier and finally to "done"
//   all warps  epilogue: TMEM -> registers (warp w owns lanes 32w..32w+31 =
//              tile rows), L = D and L_lo = D - tf32(D) or L's 16-bit split
// The trailing update is the persistent tc_update_kernel further down.
// Every mbarrier wait is bounded (2 s); on expiry the CTA records an error in
// the context's flag word, frees its TMEM and returns.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cudaTypedefs.h>

#include <cmath>

#include "hs_internal.cuh"
#include "hs_mixed.cuh"
#include "tc_common.cuh"

namespace hs {
namespace {

using namespace tc;

constexpr int kTcThreads = 128;
constexpr int kSlab = 32;               // K elements (FP32) per stage = 128 bytes
constexpr uint64_t kWaitNs = 2000000000ull;

enum { MODE_TRSM = 1 };  // the tile kernel's one mode, the panel TRSM

struct TcArgs {
    float* A32;        // packed FP32 working matrix
    float* LO;         // FP32 low parts of panel blocks and of L_kk^-T (slots below)
    int64_t blockID;   // id of the diagonal block of column k
    int k, nb;
    int* err;          // error flag (timeouts)
    // persistent update: 0 columns first_col.., 1 column first_col only, 2 columns
    // first_col+1.., 3 columns first_col .. first_col + ncols - 1
    int part, ncols;
    // panel p of the update sits in slot set set0 + p (sets 0..kPanelGroup-1 and
    // kPanelGroup..2 kPanelGroup-1 are the two banks of a group look-ahead)
    int set0;
    // non-null: the update's CTAs take tiles from this counter (zero before the
    // first launch that uses it), so that a second launch can share the tiles of
    // the first; null: CTA i takes tiles i, i + grid, ...
    unsigned long long* tile_ctr;
    const long long* abort_flag;  // smallest failing pivot row so far (INT64_MAX: none)
    // slots (bsz x bsz blocks): FP32 low parts of panel k in LO from lo_base (row r at
    // lo_base + r - k - 1), L_kk^-1 hi / lo at LO[inv], LO[inv + 1]
    int lo_base, inv;
    // persistent update with the npanels (1..kPanelGroup) consecutive panel columns
    // k + p, updating the trailing columns from first_col on.  Panel p keeps its FP32
    // low parts from LO slot (set0 + p) nb and its 16-bit split from P16 slot
    // 2 (set0 + p) nb (hi of row r at 2 (set0 + p) nb + r - (k + p) - 1, lo nb slots
    // further)
    int npanels;
    // panels summed in one TMEM accumulation before the add into C (1, 2 or
    // kPanelGroup; the last unit of a tile takes what is left of its npanels): fewer
    // panels a unit is a more accurate factor, more adds into C
    int unit_panels;
    int first_col;
    // TRSM with 16-bit split products downstream (split16 = HS_PRECISION_BF16X3 or
    // HS_PRECISION_F16X3; 0: none): the epilogue writes L's hi / lo split (P16 slots
    // 2 lo_base + r - k - 1 and nb further) instead of its TF32 low part.  The FP16
    // split is of f16_scale L (a power of two); the update multiplies its FP32
    // accumulator by f16_unscale = f16_scale^-2 (exact).
    __nv_bfloat16* P16;  // 16-bit storage: BF16 or FP16 values
    int split16;
    float f16_scale, f16_unscale;
};

// CTA-uniform early exit once a diagonal POTRF has recorded a non-positive pivot:
// the factor will be discarded, so the remaining tensor-core work is skipped.  The
// decision is taken by thread 0 and shared before any barrier or TMEM use, because
// the look-ahead POTRF may record a pivot while this kernel runs.
__device__ __forceinline__ bool factor_aborted(const long long* flag) {
    __shared__ int s_abort;
    if (threadIdx.x == 0) s_abort = (*reinterpret_cast<const volatile long long*>(flag) != INT64_MAX) ? 1 : 0;
    __syncthreads();
    return s_abort != 0;
}

template <int BSZ>
struct TcSmem {
    static constexpr int kTiles = BSZ / 128;               // 128-row tiles per block
    static constexpr int kABytes = 128 * kSlab * 4;        // 16 KB
    static constexpr int kBBytes = BSZ * kSlab * 4;        // 16 / 32 KB
    static constexpr int kStage = 2 * kABytes + 2 * kBBytes;
    static constexpr int kRowBox = 32 * kSlab * 4;         // 32 rows of B: 4 KB
    static constexpr int kStages = 2;
    static constexpr int kBytes = kStages * kStage + 1024 /* barriers, slot */ + 1024 /* alignment */;
};

template <int BSZ, int MODE>
__global__ void __launch_bounds__(kTcThreads, 1)
    tc_tile_kernel(const __grid_constant__ CUtensorMap mA128, const __grid_constant__ CUtensorMap mL128,
                   const __grid_constant__ CUtensorMap mL32, TcArgs a) {
    using SM = TcSmem<BSZ>;
    if (factor_aborted(a.abort_flag)) return;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + SM::kStages * SM::kStage);
    uint64_t* empty = full + SM::kStages;
    uint64_t* done = empty + SM::kStages;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
    __shared__ int s_fail;  // a wait of the producer or the MMA issuer ran out

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const size_t bb = (size_t)BSZ * BSZ;

    // ---- tile decode
    const int ti = (int)(blockIdx.x % SM::kTiles);
    const int64_t item = blockIdx.x / SM::kTiles;
    static_assert(MODE == MODE_TRSM, "the tile kernel runs the panel TRSM only");
    const int r = a.k + 1 + (int)item;  // block row of the panel (column k)
    // operand coordinates: (column, row, block) in the TMA maps
    const int blkA = (int)(a.blockID + (r - a.k));  // panel block of row r
    const int gA = a.lo_base + r - a.k - 1;         // its low-part slot
    const int blkB = a.inv, gB = a.inv + 1;         // L_kk^-T hi / lo

    if (tid == 0) {
        for (int s = 0; s < SM::kStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(done, 1);
        fence_barrier_init();
        s_fail = 0;
    }
    if (warp == 0) {
        tmem_alloc(tslot, BSZ);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t taddr = *tslot;
    const uint64_t deadline = globaltimer_ns() + kWaitNs;
    bool ok = true;
    constexpr int kSlabs = BSZ / kSlab;

    if (tid == 0) {
        // ---- producer.  L_kk^-1 is lower triangular: the rows of B (= output
        // columns) before 32 kc are zero in K slab kc, so only rows 32 kc .. BSZ - 1
        // of the slab are loaded (32-row boxes, at their place in the stage)
        constexpr int kRowBoxes = BSZ / 32;
        int issued = 0;
        for (int kc = 0; kc < kSlabs && ok; ++kc) {
            const int s = kc % SM::kStages, use = kc / SM::kStages;
            if (use > 0 && !mbar_wait(&empty[s], (use - 1) & 1, deadline)) { ok = false; break; }
            uint8_t* st = smem + s * SM::kStage;
            mbar_arrive_expect_tx(&full[s], 2 * SM::kABytes + 2 * (kRowBoxes - kc) * SM::kRowBox);
            tma_load_3d(st, &mA128, &full[s], kc * kSlab, ti * 128, blkA);
            tma_load_3d(st + SM::kABytes, &mL128, &full[s], kc * kSlab, ti * 128, gA);
            for (int rb = kc; rb < kRowBoxes; ++rb) {
                tma_load_3d(st + 2 * SM::kABytes + rb * SM::kRowBox, &mL32, &full[s], kc * kSlab, 32 * rb, blkB);
                tma_load_3d(st + 2 * SM::kABytes + SM::kBBytes + rb * SM::kRowBox, &mL32, &full[s], kc * kSlab,
                            32 * rb, gB);
            }
            ++issued;
        }
        if (!ok) {
            s_fail = 1;
            atomicExch(a.err, 1);
        }
        // no load may still be writing into shared memory when the CTA leaves: wait
        // (bounded) for the phase each stage was last armed with (a completed phase
        // passes at once)
        for (int kc = issued > SM::kStages ? issued - SM::kStages : 0; kc < issued; ++kc)
            if (!mbar_wait_for(&full[kc % SM::kStages], (kc / SM::kStages) & 1, kWaitNs)) atomicExch(a.err, 1);
    } else if (tid == 32) {
        // ---- MMA issuer: slab kc adds into output columns 32 kc .. BSZ - 1 only
        // (N = BSZ - 32 kc; the columns before it would get exact zeros from this slab)
        for (int kc = 0; kc < kSlabs; ++kc) {
            const int s = kc % SM::kStages, use = kc / SM::kStages;
            if (!mbar_wait(&full[s], use & 1, deadline)) { ok = false; break; }
            tc_fence_after();
            const uint32_t idesc = umma_idesc(kFmtTF32, kFmtTF32, 128, BSZ - 32 * kc);
            const uint32_t base = smem_u32(smem + s * SM::kStage);
            const uint32_t aHi = base, aLo = base + SM::kABytes;
            const uint32_t bHi = base + 2 * SM::kABytes + kc * SM::kRowBox, bLo = bHi + SM::kBBytes;
            const uint32_t dcol = taddr + (uint32_t)(32 * kc);
#pragma unroll
            for (int ks = 0; ks < kSlab / 8; ++ks) {
                const uint32_t off = ks * 32;  // 8 TF32 = 32 bytes along K
                const uint64_t dAh = umma_desc_sw128(aHi + off), dAl = umma_desc_sw128(aLo + off);
                const uint64_t dBh = umma_desc_sw128(bHi + off), dBl = umma_desc_sw128(bLo + off);
                umma_tf32(dcol, dAh, dBh, idesc, (kc | ks) != 0);
                umma_tf32(dcol, dAh, dBl, idesc, 1);
                umma_tf32(dcol, dAl, dBh, idesc, 1);
            }
            umma_commit(&empty[s]);
        }
        if (!ok) {
            s_fail = 1;
            atomicExch(a.err, 1);
        }
        // "done" arrives once every MMA this thread issued has completed, also after a
        // wait ran out: TMEM is released only after that
        umma_commit(done);
    }
    __syncthreads();  // the roles have issued all their work; s_fail is final

    // ---- epilogue: all 4 warps, thread = tile row
    int wok = 0;
    if (lane == 0) wok = mbar_wait_for(done, 0, kWaitNs) ? 1 : 0;
    const bool done_ok = __shfl_sync(0xffffffffu, wok, 0) != 0;
    __syncwarp();
    tc_fence_after();
    if (!done_ok || s_fail) {
        if (lane == 0) atomicExch(a.err, 1);
    } else {
#pragma unroll 1
        for (int j = 0; j < BSZ / 32; ++j) {
            uint32_t v[32];
            tmem_ld_32x32b_x32(taddr + ((uint32_t)(warp * 32) << 16) + j * 32, v);
            tmem_ld_wait();
            // staged through this warp's 32 x 33 shared tile (the operand ring is
            // free once the MMAs are done), then written as whole 128-byte row
            // segments: 8 lanes a row, 4 rows an instruction
            float* stg = reinterpret_cast<float*>(smem) + warp * 32 * 33;
#pragma unroll
            for (int q = 0; q < 32; ++q) stg[lane * 33 + q] = __uint_as_float(v[q]);
            __syncwarp();
            const int c4 = (lane & 7) * 4;
#pragma unroll 2
            for (int it = 0; it < 8; ++it) {
                const int rr = it * 4 + (lane >> 3);
                const float* sr = stg + rr * 33 + c4;
                const float x0 = sr[0], x1 = sr[1], x2 = sr[2], x3 = sr[3];
                const size_t off = (size_t)(ti * 128 + warp * 32 + rr) * BSZ + j * 32 + c4;
                *reinterpret_cast<float4*>(a.A32 + (size_t)blkA * bb + off) = make_float4(x0, x1, x2, x3);
                if (a.split16 == HS_PRECISION_F16X3) {
                    const float sc = a.f16_scale;
                    const float y0 = x0 * sc, y1 = x1 * sc, y2 = x2 * sc, y3 = x3 * sc;
                    const __half2 h01 = __floats2half2_rn(y0, y1), h23 = __floats2half2_rn(y2, y3);
                    const float2 f01 = __half22float2(h01), f23 = __half22float2(h23);
                    const __half2 l01 = __floats2half2_rn(y0 - f01.x, y1 - f01.y);
                    const __half2 l23 = __floats2half2_rn(y2 - f23.x, y3 - f23.y);
                    __half* ph =
                        reinterpret_cast<__half*>(a.P16) + (size_t)(2 * a.lo_base + (r - a.k - 1)) * bb + off;
                    __half2* h2 = reinterpret_cast<__half2*>(ph);
                    __half2* l2 = reinterpret_cast<__half2*>(ph + (size_t)a.nb * bb);
                    h2[0] = h01;
                    h2[1] = h23;
                    l2[0] = l01;
                    l2[1] = l23;
                } else if (a.split16 == HS_PRECISION_BF16X3) {
                    const __nv_bfloat162 h01 = __floats2bfloat162_rn(x0, x1), h23 = __floats2bfloat162_rn(x2, x3);
                    const float2 f01 = __bfloat1622float2(h01), f23 = __bfloat1622float2(h23);
                    const __nv_bfloat162 l01 = __floats2bfloat162_rn(x0 - f01.x, x1 - f01.y);
                    const __nv_bfloat162 l23 = __floats2bfloat162_rn(x2 - f23.x, x3 - f23.y);
                    __nv_bfloat16* ph = a.P16 + (size_t)(2 * a.lo_base + (r - a.k - 1)) * bb + off;
                    __nv_bfloat162* h2 = reinterpret_cast<__nv_bfloat162*>(ph);
                    __nv_bfloat162* l2 = reinterpret_cast<__nv_bfloat162*>(ph + (size_t)a.nb * bb);
                    h2[0] = h01;
                    h2[1] = h23;
                    l2[0] = l01;
                    l2[1] = l23;
                } else {
                    *reinterpret_cast<float4*>(a.LO + (size_t)gA * bb + off) =
                        make_float4(x0 - tf32_trunc(x0), x1 - tf32_trunc(x1), x2 - tf32_trunc(x2),
                                    x3 - tf32_trunc(x3));
                }
            }
            __syncwarp();
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(taddr, BSZ);
}

// ------------------------------------------------------------------ persistent trailing update
// The trailing update of block column k as one persistent launch: one CTA per
// SM walks the 128 x BSZ output tiles in a grouped order (vertical strips of
// kGroup block rows, column by column), so that the CTAs running at the same
// time share panel blocks through L2.  Warp roles:
//   warp 0 (one thread)  TMA producer: A_hi/A_lo/B_hi/B_lo slabs of kUpdK
//                        K-columns into a ring of stages, plus an L2 prefetch of
//                        the tile's C rows
//   warp 1 (one thread)  MMA issuer: kUpdK/8 x 3 tcgen05.mma per slab (hi*hi, hi*lo,
//                        lo*hi) into one of two TMEM accumulators (2 x BSZ
//                        columns), one accumulation a (tile, panel) unit, so that
//                        the epilogue of a unit overlaps the MMAs of the next
//   warps 2-9            epilogue: TMEM -> registers -> -D in a swizzled shared
//                        tile -> TMA reduce-add into C (two warps per TMEM lane
//                        quarter, half the columns each), then free the
//                        accumulator (one arrival per warp)
// (Forming the low parts in shared memory instead of loading them halves the
// L2 traffic but adds shared-memory traffic on the port the tensor core reads
// its operands through; measured slower.  Strips of 16 block rows were ~1.5 %
// faster than 8 at N=131072, strips of 32 ~8 % slower.)
constexpr int kGroup = 16;
constexpr int kUpdThreads = 320;
// K floats per stage: 32 (128-byte rows, 128-byte swizzle, 2 stages of 96 KB)
// measured faster than 16 (64-byte swizzle, 4 stages of 48 KB); the kernel is
// limited by the shared-memory traffic of TMA writes plus the tensor core's
// operand reads, not by the depth of the ring
constexpr int kUpdK = 32;
// panels per pass of the trailing update over C.  (8 and 16 cut the BF16 update by
// 3 % at N=131072 but left the factor less accurate — the unrefined backward error
// 4.3e-9 -> 6.8e-9, 10 -> 11 -> 12 CG iterations on the same right-hand side,
// plausibly from the longer FP32 accumulation chains in TMEM before each
// round-to-nearest add into C — and the solve no faster.)
constexpr int kPanelGroup = 4;
// panel slot sets: two banks of kPanelGroup, so that the next group's panels can be
// factored while the trailing update still reads the current group's
constexpr int kSets = 2 * kPanelGroup;
// tile counters of one factor: one per look-ahead by a group (a shared update)
__host__ __device__ constexpr int64_t tile_counters(int64_t nb) { return nb / kPanelGroup + 2; }
constexpr uint64_t kStepWaitNs = 2000000000ull;

// operand formats of the update: TF32 (FP32 storage, hi = the FP32 value as
// read by the tensor core, lo = x - tf32(x)), BF16 (hi = bf16(x), lo =
// bf16(x - hi)) or FP16 of the scaled panel (hi = fp16(s x), lo = fp16(s x - hi));
// all give 128-byte operand rows per slab and 32-byte K steps
template <int PREC>
struct UpdFmt;
template <>
struct UpdFmt<HS_PRECISION_TF32X3> {
    static constexpr int kK = kUpdK, kKStep = 8, kFmt = kFmtTF32;
};
template <>
struct UpdFmt<HS_PRECISION_BF16X3> {
    static constexpr int kK = 2 * kUpdK, kKStep = 16, kFmt = kFmtBF16;
};
template <>
struct UpdFmt<HS_PRECISION_F16X3> {
    static constexpr int kK = 2 * kUpdK, kKStep = 16, kFmt = kFmtF16;
};

template <int BSZ>
struct UpdSmem {
    static constexpr int kA = 128 * kUpdK * 4;       // 8 KB per 16 K-columns of FP32
    static constexpr int kB = BSZ * kUpdK * 4;       // 16 / 8 KB
    static constexpr int kRaw = kA + kB;             // one of hi / lo
    static constexpr int kStage = 2 * kRaw;          // A_hi, B_hi, A_lo, B_lo (TMA bytes per stage)
    static constexpr int kStages = kUpdK == 32 ? 2 : 4;
    static constexpr int kStaging = 8 * 32 * 32 * 4;  // one 32x32 FP32 tile per epilogue warp
    static constexpr int kBytes = kStages * kStage + kStaging + 256 /* barriers, slot */ + 1024 /* alignment */;
};

__device__ __forceinline__ uint64_t upd_desc(uint32_t addr) {
    return kUpdK == 32 ? umma_desc_sw128(addr) : umma_desc_sw64(addr);
}

__host__ __device__ __forceinline__ int64_t tri64(int64_t n) { return n * (n + 1) / 2; }

// Tile hand-off inside a CTA of the persistent update.  The producer takes the
// CTA's j-th tile (from the shared counter, or by stride) and publishes it in slot
// j % kRing as ((j + 1) << 32) | tile with a release store (kNoTile: no tiles
// left); the MMA issuer and the epilogue warps read it with acquire loads.  A slot
// is rewritten only after every reader is past its previous tile: the producer
// publishes tile j after the empty-barrier waits of tile j - 1, so the issuer has
// consumed every slab of tile j - 2 (a tile has >= kStages slabs), and before it
// began tile j - 2 the epilogue had released the accumulator of tile j - 4.
constexpr int kRing = 8;
constexpr uint32_t kNoTile = 0xffffffffu;

__device__ __forceinline__ void ring_publish(uint64_t* slot, uint32_t j, uint32_t tile) {
    const uint64_t v = ((uint64_t)(j + 1) << 32) | tile;
    asm volatile("st.release.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(slot)), "l"(v) : "memory");
}

// tile j of this CTA; kNoTile when none is left, or when the wait ran out (then
// *ok = false)
__device__ __forceinline__ uint32_t ring_take(const uint64_t* slot, uint32_t j, uint64_t timeout_ns, bool* ok) {
    const uint64_t want = (uint64_t)j + 1;
    uint64_t deadline = 0;
    for (;;) {
        uint64_t v;
        asm volatile("ld.acquire.cta.shared::cta.b64 %0, [%1];" : "=l"(v) : "r"(smem_u32(slot)) : "memory");
        if ((v >> 32) == want) return (uint32_t)v;
        if ((v >> 32) > want) break;  // overwritten before it was read: cannot happen (see above)
        const uint64_t now = globaltimer_ns();
        if (deadline == 0)
            deadline = now + timeout_ns;
        else if (now > deadline)
            break;
    }
    *ok = false;
    return kNoTile;
}

// tiles of the persistent update (128 x BSZ each, BSZ / 128 per block) for a part
__host__ __device__ __forceinline__ int64_t update_tiles(int part, int m, int ncols, int tiles_per_block) {
    int64_t blocks;
    if (part == 1)
        blocks = m;
    else if (part == 3)
        blocks = (int64_t)ncols * m - (int64_t)ncols * (ncols - 1) / 2;
    else
        blocks = tri64(part == 2 ? m - 1 : m);
    return blocks * tiles_per_block;
}

// pair p of the grouped enumeration of the m x m lower triangle -> (r', c')
__device__ __forceinline__ void grouped_pair(int64_t p, int m, int* rr, int* cc) {
    int lo = 0, hi = (m + kGroup - 1) / kGroup;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (tri64((int64_t)mid * kGroup) <= p) lo = mid; else hi = mid - 1;
    }
    const int r0 = lo * kGroup;
    const int r1 = min(r0 + kGroup, m), h = r1 - r0;
    int64_t l = p - tri64(r0);
    if (l < (int64_t)r0 * h) {
        *rr = r0 + (int)(l % h);
        *cc = (int)(l / h);
        return;
    }
    l -= (int64_t)r0 * h;
    int j = 0;
    while (l >= h - j) {
        l -= h - j;
        ++j;
    }
    *rr = r0 + j + (int)l;
    *cc = r0 + j;
}

// mU*: maps of the hi parts, mV*: of the lo parts (*128: 128-row boxes, *B: BSZ-row boxes)
template <int BSZ, int PREC>
__global__ void __launch_bounds__(kUpdThreads, 1)
    tc_update_kernel(const __grid_constant__ CUtensorMap mU128, const __grid_constant__ CUtensorMap mUB,
                     const __grid_constant__ CUtensorMap mV128, const __grid_constant__ CUtensorMap mVB,
                     const __grid_constant__ CUtensorMap mC32, TcArgs a) {
    using SM = UpdSmem<BSZ>;
    using F = UpdFmt<PREC>;
    if (factor_aborted(a.abort_flag)) return;
    constexpr int kTiles = BSZ / 128;
    constexpr int kSlabsP = BSZ / F::kK;  // slabs per panel
    static_assert(kSlabsP >= SM::kStages, "a tile needs at least kStages slabs (tile hand-off)");
    const int kSlabs = a.npanels * kSlabsP;
    constexpr uint32_t kAccCols = 2 * BSZ;  // two accumulators
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* staging = smem + SM::kStages * SM::kStage;  // 1024-aligned: the stage size is
    uint64_t* full = reinterpret_cast<uint64_t*>(staging + SM::kStaging);
    uint64_t* empty = full + SM::kStages;
    uint64_t* tfull = empty + SM::kStages;
    uint64_t* tempty = tfull + 2;
    uint64_t* drained = tempty + 2;  // every MMA of the issuer has completed
    uint32_t* tslot = reinterpret_cast<uint32_t*>(drained + 1);
    uint64_t* ring = drained + 2;    // kRing tile slots (after tslot's 8 bytes)

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m = a.nb - a.first_col;
    // part 1: the m blocks of column first_col; part 2: the lower triangle of the
    // columns after it; part 0: both (the m x m lower triangle from first_col on);
    // part 3: the blocks of columns first_col .. first_col + ncols - 1
    const int mt = a.part == 2 ? m - 1 : m;
    const int64_t ntiles = update_tiles(a.part, m, a.ncols, kTiles);

    if (tid == 0) {
        for (int s = 0; s < SM::kStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], 8);
        }
        mbar_init(drained, 1);
        for (int i = 0; i < kRing; ++i) ring[i] = 0;
        fence_barrier_init();
    }
    if (warp == 0) {
        tmem_alloc(tslot, kAccCols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t taddr = *tslot;
    bool ok = true;

    auto decode = [&](int64_t t, int* r, int* c, int* ti) {
        *ti = (int)(t % kTiles);
        const int64_t p = t / kTiles;
        if (a.part == 1) {
            *r = a.first_col + (int)p;
            *c = a.first_col;
            return;
        }
        if (a.part == 3) {  // column j of the part holds m - j blocks
            int j = 0;
            int64_t q = p;
            while (j + 1 < a.ncols && q >= m - j) {
                q -= m - j;
                ++j;
            }
            *r = a.first_col + j + (int)q;
            *c = a.first_col + j;
            return;
        }
        int rr, cc;
        grouped_pair(p, mt, &rr, &cc);
        const int base = a.first_col + (a.part == 2 ? 1 : 0);
        *r = base + rr;
        *c = base + cc;
    };

    if (warp == 0) {
        if (lane == 0) {
            // ---- producer
            uint32_t g = 0;
            for (uint32_t j = 0;; ++j) {
                int64_t t = kNoTile;
                if (ok) {
                    t = a.tile_ctr ? (int64_t)atomicAdd(a.tile_ctr, 1ull) : blockIdx.x + (int64_t)j * gridDim.x;
                    if (t >= ntiles) t = kNoTile;
                }
                ring_publish(&ring[j % kRing], j, (uint32_t)t);
                if (t == kNoTile) break;
                int r, c, ti;
                decode(t, &r, &c, &ti);
                // the tile's 128 rows of C are contiguous: bring them into L2 now, so
                // the epilogue's reduce-add finds its lines there
                prefetch_l2(a.A32 + (size_t)block_id(r, c, a.nb) * BSZ * BSZ + (size_t)ti * 128 * BSZ,
                            128 * BSZ * 4);
                const bool bf = PREC != HS_PRECISION_TF32X3;  // 16-bit split slots in P16
                for (int kc = 0; kc < kSlabs; ++kc, ++g) {
                    const uint32_t s = g % SM::kStages, use = g / SM::kStages;
                    if (use > 0 && !mbar_wait_for(&empty[s], (use - 1) & 1, kStepWaitNs)) {
                        ok = false;
                        break;
                    }
                    // panel pi = column k + pi: TF32 hi = its FP32 block in A32, lo = its
                    // LO slot; BF16 / FP16 hi / lo = its split slots in P16
                    const int pi = kc / kSlabsP, kk = kc % kSlabsP;
                    const int colp = a.k + pi;
                    const int gA = r - colp - 1, gB = c - colp - 1;
                    const int64_t dblk = block_id(colp, colp, a.nb);
                    const int lob = (a.set0 + pi) * a.nb, pb = 2 * (a.set0 + pi) * a.nb;
                    const int hiA = bf ? pb + gA : (int)(dblk + (r - colp));
                    const int loA = bf ? pb + a.nb + gA : lob + gA;
                    const int hiB = bf ? pb + gB : (int)(dblk + (c - colp));
                    const int loB = bf ? pb + a.nb + gB : lob + gB;
                    uint8_t* st = smem + s * SM::kStage;
                    mbar_arrive_expect_tx(&full[s], SM::kStage);
                    tma_load_3d(st, &mU128, &full[s], kk * F::kK, ti * 128, hiA);
                    tma_load_3d(st + SM::kA, &mUB, &full[s], kk * F::kK, 0, hiB);
                    tma_load_3d(st + SM::kRaw, &mV128, &full[s], kk * F::kK, ti * 128, loA);
                    tma_load_3d(st + SM::kRaw + SM::kA, &mVB, &full[s], kk * F::kK, 0, loB);
                }
            }
            if (!ok) atomicExch(a.err, 1);
            // no load may still be writing into shared memory when the CTA leaves: wait
            // (bounded) for the phase each stage was last armed with (slabs g - kStages ..
            // g - 1; a completed phase passes at once)
            for (uint32_t h = g > (uint32_t)SM::kStages ? g - SM::kStages : 0; h < g; ++h)
                if (!mbar_wait_for(&full[h % SM::kStages], (h / SM::kStages) & 1, kStepWaitNs)) atomicExch(a.err, 1);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // ---- MMA issuer
            // one accumulation unit = one tile x unit_panels panels: with unit_panels = 1
            // each panel's product is accumulated in TMEM on its own and the epilogue sums
            // the units in registers (FP32 round-to-nearest adds), instead of the whole
            // group's K = npanels x BSZ sum in TMEM, whose accumulation measured several
            // times less accurate (log|K|, the unrefined backward error); C still gets
            // one add a tile
            constexpr uint32_t idesc = umma_idesc(F::kFmt, F::kFmt, 128, BSZ);
            uint32_t g = 0;
            int un = 0;
            for (uint32_t j = 0; ok; ++j) {
                if (ring_take(&ring[j % kRing], j, kStepWaitNs, &ok) == kNoTile) break;
                for (int p0 = 0; p0 < a.npanels && ok; p0 += a.unit_panels, ++un) {
                    const int unit_slabs = min(a.unit_panels, a.npanels - p0) * kSlabsP;
                    const int b = un & 1, u = un >> 1;
                    if (u > 0 && !mbar_wait_for(&tempty[b], (u - 1) & 1, kStepWaitNs)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t dcol = taddr + (uint32_t)(b * BSZ);
                    for (int kk = 0; kk < unit_slabs; ++kk, ++g) {
                        const uint32_t s = g % SM::kStages, use = g / SM::kStages;
                        if (!mbar_wait_for(&full[s], use & 1, kStepWaitNs)) {
                            ok = false;
                            break;
                        }
                        tc_fence_after();
                        const uint32_t base = smem_u32(smem + s * SM::kStage);
                        const uint32_t aHi = base, bHi = base + SM::kA;
                        const uint32_t aLo = base + SM::kRaw, bLo = aLo + SM::kA;
#pragma unroll
                        for (int ks = 0; ks < F::kK / F::kKStep; ++ks) {
                            const uint32_t off = ks * 32;  // one K step = 32 bytes along K
                            const uint64_t dAh = upd_desc(aHi + off), dAl = upd_desc(aLo + off);
                            const uint64_t dBh = upd_desc(bHi + off), dBl = upd_desc(bLo + off);
                            if (PREC != HS_PRECISION_TF32X3) {
                                umma_f16(dcol, dAh, dBh, idesc, (kk | ks) != 0);
                                umma_f16(dcol, dAh, dBl, idesc, 1);
                                umma_f16(dcol, dAl, dBh, idesc, 1);
                            } else {
                                umma_tf32(dcol, dAh, dBh, idesc, (kk | ks) != 0);
                                umma_tf32(dcol, dAh, dBl, idesc, 1);
                                umma_tf32(dcol, dAl, dBh, idesc, 1);
                            }
                        }
                        umma_commit(&empty[s]);
                    }
                    if (!ok) break;
                    umma_commit(&tfull[b]);
                }
            }
            if (!ok) atomicExch(a.err, 1);
            // TMEM is released only after every MMA issued here has completed, also
            // after a wait ran out
            umma_commit(drained);
            if (!mbar_wait_for(drained, 0, kStepWaitNs)) atomicExch(a.err, 1);
        }
    } else {
        // ---- epilogue warps 2..9: lane quarter q = warp % 4 holds tile rows 32q..32q+31;
        // the two warps of a quarter split the BSZ columns.  Each 32x32 chunk of -D
        // goes to the warp's shared tile (128-byte swizzle: 16-byte unit u of row i
        // at unit u ^ (i % 8)) and is added into C by a TMA reduce, so C is read and
        // written in whole lines by L2 instead of row by row by the SM.
        const int q = warp & 3;
        const int half = (warp - 2) >> 2;  // 0: warps 2-5, 1: warps 6-9
        constexpr int kChunks = BSZ / 64;   // 32-column chunks per warp
        float4* stile = reinterpret_cast<float4*>(staging + (warp - 2) * 4096);
        const float us = PREC == HS_PRECISION_F16X3 ? a.f16_unscale : 1.0f;  // exact power of two
        int un = 0;
        bool eok = true;
        const int units = (a.npanels + a.unit_panels - 1) / a.unit_panels;
        for (uint32_t jt = 0; eok; ++jt) {
            uint32_t t = kNoTile;
            int rok = 1;
            if (lane == 0) {
                bool tok = true;
                t = ring_take(&ring[jt % kRing], jt, kStepWaitNs, &tok);
                rok = tok ? 1 : 0;
            }
            t = __shfl_sync(0xffffffffu, t, 0);
            if (!__shfl_sync(0xffffffffu, rok, 0)) {
                if (lane == 0) atomicExch(a.err, 1);
                break;
            }
            if (t == kNoTile) break;
            // the tile's accumulation units, summed in registers (round-to-nearest FP32
            // adds, in unit order): each unit's accumulator is released as soon as it is
            // read, and C receives one add per tile
            float sum[kChunks][32];
            for (int pi = 0; pi < units; ++pi, ++un) {  // accumulation units (see the issuer)
                const int b = un & 1, u = un >> 1;
                int wok = 0;
                if (lane == 0) wok = mbar_wait_for(&tfull[b], u & 1, kStepWaitNs) ? 1 : 0;
                wok = __shfl_sync(0xffffffffu, wok, 0);
                if (!wok) {
                    if (lane == 0) atomicExch(a.err, 1);
                    eok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t tcol = taddr + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * BSZ + half * (BSZ / 2));
#pragma unroll
                for (int h = 0; h < 2 * kChunks; ++h) {  // 16 columns at a time
                    uint32_t v[16];
                    tmem_ld_32x32b_x16(tcol + (uint32_t)(h * 16), v);
                    tmem_ld_wait();
#pragma unroll
                    for (int e = 0; e < 16; ++e) {
                        float& sv = sum[h >> 1][(h & 1) * 16 + e];
                        sv = (pi == 0 ? 0.0f : sv) + __uint_as_float(v[e]);
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&tempty[b]);
            }
            if (!eok) break;
            int r, c, ti;
            decode(t, &r, &c, &ti);
            const int cblk = (int)block_id(r, c, a.nb);
            const int row0 = ti * 128 + q * 32;
#pragma unroll
            for (int j = 0; j < kChunks; ++j) {
                if (lane == 0) bulk_wait_read0();  // the previous chunk's reduce has read the tile
                __syncwarp();
#pragma unroll
                for (int e = 0; e < 8; ++e)
                    stile[lane * 8 + (e ^ (lane & 7))] = make_float4(-us * sum[j][4 * e + 0], -us * sum[j][4 * e + 1],
                                                                     -us * sum[j][4 * e + 2], -us * sum[j][4 * e + 3]);
                fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0) {
                    tma_reduce_add_3d(&mC32, stile, half * (BSZ / 2) + j * 32, row0, cblk);
                    bulk_commit();
                }
            }
        }
    }
    if (warp >= 2 && lane == 0) bulk_wait0();  // every reduce into C has completed
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(taddr, kAccCols);
}

// ------------------------------------------------------------------ helpers
__global__ void f64_to_f32_kernel(const double* __restrict__ in, float* __restrict__ out, int64_t n) {
    const int64_t n2 = n / 2;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n2; i += (int64_t)gridDim.x * blockDim.x) {
        const double2 v = __ldcs(reinterpret_cast<const double2*>(in) + i);
        reinterpret_cast<float2*>(out)[i] = make_float2((float)v.x, (float)v.y);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && (n & 1)) out[n - 1] = (float)in[n - 1];
}

// sum over the CTA (fixed order: warps by shuffle butterfly, then warp 0 in order);
// the total is valid in thread 0
__device__ __forceinline__ double cta_total(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int wp = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sh[wp] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += sh[i];
    return t;
}

// the same conversion a stored block at a time, with the squared Frobenius norm of
// the symmetric matrix (off-diagonal blocks twice) summed on the way: CTA partials
// in part[blockIdx.x], blocks in a fixed order, so the norm is reproducible
__global__ void f64_to_f32_fro2_kernel(const double* __restrict__ in, float* __restrict__ out, int bsz, int nb,
                                       int64_t T, double* __restrict__ part) {
    __shared__ double sh[32];
    double acc = 0.0;
    // a thread converts 4 consecutive values a step (two 16-byte loads, one 16-byte
    // store), four steps' loads issued before their stores
    const int bb4 = bsz * bsz / 4;
    for (int64_t blk = blockIdx.x; blk < T; blk += gridDim.x) {
        int bi, bj;
        block_coords(blk, nb, &bi, &bj);
        const double2* src = reinterpret_cast<const double2*>(in) + blk * 2 * bb4;
        float4* dst = reinterpret_cast<float4*>(out) + blk * bb4;
        double sq = 0.0;
        for (int e0 = threadIdx.x; e0 < bb4; e0 += 4 * blockDim.x) {
            double2 v[4][2];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int e = e0 + u * blockDim.x;
                if (e < bb4) {
                    v[u][0] = __ldcs(src + 2 * e);
                    v[u][1] = __ldcs(src + 2 * e + 1);
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int e = e0 + u * blockDim.x;
                if (e < bb4) {
                    dst[e] = make_float4((float)v[u][0].x, (float)v[u][0].y, (float)v[u][1].x, (float)v[u][1].y);
                    sq += v[u][0].x * v[u][0].x;
                    sq += v[u][0].y * v[u][0].y;
                    sq += v[u][1].x * v[u][1].x;
                    sq += v[u][1].y * v[u][1].y;
                }
            }
        }
        acc += ((bi == bj) ? 1.0 : 2.0) * sq;
    }
    const double t = cta_total(acc, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// diagonal shift of the FP32 copy (valid rows only)
__global__ void shift_diag_kernel(float* __restrict__ A, int bsz, int nb, int64_t N, float shift) {
    const int64_t bb = (int64_t)bsz * bsz;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        const int k = (int)(i / bsz), r = (int)(i % bsz);
        A[block_id(k, k, nb) * bb + (int64_t)r * bsz + r] += shift;
    }
}

// lo[i] = a[i] - tf32(a[i]) over n floats
__global__ void lo_part_kernel(const float* __restrict__ a, float* __restrict__ lo, int64_t n4) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n4; i += (int64_t)gridDim.x * blockDim.x) {
        const float4 v = reinterpret_cast<const float4*>(a)[i];
        reinterpret_cast<float4*>(lo)[i] =
            make_float4(v.x - tf32_trunc(v.x), v.y - tf32_trunc(v.y), v.z - tf32_trunc(v.z), v.w - tf32_trunc(v.w));
    }
}

// ------------------------------------------------------------------ diagonal chain
// The FP64 work on one diagonal block in a single CTA: Cholesky of the FP32 block
// (lower triangle; rows / columns >= valid replaced by the identity) together with
// X = L^-1, by one right-looking sweep over 32-column panels p:
//   - the panel's 32 x 32 diagonal block D_p is factored by warp 0 in registers,
//     column by column, and inverted in the same pass (lane = row of L_pp and
//     column of X_pp = L_pp^-1; each column of L_pp is broadcast once for both);
//   - block row p of X is X_pp B_p (B = the identity less the updates below) and
//     the panel rows below the diagonal block become row X_pp^T;
//   - rank-32 updates in 32 x 32 warp tiles on the FP64 tensor pipe (DMMA): the
//     trailing lower triangle, S_rc -= L_rp L_cp^T, and the rows of B below,
//     B_r -= L_rp X_p.  Warp 1 first computes the diagonal block of panel p+1 (the
//     corner of the trailing triangle) and hands it to warp 0, which factors it
//     while warps 1..7 update the rest.
// S (the working matrix) and B (held transposed in Y, which ends as X^T) stay in
// global memory (L2-resident; S is read from the FP32 block directly at panel 0);
// the panel is staged in shared memory k-major, block row p of B / X as [a][c].
// Outputs: L's lower triangle in FP64 in Ld (the solves read its diagonal for log|K|,
// the mixed NLML the whole block; the FP32 block keeps its input), Y = X^T,
// invHi = float(X), invLo = invHi - tf32(invHi).
// A pivot that is not > 0 on a valid row records its global row in *info.
constexpr int kChainThreads = 256;

template <int BSZ>
struct ChainSmem {
    static constexpr int kP = BSZ / 32;       // panels
    static constexpr int kLt = BSZ - 32 + 4;  // k-major panel stride (rows below the diagonal block)
    static constexpr int kXr = BSZ + 4;       // block-row stride
    static constexpr int kD = 33;             // diagonal block / inverse stride
    static constexpr size_t kBytes = (size_t)(32 * kLt + 32 * kXr + 2 * 32 * kD + 64) * sizeof(double);
};

// two / four consecutive entries (r, c..) of the working matrix: the FP32 block with
// the identity outside the valid range (panel 0), else S
template <int BSZ>
__device__ __forceinline__ void chain_src4(const float* __restrict__ blk, const double* __restrict__ S, bool first,
                                           int valid, int r, int c, double v[4]) {
    if (first) {
        const float4 f = *reinterpret_cast<const float4*>(blk + (size_t)r * BSZ + c);
        const float fv[4] = {f.x, f.y, f.z, f.w};
#pragma unroll
        for (int q = 0; q < 4; ++q) v[q] = (r >= valid || c + q >= valid) ? (r == c + q ? 1.0 : 0.0) : (double)fv[q];
    } else {
        const double2 a = *reinterpret_cast<const double2*>(S + (size_t)r * BSZ + c);
        const double2 b = *reinterpret_cast<const double2*>(S + (size_t)r * BSZ + c + 2);
        v[0] = a.x;
        v[1] = a.y;
        v[2] = b.x;
        v[3] = b.y;
    }
}

template <int BSZ>
__device__ __forceinline__ double2 chain_src2(const float* __restrict__ blk, const double* __restrict__ S, bool first,
                                              int valid, int r, int c) {
    if (first) {
        const float2 f = *reinterpret_cast<const float2*>(blk + (size_t)r * BSZ + c);
        return make_double2((r >= valid || c >= valid) ? (r == c ? 1.0 : 0.0) : (double)f.x,
                            (r >= valid || c + 1 >= valid) ? (r == c + 1 ? 1.0 : 0.0) : (double)f.y);
    }
    return *reinterpret_cast<const double2*>(S + (size_t)r * BSZ + c);
}

// warp 0: D (32 x 32, stride kD, lower triangle read) -> L_pp in D (upper part
// zero) and Xp = L_pp^-1.  d0 = the block's first row within the diagonal block
// of the matrix.
__device__ __forceinline__ void chain_diag(double* __restrict__ D, double* __restrict__ Xp,
                                           double* __restrict__ colb, int lane, int d0, int valid,
                                           long long* __restrict__ info, long long row_base) {
    constexpr int kD = 33;
    double x[32], z[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) {
        x[j] = j <= lane ? D[lane * kD + j] : 0.0;
        z[j] = j == lane ? 1.0 : 0.0;
    }
    // the pivot of step k+1 is taken from lane k+1 as soon as that lane has its own
    // L[k+1][k], ahead of the column broadcast through shared memory
    double piv = __shfl_sync(0xffffffffu, x[0], 0);
#pragma unroll
    for (int k = 0; k < 32; ++k) {
        if (lane == 0 && d0 + k < valid && !(piv > 0.0)) {
            atomicMin(info, row_base + d0 + k);
            // info[1]: the most negative failing pivot (bit pattern of a negative double;
            // a larger signed pattern is a larger magnitude); NaN and zero pivots are not
            // recorded
            if (piv < 0.0) atomicMax(info + 1, __double_as_longlong(piv));
        }
        const double ri = rsqrt(piv);
        const double lk = lane == k ? piv * ri : (lane > k ? x[k] * ri : 0.0);  // L[lane][k]
        const double zk = z[k] * ri;                                            // X[k][lane]
        x[k] = lk;
        z[k] = zk;
        if (k + 1 < 32) piv = __shfl_sync(0xffffffffu, x[k + 1] - lk * lk, k + 1);
        double* cb = colb + 32 * (k & 1);
        cb[lane] = lk;
        __syncwarp();
#pragma unroll
        for (int j = k + 1; j < 32; ++j) {
            const double ljk = cb[j];
            x[j] = x[j] - lk * ljk;
            z[j] = z[j] - ljk * zk;
        }
    }
#pragma unroll
    for (int j = 0; j < 32; ++j) {
        D[lane * kD + j] = x[j];
        Xp[j * kD + lane] = z[j];
    }
}

// one 32 x 32 warp tile of sum_k A[m][k] B[k][n] over K = 32 on the FP64 tensor
// pipe: A[m][k] = pa[k * lda + m], B[k][n] = pb[k * ldb + n]; lane holds rows
// 8 mi + lane/4, columns 8 ni + 2 (lane%4) + {0, 1}
__device__ __forceinline__ void chain_wtile(const double* __restrict__ pa, int lda, const double* __restrict__ pb,
                                            int ldb, int lane, double (&acc)[4][4][2]) {
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) acc[mi][ni][0] = acc[mi][ni][1] = 0.0;
#pragma unroll
    for (int k0 = 0; k0 < 32; k0 += 4) {
        double a[4], b[4];
#pragma unroll
        for (int mi = 0; mi < 4; ++mi) a[mi] = pa[(k0 + t) * lda + 8 * mi + g];
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) b[ni] = pb[(k0 + t) * ldb + 8 * ni + g];
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) dmma884(acc[mi][ni], a[mi], b[ni]);
    }
}

__device__ __forceinline__ void chain_bar(int id, int count) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// block row p of X from shared memory -> Y (transposed; zero before column c0 in
// the panel's rows of Y) and invHi / invLo (zero after column w when `zero_upper`:
// the planes are shared by all diagonal blocks and only the first writes the part
// above the block diagonal).  Threads `t0`, `t0 + nt`, ... take part.
template <int BSZ>
__device__ __forceinline__ void chain_outputs(double* __restrict__ Y, float* __restrict__ invHi,
                                              float* __restrict__ invLo, const double* __restrict__ Xr, int c0,
                                              bool zero_upper, int t0, int nt) {
    using CS = ChainSmem<BSZ>;
    constexpr int n = BSZ, kXr = CS::kXr;
    const int w = c0 + 32;
    for (int e = t0; e < w * 8; e += nt) {
        const int c = e % w, a4 = e / w;
        double v[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) v[q] = Xr[(4 * a4 + q) * kXr + c];
        *reinterpret_cast<double2*>(Y + (size_t)c * n + c0 + 4 * a4) = make_double2(v[0], v[1]);
        *reinterpret_cast<double2*>(Y + (size_t)c * n + c0 + 4 * a4 + 2) = make_double2(v[2], v[3]);
    }
    for (int e = t0; e < 32 * c0 / 2; e += nt) {
        const int c = c0 + (2 * e) / c0, r = (2 * e) % c0;
        *reinterpret_cast<double2*>(Y + (size_t)c * n + r) = make_double2(0.0, 0.0);
    }
    const int cw = zero_upper ? n : w;  // columns written
    for (int e = t0; e < 8 * cw; e += nt) {
        const int a = e / (cw / 4), c = 4 * (e % (cw / 4));
        float4 f = make_float4(0.f, 0.f, 0.f, 0.f);
        if (c < w) {
            const double* xr = Xr + a * kXr + c;
            f = make_float4((float)xr[0], (float)xr[1], (float)xr[2], (float)xr[3]);
        }
        const size_t o = (size_t)(c0 + a) * n + c;
        *reinterpret_cast<float4*>(invHi + o) = f;
        *reinterpret_cast<float4*>(invLo + o) =
            make_float4(f.x - tf32_trunc(f.x), f.y - tf32_trunc(f.y), f.z - tf32_trunc(f.z), f.w - tf32_trunc(f.w));
    }
}

template <int BSZ>
__global__ void __launch_bounds__(kChainThreads, 1)
    diag_chain_kernel(const float* __restrict__ blk, double* __restrict__ S, double* __restrict__ Y,
                      double* __restrict__ Ld, float* __restrict__ invHi, float* __restrict__ invLo, int valid,
                      int zero_upper, long long* __restrict__ info, long long row_base) {
    using CS = ChainSmem<BSZ>;
    constexpr int n = BSZ, kLt = CS::kLt, kXr = CS::kXr, kD = CS::kD;
    constexpr int kIt = (n * 8 + kChainThreads - 1) / kChainThreads;  // staging steps a thread
    extern __shared__ double csm[];
    double* PsT = csm;               // [k][rr - 32]: panel rows below the diagonal block
    double* Xr = PsT + 32 * kLt;     // [a][c]: block row p of B, then of X
    double* D = Xr + 32 * kXr;       // diagonal block of the current panel (L after warp 0)
    double* Xp = D + 32 * kD;        // its inverse
    double* colb = Xp + 32 * kD;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    if (warp == 0) {  // D_0 from the FP32 block
#pragma unroll
        for (int j4 = 0; j4 < 8; ++j4) {
            double v[4];
            chain_src4<BSZ>(blk, S, true, valid, lane, 4 * j4, v);
#pragma unroll
            for (int q = 0; q < 4; ++q) D[lane * kD + 4 * j4 + q] = v[q];
        }
        __syncwarp();
        chain_diag(D, Xp, colb, lane, 0, valid, info, row_base);
    }
    __syncthreads();

    for (int p = 0; p < CS::kP; ++p) {
        const int c0 = 32 * p, mb = n - c0 - 32, w = c0 + 32;
        const bool first = p == 0;
        {
            // panel rows below the diagonal block, four columns a step (rows fastest),
            // all loads of a thread in flight before the shared stores
            double v[kIt][4];
#pragma unroll
            for (int u = 0; u < kIt; ++u) {
                const int e = tid + u * kChainThreads;
                if (e < mb * 8) chain_src4<BSZ>(blk, S, first, valid, c0 + 32 + e % mb, c0 + 4 * (e / mb), v[u]);
            }
#pragma unroll
            for (int u = 0; u < kIt; ++u) {
                const int e = tid + u * kChainThreads;
                if (e < mb * 8) {
                    const int rr = e % mb, k4 = e / mb;
#pragma unroll
                    for (int q = 0; q < 4; ++q) PsT[(4 * k4 + q) * kLt + rr] = v[u][q];
                }
            }
            // B_p[a][c]: columns before the panel from Y[c][c0 + a], the panel's own the identity
#pragma unroll
            for (int u = 0; u < kIt; ++u) {
                const int e = tid + u * kChainThreads;
                const int c = e % w, a4 = e / w;
                if (e < w * 8) {
                    if (c < c0) {
                        const double2 x0 = *reinterpret_cast<const double2*>(Y + (size_t)c * n + c0 + 4 * a4);
                        const double2 x1 = *reinterpret_cast<const double2*>(Y + (size_t)c * n + c0 + 4 * a4 + 2);
                        v[u][0] = x0.x;
                        v[u][1] = x0.y;
                        v[u][2] = x1.x;
                        v[u][3] = x1.y;
                    } else {
#pragma unroll
                        for (int q = 0; q < 4; ++q) v[u][q] = (c - c0 == 4 * a4 + q) ? 1.0 : 0.0;
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < kIt; ++u) {
                const int e = tid + u * kChainThreads;
                if (e < w * 8) {
                    const int c = e % w, a4 = e / w;
#pragma unroll
                    for (int q = 0; q < 4; ++q) Xr[(4 * a4 + q) * kXr + c] = v[u][q];
                }
            }
        }
        __syncthreads();
        if (tid < w) {
            // column tid of block row p: X_p = X_pp B_p
            double b[32], v[32];
#pragma unroll
            for (int a = 0; a < 32; ++a) {
                b[a] = Xr[a * kXr + tid];
                v[a] = 0.0;
            }
#pragma unroll
            for (int q = 0; q < 32; ++q)
#pragma unroll
                for (int a = q; a < 32; ++a) v[a] = fma(Xp[a * kD + q], b[q], v[a]);
#pragma unroll
            for (int a = 0; a < 32; ++a) Xr[a * kXr + tid] = v[a];
        } else if (tid < w + mb) {
            // panel row below the diagonal block: row X_pp^T
            const int rr = tid - w;
            double x[32], v[32];
#pragma unroll
            for (int k = 0; k < 32; ++k) {
                x[k] = PsT[k * kLt + rr];
                v[k] = 0.0;
            }
#pragma unroll
            for (int k = 0; k < 32; ++k)
#pragma unroll
                for (int j = k; j < 32; ++j) v[j] = fma(x[k], Xp[j * kD + k], v[j]);
#pragma unroll
            for (int j = 0; j < 32; ++j) PsT[j * kLt + rr] = v[j];
        }
        __syncthreads();
        // panel p of L -> Ld in FP64 (its diagonal block from D, lower triangle, and the
        // rows below from PsT; D is rewritten below); block row p of X goes out during
        // the updates
        for (int e = tid; e < 32 * 32; e += kChainThreads) {
            const int i = e >> 5, j = e & 31;
            if (j <= i) Ld[(size_t)(c0 + i) * n + c0 + j] = D[i * kD + j];
        }
        for (int e = tid; e < mb * 32; e += kChainThreads) {
            const int k = e & 31, rr = e >> 5;
            Ld[(size_t)(c0 + 32 + rr) * n + c0 + k] = PsT[k * kLt + rr];
        }
        if (mb == 0) {
            chain_outputs<BSZ>(Y, invHi, invLo, Xr, c0, zero_upper != 0, tid, kChainThreads);
            break;
        }
        __syncthreads();  // D, Xp are rewritten below
        if (warp == 0) {
            chain_bar(1, 64);  // warp 1 has written D of panel p+1
            chain_diag(D, Xp, colb, lane, c0 + 32, valid, info, row_base);
        } else {
            // 32 x 32 warp tiles over warps 1..7: the trailing lower triangle (its
            // corner, the diagonal block of panel p+1, first and into D), then the rows
            // of B below block row p (in Y[c][r]; the panel's own columns are written
            // for the first time)
            const int g = lane >> 2, t = lane & 3;
            const int q = mb >> 5, wq = w >> 5;
            const int ntri = q * (q + 1) / 2;
            const int ntiles = ntri + q * wq;
            // warp 4 shares warp 0's scheduler and stays off the tile work
            constexpr int kTw = kChainThreads / 32 - 2;
            const int tw = warp < 4 ? warp - 1 : warp - 2;
            double acc[4][4][2];
            for (int u = tw; u < ntiles && warp != 4; u += kTw) {
                if (u < ntri) {
                    int R = (int)((sqrtf(8.0f * u + 1.0f) - 1.0f) * 0.5f);
                    while (R * (R + 1) / 2 > u) --R;
                    while ((R + 1) * (R + 2) / 2 <= u) ++R;
                    const int C = u - R * (R + 1) / 2;
                    chain_wtile(PsT + 32 * R, kLt, PsT + 32 * C, kLt, lane, acc);
                    const int r0 = c0 + 32 + 32 * R, cc0 = c0 + 32 + 32 * C;
#pragma unroll
                    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                        for (int ni = 0; ni < 4; ++ni) {
                            const int r = r0 + 8 * mi + g, c = cc0 + 8 * ni + 2 * t;
                            const double2 sv = chain_src2<BSZ>(blk, S, first, valid, r, c);
                            const double2 o = make_double2(sv.x - acc[mi][ni][0], sv.y - acc[mi][ni][1]);
                            if (u == 0) {
                                D[(r - r0) * kD + (c - cc0)] = o.x;
                                D[(r - r0) * kD + (c - cc0) + 1] = o.y;
                            } else {
                                *reinterpret_cast<double2*>(S + (size_t)r * n + c) = o;
                            }
                        }
                    if (u == 0) chain_bar(1, 64);  // D of panel p+1 is ready for warp 0
                } else {
                    const int R = (u - ntri) % q, C = (u - ntri) / q;
                    chain_wtile(PsT + 32 * R, kLt, Xr + 32 * C, kXr, lane, acc);
                    const bool fresh = C == p;
                    const int r0 = c0 + 32 + 32 * R;
#pragma unroll
                    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                            for (int i = 0; i < 2; ++i) {
                                double* o = Y + (size_t)(32 * C + 8 * ni + 2 * t + i) * n + r0 + 8 * mi + g;
                                *o = (fresh ? 0.0 : *o) - acc[mi][ni][i];
                            }
                }
            }
            chain_outputs<BSZ>(Y, invHi, invLo, Xr, c0, zero_upper != 0, tid - 32, kChainThreads - 32);
        }
        __syncthreads();
    }
}

__global__ void set_int_kernel(int* p, int v) { *p = v; }

PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

hs_status get_encoder() {
    if (g_encode) return HS_OK;
    cudaDriverEntryPointQueryResult q;
    void* fn = nullptr;
    HS_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
    if (q != cudaDriverEntryPointSuccess || !fn) {
        set_error("cuTensorMapEncodeTiled is not available from the driver");
        return HS_ERR_UNSUPPORTED;
    }
    g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    return HS_OK;
}

// 3-D FP32 map over `blocks` blocks of bsz x bsz, box = 32 columns x box_rows rows x 1 block
hs_status make_map(CUtensorMap* m, void* base, int bsz, int64_t blocks, int box_rows, int box_k = kSlab,
                   int elem = 4) {
    hs_status st = get_encoder();
    if (st != HS_OK) return st;
    cuuint64_t dims[3] = {(cuuint64_t)bsz, (cuuint64_t)bsz, (cuuint64_t)blocks};
    cuuint64_t strides[2] = {(cuuint64_t)bsz * elem, (cuuint64_t)bsz * bsz * elem};
    cuuint32_t box[3] = {(cuuint32_t)box_k, (cuuint32_t)box_rows, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    // 2-byte maps are plain copies of the BF16 or FP16 split (no conversion on load)
    CUresult r = g_encode(m, elem == 2 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base,
                          dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          box_k * elem == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
        return HS_ERR_CUDA;
    }
    return HS_OK;
}

// panel TRSM of `items` blocks below the diagonal of column a.k
template <int BSZ>
hs_status tc_launch(hs_ctx ctx, const MixedWork& w, TcArgs a, int64_t items, cudaStream_t s) {
    using SM = TcSmem<BSZ>;
    const int64_t grid = items * SM::kTiles;
    if (grid <= 0) return HS_OK;
    HS_REQUIRE(grid < (1LL << 31), "too many tiles");
    ctx->launches += 1;
    tc_tile_kernel<BSZ, MODE_TRSM><<<(unsigned)grid, kTcThreads, SM::kBytes, s>>>(w.mA128, w.mL128, w.mL32, a);
    HS_CHECK_LAUNCH("tc_tile_kernel");
    return HS_OK;
}

template <int BSZ>
hs_status tc_update_launch(hs_ctx ctx, const MixedWork& w, const TcArgs& a, int precision, cudaStream_t s,
                           int max_ctas) {
    using SM = UpdSmem<BSZ>;
    const int m = a.nb - a.first_col;
    const int64_t ntiles = update_tiles(a.part, m, a.ncols, BSZ / 128);
    if (ntiles <= 0) return HS_OK;
    HS_REQUIRE(ntiles < (int64_t)kNoTile, "too many update tiles");
    HS_REQUIRE(a.part != 3 || (a.ncols >= 1 && a.ncols <= m), "update columns outside the trailing matrix");
    const int grid = (int)(ntiles < max_ctas ? ntiles : max_ctas);
    ctx->launches += 1;
    if (precision == HS_PRECISION_BF16X3)
        tc_update_kernel<BSZ, HS_PRECISION_BF16X3>
            <<<grid, kUpdThreads, SM::kBytes, s>>>(w.mP128, w.mPB, w.mP128, w.mPB, w.mC32, a);
    else if (precision == HS_PRECISION_F16X3)
        tc_update_kernel<BSZ, HS_PRECISION_F16X3>
            <<<grid, kUpdThreads, SM::kBytes, s>>>(w.mP128, w.mPB, w.mP128, w.mPB, w.mC32, a);
    else
        tc_update_kernel<BSZ, HS_PRECISION_TF32X3>
            <<<grid, kUpdThreads, SM::kBytes, s>>>(w.mU128, w.mUB, w.mV128, w.mVB, w.mC32, a);
    HS_CHECK_LAUNCH("tc_update_kernel");
    return HS_OK;
}

bool g_tc_attr[64][2] = {};

template <int BSZ>
hs_status tc_attrs() {
    int dev = 0;
    HS_CUDA(cudaGetDevice(&dev));
    const int slot = BSZ == 256 ? 1 : 0;
    if (dev < 64 && g_tc_attr[dev][slot]) return HS_OK;
    HS_CUDA(cudaFuncSetAttribute(tc_tile_kernel<BSZ, MODE_TRSM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 TcSmem<BSZ>::kBytes));
    HS_CUDA(cudaFuncSetAttribute(tc_update_kernel<BSZ, HS_PRECISION_TF32X3>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, UpdSmem<BSZ>::kBytes));
    HS_CUDA(cudaFuncSetAttribute(tc_update_kernel<BSZ, HS_PRECISION_BF16X3>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, UpdSmem<BSZ>::kBytes));
    HS_CUDA(cudaFuncSetAttribute(tc_update_kernel<BSZ, HS_PRECISION_F16X3>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, UpdSmem<BSZ>::kBytes));
    HS_CUDA(cudaFuncSetAttribute(diag_chain_kernel<BSZ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)ChainSmem<BSZ>::kBytes));
    if (dev < 64) g_tc_attr[dev][slot] = true;
    return HS_OK;
}

int grid_for_elems(int64_t n, int num_sms) {
    int64_t g = (n + 255) / 256;
    if (g > 8LL * num_sms) g = 8LL * num_sms;
    return (int)(g < 1 ? 1 : g);
}

}  // namespace

size_t mixed_workspace_bytes(int64_t N, int bsz) {
    const int64_t nb = (N + bsz - 1) / bsz;
    const size_t bb = (size_t)bsz * bsz;
    const size_t T = (size_t)(nb * (nb + 1) / 2);
    size_t bytes = 0;
    bytes += T * bb * 4;                 // A32 / L32
    bytes += (size_t)(kSets * nb + 2) * bb * 4;  // LO: two groups' low parts + L_kk^-1 hi / lo
    bytes += (size_t)nb * bb * 8;        // Ldiag64
    bytes += (size_t)nb * bb * 8;        // Yinv
    bytes += (size_t)2 * kSets * nb * bb * 2;  // 16-bit split of two groups' panels (hi / lo each)
    bytes += bb * 8;                     // S
    bytes += 1024;                       // error flags
    bytes += ((size_t)tile_counters(nb) * 8 + 255) & ~size_t(255);  // tile counters of the updates
    bytes += ((size_t)nb * 4 + 255) & ~size_t(255);  // sweep publication flags
    return bytes;
}

hs_status mixed_bind(hs_ctx ctx, void* ws, MixedWork* w) {
    const int bsz = ctx->bsz, nb = ctx->nb;
    const size_t bb = (size_t)bsz * bsz;
    const size_t T = total_blocks(nb);
    char* p = static_cast<char*>(ws);
    w->A32 = reinterpret_cast<float*>(p);
    p += T * bb * 4;
    w->LO = reinterpret_cast<float*>(p);
    p += (size_t)(kSets * nb + 2) * bb * 4;
    w->Ld = reinterpret_cast<double*>(p);
    p += (size_t)nb * bb * 8;
    w->Yinv = reinterpret_cast<double*>(p);
    p += (size_t)nb * bb * 8;
    w->P16 = reinterpret_cast<__nv_bfloat16*>(p);
    p += (size_t)2 * kSets * nb * bb * 2;
    w->S = reinterpret_cast<double*>(p);
    p += bb * 8;
    w->err = reinterpret_cast<int*>(p);
    p += 1024;
    w->tile_ctr = reinterpret_cast<unsigned long long*>(p);
    p += ((size_t)tile_counters(nb) * 8 + 255) & ~size_t(255);
    w->flags = reinterpret_cast<unsigned*>(p);
    hs_status st = make_map(&w->mA128, w->A32, bsz, (int64_t)T, 128);
    if (st == HS_OK) st = make_map(&w->mL128, w->LO, bsz, kSets * nb + 2, 128);
    if (st == HS_OK) st = make_map(&w->mL32, w->LO, bsz, kSets * nb + 2, 32);
    if (st == HS_OK) st = make_map(&w->mU128, w->A32, bsz, (int64_t)T, 128, kUpdK);
    if (st == HS_OK) st = make_map(&w->mUB, w->A32, bsz, (int64_t)T, bsz, kUpdK);
    if (st == HS_OK) st = make_map(&w->mV128, w->LO, bsz, kSets * nb + 2, 128, kUpdK);
    if (st == HS_OK) st = make_map(&w->mVB, w->LO, bsz, kSets * nb + 2, bsz, kUpdK);
    if (st == HS_OK) st = make_map(&w->mC32, w->A32, bsz, (int64_t)T, 32, 32);
    if (st == HS_OK) st = make_map(&w->mP128, w->P16, bsz, 2 * kSets * (int64_t)nb, 128, 2 * kUpdK, 2);
    if (st == HS_OK) st = make_map(&w->mPB, w->P16, bsz, 2 * kSets * (int64_t)nb, bsz, 2 * kUpdK, 2);
    return st;
}

int mixed_fro_grid(int64_t blocks) { return (int)(blocks < 1024 ? blocks : 1024); }

hs_status mixed_factor(hs_ctx ctx, const double* K64, MixedWork& w, cudaStream_t s, double shift, int precision,
                       double* fro_part, double maxdiag, int acc_panels) {
    if (acc_panels != 1 && acc_panels != 2 && acc_panels != kPanelGroup) acc_panels = kPanelGroup;
    const int bsz = ctx->bsz, nb = ctx->nb;
    HS_REQUIRE(bsz == 128 || bsz == 256, "the mixed-precision factor supports matrixBlockSize 128 or 256");
    hs_status st = bsz == 256 ? tc_attrs<256>() : tc_attrs<128>();
    if (st != HS_OK) return st;
    const size_t bb = (size_t)bsz * bsz;
    const int64_t T = total_blocks(nb);
    ctx->launches += 2;
    set_int_kernel<<<1, 1, 0, s>>>(w.err, 0);
    HS_CUDA(cudaMemsetAsync(w.tile_ctr, 0, (size_t)tile_counters(nb) * sizeof(unsigned long long), s));
    if (fro_part && bsz % 4 == 0)
        f64_to_f32_fro2_kernel<<<mixed_fro_grid(T), 256, 0, s>>>(K64, w.A32, bsz, nb, T, fro_part);
    else
        f64_to_f32_kernel<<<grid_for_elems(T * (int64_t)bb / 2, ctx->num_sms), 256, 0, s>>>(K64, w.A32,
                                                                                          T * (int64_t)bb);
    HS_CHECK_LAUNCH("f64_to_f32");
    if (shift != 0.0) {
        ctx->launches += 1;
        shift_diag_kernel<<<64, 256, 0, s>>>(w.A32, bsz, nb, ctx->N, (float)shift);
        HS_CHECK_LAUNCH("shift_diag");
    }
    // diagonal block k in FP64 (one CTA): L_kk, its FP32 copy in place, Y_k = L_kk^-T
    // and the split L_kk^-1 for the panel TRSM
    auto diag_chain = [&](int k, cudaStream_t st_) -> hs_status {
        const int64_t id = T - (int64_t)(nb - k) * (nb - k + 1) / 2;
        float* dblk = w.A32 + (size_t)id * bb;
        const int64_t rem = ctx->N - (int64_t)k * bsz;
        const int valid = rem < bsz ? (int)rem : bsz;
        float* invHi = w.LO + (size_t)kSets * nb * bb;
        prof_begin(ctx, st_, HS_KERNEL_POTRF);
        ctx->launches += 1;
        if (bsz == 256)
            diag_chain_kernel<256><<<1, kChainThreads, ChainSmem<256>::kBytes, st_>>>(
                dblk, w.S, w.Yinv + (size_t)k * bb, w.Ld + (size_t)k * bb, invHi, invHi + bb, valid, k == 0,
                ctx->d_info, (long long)k * bsz);
        else
            diag_chain_kernel<128><<<1, kChainThreads, ChainSmem<128>::kBytes, st_>>>(
                dblk, w.S, w.Yinv + (size_t)k * bb, w.Ld + (size_t)k * bb, invHi, invHi + bb, valid, k == 0,
                ctx->d_info, (long long)k * bsz);
        HS_CHECK_LAUNCH("diag_chain");
        const double nn = bsz;
        prof_end(ctx, st_, HS_KERNEL_POTRF, 2.0 * nn * nn * nn / 3.0, nn * nn * (4.0 + 8.0 * 4.0 + 4.0 + 4.0));
        return HS_OK;
    };
    // Panels are factored in groups of up to kPanelGroup (k .. k+g-1) and the columns
    // after a group are updated with all of its panels at once (K = g bsz per pass
    // over C), which divides the read-modify-write traffic on the trailing matrix by
    // g.  Inside a group, column k+i+1 is brought up to date with panels k..k+i just
    // before its diagonal chain and panel.  Panel k+i keeps its low parts and 16-bit
    // split in slot set kPanelGroup bank + i; consecutive groups alternate banks.
    // Look-ahead by a group, while the trailing matrix is large: the update after a
    // group first brings the next group's columns up to date (part 3); the next
    // group's chains, panels and inner updates then run on the high-priority side
    // stream, on the side_sms SMs that the update of the remaining columns (part 0)
    // leaves free, and once they are done a second launch of that update joins on
    // those SMs, taking tiles from the same counter.  Near the end, with too little
    // update left to hide a group behind, the look-ahead is by one diagonal chain: the
    // update runs as part 1 (the next column) and part 2 (the rest), with that
    // column's chain on the side stream beside part 2.  Both orders add the same
    // products into every block in the same sequence.
    cudaStream_t sd = ctx->side_hi;
    const bool lookahead = sd != nullptr && ctx->num_sms > 8;
    const int kFree = 2;
    const int side_sms = ctx->mixed_side_sms < ctx->num_sms / 2 ? ctx->mixed_side_sms : ctx->num_sms / 2;
    const bool group_ahead = lookahead && side_sms > 0;
    int next_ctr = 0;  // tile counters used so far (one per group look-ahead)
    const double n3 = (double)bsz * bb;
    auto diag_id = [&](int k) { return T - (int64_t)(nb - k) * (nb - k + 1) / 2; };
    TcArgs base{};
    base.A32 = w.A32;
    base.LO = w.LO;
    base.nb = nb;
    base.err = w.err;
    base.abort_flag = ctx->d_info;
    base.inv = kSets * nb;
    // FP16 split: scale s = 2^e, the largest e with s sqrt(maxdiag) <= 2^15.  Every
    // |L_ij| <= sqrt(K_ii) <= sqrt(maxdiag), so s L stays below 2^15 (FP16 holds up to
    // 65504), and entries small enough to reach FP16's subnormal range carry an absolute
    // error below 2^-25 / s, far below the products that matter.  A matrix that is not
    // positive definite can overflow it; its factor then fails a pivot check and is
    // redone with 3xTF32 products.
    base.f16_scale = base.f16_unscale = 1.0f;
    if (precision == HS_PRECISION_F16X3) {
        int e = 0;
        if (maxdiag > 0.0 && std::isfinite(maxdiag)) {
            e = (int)std::floor(std::log2(32768.0 / std::sqrt(maxdiag)));
            e = e < -60 ? -60 : (e > 60 ? 60 : e);
        }
        base.f16_scale = std::ldexp(1.0f, e);
        base.f16_unscale = std::ldexp(1.0f, -2 * e);
    }
    // blocks k+1..nb-1 of column k: FP32 low parts into set `set`, TRSM-as-GEMM with
    // L_kk^-T (writes L and its low part), and for BF16 / FP16 the split of L into P16
    auto panel = [&](int k, int set, cudaStream_t st_) -> hs_status {
        const int64_t blockID = diag_id(k);
        float* dblk = w.A32 + (size_t)blockID * bb;
        const int m = nb - k - 1;
        ctx->launches += 1;
        lo_part_kernel<<<grid_for_elems((int64_t)m * bb / 4, ctx->num_sms), 256, 0, st_>>>(
            dblk + bb, w.LO + (size_t)set * nb * bb, (int64_t)m * bb / 4);
        HS_CHECK_LAUNCH("lo_part");
        TcArgs a = base;
        a.blockID = blockID;
        a.k = k;
        a.lo_base = set * nb;
        // 16-bit products downstream: the TRSM writes L's 16-bit split itself
        a.split16 = (precision == HS_PRECISION_BF16X3 || precision == HS_PRECISION_F16X3) ? precision : 0;
        a.P16 = w.P16;
        prof_begin(ctx, st_, HS_KERNEL_TRSM);
        hs_status r = bsz == 256 ? tc_launch<256>(ctx, w, a, m, st_) : tc_launch<128>(ctx, w, a, m, st_);
        if (r != HS_OK) return r;
        prof_end(ctx, st_, HS_KERNEL_TRSM, (double)m * 2.0 * bsz * bb, 4.0 * m * bb * 4.0);
        return HS_OK;
    };
    // trailing update with panels k .. k + npanels - 1 (slot sets set0 ..) of the
    // columns from c0 on: part 1 = column c0, part 2 = the columns after it, part 0 =
    // both, part 3 = columns c0 .. c0 + ncols - 1.  ctr >= 0: tiles from that counter.
    auto update = [&](int k, int npanels, int c0, int part, int ncols, int set0, cudaStream_t st_, int cap,
                      int ctr) -> hs_status {
        TcArgs a = base;
        a.k = k;
        a.blockID = diag_id(k);
        a.npanels = npanels;
        a.unit_panels = acc_panels < npanels ? acc_panels : npanels;
        a.first_col = c0;
        a.part = part;
        a.ncols = ncols;
        a.set0 = set0;
        a.tile_ctr = ctr >= 0 ? w.tile_ctr + ctr : nullptr;
        // the part's columns hold hi, hi - 1, ..., lo blocks (diagonal block included)
        const int m = nb - c0;
        const int hi = part == 2 ? m - 1 : m;
        const int lo = part == 1 ? m : (part == 3 ? m - ncols + 1 : 1);
        const double cols = hi - lo + 1.0, blocks = cols * (hi + lo) / 2.0, np = npanels;
        // the second launch of a shared update: its tiles are counted with the first
        const bool joining = st_ != s && ctr >= 0;
        const double flops = joining ? 0.0 : np * ((blocks - cols) * 2.0 * n3 + cols * bsz * bsz * (bsz + 1.0));
        const double bytes = joining ? 0.0 : (blocks * 2.0 + 2.0 * np * m) * bb * 4.0;
        const int pk = st_ == s ? HS_KERNEL_UPDATE : HS_KERNEL_UPDATE_SIDE;
        prof_begin(ctx, st_, pk);
        hs_status r = bsz == 256 ? tc_update_launch<256>(ctx, w, a, precision, st_, cap)
                                 : tc_update_launch<128>(ctx, w, a, precision, st_, cap);
        if (r != HS_OK) return r;
        prof_end(ctx, st_, pk, flops, bytes);
        return HS_OK;
    };
    // panels k .. k+g-1 of a group whose first diagonal block is factored, with the
    // updates and chains between them
    auto in_group = [&](int k, int g, int bank, cudaStream_t st_, int cap) -> hs_status {
        hs_status r;
        for (int i = 0; i < g; ++i) {
            if ((r = panel(k + i, kPanelGroup * bank + i, st_)) != HS_OK) return r;
            if (i + 1 < g) {
                if ((r = update(k, i + 1, k + i + 1, 1, 1, kPanelGroup * bank, st_, cap, -1)) != HS_OK) return r;
                if ((r = diag_chain(k + i + 1, st_)) != HS_OK) return r;
            }
        }
        return HS_OK;
    };
    if ((st = diag_chain(0, s)) != HS_OK) return st;
    bool ready = false;  // the group at k has been factored ahead
    for (int k = 0, bank = 0; k < nb - 1; bank ^= 1) {
        // precondition: column k has seen every panel before it and its diagonal
        // block is factored
        const int g = kPanelGroup < nb - 1 - k ? kPanelGroup : nb - 1 - k;
        const int set0 = kPanelGroup * bank;
        if (!ready && (st = in_group(k, g, bank, s, ctx->num_sms)) != HS_OK) return st;
        const int c0 = k + g;
        const int g2 = c0 < nb - 1 ? (kPanelGroup < nb - 1 - c0 ? kPanelGroup : nb - 1 - c0) : 0;
        const int64_t rest_rows = ctx->N - (int64_t)(c0 + g2) * bsz;  // rows after the next group
        if (group_ahead && g2 > 0 && rest_rows >= ctx->mixed_min_rows) {
            HS_REQUIRE(next_ctr < tile_counters(nb), "tile counters exhausted");
            if ((st = update(k, g, c0, 3, g2, set0, s, ctx->num_sms, -1)) != HS_OK) return st;
            HS_CUDA(cudaEventRecord(ctx->ev_a, s));
            HS_CUDA(cudaStreamWaitEvent(sd, ctx->ev_a, 0));
            if ((st = diag_chain(c0, sd)) != HS_OK) return st;
            if ((st = in_group(c0, g2, bank ^ 1, sd, side_sms)) != HS_OK) return st;
            const int ctr = next_ctr++;
            if ((st = update(k, g, c0 + g2, 0, 0, set0, s, ctx->num_sms - side_sms, ctr)) != HS_OK) return st;
            if ((st = update(k, g, c0 + g2, 0, 0, set0, sd, side_sms, ctr)) != HS_OK) return st;
            HS_CUDA(cudaEventRecord(ctx->ev_b, sd));
            HS_CUDA(cudaStreamWaitEvent(s, ctx->ev_b, 0));
            ready = true;
        } else {
            if ((st = update(k, g, c0, 1, 1, set0, s, ctx->num_sms, -1)) != HS_OK) return st;
            const bool more = c0 + 1 < nb;  // columns after c0
            const bool side = lookahead && more;
            if (side) {
                HS_CUDA(cudaEventRecord(ctx->ev_a, s));
                HS_CUDA(cudaStreamWaitEvent(sd, ctx->ev_a, 0));
                if ((st = diag_chain(c0, sd)) != HS_OK) return st;
                HS_CUDA(cudaEventRecord(ctx->ev_b, sd));
            }
            if (more && (st = update(k, g, c0, 2, 0, set0, s, side ? ctx->num_sms - kFree : ctx->num_sms, -1)) !=
                            HS_OK)
                return st;
            if (side) {
                HS_CUDA(cudaStreamWaitEvent(s, ctx->ev_b, 0));
            } else if ((st = diag_chain(c0, s)) != HS_OK) {
                return st;
            }
            ready = false;
        }
        k = c0;
    }
    return HS_OK;
}

hs_status mixed_check_error(hs_ctx ctx, const MixedWork& w) {
    int e[2] = {0, 0};
    HS_CUDA(cudaMemcpy(e, w.err, sizeof(e), cudaMemcpyDeviceToHost));
    if (e[0]) {
        set_error("mixed-precision factor: a tensor-core tile gave up waiting for its operands (timeout)");
        return HS_ERR_TIMEOUT;
    }
    if (e[1]) {
        set_error("mixed-precision solve: a triangular sweep gave up waiting for a block row (timeout)");
        return HS_ERR_TIMEOUT;
    }
    (void)ctx;
    return HS_OK;
}

}  // namespace hs
