// Device-side building blocks shared by the factorisation and the solves: the front descriptors, the FP64 tensor-core
// tile product (mma.sync m8n8k4 .f64, the FP64 MMA path of sm_100a) and small helpers.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace oosgpu::device
{

// One supernode's front (the multifrontal factorisation of the reference, MultifrontalDriver.cpp:257-344): its panel
// (c + r rows by c columns, column-major, leading dimension c + r) in the factor's value array, its update matrix
// (r by r, column-major, leading dimension r, lower triangle) in the update arena, its rows R(s) (and their positions
// in its parent's front) at rowStart in the row arrays.
struct FrontDesc
{
    std::int64_t panel;
    std::int64_t update;
    std::int64_t rowStart;
    std::int32_t first;
    std::int32_t c;
    std::int32_t r;
    std::int32_t childStart;
    std::int32_t childCount;
    std::int32_t parent;
};

// A 64 x 64 output tile of a batched product: front, first row, first column (meaning set by the launch).
struct TileTask
{
    std::int32_t front;
    std::int32_t i0;
    std::int32_t j0;
    std::int32_t k0;
};

// A range of a front's columns assembled by one block.
struct AssemblyTask
{
    std::int32_t front;
    std::int32_t j0;
    std::int32_t j1;
    std::int32_t pad;
};

constexpr int TILE = 64;
constexpr int MIXED_TILE = 128; // the tiles of the mixed-precision (tcgen05) update matrices
// Shared-memory row strides of the tiles: 68 doubles, 4 more than a multiple of 16, so that the m8n8k4 fragment loads
// (lanes 4 apart differ by one row) hit 16 distinct 8-byte banks in each half-warp.
constexpr int TILE_PAD = 4;
// The row stride of a staged 64 x 64 inverse block read as an m8n8k4 operand (either orientation): conflict-free too.
constexpr int INVERSE_LD = TILE + TILE_PAD;
constexpr int TILE_THREADS = 128;
// The columns of a macro panel of the factorisation: the 64-column steps inside it update its own later columns, and
// once it is done it updates the rest of the front's panel in one product of K = PANEL_MACRO.
constexpr int PANEL_MACRO = 256;
// The staged extend-add (assembleStaged): a piece of a front is STAGE_COLUMNS columns by up to STAGE_ROWS front
// positions, built in STAGE_SMEM bytes of shared memory (two blocks per SM).
constexpr int STAGE_COLUMNS = 32;
constexpr int STAGE_ROWS = 384;
constexpr int STAGE_THREADS = 256;
constexpr std::size_t STAGE_SMEM = static_cast<std::size_t>(STAGE_COLUMNS) * STAGE_ROWS * sizeof(double);
// The TMA-fed update-matrix kernel (updateMatrixTma): 128 x 128 tiles, 16 warps, UPDATE_STAGES stages of UPDATE_SLICE
// columns of K (A and B: 32 KB a stage), plus 1 KB to align the stages to the 128-byte swizzle's 1024-byte atoms.
constexpr int UPDATE_TILE = 128;
constexpr int UPDATE_THREADS = 512;
constexpr int UPDATE_STAGES = 4;
constexpr int UPDATE_SLICE = 16;
constexpr std::size_t UPDATE_TMA_SMEM = static_cast<std::size_t>(UPDATE_STAGES) * 2 * UPDATE_TILE * UPDATE_SLICE *
                                            sizeof(double) + 1024;
// panelRowsInverse: the 64-row halves of one task (a task covers TILE * PANEL_ROW_HALVES rows below the block).
constexpr int PANEL_ROW_HALVES = 1;
// The rows of R(s) one block of the backward product x_F -= L21^T X[R(s)] takes; longer R(s) are split into chunks
// whose partial products are summed in chunk order.
constexpr int SOLVE_ROWS_CHUNK = 512;

__device__ __forceinline__ void dmma8x8x4(double (&d)[2], double a, double b)
{
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

__device__ __forceinline__ bool isBadPivot(double d)
{
    return d == 0.0 || !isfinite(d);
}

// The operands of one tile product C(ii, jj) -= sum_p A(ii, p) * B(jj, p) * d_p over p < K, for ii < m, jj < n:
//   A(ii, p) = a[ii * aRowStride + p * aColStride]
//   B(jj, p) = b[rowOf(p) * bRowStride... ] expressed as b[jj * bRowStride + bRow(p) * bColStride]
//   d_p      = d[p * dStride] (d null: 1)
//   C(ii, jj) = c[ii * cRowStride + jj * cColStride], written where the mask keeps it:
//   lowerOffset >= -TILE... : keep (ii + lowerOffset >= jj) when lower is set.
// bIndex, when not null, maps p to the row index fed to bColStride (a gathered B).
struct TileOperands
{
    const double* a;
    std::int64_t aRowStride;
    std::int64_t aColStride;
    const double* b;
    std::int64_t bRowStride;
    std::int64_t bColStride;
    const std::int32_t* bIndex;
    const double* d;
    std::int64_t dStride;
    double* c;
    std::int64_t cRowStride;
    std::int64_t cColStride;
    int m;
    int n;
    int k;
    bool lower;
    int lowerOffset;
};

// The K pipeline of tileProduct: TILE_STAGES slices of TILE_SLICE columns of K in flight, each slice holding A and B
// (TILE_SLICE rows of TILE + TILE_PAD doubles) and the slice's d values.
constexpr int TILE_SLICE = 8;
constexpr int TILE_STAGES = 4;
constexpr int NARROW_COLUMNS = 16; // a product with at most this many columns of C runs narrow (tileAccumulate)
constexpr int TILE_STAGE_DOUBLES = 2 * TILE_SLICE * (TILE + TILE_PAD) + TILE_SLICE;
constexpr int TILE_SMEM_DOUBLES = TILE_STAGES * TILE_STAGE_DOUBLES; // 37,120 bytes

// An 8-byte asynchronous copy global -> shared; zero-filled (nothing read) when `valid` is false.
__device__ __forceinline__ void copyAsync8(double* sharedDst, const double* globalSrc, bool valid)
{
    const unsigned dst = static_cast<unsigned>(__cvta_generic_to_shared(sharedDst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(globalSrc), "r"(valid ? 8 : 0)
                 : "memory");
}

// A 16-byte asynchronous copy global -> shared through L2 only (both addresses 16-byte aligned); zero-filled when
// `valid` is false.
__device__ __forceinline__ void copyAsync16(double* sharedDst, const double* globalSrc, bool valid)
{
    const unsigned dst = static_cast<unsigned>(__cvta_generic_to_shared(sharedDst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(globalSrc), "r"(valid ? 16 : 0)
                 : "memory");
}

__device__ __forceinline__ void commitAsyncCopies()
{
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}

template <int PENDING> __device__ __forceinline__ void waitAsyncCopies()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(PENDING) : "memory");
}

// The accumulators of one thread: acc[mi][ni][h] is element (tileRow(mi), tileColumn(ni, h)) of the 64 x 64 tile.
using TileAccumulators = double[4][4][2];

__device__ __forceinline__ int tileRow(int mi)
{
    return ((threadIdx.x >> 5) >> 1) * 32 + mi * 8 + ((threadIdx.x & 31) >> 2);
}

__device__ __forceinline__ int tileColumn(int ni, int h)
{
    return ((threadIdx.x >> 5) & 1) * 32 + ni * 8 + (threadIdx.x & 3) * 2 + h;
}

// One 64 x 64 tile on a block of TILE_THREADS threads (4 warps of 32 x 32): acc = A B (D) over the K range of `op`
// (op.c and op.lower unused). The K loop streams slices of A and B (TILE_SLICE deep) and of d into shared memory by
// asynchronous copies, TILE_STAGES slices in flight, so the loads of later slices overlap the products of the current
// one; the products run on the FP64 tensor cores (DMMA m8n8k4), each fragment of B multiplied by its d_p as it is read
// (W = B D, rounded once); ACCUMULATE: onto the values acc holds (else from zero). smem: TILE_SMEM_DOUBLES doubles. B's rows are contiguous in memory (bRowStride 1 in every
// caller); A_BY_ROWS: A's rows are contiguous along p (aColStride 1), else along the rows (aRowStride 1). Every
// asynchronous copy of the block has completed on return, but other threads may still read `smem`: synchronise before
// reusing it.
template <bool A_BY_ROWS = false, bool ACCUMULATE = false>
__device__ __forceinline__ void tileAccumulate(const TileOperands& op, double* smem, TileAccumulators& acc)
{
    constexpr int LD = TILE + TILE_PAD;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int wm = (warp >> 1) * 32;
    const int wn = (warp & 1) * 32;
    const bool scaled = op.d != nullptr;
    // A narrow product (n <= 16 columns: the solves' 8-column blocks, the edges of a panel) has only the two column
    // tiles of the even warps to fill: the odd warps take every other slice of K for the same tiles instead (the
    // slices' parities split between the pair), and hand their sums to their even partner at the end (in slice
    // order per parity, so the sums do not depend on timing).
    const bool narrow = op.n <= NARROW_COLUMNS;
    const bool helper = narrow && (warp & 1) != 0;

    if (!ACCUMULATE || helper)
    {
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
            {
                acc[mi][ni][0] = 0.0;
                acc[mi][ni][1] = 0.0;
            }
    }

    const int slices = (op.k + TILE_SLICE - 1) / TILE_SLICE;
    const auto issue = [&](int slice)
    {
        double* sA = smem + (slice % TILE_STAGES) * TILE_STAGE_DOUBLES;
        double* sB = sA + TILE_SLICE * LD;
        double* sD = sB + TILE_SLICE * LD;
        const int kbase = slice * TILE_SLICE;
#pragma unroll
        for (int q = 0; q < TILE * TILE_SLICE / TILE_THREADS; ++q)
        {
            const int e = tid + q * TILE_THREADS;
            const int ii = A_BY_ROWS ? (e / TILE_SLICE) : (e & (TILE - 1));
            const int pa = A_BY_ROWS ? (e & (TILE_SLICE - 1)) : (e / TILE);
            const int kpa = kbase + pa;
            const bool okA = kpa < op.k && ii < op.m;
            copyAsync8(sA + pa * LD + ii,
                       okA ? op.a + ii * op.aRowStride + static_cast<std::int64_t>(kpa) * op.aColStride : op.a, okA);
            const int jj = e & (TILE - 1);
            const int pb = e / TILE;
            const int kpb = kbase + pb;
            const bool okB = kpb < op.k && jj < op.n;
            const double* srcB = op.b;
            if (okB)
            {
                const std::int64_t row = op.bIndex != nullptr ? op.bIndex[kpb] : kpb;
                srcB = op.b + jj * op.bRowStride + row * op.bColStride;
            }
            if (!narrow || jj < NARROW_COLUMNS) // a narrow product reads no column of B beyond the first 16
                copyAsync8(sB + pb * LD + jj, srcB, okB);
        }
        if (tid < TILE_SLICE)
        {
            const bool okD = scaled && kbase + tid < op.k;
            copyAsync8(sD + tid, okD ? op.d + static_cast<std::int64_t>(kbase + tid) * op.dStride : op.b, okD);
        }
        commitAsyncCopies();
    };

#pragma unroll
    for (int s = 0; s < TILE_STAGES - 1; ++s)
    {
        if (s < slices)
            issue(s);
        else
            commitAsyncCopies();
    }
    for (int t = 0; t < slices; ++t)
    {
        waitAsyncCopies<TILE_STAGES - 2>();
        __syncthreads();
        if (t + TILE_STAGES - 1 < slices)
            issue(t + TILE_STAGES - 1);
        else
            commitAsyncCopies();
        const double* sA = smem + (t % TILE_STAGES) * TILE_STAGE_DOUBLES;
        const double* sB = sA + TILE_SLICE * LD;
        const double* sD = sB + TILE_SLICE * LD;
        if (narrow)
        {
            if ((warp & 1) != (t & 1))
                continue; // the partner's slice
#pragma unroll
            for (int kk = 0; kk < TILE_SLICE; kk += 4)
            {
                const int pr = kk + (lane & 3);
                const double dp = scaled ? sD[pr] : 1.0;
                double fa[4];
                double fb[2];
#pragma unroll
                for (int mi = 0; mi < 4; ++mi)
                    fa[mi] = sA[pr * LD + wm + mi * 8 + (lane >> 2)];
#pragma unroll
                for (int ni = 0; ni < 2; ++ni)
                    fb[ni] = scaled ? sB[pr * LD + ni * 8 + (lane >> 2)] * dp : sB[pr * LD + ni * 8 + (lane >> 2)];
#pragma unroll
                for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                    for (int ni = 0; ni < 2; ++ni)
                        dmma8x8x4(acc[mi][ni], fa[mi], fb[ni]);
            }
            continue;
        }
#pragma unroll
        for (int kk = 0; kk < TILE_SLICE; kk += 4)
        {
            const int pr = kk + (lane & 3);
            const double dp = scaled ? sD[pr] : 1.0;
            double fa[4];
            double fb[4];
#pragma unroll
            for (int mi = 0; mi < 4; ++mi)
                fa[mi] = sA[pr * LD + wm + mi * 8 + (lane >> 2)];
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
                fb[ni] = scaled ? sB[pr * LD + wn + ni * 8 + (lane >> 2)] * dp : sB[pr * LD + wn + ni * 8 + (lane >> 2)];
#pragma unroll
            for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni)
                    dmma8x8x4(acc[mi][ni], fa[mi], fb[ni]);
        }
    }
    waitAsyncCopies<0>();
    if (narrow)
    {
        // the odd warps' sums into their even partners' tiles (the pipeline's shared memory, every stage read)
        __syncthreads();
        double* hand = smem + (warp >> 1) * (32 * 16) + lane * 16;
        if (helper)
        {
#pragma unroll
            for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                for (int ni = 0; ni < 2; ++ni)
                {
                    hand[(mi * 2 + ni) * 2] = acc[mi][ni][0];
                    hand[(mi * 2 + ni) * 2 + 1] = acc[mi][ni][1];
                }
        }
        __syncthreads();
        if (!helper)
        {
#pragma unroll
            for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                for (int ni = 0; ni < 2; ++ni)
                {
                    acc[mi][ni][0] += hand[(mi * 2 + ni) * 2];
                    acc[mi][ni][1] += hand[(mi * 2 + ni) * 2 + 1];
                }
        }
    }
}

// acc += A B on one 64 x 64 tile with both operands in shared memory (TILE_THREADS threads, the fragments of
// tileAccumulate): A(ii, p) = a[ii * lda + p], or a[p * lda + ii] when A_TRANSPOSED; B(p, jj) = b[p * ldb + jj];
// p < k, k a multiple of 4, and A and B hold zeros (not garbage) wherever a product term lies outside their extents.
// ldb = TILE + TILE_PAD keeps the B fragments free of bank conflicts.
template <bool A_TRANSPOSED>
__device__ __forceinline__ void sharedTileProduct(const double* a, int lda, const double* b, int ldb, int k,
                                                  TileAccumulators& acc)
{
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int wm = (warp >> 1) * 32;
    const int wn = (warp & 1) * 32;
#pragma unroll 4
    for (int kk = 0; kk < k; kk += 4)
    {
        const int pr = kk + (lane & 3);
        double fa[4];
        double fb[4];
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
        {
            const int ii = wm + mi * 8 + (lane >> 2);
            fa[mi] = A_TRANSPOSED ? a[pr * lda + ii] : a[ii * lda + pr];
        }
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
            fb[ni] = b[pr * ldb + wn + ni * 8 + (lane >> 2)];
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
                dmma8x8x4(acc[mi][ni], fa[mi], fb[ni]);
    }
}

// C -= A B (D) on one 64 x 64 tile (tileAccumulate), C read, reduced and written once; op.lower keeps the elements
// ii + lowerOffset >= jj only.
// The lines of C's tile (column-major: op.cRowStride 1) asked into L2 ahead of the product, so that the epilogue's
// read of C, after K columns of products, finds them there instead of in HBM.
__device__ __forceinline__ void prefetchColumnTile(const TileOperands& op)
{
    // 64 columns of up to 64 rows: 512 bytes, four 128-byte lines, per column
    const int column = threadIdx.x >> 1;
    if (op.cRowStride != 1 || column >= op.n)
        return;
    const double* top = op.c + column * op.cColStride;
    for (int line = (threadIdx.x & 1) * 2; line < (threadIdx.x & 1) * 2 + 2; ++line)
        if (line * 16 < op.m)
            asm volatile("prefetch.global.L2 [%0];\n" ::"l"(top + line * 16));
}

template <bool A_BY_ROWS = false>
__device__ __forceinline__ void tileProduct(const TileOperands& op, double* smem)
{
    TileAccumulators acc;
    if (op.k >= 2 * TILE_SLICE * TILE_STAGES)
        prefetchColumnTile(op);
    tileAccumulate<A_BY_ROWS>(op, smem, acc);
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int h = 0; h < 2; ++h)
            {
                const int ii = tileRow(mi);
                const int jj = tileColumn(ni, h);
                if (ii < op.m && jj < op.n && (!op.lower || ii + op.lowerOffset >= jj))
                {
                    double* target = op.c + ii * op.cRowStride + jj * op.cColStride;
                    *target = *target - acc[mi][ni][h];
                }
            }
}

} // namespace oosgpu::device
