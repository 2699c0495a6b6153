// The kernels of the solves with a positive definite supernodal factor: X = L^-T D^-1 L^-1 B, forward over the
// supernodes children first, then the diagonal, then backward (FactorSolve.cpp:31-158).
//
// The right-hand sides are held by rows on the device (the values of an equation for the tile's columns contiguous,
// as the reference's row-stored blocks, FactorSolve.hpp): X[eq * width + col]. The forward sweep is multifrontal: a
// supernode receives its children's update rows (in increasing child order, each row's sum fixed), eliminates its own
// rows and leaves the update rows of R(s) for its parent, so no two supernodes write one value and the sums do not
// depend on the scheduling. The backward sweep gathers the solved rows R(s) and substitutes back.
//
// Small supernodes (c <= 64) run one block each; the larger ones of a level run as one launch of dataflow tasks, one
// per 64-row block (the chains, below), their products on the FP64 tensor cores.

#include "kernels.cuh"

#include <cstdint>

namespace oosgpu::device
{


constexpr int SOLVE_BLOCK = 64;

// g += the children's update rows that land at the slots of a tile's rows (slotOf(ii) for the rows ii < rows, all
// width columns), element (tileRow(mi), tileColumn(ni, h)) of the tile in g[mi][ni][h] as the tile products hold it.
// The rows are added in rounds (the k-th entry of every row's gather list in round k), so each value takes its
// children in increasing order and every round's loads are independent of each other.
template <typename SlotOf>
__device__ __forceinline__ void gatherTile(const SolveArgs& a, int rows, SlotOf slotOf, TileAccumulators& g)
{
    std::int64_t next[4];
    std::int64_t end[4];
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
    {
        const int ii = tileRow(mi);
        next[mi] = 0;
        end[mi] = 0;
        if (ii < rows)
        {
            const std::int64_t slot = slotOf(ii);
            next[mi] = a.gatherStart[slot];
            end[mi] = a.gatherStart[slot + 1];
        }
    }
    for (;;)
    {
        std::int64_t row[4];
        bool any = false;
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
        {
            row[mi] = next[mi] < end[mi] ? a.gatherRows[next[mi]] : -1;
            any = any || row[mi] >= 0;
            ++next[mi];
        }
        if (!any)
            break;
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
        {
            if (row[mi] < 0)
                continue;
            const double* source = a.updates + row[mi] * a.width;
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                for (int h = 0; h < 2; ++h)
                {
                    const int jj = tileColumn(ni, h);
                    if (jj < a.width)
                        g[mi][ni][h] += source[jj];
                }
        }
    }
}

// The gather slot of column position p < c of a supernode (in pivot order after an indefinite factorisation), and of
// its update row k.
__device__ __forceinline__ std::int64_t columnSlot(const SolveArgs& a, const FrontDesc& f, int p)
{
    return a.perm != nullptr ? a.perm[f.first + p] : f.first + p;
}

__device__ __forceinline__ std::int64_t rowSlot(const SolveArgs& a, const FrontDesc& f, int k)
{
    return a.dimension + f.rowStart + k;
}

// The columns of a small supernode rounded up to the product's K step (4), and the leading dimension of the
// x_F block in shared memory (conflict-free B fragments).
__device__ __forceinline__ int roundFour(int c)
{
    return (c + 3) & ~3;
}
constexpr int XF_LD = TILE + TILE_PAD;

// The strict lower triangle of a small supernode's L11^-1 (c <= 64) from the strict upper triangle of its diagonal
// block: inv[i * smallInverseLd(c4) + q] = L11^-1(i, q) for q < i < c, zero elsewhere in the c4 x c4 square (c4 = c
// rounded up to 4); asynchronous copies, committed by the caller. The region holds smallInverseDoubles(c4) doubles, so that the
// product's fragment reads of rows up to 63 stay inside it.
__device__ __forceinline__ void stageSmallInverse(const double* panel, std::int64_t n, int c, double* inv)
{
    const int c4 = roundFour(c);
    for (int e = threadIdx.x; e < c4 * c4; e += blockDim.x)
    {
        const int i = e / c4;
        const int q = e - i * c4;
        const bool inside = q < i && i < c;
        copyAsync8(inv + i * smallInverseLd(c4) + q, inside ? panel + q + static_cast<std::int64_t>(i) * n : panel,
                   inside);
    }
}

// Forward sweep of a small supernode (c <= 64), one block of TILE_THREADS: x_F <- L11^-1 (b_F + children's rows at
// F), as the product with the inverse of L11 (every value independent); then the update rows by 64-row tiles,
// u_s = (children's rows at R(s), in the children's order) - L21 x_F, the product on the FP64 tensor cores
// (tileAccumulate) and each tile written once. The children's rows come by the gather lists: every value has one
// owner thread, no barrier between children. Dynamic shared memory: smallSolveSmem(cmax, width) with cmax the launch's
// largest c. At most 128 registers, so that four blocks fit an SM (the shared memory of the narrowest class allows
// four as well): these launches wait on their loads, and the fourth block took the plate's 64-column forward sweep of
// small supernodes from 4.35 to 3.93 ms.
__global__ void __launch_bounds__(TILE_THREADS, 4) forwardSmall(SolveArgs a, const std::int32_t* list, int cmax)
{
    extern __shared__ double stage[];
    double* pipe = stage;                                      // the tile pipeline
    double* inv = stage + TILE_SMEM_DOUBLES;                   // L11^-1, c4 rows of smallInverseLd(c4)
    double* xF = inv + smallInverseDoubles(roundFour(cmax));   // c4 x XF_LD
    const FrontDesc f = a.fronts[list[blockIdx.x]];
    const int w = a.width;
    const int c = f.c;
    const std::int64_t n = f.c + f.r;
    const double* panel = a.panels + f.panel;
    double* xRows = a.x + static_cast<std::int64_t>(f.first) * w;
    stageSmallInverse(panel, n, c, inv);
    commitAsyncCopies();
    {
        TileAccumulators g;
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                for (int h = 0; h < 2; ++h)
                {
                    const int ii = tileRow(mi);
                    const int jj = tileColumn(ni, h);
                    g[mi][ni][h] = ii < c && jj < w ? xRows[ii * w + jj] : 0.0;
                }
        gatherTile(a, c, [&](int ii) { return columnSlot(a, f, ii); }, g);
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                for (int h = 0; h < 2; ++h)
                {
                    const int ii = tileRow(mi);
                    const int jj = tileColumn(ni, h);
                    if (ii < roundFour(c))
                        xF[ii * XF_LD + jj] = ii < c && jj < w ? g[mi][ni][h] : 0.0;
                }
    }
    waitAsyncCopies<0>();
    __syncthreads();
    // x_F = (I + strict lower of L11^-1) b on the tensor cores
    {
        TileAccumulators t;
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
            {
                t[mi][ni][0] = 0.0;
                t[mi][ni][1] = 0.0;
            }
        sharedTileProduct<false>(inv, smallInverseLd(roundFour(c)), xF, XF_LD, roundFour(c), t);
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                for (int h = 0; h < 2; ++h)
                {
                    const int ii = tileRow(mi);
                    const int jj = tileColumn(ni, h);
                    if (ii < c && jj < w)
                        xRows[ii * w + jj] = xF[ii * XF_LD + jj] + t[mi][ni][h];
                }
    }
    __syncthreads();
    double* own = a.updates + f.rowStart * w;
    for (int i0 = 0; i0 < f.r; i0 += TILE)
    {
        TileOperands op;
        op.a = panel + c + i0; // A(ii, p) = L(c + i0 + ii, p)
        op.aRowStride = 1;
        op.aColStride = n;
        op.b = xRows;
        op.bRowStride = 1;
        op.bColStride = w;
        op.bIndex = nullptr;
        op.d = nullptr;
        op.dStride = 0;
        op.c = nullptr;
        op.cRowStride = 0;
        op.cColStride = 0;
        op.m = min(TILE, f.r - i0);
        op.n = w;
        op.k = c;
        op.lower = false;
        op.lowerOffset = 0;
        // acc = -(children's rows) + L21 x_F; the update rows are -acc
        TileAccumulators acc;
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
            {
                acc[mi][ni][0] = 0.0;
                acc[mi][ni][1] = 0.0;
            }
        gatherTile(a, op.m, [&](int ii) { return rowSlot(a, f, i0 + ii); }, acc);
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
            {
                acc[mi][ni][0] = -acc[mi][ni][0];
                acc[mi][ni][1] = -acc[mi][ni][1];
            }
        tileAccumulate<false, true>(op, pipe, acc);
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                for (int h = 0; h < 2; ++h)
                {
                    const int ii = tileRow(mi);
                    const int jj = tileColumn(ni, h);
                    if (ii < op.m && jj < w)
                        own[static_cast<std::int64_t>(i0 + ii) * w + jj] = -acc[mi][ni][h];
                }
        __syncthreads();
    }
}

// The children's update rows gathered into the columns of supernode s, one thread per value, the children in
// increasing order (forwardGather's sums): the forward sweep's first step of a supernode whose elimination is left
// out (the trailing supernode of a partial factorisation, whose columns then hold f* = f_b - K_bi K_ii^-1 f_i).
__global__ void gatherColumns(SolveArgs a, std::int32_t s)
{
    const FrontDesc f = a.fronts[s];
    const int w = a.width;
    const std::int64_t e = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= static_cast<std::int64_t>(f.c) * w)
        return;
    const int p = static_cast<int>(e / w);
    const int col = static_cast<int>(e - static_cast<std::int64_t>(p) * w);
    const std::int64_t slot = columnSlot(a, f, p);
    double* x = a.x + static_cast<std::int64_t>(f.first + p) * w + col;
    double value = *x;
    for (std::int64_t q = a.gatherStart[slot]; q < a.gatherStart[slot + 1]; ++q)
        value += a.updates[static_cast<std::int64_t>(a.gatherRows[q]) * w + col];
    *x = value;
}

// The children's update rows of a large supernode, for the front positions [i0, j0) of a task (at most 64): added into
// X's rows of its columns (in place) and into its own update rows (which they set), by the gather lists (gatherTile):
// every value one thread, the children in increasing order, so every sum is the same whatever the split. One block
// of TILE_THREADS.
__global__ void __launch_bounds__(TILE_THREADS) forwardGather(SolveArgs a, const TileTask* tasks)
{
    const TileTask task = tasks[blockIdx.x];
    const FrontDesc f = a.fronts[task.front];
    const int w = a.width;
    const int rows = min(task.j0 - task.i0, TILE);
    double* xF = a.x + static_cast<std::int64_t>(f.first) * w;
    double* own = a.updates + f.rowStart * w;
    TileAccumulators g;
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int h = 0; h < 2; ++h)
            {
                const int p = task.i0 + tileRow(mi);
                const int jj = tileColumn(ni, h);
                g[mi][ni][h] = tileRow(mi) < rows && jj < w && p < f.c ? xF[static_cast<std::int64_t>(p) * w + jj] : 0.0;
            }
    gatherTile(a, rows,
               [&](int ii)
               {
                   const int p = task.i0 + ii;
                   return p < f.c ? columnSlot(a, f, p) : rowSlot(a, f, p - f.c);
               },
               g);
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int h = 0; h < 2; ++h)
            {
                const int p = task.i0 + tileRow(mi);
                const int jj = tileColumn(ni, h);
                if (tileRow(mi) >= rows || jj >= w)
                    continue;
                if (p < f.c)
                    xF[static_cast<std::int64_t>(p) * w + jj] = g[mi][ni][h];
                else
                    own[static_cast<std::int64_t>(p - f.c) * w + jj] = g[mi][ni][h];
            }
}

// The inverse of the unit lower diagonal block (kb <= 64 columns) of step k0 of a supernode, after each
// factorisation: one thread per column j of L11^-1 carries it through the forward substitution of e_j in registers,
// reading L11 from shared memory by broadcast; the strict lower part of L11^-1 is written transposed into the block's
// strict upper triangle (unused by the factor: L11^-1(i, j) at panel position (k0 + j, k0 + i)), where the solves'
// diagonal steps read it. The substitution is unrolled for the smallest of 8, 16, 32 or 64 columns that holds kb, so
// a supernode of a few columns costs a few terms per thread.
template <int N>
__device__ __forceinline__ void invertUnitLower(const double* l, int ld, int j, int kb, double* block, std::int64_t n)
{
    double x[N];
#pragma unroll
    for (int i = 0; i < N; ++i)
        x[i] = i == j ? 1.0 : 0.0;
#pragma unroll
    for (int i = 1; i < N; ++i)
    {
        double v = x[i];
#pragma unroll
        for (int q = 0; q < i; ++q)
            v -= l[q * ld + i] * x[q];
        x[i] = v;
    }
#pragma unroll
    for (int i = 1; i < N; ++i)
        if (i > j && i < kb)
            block[j + static_cast<std::int64_t>(i) * n] = x[i];
}

__global__ void __launch_bounds__(SOLVE_BLOCK) invertDiagonal(FactorArgs args, const TileTask* tasks)
{
    constexpr int LD = SOLVE_BLOCK + 1;
    __shared__ double l[SOLVE_BLOCK * LD]; // l[q * LD + i] = L(k0 + i, k0 + q), i > q; zero elsewhere below kb
    const TileTask task = tasks[blockIdx.x];
    const FrontDesc f = args.fronts[task.front];
    const std::int64_t n = f.c + f.r;
    const int k0 = task.i0;
    const int kb = min(SOLVE_BLOCK, f.c - k0);
    const int width = kb <= 8 ? 8 : kb <= 16 ? 16 : kb <= 32 ? 32 : SOLVE_BLOCK;
    double* block = args.panels + f.panel + k0 + static_cast<std::int64_t>(k0) * n;
    for (int e = threadIdx.x; e < width * width; e += blockDim.x)
    {
        const int q = e / width;
        const int i = e - q * width;
        const bool inside = q < kb && i < kb && i > q;
        copyAsync8(l + q * LD + i, inside ? block + i + static_cast<std::int64_t>(q) * n : block, inside);
    }
    commitAsyncCopies();
    waitAsyncCopies<0>();
    __syncthreads();
    const int j = threadIdx.x;
    if (j >= kb)
        return;
    if (width == 8)
        invertUnitLower<8>(l, LD, j, kb, block, n);
    else if (width == 16)
        invertUnitLower<16>(l, LD, j, kb, block, n);
    else if (width == 32)
        invertUnitLower<32>(l, LD, j, kb, block, n);
    else
        invertUnitLower<SOLVE_BLOCK>(l, LD, j, kb, block, n);
}

// Stages the strict lower triangle of the inverse of the unit lower 64 x 64 diagonal block at column k0 of a large
// supernode (kept in that block's strict upper triangle): inv[i * INVERSE_LD + q] = L11^-1(i, q) for q < i < kb.
// Asynchronous copies, committed by the caller.
__device__ __forceinline__ void stageBlockInverse(const SolveArgs& a, const FrontDesc& f, int k0, int kb, double* inv)
{
    constexpr int LD = INVERSE_LD;
    const std::int64_t n = f.c + f.r;
    const double* block = a.panels + f.panel + k0 + static_cast<std::int64_t>(k0) * n;
    for (int e = threadIdx.x; e < SOLVE_BLOCK * SOLVE_BLOCK; e += blockDim.x)
    {
        const int i = e / SOLVE_BLOCK;
        const int q = e - i * SOLVE_BLOCK;
        const bool inside = q < i && i < kb;
        copyAsync8(inv + i * LD + q, inside ? block + q + static_cast<std::int64_t>(i) * n : block, inside);
    }
}

// x = (I + strict lower of L_jj^-1) b (TRANSPOSED: its transpose) for a 64 x 64 diagonal block of a large
// supernode, b in shared memory (64 x XF_LD, zero beyond its jb rows and w columns), inv as stageBlockInverse leaves
// it; the product on the tensor cores, x written to the jb x w rows of X at xBlock. acc is scratch.
template <bool TRANSPOSED>
__device__ __forceinline__ void stepTriangle(const double* inv, const double* b, int jb, int w, double* xBlock,
                                             TileAccumulators& acc)
{
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
        {
            acc[mi][ni][0] = 0.0;
            acc[mi][ni][1] = 0.0;
        }
    sharedTileProduct<TRANSPOSED>(inv, INVERSE_LD, b, XF_LD, SOLVE_BLOCK, acc);
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int h = 0; h < 2; ++h)
            {
                const int ii = tileRow(mi);
                const int jj = tileColumn(ni, h);
                if (ii < jb && jj < w)
                    xBlock[ii * w + jj] = b[ii * XF_LD + jj] + acc[mi][ni][h];
            }
}

// The diagonal sweep: X[eq] /= d_eq.
__global__ void diagonalSweep(SolveArgs a, const double* diagonal, int dimension)
{
    const std::int64_t e = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int w = a.width;
    if (e >= static_cast<std::int64_t>(dimension) * w)
        return;
    a.x[e] = a.x[e] / diagonal[e / w];
}

__global__ void gatherDiagonal(FactorArgs args, const std::int32_t* supernodeOfColumn, int dimension, double* diagonal)
{
    const int eq = blockIdx.x * blockDim.x + threadIdx.x;
    if (eq >= dimension)
        return;
    const FrontDesc f = args.fronts[supernodeOfColumn[eq]];
    const int k = eq - f.first;
    const std::int64_t n = f.c + f.r;
    diagonal[eq] = args.panels[f.panel + k + k * n];
}

// Backward sweep of a small supernode (c <= 64), one block of TILE_THREADS: x_F <- L11^-T (x_F - L21^T X[R(s)]),
// L21^T X[R(s)] as one tile product over K = r on the FP64 tensor cores (the rows of X gathered by R(s)), the
// triangle as the product with the transposed inverse. Dynamic shared memory: smallSolveSmem(cmax, width).
__global__ void __launch_bounds__(TILE_THREADS) backwardSmall(SolveArgs a, const std::int32_t* list, int cmax)
{
    extern __shared__ double stage[];
    double* pipe = stage;                    // the tile pipeline, then x_F (c4 x XF_LD)
    double* inv = stage + TILE_SMEM_DOUBLES; // L11^-1, c4 rows of smallInverseLd(c4)
    (void)cmax;
    const FrontDesc f = a.fronts[list[blockIdx.x]];
    const int w = a.width;
    const int c = f.c;
    const std::int64_t n = f.c + f.r;
    const double* panel = a.panels + f.panel;
    double* xRows = a.x + static_cast<std::int64_t>(f.first) * w;
    stageSmallInverse(panel, n, c, inv);
    commitAsyncCopies();
    TileOperands op;
    op.a = panel + c; // A(q, i) = L(c + i, q)
    op.aRowStride = n;
    op.aColStride = 1;
    op.b = a.x;
    op.bRowStride = 1;
    op.bColStride = w;
    op.bIndex = a.rows + f.rowStart;
    op.d = nullptr;
    op.dStride = 0;
    op.c = nullptr;
    op.cRowStride = 0;
    op.cColStride = 0;
    op.m = c;
    op.n = w;
    op.k = f.r;
    op.lower = false;
    op.lowerOffset = 0;
    TileAccumulators acc;
    tileAccumulate<true>(op, pipe, acc);
    __syncthreads();
    double* xF = pipe;
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int h = 0; h < 2; ++h)
            {
                const int ii = tileRow(mi);
                const int jj = tileColumn(ni, h);
                if (ii < roundFour(c))
                    xF[ii * XF_LD + jj] = ii < c && jj < w ? xRows[ii * w + jj] - acc[mi][ni][h] : 0.0;
            }
    __syncthreads();
    // x_F = (I + strict lower of L11^-1)^T b on the tensor cores
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
        {
            acc[mi][ni][0] = 0.0;
            acc[mi][ni][1] = 0.0;
        }
    sharedTileProduct<true>(inv, smallInverseLd(roundFour(c)), xF, XF_LD, roundFour(c), acc);
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int h = 0; h < 2; ++h)
            {
                const int ii = tileRow(mi);
                const int jj = tileColumn(ni, h);
                if (ii < c && jj < w)
                    xRows[ii * w + jj] = xF[ii * XF_LD + jj] + acc[mi][ni][h];
            }
}

// x_F -= L21^T X[R(s)] for a large supernode, by tiles of 64 of its columns (A = L21^T read along its rows). A task
// covers the rows [j0, j0 + SOLVE_ROWS_CHUNK) of R(s) and writes its partial product to slot k0 when R(s) is split
// (k0 >= 0), or all of R(s) straight into x_F (k0 = -1).
__global__ void __launch_bounds__(TILE_THREADS, 5) backwardRows(SolveArgs a, const TileTask* tasks)
{
    __shared__ double smem[TILE_SMEM_DOUBLES];
    const TileTask task = tasks[blockIdx.x];
    const FrontDesc f = a.fronts[task.front];
    const std::int64_t n = f.c + f.r;
    const int w = a.width;
    TileOperands op;
    // A(ii, p) = L(c + j0 + p, i0 + ii)
    op.a = a.panels + f.panel + f.c + task.j0 + static_cast<std::int64_t>(task.i0) * n;
    op.aRowStride = n;
    op.aColStride = 1;
    op.b = a.x;
    op.bRowStride = 1;
    op.bColStride = w;
    op.bIndex = a.rows + f.rowStart + task.j0;
    op.d = nullptr;
    op.dStride = 0;
    op.c = a.x + static_cast<std::int64_t>(f.first + task.i0) * w;
    op.cRowStride = w;
    op.cColStride = 1;
    op.m = min(TILE, f.c - task.i0);
    op.n = w;
    op.k = task.k0 < 0 ? f.r : min(SOLVE_ROWS_CHUNK, f.r - task.j0);
    op.lower = false;
    op.lowerOffset = 0;
    if (task.k0 < 0)
    {
        tileProduct<true>(op, smem);
        return;
    }
    TileAccumulators acc;
    tileAccumulate<true>(op, smem, acc);
    double* partial = a.rowPartials + static_cast<std::int64_t>(task.k0) * (TILE * TILE);
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int h = 0; h < 2; ++h)
                partial[tileRow(mi) * TILE + tileColumn(ni, h)] = acc[mi][ni][h];
}

// x_F tile -= the sum of its split partial products (task: front, i0, first slot j0, chunks k0), summed in chunk order.
__global__ void __launch_bounds__(TILE_THREADS) backwardRowsReduce(SolveArgs a, const TileTask* tasks)
{
    const TileTask task = tasks[blockIdx.x];
    const FrontDesc f = a.fronts[task.front];
    const int w = a.width;
    const int m = min(TILE, f.c - task.i0);
    double* xTile = a.x + static_cast<std::int64_t>(f.first + task.i0) * w;
    const double* partials = a.rowPartials + static_cast<std::int64_t>(task.j0) * (TILE * TILE);
    for (int e = threadIdx.x; e < m * w; e += blockDim.x)
    {
        const int ii = e / w;
        const int jj = e - ii * w;
        double sum = 0.0;
        for (int q = 0; q < task.k0; ++q)
            sum += partials[static_cast<std::int64_t>(q) * (TILE * TILE) + ii * TILE + jj];
        xTile[e] -= sum;
    }
}

// ------------------------------------------------------------------------------------------------------------------
// The chains of the large supernodes. The triangular solves with a large supernode's L11 are chains of 64-row blocks:
// forward, block i needs the blocks before it (x_i = L_ii^-1 (x_i - sum_{q<i} L_iq x_q)), backward the blocks after it.
// One launch per level runs every large supernode's chain as dataflow tasks, one 64-row block each: a task streams
// its row of L through a cp.async pipeline from the start (L is constant), takes the solved blocks x_q as their ready
// flags are set, a chunk of ready blocks at a time, then applies the stored inverse of its diagonal block, stores its
// rows and sets its own flag. The forward launch also carries the update rows' blocks (u_i -= sum_q L_iq x_q), which
// wait on every block of x_F.
//
// Progress: a task takes a ticket (atomicAdd on the launch's counter) as it starts and runs the task at that place
// of the launch's list, which puts every block a task waits on earlier in the list (blocks by block index, forward;
// by distance from the last, backward; update rows last). So every task waited on has started before: it runs or has
// finished, and waits only on earlier ones itself. Every wait is bounded as well (CHAIN_WAIT_NS, CHAIN_WAIT_POLLS); a
// wait that runs out sets chainStop, which ends every other wait of the sweep at once, and chainFailed, which the host
// reads after the solve (the sweep's results are then void).
//
// The solved rows of x are written by other blocks of the launch while it runs, so they are read through L2 only
// (ld.global.cg), after the acquire of their flag; a block publishes its rows with a fence and a release store.
// Each sum runs in a fixed order (the chain's block order, each block's products in column order, the narrow
// products' two slice parities added at the end), so the result does not depend on the timing.
// ------------------------------------------------------------------------------------------------------------------

constexpr unsigned long long CHAIN_WAIT_NS = 2000000000ull; // a wait gives up after 2 s of global time
constexpr unsigned CHAIN_WAIT_POLLS = 1u << 26;              // or after this many polls

__device__ __forceinline__ int loadAcquire(const int* p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void storeRelease(int* p, int v)
{
    asm volatile("st.release.gpu.global.s32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned long long globalNanoseconds()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
    return t;
}

// One task's product: acc += sum over the chain's blocks in its order o = 0 .. count - 1 (block q = first + step * o)
// of A_q x_q, with A_q(ii, p) = a[ii * aRowStride + (64 q + p) * aColStride] for ii < m and p < kb(q) =
// min(64, c - 64 q), and x_q the rows 64 q + p of x (w values each, by rows).
struct ChainProduct
{
    const double* a;
    std::int64_t aRowStride;
    std::int64_t aColStride;
    const double* x;
    const int* flags;
    int first;
    int step;
    int count;
    int c;
    int m;
    int w;
};

// Warp 0 (all its lanes): waits (lane 0, bounded) until block o of the chain is solved, then counts the solved blocks
// after it, up to `limit`, 32 flags at a time; returns one past the last. After a wait that ran out (here or in another
// task) it returns `limit` without waiting further.
__device__ int waitReady(const ChainProduct& op, const SolveArgs& a, int o, int limit)
{
    const int lane = threadIdx.x & 31;
    int stopped = 0;
    if (lane == 0)
    {
        const int* flag = op.flags + op.first + op.step * o;
        if (loadAcquire(flag) == 0)
        {
            const unsigned long long start = globalNanoseconds();
            for (unsigned polls = 0;; ++polls)
            {
                __nanosleep(32);
                if (loadAcquire(flag) != 0)
                    break;
                if (*reinterpret_cast<volatile int*>(a.chainStop) != 0)
                {
                    stopped = 1;
                    break;
                }
                if (polls >= CHAIN_WAIT_POLLS || globalNanoseconds() - start > CHAIN_WAIT_NS)
                {
                    atomicExch(a.chainStop, 1);
                    *reinterpret_cast<volatile int*>(a.chainFailed) = 1;
                    stopped = 1;
                    break;
                }
            }
        }
    }
    if (__shfl_sync(0xffffffffu, stopped, 0) != 0)
        return limit;
    int end = o + 1;
    while (end < limit)
    {
        const int k = end + lane;
        const bool set = k < limit && loadAcquire(op.flags + op.first + op.step * k) != 0;
        const unsigned solved = __ballot_sync(0xffffffffu, set);
        if (solved != 0xffffffffu)
            return end + __ffs(~solved) - 1;
        end += 32;
    }
    return limit;
}

// Does this thread hold element (tileRow(mi), tileColumn(ni, h)) of a chain task's result? A narrow product (at most
// NARROW_COLUMNS right-hand sides) keeps it in the even warps' first two column fragments.
__device__ __forceinline__ bool chainOwner(bool narrow, int ni)
{
    return narrow ? ((threadIdx.x >> 5) & 1) == 0 && ni < 2 : true;
}

// acc = -(the task's own rows): the sums then end at -(rows - products).
__device__ __forceinline__ void chainStart(const double* rows, int m, int w, TileAccumulators& acc)
{
    const bool narrow = w <= NARROW_COLUMNS;
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int h = 0; h < 2; ++h)
            {
                const int ii = tileRow(mi);
                const int jj = tileColumn(ni, h);
                acc[mi][ni][h] = chainOwner(narrow, ni) && ii < m && jj < w ? -__ldcg(rows + ii * w + jj) : 0.0;
            }
}

// The product of a task (ChainProduct), A_BY_ROWS: A's rows run along p (aColStride 1), in the CHAIN_REGION_DOUBLES
// of shared memory at `region`; readyShared: a shared int. With an even number of right-hand sides, the slices of x
// come through the same cp.async pipeline as those of A (16-byte copies, through L2 only), issued once their block is
// known solved; with an odd number (no 16-byte alignment), the solved blocks are read a chunk at a time into a buffer
// of their own. Every asynchronous copy of the block has completed on return, and the threads are synchronised.
template <bool A_BY_ROWS>
__device__ void chainAccumulate(const ChainProduct& op, const SolveArgs& args, double* region, int* readyShared,
                                TileAccumulators& acc)
{
    constexpr int LD = CHAIN_LD;
    constexpr int SLICES_PER_BLOCK = SOLVE_BLOCK / CHAIN_SLICE;
    constexpr int A_DOUBLES = CHAIN_SLICE * LD;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int wm = (warp >> 1) * 32;
    const int wn = (warp & 1) * 32;
    const bool narrow = op.w <= NARROW_COLUMNS;
    const bool helper = narrow && (warp & 1) != 0;
    const bool pipelined = (op.w & 1) == 0 && (reinterpret_cast<std::uintptr_t>(op.x) & 15) == 0;
    const int columns = narrow ? NARROW_COLUMNS : TILE; // the columns of x the products read
    const int ldb = narrow ? NARROW_COLUMNS + TILE_PAD : LD;
    const int stageDoubles = pipelined ? A_DOUBLES + CHAIN_SLICE * ldb : A_DOUBLES;
    double* ready = region + CHAIN_STAGES * A_DOUBLES; // the unpipelined path's solved blocks
    const int chunkBlocks = CHAIN_B_DOUBLES / (SOLVE_BLOCK * ldb);
    const int slices = op.count * SLICES_PER_BLOCK;
    int readyEnd = 0; // the blocks [0, readyEnd) of the order are known solved

    // (pipelined) the columns [w, columns) of every stage's x slice stay zero: the copies write columns < w only
    if (pipelined)
        for (int e = tid; e < CHAIN_STAGES * CHAIN_SLICE * columns; e += TILE_THREADS)
        {
            const int row = e / columns;
            const int jj = e - row * columns;
            if (jj >= op.w)
                region[(row / CHAIN_SLICE) * stageDoubles + A_DOUBLES + (row % CHAIN_SLICE) * ldb + jj] = 0.0;
        }
    // block o of the order known solved (thread 0 waits; a barrier for all)
    const auto ensureReady = [&](int o)
    {
        if (o < readyEnd)
            return;
        if (warp == 0)
        {
            const int solved = waitReady(op, args, o, op.count);
            if (lane == 0)
                *readyShared = solved;
        }
        __syncthreads();
        readyEnd = *readyShared;
        __syncthreads();
    };
    const auto issue = [&](int t)
    {
        double* sA = region + (t % CHAIN_STAGES) * stageDoubles;
        const int o = t / SLICES_PER_BLOCK;
        const int q = op.first + op.step * o;
        const int kb = min(SOLVE_BLOCK, op.c - q * SOLVE_BLOCK);
        const int p0 = (t % SLICES_PER_BLOCK) * CHAIN_SLICE;
        const double* base = op.a + static_cast<std::int64_t>(q) * SOLVE_BLOCK * op.aColStride;
#pragma unroll
        for (int r = 0; r < TILE * CHAIN_SLICE / TILE_THREADS; ++r)
        {
            const int e = tid + r * TILE_THREADS;
            const int ii = A_BY_ROWS ? e / CHAIN_SLICE : (e & (TILE - 1));
            const int pp = A_BY_ROWS ? (e & (CHAIN_SLICE - 1)) : e / TILE;
            const int p = p0 + pp;
            const bool ok = ii < op.m && p < kb;
            copyAsync8(sA + pp * LD + ii,
                       ok ? base + ii * op.aRowStride + static_cast<std::int64_t>(p) * op.aColStride : op.a, ok);
        }
        if (pipelined)
        {
            // x rows 64 q + p0 + pp, w values each (pairs of 16 bytes), zero beyond the block's columns
            double* sB = sA + A_DOUBLES;
            const int pairs = op.w >> 1;
            for (int e = tid; e < CHAIN_SLICE * pairs; e += TILE_THREADS)
            {
                const int pp = e / pairs;
                const int jj = (e - pp * pairs) * 2;
                const int p = p0 + pp;
                const bool ok = p < kb;
                copyAsync16(sB + pp * ldb + jj,
                            ok ? op.x + static_cast<std::int64_t>(q * SOLVE_BLOCK + p) * op.w + jj : op.x, ok);
            }
        }
        commitAsyncCopies();
    };

#pragma unroll
    for (int t = 0; t < CHAIN_STAGES - 1; ++t)
    {
        if (t < slices)
        {
            if (pipelined)
                ensureReady(t / SLICES_PER_BLOCK);
            issue(t);
        }
        else
            commitAsyncCopies();
    }
    int oBase = 0; // (unpipelined) the blocks [oBase, oLoaded) of the order are in `ready`
    int oLoaded = 0;
    for (int t = 0; t < slices; ++t)
    {
        waitAsyncCopies<CHAIN_STAGES - 2>();
        __syncthreads();
        const int next = t + CHAIN_STAGES - 1;
        if (next < slices)
        {
            if (pipelined)
                ensureReady(next / SLICES_PER_BLOCK);
            issue(next);
        }
        else
            commitAsyncCopies();
        const int o = t / SLICES_PER_BLOCK;
        const double* sA = region + (t % CHAIN_STAGES) * stageDoubles;
        const double* sB;
        if (pipelined)
            sB = sA + A_DOUBLES;
        else
        {
            if (o >= oLoaded)
            {
                // the next solved blocks into `ready` (every thread is done with the last ones: the barrier above)
                if (warp == 0)
                {
                    const int solved = waitReady(op, args, o, min(op.count, o + chunkBlocks));
                    if (lane == 0)
                        *readyShared = solved;
                }
                __syncthreads();
                oBase = o;
                oLoaded = *readyShared;
                const int rows = (oLoaded - oBase) * SOLVE_BLOCK;
                for (int e = tid; e < rows * columns; e += TILE_THREADS)
                {
                    const int row = e / columns;
                    const int jj = e - row * columns;
                    const int q = op.first + op.step * (oBase + row / SOLVE_BLOCK);
                    const int p = row % SOLVE_BLOCK;
                    const bool inside = p < op.c - q * SOLVE_BLOCK && jj < op.w;
                    ready[row * ldb + jj] =
                        inside ? __ldcg(op.x + static_cast<std::int64_t>(q * SOLVE_BLOCK + p) * op.w + jj) : 0.0;
                }
                __syncthreads();
            }
            sB = ready + ((o - oBase) * SOLVE_BLOCK + (t % SLICES_PER_BLOCK) * CHAIN_SLICE) * ldb;
        }
        if (narrow)
        {
            if ((warp & 1) != (t & 1))
                continue; // the partner's slice
#pragma unroll
            for (int kk = 0; kk < CHAIN_SLICE; kk += 4)
            {
                const int pr = kk + (lane & 3);
                double fa[4];
                double fb[2];
#pragma unroll
                for (int mi = 0; mi < 4; ++mi)
                    fa[mi] = sA[pr * LD + wm + mi * 8 + (lane >> 2)];
#pragma unroll
                for (int ni = 0; ni < 2; ++ni)
                    fb[ni] = sB[pr * ldb + ni * 8 + (lane >> 2)];
#pragma unroll
                for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                    for (int ni = 0; ni < 2; ++ni)
                        dmma8x8x4(acc[mi][ni], fa[mi], fb[ni]);
            }
            continue;
        }
#pragma unroll
        for (int kk = 0; kk < CHAIN_SLICE; kk += 4)
        {
            const int pr = kk + (lane & 3);
            double fa[4];
            double fb[4];
#pragma unroll
            for (int mi = 0; mi < 4; ++mi)
                fa[mi] = sA[pr * LD + wm + mi * 8 + (lane >> 2)];
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
                fb[ni] = sB[pr * ldb + wn + ni * 8 + (lane >> 2)];
#pragma unroll
            for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni)
                    dmma8x8x4(acc[mi][ni], fa[mi], fb[ni]);
        }
    }
    waitAsyncCopies<0>();
    __syncthreads();
    if (narrow)
    {
        // the odd warps' sums into their even partners' (through the first stage's shared memory)
        double* hand = region + (warp >> 1) * (32 * 16) + lane * 16;
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
        __syncthreads();
    }
}

// The end of a task of x_F: b = -acc (the task's rows less the products) in shared memory (64 x XF_LD at `b`), then
// x = b + (strict lower of L_ii^-1) b (TRANSPOSED: of L_ii^-T) with the staged inverse, into the task's rows; then its
// flag. A narrow product (at most NARROW_COLUMNS right-hand sides) splits the inverse's K between the warps of a pair
// (the odd warps' half added through `scratch`, at least 1024 doubles).
template <bool TRANSPOSED>
__device__ __forceinline__ void chainFinish(const double* inv, double* b, double* scratch, int m, int w, double* rows,
                                            int* flag, TileAccumulators& acc)
{
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const bool narrow = w <= NARROW_COLUMNS;
    for (int e = threadIdx.x; e < SOLVE_BLOCK * XF_LD; e += blockDim.x)
        b[e] = 0.0;
    __syncthreads();
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int h = 0; h < 2; ++h)
            {
                const int ii = tileRow(mi);
                const int jj = tileColumn(ni, h);
                if (chainOwner(narrow, ni) && ii < m && jj < w)
                    b[ii * XF_LD + jj] = -acc[mi][ni][h];
            }
    __syncthreads();
    if (!narrow)
        stepTriangle<TRANSPOSED>(inv, b, m, w, rows, acc);
    else
    {
        const int wm = (warp >> 1) * 32;
        const int k0 = (warp & 1) * (SOLVE_BLOCK / 2);
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int ni = 0; ni < 2; ++ni)
            {
                acc[mi][ni][0] = 0.0;
                acc[mi][ni][1] = 0.0;
            }
#pragma unroll
        for (int kk = 0; kk < SOLVE_BLOCK / 2; kk += 4)
        {
            const int pr = k0 + kk + (lane & 3);
            double fa[4];
            double fb[2];
#pragma unroll
            for (int mi = 0; mi < 4; ++mi)
            {
                const int ii = wm + mi * 8 + (lane >> 2);
                fa[mi] = TRANSPOSED ? inv[pr * INVERSE_LD + ii] : inv[ii * INVERSE_LD + pr];
            }
#pragma unroll
            for (int ni = 0; ni < 2; ++ni)
                fb[ni] = b[pr * XF_LD + ni * 8 + (lane >> 2)];
#pragma unroll
            for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                for (int ni = 0; ni < 2; ++ni)
                    dmma8x8x4(acc[mi][ni], fa[mi], fb[ni]);
        }
        double* hand = scratch + (warp >> 1) * (32 * 16) + lane * 16;
        if (warp & 1)
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
        if ((warp & 1) == 0)
        {
#pragma unroll
            for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                for (int ni = 0; ni < 2; ++ni)
#pragma unroll
                    for (int h = 0; h < 2; ++h)
                    {
                        const int ii = tileRow(mi);
                        const int jj = tileColumn(ni, h);
                        if (ii < m && jj < w)
                            rows[ii * w + jj] =
                                b[ii * XF_LD + jj] + (acc[mi][ni][h] + hand[(mi * 2 + ni) * 2 + h]);
                    }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        __threadfence();
        storeRelease(flag, 1);
    }
}

// The forward chains of one level (tasks: front, first row i0, own block (-1: update rows), first flag).
__global__ void __launch_bounds__(TILE_THREADS) forwardChain(SolveArgs a, const TileTask* tasks, int slot)
{
    extern __shared__ double chainShared[];
    __shared__ int ticket[2];
    double* region = chainShared;
    double* inv = region + CHAIN_REGION_DOUBLES;
    if (threadIdx.x == 0)
        ticket[0] = atomicAdd(a.chainTickets + slot, 1);
    __syncthreads();
    const TileTask task = tasks[ticket[0]];
    const FrontDesc f = a.fronts[task.front];
    const std::int64_t n = f.c + f.r;
    const int w = a.width;
    const bool pivotRows = task.j0 >= 0;
    const int m = pivotRows ? min(TILE, f.c - task.i0) : static_cast<int>(n - task.i0 < TILE ? n - task.i0 : TILE);
    double* rows = pivotRows ? a.x + static_cast<std::int64_t>(f.first + task.i0) * w
                             : a.updates + (f.rowStart + (task.i0 - f.c)) * w;
    if (pivotRows)
    {
        stageBlockInverse(a, f, task.i0, m, inv);
        commitAsyncCopies();
    }
    TileAccumulators acc;
    chainStart(rows, m, w, acc);
    ChainProduct op;
    op.a = a.panels + f.panel + task.i0; // A(ii, p) = L(i0 + ii, 64 q + p)
    op.aRowStride = 1;
    op.aColStride = n;
    op.x = a.x + static_cast<std::int64_t>(f.first) * w;
    op.flags = a.chainFlags + task.k0;
    op.first = 0;
    op.step = 1;
    op.count = pivotRows ? task.j0 : (f.c + SOLVE_BLOCK - 1) / SOLVE_BLOCK;
    op.c = f.c;
    op.m = m;
    op.w = w;
    chainAccumulate<false>(op, a, region, ticket + 1, acc);
    if (pivotRows)
    {
        chainFinish<false>(inv, region + CHAIN_REGION_DOUBLES - SOLVE_BLOCK * XF_LD, region, m, w, rows,
                           a.chainFlags + task.k0 + task.j0, acc);
        return;
    }
    const bool narrow = w <= NARROW_COLUMNS;
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int h = 0; h < 2; ++h)
            {
                const int ii = tileRow(mi);
                const int jj = tileColumn(ni, h);
                if (chainOwner(narrow, ni) && ii < m && jj < w)
                    rows[ii * w + jj] = -acc[mi][ni][h];
            }
}

// The backward chains of one level (tasks: front, first row i0, own block, first flag), after the products with the
// rows R(s) (backwardRows): x_i = L_ii^-T (x_i - sum_{q>i} L_qi^T x_q), the blocks q from the last.
__global__ void __launch_bounds__(TILE_THREADS) backwardChain(SolveArgs a, const TileTask* tasks, int slot)
{
    extern __shared__ double chainShared[];
    __shared__ int ticket[2];
    double* region = chainShared;
    double* inv = region + CHAIN_REGION_DOUBLES;
    if (threadIdx.x == 0)
        ticket[0] = atomicAdd(a.chainTickets + slot, 1);
    __syncthreads();
    const TileTask task = tasks[ticket[0]];
    const FrontDesc f = a.fronts[task.front];
    const std::int64_t n = f.c + f.r;
    const int w = a.width;
    const int blocks = (f.c + SOLVE_BLOCK - 1) / SOLVE_BLOCK;
    const int m = min(TILE, f.c - task.i0);
    double* rows = a.x + static_cast<std::int64_t>(f.first + task.i0) * w;
    stageBlockInverse(a, f, task.i0, m, inv);
    commitAsyncCopies();
    TileAccumulators acc;
    chainStart(rows, m, w, acc);
    ChainProduct op;
    op.a = a.panels + f.panel + static_cast<std::int64_t>(task.i0) * n; // A(ii, p) = L(64 q + p, i0 + ii)
    op.aRowStride = n;
    op.aColStride = 1;
    op.x = a.x + static_cast<std::int64_t>(f.first) * w;
    op.flags = a.chainFlags + task.k0;
    op.first = blocks - 1;
    op.step = -1;
    op.count = blocks - 1 - task.j0;
    op.c = f.c;
    op.m = m;
    op.w = w;
    chainAccumulate<true>(op, a, region, ticket + 1, acc);
    chainFinish<true>(inv, region + CHAIN_REGION_DOUBLES - SOLVE_BLOCK * XF_LD, region, m, w, rows,
                      a.chainFlags + task.k0 + task.j0, acc);
}

// Column-major B (ld) <-> rows of X (width columns from column c0), by 32 x 32 tiles transposed in shared memory so
// that both the column reads and the row writes are coalesced. Block (32, 8); grid (rows / 32, width / 32).
__global__ void toRows(const double* b, std::int64_t ld, int c0, int width, int dimension, double* x,
                       const double* scale)
{
    __shared__ double tile[32][33];
    const int i0 = blockIdx.x * 32;
    const int col0 = blockIdx.y * 32;
    const int tx = threadIdx.x;
    for (int c = threadIdx.y; c < 32; c += blockDim.y)
    {
        const int col = col0 + c;
        const int i = i0 + tx;
        if (col < width && i < dimension)
            tile[c][tx] = b[static_cast<std::int64_t>(c0 + col) * ld + i] * (scale != nullptr ? scale[i] : 1.0);
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y)
    {
        const int i = i0 + r;
        const int col = col0 + tx;
        if (col < width && i < dimension)
            x[static_cast<std::int64_t>(i) * width + col] = tile[tx][r];
    }
}

__global__ void fromRows(const double* x, int c0, int width, int dimension, double* b, std::int64_t ld,
                         const double* scale)
{
    __shared__ double tile[32][33];
    const int i0 = blockIdx.x * 32;
    const int col0 = blockIdx.y * 32;
    const int tx = threadIdx.x;
    for (int r = threadIdx.y; r < 32; r += blockDim.y)
    {
        const int i = i0 + r;
        const int col = col0 + tx;
        if (col < width && i < dimension)
            tile[tx][r] = x[static_cast<std::int64_t>(i) * width + col];
    }
    __syncthreads();
    for (int c = threadIdx.y; c < 32; c += blockDim.y)
    {
        const int col = col0 + c;
        const int i = i0 + tx;
        // x + 0.0: a solved value is never -0 (the reference writes x + 0 back, SolveSweeps.cpp:448-457).
        if (col < width && i < dimension)
            b[static_cast<std::int64_t>(c0 + col) * ld + i] = tile[c][tx] * (scale != nullptr ? scale[i] : 1.0) + 0.0;
    }
}

} // namespace oosgpu::device

namespace oosgpu::device
{

// ------------------------------------------------------------------------------------------------------------------
// Iterative refinement in FP64 (the fixed-precision refinement of LAPACK xPORFS, which the reference applies to free
// bodies, include/oos/linalg/dense/IterativeRefinement.hpp:39-64): R = B - A X on the rows of a tile, with A given by
// the full symmetric pattern of its lower CSC (both triangles, each row's columns ascending, `source` the index of
// each term in the CSC's values), one warp per group of rows with the same columns, each lane its columns. For the convergence test it accumulates,
// per column, the squared 2-norms of R and B and the infinity norms of R, B and X, and the infinity norm of A (the
// largest row sum of |a_ij|): the normwise backward error ||r||_inf / (||A||_inf ||x||_inf + ||b||_inf) (Rigal and
// Gaches) and the relative residual ||r||_2 / ||b||_2 follow. norms: [0, 64) sum r^2, [64, 128) sum b^2,
// [128, 192) max |r|, [192, 256) max |b|, [256, 320) max |x|, [320] ||A||_inf.
// ------------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ void atomicMaxNonNegative(double* target, double value)
{
    // For non-negative doubles the order of their bit patterns as integers is their order.
    atomicMax(reinterpret_cast<unsigned long long*>(target), static_cast<unsigned long long>(__double_as_longlong(value)));
}

// Each warp takes a group of consecutive rows with the same columns (the DOFs of one node: at most RESIDUAL_GROUP
// rows, groupFirst[g] .. groupFirst[g + 1] - 1), groups g0, g0 + (all warps), ...; each lane holds its columns (at
// most two, width <= 64). The group's terms are read 32 at a time, one per lane (its column and each row's value),
// then passed round by shuffles, so every row of X is read once per group instead of once per row. Each row's sum
// still takes its terms in increasing column order, and each row's |a_ij| sum its lane-strided partial sums, so R
// and the norms are those of a warp per row. The norms stay in registers and reach the accumulators once at the end.
__global__ void residualRows(const std::int64_t* rowStart, const std::int32_t* columns, const std::int32_t* source,
                             const std::int32_t* groupFirst, int groups, const double* values, const double* b,
                             const double* x, double* r, int width, double* norms)
{
    constexpr unsigned FULL = 0xffffffffu;
    const int warpsPerBlock = blockDim.x >> 5;
    const int lane = threadIdx.x & 31;
    const int totalWarps = gridDim.x * warpsPerBlock;
    double sumR[2] = {0.0, 0.0};
    double sumB[2] = {0.0, 0.0};
    double maxR[2] = {0.0, 0.0};
    double maxB[2] = {0.0, 0.0};
    double maxX[2] = {0.0, 0.0};
    double maxRowSum = 0.0;
    for (int g = blockIdx.x * warpsPerBlock + (threadIdx.x >> 5); g < groups; g += totalWarps)
    {
        const int first = groupFirst[g];
        const int count = groupFirst[g + 1] - first;
        const std::int64_t begin = rowStart[first];
        const int length = static_cast<int>(rowStart[first + 1] - begin);
        double acc[RESIDUAL_GROUP][2];
        double rowSum[RESIDUAL_GROUP];
#pragma unroll
        for (int u = 0; u < RESIDUAL_GROUP; ++u)
        {
            acc[u][0] = 0.0;
            acc[u][1] = 0.0;
            rowSum[u] = 0.0;
        }
        for (int t0 = 0; t0 < length; t0 += 32)
        {
            const int t = t0 + lane;
            const bool live = t < length;
            const int myColumn = live ? columns[begin + t] : 0;
            double myValue[RESIDUAL_GROUP];
#pragma unroll
            for (int u = 0; u < RESIDUAL_GROUP; ++u)
            {
                myValue[u] = u < count && live ? values[source[rowStart[first + u] + t]] : 0.0;
                rowSum[u] += fabs(myValue[u]);
            }
            const int chunk = min(32, length - t0);
            for (int q = 0; q < chunk; ++q)
            {
                const double* xRow = x + static_cast<std::int64_t>(__shfl_sync(FULL, myColumn, q)) * width;
                const double x0 = lane < width ? xRow[lane] : 0.0;
                const double x1 = lane + 32 < width ? xRow[lane + 32] : 0.0;
#pragma unroll
                for (int u = 0; u < RESIDUAL_GROUP; ++u)
                    if (u < count) // the same on every lane
                    {
                        const double v = __shfl_sync(FULL, myValue[u], q);
                        acc[u][0] += v * x0;
                        acc[u][1] += v * x1;
                    }
            }
        }
#pragma unroll
        for (int u = 0; u < RESIDUAL_GROUP; ++u)
        {
            if (u >= count)
                break;
            double sum = rowSum[u];
            for (int offset = 16; offset > 0; offset >>= 1)
                sum += __shfl_xor_sync(FULL, sum, offset);
            maxRowSum = fmax(maxRowSum, sum);
#pragma unroll
            for (int h = 0; h < 2; ++h)
            {
                const int c = lane + 32 * h;
                if (c >= width)
                    continue;
                const std::int64_t at = static_cast<std::int64_t>(first + u) * width + c;
                const double bc = b[at];
                const double rc = bc - acc[u][h];
                r[at] = rc;
                sumR[h] += rc * rc;
                sumB[h] += bc * bc;
                maxR[h] = fmax(maxR[h], fabs(rc));
                maxB[h] = fmax(maxB[h], fabs(bc));
                maxX[h] = fmax(maxX[h], fabs(x[at]));
            }
        }
    }
#pragma unroll
    for (int h = 0; h < 2; ++h)
    {
        const int c = lane + 32 * h;
        if (c >= width)
            continue;
        atomicAdd(norms + c, sumR[h]);
        atomicAdd(norms + 64 + c, sumB[h]);
        atomicMaxNonNegative(norms + 128 + c, maxR[h]);
        atomicMaxNonNegative(norms + 192 + c, maxB[h]);
        atomicMaxNonNegative(norms + 256 + c, maxX[h]);
    }
    if (lane == 0)
        atomicMaxNonNegative(norms + 320, maxRowSum);
}

// X += R on a tile's rows.
__global__ void addRows(double* x, const double* r, std::int64_t count)
{
    const std::int64_t e = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e < count)
        x[e] += r[e];
}

} // namespace oosgpu::device
