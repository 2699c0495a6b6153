// The kernels of the solves with a positive definite supernodal factor: X = L^-T D^-1 L^-1 B, forward over the
// supernodes children first, then the diagonal, then backward (FactorSolve.cpp:31-158).
//
// The right-hand sides are held by rows on the device (the values of an equation for the tile's columns contiguous,
// as the reference's row-stored blocks, FactorSolve.hpp): X[eq * width + col]. The forward sweep is multifrontal: a
// supernode receives its children's update rows (in increasing child order, each row's sum fixed), eliminates its own
// rows and leaves the update rows of R(s) for its parent, so no two supernodes write one value and the sums do not
// depend on the scheduling. The backward sweep gathers the solved rows R(s) and substitutes back.
//
// Small supernodes (c <= 64) run one block each; larger ones run as 64-column steps of a diagonal block solve and tile
// products on the FP64 tensor cores (tileProduct).

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
// largest c.
__global__ void __launch_bounds__(TILE_THREADS) forwardSmall(SolveArgs a, const std::int32_t* list, int cmax)
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

// The rows [k0, k0 + kb) of x_F of a large supernode, kb <= SOLVE_STEP, by 64-row blocks j: b_j = x_j - L(j, <j) x_<j
// (the earlier blocks of the step, one tile product on the FP64 tensor cores), then x_j = L_jj^-1 b_j as the product
// with the stored inverse (every value independent). One block of TILE_THREADS per supernode; dynamic shared memory
// STEP_SOLVE_SMEM.
__global__ void __launch_bounds__(TILE_THREADS) forwardDiagonal(SolveArgs a, const std::int32_t* list, int k0)
{
    constexpr int LD = INVERSE_LD;
    extern __shared__ double stage[];
    double* pipe = stage;
    double* inv = stage + TILE_SMEM_DOUBLES;  // 64 x INVERSE_LD
    double* b = inv + SOLVE_BLOCK * LD;       // 64 x XF_LD
    const FrontDesc f = a.fronts[list[blockIdx.x]];
    const int w = a.width;
    const std::int64_t n = f.c + f.r;
    const int kb = min(SOLVE_STEP, f.c - k0);
    double* xStep = a.x + static_cast<std::int64_t>(f.first + k0) * w;
    for (int j0 = 0; j0 < kb; j0 += SOLVE_BLOCK)
    {
        const int jb = min(SOLVE_BLOCK, kb - j0);
        stageBlockInverse(a, f, k0 + j0, jb, inv);
        commitAsyncCopies();
        TileOperands op;
        op.a = a.panels + f.panel + (k0 + j0) + static_cast<std::int64_t>(k0) * n; // A(ii, p) = L(k0 + j0 + ii, k0 + p)
        op.aRowStride = 1;
        op.aColStride = n;
        op.b = xStep;
        op.bRowStride = 1;
        op.bColStride = w;
        op.bIndex = nullptr;
        op.d = nullptr;
        op.dStride = 0;
        op.c = nullptr;
        op.cRowStride = 0;
        op.cColStride = 0;
        op.m = jb;
        op.n = w;
        op.k = j0;
        op.lower = false;
        op.lowerOffset = 0;
        TileAccumulators acc;
        tileAccumulate(op, pipe, acc);
        double* xBlock = xStep + static_cast<std::int64_t>(j0) * w;
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                for (int h = 0; h < 2; ++h)
                {
                    const int ii = tileRow(mi);
                    const int jj = tileColumn(ni, h);
                    b[ii * XF_LD + jj] = ii < jb && jj < w ? xBlock[ii * w + jj] - acc[mi][ni][h] : 0.0;
                }
        __syncthreads();
        stepTriangle<false>(inv, b, jb, w, xBlock, acc);
        __syncthreads();
    }
}

// Step t's block applied to the rows below it: a tile of 64 rows either in x_F (i0 < c, task.k0 = 0) or in the update
// rows (i0 >= c, task.k0 = 1); C -= L(i, k0:k0+kb) x_block.
__global__ void __launch_bounds__(TILE_THREADS) forwardUpdate(SolveArgs a, const TileTask* tasks, int k0)
{
    __shared__ double smem[TILE_SMEM_DOUBLES];
    const TileTask task = tasks[blockIdx.x];
    const FrontDesc f = a.fronts[task.front];
    const std::int64_t n = f.c + f.r;
    const int w = a.width;
    const double* panel = a.panels + f.panel;
    TileOperands op;
    op.a = panel + task.i0 + static_cast<std::int64_t>(k0) * n;
    op.aRowStride = 1;
    op.aColStride = n;
    op.b = a.x + static_cast<std::int64_t>(f.first + k0) * w;
    op.bRowStride = 1;
    op.bColStride = w;
    op.bIndex = nullptr;
    op.d = nullptr;
    op.dStride = 0;
    if (task.i0 < f.c)
    {
        op.c = a.x + static_cast<std::int64_t>(f.first + task.i0) * w;
        op.m = min(TILE, f.c - task.i0);
    }
    else
    {
        op.c = a.updates + (f.rowStart + (task.i0 - f.c)) * w;
        op.m = static_cast<int>(n - task.i0 < TILE ? n - task.i0 : TILE);
    }
    op.cRowStride = w;
    op.cColStride = 1;
    op.n = w;
    op.k = min(SOLVE_STEP, f.c - k0);
    op.lower = false;
    op.lowerOffset = 0;
    tileProduct(op, smem);
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
__global__ void __launch_bounds__(TILE_THREADS) backwardRows(SolveArgs a, const TileTask* tasks)
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

// The rows [k0, k0 + kb) of x_F of a large supernode in the backward sweep, by 64-row blocks j from the last:
// b_j = x_j - L(>j, j)^T x_>j (the later blocks of the step, one tile product), then x_j = L_jj^-T b_j as the product
// with the transposed inverse. One block of TILE_THREADS per supernode; dynamic shared memory STEP_SOLVE_SMEM.
__global__ void __launch_bounds__(TILE_THREADS) backwardDiagonal(SolveArgs a, const std::int32_t* list, int k0)
{
    constexpr int LD = INVERSE_LD;
    extern __shared__ double stage[];
    double* pipe = stage;
    double* inv = stage + TILE_SMEM_DOUBLES;  // 64 x INVERSE_LD
    double* b = inv + SOLVE_BLOCK * LD;       // 64 x XF_LD
    const FrontDesc f = a.fronts[list[blockIdx.x]];
    const int w = a.width;
    const std::int64_t n = f.c + f.r;
    const int kb = min(SOLVE_STEP, f.c - k0);
    double* xStep = a.x + static_cast<std::int64_t>(f.first + k0) * w;
    for (int j0 = ((kb - 1) / SOLVE_BLOCK) * SOLVE_BLOCK; j0 >= 0; j0 -= SOLVE_BLOCK)
    {
        const int jb = min(SOLVE_BLOCK, kb - j0);
        stageBlockInverse(a, f, k0 + j0, jb, inv);
        commitAsyncCopies();
        const int later = j0 + jb;
        TileOperands op;
        // A(ii, p) = L(k0 + later + p, k0 + j0 + ii)
        op.a = a.panels + f.panel + (k0 + later) + static_cast<std::int64_t>(k0 + j0) * n;
        op.aRowStride = n;
        op.aColStride = 1;
        op.b = xStep + static_cast<std::int64_t>(later) * w;
        op.bRowStride = 1;
        op.bColStride = w;
        op.bIndex = nullptr;
        op.d = nullptr;
        op.dStride = 0;
        op.c = nullptr;
        op.cRowStride = 0;
        op.cColStride = 0;
        op.m = jb;
        op.n = w;
        op.k = kb - later;
        op.lower = false;
        op.lowerOffset = 0;
        TileAccumulators acc;
        tileAccumulate<true>(op, pipe, acc);
        double* xBlock = xStep + static_cast<std::int64_t>(j0) * w;
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                for (int h = 0; h < 2; ++h)
                {
                    const int ii = tileRow(mi);
                    const int jj = tileColumn(ni, h);
                    b[ii * XF_LD + jj] = ii < jb && jj < w ? xBlock[ii * w + jj] - acc[mi][ni][h] : 0.0;
                }
        __syncthreads();
        stepTriangle<true>(inv, b, jb, w, xBlock, acc);
        __syncthreads();
    }
}

// After step t's block is solved, its terms leave the rows above it: x_F[q] -= sum_{i in block} L(i, q) x_F[i] for
// q in a tile of [0, k0).
__global__ void __launch_bounds__(TILE_THREADS) backwardUpdate(SolveArgs a, const TileTask* tasks, int k0)
{
    __shared__ double smem[TILE_SMEM_DOUBLES];
    const TileTask task = tasks[blockIdx.x];
    const FrontDesc f = a.fronts[task.front];
    const std::int64_t n = f.c + f.r;
    const int w = a.width;
    TileOperands op;
    // A(ii, p) = L(k0 + p, i0 + ii) = panel[k0 + p + (i0 + ii) n]
    op.a = a.panels + f.panel + k0 + static_cast<std::int64_t>(task.i0) * n;
    op.aRowStride = n;
    op.aColStride = 1;
    op.b = a.x + static_cast<std::int64_t>(f.first + k0) * w;
    op.bRowStride = 1;
    op.bColStride = w;
    op.bIndex = nullptr;
    op.d = nullptr;
    op.dStride = 0;
    op.c = a.x + static_cast<std::int64_t>(f.first + task.i0) * w;
    op.cRowStride = w;
    op.cColStride = 1;
    op.m = min(TILE, k0 - task.i0);
    op.n = w;
    op.k = min(SOLVE_STEP, f.c - k0);
    op.lower = false;
    op.lowerOffset = 0;
    tileProduct<true>(op, smem);
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
