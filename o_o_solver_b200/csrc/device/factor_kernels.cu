// The kernels of the positive definite multifrontal LDL^T on the GPU, FP64 (the plain form):
//   - assembleFronts: extend-add of a level's large fronts by column ranges (FrontAssembly.cpp:166-300);
//   - smallFronts: a whole small front per block, assembled, eliminated and written out from shared memory;
//   - diagonalBlocks / panelRows / tile products: the blocked LDL^T of a large front's panel
//     (DenseBlockKernels.cpp:395-446, factorFrontWithoutPivoting), then the Schur update of its update matrix;
//   - pivotSummary: inertia, zero pivots and the MaxDiagonalRatio test over the eliminated columns
//     (MultifrontalDriver.cpp:704-817).
// Every element of a front receives its matrix entry then its children's update matrices in increasing child order,
// as in the reference; the Schur terms are summed by the FP64 tensor cores (each product fused with its sum), so the
// factor agrees with the reference's to rounding, not bit for bit.

#include "kernels.cuh"

#include <cstdint>
#include <climits>

namespace oosgpu::device
{


// The position of DOF `row` in the front of `f` (columns first, then R(s)); -1 when outside its structure.
__device__ __forceinline__ int positionInFront(const FrontDesc& f, const std::int32_t* rows, std::int32_t row)
{
    if (row < f.first)
        return -1;
    if (row < f.first + f.c)
        return row - f.first;
    const std::int32_t* r = rows + f.rowStart;
    int lo = 0;
    int hi = f.r;
    while (lo < hi)
    {
        const int mid = (lo + hi) >> 1;
        if (r[mid] < row)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo < f.r && r[lo] == row ? f.c + lo : -1;
}

// ------------------------------------------------------------------------------------------------------------------
// Extend-add of large fronts, one block per range of front columns [j0, j1): clear, the matrix's entries in the
// supernode's columns, then each child's update matrix in increasing child order (a __syncthreads between them keeps
// every element's sum in that order).
// ------------------------------------------------------------------------------------------------------------------
__global__ void assembleFronts(FactorArgs args, const AssemblyTask* tasks, std::int32_t* structureError)
{
    const AssemblyTask task = tasks[blockIdx.x];
    const FrontDesc f = args.fronts[task.front];
    const int n = f.c + f.r;
    double* panel = args.panels + f.panel;
    double* update = args.updates + f.update;
    const int tid = threadIdx.x;
    const int threads = blockDim.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;
    const int warps = threads >> 5;

    // Clear: a panel column whole (its entries above the diagonal are the factor's zeros), an update column from its
    // diagonal down.
    for (int j = task.j0; j < task.j1; ++j)
    {
        if (j < f.c)
        {
            double* column = panel + static_cast<std::int64_t>(j) * n;
            for (int i = tid; i < n; i += threads)
                column[i] = 0.0;
        }
        else
        {
            const int t = j - f.c;
            double* column = update + static_cast<std::int64_t>(t) * f.r;
            for (int i = t + tid; i < f.r; i += threads)
                column[i] = 0.0;
        }
    }
    __syncthreads();
    // The matrix's entries of the supernode's columns in range.
    const int lastEntryColumn = min(task.j1, f.c);
    for (int j = task.j0 + warp; j < lastEntryColumn; j += warps)
    {
        const std::int32_t column = f.first + j;
        const std::int64_t begin = args.colOffsets[column];
        const std::int64_t end = args.colOffsets[column + 1];
        double* target = panel + static_cast<std::int64_t>(j) * n;
        for (std::int64_t k = begin + lane; k < end; k += 32)
        {
            const std::int32_t row = args.colRows[k];
            const int position = row < column ? -1 : positionInFront(f, args.rows, row);
            if (position < 0)
            {
                atomicMin(structureError, column);
                continue;
            }
            target[position] += args.colValues[k];
        }
    }
    __syncthreads();
    // The children's update matrices, one after the other.
    __shared__ int range[2];
    for (int q = 0; q < f.childCount; ++q)
    {
        const std::int32_t child = args.children[f.childStart + q];
        const FrontDesc ch = args.fronts[child];
        if (ch.r == 0)
            continue;
        const std::int32_t* map = args.relpos + ch.rowStart;
        if (tid == 0)
        {
            // The child's columns whose positions fall in [j0, j1) (positions increase with the rows).
            int lo = 0;
            int hi = ch.r;
            while (lo < hi)
            {
                const int mid = (lo + hi) >> 1;
                if (map[mid] < task.j0)
                    lo = mid + 1;
                else
                    hi = mid;
            }
            int lo2 = lo;
            int hi2 = ch.r;
            while (lo2 < hi2)
            {
                const int mid = (lo2 + hi2) >> 1;
                if (map[mid] < task.j1)
                    lo2 = mid + 1;
                else
                    hi2 = mid;
            }
            range[0] = lo;
            range[1] = lo2;
        }
        __syncthreads();
        const int begin = range[0];
        const int end = range[1];
        const double* source = args.updates + ch.update;
        for (int jc = begin + warp; jc < end; jc += warps)
        {
            const int pj = map[jc];
            const double* column = source + static_cast<std::int64_t>(jc) * ch.r;
            if (pj < f.c)
            {
                double* target = panel + static_cast<std::int64_t>(pj) * n;
                for (int ic = jc + lane; ic < ch.r; ic += 32)
                    target[map[ic]] += column[ic];
            }
            else
            {
                double* target = update + static_cast<std::int64_t>(pj - f.c) * f.r - f.c;
                for (int ic = jc + lane; ic < ch.r; ic += 32)
                    target[map[ic]] += column[ic];
            }
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------------------------------------------------------
// Small fronts: one block per front of order n <= maxOrder, the lower triangle of the front in shared memory (packed by
// columns, then R(s) for the searches of the assembly): assembled, then
//   - the c columns eliminated right-looking within the panel (columns < c): l_ik = a_ik / d_k, a_ij -= l_ik (l_jk d_k);
//   - the update matrix, U_ij = a_ij - sum_k l_ik (l_jk d_k) for k = 0, 1, ..., c - 1, each element by one thread
//     straight into global memory (no barrier between the terms).
// Every element receives its terms in k order with the same products as the reference's unblocked algorithm.
// ------------------------------------------------------------------------------------------------------------------
__global__ void smallFronts(FactorArgs args, const std::int32_t* list, std::int32_t* structureError)
{
    extern __shared__ double front[];
    const std::int32_t s = list[blockIdx.x];
    const FrontDesc f = args.fronts[s];
    const int n = f.c + f.r;
    const int c = f.c;
    // element (i, j), i >= j, of the packed lower triangle
    const auto at = [n](int i, int j) { return j * n - ((j * (j - 1)) >> 1) + (i - j); };
    const int tid = threadIdx.x;
    const int threads = blockDim.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;
    const int warps = threads >> 5;
    const int packed = n * (n + 1) / 2;
    std::int32_t* rows = reinterpret_cast<std::int32_t*>(front + packed);

    for (int e = tid; e < packed; e += threads)
        front[e] = 0.0;
    for (int e = tid; e < f.r; e += threads)
        rows[e] = args.rows[f.rowStart + e];
    __syncthreads();
    for (int j = warp; j < c; j += warps)
    {
        const std::int32_t column = f.first + j;
        const std::int64_t begin = args.colOffsets[column];
        const std::int64_t end = args.colOffsets[column + 1];
        for (std::int64_t k = begin + lane; k < end; k += 32)
        {
            const std::int32_t row = args.colRows[k];
            int position = -1;
            if (row >= column)
            {
                if (row < f.first + c)
                    position = row - f.first;
                else
                {
                    int lo = 0;
                    int hi = f.r;
                    while (lo < hi)
                    {
                        const int mid = (lo + hi) >> 1;
                        if (rows[mid] < row)
                            lo = mid + 1;
                        else
                            hi = mid;
                    }
                    position = lo < f.r && rows[lo] == row ? c + lo : -1;
                }
            }
            if (position < 0)
            {
                atomicMin(structureError, column);
                continue;
            }
            front[at(position, j)] += args.colValues[k];
        }
    }
    __syncthreads();
    for (int q = 0; q < f.childCount; ++q)
    {
        const FrontDesc ch = args.fronts[args.children[f.childStart + q]];
        const std::int32_t* map = args.relpos + ch.rowStart;
        const double* source = args.updates + ch.update;
        for (int jc = warp; jc < ch.r; jc += warps)
        {
            const int pj = map[jc];
            const double* column = source + static_cast<std::int64_t>(jc) * ch.r;
            for (int ic = jc + lane; ic < ch.r; ic += 32)
                front[at(map[ic], pj)] += column[ic];
        }
        __syncthreads();
    }
    // The panel: the c columns eliminated, each step updating the later panel columns only.
    for (int k = 0; k < c; ++k)
    {
        const double pivot = front[at(k, k)];
        if (isBadPivot(pivot))
        {
            if (tid == 0)
                atomicMin(args.zeroPivot + s, k);
        }
        for (int i = k + 1 + tid; i < n; i += threads)
            front[at(i, k)] = front[at(i, k)] / pivot;
        __syncthreads();
        for (int j = k + 1 + warp; j < c; j += warps)
        {
            const double w = front[at(j, k)] * pivot;
            for (int i = j + lane; i < n; i += 32)
                front[at(i, j)] -= front[at(i, k)] * w;
        }
        __syncthreads();
    }
    double* panel = args.panels + f.panel;
    for (int e = tid; e < n * c; e += threads)
    {
        const int j = e / n;
        const int i = e - j * n;
        panel[e] = i >= j ? front[at(i, j)] : 0.0;
    }
    // The update matrix: a warp per column, a lane per row (four rows in flight), the c terms of each element in order.
    if (f.r > 0)
    {
        double* update = args.updates + f.update;
        const int r = f.r;
        for (int jj = warp; jj < r; jj += warps)
        {
            const int j = c + jj;
            for (int i0 = jj + lane; i0 < r; i0 += 128)
            {
                double acc[4];
#pragma unroll
                for (int u = 0; u < 4; ++u)
                {
                    const int ii = i0 + 32 * u;
                    acc[u] = ii < r ? front[at(c + ii, j)] : 0.0;
                }
                for (int k = 0; k < c; ++k)
                {
                    const double w = front[at(j, k)] * front[at(k, k)];
#pragma unroll
                    for (int u = 0; u < 4; ++u)
                    {
                        const int ii = i0 + 32 * u;
                        if (ii < r)
                            acc[u] -= front[at(c + ii, k)] * w;
                    }
                }
#pragma unroll
                for (int u = 0; u < 4; ++u)
                {
                    const int ii = i0 + 32 * u;
                    if (ii < r)
                        update[ii + static_cast<std::int64_t>(jj) * r] = acc[u];
                }
            }
        }
    }
}

// ------------------------------------------------------------------------------------------------------------------
// Blocked elimination of a large front's panel, step t (columns [k0, k0 + kb), k0 = 64 t):
//   diagonalBlocks: the kb x kb diagonal block eliminated in shared memory by one block per front;
//   panelRowsInverse: the rows below it, L(i, :) = A(i, :) L11^-T D^-1, as a product with the block's inverse on the
//              FP64 tensor cores, one block per front and 128 rows;
//   trailing panel update and final update-matrix SYRK: tile products (tileProduct).
// ------------------------------------------------------------------------------------------------------------------
constexpr int BLOCK = 64;
constexpr int INVERSE_SUB = 16; // the blocks of the diagonal block's inverse

// The diagonal block's LDL^T and the inverse of its unit lower factor, in shared memory by DIAGONAL_THREADS threads
// with loops kept rolled: a single block runs at the top of the tree, where every instruction is fetched once, so the
// code stays small enough for the instruction cache (a fully unrolled register version stalled on instruction fetch).
//   elimination: for k = 0, 1, ...: l_ik = a_ik / d_k, then a_ij -= l_ik (l_jk d_k) for k < j <= i, each element's
//   terms in k order as the reference's unblocked algorithm, one barrier per column;
//   inverse: X = L11^-1 by 16 x 16 blocks (the diagonal blocks by substitution, one thread per column, then the
//   off-diagonal blocks by block diagonals: eight barrier phases in all), kept in the strict upper triangle
//   (X(i, j) at (j, i)), where panelRowsInverse and the solves read it.
__global__ void __launch_bounds__(DIAGONAL_THREADS) diagonalBlocksByColumn(FactorArgs args, const std::int32_t* list,
                                                                          int k0)
{
    constexpr int LD = BLOCK + 1;
    constexpr int PARTS = DIAGONAL_THREADS / BLOCK;
    __shared__ double a[BLOCK * LD];
    __shared__ double scaled[2][BLOCK];      // w_j = l_jk d_k of step k in scaled[k & 1]
    // products T of the inverse's off-diagonal blocks (at most three 16 x 16 blocks at a time)
    __shared__ double products[(BLOCK / INVERSE_SUB - 1) * INVERSE_SUB * INVERSE_SUB];
    const std::int32_t s = list[blockIdx.x];
    const FrontDesc f = args.fronts[s];
    const int n = f.c + f.r;
    const int kb = min(BLOCK, f.c - k0);
    double* panel = args.panels + f.panel + static_cast<std::int64_t>(k0) * n + k0;
    const int t = threadIdx.x;
    for (int e = t; e < BLOCK * BLOCK; e += DIAGONAL_THREADS)
    {
        const int j = e / BLOCK;
        const int i = e - j * BLOCK;
        const bool inside = i < kb && j < kb;
        copyAsync8(a + i + j * LD, inside ? panel + i + static_cast<std::int64_t>(j) * n : panel, inside);
    }
    commitAsyncCopies();
    waitAsyncCopies<0>();
    __syncthreads();
    const int row = t & (BLOCK - 1);
    const int part = t / BLOCK;
    // Column 0: l_i0 = a_i0 / d_0 and the scaled values w_i = l_i0 d_0.
    if (t == 0 && kb > 0 && isBadPivot(a[0]))
        atomicMin(args.zeroPivot + s, k0);
    if (t > 0 && t < kb)
    {
        const double pivot = a[0];
        const double l = a[t] / pivot;
        a[t] = l;
        scaled[0][t] = l * pivot;
    }
    __syncthreads();
    // Step k, one barrier: the rows below k take column k's terms, a_ij -= l_ik w_j (thread (row, part): the columns
    // j = k + 1 + part, k + 1 + part + PARTS, ... of its row), and column k + 1 is finished in the same phase: the
    // thread holding a_{i,k+1} (part 0) forms the pivot d_{k+1} = a_{k+1,k+1} - l_{k+1,k} w_{k+1} itself (every one
    // of them from the same values, so the same bits; the pivot's own thread leaves a_{k+1,k+1} unchanged in this
    // step and stores d_{k+1} at the start of the next), then l_{i,k+1} = a_{i,k+1} / d_{k+1} and its scaled value.
    double pendingPivot = 0.0;
#pragma unroll 1
    for (int k = 0; k < kb; ++k)
    {
        const double* w = scaled[k & 1];
        double* wNext = scaled[(k + 1) & 1];
        if (k > 0 && part == 0 && row == k)
        {
            a[k + k * LD] = pendingPivot;
            if (isBadPivot(pendingPivot))
                atomicMin(args.zeroPivot + s, k0 + k);
        }
        if (row > k && row < kb)
        {
            const double l = a[row + k * LD];
#pragma unroll 4
            for (int j = k + 1 + part; j <= row; j += PARTS)
                if (j != row || j != k + 1) // the next pivot waits for its own step
                    a[row + j * LD] -= l * w[j];
            if (part == 0 && k + 1 < kb)
            {
                double pivot = a[(k + 1) + (k + 1) * LD];
                pivot -= a[(k + 1) + k * LD] * w[k + 1];
                if (row == k + 1)
                {
                    pendingPivot = pivot;
                }
                else
                {
                    const double next = a[row + (k + 1) * LD] / pivot;
                    a[row + (k + 1) * LD] = next;
                    wNext[row] = next * pivot;
                }
            }
        }
        __syncthreads();
    }
    // the inverse by 16 x 16 blocks, X(i, j) kept at (j, i)
    if (t >= kb && t < BLOCK)
        a[t + t * LD] = 1.0;
    __syncthreads();
    invertUnitLowerBlocked(a, products);
    // L and D (lower triangle) and L11^-1 (strict upper triangle) back into the panel
    for (int e = t; e < BLOCK * BLOCK; e += DIAGONAL_THREADS)
    {
        const int j = e / BLOCK;
        const int i = e - j * BLOCK;
        if (i < kb && j < kb)
            panel[i + static_cast<std::int64_t>(j) * n] = a[i + j * LD];
    }
}

// The diagonal block's LDL^T by 16-column sub-panels, and the inverse of its unit lower factor (the same results as
// diagonalBlocksByColumn, to rounding: the rows below each 16 x 16 block take their L as products with its inverse).
// For each sub-panel J (columns j0 = 16 J ...):
//   1. one warp eliminates the 16 x 16 diagonal block in registers (lane i holds row j0 + i): per column k the pivot
//      d_k is shuffled from lane k, l_ik = a_ik / d_k, w_ik = l_ik d_k, and a_ij -= l_ik w_jk for k < j <= i, w_jk
//      shuffled from lane j; then the same lanes invert the unit lower block, X_JJ = L_JJ^-1 (lane j: column j,
//      X(i, j) = -sum_{j <= q < i} L(i, q) X(q, j)), into the block's strict upper triangle (X(i, j) at (j, i));
//   2. the rows below the sub-panel: Y = A X_JJ^T on the FP64 tensor cores, then l_iq = y_iq / d_q and w_iq = y_iq;
//   3. the trailing lower triangle: A -= L W^T on the tensor cores, lower 8 x 8 tiles.
// The 64 x 64 inverse then needs only its off-diagonal 16 x 16 blocks, by block diagonals on the tensor cores:
// T_IJ = sum_{J <= K < I} L_IK X_KJ, X_IJ = -X_II T_IJ. Products of 8 x 8 tiles (DMMA m8n8k4: lane g = lane / 4
// holds row g of A and column g of B at k = lane mod 4, and results (g, 2 (lane mod 4)) and the next column), spread
// over the block's warps; beyond kb the block is the identity, so the tiles run over all 64 rows.
constexpr int DIAGONAL_LD = BLOCK + 1;                        // the block in shared memory, by columns
constexpr int DIAGONAL_W_LD = INVERSE_SUB + 1;                // rows of W apart by 17 doubles (distinct banks)
constexpr int DIAGONAL_P_BLOCK = INVERSE_SUB * (INVERSE_SUB + 1);

// The elimination of a 64 x 64 diagonal block held in shared memory (a: column-major, leading dimension 65, loaded,
// zero outside its kb x kb corner) by the DIAGONAL_THREADS threads of a block, as diagonalBlocks describes; wRows
// (64 x 17) and products (3 x 16 x 17) are its scratch. Leaves L below the diagonal, D on it and L^-1 transposed in the
// strict upper triangle; a zero or non-finite pivot recorded for supernode s.
__device__ void eliminateDiagonalBlock(const FactorArgs& args, std::int32_t s, int k0, int kb, double* a,
                                       double* wRows, double* products)
{
    constexpr int LD = DIAGONAL_LD;
    constexpr int SUB = INVERSE_SUB; // 16
    constexpr int W_LD = DIAGONAL_W_LD;
    constexpr int P_LD = SUB + 1;
    constexpr int P_BLOCK = DIAGONAL_P_BLOCK;
    const int t = threadIdx.x;
    const int lane = t & 31;
    // Beyond kb the block is the identity (its L rows are zero from the load), so the inverse stays finite.
    if (t >= kb && t < BLOCK)
        a[t + t * LD] = 1.0;
    __syncthreads();

#pragma unroll 1
    for (int j0 = 0; j0 < kb; j0 += SUB)
    {
        const int width = min(SUB, kb - j0); // columns of this sub-panel
        // 1. the 16 x 16 diagonal block and its inverse, warp 0
        if (t < 32)
        {
            const int i = lane; // row j0 + i; lanes 16..31 take part in the shuffles only
            const bool row = i < width;
            double x[SUB];
#pragma unroll
            for (int q = 0; q < SUB; ++q)
                x[q] = row && q <= i ? a[(j0 + i) + (j0 + q) * LD] : 0.0;
            // The reciprocal of each pivot by every lane, outside any branch (a division under a branch keeps the
            // row in local memory), l_ik = a_ik (1 / d_k); the pivots checked once the block is eliminated.
#pragma unroll
            for (int k = 0; k < SUB; ++k)
            {
                if (k < width)
                {
                    const double d = __shfl_sync(0xffffffffu, x[k], k);
                    const double reciprocal = 1.0 / d;
                    const double l = row && i > k ? x[k] * reciprocal : 0.0;
                    if (row && i > k)
                        x[k] = l;
                    const double w = l * d; // w_ik, for the lanes below the pivot
#pragma unroll
                    for (int j = k + 1; j < SUB; ++j)
                    {
                        const double wj = __shfl_sync(0xffffffffu, w, j);
                        if (row && j <= i)
                            x[j] = fma(-l, wj, x[j]);
                    }
                }
            }
            if (row)
            {
#pragma unroll
                for (int q = 0; q < SUB; ++q)
                    if (q <= i)
                        a[(j0 + i) + (j0 + q) * LD] = x[q];
                if (isBadPivot(a[(j0 + i) + (j0 + i) * LD]))
                    atomicMin(args.zeroPivot + s, k0 + j0 + i);
            }
            __syncwarp();
            // X = L_JJ^-1, lane j: column j (unit diagonal; rows and columns beyond width give the identity)
            if (i < SUB)
            {
                double column[SUB];
#pragma unroll
                for (int r = 0; r < SUB; ++r)
                {
                    double sum = 0.0;
#pragma unroll
                    for (int q = 0; q < r; ++q)
                        if (q >= i)
                            sum += a[(j0 + r) + (j0 + q) * LD] * column[q];
                    column[r] = r == i ? 1.0 : (r > i ? -sum : 0.0);
                    if (r > i)
                        a[(j0 + i) + (j0 + r) * LD] = column[r]; // X(r, i) at (i, r)
                }
            }
        }
        __syncthreads();
        // 2. the rows below the sub-panel: Y = A X_JJ^T (8-row tiles x 2 column halves), then L = Y / d and W = Y
        const int below = BLOCK - (j0 + SUB);
        const int g = lane >> 2;
        const int tq = lane & 3;
        const int warp = t >> 5;
        constexpr int WARPS = DIAGONAL_THREADS / 32;
        double y[2][2];
        const int rowTasks = below / 8 * 2;
        for (int u = 0; u < 2; ++u)
        {
            const int task = warp + u * WARPS;
            y[u][0] = 0.0;
            y[u][1] = 0.0;
            if (task >= rowTasks)
                continue;
            const int i0 = j0 + SUB + (task >> 1) * 8;
            const int nn = (task & 1) * 8 + g;
#pragma unroll
            for (int ks = 0; ks < SUB; ks += 4)
            {
                const int k = ks + tq;
                const double fa = a[(i0 + g) + (j0 + k) * LD];
                const double fb = nn > k ? a[(j0 + k) + (j0 + nn) * LD] : (nn == k ? 1.0 : 0.0);
                dmma8x8x4(y[u], fa, fb);
            }
        }
        __syncthreads();
        for (int u = 0; u < 2; ++u)
        {
            const int task = warp + u * WARPS;
            if (task >= rowTasks)
                continue;
            const int i = j0 + SUB + (task >> 1) * 8 + g;
#pragma unroll
            for (int h = 0; h < 2; ++h)
            {
                const int q = (task & 1) * 8 + 2 * tq + h;
                a[i + (j0 + q) * LD] = y[u][h] / a[(j0 + q) + (j0 + q) * LD];
                wRows[i * W_LD + q] = y[u][h];
            }
        }
        __syncthreads();
        // 3. the trailing lower triangle, A -= L W^T by lower 8 x 8 tiles (each tile's terms in q order on its lanes)
        const int tilesAcross = below / 8;
        for (int task = warp; task < tilesAcross * (tilesAcross + 1) / 2; task += WARPS)
        {
            int ti = 0;
            while ((ti + 1) * (ti + 2) / 2 <= task)
                ++ti;
            const int tj = task - ti * (ti + 1) / 2;
            const int i0 = j0 + SUB + ti * 8;
            const int c0 = j0 + SUB + tj * 8;
            double acc[2] = {a[(i0 + g) + (c0 + 2 * tq) * LD], a[(i0 + g) + (c0 + 2 * tq + 1) * LD]};
#pragma unroll
            for (int ks = 0; ks < SUB; ks += 4)
            {
                const int k = ks + tq;
                dmma8x8x4(acc, -a[(i0 + g) + (j0 + k) * LD], wRows[(c0 + g) * W_LD + k]);
            }
#pragma unroll
            for (int h = 0; h < 2; ++h)
                if (i0 + g >= c0 + 2 * tq + h)
                    a[(i0 + g) + (c0 + 2 * tq + h) * LD] = acc[h];
        }
        __syncthreads();
    }
    // the inverse's off-diagonal 16 x 16 blocks by block diagonals: T_IJ = sum_{J <= K < I} L_IK X_KJ, then
    // X_IJ = -X_II T_IJ (X stored transposed: X(i, j) at (j, i)); a task is one 8 x 8 quarter of a block
    const int warp = t >> 5;
    const int g = lane >> 2;
    const int tq = lane & 3;
    constexpr int WARPS = DIAGONAL_THREADS / 32;
#pragma unroll 1
    for (int d = 1; d < BLOCK / SUB; ++d)
    {
        const int tasks = (BLOCK / SUB - d) * 4;
        for (int task = warp; task < tasks; task += WARPS)
        {
            const int b = task >> 2;
            const int m0 = ((task >> 1) & 1) * 8;
            const int nn = (task & 1) * 8 + g;
            const int bj = b * SUB;
            const int bi = (b + d) * SUB;
            double acc[2] = {0.0, 0.0};
            for (int bk = bj; bk < bi; bk += SUB)
            {
#pragma unroll
                for (int ks = 0; ks < SUB; ks += 4)
                {
                    const int k = ks + tq;
                    const double fa = a[(bi + m0 + g) + (bk + k) * LD];
                    const double fb = bk > bj ? a[(bj + nn) + (bk + k) * LD]
                                              : (k > nn ? a[(bj + nn) + (bj + k) * LD] : (k == nn ? 1.0 : 0.0));
                    dmma8x8x4(acc, fa, fb);
                }
            }
#pragma unroll
            for (int h = 0; h < 2; ++h)
                products[b * P_BLOCK + (m0 + g) * P_LD + (task & 1) * 8 + 2 * tq + h] = acc[h];
        }
        __syncthreads();
        for (int task = warp; task < tasks; task += WARPS)
        {
            const int b = task >> 2;
            const int m0 = ((task >> 1) & 1) * 8;
            const int n0 = (task & 1) * 8;
            const int bj = b * SUB;
            const int bi = (b + d) * SUB;
            const int m = m0 + g;
            double acc[2] = {0.0, 0.0};
#pragma unroll
            for (int ks = 0; ks < SUB; ks += 4)
            {
                const int k = ks + tq;
                const double fa = m > k ? a[(bi + k) + (bi + m) * LD] : (m == k ? 1.0 : 0.0);
                dmma8x8x4(acc, fa, products[b * P_BLOCK + k * P_LD + n0 + g]);
            }
#pragma unroll
            for (int h = 0; h < 2; ++h)
                a[(bj + n0 + 2 * tq + h) + (bi + m) * LD] = -acc[h];
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(DIAGONAL_THREADS, 2) diagonalBlocks(FactorArgs args, const std::int32_t* list, int k0)
{
    constexpr int LD = DIAGONAL_LD;
    __shared__ double a[BLOCK * LD];
    __shared__ double wRows[BLOCK * DIAGONAL_W_LD]; // w(i, q) = y_iq of the current sub-panel
    __shared__ double products[(BLOCK / INVERSE_SUB - 1) * DIAGONAL_P_BLOCK];
    const std::int32_t s = list[blockIdx.x];
    const FrontDesc f = args.fronts[s];
    const int n = f.c + f.r;
    const int kb = min(BLOCK, f.c - k0);
    double* panel = args.panels + f.panel + static_cast<std::int64_t>(k0) * n + k0;
    const int t = threadIdx.x;
    for (int e = t; e < BLOCK * BLOCK; e += DIAGONAL_THREADS)
    {
        const int j = e / BLOCK;
        const int i = e - j * BLOCK;
        const bool inside = i < kb && j < kb;
        copyAsync8(a + i + j * LD, inside ? panel + i + static_cast<std::int64_t>(j) * n : panel, inside);
    }
    commitAsyncCopies();
    waitAsyncCopies<0>();
    __syncthreads();
    eliminateDiagonalBlock(args, s, k0, kb, a, wRows, products);
    for (int e = t; e < BLOCK * BLOCK; e += DIAGONAL_THREADS)
    {
        const int j = e / BLOCK;
        const int i = e - j * BLOCK;
        if (i < kb && j < kb)
            panel[i + static_cast<std::int64_t>(j) * n] = a[i + j * LD];
    }
}

// The rows below step k0's diagonal block, L21 = A21 L11^-T D^-1, as products on the FP64 tensor cores: for each
// 64-row half of a task (64 * PANEL_ROW_HALVES rows), Y = A21 (L11^-1)^T with L11^-1 from the block's strict upper
// triangle (unit diagonal), then l_ij = y_ij (1 / d_j), written in place (a block stages its rows before it writes
// them). The inverse and the first rows arrive in one group of asynchronous copies.
// Dynamic shared memory: PANEL_ROWS_INVERSE_SMEM bytes.
__global__ void __launch_bounds__(TILE_THREADS) panelRowsInverse(FactorArgs args, const TileTask* tasks, int k0)
{
    constexpr int LD = TILE + TILE_PAD;
    extern __shared__ double stage[];
    double* sA = stage;           // sA[p * LD + ii] = A21(ii, p)
    double* sB = sA + BLOCK * LD; // sB[p * LD + jj] = L11^-1(jj, p) for p < jj, 1 for p == jj, 0 above
    double* sd = sB + BLOCK * LD; // d_j
    const TileTask task = tasks[blockIdx.x];
    const FrontDesc f = args.fronts[task.front];
    const std::int64_t n = f.c + f.r;
    const int kb = min(BLOCK, f.c - k0);
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int wm = (warp >> 1) * 32;
    const int wn = (warp & 1) * 32;
    const double* block = args.panels + f.panel + k0 + static_cast<std::int64_t>(k0) * n;
    // The block's strict upper triangle (L11^-1 transposed) and its diagonal, by asynchronous copies; the diagonal
    // slots then become the unit diagonal of L11^-1 and everything below it zero.
    for (int e = tid; e < BLOCK * BLOCK; e += blockDim.x)
    {
        const int jj = e / BLOCK;
        const int p = e - jj * BLOCK;
        const bool inside = p <= jj && jj < kb;
        copyAsync8(sB + p * LD + jj, inside ? block + p + static_cast<std::int64_t>(jj) * n : block, inside);
    }
    // The rows of a half into sA, as asynchronous copies (the first half's in flight with the inverse's).
    const auto loadRows = [&](std::int64_t i0)
    {
        const int m = static_cast<int>(n - i0 < TILE ? n - i0 : TILE);
        const double* rows = args.panels + f.panel + i0 + static_cast<std::int64_t>(k0) * n;
        for (int e = tid; e < BLOCK * TILE; e += blockDim.x)
        {
            const int p = e / TILE;
            const int ii = e - p * TILE;
            const bool inside = p < kb && ii < m;
            copyAsync8(sA + p * LD + ii, inside ? rows + ii + static_cast<std::int64_t>(p) * n : rows, inside);
        }
    };
    if (task.i0 < n)
        loadRows(task.i0);
    commitAsyncCopies();
    waitAsyncCopies<0>();
    __syncthreads();
    // sd: 1 / d_j, applied as a product in the write-out
    for (int j = tid; j < BLOCK; j += blockDim.x)
    {
        sd[j] = j < kb ? 1.0 / sB[j * LD + j] : 1.0;
        sB[j * LD + j] = j < kb ? 1.0 : 0.0;
    }
    for (int half = 0; half < PANEL_ROW_HALVES; ++half)
    {
        const std::int64_t i0 = task.i0 + half * TILE;
        if (i0 >= n)
            break;
        const int m = static_cast<int>(n - i0 < TILE ? n - i0 : TILE);
        double* rows = args.panels + f.panel + i0 + static_cast<std::int64_t>(k0) * n;
        if (half > 0)
        {
            loadRows(i0);
            commitAsyncCopies();
            waitAsyncCopies<0>();
        }
        __syncthreads();
        double acc[4][4][2];
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
            {
                acc[mi][ni][0] = 0.0;
                acc[mi][ni][1] = 0.0;
            }
#pragma unroll 4
        for (int kk = 0; kk < BLOCK; kk += 4)
        {
            const int pr = kk + (lane & 3);
            double fa[4];
            double fb[4];
#pragma unroll
            for (int mi = 0; mi < 4; ++mi)
                fa[mi] = sA[pr * LD + wm + mi * 8 + (lane >> 2)];
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
                fb[ni] = sB[pr * LD + wn + ni * 8 + (lane >> 2)];
#pragma unroll
            for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni)
                    dmma8x8x4(acc[mi][ni], fa[mi], fb[ni]);
        }
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                for (int h = 0; h < 2; ++h)
                {
                    const int ii = wm + mi * 8 + (lane >> 2);
                    const int jj = wn + ni * 8 + (lane & 3) * 2 + h;
                    if (ii < m && jj < kb)
                        rows[ii + static_cast<std::int64_t>(jj) * n] = acc[mi][ni][h] * sd[jj];
                }
        __syncthreads();
    }
}

// Trailing panel update: the tile (i0, j0) of the panel's columns minus the products with the K = task.k0 columns from
// k0 (a 64-column step within its macro panel, or a finished macro panel of PANEL_MACRO columns).
__global__ void __launch_bounds__(TILE_THREADS, 5) panelUpdate(FactorArgs args, const TileTask* tasks, int k0)
{
    __shared__ double smem[TILE_SMEM_DOUBLES];
    const TileTask task = tasks[blockIdx.x];
    const FrontDesc f = args.fronts[task.front];
    const std::int64_t n = f.c + f.r;
    double* panel = args.panels + f.panel;
    TileOperands op;
    op.a = panel + task.i0 + static_cast<std::int64_t>(k0) * n;
    op.aRowStride = 1;
    op.aColStride = n;
    op.b = panel + task.j0 + static_cast<std::int64_t>(k0) * n;
    op.bRowStride = 1;
    op.bColStride = n;
    op.bIndex = nullptr;
    op.d = panel + k0 + static_cast<std::int64_t>(k0) * n;
    op.dStride = n + 1;
    op.c = panel + task.i0 + static_cast<std::int64_t>(task.j0) * n;
    op.cRowStride = 1;
    op.cColStride = n;
    op.m = static_cast<int>(n - task.i0 < TILE ? n - task.i0 : TILE);
    op.n = min(TILE, f.c - task.j0);
    op.k = task.k0;
    op.lower = task.i0 == task.j0;
    op.lowerOffset = 0;
    tileProduct(op, smem);
}

// The Schur update of the update matrix: U(i, j) -= sum_{k < c} L(c + i, k) d_k L(c + j, k), lower tiles.
__global__ void __launch_bounds__(TILE_THREADS) updateMatrix(FactorArgs args, const TileTask* tasks)
{
    __shared__ double smem[TILE_SMEM_DOUBLES];
    const TileTask task = tasks[blockIdx.x];
    const FrontDesc f = args.fronts[task.front];
    const std::int64_t n = f.c + f.r;
    const double* panel = args.panels + f.panel;
    TileOperands op;
    op.a = panel + f.c + task.i0;
    op.aRowStride = 1;
    op.aColStride = n;
    op.b = panel + f.c + task.j0;
    op.bRowStride = 1;
    op.bColStride = n;
    op.bIndex = nullptr;
    op.d = panel;
    op.dStride = n + 1;
    op.c = args.updates + f.update + task.i0 + static_cast<std::int64_t>(task.j0) * f.r;
    op.cRowStride = 1;
    op.cColStride = f.r;
    op.m = min(TILE, f.r - task.i0);
    op.n = min(TILE, f.r - task.j0);
    op.k = f.c;
    op.lower = task.i0 == task.j0;
    op.lowerOffset = 0;
    tileProduct(op, smem);
}

// ------------------------------------------------------------------------------------------------------------------
// Pivot summary over the eliminated columns (one thread per equation): inertia counts, the MaxDiagonalRatio test
// (a_jj / d_j against maxRatio, a negative pivot always flagged; MultifrontalDriver.cpp:793-817) and the largest
// ratio. counters: [positive, negative, zero, issues]; issues: equations flagged, compacted (order fixed on the host).
// largest: per block, the largest ratio and the smallest equation reaching it.
// ------------------------------------------------------------------------------------------------------------------
__global__ void pivotSummary(FactorArgs args, const std::int32_t* supernodeOfColumn, int dimension,
                             const double* referenceDiagonal, double maxRatio, unsigned long long* counters,
                             std::int32_t* issues, int issueCapacity, double* blockRatio, std::int32_t* blockEquation)
{
    __shared__ double bestRatio[256];
    __shared__ int bestEquation[256];
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    double ratio = -INFINITY;
    int equation = INT_MAX;
    if (j < dimension)
    {
        const FrontDesc f = args.fronts[supernodeOfColumn[j]];
        const int k = j - f.first;
        const std::int64_t n = f.c + f.r;
        const double pivot = args.panels[f.panel + k + k * n];
        if (pivot > 0.0)
            atomicAdd(counters + 0, 1ull);
        else if (pivot < 0.0)
            atomicAdd(counters + 1, 1ull);
        else
            atomicAdd(counters + 2, 1ull);
        double diagonal = 0.0;
        const std::int64_t begin = args.colOffsets[j];
        if (begin < args.colOffsets[j + 1] && args.colRows[begin] == j)
            diagonal = args.colValues[begin];
        if (referenceDiagonal != nullptr && referenceDiagonal[j] >= 0.0)
            diagonal = referenceDiagonal[j];
        ratio = diagonal / pivot;
        equation = j;
        const bool isNegative = ratio < 0.0 || pivot < 0.0;
        if (ratio > maxRatio || isNegative)
        {
            const unsigned long long at = atomicAdd(counters + 3, 1ull);
            if (at < static_cast<unsigned long long>(issueCapacity))
                issues[at] = j;
        }
        if (!(ratio == ratio))
        {
            ratio = -INFINITY; // a NaN ratio never is the largest (the reference's `ratio > largest` is false)
            equation = INT_MAX;
        }
    }
    bestRatio[threadIdx.x] = ratio;
    bestEquation[threadIdx.x] = equation;
    __syncthreads();
    for (int stride = blockDim.x / 2; stride > 0; stride >>= 1)
    {
        if (threadIdx.x < stride)
        {
            const double other = bestRatio[threadIdx.x + stride];
            const int otherEquation = bestEquation[threadIdx.x + stride];
            if (other > bestRatio[threadIdx.x] ||
                (other == bestRatio[threadIdx.x] && otherEquation < bestEquation[threadIdx.x]))
            {
                bestRatio[threadIdx.x] = other;
                bestEquation[threadIdx.x] = otherEquation;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
    {
        blockRatio[blockIdx.x] = bestRatio[0];
        blockEquation[blockIdx.x] = bestEquation[0];
    }
}

} // namespace oosgpu::device
