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
// Small fronts: one block per front of order n <= maxOrder, the whole front in shared memory (column-major,
// leading dimension ld = n + 1): assembled, its c columns eliminated right-looking (each element receives its terms
// k = 0, 1, ... in order, as the reference's unblocked algorithm), then the panel and the update matrix written out.
// ------------------------------------------------------------------------------------------------------------------
__global__ void smallFronts(FactorArgs args, const std::int32_t* list, std::int32_t* structureError)
{
    extern __shared__ double front[];
    const std::int32_t s = list[blockIdx.x];
    const FrontDesc f = args.fronts[s];
    const int n = f.c + f.r;
    const int ld = n + 1;
    const int tid = threadIdx.x;
    const int threads = blockDim.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;
    const int warps = threads >> 5;

    for (int e = tid; e < n * ld; e += threads)
        front[e] = 0.0;
    __syncthreads();
    for (int j = warp; j < f.c; j += warps)
    {
        const std::int32_t column = f.first + j;
        const std::int64_t begin = args.colOffsets[column];
        const std::int64_t end = args.colOffsets[column + 1];
        for (std::int64_t k = begin + lane; k < end; k += 32)
        {
            const std::int32_t row = args.colRows[k];
            const int position = row < column ? -1 : positionInFront(f, args.rows, row);
            if (position < 0)
            {
                atomicMin(structureError, column);
                continue;
            }
            front[position + j * ld] += args.colValues[k];
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
                front[map[ic] + pj * ld] += column[ic];
        }
        __syncthreads();
    }
    // Elimination of the c columns.
    for (int k = 0; k < f.c; ++k)
    {
        const double pivot = front[k + k * ld];
        if (isBadPivot(pivot))
        {
            if (tid == 0)
                atomicMin(args.zeroPivot + s, k);
        }
        for (int i = k + 1 + tid; i < n; i += threads)
            front[i + k * ld] = front[i + k * ld] / pivot;
        __syncthreads();
        for (int j = k + 1 + warp; j < n; j += warps)
        {
            const double w = front[j + k * ld] * pivot;
            for (int i = j + lane; i < n; i += 32)
                front[i + j * ld] -= front[i + k * ld] * w;
        }
        __syncthreads();
    }
    double* panel = args.panels + f.panel;
    for (int e = tid; e < n * f.c; e += threads)
    {
        const int j = e / n;
        const int i = e - j * n;
        panel[e] = i >= j ? front[i + j * ld] : 0.0;
    }
    if (f.r > 0)
    {
        double* update = args.updates + f.update;
        for (int e = tid; e < f.r * f.r; e += threads)
        {
            const int j = e / f.r;
            const int i = e - j * f.r;
            if (i >= j)
                update[e] = front[(f.c + i) + (f.c + j) * ld];
        }
    }
}

// ------------------------------------------------------------------------------------------------------------------
// Blocked elimination of a large front's panel, step t (columns [k0, k0 + kb), k0 = 64 t):
//   diagonalBlocks: the kb x kb diagonal block eliminated in shared memory by one block per front;
//   panelRows: the rows below it, L(i, :) = A(i, :) L11^-T D^-1, one block per front and 128 rows, each thread a row
//              (the chain of the right-looking algorithm: a_ij - sum_k l_ik w_jk, then / d_j);
//   trailing panel update and final update-matrix SYRK: tile products (tileProduct).
// ------------------------------------------------------------------------------------------------------------------
constexpr int BLOCK = 64;

__global__ void diagonalBlocks(FactorArgs args, const std::int32_t* list, int k0)
{
    __shared__ double a[BLOCK * (BLOCK + 1)];
    const std::int32_t s = list[blockIdx.x];
    const FrontDesc f = args.fronts[s];
    const int n = f.c + f.r;
    const int kb = min(BLOCK, f.c - k0);
    constexpr int LD = BLOCK + 1;
    double* panel = args.panels + f.panel + static_cast<std::int64_t>(k0) * n + k0;
    const int tid = threadIdx.x;
    const int threads = blockDim.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;
    const int warps = threads >> 5;
    for (int e = tid; e < kb * kb; e += threads)
    {
        const int j = e / kb;
        const int i = e - j * kb;
        a[i + j * LD] = panel[i + static_cast<std::int64_t>(j) * n];
    }
    __syncthreads();
    for (int k = 0; k < kb; ++k)
    {
        const double pivot = a[k + k * LD];
        if (isBadPivot(pivot) && tid == 0)
            atomicMin(args.zeroPivot + s, k0 + k);
        for (int i = k + 1 + tid; i < kb; i += threads)
            a[i + k * LD] = a[i + k * LD] / pivot;
        __syncthreads();
        for (int j = k + 1 + warp; j < kb; j += warps)
        {
            const double w = a[j + k * LD] * pivot;
            for (int i = j + lane; i < kb; i += 32)
                a[i + j * LD] -= a[i + k * LD] * w;
        }
        __syncthreads();
    }
    for (int e = tid; e < kb * kb; e += threads)
    {
        const int j = e / kb;
        const int i = e - j * kb;
        if (i >= j)
            panel[i + static_cast<std::int64_t>(j) * n] = a[i + j * LD];
    }
}

constexpr int ROWS_PER_BLOCK = 128;

__global__ void __launch_bounds__(ROWS_PER_BLOCK) panelRows(FactorArgs args, const TileTask* tasks, int k0)
{
    __shared__ double w[BLOCK * BLOCK]; // w[j * BLOCK + k] = L11(j, k) * d_k
    __shared__ double dinv[BLOCK];
    const TileTask task = tasks[blockIdx.x];
    const FrontDesc f = args.fronts[task.front];
    const int n = f.c + f.r;
    const int kb = min(BLOCK, f.c - k0);
    const double* diag = args.panels + f.panel + static_cast<std::int64_t>(k0) * n + k0;
    for (int e = threadIdx.x; e < BLOCK * BLOCK; e += blockDim.x)
    {
        const int j = e / BLOCK;
        const int k = e - j * BLOCK;
        double value = 0.0;
        if (j < kb && k < j)
            value = diag[j + static_cast<std::int64_t>(k) * n] * diag[k + static_cast<std::int64_t>(k) * n];
        w[e] = value;
    }
    for (int k = threadIdx.x; k < BLOCK; k += blockDim.x)
        dinv[k] = k < kb ? diag[k + static_cast<std::int64_t>(k) * n] : 1.0;
    __syncthreads();
    const int row = task.i0 + threadIdx.x;
    if (row >= n)
        return;
    double* base = args.panels + f.panel + static_cast<std::int64_t>(k0) * n + row;
    double x[BLOCK];
#pragma unroll
    for (int j = 0; j < BLOCK; ++j)
        x[j] = j < kb ? base[static_cast<std::int64_t>(j) * n] : 0.0;
#pragma unroll
    for (int j = 0; j < BLOCK; ++j)
    {
        double v = x[j];
#pragma unroll
        for (int k = 0; k < j; ++k)
            v -= x[k] * w[j * BLOCK + k];
        x[j] = v / dinv[j];
    }
#pragma unroll
    for (int j = 0; j < BLOCK; ++j)
        if (j < kb)
            base[static_cast<std::int64_t>(j) * n] = x[j];
}

// Trailing panel update of step t: columns [o, c), rows [o, n), o = k0 + 64, K = the step's 64 columns.
__global__ void __launch_bounds__(TILE_THREADS) panelUpdate(FactorArgs args, const TileTask* tasks, int k0)
{
    __shared__ double smemA[TILE_K * (TILE + TILE_PAD)];
    __shared__ double smemB[TILE_K * (TILE + TILE_PAD)];
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
    op.k = BLOCK;
    op.lower = task.i0 == task.j0;
    op.lowerOffset = 0;
    tileProduct(op, smemA, smemB);
}

// The Schur update of the update matrix: U(i, j) -= sum_{k < c} L(c + i, k) d_k L(c + j, k), lower tiles.
__global__ void __launch_bounds__(TILE_THREADS) updateMatrix(FactorArgs args, const TileTask* tasks)
{
    __shared__ double smemA[TILE_K * (TILE + TILE_PAD)];
    __shared__ double smemB[TILE_K * (TILE + TILE_PAD)];
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
    tileProduct(op, smemA, smemB);
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
