// Extend-add of the large fronts through shared memory (the reference's FrontAssembler::assembleColumns,
// src/linalg/supernodal/FrontAssembly.cpp:166-300, on the GPU).
//
// One block per piece of a front: STAGE_COLUMNS front columns [j0, j1) by up to STAGE_ROWS front positions [i0, i1)
// (a piece lies inside the panel's columns or inside the update matrix's, never across). The piece is built in shared
// memory and written out once:
//   zeros; the matrix's entries of its panel columns (each element receives at most one); then each child's update
//   matrix in increasing child order, a barrier between two children, so that every element's sum is
//   0 + a_ij + u1_ij + u2_ij + ... exactly as the reference forms it (and as the element-wise kernel did);
//   the piece's columns written to the panel (every row: the panel's zeros above the diagonal too) or to the update
//   matrix (from the diagonal down), coalesced, two values per store where the column allows.
// HBM traffic: every front element written once, every child's update element and matrix entry read once. The
// element-wise kernel cleared the front in HBM, then read, added and wrote an element for every child term.

#include "assembly.cuh"
#include "kernels.cuh"

#include <climits>
#include <cstdint>

namespace oosgpu::device
{

namespace
{

// The first index k of the ascending map[0 .. count) with map[k] >= value.
__device__ __forceinline__ int firstAtLeast(const std::int32_t* map, int count, int value)
{
    int lo = 0;
    int hi = count;
    while (lo < hi)
    {
        const int mid = (lo + hi) >> 1;
        if (map[mid] < value)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// The equation at front position p of f (columns first, then R(s)).
__device__ __forceinline__ std::int32_t equationAt(const FrontDesc& f, const std::int32_t* rows, int p)
{
    return p < f.c ? f.first + p : rows[f.rowStart + p - f.c];
}

} // namespace

__global__ void __launch_bounds__(STAGE_THREADS) assembleStaged(FactorArgs args, const AssemblyTask* pieces,
                                                                 std::int32_t* structureError)
{
    extern __shared__ double tile[]; // the piece, column-major, leading dimension STAGE_ROWS
    __shared__ int range[4];
    const AssemblyTask piece = pieces[blockIdx.x];
    const FrontDesc f = args.fronts[piece.front];
    const int n = f.c + f.r;
    const int j0 = piece.j0;
    const int j1 = piece.j1;
    const int i0 = piece.pad; // the piece's first front position
    const int i1 = min(i0 + STAGE_ROWS, n);
    const int columns = j1 - j0;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    constexpr int WARPS = STAGE_THREADS / 32;
    const bool inPanel = j0 < f.c;

    for (int e = tid; e < STAGE_ROWS * columns; e += STAGE_THREADS)
        tile[e] = 0.0;
    // A piece wholly above its columns' diagonal holds the panel's zeros only.
    if (i1 > j0)
    {
        __syncthreads();
        if (inPanel)
        {
            // The piece's positions as equations: a matrix entry lands in it when its row lies in [low, high].
            const std::int32_t low = i0 == 0 ? INT_MIN : equationAt(f, args.rows, i0);
            const std::int32_t high = i1 == n ? INT_MAX : equationAt(f, args.rows, i1 - 1);
            for (int j = j0 + warp; j < j1; j += WARPS)
            {
                const std::int32_t column = f.first + j;
                const std::int64_t begin = args.colOffsets[column];
                const std::int64_t end = args.colOffsets[column + 1];
                double* target = tile + (j - j0) * STAGE_ROWS - i0;
                for (std::int64_t k = begin + lane; k < end; k += 32)
                {
                    const std::int32_t row = args.colRows[k];
                    if (row < column)
                    {
                        atomicMin(structureError, column);
                        continue;
                    }
                    if (row < low || row > high)
                        continue; // another piece of these columns takes it
                    const int position = positionInFront(f, args.rows, row);
                    if (position < 0)
                    {
                        atomicMin(structureError, column);
                        continue;
                    }
                    target[position] += args.colValues[k];
                }
            }
        }
        __syncthreads();
        for (int q = 0; q < f.childCount; ++q)
        {
            const std::int32_t child = args.children[f.childStart + q];
            const FrontDesc ch = args.fronts[child];
            if (ch.r == 0)
                continue;
            const std::int32_t* map = args.relpos + ch.rowStart;
            if (tid == 0)
            {
                // the child's rows whose positions fall in the piece's columns, and in its rows (positions ascend)
                range[0] = firstAtLeast(map, ch.r, j0);
                range[1] = firstAtLeast(map, ch.r, j1);
                range[2] = firstAtLeast(map, ch.r, i0);
                range[3] = firstAtLeast(map, ch.r, i1);
            }
            __syncthreads();
            const int ja = range[0];
            const int jb = range[1];
            const int ia = range[2];
            const int ib = range[3];
            const double* source = args.updates + ch.update;
            for (int jc = ja + warp; jc < jb; jc += WARPS)
            {
                double* target = tile + (map[jc] - j0) * STAGE_ROWS - i0;
                const double* column = source + static_cast<std::int64_t>(jc) * ch.r;
                for (int ic = max(ia, jc) + lane; ic < ib; ic += 32)
                    target[map[ic]] += column[ic];
            }
            __syncthreads();
        }
    }
    __syncthreads();
    // Out: a warp per column, two values per store from the first 16-byte boundary on.
    for (int jl = warp; jl < columns; jl += WARPS)
    {
        const int j = j0 + jl;
        double* destination = inPanel ? args.panels + f.panel + static_cast<std::int64_t>(j) * n
                                      : args.updates + f.update + static_cast<std::int64_t>(j - f.c) * f.r - f.c;
        const int first = inPanel ? i0 : max(i0, j);
        const double* source = tile + jl * STAGE_ROWS - i0;
        int i = first;
        if (i < i1 && (reinterpret_cast<std::uintptr_t>(destination + i) & 15) != 0)
        {
            if (lane == 0)
                destination[i] = source[i];
            ++i;
        }
        for (int p = i + 2 * lane; p + 1 < i1; p += 64)
            *reinterpret_cast<double2*>(destination + p) = make_double2(source[p], source[p + 1]);
        const int pairs = (i1 - i) / 2;
        if (lane == 0 && i + 2 * pairs < i1)
            destination[i1 - 1] = source[i1 - 1];
    }
}

} // namespace oosgpu::device
