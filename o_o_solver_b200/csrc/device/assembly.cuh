// The assembly of one front by one thread block (FrontAssembly.cpp:166-300): cleared, the matrix's entries of the
// supernode's columns added, then the children's update matrices in increasing child order (a __syncthreads between
// them keeps every element's sum in the reference's order). The front is any column-major store reached through an
// accessor (shared memory for a small front, global memory for a whole front).
#pragma once

#include "kernels.cuh"

#include <cstdint>

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

// element(i, j): a reference to the front's element (i, j), i >= j.
template <typename Element>
__device__ void assembleFrontBy(const FactorArgs& args, const FrontDesc& f, Element element,
                                std::int32_t* structureError)
{
    const int n = f.c + f.r;
    const int tid = threadIdx.x;
    const int threads = blockDim.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;
    const int warps = threads >> 5;
    for (std::int64_t e = tid; e < static_cast<std::int64_t>(n) * n; e += threads)
    {
        const int j = static_cast<int>(e / n);
        const int i = static_cast<int>(e - static_cast<std::int64_t>(j) * n);
        if (i >= j)
            element(i, j) = 0.0;
    }
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
            element(position, j) += args.colValues[k];
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
                element(map[ic], pj) += column[ic];
        }
        __syncthreads();
    }
}

} // namespace oosgpu::device
