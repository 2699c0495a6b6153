// Device-side building blocks shared by the factorisation and the solves: the front descriptors, the FP64 tensor-core
// tile product (mma.sync m8n8k4 .f64, the FP64 MMA path of sm_100a) and small helpers.
#pragma once

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
constexpr int TILE_K = 16;
constexpr int TILE_PAD = 8; // smem row stride 72 doubles: the m8n8k4 fragment loads take 2 wavefronts (no conflict)
constexpr int TILE_THREADS = 128;

__device__ __forceinline__ void dmma8x8x4(double (&d)[2], double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
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

// One 64 x 64 tile on a block of TILE_THREADS threads (4 warps of 32 x 32). The K loop stages TILE_K-deep slices of A
// and of W = B * D in shared memory (register double buffering: the next slice is loaded while the current one is
// multiplied), the products run on the FP64 tensor cores (DMMA m8n8k4), and C is read, reduced and written once.
// smemA/smemB: TILE_K * (TILE + TILE_PAD) doubles each. A_BY_ROWS: A's rows are contiguous in memory (aColStride 1),
// so the loads of A run along p (16 consecutive doubles per row) instead of along the rows.
template <bool A_BY_ROWS = false>
__device__ __forceinline__ void tileProduct(const TileOperands& op, double* smemA, double* smemB)
{
    constexpr int LD = TILE + TILE_PAD;
    constexpr int PER_THREAD = TILE * TILE_K / TILE_THREADS; // 8
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int wm = (warp >> 1) * 32;
    const int wn = (warp & 1) * 32;

    double acc[4][4][2];
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
        {
            acc[mi][ni][0] = 0.0;
            acc[mi][ni][1] = 0.0;
        }

    double ra[PER_THREAD];
    double rb[PER_THREAD];
    const auto load = [&](int kbase)
    {
#pragma unroll
        for (int q = 0; q < PER_THREAD; ++q)
        {
            const int e = tid + q * TILE_THREADS;
            const int ii = e & (TILE - 1);
            const int p = e >> 6;
            const int kp = kbase + p;
            const int iiA = A_BY_ROWS ? (e >> 4) : ii;
            const int pA = A_BY_ROWS ? (e & (TILE_K - 1)) : p;
            const int kpA = kbase + pA;
            double va = 0.0;
            double vb = 0.0;
            if (kpA < op.k && iiA < op.m)
                va = op.a[iiA * op.aRowStride + static_cast<std::int64_t>(kpA) * op.aColStride];
            if (kp < op.k)
            {
                if (ii < op.n)
                {
                    const std::int64_t row = op.bIndex != nullptr ? op.bIndex[kp] : kp;
                    vb = op.b[ii * op.bRowStride + row * op.bColStride];
                    if (op.d != nullptr)
                        vb *= op.d[static_cast<std::int64_t>(kp) * op.dStride];
                }
            }
            ra[q] = va;
            rb[q] = vb;
        }
    };
    const auto store = [&]()
    {
#pragma unroll
        for (int q = 0; q < PER_THREAD; ++q)
        {
            const int e = tid + q * TILE_THREADS;
            const int ii = e & (TILE - 1);
            const int p = e >> 6;
            if (A_BY_ROWS)
                smemA[(e & (TILE_K - 1)) * LD + (e >> 4)] = ra[q];
            else
                smemA[p * LD + ii] = ra[q];
            smemB[p * LD + ii] = rb[q];
        }
    };

    load(0);
    store();
    __syncthreads();
    for (int kbase = 0; kbase < op.k; kbase += TILE_K)
    {
        const bool more = kbase + TILE_K < op.k;
        if (more)
            load(kbase + TILE_K);
#pragma unroll
        for (int kk = 0; kk < TILE_K; kk += 4)
        {
            const int pr = kk + (lane & 3);
            double fa[4];
            double fb[4];
#pragma unroll
            for (int mi = 0; mi < 4; ++mi)
                fa[mi] = smemA[pr * LD + wm + mi * 8 + (lane >> 2)];
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
                fb[ni] = smemB[pr * LD + wn + ni * 8 + (lane >> 2)];
#pragma unroll
            for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni)
                    dmma8x8x4(acc[mi][ni], fa[mi], fb[ni]);
        }
        __syncthreads();
        if (more)
        {
            store();
            __syncthreads();
        }
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
                if (ii < op.m && jj < op.n && (!op.lower || ii + op.lowerOffset >= jj))
                {
                    double* target = op.c + ii * op.cRowStride + jj * op.cColStride;
                    *target = *target - acc[mi][ni][h];
                }
            }
}

} // namespace oosgpu::device
