// The dense block kernels of the block Lanczos run (the reference's MassOrthogonalizer and the basis products of
// LanczosRun, src/linalg/eigen/MassOrthogonalizer.cpp:236-425 and LanczosRun.cpp:38-58): tall blocks of vectors,
// column-major with a leading dimension, in HBM. Every reduction over the rows has a fixed order that depends on the
// row count only (blocks of rows fixed by the row count, lanes and warps combined in a fixed tree, the blocks' sums
// added in increasing order): the same bits on every run.

#include "kernels.cuh"

#include <cstdint>

namespace oosgpu::device
{

namespace
{

constexpr std::uint64_t GOLDEN_GAMMA = 0x9E3779B97F4A7C15ULL;

// splitmix64's output function (Steele, Lea & Flood, OOPSLA 2014) of a state.
__device__ __forceinline__ std::uint64_t mix64(std::uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

__device__ __forceinline__ double warpSum(double v)
{
    for (int offset = 16; offset > 0; offset >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, offset);
    return v;
}

} // namespace

// x(i, j) = the draw number j * rows + i + 1 after `state` of splitmix64, as a uniform value in [-1, 1) from its 53
// high bits: the values the reference's fillRandom (LanczosRun.cpp:93-101) writes column by column from that state.
__global__ void randomBlock(double* x, std::int64_t ld, int rows, int columns, std::uint64_t state)
{
    const std::int64_t e = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= static_cast<std::int64_t>(rows) * columns)
        return;
    const int j = static_cast<int>(e / rows);
    const int i = static_cast<int>(e - static_cast<std::int64_t>(j) * rows);
    const std::uint64_t z = mix64(state + static_cast<std::uint64_t>(e + 1) * GOLDEN_GAMMA);
    constexpr double TWO_TO_MINUS_52 = 1.0 / 4503599627370496.0;
    x[static_cast<std::int64_t>(j) * ld + i] = static_cast<double>(z >> 11) * TWO_TO_MINUS_52 - 1.0;
}

// partials[(block * w + j) * m + i] = sum over the block's rows r of a(r, i) y(r, j), for the rows
// [block * rowsPerBlock, +rowsPerBlock). The columns of `a` go by groups of 8 to the warps; when there are fewer than
// 8 groups, the warps of one group split the block's rows into slices, combined in slice order.
__global__ void __launch_bounds__(GRAM_THREADS) gramPartials(const double* a, std::int64_t lda, int m, const double* y,
                                                             std::int64_t ldy, int w, int rows, int rowsPerBlock,
                                                             double* partials)
{
    __shared__ double slices[GRAM_THREADS / 32][64];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    constexpr int WARPS = GRAM_THREADS / 32;
    const int start = blockIdx.x * rowsPerBlock;
    const int end = min(start + rowsPerBlock, rows);
    const int groups = (m + 7) / 8;
    const int sliceCount = groups >= WARPS ? 1 : WARPS / groups;
    const int rowsPerSlice = (max(end - start, 0) + sliceCount - 1) / sliceCount;
    for (int j0 = 0; j0 < w; j0 += 8)
    {
        const int wUsed = min(8, w - j0);
        // Rounds: groups handled by the warps together (sliceCount warps per group when sliceCount > 1).
        const int groupsPerRound = sliceCount > 1 ? groups : WARPS;
        for (int g0 = 0; g0 < groups; g0 += groupsPerRound)
        {
            const int group = g0 + (sliceCount > 1 ? warp / sliceCount : warp);
            const int slice = sliceCount > 1 ? warp % sliceCount : 0;
            const bool active = (sliceCount > 1 ? warp < groups * sliceCount : true) && group < groups;
            double acc[8][8];
#pragma unroll
            for (int ii = 0; ii < 8; ++ii)
#pragma unroll
                for (int jj = 0; jj < 8; ++jj)
                    acc[ii][jj] = 0.0;
            if (active)
            {
                const int i0 = group * 8;
                const int iUsed = min(8, m - i0);
                const int sliceStart = start + slice * rowsPerSlice;
                const int sliceEnd = min(sliceStart + rowsPerSlice, end);
                for (int r = sliceStart + lane; r < sliceEnd; r += 32)
                {
                    double yv[8];
#pragma unroll
                    for (int jj = 0; jj < 8; ++jj)
                        yv[jj] = jj < wUsed ? y[static_cast<std::int64_t>(j0 + jj) * ldy + r] : 0.0;
#pragma unroll
                    for (int ii = 0; ii < 8; ++ii)
                    {
                        if (ii < iUsed)
                        {
                            const double av = a[static_cast<std::int64_t>(i0 + ii) * lda + r];
#pragma unroll
                            for (int jj = 0; jj < 8; ++jj)
                                acc[ii][jj] = fma(av, yv[jj], acc[ii][jj]);
                        }
                    }
                }
#pragma unroll
                for (int ii = 0; ii < 8; ++ii)
#pragma unroll
                    for (int jj = 0; jj < 8; ++jj)
                        acc[ii][jj] = warpSum(acc[ii][jj]);
            }
            if (sliceCount == 1)
            {
                if (active && lane == 0)
                {
                    const int i0 = group * 8;
                    for (int ii = 0; ii < min(8, m - i0); ++ii)
                        for (int jj = 0; jj < wUsed; ++jj)
                            partials[(static_cast<std::int64_t>(blockIdx.x) * w + j0 + jj) * m + i0 + ii] =
                                acc[ii][jj];
                }
            }
            else
            {
                if (active && lane == 0)
                {
#pragma unroll
                    for (int ii = 0; ii < 8; ++ii)
#pragma unroll
                        for (int jj = 0; jj < 8; ++jj)
                            slices[warp][ii * 8 + jj] = acc[ii][jj];
                }
                __syncthreads();
                // One thread per (group, ii, jj): the slices of its group in increasing order.
                for (int t = threadIdx.x; t < groups * 64; t += blockDim.x)
                {
                    const int g = t / 64;
                    const int ii = (t / 8) % 8;
                    const int jj = t % 8;
                    const int i = g * 8 + ii;
                    if (i >= m || jj >= wUsed)
                        continue;
                    double sum = 0.0;
                    for (int s = 0; s < sliceCount; ++s)
                        sum += slices[g * sliceCount + s][ii * 8 + jj];
                    partials[(static_cast<std::int64_t>(blockIdx.x) * w + j0 + jj) * m + i] = sum;
                }
                __syncthreads();
            }
        }
    }
}

// out[k] = sum over the blocks b (increasing) of partials[b * count + k].
__global__ void reducePartials(const double* partials, int blocks, int count, double* out)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count)
        return;
    double sum = 0.0;
    for (int b = 0; b < blocks; ++b)
        sum += partials[static_cast<std::int64_t>(b) * count + k];
    out[k] = sum;
}

// w(r, j) <- w(r, j) - sum_i a(r, i) c(i, j) for j < width, c m x width column-major (leading dimension ldc): each
// value one chain over i in increasing order (the reference's subtractRows, MassOrthogonalizer.cpp:96-112). One thread
// per row, c in shared memory (m x width, leading dimension m).
__global__ void subtractProduct(double* w, std::int64_t ldw, int width, const double* a, std::int64_t lda, int m,
                                const double* c, std::int64_t ldc, int rows)
{
    extern __shared__ double cs[];
    for (int t = threadIdx.x; t < m * width; t += blockDim.x)
        cs[t] = c[(t / m) * ldc + t % m];
    __syncthreads();
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows)
        return;
    for (int j0 = 0; j0 < width; j0 += 8)
    {
        const int used = min(8, width - j0);
        double acc[8];
#pragma unroll
        for (int jj = 0; jj < 8; ++jj)
            acc[jj] = jj < used ? w[static_cast<std::int64_t>(j0 + jj) * ldw + r] : 0.0;
        for (int i = 0; i < m; ++i)
        {
            const double av = a[static_cast<std::int64_t>(i) * lda + r];
#pragma unroll
            for (int jj = 0; jj < 8; ++jj)
                acc[jj] = fma(-av, cs[i + (j0 + jj < width ? (j0 + jj) : 0) * m], acc[jj]);
        }
#pragma unroll
        for (int jj = 0; jj < 8; ++jj)
            if (jj < used)
                w[static_cast<std::int64_t>(j0 + jj) * ldw + r] = acc[jj];
    }
}

// out(r, j) = sum_i a(r, i) s(i, j) - sum_t next(r, t) correction(t, j) for j < k (the second sum only when `next` is
// given; correction b x k, leading dimension b): the basis times the Ritz vectors of a restart or of the converged
// pairs (LanczosRun.cpp:38-58, 383-390). A block reads its BLOCK_ROWS rows of `a` into shared memory before it writes
// any output row, so `out` may be the first columns of `a`.
__global__ void combineRows(const double* a, std::int64_t lda, int m, const double* s, std::int64_t lds, int k,
                            double* out, std::int64_t ldo, int rows, const double* next, std::int64_t ldn, int b,
                            const double* correction)
{
    extern __shared__ double tile[]; // m x COMBINE_ROWS, row index fastest
    const int r0 = blockIdx.x * COMBINE_ROWS;
    for (int t = threadIdx.x; t < m * COMBINE_ROWS; t += blockDim.x)
    {
        const int rr = t % COMBINE_ROWS;
        const int i = t / COMBINE_ROWS;
        tile[t] = r0 + rr < rows ? a[static_cast<std::int64_t>(i) * lda + r0 + rr] : 0.0;
    }
    __syncthreads();
    const int rr = threadIdx.x % COMBINE_ROWS;
    const int r = r0 + rr;
    if (r >= rows)
        return;
    for (int j = threadIdx.x / COMBINE_ROWS; j < k; j += blockDim.x / COMBINE_ROWS)
    {
        double acc = 0.0;
        for (int i = 0; i < m; ++i)
            acc = fma(tile[i * COMBINE_ROWS + rr], s[static_cast<std::int64_t>(j) * lds + i], acc);
        if (next != nullptr)
            for (int t = 0; t < b; ++t)
                acc = fma(-next[static_cast<std::int64_t>(t) * ldn + r], correction[static_cast<std::int64_t>(j) * b + t],
                          acc);
        out[static_cast<std::int64_t>(j) * ldo + r] = acc;
    }
}

// Column c of a block after its Gram-Schmidt passes, decided on the device: its M-norm sqrt(max(0, *dot)) against the
// dependence threshold factor * reference, where reference is the M-norm the block's column c had before its
// projections (perColumn: sqrt(max(0, gram(c, c)))) or the largest such norm of the block and floorNorm (otherwise;
// gram width x width, leading dimension width). Above it, x and its M-image mx are scaled to unit M-norm and the norm
// is written to *diagonal; at or below it (or not a number), the column is left as it is, *diagonal is 0 and
// *accepted 0: the host redoes that block along the path with random replacements. Every thread forms the same
// scalars from the same values, so the whole grid agrees.
__global__ void acceptColumn(double* x, double* mx, int rows, const double* dot, const double* gram, int width, int c,
                             int perColumn, double floorNorm, double factor, double* diagonal, double* accepted)
{
    double reference = floorNorm;
    if (perColumn != 0)
        reference = sqrt(fmax(0.0, gram[c + c * width]));
    else
        for (int j = 0; j < width; ++j)
            reference = fmax(reference, sqrt(fmax(0.0, gram[j + j * width])));
    const double norm = sqrt(fmax(0.0, *dot));
    const bool keep = norm > factor * reference;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0)
    {
        *diagonal = keep ? norm : 0.0;
        *accepted = keep ? 1.0 : 0.0;
    }
    if (!keep || i >= rows)
        return;
    const double inverse = 1.0 / norm;
    x[i] *= inverse;
    mx[i] *= inverse;
}

// x <- s x, and y <- s y when y is given (one column).
__global__ void scaleColumn(double* x, double* y, double s, int rows)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows)
        return;
    x[i] *= s;
    if (y != nullptr)
        y[i] *= s;
}

// x(:, j) <- s_j x(:, j), and y(:, j) <- s_j y(:, j) when y is given (each value alone).
__global__ void scaleColumns(double* x, std::int64_t ldx, double* y, std::int64_t ldy, const double* s, int rows,
                             int columns)
{
    const std::int64_t e = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= static_cast<std::int64_t>(rows) * columns)
        return;
    const int j = static_cast<int>(e / rows);
    const int i = static_cast<int>(e - static_cast<std::int64_t>(j) * rows);
    x[static_cast<std::int64_t>(j) * ldx + i] *= s[j];
    if (y != nullptr)
        y[static_cast<std::int64_t>(j) * ldy + i] *= s[j];
}

} // namespace oosgpu::device
