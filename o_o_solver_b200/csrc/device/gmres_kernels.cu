// The kernels of the GMRES refinement of the solves (GpuFactor::solveRefined with a Krylov basis): blocks of
// right-hand sides held by rows (X[eq * width + col]), each column an independent system. The products with A use the
// full symmetric pattern of the matrix; the inner products sum fixed row blocks, their partial sums added in block
// order (reducePartials), so every coefficient has the same bits on every run.

#include "kernels.cuh"

#include <cstdint>

namespace oosgpu::device
{

// y = A x for a block of rows: one warp per row (a grid-stride loop), each lane its columns.
__global__ void multiplyRows(const std::int64_t* rowStart, const std::int32_t* columns, const std::int32_t* source,
                             const double* values, const double* x, double* y, int width, int dimension)
{
    const int warpsPerBlock = blockDim.x >> 5;
    const int lane = threadIdx.x & 31;
    const int totalWarps = gridDim.x * warpsPerBlock;
    for (int row = blockIdx.x * warpsPerBlock + (threadIdx.x >> 5); row < dimension; row += totalWarps)
    {
        const std::int64_t begin = rowStart[row];
        const std::int64_t end = rowStart[row + 1];
#pragma unroll
        for (int h = 0; h < 2; ++h)
        {
            const int c = lane + 32 * h;
            if (c >= width)
                continue;
            double sum = 0.0;
            for (std::int64_t k = begin; k < end; ++k)
                sum += values[source[k]] * x[static_cast<std::int64_t>(columns[k]) * width + c];
            y[static_cast<std::int64_t>(row) * width + c] = sum;
        }
    }
}

// partials[block * (vectors * width) + i * width + c] = sum over the block's rows r of v_i[r, c] w[r, c]: the vectors
// v_i are `stride` values apart. 256 threads: column tid % 64, row group tid / 64 (rows r = g, g + 4, ...), the four
// groups added in order.
__global__ void __launch_bounds__(256) dotRowsPartials(const double* v, std::int64_t stride, int vectors,
                                                       const double* w, int width, int dimension, int rowsPerBlock,
                                                       double* partials)
{
    __shared__ double sums[4][GMRES_MAX_VECTORS][64];
    const int c = threadIdx.x & 63;
    const int g = threadIdx.x >> 6;
    const int start = blockIdx.x * rowsPerBlock;
    const int end = min(start + rowsPerBlock, dimension);
    double acc[GMRES_MAX_VECTORS];
#pragma unroll
    for (int i = 0; i < GMRES_MAX_VECTORS; ++i)
        acc[i] = 0.0;
    if (c < width)
        for (int r = start + g; r < end; r += 4)
        {
            const std::int64_t at = static_cast<std::int64_t>(r) * width + c;
            const double wv = w[at];
#pragma unroll
            for (int i = 0; i < GMRES_MAX_VECTORS; ++i)
                if (i < vectors)
                    acc[i] += v[i * stride + at] * wv;
        }
#pragma unroll
    for (int i = 0; i < GMRES_MAX_VECTORS; ++i)
        sums[g][i][c] = acc[i];
    __syncthreads();
    if (g == 0 && c < width)
        for (int i = 0; i < vectors; ++i)
            partials[static_cast<std::int64_t>(blockIdx.x) * vectors * width + i * width + c] =
                ((sums[0][i][c] + sums[1][i][c]) + sums[2][i][c]) + sums[3][i][c];
}

// w[r, c] -= sum_i coef[i * width + c] v_i[r, c], i increasing.
__global__ void subtractRowsCombination(double* w, const double* v, std::int64_t stride, int vectors,
                                        const double* coef, int width, std::int64_t items)
{
    const std::int64_t e = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= items)
        return;
    const int c = static_cast<int>(e % width);
    double value = w[e];
    for (int i = 0; i < vectors; ++i)
        value -= coef[i * width + c] * v[i * stride + e];
    w[e] = value;
}

// x[r, c] += sum_i y[i * width + c] v_i[r, c], i increasing.
__global__ void addRowsCombination(double* x, const double* v, std::int64_t stride, int vectors, const double* y,
                                   int width, std::int64_t items)
{
    const std::int64_t e = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= items)
        return;
    const int c = static_cast<int>(e % width);
    double sum = 0.0;
    for (int i = 0; i < vectors; ++i)
        sum += y[i * width + c] * v[i * stride + e];
    x[e] += sum;
}

// out[r, c] = in[r, c] * s[c].
__global__ void scaleRowsColumns(const double* in, double* out, const double* s, int width, std::int64_t items)
{
    const std::int64_t e = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= items)
        return;
    out[e] = in[e] * s[e % width];
}

} // namespace oosgpu::device
