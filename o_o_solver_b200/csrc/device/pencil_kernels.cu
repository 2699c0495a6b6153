// The kernels of the shifted pencil (the reference's SparsePencil, src/linalg/eigen/SparsePencil.cpp:55-157):
// the shifted, scaled matrix S (K - sigma M) S on the pattern of K, and the products with M.

#include "kernels.cuh"

#include <cstdint>

namespace oosgpu::device
{

// values[k] = s_i (K_k + (-sigma) M_k) s_j for the term k of column j, row i: each product rounded, then the sum
// (SymmetricCsc::combine, SymmetricCsc.cpp:209-238: "rounded once per product and once for the sum"), then the
// powers-of-two scales, which round nothing (scaleSymmetric). One warp per column.
__global__ void shiftedMatrix(const std::int64_t* offsets, const std::int32_t* rows, const double* stiffness,
                              const double* mass, double sigma, const double* scale, double* values, int dimension)
{
    const int column = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (column >= dimension)
        return;
    const double sj = scale[column];
    for (std::int64_t k = offsets[column] + lane; k < offsets[column + 1]; k += 32)
    {
        const double product = __dmul_rn(-sigma, mass[k]);
        const double sum = __dadd_rn(stiffness[k], product);
        values[k] = __dmul_rn(__dmul_rn(scale[rows[k]], sum), sj);
    }
}

// Y = diag(m) X for column-major blocks (a lumped mass: the reference's diagonal product, SparsePencil.cpp:147-156).
__global__ void diagonalProduct(const double* m, const double* x, std::int64_t ldx, double* y, std::int64_t ldy,
                                int dimension, int columns)
{
    const std::int64_t e = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= static_cast<std::int64_t>(dimension) * columns)
        return;
    const int col = static_cast<int>(e / dimension);
    const int i = static_cast<int>(e - static_cast<std::int64_t>(col) * dimension);
    y[static_cast<std::int64_t>(col) * ldy + i] = m[i] * x[static_cast<std::int64_t>(col) * ldx + i];
}

// Y = A X for column-major blocks, A symmetric given by its full pattern (both triangles, rows ascending, `source`
// the index of each term in the lower CSC's values): one warp per row, each lane its columns, each value one sum in
// the row's order of terms.
__global__ void symmetricProduct(const std::int64_t* rowStart, const std::int32_t* columns, const std::int32_t* source,
                                 const double* values, const double* x, std::int64_t ldx, double* y, std::int64_t ldy,
                                 int dimension, int width)
{
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= dimension)
        return;
    const std::int64_t begin = rowStart[row];
    const std::int64_t end = rowStart[row + 1];
    for (int c = lane; c < width; c += 32)
    {
        double sum = 0.0;
        for (std::int64_t k = begin; k < end; ++k)
            sum += values[source[k]] * x[static_cast<std::int64_t>(c) * ldx + columns[k]];
        y[static_cast<std::int64_t>(c) * ldy + row] = sum;
    }
}

} // namespace oosgpu::device
