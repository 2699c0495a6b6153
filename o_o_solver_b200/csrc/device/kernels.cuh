// The argument blocks and the kernels of the factorisation and the solves (defined in factor_kernels.cu and
// solve_kernels.cu, launched by the host engine).
#pragma once

#include "common.cuh"

#include <cstdint>

namespace oosgpu::device
{

struct FactorArgs
{
    const FrontDesc* fronts;
    const std::int32_t* children;   // children of each front, increasing, at childStart
    const std::int32_t* rows;       // R(s) of every supernode, at rowStart
    const std::int32_t* relpos;     // position in the parent's front of each row of R(s), at rowStart
    const std::int64_t* colOffsets; // the CSC of the matrix
    const std::int32_t* colRows;
    const double* colValues;
    double* panels;
    double* updates;
    std::int32_t* zeroPivot; // per supernode: the first zero (or non-finite) pivot's column in it
};

struct SolveArgs
{
    const FrontDesc* fronts;
    const std::int32_t* children;
    const std::int32_t* rows;
    const std::int32_t* relpos;
    const double* panels;
    double* x;       // n x width, by rows
    double* updates; // update rows of every supernode: rowStart[s] * width, r x width by rows
    int width;
};

__global__ void assembleFronts(FactorArgs args, const AssemblyTask* tasks, std::int32_t* structureError);
__global__ void smallFronts(FactorArgs args, const std::int32_t* list, std::int32_t* structureError);
__global__ void diagonalBlocks(FactorArgs args, const std::int32_t* list, int k0);
__global__ void panelRows(FactorArgs args, const TileTask* tasks, int k0);
__global__ void panelUpdate(FactorArgs args, const TileTask* tasks, int k0);
__global__ void updateMatrix(FactorArgs args, const TileTask* tasks);
__global__ void pivotSummary(FactorArgs args, const std::int32_t* supernodeOfColumn, int dimension,
                             const double* referenceDiagonal, double maxRatio, unsigned long long* counters,
                             std::int32_t* issues, int issueCapacity, double* blockRatio, std::int32_t* blockEquation);
__global__ void forwardSmall(SolveArgs a, const std::int32_t* list);
__global__ void forwardGather(SolveArgs a, const TileTask* tasks);
__global__ void forwardDiagonal(SolveArgs a, const std::int32_t* list, int k0);
__global__ void forwardUpdate(SolveArgs a, const TileTask* tasks, int k0);
__global__ void diagonalSweep(SolveArgs a, const std::int32_t* supernodeOfColumn, int dimension);
__global__ void backwardSmall(SolveArgs a, const std::int32_t* list);
__global__ void backwardRows(SolveArgs a, const TileTask* tasks);
__global__ void backwardDiagonal(SolveArgs a, const std::int32_t* list, int k0);
__global__ void backwardUpdate(SolveArgs a, const TileTask* tasks, int k0);
__global__ void toRows(const double* b, std::int64_t ld, int c0, int width, int dimension, double* x,
                       const double* scale);
__global__ void fromRows(const double* x, int c0, int width, int dimension, double* b, std::int64_t ld,
                         const double* scale);
__global__ void residualRows(const std::int64_t* rowStart, const std::int32_t* columns, const std::int32_t* source,
                             const double* values, const double* b, const double* x, double* r, int width,
                             int dimension, double* norms);
__global__ void addRows(double* x, const double* r, std::int64_t count);

} // namespace oosgpu::device
