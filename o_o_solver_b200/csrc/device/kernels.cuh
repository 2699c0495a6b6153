// The argument blocks and the kernels of the factorisation and the solves (defined in factor_kernels.cu and
// solve_kernels.cu, launched by the host engine).
#pragma once

#include "common.cuh"

#include <cstddef>
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

// The state of an indefinite factorisation beside its panels.
struct PivotArgs
{
    std::int32_t* perm;        // per pivot position: its natural equation (a permutation within each supernode)
    double* subdiagonal;       // per pivot position: e_k of a 2x2 block at its first column, 0 elsewhere
    std::int32_t* status;      // per supernode: bit 1 the block path's threshold test failed, bit 2 a pivot delayed
    std::int32_t* stepPerm;    // per supernode, 64 values: the interchanges of the current step's diagonal block
    std::int32_t* stepSwapped; // per supernode: the current step's diagonal block interchanged columns
    double* w;                 // W = L D of the current step's rows, n x 64 per large front at wOffset
    const std::int64_t* wOffset;
};

// A source of an exact front's assembly: a child's update matrix (order x order, lower triangle, column-major) and
// the front position of each of its rows.
struct FrontSource
{
    const double* values;
    const std::int32_t* positions;
    std::int32_t order;
    std::int32_t unused;
};

// One front of the exact path: its order (candidates, then its rows R(s)), its candidates (its c columns, then the
// columns its children delayed), its sources (children in increasing order) and where its panel goes (order x
// candidates, leading dimension order).
struct ExactFront
{
    std::int32_t supernode;
    std::int32_t order;
    std::int32_t candidates;
    std::int32_t sourceCount;
    const FrontSource* sources;
    double* panel;
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
    // The gather lists of the forward sweep (slot first + p for a column position p < c, dimension + rowStart + k for
    // an update row; entries: indexes of children's update rows, children in increasing order) and, after an
    // indefinite factorisation, the pivot order (the column at pivot position j is perm[j]; null otherwise).
    const std::int64_t* gatherStart;
    const std::int32_t* gatherRows;
    const std::int32_t* perm;
    int dimension;
    // The partial products of split backward row tiles: slot q at rowPartials + q * TILE * TILE (64 x 64 by rows).
    double* rowPartials;
    // The chain launches' ticket counters and ready flags (zero before each sweep), the word that makes every chain
    // task stop waiting once one wait has run out, and the host-visible record of that (mapped host memory).
    int* chainTickets;
    int* chainFlags;
    int* chainStop;
    int* chainFailed;
};

__global__ void assembleFronts(FactorArgs args, const AssemblyTask* tasks, std::int32_t* structureError);
__global__ void smallFronts(FactorArgs args, const std::int32_t* list, std::int32_t* structureError);
// Dynamic shared memory of smallFronts for fronts of order at most `order`: the front's packed lower triangle
// (order (order + 1) / 2 values) and its rows R(s).
constexpr std::size_t smallFrontSmem(int order)
{
    return static_cast<std::size_t>(order) * (order + 1) / 2 * sizeof(double) +
           static_cast<std::size_t>(order) * sizeof(std::int32_t);
}
constexpr int DIAGONAL_THREADS = 256;
// The inverse of a 64 x 64 unit lower block by 16 x 16 blocks, in shared memory by DIAGONAL_THREADS threads: `a`
// (leading dimension 65) holds L's strict lower triangle (the diagonal taken as 1; beyond the block's order the
// caller puts the identity); X = L^-1 is written into the strict upper triangle, X(i, j) at (j, i). First the four
// diagonal blocks by substitution (thread t < 64 takes column t of its block, X(i, j) = -sum_{j <= q < i} L(i, q)
// X(q, j) in q order), then the off-diagonal blocks by block diagonals, X_IJ = -X_II (sum_{J <= K < I} L_IK X_KJ).
// products: 3 x 16 x 16 doubles of shared memory. Synchronises before and after.
__device__ __forceinline__ void invertUnitLowerBlocked(double* a, double* products)
{
    constexpr int B = 64;
    constexpr int LD = B + 1;
    constexpr int SUB = 16;
    const int t = threadIdx.x;
    __syncthreads();
    if (t < B)
    {
        const int j0 = t & ~(SUB - 1);
        const int jj = t - j0;
        double x[SUB];
#pragma unroll
        for (int i = 0; i < SUB; ++i)
        {
            double sum = 0.0;
#pragma unroll
            for (int q = 0; q < i; ++q)
                if (q >= jj)
                    sum += a[(j0 + i) + (j0 + q) * LD] * x[q];
            x[i] = i == jj ? 1.0 : -sum;
            if (i > jj)
                a[t + (j0 + i) * LD] = x[i];
        }
    }
    __syncthreads();
#pragma unroll 1
    for (int d = 1; d < B / SUB; ++d)
    {
        const int count = (B / SUB - d) * SUB * SUB;
        for (int e = t; e < count; e += DIAGONAL_THREADS) // T_IJ = sum_{J <= K < I} L_IK X_KJ
        {
            const int b = e / (SUB * SUB);
            const int p = (e / SUB) % SUB;
            const int q = e % SUB;
            const int jBase = b * SUB;
            const int iRow = (b + d) * SUB + p;
            double sum = a[iRow + (jBase + q) * LD]; // X_JJ(q, q) = 1
#pragma unroll 1
            for (int r = q + 1; r < SUB; ++r)
                sum += a[iRow + (jBase + r) * LD] * a[(jBase + q) + (jBase + r) * LD];
#pragma unroll 1
            for (int kBase = jBase + SUB; kBase < (b + d) * SUB; kBase += SUB)
#pragma unroll 4
                for (int r = 0; r < SUB; ++r)
                    sum += a[iRow + (kBase + r) * LD] * a[(jBase + q) + (kBase + r) * LD];
            products[e] = sum;
        }
        __syncthreads();
        for (int e = t; e < count; e += DIAGONAL_THREADS) // X_IJ = -X_II T_IJ
        {
            const int b = e / (SUB * SUB);
            const int p = (e / SUB) % SUB;
            const int q = e % SUB;
            const int iBase = (b + d) * SUB;
            double sum = products[e];
#pragma unroll 1
            for (int r = 0; r < p; ++r)
                sum += a[(iBase + r) + (iBase + p) * LD] * products[b * SUB * SUB + r * SUB + q];
            a[(b * SUB + q) + (iBase + p) * LD] = -sum;
        }
        __syncthreads();
    }
}
// ---- the workload models' stiffness on the GPU (model_kernels.cu) ----
// One kind of element matrix (family 0 flat shell of a x b, thickness, young, poisson, turned by orientation 0..2;
// 1 hexahedron of edge a; 2 given at `given` + givenOffset, row-major); dofs x dofs, at most 24.
struct ElementKindDesc
{
    int family;
    int orientation;
    int dofs;
    int givenOffset;
    double a;
    double b;
    double thickness;
    double young;
    double poisson;
};
// A model's graph (CSR, sorted neighbours), its elements (nodes at elementStart, -1 for a clamped node; kind per
// element), the elements of each node in increasing order (CSR), and the element matrices (576 values per kind).
struct ModelArgs
{
    int nodes;
    int nodeDofs;
    std::int64_t slots;
    const std::int64_t* graphOffsets;
    const std::int32_t* neighbours;
    const std::int64_t* elementStart;
    const std::int32_t* elementNodes;
    const std::int32_t* elementKind;
    const std::int64_t* elementsOfNodeStart;
    const std::int32_t* elementsOfNode;
    const double* matrices;
};
__global__ void elementMatrices(const ElementKindDesc* kinds, const double* given, double* out);
__global__ void nodeBlocks(ModelArgs m, double* diagonalBlocks, double* offBlocks);
__global__ void cscCounts(ModelArgs m, const std::int32_t* nodeAtPosition, const std::int32_t* positionOf,
                          std::int64_t* terms);
__global__ void cscFill(ModelArgs m, const std::int32_t* nodeAtPosition, const std::int32_t* positionOf,
                        const std::int64_t* termStart, const double* diagonalBlocks, const double* offBlocks,
                        const double* lumpedMass, int which, std::int64_t* offsets, std::int32_t* rows, double* values);
__global__ void scatterPositions(const std::int32_t* nodeAtPosition, std::int32_t* positionOf, int nodes);

// The extend-add of the large fronts by pieces staged in shared memory (assembly_kernels.cu); AssemblyTask.pad holds
// the piece's first front position. Dynamic shared memory: STAGE_SMEM bytes.
__global__ void assembleStaged(FactorArgs args, const AssemblyTask* pieces, std::int32_t* structureError);
// The update matrices' Schur products fed by TMA (update_tma_kernels.cu): 128 x 128 lower tiles {front, i0, j0,
// tensor map index}; maps: the fronts' tensor maps (128 bytes each); error set to 1 when a bounded wait ran out.
// Dynamic shared memory: UPDATE_TMA_SMEM bytes.
__global__ void updateMatrixTma(FactorArgs args, const TileTask* tasks, const void* maps, int* error);
__global__ void diagonalBlocks(FactorArgs args, const std::int32_t* list, int k0);
__global__ void diagonalBlocksByColumn(FactorArgs args, const std::int32_t* list, int k0);
__global__ void panelRowsInverse(FactorArgs args, const TileTask* tasks, int k0);
constexpr std::size_t PANEL_ROWS_INVERSE_SMEM = (2 * 64 * (TILE + TILE_PAD) + 64) * sizeof(double);
__global__ void panelUpdate(FactorArgs args, const TileTask* tasks, int k0);
__global__ void updateMatrix(FactorArgs args, const TileTask* tasks);
// The mixed-precision update matrix (3xTF32 on tcgen05, mixed_kernels.cu): 128 x 128 tiles; error set to 1 when a
// bounded wait on the tensor cores ran out.
__global__ void updateMatrixMixed(FactorArgs args, const TileTask* tasks, int* error);
constexpr std::size_t MIXED_UPDATE_SMEM = 2 * 4 * 128 * 16 * 4 + 1024;
__global__ void pivotSummary(FactorArgs args, const std::int32_t* supernodeOfColumn, int dimension,
                             const double* referenceDiagonal, double maxRatio, unsigned long long* counters,
                             std::int32_t* issues, int issueCapacity, double* blockRatio, std::int32_t* blockEquation);
__global__ void forwardSmall(SolveArgs a, const std::int32_t* list, int cmax);
__global__ void gatherColumns(SolveArgs a, std::int32_t s);
__global__ void forwardGather(SolveArgs a, const TileTask* tasks);
__global__ void invertDiagonal(FactorArgs args, const TileTask* tasks);
// The row stride of a small supernode's staged inverse for c4 (its columns rounded up to 4): at least c4 and 4 more than
// a multiple of 16 (conflict-free fragment reads).
__host__ __device__ constexpr int smallInverseLd(int c4)
{
    return (c4 + 11) / 16 * 16 + 4;
}
// The inverse region of forwardSmall / backwardSmall for c4: c4 rows of smallInverseLd(c4) and room for the
// tensor-core fragment reads of rows up to 63.
__host__ __device__ constexpr int smallInverseDoubles(int c4)
{
    return 64 * smallInverseLd(c4) + 64;
}
// Dynamic shared memory of forwardSmall / backwardSmall for supernodes of at most `columns` columns: the tile
// pipeline, the inverse region and an x_F block of c4 rows by TILE + TILE_PAD (laid out for the widest tile of
// right-hand sides).
constexpr std::size_t smallSolveSmem(int columns)
{
    return static_cast<std::size_t>(TILE_SMEM_DOUBLES + smallInverseDoubles((columns + 3) & ~3) +
                                    ((columns + 3) & ~3) * (TILE + TILE_PAD)) *
           sizeof(double);
}
// The chains of the large supernodes (solve_kernels.cu). A task's shared memory: a region for its product's pipeline
// (CHAIN_STAGES slices of CHAIN_SLICE columns of A and of x; or, with an odd number of right-hand sides, the A slices
// and then CHAIN_B_DOUBLES for a chunk of solved blocks of x), reused at the end for the 64-row block b, and the
// inverse of its diagonal block.
constexpr int CHAIN_SLICE = 16;
constexpr int CHAIN_STAGES = 4;
constexpr int CHAIN_LD = TILE + TILE_PAD;
constexpr int CHAIN_B_DOUBLES = TILE * CHAIN_LD;
constexpr int CHAIN_REGION_DOUBLES = CHAIN_STAGES * 2 * CHAIN_SLICE * CHAIN_LD;
static_assert(CHAIN_REGION_DOUBLES >= CHAIN_STAGES * CHAIN_SLICE * CHAIN_LD + CHAIN_B_DOUBLES, "chain region");
constexpr std::size_t CHAIN_SMEM = static_cast<std::size_t>(CHAIN_REGION_DOUBLES + 64 * INVERSE_LD) * sizeof(double);
__global__ void forwardChain(SolveArgs a, const TileTask* tasks, int slot);
__global__ void backwardChain(SolveArgs a, const TileTask* tasks, int slot);
__global__ void diagonalSweep(SolveArgs a, const double* diagonal, int dimension);
// D of a positive definite factor as one contiguous vector (diagonal[eq] = d_eq), gathered once per factorisation.
__global__ void gatherDiagonal(FactorArgs args, const std::int32_t* supernodeOfColumn, int dimension, double* diagonal);
__global__ void backwardSmall(SolveArgs a, const std::int32_t* list, int cmax);
__global__ void backwardRows(SolveArgs a, const TileTask* tasks);
__global__ void backwardRowsReduce(SolveArgs a, const TileTask* tasks);
__global__ void toRows(const double* b, std::int64_t ld, int c0, int width, int dimension, double* x,
                       const double* scale);
__global__ void fromRows(const double* x, int c0, int width, int dimension, double* b, std::int64_t ld,
                         const double* scale);
// Rows of one group (consecutive rows with the same columns, at most RESIDUAL_GROUP) share one warp in residualRows.
constexpr int RESIDUAL_GROUP = 8;
__global__ void residualRows(const std::int64_t* rowStart, const std::int32_t* columns, const std::int32_t* source,
                             const std::int32_t* groupFirst, int groups, const double* values, const double* b,
                             const double* x, double* r, int width, double* norms);
__global__ void addRows(double* x, const double* r, std::int64_t count);

// The GMRES refinement (gmres_kernels.cu).
constexpr int GMRES_MAX_VECTORS = 12; // the Krylov vectors of one correction
__global__ void multiplyRows(const std::int64_t* rowStart, const std::int32_t* columns, const std::int32_t* source,
                             const double* values, const double* x, double* y, int width, int dimension);
__global__ void dotRowsPartials(const double* v, std::int64_t stride, int vectors, const double* w, int width,
                                int dimension, int rowsPerBlock, double* partials);
__global__ void subtractRowsCombination(double* w, const double* v, std::int64_t stride, int vectors,
                                        const double* coef, int width, std::int64_t items);
__global__ void addRowsCombination(double* x, const double* v, std::int64_t stride, int vectors, const double* y,
                                   int width, std::int64_t items);
__global__ void scaleRowsColumns(const double* in, double* out, const double* s, int width, std::int64_t items);

__global__ void smallFrontsPivoted(FactorArgs args, PivotArgs pivots, const std::int32_t* list,
                                   std::int32_t* structureError);
__global__ void pivotedDiagonal(FactorArgs args, PivotArgs pivots, const std::int32_t* list, int k0);
__global__ void permuteEarlierRows(FactorArgs args, PivotArgs pivots, const TileTask* tasks, int k0);
__global__ void panelRowsPivotedInverse(FactorArgs args, PivotArgs pivots, const TileTask* tasks, int k0);
constexpr std::size_t PANEL_ROWS_PIVOTED_SMEM = PANEL_ROWS_INVERSE_SMEM + 64 * (sizeof(double) + sizeof(int));
__global__ void updatePivoted(FactorArgs args, PivotArgs pivots, const TileTask* tasks, int k0);
__global__ void exactFront(FactorArgs args, ExactFront x, double* work, std::int32_t* perm, double* sub,
                           std::int32_t* eliminated, std::int32_t* structureError);
__global__ void copyTrailing(const double* work, std::int64_t ld, int from, int count, double* update);
__global__ void trailingFront(FactorArgs args, ExactFront x, double* schur, std::int32_t* structureError);
__global__ void inertiaPivoted(FactorArgs args, PivotArgs pivots, const std::int32_t* supernodeOfColumn, int dimension,
                               unsigned long long* counters);
__global__ void identityPermutation(std::int32_t* perm, int dimension);
__global__ void invertPermutation(const std::int32_t* perm, std::int32_t* inverse, int dimension);
__global__ void remapPivotOrder(const FrontDesc* fronts, const std::int32_t* rows, const std::int32_t* relpos,
                                const std::int32_t* inverse, std::int32_t* rowsPivot, std::int32_t* relposPivot,
                                int supernodes);
__global__ void toRowsPivoted(const double* b, std::int64_t ld, int c0, int width, int dimension, double* x,
                              const std::int32_t* perm, const double* scale);
__global__ void fromRowsPivoted(const double* x, int c0, int width, int dimension, double* b, std::int64_t ld,
                                const std::int32_t* perm, const double* scale);
__global__ void diagonalSweepPivoted(SolveArgs a, const std::int32_t* supernodeOfColumn, const double* subdiagonal,
                                     int dimension);

// The block kernels of the Lanczos run (block_kernels.cu).
constexpr int GRAM_THREADS = 256;
constexpr int GRAM_BLOCKS_MAX = 296; // 2 per SM
constexpr int COMBINE_ROWS = 32;
constexpr int COMBINE_THREADS = 256;

__global__ void randomBlock(double* x, std::int64_t ld, int rows, int columns, std::uint64_t state);
__global__ void gramPartials(const double* a, std::int64_t lda, int m, const double* y, std::int64_t ldy, int w,
                             int rows, int rowsPerBlock, double* partials);
__global__ void reducePartials(const double* partials, int blocks, int count, double* out);
__global__ void subtractProduct(double* w, std::int64_t ldw, int width, const double* a, std::int64_t lda, int m,
                                const double* c, std::int64_t ldc, int rows);
__global__ void combineRows(const double* a, std::int64_t lda, int m, const double* s, std::int64_t lds, int k,
                            double* out, std::int64_t ldo, int rows, const double* next, std::int64_t ldn, int b,
                            const double* correction);
__global__ void scaleColumn(double* x, double* y, double s, int rows);
__global__ void acceptColumn(double* x, double* mx, int rows, const double* dot, const double* gram, int width, int c,
                             int perColumn, double floorNorm, double factor, double* diagonal, double* accepted);
__global__ void scaleColumns(double* x, std::int64_t ldx, double* y, std::int64_t ldy, const double* s, int rows,
                             int columns);

__global__ void shiftedMatrix(const std::int64_t* offsets, const std::int32_t* rows, const double* stiffness,
                              const double* mass, double sigma, const double* scale, double* values, int dimension);
__global__ void diagonalProduct(const double* m, const double* x, std::int64_t ldx, double* y, std::int64_t ldy,
                                int dimension, int columns);
__global__ void symmetricProduct(const std::int64_t* rowStart, const std::int32_t* columns, const std::int32_t* source,
                                 const double* values, const double* x, std::int64_t ldx, double* y, std::int64_t ldy,
                                 int dimension, int width);

} // namespace oosgpu::device
