// C entry points over the reference's own linear algebra, declared in ref_shim.h. TEST INFRASTRUCTURE ONLY: the
// checker of the GPU path and the timed CPU baseline; the product never links it.
//
// Each function calls the reference's public API as its own callers do (FsetOrdering.cpp:16-105 for the ordering and
// the analysis, FsetSolver.cpp:136,171 for the factor and the solve, FullPathEigen.cpp:163-207 for the modes).

#include "ref_shim.h"

#include "oos/base/memory/MemoryBudget.hpp"
#include "oos/base/threading/ThreadPool.hpp"
#include "oos/linalg/dense/DenseKernels.hpp"
#include "oos/linalg/dense/KernelSelection.hpp"
#include "oos/linalg/dense/SmallEigenSolver.hpp"
#include "oos/linalg/eigen/BlockLanczos.hpp"
#include "oos/linalg/eigen/BucklingPencil.hpp"
#include "oos/linalg/eigen/PencilScaling.hpp"
#include "oos/linalg/eigen/ShiftStrategy.hpp"
#include "oos/linalg/eigen/SparsePencil.hpp"
#include "oos/linalg/eigen/SturmCheck.hpp"
#include "oos/linalg/ordering/ConstrainedOrdering.hpp"
#include "oos/linalg/ordering/NodeGraph.hpp"
#include "oos/linalg/ordering/NodePermutation.hpp"
#include "oos/linalg/sparse/SymmetricCsc.hpp"
#include "oos/linalg/supernodal/FactorSolve.hpp"
#include "oos/linalg/supernodal/PartialFactor.hpp"
#include "oos/linalg/supernodal/SupernodalFactor.hpp"
#include "oos/linalg/symbolic/SymbolicFactor.hpp"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <vector>

namespace
{
using namespace oos;
using namespace oos::linalg;

thread_local std::string g_error;

constexpr std::uint64_t UNBOUNDED = std::uint64_t{1} << 46;

double secondsSince(std::chrono::steady_clock::time_point start)
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
}

KernelKind kindOf(int family)
{
    switch (family)
    {
    case 0:
        return KernelKind::Reference;
    case 1:
        return KernelKind::Avx2;
    case 2:
        return KernelKind::Avx512;
    default:
        return KernelSelection::selectForThisProcess().kind();
    }
}

template <typename F> int guarded(F&& body)
{
    try
    {
        body();
        return 0;
    }
    catch (const std::exception& error)
    {
        g_error = error.what();
    }
    catch (...)
    {
        g_error = "unknown exception";
    }
    return -1;
}

} // namespace

struct ref_symbolic
{
    base::MemoryBudget budget{UNBOUNDED};
    NodeGraph graph;
    std::vector<std::int32_t> weights;
    SymbolicFactor symbolic;
    double orderingSeconds = 0.0;
    double analyseSeconds = 0.0;
};

struct ref_factor
{
    base::MemoryBudget budget{UNBOUNDED};
    std::unique_ptr<base::ThreadPool> pool;
    std::unique_ptr<DenseKernels> kernels;
    SymmetricCsc matrix;
    SupernodalFactor factor;
};

extern "C" const char* ref_last_error(void)
{
    return g_error.c_str();
}

extern "C" ref_symbolic* ref_analyse_trailing(int32_t node_count, const int64_t* offsets, const int32_t* neighbours,
                                              const int32_t* weights, const double* coords, int method,
                                              const int32_t* given_order, int amalgamate, int threads,
                                              const int32_t* trailing_nodes, int32_t trailing_count);

extern "C" ref_symbolic* ref_analyse(int32_t node_count, const int64_t* offsets, const int32_t* neighbours,
                                     const int32_t* weights, const double* coords, int method,
                                     const int32_t* given_order, int amalgamate, int threads)
{
    return ref_analyse_trailing(node_count, offsets, neighbours, weights, coords, method, given_order, amalgamate,
                                threads, nullptr, 0);
}

// The same with a trailing set (the boundary of a unit, ordered last: ConstrainedOrdering's trailing nodes, the last
// supernode of SymbolicFactor::analyse).
extern "C" ref_symbolic* ref_analyse_trailing(int32_t node_count, const int64_t* offsets, const int32_t* neighbours,
                                              const int32_t* weights, const double* coords, int method,
                                              const int32_t* given_order, int amalgamate, int threads,
                                              const int32_t* trailing_nodes, int32_t trailing_count)
{
    auto result = std::make_unique<ref_symbolic>();
    const int status = guarded(
        [&]
        {
            const auto adjacency = static_cast<std::size_t>(offsets[node_count]);
            result->graph = NodeGraph::fromAdjacency(
                node_count, std::span<const std::int64_t>(offsets, static_cast<std::size_t>(node_count) + 1),
                std::span<const std::int32_t>(neighbours, adjacency), result->budget);
            result->weights.assign(weights, weights + node_count);
            std::vector<base::Vec3> positions;
            if (coords != nullptr)
                for (std::int32_t k = 0; k < node_count; ++k)
                    positions.push_back(base::Vec3{coords[3 * k], coords[3 * k + 1], coords[3 * k + 2]});
            const auto start = std::chrono::steady_clock::now();
            NodePermutation order;
            if (method == 4)
                order = NodePermutation(std::span<const std::int32_t>(given_order, static_cast<std::size_t>(node_count)),
                                        result->budget);
            else
            {
                std::unique_ptr<base::ThreadPool> pool;
                if (threads > 1)
                    pool = std::make_unique<base::ThreadPool>(static_cast<std::size_t>(threads));
                const OrderingMethod chosen = method == 1   ? OrderingMethod::MinimumDegree
                                              : method == 2 ? OrderingMethod::NestedDissection
                                              : method == 3 ? OrderingMethod::Natural
                                                            : OrderingMethod::Automatic;
                const std::span<const std::int32_t> trailing(trailing_nodes,
                                                             static_cast<std::size_t>(trailing_count));
                order = ConstrainedOrdering().order(result->graph, result->weights, positions, trailing, chosen,
                                                    result->budget, pool.get());
            }
            result->orderingSeconds = secondsSince(start);
            const auto analyseStart = std::chrono::steady_clock::now();
            const AmalgamationThresholds thresholds =
                amalgamate != 0 ? AmalgamationThresholds{} : AmalgamationThresholds::none();
            result->symbolic = SymbolicFactor::analyse(result->graph, result->weights, order, trailing_count,
                                                       thresholds, result->budget);
            result->analyseSeconds = secondsSince(analyseStart);
        });
    return status == 0 ? result.release() : nullptr;
}

extern "C" void ref_symbolic_free(ref_symbolic* s)
{
    delete s;
}

extern "C" void ref_sym_sizes(const ref_symbolic* s, int64_t sizes[10])
{
    const SymbolicFactor& f = s->symbolic;
    std::int64_t rowEntries = 0;
    for (std::int32_t k = 0; k < f.supernodeCount(); ++k)
        rowEntries += f.rowCount(k);
    sizes[0] = f.nodeCount();
    sizes[1] = f.dofCount();
    sizes[2] = f.supernodeCount();
    sizes[3] = rowEntries;
    sizes[4] = f.panelValueCount();
    sizes[5] = f.factorEntryCount();
    sizes[6] = f.largestFrontValues();
    sizes[7] = f.updateStackPeakValues();
    sizes[8] = f.trailingDofCount();
    sizes[9] = 0;
}

extern "C" double ref_sym_flops(const ref_symbolic* s)
{
    return s->symbolic.flopCount();
}

extern "C" void ref_sym_times(const ref_symbolic* s, double times[2])
{
    times[0] = s->orderingSeconds;
    times[1] = s->analyseSeconds;
}

extern "C" void ref_sym_node_order(const ref_symbolic* s, int32_t* node_at_position)
{
    const NodePermutation& order = s->symbolic.nodeOrder();
    for (std::int32_t k = 0; k < order.size(); ++k)
        node_at_position[k] = order.nodeAt(k);
}

extern "C" void ref_sym_first_columns(const ref_symbolic* s, int32_t* first_column_of_position)
{
    for (std::int32_t k = 0; k <= s->symbolic.nodeCount(); ++k)
        first_column_of_position[k] = s->symbolic.firstColumnOfPosition(k);
}

extern "C" void ref_sym_supernodes(const ref_symbolic* s, int32_t* first_position, int32_t* parent)
{
    const Supernodes& supernodes = s->symbolic.supernodes();
    for (std::int32_t k = 0; k <= supernodes.count(); ++k)
        first_position[k] = supernodes.firstPosition(k);
    for (std::int32_t k = 0; k < supernodes.count(); ++k)
        parent[k] = supernodes.parent(k);
}

extern "C" void ref_sym_rows(const ref_symbolic* s, int64_t* row_start, int32_t* rows)
{
    const SymbolicFactor& f = s->symbolic;
    row_start[0] = 0;
    for (std::int32_t k = 0; k < f.supernodeCount(); ++k)
    {
        const auto r = f.rows(k);
        std::copy(r.begin(), r.end(), rows + row_start[k]);
        row_start[k + 1] = row_start[k] + static_cast<std::int64_t>(r.size());
    }
}

extern "C" ref_factor* ref_factorise(const ref_symbolic* s, int32_t dimension, const int64_t* col_offsets,
                                     const int32_t* rows, const double* values, int pivoting, int family, int threads,
                                     double max_ratio, int bailout, double* seconds)
{
    auto result = std::make_unique<ref_factor>();
    const int status = guarded(
        [&]
        {
            const auto terms = static_cast<std::size_t>(col_offsets[dimension]);
            result->matrix = SymmetricCsc::fromCompressedColumns(
                dimension, std::span<const std::int64_t>(col_offsets, static_cast<std::size_t>(dimension) + 1),
                std::span<const std::int32_t>(rows, terms), std::span<const double>(values, terms), result->budget);
            DenseKernelOptions options;
            if (threads > 1)
            {
                result->pool = std::make_unique<base::ThreadPool>(static_cast<std::size_t>(threads));
                options.pool = result->pool.get();
            }
            result->kernels = std::make_unique<DenseKernels>(kindOf(family), options);
            FactorOptions factorOptions;
            factorOptions.pivoting = pivoting != 0 ? PivotingMode::Indefinite : PivotingMode::PositiveDefinite;
            factorOptions.pivotPolicy.maxRatio = max_ratio;
            factorOptions.pivotPolicy.bailout = bailout;
            const auto start = std::chrono::steady_clock::now();
            result->factor = SupernodalFactor::factorise(s->symbolic, result->matrix, *result->kernels, factorOptions,
                                                         result->budget);
            if (seconds != nullptr)
                seconds[0] = secondsSince(start);
        });
    return status == 0 ? result.release() : nullptr;
}

extern "C" void ref_factor_free(ref_factor* f)
{
    delete f;
}

extern "C" void ref_factor_info(const ref_factor* f, int64_t info[8], double* largest_ratio)
{
    const SupernodalFactor& factor = f->factor;
    info[0] = static_cast<int64_t>(factor.inertia().positive);
    info[1] = static_cast<int64_t>(factor.inertia().negative);
    info[2] = static_cast<int64_t>(factor.inertia().zero);
    info[3] = factor.delayedPivotCount();
    info[4] = factor.twoByTwoPivotCount();
    info[5] = factor.pivotDiagnostics().issueCount();
    info[6] = factor.pivotDiagnostics().equationOfLargestRatio();
    info[7] = static_cast<int64_t>(factor.kernel());
    if (largest_ratio != nullptr)
        *largest_ratio = factor.pivotDiagnostics().largestRatio();
}

extern "C" int ref_factor_panel(const ref_factor* f, int32_t s, int64_t* eliminated, int64_t* row_count,
                                double* values, int32_t* rows, double* subdiagonal)
{
    return guarded(
        [&]
        {
            const FactorPanel panel = f->factor.panel(s);
            *eliminated = static_cast<int64_t>(panel.eliminatedCount());
            *row_count = static_cast<int64_t>(panel.rows.size());
            if (values != nullptr)
                for (std::size_t j = 0; j < panel.eliminatedCount(); ++j)
                    for (std::size_t i = 0; i < panel.rows.size(); ++i)
                        values[i + j * panel.rows.size()] = panel.values(i, j);
            if (rows != nullptr)
                std::copy(panel.rows.begin(), panel.rows.end(), rows);
            if (subdiagonal != nullptr)
                for (std::size_t k = 0; k < panel.eliminatedCount(); ++k)
                    subdiagonal[k] = panel.subdiagonal != nullptr ? panel.subdiagonal[k] : 0.0;
        });
}

extern "C" int ref_solve(const ref_factor* f, double* b, int64_t ld, int64_t columns, int threads, double* seconds)
{
    return guarded(
        [&]
        {
            (void)threads;
            const DenseMatrixView view{b, static_cast<std::size_t>(f->factor.dimension()),
                                       static_cast<std::size_t>(columns), static_cast<std::size_t>(ld)};
            const auto start = std::chrono::steady_clock::now();
            FactorSolve(f->factor, *f->kernels).solve(view);
            if (seconds != nullptr)
                seconds[0] = secondsSince(start);
        });
}

// PartialFactor (src/linalg/supernodal/PartialFactor.cpp): K*, condensed loads and recovery.
struct ref_partial
{
    base::MemoryBudget budget{UNBOUNDED};
    std::unique_ptr<DenseKernels> kernels;
    SymmetricCsc matrix;
    PartialFactor factor;
};

extern "C" ref_partial* ref_partial_factorise(const ref_symbolic* s, int32_t dimension, const int64_t* col_offsets,
                                              const int32_t* rows, const double* values, int family,
                                              double* schur_complement)
{
    auto result = std::make_unique<ref_partial>();
    const int status = guarded(
        [&]
        {
            const auto terms = static_cast<std::size_t>(col_offsets[dimension]);
            result->matrix = SymmetricCsc::fromCompressedColumns(
                dimension, std::span<const std::int64_t>(col_offsets, static_cast<std::size_t>(dimension) + 1),
                std::span<const std::int32_t>(rows, terms), std::span<const double>(values, terms), result->budget);
            result->kernels = std::make_unique<DenseKernels>(kindOf(family), DenseKernelOptions{});
            result->factor = PartialFactor::factorise(s->symbolic, result->matrix, *result->kernels, FactorOptions{},
                                                      result->budget);
            const DenseMatrix& k = result->factor.schurComplement();
            for (std::size_t j = 0; j < k.columns(); ++j)
                for (std::size_t i = 0; i < k.rows(); ++i)
                    schur_complement[i + j * k.rows()] = k(i, j);
        });
    return status == 0 ? result.release() : nullptr;
}

extern "C" void ref_partial_free(ref_partial* p)
{
    delete p;
}

// f* (trailing x columns, column-major) of loads (dimension x columns, column-major).
extern "C" int ref_partial_condense(const ref_partial* p, const double* loads, int64_t columns, double* condensed)
{
    return guarded(
        [&]
        {
            const auto n = static_cast<std::size_t>(p->factor.dimension());
            const ConstDenseMatrixView view{loads, n, static_cast<std::size_t>(columns), n};
            base::MemoryBudget budget{UNBOUNDED};
            const DenseMatrix f = p->factor.condenseLoads(view, *p->kernels, budget);
            for (std::size_t j = 0; j < f.columns(); ++j)
                for (std::size_t i = 0; i < f.rows(); ++i)
                    condensed[i + j * f.rows()] = f(i, j);
        });
}

// loads (dimension x columns) -> the solution with the trailing rows given (trailing x columns).
extern "C" int ref_partial_recover(const ref_partial* p, double* loads, int64_t columns, const double* trailing)
{
    return guarded(
        [&]
        {
            const auto n = static_cast<std::size_t>(p->factor.dimension());
            const auto t = static_cast<std::size_t>(p->factor.trailingDofCount());
            const DenseMatrixView x{loads, n, static_cast<std::size_t>(columns), n};
            const ConstDenseMatrixView b{trailing, t, static_cast<std::size_t>(columns), t};
            p->factor.recover(x, b, *p->kernels);
        });
}

namespace
{

// SparsePencil (buckling false) or BucklingPencil (the second matrix K_d) + BlockLanczos::solve of one request.
int eigenSolve(bool buckling, const ref_symbolic* s, int32_t dimension, const int64_t* col_offsets, const int32_t* rows,
                         const double* stiffness, const double* mass, double lower, double upper, int64_t mode_count,
                         int64_t block_size, int64_t modes_per_shift, int family, int threads, double* eigenvalues,
                         int64_t capacity, double* eigenvectors, double* shifts, int64_t max_shifts,
                         int64_t counts[5], double* seconds)
{
    return guarded(
        [&]
        {
            base::MemoryBudget budget{UNBOUNDED};
            const auto terms = static_cast<std::size_t>(col_offsets[dimension]);
            const std::span<const std::int64_t> offsets(col_offsets, static_cast<std::size_t>(dimension) + 1);
            const std::span<const std::int32_t> rowSpan(rows, terms);
            const SymmetricCsc k = SymmetricCsc::fromCompressedColumns(
                dimension, offsets, rowSpan, std::span<const double>(stiffness, terms), budget);
            const SymmetricCsc m = SymmetricCsc::fromCompressedColumns(dimension, offsets, rowSpan,
                                                                       std::span<const double>(mass, terms), budget);
            std::unique_ptr<base::ThreadPool> pool;
            DenseKernelOptions options;
            if (threads > 1)
            {
                pool = std::make_unique<base::ThreadPool>(static_cast<std::size_t>(threads));
                options.pool = pool.get();
            }
            const DenseKernels kernels(kindOf(family), options);
            FactorOptions factorOptions;
            const auto start = std::chrono::steady_clock::now();
            std::unique_ptr<ShiftedPencil> pencil;
            if (buckling)
                pencil = std::make_unique<BucklingPencil>(s->symbolic, k, m, kernels, factorOptions, budget);
            else
                pencil = std::make_unique<SparsePencil>(s->symbolic, k, m, kernels, factorOptions, budget);
            LanczosOptions lanczos;
            if (block_size > 0)
                lanczos.blockSize = static_cast<std::size_t>(block_size);
            if (modes_per_shift > 0)
                lanczos.modesPerShift = static_cast<std::size_t>(modes_per_shift);
            EigenRequest request;
            request.lowerBound = lower;
            request.upperBound = upper;
            request.modeCount = static_cast<std::size_t>(mode_count);
            const EigenSolution solution = BlockLanczos(lanczos).solve(*pencil, request, kernels, budget);
            if (seconds != nullptr)
                seconds[0] = secondsSince(start);
            const std::size_t found = std::min<std::size_t>(solution.eigenvalues.size(),
                                                            static_cast<std::size_t>(capacity));
            for (std::size_t j = 0; j < found; ++j)
            {
                eigenvalues[j] = solution.eigenvalues[j];
                if (eigenvectors != nullptr)
                    for (std::size_t i = 0; i < static_cast<std::size_t>(dimension); ++i)
                        eigenvectors[i + j * static_cast<std::size_t>(dimension)] =
                            solution.eigenvectors.data()[i + j * solution.eigenvectors.leadingDimension()];
            }
            const std::size_t records = std::min<std::size_t>(solution.shifts.size(), static_cast<std::size_t>(max_shifts));
            for (std::size_t r = 0; r < records && shifts != nullptr; ++r)
            {
                const ShiftRecord& record = solution.shifts[r];
                double* out = shifts + 7 * r;
                out[0] = record.shift;
                out[1] = static_cast<double>(static_cast<int>(record.purpose));
                out[2] = static_cast<double>(record.sturmCount);
                out[3] = record.hasLanczosRun ? 1.0 : 0.0;
                out[4] = static_cast<double>(record.blockSteps);
                out[5] = static_cast<double>(record.restarts);
                out[6] = static_cast<double>(record.convergedCount);
            }
            counts[0] = static_cast<int64_t>(found);
            counts[1] = static_cast<int64_t>(solution.factorisationCount);
            counts[2] = static_cast<int64_t>(solution.shifts.size());
            counts[3] = static_cast<int64_t>(solution.verifiedCount);
            counts[4] = solution.isComplete ? 1 : 0;
        });
}

} // namespace

extern "C" int ref_modes(const ref_symbolic* s, int32_t dimension, const int64_t* col_offsets, const int32_t* rows,
                         const double* stiffness, const double* mass, double lower, double upper, int64_t mode_count,
                         int64_t block_size, int64_t modes_per_shift, int family, int threads, double* eigenvalues,
                         int64_t capacity, double* eigenvectors, double* shifts, int64_t max_shifts,
                         int64_t counts[5], double* seconds)
{
    return eigenSolve(false, s, dimension, col_offsets, rows, stiffness, mass, lower, upper, mode_count, block_size,
                      modes_per_shift, family, threads, eigenvalues, capacity, eigenvectors, shifts, max_shifts, counts,
                      seconds);
}

extern "C" int ref_buckling(const ref_symbolic* s, int32_t dimension, const int64_t* col_offsets,
                            const int32_t* rows, const double* stiffness, const double* differential, double lower,
                            double upper, int64_t mode_count, int64_t block_size, int64_t modes_per_shift, int family,
                            int threads, double* eigenvalues, int64_t capacity, double* eigenvectors, double* shifts,
                            int64_t max_shifts, int64_t counts[5], double* seconds)
{
    return eigenSolve(true, s, dimension, col_offsets, rows, stiffness, differential, lower, upper, mode_count,
                      block_size, modes_per_shift, family, threads, eigenvalues, capacity, eigenvectors, shifts,
                      max_shifts, counts, seconds);
}

extern "C" int ref_pencil_scale(int32_t dimension, const int64_t* col_offsets, const int32_t* rows,
                                const double* values, double* scale)
{
    return guarded(
        [&]
        {
            base::MemoryBudget budget{UNBOUNDED};
            const auto terms = static_cast<std::size_t>(col_offsets[dimension]);
            const SymmetricCsc k = SymmetricCsc::fromCompressedColumns(
                dimension, std::span<const std::int64_t>(col_offsets, static_cast<std::size_t>(dimension) + 1),
                std::span<const std::int32_t>(rows, terms), std::span<const double>(values, terms), budget);
            const auto scales = pencilScaleOf(k, budget);
            std::copy(scales.span().begin(), scales.span().end(), scale);
        });
}

extern "C" int ref_sturm_verify(int64_t points, const double* shifts, const int64_t* counts, int64_t values,
                                const double* sorted, double result[6])
{
    return guarded(
        [&]
        {
            SturmCheck sturm;
            for (int64_t k = 0; k < points; ++k)
                sturm.addPoint({shifts[k], static_cast<std::size_t>(counts[k])});
            const SturmVerification v =
                sturm.verify(std::span<const double>(sorted, static_cast<std::size_t>(values)));
            result[0] = v.verifiedUpTo;
            result[1] = static_cast<double>(v.verifiedCount);
            result[2] = v.hasMismatch ? 1.0 : 0.0;
            result[3] = v.mismatch.lower;
            result[4] = v.mismatch.upper;
            result[5] = static_cast<double>(v.mismatch.expectedCount) * 1e6 + static_cast<double>(v.mismatch.foundCount);
        });
}

extern "C" int ref_shift_next(double lower, double upper, int64_t mode_count, double scale, const double verification[6],
                              int64_t values, const double* sorted, int64_t ritz_count, const double* ritz,
                              int64_t shift_count, const double* lanczos_shifts, double* shift, int32_t* purpose)
{
    return guarded(
        [&]
        {
            EigenRequest request;
            request.lowerBound = lower;
            request.upperBound = upper;
            request.modeCount = static_cast<std::size_t>(mode_count);
            const ShiftStrategy strategy(request, scale);
            SturmVerification v;
            v.verifiedUpTo = verification[0];
            v.verifiedCount = static_cast<std::size_t>(verification[1]);
            v.hasMismatch = verification[2] != 0.0;
            v.mismatch.lower = verification[3];
            v.mismatch.upper = verification[4];
            const ShiftChoice choice = strategy.nextShift(
                v, std::span<const double>(sorted, static_cast<std::size_t>(values)),
                std::span<const double>(ritz, static_cast<std::size_t>(ritz_count)),
                std::span<const double>(lanczos_shifts, static_cast<std::size_t>(shift_count)));
            *shift = choice.shift;
            *purpose = static_cast<int32_t>(choice.purpose);
        });
}

extern "C" int ref_symmetric_eigen(const double* a, int64_t p, int64_t ld, double* eigenvalues, double* eigenvectors)
{
    return guarded(
        [&]
        {
            base::MemoryBudget budget{UNBOUNDED};
            const auto n = static_cast<std::size_t>(p);
            const SymmetricEigenDecomposition d =
                SmallEigenSolver::decompose(ConstDenseMatrixView(a, n, n, static_cast<std::size_t>(ld)), budget);
            for (std::size_t j = 0; j < n; ++j)
            {
                eigenvalues[j] = d.eigenvalues[j];
                for (std::size_t i = 0; i < n; ++i)
                    eigenvectors[i + j * n] = d.eigenvectors(i, j);
            }
        });
}
