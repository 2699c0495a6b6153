// The block shift-invert Lanczos solver on the GPU (declared in lanczos.hpp): the reference's BlockLanczos::solve
// (src/linalg/eigen/BlockLanczos.cpp:84-246), LanczosRun (src/linalg/eigen/LanczosRun.cpp), MassOrthogonalizer
// (src/linalg/eigen/MassOrthogonalizer.cpp), the resident part of EigenvectorStore (src/linalg/eigen/
// EigenvectorStore.cpp), ShiftStrategy (src/linalg/eigen/ShiftStrategy.cpp) and SturmCheck (src/linalg/eigen/
// SturmCheck.cpp).
//
// Device side: the basis (dimension x basisColumns), four blocks, the eigenvectors found, and every product over the
// rows (the block kernels of block_kernels.cu, on the pencil's stream). Host side: the projected matrix T, its
// eigen-decomposition, the Sturm walk and the shift strategy; the host reads back the projection coefficients and the
// norms of each step (a few hundred values).

#include "lanczos.hpp"

#include "../device/kernels.cuh"
#include "host_api.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <numeric>
#include <string>

namespace oosgpu::eigen
{

void DeviceFree::operator()(double* p) const noexcept
{
    if (p != nullptr)
        cudaFree(p);
}

namespace
{

constexpr double INFINITE = std::numeric_limits<double>::infinity();
constexpr double EPSILON = std::numeric_limits<double>::epsilon();
constexpr std::uint64_t GOLDEN_GAMMA = 0x9E3779B97F4A7C15ULL;

// LanczosRun's constants (src/linalg/eigen/LanczosRun.hpp:103-115): the deflation threshold relative to
// eps sqrt(n) |Op|, the random replacements of a deflated column, the negligible and the accurate Ritz values.
constexpr double DEFLATION_FACTOR = 100.0;
constexpr std::size_t REPLACEMENT_ATTEMPTS = 3;
constexpr double NEGLIGIBLE_RITZ_VALUE = 1.0e-14;
constexpr double ACCURATE_RITZ_RATIO = 1.0e-3;
// Block classical Gram-Schmidt twice ("twice is enough").
constexpr int ORTHOGONALISATION_PASSES = 2;
// BlockLanczos's (src/linalg/eigen/SolveSupport.hpp:19-22): the moves off a singular shift, the seed step of a run.
constexpr std::size_t MAX_SINGULAR_MOVES = 3;
constexpr std::uint64_t SEED_STEP = 0x9E3779B97F4A7C15ULL;
constexpr double MAXIMUM_CONVERGENCE_TOLERANCE = 1.0e-2;
// ShiftStrategy's (src/linalg/eigen/ShiftStrategy.cpp:20-27).
constexpr double SAME_SHIFT_TOLERANCE = 1.0e-3;
constexpr std::size_t MAX_CLEARANCE_PASSES = 64;
// The sweeps of the implicit QL method allowed per eigenvalue.
constexpr int MAX_QL_SWEEPS = 60;
// The largest shared memory of one block (the basis rows of combineRows).
constexpr std::size_t MAX_SHARED_BYTES = 227 * 1024;

void check(cudaError_t status, const char* what)
{
    if (status != cudaSuccess)
        throw Error(status == cudaErrorMemoryAllocation ? STATUS_MEMORY_BUDGET : STATUS_CUDA,
                    std::string(what) + ": " + cudaGetErrorString(status));
}

std::unique_ptr<double, DeviceFree> deviceValues(std::size_t count, const char* what)
{
    void* p = nullptr;
    check(cudaMalloc(&p, std::max<std::size_t>(count, 1) * sizeof(double)), what);
    return std::unique_ptr<double, DeviceFree>(static_cast<double*>(p));
}

// A device buffer that grows on demand.
class Scratch
{
public:
    double* reserve(std::size_t count, const char* what)
    {
        if (count > m_count || !m_data)
        {
            m_data.reset();
            m_data = deviceValues(std::max(count, m_count * 3 / 2), what);
            m_count = std::max(count, m_count * 3 / 2);
        }
        return m_data.get();
    }

private:
    std::unique_ptr<double, DeviceFree> m_data;
    std::size_t m_count = 0;
};

std::size_t roundUp(std::size_t value, std::size_t multiple)
{
    return (value + multiple - 1) / multiple * multiple;
}

unsigned blocksFor(std::int64_t items, int threads)
{
    return static_cast<unsigned>(std::max<std::int64_t>((items + threads - 1) / threads, 1));
}

// sqrt(a^2 + b^2) from sqrt and divisions (no overflow for finite inputs).
double hypotenuse(double a, double b)
{
    a = std::abs(a);
    b = std::abs(b);
    const double big = std::max(a, b);
    if (big == 0.0)
        return 0.0;
    const double small = std::min(a, b) / big;
    return big * std::sqrt(1.0 + small * small);
}

// Wall seconds of the phases of the runs; each timed phase ends with its stream drained.
struct Phases
{
    double operatorSeconds = 0.0;
    double orthogonalisationSeconds = 0.0;
    double projectedSeconds = 0.0;
};

template <typename Body> void timed(double& counter, cudaStream_t stream, Body&& body)
{
    const auto start = std::chrono::steady_clock::now();
    body();
    check(cudaStreamSynchronize(stream), "Lanczos");
    counter += std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
}

// The block operations over the rows of the pencil's dimension, on one stream.
class BlockOps
{
public:
    BlockOps(cudaStream_t stream, int rows) : m_stream(stream), m_rows(rows)
    {
        m_blocks = std::clamp((rows + 255) / 256, 1, device::GRAM_BLOCKS_MAX);
        m_rowsPerBlock = (rows + m_blocks - 1) / m_blocks;
    }

    [[nodiscard]] cudaStream_t stream() const noexcept { return m_stream; }
    [[nodiscard]] int rows() const noexcept { return m_rows; }
    [[nodiscard]] std::int64_t launches() const noexcept { return m_launches; }

    // out (device, m x w, leading dimension m) = a^T y over the rows.
    void gram(const double* a, std::int64_t lda, std::size_t m, const double* y, std::int64_t ldy, std::size_t w,
              double* out)
    {
        if (m == 0 || w == 0)
            return;
        const std::size_t count = m * w;
        double* partials = m_partials.reserve(count * static_cast<std::size_t>(m_blocks), "Lanczos: partial sums");
        device::gramPartials<<<m_blocks, device::GRAM_THREADS, 0, m_stream>>>(
            a, lda, static_cast<int>(m), y, ldy, static_cast<int>(w), m_rows, m_rowsPerBlock, partials);
        device::reducePartials<<<blocksFor(static_cast<std::int64_t>(count), 128), 128, 0, m_stream>>>(
            partials, m_blocks, static_cast<int>(count), out);
        m_launches += 2;
        check(cudaGetLastError(), "Lanczos: inner products");
    }

    // w(:, 0:width) -= a(:, 0:m) c, c m x width with leading dimension m (device).
    void subtract(double* w, std::int64_t ldw, std::size_t width, const double* a, std::int64_t lda, std::size_t m,
                  const double* c)
    {
        if (m == 0 || width == 0)
            return;
        const std::size_t chunk = std::max<std::size_t>(1, 4096 / width);
        for (std::size_t i0 = 0; i0 < m; i0 += chunk)
        {
            const std::size_t mm = std::min(chunk, m - i0);
            device::subtractProduct<<<blocksFor(m_rows, 256), 256, mm * width * sizeof(double), m_stream>>>(
                w, ldw, static_cast<int>(width), a + static_cast<std::int64_t>(i0) * lda, lda, static_cast<int>(mm),
                c + i0, static_cast<std::int64_t>(m), m_rows);
            ++m_launches;
        }
        check(cudaGetLastError(), "Lanczos: block update");
    }

    // out(:, 0:k) = a(:, 0:m) s - next correction (the second term when `next` is given); out may be a's first columns.
    void combine(const double* a, std::int64_t lda, std::size_t m, const double* s, std::int64_t lds, std::size_t k,
                 double* out, std::int64_t ldo, const double* next, std::int64_t ldn, std::size_t b,
                 const double* correction)
    {
        if (k == 0)
            return;
        const std::size_t shared = std::max<std::size_t>(m, 1) * device::COMBINE_ROWS * sizeof(double);
        if (shared > MAX_SHARED_BYTES)
            throw Error(STATUS_INVALID_ARGUMENT, "Lanczos: a basis of " + std::to_string(m) +
                                                     " columns is wider than the products by rows allow (" +
                                                     std::to_string(MAX_SHARED_BYTES / device::COMBINE_ROWS / 8) +
                                                     "); lower the modes per shift or the block size");
        if (shared > 48 * 1024)
            // The limit is the process's: the largest, so that no solve lowers another's.
            check(cudaFuncSetAttribute(device::combineRows, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(MAX_SHARED_BYTES)),
                  "Lanczos: shared memory of the basis products");
        device::combineRows<<<blocksFor(m_rows, device::COMBINE_ROWS), device::COMBINE_THREADS, shared, m_stream>>>(
            a, lda, static_cast<int>(m), s, lds, static_cast<int>(k), out, ldo, m_rows, next, ldn,
            static_cast<int>(b), correction);
        ++m_launches;
        check(cudaGetLastError(), "Lanczos: basis products");
    }

    // The reference's fillRandom from `state`, which advances by one draw per value.
    void random(double* x, std::int64_t ld, std::size_t columns, std::uint64_t& state)
    {
        const std::int64_t items = static_cast<std::int64_t>(m_rows) * static_cast<std::int64_t>(columns);
        device::randomBlock<<<blocksFor(items, 256), 256, 0, m_stream>>>(x, ld, m_rows, static_cast<int>(columns),
                                                                         state);
        ++m_launches;
        check(cudaGetLastError(), "Lanczos: random block");
        state += static_cast<std::uint64_t>(items) * GOLDEN_GAMMA;
    }

    void scale(double* x, double* y, double s)
    {
        device::scaleColumn<<<blocksFor(m_rows, 256), 256, 0, m_stream>>>(x, y, s, m_rows);
        ++m_launches;
        check(cudaGetLastError(), "Lanczos: scale");
    }

    void scaleColumns(double* x, std::int64_t ldx, const double* s, std::size_t columns)
    {
        const std::int64_t items = static_cast<std::int64_t>(m_rows) * static_cast<std::int64_t>(columns);
        device::scaleColumns<<<blocksFor(items, 256), 256, 0, m_stream>>>(x, ldx, nullptr, 0, s, m_rows,
                                                                          static_cast<int>(columns));
        ++m_launches;
        check(cudaGetLastError(), "Lanczos: scale");
    }

    void copy(double* dst, std::int64_t ldd, const double* src, std::int64_t lds, std::size_t columns)
    {
        if (columns == 0)
            return;
        check(cudaMemcpy2DAsync(dst, static_cast<std::size_t>(ldd) * sizeof(double), src,
                                static_cast<std::size_t>(lds) * sizeof(double),
                                static_cast<std::size_t>(m_rows) * sizeof(double), columns, cudaMemcpyDeviceToDevice,
                                m_stream),
              "Lanczos: block copy");
    }

    void zero(double* x, std::int64_t ld, std::size_t columns)
    {
        check(cudaMemset2DAsync(x, static_cast<std::size_t>(ld) * sizeof(double), 0,
                                static_cast<std::size_t>(m_rows) * sizeof(double), columns, m_stream),
              "Lanczos: zero block");
    }

    void download(const double* device, std::size_t count, double* host)
    {
        if (count == 0)
            return;
        check(cudaMemcpyAsync(host, device, count * sizeof(double), cudaMemcpyDeviceToHost, m_stream),
              "Lanczos: read back");
        check(cudaStreamSynchronize(m_stream), "Lanczos: read back");
    }

    void upload(double* device, const double* host, std::size_t count)
    {
        if (count == 0)
            return;
        check(cudaMemcpyAsync(device, host, count * sizeof(double), cudaMemcpyHostToDevice, m_stream),
              "Lanczos: upload");
    }

private:
    cudaStream_t m_stream;
    int m_rows;
    int m_blocks = 1;
    int m_rowsPerBlock = 1;
    Scratch m_partials;
    std::int64_t m_launches = 0;
};

// The basis and its blocks (LanczosWorkspace, LanczosRun.cpp:61-76), column-major with leading dimension n.
struct Workspace
{
    Workspace(std::size_t n, std::size_t basisColumns, std::size_t b)
        : basis(deviceValues(n * basisColumns, "Lanczos: basis")),
          next(deviceValues(n * b, "Lanczos: blocks")),
          product(deviceValues(n * b, "Lanczos: blocks")),
          massScratch(deviceValues(n * b, "Lanczos: blocks")),
          massOfNext(deviceValues(n * b, "Lanczos: blocks")),
          small(deviceValues(basisColumns * basisColumns + b * basisColumns + b, "Lanczos: projected vectors"))
    {
    }

    std::unique_ptr<double, DeviceFree> basis;
    std::unique_ptr<double, DeviceFree> next;
    std::unique_ptr<double, DeviceFree> product;
    std::unique_ptr<double, DeviceFree> massScratch;
    std::unique_ptr<double, DeviceFree> massOfNext;
    // The Ritz vectors of a restart or of the converged pairs, and the purification terms (uploaded).
    std::unique_ptr<double, DeviceFree> small;
};

// The eigenvectors found, resident in device memory (EigenvectorStore without its spool: 180 GB hold them), with
// their eigenvalues and residual bounds in the order found.
class Store
{
public:
    Store(cudaStream_t stream, std::size_t n, std::size_t initialCapacity)
        : m_stream(stream), m_n(n), m_capacity(std::max<std::size_t>(initialCapacity, 1)),
          m_vectors(deviceValues(n * m_capacity, "Lanczos: eigenvectors found"))
    {
    }

    [[nodiscard]] const double* vectors() const noexcept { return m_vectors.get(); }
    [[nodiscard]] std::size_t count() const noexcept { return m_values.size(); }
    [[nodiscard]] const std::vector<double>& eigenvalues() const noexcept { return m_values; }
    [[nodiscard]] const std::vector<double>& residualBounds() const noexcept { return m_bounds; }

    double* prepareColumns(std::size_t columns)
    {
        const std::size_t needed = count() + columns;
        if (needed > m_capacity)
        {
            const std::size_t grown = std::max(needed, static_cast<std::size_t>(std::ceil(1.5 * m_capacity)));
            auto larger = deviceValues(m_n * grown, "Lanczos: eigenvectors found");
            if (count() > 0)
                check(cudaMemcpyAsync(larger.get(), m_vectors.get(), m_n * count() * sizeof(double),
                                      cudaMemcpyDeviceToDevice, m_stream),
                      "Lanczos: grow the eigenvectors");
            check(cudaStreamSynchronize(m_stream), "Lanczos: grow the eigenvectors");
            m_vectors = std::move(larger);
            m_capacity = grown;
        }
        return m_vectors.get() + m_n * count();
    }

    void commit(const std::vector<double>& values, const std::vector<double>& bounds)
    {
        m_values.insert(m_values.end(), values.begin(), values.end());
        m_bounds.insert(m_bounds.end(), bounds.begin(), bounds.end());
    }

private:
    cudaStream_t m_stream;
    std::size_t m_n;
    std::size_t m_capacity;
    std::unique_ptr<double, DeviceFree> m_vectors;
    std::vector<double> m_values;
    std::vector<double> m_bounds;
};

struct RunSettings
{
    std::size_t blockSize = 1;
    std::size_t basisColumns = 3;
    std::size_t target = 1;
    double convergenceTolerance = 1.0e-10;
    std::size_t maximumRestarts = 1;
    std::uint64_t seed = 0;
    // A start block given by the caller (device, n x blockSize, leading dimension startLd), in place of the random one.
    const double* startBlock = nullptr;
    std::int64_t startLd = 0;
};

struct RunResult
{
    std::size_t convergedCount = 0;
    std::vector<double> ritzEstimates;
    std::size_t blockSteps = 0;
    std::size_t restarts = 0;
    bool isSpaceExhausted = false;
};

// One Lanczos run at the shift of the pencil's current factor (LanczosRun::run, LanczosRun.cpp:447-534): thick
// restarts, full reorthogonalisation in the M inner product, purified Ritz vectors.
class Run
{
public:
    Run(ShiftedPencil& pencil, BlockOps& ops, Workspace& workspace, const RunSettings& settings, Phases& phases)
        : m_pencil(pencil), m_ops(ops), m_ws(workspace), m_settings(settings), m_phases(phases),
          m_n(static_cast<std::size_t>(pencil.dimension())), m_capacity(settings.basisColumns)
    {
    }

    RunResult run(double shift, Store& store)
    {
        RunResult result;
        const std::size_t b = m_settings.blockSize;
        const std::size_t ld = m_settings.basisColumns;
        m_randomState = m_settings.seed;
        m_projected.assign(ld * ld, 0.0);
        m_coupling.assign(b * ld, 0.0);
        m_columns = 0;
        m_operatorNorm = 0.0;
        const cudaStream_t stream = m_ops.stream();
        startBlock(store);
        if (m_nextColumnCount == 0)
        {
            result.isSpaceExhausted = !probeBeyondLocked(shift, store, result);
            return result;
        }
        Ritz ritz;
        std::vector<double> coefficients;
        std::vector<double> secondCoefficients;
        std::vector<double> triangle;
        std::vector<double> norms(b, 0.0);
        const auto n = static_cast<std::int64_t>(m_n);
        while (true)
        {
            if (m_columns + b > m_capacity)
            {
                if (result.restarts >= m_settings.maximumRestarts || m_capacity < 3 * b)
                    break;
                timed(m_phases.orthogonalisationSeconds, stream, [&] { restart(ritz); });
                ++result.restarts;
            }
            const std::size_t p = m_columns;
            for (std::size_t j = 0; j < p; ++j)
                for (std::size_t r = 0; r < b; ++r)
                {
                    m_projected[(p + r) + j * ld] = m_coupling[r + j * b];
                    m_projected[j + (p + r) * ld] = m_coupling[r + j * b];
                }
            double* basis = m_ws.basis.get();
            m_ops.copy(basis + n * static_cast<std::int64_t>(p), n, m_ws.next.get(), n, b);
            m_basisInUse = p + b;

            double* w = m_ws.product.get();
            m_ops.copy(w, n, basis + n * static_cast<std::int64_t>(p), n, b);
            timed(m_phases.operatorSeconds, stream, [&] { applyOperator(w, b); });
            timed(m_phases.orthogonalisationSeconds, stream,
                  [&]
                  {
                      projectOut(w, b, store, p + b, &coefficients, norms.data());
                      projectOut(w, b, store, p + b, &secondCoefficients, nullptr);
                  });
            for (const double norm : norms)
                m_operatorNorm = std::max(m_operatorNorm, norm);
            const std::size_t rows = p + b;
            for (std::size_t c = 0; c < b; ++c)
                for (std::size_t r = 0; r <= c; ++r)
                {
                    const double upper = coefficients[(p + r) + c * rows] + secondCoefficients[(p + r) + c * rows];
                    const double lower = coefficients[(p + c) + r * rows] + secondCoefficients[(p + c) + r * rows];
                    const double value = 0.5 * (upper + lower);
                    m_projected[(p + r) + (p + c) * ld] = value;
                    m_projected[(p + c) + (p + r) * ld] = value;
                }
            m_referenceNorms.assign(b, m_operatorNorm);
            timed(m_phases.orthogonalisationSeconds, stream,
                  [&] { m_nextColumnCount = factoriseBlock(w, b, &triangle, store); });
            std::swap(m_ws.next, m_ws.product);
            std::fill(m_coupling.begin(), m_coupling.end(), 0.0);
            for (std::size_t c = 0; c < b; ++c)
                for (std::size_t r = 0; r < b; ++r)
                    m_coupling[r + (p + c) * b] = triangle[r + c * b];
            m_columns = p + b;
            ++result.blockSteps;

            timed(m_phases.projectedSeconds, stream, [&] { ritz = computeRitzPairs(); });
            if (hasConvergedTarget(ritz) || m_nextColumnCount == 0)
                break;
        }
        timed(m_phases.orthogonalisationSeconds, stream, [&] { extractConverged(ritz, shift, store, result); });
        return result;
    }

private:
    struct Ritz
    {
        std::vector<double> values;
        std::vector<double> vectors;
        std::vector<double> residuals;
        std::vector<unsigned char> isConverged;
        std::size_t accurateCount = 0;
    };

    // Op X = (K - sigma M)^-1 (M X).
    void applyOperator(double* block, std::size_t width)
    {
        const auto n = static_cast<std::int64_t>(m_n);
        double* mass = m_ws.massScratch.get();
        m_pencil.multiplyMass(block, n, mass, n, static_cast<std::int64_t>(width));
        m_ops.copy(block, n, mass, n, width);
        m_pencil.solve(block, n, static_cast<std::int64_t>(width));
    }

    // One pass of block classical Gram-Schmidt in the M inner product against the locked eigenvectors and the first
    // basisCount basis columns (MassOrthogonalizer::projectOut): W <- W - L (L^T M W) - Q (Q^T M W). coefficients
    // receives Q^T M W (basisCount x width); normsBefore the M-norms of W's columns before the pass.
    void projectOut(double* w, std::size_t width, const Store& store, std::size_t basisCount,
                    std::vector<double>* coefficients, double* normsBefore)
    {
        const auto n = static_cast<std::int64_t>(m_n);
        double* mw = m_ws.massScratch.get();
        m_pencil.multiplyMass(w, n, mw, n, static_cast<std::int64_t>(width));
        const std::size_t lockedCount = store.count();
        double* dLocked = m_values.reserve((lockedCount + basisCount + width) * width, "Lanczos: coefficients");
        double* dBasis = dLocked + lockedCount * width;
        double* dNorms = dBasis + basisCount * width;
        m_ops.gram(store.vectors(), n, lockedCount, mw, n, width, dLocked);
        m_ops.gram(m_ws.basis.get(), n, basisCount, mw, n, width, dBasis);
        if (normsBefore != nullptr)
            m_ops.gram(w, n, width, mw, n, width, dNorms);
        m_ops.subtract(w, n, width, store.vectors(), n, lockedCount, dLocked);
        m_ops.subtract(w, n, width, m_ws.basis.get(), n, basisCount, dBasis);
        if (coefficients != nullptr || normsBefore != nullptr)
        {
            m_host.resize((basisCount + width) * width);
            m_ops.download(dBasis, (basisCount + (normsBefore != nullptr ? width : 0)) * width, m_host.data());
            if (coefficients != nullptr)
                coefficients->assign(m_host.begin(), m_host.begin() + static_cast<std::ptrdiff_t>(basisCount * width));
            if (normsBefore != nullptr)
                for (std::size_t j = 0; j < width; ++j)
                    normsBefore[j] = std::sqrt(std::max(0.0, m_host[basisCount * width + j + j * width]));
        }
    }

    // Column c of the block against the columns before it, classical Gram-Schmidt twice (LanczosRun.cpp:127-150);
    // the coefficients are added to column c of the triangle when one is given.
    void subtractEarlierColumns(double* block, std::size_t c, std::size_t width, std::vector<double>* triangle)
    {
        if (c == 0)
            return;
        const auto n = static_cast<std::int64_t>(m_n);
        double* w = block + n * static_cast<std::int64_t>(c);
        const double* earlierMass = m_ws.massOfNext.get();
        double* d = m_columnValues.reserve(2 * c, "Lanczos: column coefficients");
        for (int pass = 0; pass < ORTHOGONALISATION_PASSES; ++pass)
        {
            double* coefficients = d + static_cast<std::size_t>(pass) * c;
            m_ops.gram(earlierMass, n, c, w, n, 1, coefficients);
            m_ops.subtract(w, n, 1, block, n, c, coefficients);
        }
        if (triangle != nullptr)
        {
            m_host.resize(2 * c);
            m_ops.download(d, 2 * c, m_host.data());
            for (int pass = 0; pass < ORTHOGONALISATION_PASSES; ++pass)
                for (std::size_t i = 0; i < c; ++i)
                    (*triangle)[i + c * width] += m_host[static_cast<std::size_t>(pass) * c + i];
        }
    }

    // M-normalises column c (its M-product in massOfNext) when its M-norm is above the threshold; returns the norm,
    // 0 for a deflated column.
    double normalise(double* block, std::size_t c, double threshold)
    {
        const auto n = static_cast<std::int64_t>(m_n);
        double* x = block + n * static_cast<std::int64_t>(c);
        double* mx = m_ws.massOfNext.get() + n * static_cast<std::int64_t>(c);
        m_pencil.multiplyMass(x, n, mx, n, 1);
        double* d = m_columnValues.reserve(1, "Lanczos: column coefficients");
        m_ops.gram(x, n, 1, mx, n, 1, d);
        double dot = 0.0;
        m_ops.download(d, 1, &dot);
        const double norm = std::sqrt(std::max(0.0, dot));
        if (!(norm > threshold))
            return 0.0;
        m_ops.scale(x, mx, 1.0 / norm);
        return norm;
    }

    // W = V_next B column by column (LanczosRun::factoriseBlock, LanczosRun.cpp:112-204); returns the columns filled.
    std::size_t factoriseBlock(double* block, std::size_t width, std::vector<double>* triangle, const Store& store)
    {
        const auto n = static_cast<std::int64_t>(m_n);
        const double rootDimension = std::sqrt(static_cast<double>(std::max<std::size_t>(m_n, 1)));
        if (triangle != nullptr)
            triangle->assign(width * width, 0.0);
        std::size_t filled = 0;
        for (std::size_t c = 0; c < width; ++c)
        {
            subtractEarlierColumns(block, c, width, triangle);
            const double norm = normalise(block, c, DEFLATION_FACTOR * EPSILON * rootDimension * m_referenceNorms[c]);
            if (norm > 0.0)
            {
                if (triangle != nullptr)
                    (*triangle)[c + c * width] = norm;
                ++filled;
                continue;
            }
            bool isReplaced = false;
            double* column = block + n * static_cast<std::int64_t>(c);
            for (std::size_t attempt = 0; attempt < REPLACEMENT_ATTEMPTS && !isReplaced; ++attempt)
            {
                m_ops.random(column, n, 1, m_randomState);
                applyOperator(column, 1);
                double referenceNorm = 0.0;
                for (int pass = 0; pass < ORTHOGONALISATION_PASSES; ++pass)
                    projectOut(column, 1, store, m_basisInUse, nullptr, pass == 0 ? &referenceNorm : nullptr);
                subtractEarlierColumns(block, c, width, nullptr);
                isReplaced = normalise(block, c, DEFLATION_FACTOR * EPSILON * rootDimension * referenceNorm) > 0.0;
            }
            if (!isReplaced)
            {
                m_ops.zero(column, n, 1);
                m_ops.zero(m_ws.massOfNext.get() + n * static_cast<std::int64_t>(c), n, 1);
            }
            else
            {
                ++filled;
            }
        }
        return filled;
    }

    void startBlock(const Store& store)
    {
        const auto n = static_cast<std::int64_t>(m_n);
        const std::size_t b = m_settings.blockSize;
        double* next = m_ws.next.get();
        const cudaStream_t stream = m_ops.stream();
        // Op applied once puts the block in the range of Op, which excludes the null space of M.
        timed(m_phases.operatorSeconds, stream,
              [&]
              {
                  if (m_settings.startBlock != nullptr)
                      m_ops.copy(next, n, m_settings.startBlock, m_settings.startLd, b);
                  else
                      m_ops.random(next, n, b, m_randomState);
                  applyOperator(next, b);
              });
        m_referenceNorms.assign(b, 0.0);
        m_basisInUse = 0;
        timed(m_phases.orthogonalisationSeconds, stream,
              [&]
              {
                  for (int pass = 0; pass < ORTHOGONALISATION_PASSES; ++pass)
                      projectOut(next, b, store, 0, nullptr, pass == 0 ? m_referenceNorms.data() : nullptr);
                  m_nextColumnCount = factoriseBlock(next, b, nullptr, store);
              });
    }

    // After a start block that deflated whole: P Op P R off the locked set; true when a direction is left, with the
    // Rayleigh estimates of the roots left (LanczosRun::probeBeyondLocked, LanczosRun.cpp:225-289).
    bool probeBeyondLocked(double shift, const Store& store, RunResult& result)
    {
        if (store.count() == 0)
            return false;
        const auto n = static_cast<std::int64_t>(m_n);
        const std::vector<double> startNorms = m_referenceNorms;
        double* probe = m_ws.next.get();
        const std::size_t width = m_settings.blockSize;
        m_ops.random(probe, n, width, m_randomState);
        for (int pass = 0; pass < ORTHOGONALISATION_PASSES; ++pass)
            projectOut(probe, width, store, 0, nullptr, nullptr);
        applyOperator(probe, width);
        for (int pass = 0; pass < ORTHOGONALISATION_PASSES; ++pass)
            projectOut(probe, width, store, 0, nullptr, nullptr);
        double* massOfProbe = m_ws.massOfNext.get();
        const double rounding = DEFLATION_FACTOR * EPSILON * std::sqrt(static_cast<double>(std::max<std::size_t>(m_n, 1)));
        std::vector<unsigned char> isDirection(width, 0);
        bool hasDirection = false;
        double* d = m_columnValues.reserve(1, "Lanczos: column coefficients");
        for (std::size_t c = 0; c < width && c < startNorms.size(); ++c)
        {
            double* x = probe + n * static_cast<std::int64_t>(c);
            double* mx = massOfProbe + n * static_cast<std::int64_t>(c);
            m_pencil.multiplyMass(x, n, mx, n, 1);
            m_ops.gram(x, n, 1, mx, n, 1, d);
            double dot = 0.0;
            m_ops.download(d, 1, &dot);
            const double norm = std::sqrt(std::max(0.0, dot));
            if (!(startNorms[c] > 0.0) || !(norm > rounding * rounding * startNorms[c]))
                continue;
            m_ops.scale(x, mx, 1.0 / norm);
            isDirection[c] = 1;
            hasDirection = true;
        }
        if (!hasDirection)
            return false;
        double* image = m_ws.product.get();
        m_ops.copy(image, n, probe, n, width);
        applyOperator(image, width);
        for (std::size_t c = 0; c < width; ++c)
        {
            if (isDirection[c] == 0)
                continue;
            m_ops.gram(massOfProbe + n * static_cast<std::int64_t>(c), n, 1, image + n * static_cast<std::int64_t>(c),
                       n, 1, d);
            double theta = 0.0;
            m_ops.download(d, 1, &theta);
            const double estimate = shift + 1.0 / theta;
            if (theta != 0.0 && std::isfinite(estimate))
                result.ritzEstimates.push_back(estimate);
        }
        std::sort(result.ritzEstimates.begin(), result.ritzEstimates.end());
        return true;
    }

    Ritz computeRitzPairs() const
    {
        const std::size_t p = m_columns;
        const std::size_t b = m_settings.blockSize;
        const std::size_t ld = m_settings.basisColumns;
        std::vector<double> values;
        std::vector<double> vectors;
        decomposeSymmetric(m_projected.data(), p, std::max<std::size_t>(ld, 1), values, vectors);
        std::vector<std::size_t> order(p);
        std::iota(order.begin(), order.end(), std::size_t{0});
        std::stable_sort(order.begin(), order.end(),
                         [&](std::size_t x, std::size_t y) { return std::abs(values[x]) > std::abs(values[y]); });
        Ritz ritz;
        ritz.values.resize(p);
        ritz.vectors.resize(p * p);
        ritz.residuals.resize(p);
        ritz.isConverged.assign(p, 0);
        const double largest = p > 0 ? std::abs(values[order[0]]) : 0.0;
        for (std::size_t k = 0; k < p; ++k)
        {
            const std::size_t from = order[k];
            ritz.values[k] = values[from];
            std::copy_n(vectors.data() + from * p, p, ritz.vectors.data() + k * p);
            double squares = 0.0;
            for (std::size_t r = 0; r < b; ++r)
            {
                double value = 0.0;
                for (std::size_t i = 0; i < p; ++i)
                    value += m_coupling[r + i * b] * ritz.vectors[i + k * p];
                squares += value * value;
            }
            ritz.residuals[k] = std::sqrt(squares);
            const double theta = std::abs(ritz.values[k]);
            const bool isAccurate = theta > 0.0 && theta >= ACCURATE_RITZ_RATIO * largest;
            ritz.accurateCount += isAccurate ? 1 : 0;
            ritz.isConverged[k] = isAccurate && ritz.residuals[k] <= m_settings.convergenceTolerance * theta ? 1 : 0;
        }
        return ritz;
    }

    bool hasConvergedTarget(const Ritz& ritz) const
    {
        if (ritz.values.size() < m_settings.target)
            return false;
        const std::size_t wanted = std::min(m_settings.target, ritz.accurateCount);
        if (wanted == 0)
            return false;
        for (std::size_t k = 0; k < wanted; ++k)
            if (ritz.isConverged[k] == 0)
                return false;
        return true;
    }

    // Thick restart (LanczosRun::restart, LanczosRun.cpp:346-378): the basis becomes V S_k, T diag(theta_k), G G S_k.
    void restart(const Ritz& ritz)
    {
        const std::size_t p = m_columns;
        const std::size_t b = m_settings.blockSize;
        const std::size_t ld = m_settings.basisColumns;
        const std::size_t room = m_capacity - 2 * b;
        const std::size_t kept = std::min({room, p - b, std::max(m_capacity / 2, std::min(m_settings.target + b, room))});
        const auto n = static_cast<std::int64_t>(m_n);
        m_ops.upload(m_ws.small.get(), ritz.vectors.data(), p * kept);
        m_ops.combine(m_ws.basis.get(), n, p, m_ws.small.get(), static_cast<std::int64_t>(p), kept, m_ws.basis.get(),
                      n, nullptr, 0, 0, nullptr);
        std::vector<double> coupling(b * kept, 0.0);
        for (std::size_t k = 0; k < kept; ++k)
            for (std::size_t r = 0; r < b; ++r)
            {
                double value = 0.0;
                for (std::size_t i = 0; i < p; ++i)
                    value += m_coupling[r + i * b] * ritz.vectors[i + k * p];
                coupling[r + k * b] = value;
            }
        std::fill(m_coupling.begin(), m_coupling.end(), 0.0);
        std::copy(coupling.begin(), coupling.end(), m_coupling.begin());
        std::fill(m_projected.begin(), m_projected.end(), 0.0);
        for (std::size_t k = 0; k < kept; ++k)
            m_projected[k + k * ld] = ritz.values[k];
        m_columns = kept;
        // The upload's host buffer must outlive the copy: the product is ordered after it on the stream.
        check(cudaStreamSynchronize(m_ops.stream()), "Lanczos: restart");
    }

    // The converged pairs, purified and M-normalised, into the store (LanczosRun::extractConverged,
    // LanczosRun.cpp:380-445); the other Ritz values give estimates sigma + 1/theta.
    void extractConverged(const Ritz& ritz, double shift, Store& store, RunResult& result)
    {
        const std::size_t p = m_columns;
        const std::size_t b = m_settings.blockSize;
        std::vector<std::size_t> converged;
        const double largest = ritz.values.empty() ? 0.0 : std::abs(ritz.values[0]);
        for (std::size_t k = 0; k < ritz.values.size(); ++k)
        {
            if (ritz.isConverged[k] != 0)
                converged.push_back(k);
            else if (std::abs(ritz.values[k]) > NEGLIGIBLE_RITZ_VALUE * largest)
                result.ritzEstimates.push_back(shift + 1.0 / ritz.values[k]);
        }
        std::sort(result.ritzEstimates.begin(), result.ritzEstimates.end());
        const std::size_t count = converged.size();
        result.convergedCount = count;
        if (count == 0)
            return;
        std::vector<double> selected(p * count);
        std::vector<double> negatedCorrection(b * count, 0.0);
        std::vector<double> values(count);
        std::vector<double> bounds(count);
        for (std::size_t j = 0; j < count; ++j)
        {
            const std::size_t k = converged[j];
            std::copy_n(ritz.vectors.data() + k * p, p, selected.data() + j * p);
            const double theta = ritz.values[k];
            for (std::size_t r = 0; r < b; ++r)
            {
                double value = 0.0;
                for (std::size_t i = 0; i < p; ++i)
                    value += m_coupling[r + i * b] * ritz.vectors[i + k * p];
                negatedCorrection[r + j * b] = -value / theta;
            }
            values[j] = shift + 1.0 / theta;
            bounds[j] = ritz.residuals[k] / std::abs(theta);
        }
        const auto n = static_cast<std::int64_t>(m_n);
        double* out = store.prepareColumns(count);
        double* dSelected = m_selected.reserve(p * count + b * count + count, "Lanczos: converged Ritz vectors");
        double* dCorrection = dSelected + p * count;
        double* dInverse = dCorrection + b * count;
        m_ops.upload(dSelected, selected.data(), p * count);
        m_ops.upload(dCorrection, negatedCorrection.data(), b * count);
        m_ops.combine(m_ws.basis.get(), n, p, dSelected, static_cast<std::int64_t>(p), count, out, n, m_ws.next.get(),
                      n, b, dCorrection);
        double* mass = m_ws.massScratch.get();
        double* dDots = m_values.reserve(b * b, "Lanczos: coefficients");
        std::vector<double> dots(b * b);
        std::vector<double> inverse(count, 0.0);
        for (std::size_t first = 0; first < count; first += b)
        {
            const std::size_t width = std::min(b, count - first);
            double* columns = out + n * static_cast<std::int64_t>(first);
            m_pencil.multiplyMass(columns, n, mass, n, static_cast<std::int64_t>(width));
            m_ops.gram(columns, n, width, mass, n, width, dDots);
            m_ops.download(dDots, width * width, dots.data());
            for (std::size_t j = 0; j < width; ++j)
            {
                const double norm = std::sqrt(std::max(0.0, dots[j + j * width]));
                inverse[first + j] = norm > 0.0 ? 1.0 / norm : 0.0;
            }
        }
        m_ops.upload(dInverse, inverse.data(), count);
        m_ops.scaleColumns(out, n, dInverse, count);
        check(cudaStreamSynchronize(m_ops.stream()), "Lanczos: converged vectors");
        store.commit(values, bounds);
    }

    ShiftedPencil& m_pencil;
    BlockOps& m_ops;
    Workspace& m_ws;
    RunSettings m_settings;
    Phases& m_phases;
    std::size_t m_n;
    std::size_t m_capacity;
    std::vector<double> m_projected;
    std::vector<double> m_coupling;
    std::vector<double> m_referenceNorms;
    std::vector<double> m_host;
    std::size_t m_columns = 0;
    std::size_t m_basisInUse = 0;
    std::size_t m_nextColumnCount = 0;
    double m_operatorNorm = 0.0;
    std::uint64_t m_randomState = 0;
    Scratch m_values;
    Scratch m_columnValues;
    Scratch m_selected;
};

std::string text(double value)
{
    return std::to_string(value);
}

void requireNoExtraEigenvalue(const SturmVerification& verification)
{
    if (verification.hasMismatch && verification.mismatch.foundCount > verification.mismatch.expectedCount)
        throw Error(STATUS_SOLVER,
                    "eigenvalue analysis: " + std::to_string(verification.mismatch.foundCount) +
                        " eigenvalues found in [" + text(verification.mismatch.lower) + ", " +
                        text(verification.mismatch.upper) + ") where the Sturm counts allow " +
                        std::to_string(verification.mismatch.expectedCount) +
                        "; the factorisations are not reliable there (an eigenvalue on a bound of the range, or a "
                        "pencil close to singular): move the bounds of the range or check the model for massless "
                        "mechanisms");
}

void requireNoEigenvalueBelow(double lowestPoint, std::span<const double> sortedEigenvalues)
{
    if (sortedEigenvalues.empty() || !(sortedEigenvalues.front() < lowestPoint))
        return;
    throw Error(STATUS_SOLVER, "eigenvalue analysis: the eigenvalue " + text(sortedEigenvalues.front()) +
                                   " was found below the shift " + text(lowestPoint) +
                                   ", where the Sturm count says no eigenvalue lies; the factorisation there is not "
                                   "reliable (a pencil close to singular, or a mass matrix that is not positive "
                                   "semi-definite): check the model for massless mechanisms and negative masses");
}

} // namespace

// ---- SturmCheck --------------------------------------------------------------------------------------------------

void SturmCheck::addPoint(SturmPoint point)
{
    const auto at = std::lower_bound(m_points.begin(), m_points.end(), point.shift,
                                     [](const SturmPoint& p, double shift) { return p.shift < shift; });
    const bool isSameShift = at != m_points.end() && at->shift == point.shift;
    const bool isBelowNext =
        at == m_points.end() || (isSameShift ? at->countBelow == point.countBelow : at->countBelow >= point.countBelow);
    const bool isAbovePrevious = at == m_points.begin() || std::prev(at)->countBelow <= point.countBelow;
    if (!isBelowNext || !isAbovePrevious)
    {
        const SturmPoint& other = !isBelowNext ? *at : *std::prev(at);
        const auto describe = [](const SturmPoint& p)
        { return "shift " + text(p.shift) + " (" + std::to_string(p.countBelow) + " eigenvalues below)"; };
        throw Error(STATUS_SOLVER, "eigenvalue analysis: the Sturm counts contradict each other: " + describe(point) +
                                       " against " + describe(other) +
                                       "; the factorisations of K - sigma*M are not reliable (a nearly singular "
                                       "pencil, or a mass matrix that is not positive semi-definite): check the model "
                                       "for mechanisms without mass and negative masses");
    }
    if (!isSameShift)
        m_points.insert(at, point);
}

std::size_t SturmCheck::countBelow(double shift) const
{
    for (const SturmPoint& point : m_points)
        if (point.shift == shift)
            return point.countBelow;
    throw Error(STATUS_INVALID_ARGUMENT, "SturmCheck::countBelow: no Sturm point at the shift " + text(shift));
}

SturmVerification SturmCheck::verify(std::span<const double> sortedEigenvalues) const
{
    if (m_points.empty())
        throw Error(STATUS_INVALID_ARGUMENT, "SturmCheck::verify: no Sturm point; factorise at a shift first");
    SturmVerification result;
    result.verifiedUpTo = m_points.front().shift;
    auto next = std::lower_bound(sortedEigenvalues.begin(), sortedEigenvalues.end(), m_points.front().shift);
    for (std::size_t k = 0; k + 1 < m_points.size(); ++k)
    {
        const SturmPoint& lower = m_points[k];
        const SturmPoint& upper = m_points[k + 1];
        const auto end = std::lower_bound(next, sortedEigenvalues.end(), upper.shift);
        const auto found = static_cast<std::size_t>(end - next);
        const std::size_t expected = upper.countBelow - lower.countBelow;
        if (found != expected)
        {
            result.hasMismatch = true;
            result.mismatch = {lower.shift, upper.shift, expected, found};
            return result;
        }
        result.verifiedUpTo = upper.shift;
        result.verifiedCount += found;
        next = end;
    }
    return result;
}

// ---- ShiftStrategy -----------------------------------------------------------------------------------------------

ShiftStrategy::ShiftStrategy(const EigenRequest& request, double scale) : m_request(request)
{
    if (request.modeCount == 0 && !request.hasUpperBound())
        throw Error(STATUS_INVALID_ARGUMENT, "eigenvalue request: neither a mode count nor an upper bound; give a mode "
                                             "count, or an upper bound to bound the range");
    if (request.hasUpperBound() && !request.startsFromLowest() && !(request.upperBound > request.lowerBound))
        throw Error(STATUS_INVALID_ARGUMENT, "eigenvalue request: the upper bound " + text(request.upperBound) +
                                                 " must be above the lower bound " + text(request.lowerBound) +
                                                 "; check that the lower bound is below the upper bound");
    if (request.hasUpperBound() && request.startsFromLowest() && !(request.upperBound > 0.0))
        throw Error(STATUS_INVALID_ARGUMENT, "eigenvalue request: the upper bound " + text(request.upperBound) +
                                                 " must be above 0; check the upper bound");
    m_scale = std::isfinite(scale) && scale > 0.0 ? scale : 1.0;
}

ShiftChoice ShiftStrategy::firstShift() const noexcept
{
    if (m_request.startsFromLowest())
        return {-RIGID_SHIFT_FRACTION * m_scale, ShiftPurpose::LowestBound};
    return {m_request.lowerBound, ShiftPurpose::LowerBound};
}

double ShiftStrategy::descend(double shift) const noexcept
{
    return shift < 0.0 ? shift * DESCENT_FACTOR : -RIGID_SHIFT_FRACTION * m_scale;
}

double ShiftStrategy::moveOffEigenvalue(double shift, bool isUpward, std::size_t attempt) const noexcept
{
    const double step =
        SINGULAR_SHIFT_MOVE * static_cast<double>(attempt) * std::max(std::abs(shift), RIGID_SHIFT_FRACTION * m_scale);
    return isUpward ? shift + step : shift - step;
}

bool ShiftStrategy::isComplete(const SturmVerification& verification) const noexcept
{
    if (m_request.modeCount > 0 && verification.verifiedCount >= m_request.modeCount)
        return true;
    return m_request.hasUpperBound() && verification.verifiedUpTo >= m_request.upperBound;
}

ShiftStrategy::Selection ShiftStrategy::select(std::span<const double> sortedEigenvalues, double lowerPoint,
                                               double upperPoint) const noexcept
{
    const auto first = std::lower_bound(sortedEigenvalues.begin(), sortedEigenvalues.end(), lowerPoint);
    const auto end = std::lower_bound(first, sortedEigenvalues.end(), upperPoint);
    Selection selection;
    selection.first = static_cast<std::size_t>(first - sortedEigenvalues.begin());
    selection.count = static_cast<std::size_t>(end - first);
    if (m_request.modeCount > 0)
        selection.count = std::min(selection.count, m_request.modeCount);
    return selection;
}

double ShiftStrategy::clearanceAt(double value, double shift) const noexcept
{
    return SHIFT_CLEARANCE * std::max({std::abs(value), std::abs(shift), RIGID_SHIFT_FRACTION * m_scale});
}

double ShiftStrategy::clear(double shift, std::span<const double> sortedEigenvalues) const noexcept
{
    for (std::size_t pass = 0; pass < MAX_CLEARANCE_PASSES; ++pass)
    {
        bool isClear = true;
        for (const double value : sortedEigenvalues)
        {
            if (std::abs(shift - value) < clearanceAt(value, shift))
            {
                shift = value + clearanceAt(value, shift);
                isClear = false;
            }
        }
        if (isClear)
            break;
    }
    return shift;
}

bool ShiftStrategy::isNearShift(double shift, std::span<const double> lanczosShifts) const noexcept
{
    return std::any_of(lanczosShifts.begin(), lanczosShifts.end(),
                       [&](double used)
                       {
                           return std::abs(shift - used) <=
                                  SAME_SHIFT_TOLERANCE *
                                      std::max({std::abs(used), std::abs(shift), RIGID_SHIFT_FRACTION * m_scale});
                       });
}

ShiftChoice ShiftStrategy::nextShift(const SturmVerification& verification, std::span<const double> sortedEigenvalues,
                                     std::span<const double> ritzEstimates, std::span<const double> lanczosShifts) const
{
    const double a = verification.verifiedUpTo;
    const double b = verification.hasMismatch ? verification.mismatch.upper : INFINITE;
    const ShiftPurpose purpose = verification.hasMismatch ? ShiftPurpose::FillGap : ShiftPurpose::Advance;
    const auto firstFound = std::lower_bound(sortedEigenvalues.begin(), sortedEigenvalues.end(), a);
    const auto endFound = std::lower_bound(firstFound, sortedEigenvalues.end(), b);
    const auto ritzAbove = [&](double value)
    {
        const auto at = std::upper_bound(ritzEstimates.begin(), ritzEstimates.end(), value);
        return at != ritzEstimates.end() && *at < b ? *at : INFINITE;
    };
    // A mismatch: an unconverged Ritz estimate inside the interval points at a missing root.
    if (verification.hasMismatch)
        for (const double estimate : ritzEstimates)
            if (estimate > a && estimate < b && !isNearShift(estimate, lanczosShifts))
                return {clear(estimate, sortedEigenvalues), purpose};
    double shift = 0.0;
    if (firstFound != endFound)
    {
        const double highest = *(endFound - 1);
        const double estimate = ritzAbove(highest + clearanceAt(highest, highest));
        if (estimate < INFINITE)
            shift = 0.5 * (highest + estimate);
        else
        {
            const double extent = std::max(highest - a, RIGID_SHIFT_FRACTION * m_scale);
            shift = highest + STEP_FRACTION * extent;
            if (b < INFINITE)
                shift = std::min(shift, 0.5 * (highest + b));
        }
    }
    else
    {
        const double estimate = ritzAbove(a);
        if (estimate < INFINITE)
            shift = estimate;
        else
            shift = b < INFINITE ? 0.5 * (a + b) : a + std::max(std::abs(a), m_scale);
    }
    if (isNearShift(shift, lanczosShifts))
    {
        // The widest gap between the ends of the interval and the eigenvalues found in it.
        std::vector<double> ends;
        ends.push_back(a);
        ends.insert(ends.end(), firstFound, endFound);
        const double top = ends.back();
        ends.push_back(b < INFINITE ? b : top + std::max(top - a, m_scale));
        std::size_t widest = 0;
        for (std::size_t k = 1; k + 1 < ends.size(); ++k)
            if (ends[k + 1] - ends[k] > ends[widest + 1] - ends[widest])
                widest = k;
        shift = 0.5 * (ends[widest] + ends[widest + 1]);
        if (isNearShift(shift, lanczosShifts))
            shift = ends[widest] + 0.25 * (ends[widest + 1] - ends[widest]);
    }
    return {clear(shift, sortedEigenvalues), purpose};
}

// ---- the projected problem ---------------------------------------------------------------------------------------

void decomposeSymmetric(const double* a, std::size_t p, std::size_t ld, std::vector<double>& values,
                        std::vector<double>& vectors)
{
    values.assign(p, 0.0);
    vectors.assign(p * p, 0.0);
    if (p == 0)
        return;
    std::vector<double> m(p * p);
    for (std::size_t j = 0; j < p; ++j)
        for (std::size_t i = j; i < p; ++i)
        {
            if (!std::isfinite(a[i + j * ld]))
                throw Error(STATUS_SOLVER, "symmetric eigenproblem: the term (" + std::to_string(i) + ", " +
                                               std::to_string(j) + ") of the matrix is not finite");
            m[i + j * p] = a[i + j * ld];
            m[j + i * p] = a[i + j * ld];
        }
    std::vector<double>& z = vectors;
    for (std::size_t i = 0; i < p; ++i)
        z[i + i * p] = 1.0;
    // Householder reduction: step k zeroes rows k+2.. of column k with H = I - beta v v^T on rows and columns k+1..;
    // the trailing block becomes H B H = B - v w^T - w v^T (u = beta B v, w = u - (beta/2)(v^T u) v), and Z <- Z H.
    std::vector<double> v(p);
    std::vector<double> u(p);
    for (std::size_t k = 0; k + 2 < p; ++k)
    {
        double scale = 0.0;
        for (std::size_t i = k + 1; i < p; ++i)
            scale = std::max(scale, std::abs(m[i + k * p]));
        if (scale == 0.0)
            continue;
        double sigma = 0.0;
        for (std::size_t i = k + 1; i < p; ++i)
        {
            v[i] = m[i + k * p] / scale;
            sigma += v[i] * v[i];
        }
        double alpha = std::sqrt(sigma);
        if (v[k + 1] > 0.0)
            alpha = -alpha;
        v[k + 1] -= alpha;
        double vv = 0.0;
        for (std::size_t i = k + 1; i < p; ++i)
            vv += v[i] * v[i];
        if (vv == 0.0)
            continue;
        const double beta = 2.0 / vv;
        double vu = 0.0;
        for (std::size_t i = k + 1; i < p; ++i)
        {
            double sum = 0.0;
            for (std::size_t j = k + 1; j < p; ++j)
                sum += m[i + j * p] * v[j];
            u[i] = beta * sum;
            vu += v[i] * u[i];
        }
        const double half = 0.5 * beta * vu;
        for (std::size_t i = k + 1; i < p; ++i)
            u[i] -= half * v[i];
        for (std::size_t j = k + 1; j < p; ++j)
            for (std::size_t i = k + 1; i < p; ++i)
                m[i + j * p] -= v[i] * u[j] + u[i] * v[j];
        m[(k + 1) + k * p] = alpha * scale;
        m[k + (k + 1) * p] = alpha * scale;
        for (std::size_t i = k + 2; i < p; ++i)
        {
            m[i + k * p] = 0.0;
            m[k + i * p] = 0.0;
        }
        for (std::size_t r = 0; r < p; ++r)
        {
            double sum = 0.0;
            for (std::size_t i = k + 1; i < p; ++i)
                sum += z[r + i * p] * v[i];
            sum *= beta;
            for (std::size_t i = k + 1; i < p; ++i)
                z[r + i * p] -= sum * v[i];
        }
    }
    std::vector<double>& d = values;
    std::vector<double> e(p, 0.0); // e[i] couples i and i + 1
    for (std::size_t i = 0; i < p; ++i)
    {
        d[i] = m[i + i * p];
        if (i + 1 < p)
            e[i] = m[(i + 1) + i * p];
    }
    // Implicit QL with Wilkinson's shift: a chase of plane rotations from the bottom of the unreduced block [l, mm].
    for (std::size_t l = 0; l < p; ++l)
    {
        int sweeps = 0;
        while (true)
        {
            std::size_t mm = l;
            for (; mm + 1 < p; ++mm)
            {
                const double dd = std::abs(d[mm]) + std::abs(d[mm + 1]);
                if (std::abs(e[mm]) <= EPSILON * dd)
                    break;
            }
            if (mm == l)
                break;
            if (++sweeps > MAX_QL_SWEEPS)
                throw Error(STATUS_SOLVER, "eigenvalue analysis: the projected eigenproblem did not converge in " +
                                               std::to_string(MAX_QL_SWEEPS) + " QL sweeps");
            double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
            double r = hypotenuse(g, 1.0);
            g = d[mm] - d[l] + e[l] / (g + (g >= 0.0 ? r : -r));
            double s = 1.0;
            double c = 1.0;
            double shiftSum = 0.0;
            bool isSplit = false;
            for (std::size_t i = mm; i-- > l;)
            {
                const double f = s * e[i];
                const double bb = c * e[i];
                r = hypotenuse(f, g);
                e[i + 1] = r;
                if (r == 0.0)
                {
                    d[i + 1] -= shiftSum;
                    e[mm] = 0.0;
                    isSplit = true;
                    break;
                }
                s = f / r;
                c = g / r;
                g = d[i + 1] - shiftSum;
                r = (d[i] - g) * s + 2.0 * c * bb;
                shiftSum = s * r;
                d[i + 1] = g + shiftSum;
                g = c * r - bb;
                for (std::size_t k = 0; k < p; ++k)
                {
                    const double zf = z[k + (i + 1) * p];
                    z[k + (i + 1) * p] = s * z[k + i * p] + c * zf;
                    z[k + i * p] = c * z[k + i * p] - s * zf;
                }
            }
            if (isSplit)
                continue;
            d[l] -= shiftSum;
            e[l] = g;
            e[mm] = 0.0;
        }
    }
    // Increasing order (the first minimum each time), each vector signed by its largest component.
    for (std::size_t i = 0; i + 1 < p; ++i)
    {
        std::size_t k = i;
        for (std::size_t j = i + 1; j < p; ++j)
            if (d[j] < d[k])
                k = j;
        if (k != i)
        {
            std::swap(d[i], d[k]);
            for (std::size_t r = 0; r < p; ++r)
                std::swap(z[r + i * p], z[r + k * p]);
        }
    }
    for (std::size_t j = 0; j < p; ++j)
    {
        std::size_t largest = 0;
        for (std::size_t r = 1; r < p; ++r)
            if (std::abs(z[r + j * p]) > std::abs(z[largest + j * p]))
                largest = r;
        if (z[largest + j * p] < 0.0)
            for (std::size_t r = 0; r < p; ++r)
                z[r + j * p] = -z[r + j * p];
    }
}

// ---- BlockLanczos --------------------------------------------------------------------------------------------------

void validate(const LanczosOptions& options)
{
    if (options.blockSize == 0 || options.modesPerShift == 0)
        throw Error(STATUS_INVALID_ARGUMENT, "BlockLanczos: the block size (" + std::to_string(options.blockSize) +
                                                 ") and the modes per shift (" +
                                                 std::to_string(options.modesPerShift) + ") must be at least 1");
    if (!(options.convergenceTolerance > 0.0 && options.convergenceTolerance <= MAXIMUM_CONVERGENCE_TOLERANCE))
        throw Error(STATUS_INVALID_ARGUMENT, "BlockLanczos: the convergence tolerance must be in (0, 1e-2], found " +
                                                 text(options.convergenceTolerance));
    if (options.maximumShifts == 0 || options.maximumRestarts == 0)
        throw Error(STATUS_INVALID_ARGUMENT, "BlockLanczos: at least one shift and one restart must be allowed");
}

BasisShape shapeFor(const LanczosOptions& options, std::size_t dimension, const EigenRequest& request) noexcept
{
    BasisShape shape;
    if (dimension == 0)
        return shape;
    shape.blockSize = std::max<std::size_t>(1, std::min(options.blockSize, dimension / 3));
    shape.modesPerShift =
        request.modeCount > 0 ? std::min(options.modesPerShift, request.modeCount) : options.modesPerShift;
    const std::size_t wanted = roundUp(2 * shape.modesPerShift + 3 * shape.blockSize, shape.blockSize);
    const std::size_t room = std::max(dimension / shape.blockSize * shape.blockSize, std::min<std::size_t>(dimension, 3));
    shape.basisColumns = std::min(wanted, room);
    return shape;
}

EigenSolution solveModes(ShiftedPencil& pencil, const EigenRequest& request, const LanczosOptions& options,
                         const double* startBlock, std::int64_t startLd)
{
    validate(options);
    const auto started = std::chrono::steady_clock::now();
    const ShiftStrategy strategy(request, pencil.diagonalRayleighBound());
    const auto dimension = static_cast<std::size_t>(pencil.dimension());
    EigenSolution solution;
    solution.dimension = static_cast<std::int64_t>(dimension);
    if (dimension == 0)
    {
        solution.isComplete = true;
        return solution;
    }
    const BasisShape shape = shapeFor(options, dimension, request);
    BlockOps ops(pencil.stream(), static_cast<int>(dimension));
    auto workspace = std::make_unique<Workspace>(dimension, shape.basisColumns, shape.blockSize);
    Store store(pencil.stream(), dimension,
                (request.modeCount > 0 ? std::min(request.modeCount, dimension) : 0) + shape.basisColumns);

    SturmCheck sturm;
    Phases phases;
    const auto factoriseAt = [&](double shift, ShiftPurpose purpose, bool isUpward)
    {
        double trial = shift;
        for (std::size_t attempt = 0; attempt <= MAX_SINGULAR_MOVES; ++attempt)
        {
            Inertia inertia;
            bool refused = false;
            try
            {
                timed(solution.factorWallSeconds, pencil.stream(), [&] { inertia = pencil.factorise(trial); });
            }
            catch (const DelayedPivotError&)
            {
                // a front of K - sigma M too near singular for a pivot within it: moved off like a singular shift
                refused = true;
            }
            ++solution.factorisationCount;
            solution.factorSeconds += refused ? 0.0 : pencil.lastFactorSeconds();
            if (!refused && inertia.zero == 0)
            {
                sturm.addPoint({trial, static_cast<std::size_t>(inertia.negative)});
                ShiftRecord record;
                record.shift = trial;
                record.purpose = purpose;
                record.sturmCount = static_cast<std::size_t>(inertia.negative);
                solution.shifts.push_back(record);
                return trial;
            }
            trial = strategy.moveOffEigenvalue(shift, isUpward, attempt + 1);
        }
        throw Error(STATUS_SOLVER, "eigenvalue analysis: K - sigma*M is singular at " +
                                       std::to_string(MAX_SINGULAR_MOVES + 1) + " shifts around " + text(shift) +
                                       ": a degree of freedom has neither mass nor stiffness (a massless mechanism); "
                                       "constrain it (single-point constraints) or give it a mass");
    };

    double lowerPoint = -INFINITE;
    double upperPoint = INFINITE;
    if (request.hasUpperBound())
        upperPoint = factoriseAt(request.upperBound, ShiftPurpose::UpperBound, true);
    double current = 0.0;
    if (request.startsFromLowest())
    {
        current = factoriseAt(strategy.firstShift().shift, ShiftPurpose::LowestBound, false);
        for (std::size_t descents = 0; sturm.countBelow(current) > 0; ++descents)
        {
            if (descents == ShiftStrategy::MAX_DESCENTS)
                throw Error(STATUS_SOLVER, "eigenvalue analysis: " + std::to_string(sturm.countBelow(current)) +
                                               " eigenvalues lie below the shift " + text(current) +
                                               "; the stiffness has unbounded negative roots: check the model for "
                                               "negative stiffness or a mass matrix that is not positive "
                                               "semi-definite");
            current = factoriseAt(strategy.descend(current), ShiftPurpose::LowestBound, false);
        }
    }
    else
    {
        current = factoriseAt(request.lowerBound, ShiftPurpose::LowerBound, false);
        lowerPoint = current;
    }
    const std::size_t lowestCount = sturm.countBelow(current);
    std::size_t wanted = request.modeCount;
    if (request.hasUpperBound())
    {
        const std::size_t inRange = sturm.countBelow(upperPoint) - lowestCount;
        wanted = wanted > 0 ? std::min(wanted, inRange) : inRange;
    }

    std::vector<double> lanczosShifts;
    std::vector<double> sorted;
    SturmVerification verification = sturm.verify(sorted);
    bool isComplete = wanted == 0;
    for (std::size_t runIndex = 0; !isComplete; ++runIndex)
    {
        const auto inRequest = static_cast<std::size_t>(std::lower_bound(sorted.begin(), sorted.end(), upperPoint) -
                                                        std::lower_bound(sorted.begin(), sorted.end(), lowerPoint));
        const std::size_t remaining = wanted > inRequest ? wanted - inRequest : 0;
        RunSettings settings;
        settings.blockSize = shape.blockSize;
        settings.basisColumns = shape.basisColumns;
        settings.target = std::min(shape.modesPerShift, std::max(remaining, shape.blockSize));
        settings.convergenceTolerance = options.convergenceTolerance;
        settings.maximumRestarts = options.maximumRestarts;
        settings.seed = options.seed + SEED_STEP * (runIndex + 1);
        if (runIndex == 0)
        {
            settings.startBlock = startBlock;
            settings.startLd = startLd;
        }
        Run run(pencil, ops, *workspace, settings, phases);
        const RunResult result = run.run(current, store);
        solution.blockSteps += result.blockSteps;
        for (auto record = solution.shifts.rbegin(); record != solution.shifts.rend(); ++record)
            if (record->shift == current)
            {
                record->hasLanczosRun = true;
                record->blockSteps = result.blockSteps;
                record->restarts = result.restarts;
                record->convergedCount = result.convergedCount;
                break;
            }
        lanczosShifts.push_back(current);

        sorted = store.eigenvalues();
        std::sort(sorted.begin(), sorted.end());
        verification = sturm.verify(sorted);
        requireNoExtraEigenvalue(verification);
        if (request.startsFromLowest())
            requireNoEigenvalueBelow(sturm.points().front().shift, sorted);
        if (strategy.isComplete(verification) || (result.isSpaceExhausted && !verification.hasMismatch))
        {
            isComplete = true;
            break;
        }
        if (solution.shifts.size() >= options.maximumShifts)
            break;
        const ShiftChoice next = strategy.nextShift(verification, sorted, result.ritzEstimates, lanczosShifts);
        current = factoriseAt(next.shift, next.purpose, true);
        verification = sturm.verify(sorted);
        requireNoExtraEigenvalue(verification);
        isComplete = strategy.isComplete(verification);
    }

    workspace.reset();
    const std::vector<double>& values = store.eigenvalues();
    std::vector<std::size_t> order(values.size());
    std::iota(order.begin(), order.end(), std::size_t{0});
    std::stable_sort(order.begin(), order.end(), [&](std::size_t x, std::size_t y) { return values[x] < values[y]; });
    const ShiftStrategy::Selection selection = strategy.select(sorted, lowerPoint, upperPoint);
    solution.eigenvectors = deviceValues(dimension * std::max<std::size_t>(selection.count, 1), "Lanczos: eigenvectors");
    for (std::size_t k = 0; k < selection.count; ++k)
    {
        const std::size_t from = order[selection.first + k];
        solution.eigenvalues.push_back(values[from]);
        solution.residualBounds.push_back(store.residualBounds()[from]);
        check(cudaMemcpyAsync(solution.eigenvectors.get() + dimension * k, store.vectors() + dimension * from,
                              dimension * sizeof(double), cudaMemcpyDeviceToDevice, pencil.stream()),
              "Lanczos: eigenvectors");
    }
    check(cudaStreamSynchronize(pencil.stream()), "Lanczos: eigenvectors");
    solution.isComplete = isComplete;
    solution.verifiedCount = static_cast<std::size_t>(
        std::count_if(solution.eigenvalues.begin(), solution.eigenvalues.end(),
                      [&](double value) { return isComplete || value < verification.verifiedUpTo; }));
    solution.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - started).count();
    solution.operatorSeconds = phases.operatorSeconds;
    solution.orthogonalisationSeconds = phases.orthogonalisationSeconds;
    solution.projectedSeconds = phases.projectedSeconds;
    return solution;
}

} // namespace oosgpu::eigen
