// The factor object on the GPU and the C ABI of include/oos_gpu.h.
//
// A factor owns, on its device: the plan's arrays (descriptors, children, rows, positions, task lists), the panels
// (the reference's layout: supernode s at the sum of c(c + r) before it, column-major, leading dimension c + r), the
// update matrices of every supernode (each r x r), a copy of the matrix, and the solve's work rows. It runs every
// launch of a factorisation or a solve on its own stream; a factorisation reads back only its pivot summary.

#include "../device/kernels.cuh"
#include "delayed.hpp"
#include "factor_internal.hpp"
#include "host_api.hpp"
#include "spectrum.hpp"
#include "plan.hpp"

#include "oos_gpu.h"

#include <cuda.h> // CUtensorMap and the types of cuTensorMapEncodeTiled

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <string>
#include <vector>

namespace oosgpu
{

namespace
{

thread_local std::string g_lastError;

void check(cudaError_t status, const char* what)
{
    if (status != cudaSuccess)
        throw Error(status == cudaErrorMemoryAllocation ? STATUS_MEMORY_BUDGET : STATUS_CUDA,
                    std::string(what) + ": " + cudaGetErrorString(status));
}

constexpr int NO_PIVOT = 0x7f7f7f7f; // the byte pattern 0x7f: "no zero pivot"
constexpr int ISSUE_CAPACITY = 1 << 16;
constexpr int SOLVE_WIDTH = 64;
constexpr int SMALL_THREADS = 256;
// The relative fall of each column's preconditioned residual that ends a GMRES correction.
constexpr double GMRES_INNER_TOLERANCE = 1.0e-4;

// A device allocation owned by the factor.
template <typename T> class DeviceArray
{
public:
    DeviceArray() = default;
    DeviceArray(const DeviceArray&) = delete;
    DeviceArray& operator=(const DeviceArray&) = delete;
    ~DeviceArray() { release(); }
    void allocate(std::size_t count, const char* what)
    {
        if (count <= m_count && m_data != nullptr)
            return;
        release();
        void* p = nullptr;
        check(cudaMalloc(&p, std::max<std::size_t>(count, 1) * sizeof(T)), what);
        m_data = static_cast<T*>(p);
        m_count = count;
    }
    void upload(const std::vector<T>& host, cudaStream_t stream, const char* what)
    {
        allocate(host.size(), what);
        if (!host.empty())
            check(cudaMemcpyAsync(m_data, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice, stream), what);
    }
    void release()
    {
        if (m_data != nullptr)
            cudaFree(m_data);
        m_data = nullptr;
        m_count = 0;
    }
    [[nodiscard]] T* get() const noexcept { return m_data; }
    [[nodiscard]] std::size_t size() const noexcept { return m_count; }

private:
    T* m_data = nullptr;
    std::size_t m_count = 0;
};

// cuTensorMapEncodeTiled, reached through the runtime's driver entry point (no link against the driver library).
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled tensorMapEncoder()
{
    static EncodeTiled encoder = nullptr;
    if (encoder == nullptr)
    {
        void* function = nullptr;
        cudaDriverEntryPointQueryResult found = cudaDriverEntryPointSymbolNotFound;
        check(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &function, cudaEnableDefault, &found),
              "cuTensorMapEncodeTiled entry point");
        if (function == nullptr || found != cudaDriverEntryPointSuccess)
            throw Error(STATUS_CUDA, "the driver offers no cuTensorMapEncodeTiled");
        encoder = reinterpret_cast<EncodeTiled>(function);
    }
    return encoder;
}

unsigned blocksFor(std::int64_t items, int threads)
{
    return static_cast<unsigned>((items + threads - 1) / threads);
}

// A fixed sequence of launches on one stream replayed as a CUDA graph: captured the first time it runs with a given
// key (the device buffers and settings the launches are given) and replayed whenever that key comes back; the last
// GRAPHS keys are kept (a refinement or a GMRES correction alternates between a few buffers). The launches then reach
// the GPU as one submission, without the host's cost and the gaps per launch.
class LaunchGraph
{
public:
    static constexpr std::size_t GRAPHS = 16;

    LaunchGraph() = default;
    LaunchGraph(const LaunchGraph&) = delete;
    LaunchGraph& operator=(const LaunchGraph&) = delete;
    ~LaunchGraph() { reset(); }

    template <typename Launches> void run(cudaStream_t stream, const std::vector<std::uintptr_t>& key, Launches launches)
    {
        auto found = std::find_if(m_graphs.begin(), m_graphs.end(), [&](const Entry& e) { return e.key == key; });
        if (found == m_graphs.end())
        {
            if (m_graphs.size() == GRAPHS)
            {
                cudaGraphExecDestroy(m_graphs.front().exec);
                m_graphs.erase(m_graphs.begin());
            }
            check(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "graph capture");
            try
            {
                launches();
            }
            catch (...)
            {
                cudaGraph_t discarded = nullptr;
                cudaStreamEndCapture(stream, &discarded);
                if (discarded != nullptr)
                    cudaGraphDestroy(discarded);
                throw;
            }
            cudaGraph_t graph = nullptr;
            check(cudaStreamEndCapture(stream, &graph), "graph capture");
            cudaGraphExec_t exec = nullptr;
            const cudaError_t status = cudaGraphInstantiate(&exec, graph, 0);
            cudaGraphDestroy(graph);
            check(status, "graph instantiation");
            m_graphs.push_back({key, exec});
            found = m_graphs.end() - 1;
        }
        check(cudaGraphLaunch(found->exec, stream), "graph launch");
    }

    void reset()
    {
        for (const Entry& e : m_graphs)
            cudaGraphExecDestroy(e.exec);
        m_graphs.clear();
    }

private:
    struct Entry
    {
        std::vector<std::uintptr_t> key;
        cudaGraphExec_t exec;
    };
    std::vector<Entry> m_graphs;
};

std::uintptr_t keyOf(const void* p)
{
    return reinterpret_cast<std::uintptr_t>(p);
}

} // namespace

class GpuFactor
{
public:
    // prebuilt: the structure's plan when the caller has it already (a copy is taken: the factor's own choices change
    // its launches), else it is built here.
    GpuFactor(const Symbolic& symbolic, int device, const Plan* prebuilt = nullptr)
        : m_symbolic(symbolic), m_device(device)
    {
        check(cudaSetDevice(device), "cudaSetDevice");
        m_plan = prebuilt != nullptr ? *prebuilt : buildPlan(symbolic);
        // The main stream at the highest priority, the lookahead's side stream at the lowest: when an SM frees up,
        // the chain of a front's steps (one or a few blocks a launch) is scheduled before the side's update tiles.
        int leastPriority = 0;
        int greatestPriority = 0;
        check(cudaDeviceGetStreamPriorityRange(&leastPriority, &greatestPriority), "stream priorities");
        check(cudaStreamCreateWithPriority(&m_stream, cudaStreamNonBlocking, greatestPriority), "cudaStreamCreate");
        check(cudaStreamCreateWithPriority(&m_side, cudaStreamNonBlocking, leastPriority), "cudaStreamCreate");
        check(cudaStreamCreateWithFlags(&m_copyStream, cudaStreamNonBlocking), "cudaStreamCreate");
        check(cudaEventCreateWithFlags(&m_prefetchDone, cudaEventDisableTiming), "cudaEventCreate");
        check(cudaEventCreateWithFlags(&m_prefetchStart, cudaEventDisableTiming), "cudaEventCreate");
        check(cudaEventCreateWithFlags(&m_fork, cudaEventDisableTiming), "cudaEventCreate");
        for (cudaEvent_t& e : m_groupDone)
            check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
        check(cudaEventCreate(&m_start), "cudaEventCreate");
        check(cudaEventCreate(&m_stop), "cudaEventCreate");
        m_fronts.upload(m_plan.fronts, m_stream, "plan: fronts");
        m_children.upload(m_plan.children, m_stream, "plan: children");
        m_rows.upload(m_plan.rows, m_stream, "plan: rows");
        m_relpos.upload(m_plan.relpos, m_stream, "plan: positions");
        m_gatherStart.upload(m_plan.gatherStart, m_stream, "plan: gather lists");
        m_gatherRows.upload(m_plan.gatherRows, m_stream, "plan: gather lists");
        if (m_plan.rowPartialSlots > 0)
            m_rowPartials.allocate(static_cast<std::size_t>(m_plan.rowPartialSlots) * device::TILE * device::TILE,
                                   "solve: split products");
        allocateChains(m_plan);
        void* failed = nullptr;
        check(cudaHostAlloc(&failed, sizeof(int), cudaHostAllocMapped), "solve: chain status");
        m_chainFailed = static_cast<int*>(failed);
        *m_chainFailed = 0;
        m_supernodeOfColumn.upload(m_plan.supernodeOfColumn, m_stream, "plan: columns");
        m_lists.upload(m_plan.lists, m_stream, "plan: lists");
        m_tiles.upload(m_plan.tiles, m_stream, "plan: tiles");
        m_pieces.upload(m_plan.pieces, m_stream, "plan: pieces");
        m_stagedPieces.upload(m_plan.stagedPieces, m_stream, "plan: staged pieces");
        m_zeroPivot.allocate(static_cast<std::size_t>(m_plan.supernodeCount), "factor: zero pivots");
        m_diagonal.allocate(static_cast<std::size_t>(std::max(m_plan.dimension, 1)), "factor: diagonal");
        m_counters.allocate(8, "factor: counters");
        m_issues.allocate(ISSUE_CAPACITY, "factor: issues");
        const std::size_t summaryBlocks = blocksFor(std::max(m_plan.dimension, 1), 256);
        m_blockRatio.allocate(summaryBlocks, "factor: ratios");
        m_blockEquation.allocate(summaryBlocks, "factor: ratio equations");
        m_structureError.allocate(1, "factor: structure check");
        m_mixedError.allocate(1, "factor: tensor-core status");
        // Shared memory of the small-front kernel: the largest small front, square.
        const int order = m_plan.largestSmallOrder;
        m_smallSmem = static_cast<std::size_t>(order) * (order + 1) * sizeof(double);
        // A kernel's shared-memory limit is the process's, not this factor's: every factor sets the largest any plan
        // can need, so that no factor lowers another's.
        const auto smallLimit = static_cast<int>(static_cast<std::size_t>(SMALL_ORDER) * (SMALL_ORDER + 1) * sizeof(double));
        check(cudaFuncSetAttribute(device::smallFronts, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(device::smallFrontSmem(SMALL_ORDER))),
              "smallFronts shared memory");
        check(cudaFuncSetAttribute(device::smallFrontsPivoted, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   smallLimit),
              "smallFrontsPivoted shared memory");
        check(cudaFuncSetAttribute(device::updateMatrixTma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(device::UPDATE_TMA_SMEM)),
              "TMA update shared memory");
        check(cudaFuncSetAttribute(device::assembleStaged, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(device::STAGE_SMEM)),
              "staged assembly shared memory");
        check(cudaFuncSetAttribute(device::updateMatrixMixed, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(device::MIXED_UPDATE_SMEM)),
              "mixed update shared memory");
        check(cudaFuncSetAttribute(device::panelRowsInverse, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(device::PANEL_ROWS_INVERSE_SMEM)),
              "panel rows shared memory");
        check(cudaFuncSetAttribute(device::panelRowsPivotedInverse, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(device::PANEL_ROWS_PIVOTED_SMEM)),
              "pivoted panel rows shared memory");
        // The chains of the solves: the A pipeline, the ready rows of x and a block's inverse.
        for (const void* kernel : {reinterpret_cast<const void*>(device::forwardChain),
                                   reinterpret_cast<const void*>(device::backwardChain)})
            check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(device::CHAIN_SMEM)),
                  "chain solve shared memory");
        for (const void* kernel : {reinterpret_cast<const void*>(device::forwardSmall),
                                   reinterpret_cast<const void*>(device::backwardSmall)})
            check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(device::smallSolveSmem(SOLVE_SMALL_COLUMNS))),
                  "small solve shared memory");
        check(cudaStreamSynchronize(m_stream), "plan upload");
    }

    ~GpuFactor()
    {
        cudaSetDevice(m_device);
        if (m_stream != nullptr)
            cudaStreamSynchronize(m_stream);
        if (m_side != nullptr)
            cudaStreamSynchronize(m_side);
        if (m_copyStream != nullptr)
            cudaStreamSynchronize(m_copyStream);
        cudaEventDestroy(m_prefetchDone);
        cudaEventDestroy(m_prefetchStart);
        cudaEventDestroy(m_fork);
        for (cudaEvent_t e : m_groupDone)
            cudaEventDestroy(e);
        cudaEventDestroy(m_start);
        cudaEventDestroy(m_stop);
        for (cudaEvent_t e : m_profileEvents)
            cudaEventDestroy(e);
        for (cudaEvent_t e : m_solveEvents)
            cudaEventDestroy(e);
        if (m_stream != nullptr)
            cudaStreamDestroy(m_stream);
        if (m_side != nullptr)
            cudaStreamDestroy(m_side);
        if (m_copyStream != nullptr)
            cudaStreamDestroy(m_copyStream);
        if (m_chainFailed != nullptr)
            cudaFreeHost(m_chainFailed);
    }

    [[nodiscard]] cudaStream_t stream() const noexcept { return m_stream; }

    // The chain state for a plan's sweeps (ticket counters, ready flags, the stop word), grown when a plan needs more;
    // a new array starts cleared.
    void allocateChains(const Plan& plan)
    {
        const std::size_t needed = static_cast<std::size_t>(plan.chainSlots) + static_cast<std::size_t>(plan.chainFlags) + 1;
        if (m_chainState.get() != nullptr && needed <= m_chainState.size())
            return;
        m_chainState.allocate(needed, "solve: chain state");
        check(cudaMemsetAsync(m_chainState.get(), 0, m_chainState.size() * sizeof(int), m_stream), "chain state");
    }

    // A sweep whose chain wait ran out (the mapped status the kernels set) voids the factor's solves from then on.
    void checkChains() const
    {
        if (m_chainFailed != nullptr && *reinterpret_cast<volatile int*>(m_chainFailed) != 0)
            throw Error(STATUS_INTERNAL, "FactorSolve: a solve's chain step waited past its limit (the results are "
                                         "void; the factor's solves are disabled)");
    }

    // Right-hand sides copied ahead of a solve (oosgpu_solve_prefetch): host B (n x columns, ld) into the device
    // buffer the next host-array solve of the same B uses, on a copy stream of its own, so that the copy overlaps
    // whatever the factor does meanwhile. The copy starts at once, or, when a factorisation follows, once that
    // factorisation's matrix is on the device (the two copies would otherwise share the host link and delay the
    // factorisation's start). B must stay unchanged until the solve.
    void prefetch(const double* b, std::int64_t ld, std::int64_t columns, bool deferred)
    {
        check(cudaSetDevice(m_device), "cudaSetDevice");
        const std::int32_t n = m_plan.dimension;
        if (b == nullptr || ld < n || columns < 0)
            throw Error(STATUS_INVALID_ARGUMENT, "solve prefetch: expected " + std::to_string(n) +
                                                     " rows (leading dimension >= rows) and columns >= 0");
        check(cudaStreamSynchronize(m_copyStream), "an earlier prefetch");
        m_prefetch = {b, ld, columns, false};
        m_hostB.allocate(static_cast<std::size_t>(n) * static_cast<std::size_t>(columns), "solve: right-hand sides");
        if (!deferred)
            issuePrefetch();
    }

    // The copy of a prefetch not yet issued, on the copy stream after the work the main stream has queued so far.
    void issuePrefetch()
    {
        if (m_prefetch.host == nullptr || m_prefetch.issued)
            return;
        const std::int32_t n = m_plan.dimension;
        check(cudaEventRecord(m_prefetchStart, m_stream), "prefetch event");
        check(cudaStreamWaitEvent(m_copyStream, m_prefetchStart, 0), "prefetch after the matrix");
        if (m_prefetch.columns > 0 && n > 0)
            check(cudaMemcpy2DAsync(m_hostB.get(), static_cast<std::size_t>(n) * sizeof(double), m_prefetch.host,
                                    static_cast<std::size_t>(m_prefetch.ld) * sizeof(double),
                                    static_cast<std::size_t>(n) * sizeof(double),
                                    static_cast<std::size_t>(m_prefetch.columns), cudaMemcpyHostToDevice,
                                    m_copyStream),
                  "prefetch right-hand sides");
        check(cudaEventRecord(m_prefetchDone, m_copyStream), "prefetch event");
        m_prefetch.issued = true;
    }

    // The device copy (n x columns, leading dimension n) of host right-hand sides for a solve on the main stream: the
    // prefetched one when it is this B, else uploaded now.
    double* rightHandSides(const double* b, std::int64_t ld, std::int64_t columns, const char* what)
    {
        const std::int32_t n = m_plan.dimension;
        const Prefetch ahead = m_prefetch;
        m_prefetch = {};
        if (ahead.host == b && ahead.ld == ld && ahead.columns == columns && b != nullptr && ahead.issued)
        {
            check(cudaStreamWaitEvent(m_stream, m_prefetchDone, 0), "wait for the prefetched right-hand sides");
            return m_hostB.get();
        }
        check(cudaStreamSynchronize(m_copyStream), "an unused prefetch");
        m_hostB.allocate(static_cast<std::size_t>(n) * static_cast<std::size_t>(columns), what);
        check(cudaMemcpy2DAsync(m_hostB.get(), static_cast<std::size_t>(n) * sizeof(double), b,
                                static_cast<std::size_t>(ld) * sizeof(double), static_cast<std::size_t>(n) * sizeof(double),
                                static_cast<std::size_t>(columns), cudaMemcpyHostToDevice, m_stream),
              "upload right-hand sides");
        return m_hostB.get();
    }
    [[nodiscard]] const Plan& plan() const noexcept { return m_plan; }

    // trailing > 0: the partial factorisation (PartialFactor::factorise): every supernode below the trailing one
    // (the last supernode: the trailing set's equations, a root alone in its level, no rows below) factorised in
    // positive definite mode; its front, assembled from the matrix's boundary entries and its children's update
    // matrices, is K* = K_bb - K_bi K_ii^-1 K_ib, written to `schur` (host, trailing x trailing, both triangles).
    void factorise(std::int32_t dimension, std::int64_t terms, const std::int64_t* offsets, const std::int32_t* rows,
                   const double* values, bool onDevice, const oosgpu_factor_options* options, oosgpu_factor_info* info,
                   std::int32_t trailing = 0, double* schur = nullptr)
    {
        check(cudaSetDevice(m_device), "cudaSetDevice");
        m_partialLevel = -1;
        m_isPartial = false;
        if (trailing != 0)
            preparePartial(dimension, trailing, options);
        if (dimension != m_plan.dimension)
            throw Error(STATUS_INVALID_ARGUMENT,
                        "supernodal factorisation: the matrix has " + std::to_string(dimension) +
                            " equations and the symbolic factor " + std::to_string(m_plan.dimension) +
                            "; factorise the matrix assembled on the graph and in the order of its symbolic analysis");
        const double maxRatio = options != nullptr ? options->max_ratio : 1.0e7;
        const int bailout = options != nullptr ? options->bailout : 0;
        m_panels.allocate(static_cast<std::size_t>(m_plan.panelValues), "factor: panels");
        m_updates.allocate(static_cast<std::size_t>(m_plan.updateValues), "factor: update matrices");
        buildTensorMaps();
        const std::int64_t* dOffsets = offsets;
        const std::int32_t* dRows = rows;
        const double* dValues = values;
        if (!onDevice)
        {
            if (offsets[dimension] != terms && terms >= 0)
                throw Error(STATUS_INVALID_ARGUMENT, "supernodal factorisation: the offsets do not end at the terms");
            terms = offsets[dimension];
            m_cscOffsets.allocate(static_cast<std::size_t>(dimension) + 1, "factor: matrix offsets");
            m_cscRows.allocate(static_cast<std::size_t>(terms), "factor: matrix rows");
            m_cscValues.allocate(static_cast<std::size_t>(terms), "factor: matrix values");
            check(cudaMemcpyAsync(m_cscOffsets.get(), offsets, (static_cast<std::size_t>(dimension) + 1) * sizeof(std::int64_t),
                                  cudaMemcpyHostToDevice, m_stream),
                  "upload offsets");
            check(cudaMemcpyAsync(m_cscRows.get(), rows, static_cast<std::size_t>(terms) * sizeof(std::int32_t),
                                  cudaMemcpyHostToDevice, m_stream),
                  "upload rows");
            check(cudaMemcpyAsync(m_cscValues.get(), values, static_cast<std::size_t>(terms) * sizeof(double),
                                  cudaMemcpyHostToDevice, m_stream),
                  "upload values");
            dOffsets = m_cscOffsets.get();
            dRows = m_cscRows.get();
            dValues = m_cscValues.get();
        }
        issuePrefetch(); // loads prefetched for the solve travel once the matrix has
        if (!m_annotated)
        {
            // The matrix terms of each supernode's columns, for the launches' algorithmic bytes.
            std::vector<std::int64_t> hostOffsets(static_cast<std::size_t>(dimension) + 1);
            if (onDevice)
                check(cudaMemcpy(hostOffsets.data(), offsets, hostOffsets.size() * sizeof(std::int64_t),
                                 cudaMemcpyDeviceToHost),
                      "download offsets");
            else
                std::copy_n(offsets, hostOffsets.size(), hostOffsets.begin());
            std::vector<std::int64_t> termsOfFront(static_cast<std::size_t>(m_plan.supernodeCount));
            for (std::int32_t s = 0; s < m_plan.supernodeCount; ++s)
            {
                const device::FrontDesc& f = m_plan.fronts[static_cast<std::size_t>(s)];
                termsOfFront[static_cast<std::size_t>(s)] =
                    hostOffsets[static_cast<std::size_t>(f.first + f.c)] - hostOffsets[static_cast<std::size_t>(f.first)];
            }
            annotate(m_plan, termsOfFront);
            m_annotated = true;
        }
        const double* referenceDiagonal = nullptr;
        if (options != nullptr && options->reference_diagonal != nullptr)
        {
            m_referenceDiagonal.allocate(static_cast<std::size_t>(dimension), "factor: reference diagonal");
            check(cudaMemcpyAsync(m_referenceDiagonal.get(), options->reference_diagonal,
                                  static_cast<std::size_t>(dimension) * sizeof(double), cudaMemcpyHostToDevice, m_stream),
                  "upload reference diagonal");
            referenceDiagonal = m_referenceDiagonal.get();
        }

        m_matrixOffsets = dOffsets;
        m_matrixRows = dRows;
        m_matrixValues = dValues;
        m_matrixTerms = onDevice ? terms : offsets[dimension];
        device::FactorArgs args{m_fronts.get(),   m_children.get(), m_rows.get(),  m_relpos.get(),
                                dOffsets,         dRows,            dValues,       m_panels.get(),
                                m_updates.get(),  m_zeroPivot.get()};
        check(cudaEventRecord(m_start, m_stream), "event");
        check(cudaMemsetAsync(m_zeroPivot.get(), 0x7f, static_cast<std::size_t>(m_plan.supernodeCount) * sizeof(std::int32_t),
                              m_stream),
              "memset");
        check(cudaMemsetAsync(m_structureError.get(), 0x7f, sizeof(std::int32_t), m_stream), "memset");
        check(cudaMemsetAsync(m_counters.get(), 0, 8 * sizeof(unsigned long long), m_stream), "memset");
        if (options != nullptr && options->pivoting != 0)
        {
            factoriseIndefinite(args, dimension, info);
            return;
        }
        m_pivoted = false;
        m_singular = false;
        m_mixed = options != nullptr && options->precision == 1;
        if (options != nullptr && options->precision != 0 && options->precision != 1)
            throw Error(STATUS_INVALID_ARGUMENT, "FactorOptions: precision must be 0 (FP64) or 1 (mixed), found " +
                                                     std::to_string(options->precision));
        check(cudaMemsetAsync(m_mixedError.get(), 0, sizeof(int), m_stream), "memset"); // tcgen05 and TMA waits
        // the equations the pivot summary covers: all of them, or the interior of a partial factorisation
        const std::int32_t summarised = m_partialLevel >= 0 ? dimension - m_trailing : dimension;
        const unsigned summaryBlocks = blocksFor(std::max(summarised, 1), 256);
        const auto launches = [&]
        {
            // the pivot summary's counters from zero in every run of the sequence (the autotuner's timing runs, the
            // graph's replays)
            check(cudaMemsetAsync(m_counters.get(), 0, 8 * sizeof(unsigned long long), m_stream), "memset");
            runFactorLaunches(args);
            invertDiagonalBlocks(args, false);
            device::pivotSummary<<<summaryBlocks, 256, 0, m_stream>>>(args, m_supernodeOfColumn.get(), summarised,
                                                                       referenceDiagonal, maxRatio, m_counters.get(),
                                                                       m_issues.get(), ISSUE_CAPACITY,
                                                                       m_blockRatio.get(), m_blockEquation.get());
            device::gatherDiagonal<<<summaryBlocks, 256, 0, m_stream>>>(args, m_supernodeOfColumn.get(), summarised,
                                                                         m_diagonal.get());
            check(cudaGetLastError(), "pivot summary launch");
        };
        if (m_tuning && !m_tuned && !m_mixed)
            tune(launches);
        // Profiled factorisations launch one by one (events between the launches); the others replay a graph.
        if (m_profile)
            launches();
        else
        {
            std::uint64_t ratioBits = 0;
            std::memcpy(&ratioBits, &maxRatio, sizeof ratioBits);
            m_factorGraph.run(m_stream,
                              {keyOf(dOffsets), keyOf(dRows), keyOf(dValues), keyOf(referenceDiagonal),
                               static_cast<std::uintptr_t>(ratioBits), static_cast<std::uintptr_t>(m_mixed),
                               static_cast<std::uintptr_t>(dimension), static_cast<std::uintptr_t>(m_partialLevel + 1)},
                              launches);
        }
        check(cudaEventRecord(m_stop, m_stream), "event");

        // The summary back on the host.
        std::vector<unsigned long long> counters(8);
        std::vector<std::int32_t> zeroPivot(static_cast<std::size_t>(m_plan.supernodeCount));
        std::vector<double> blockRatio(summaryBlocks);
        std::vector<std::int32_t> blockEquation(summaryBlocks);
        std::int32_t structureError = 0;
        check(cudaMemcpyAsync(counters.data(), m_counters.get(), 8 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                              m_stream),
              "download counters");
        check(cudaMemcpyAsync(zeroPivot.data(), m_zeroPivot.get(), zeroPivot.size() * sizeof(std::int32_t),
                              cudaMemcpyDeviceToHost, m_stream),
              "download zero pivots");
        check(cudaMemcpyAsync(blockRatio.data(), m_blockRatio.get(), summaryBlocks * sizeof(double),
                              cudaMemcpyDeviceToHost, m_stream),
              "download ratios");
        check(cudaMemcpyAsync(blockEquation.data(), m_blockEquation.get(), summaryBlocks * sizeof(std::int32_t),
                              cudaMemcpyDeviceToHost, m_stream),
              "download ratio equations");
        check(cudaMemcpyAsync(&structureError, m_structureError.get(), sizeof(std::int32_t), cudaMemcpyDeviceToHost,
                              m_stream),
              "download structure check");
        int mixedError = 0;
        check(cudaMemcpyAsync(&mixedError, m_mixedError.get(), sizeof(int), cudaMemcpyDeviceToHost, m_stream),
              "download tensor-core status");
        check(cudaStreamSynchronize(m_stream), "factorisation");
        m_profileValid = m_profile;
        m_profiledPivoted = false;
        if (mixedError != 0)
        {
            m_factorised = false;
            throw Error(STATUS_INTERNAL, "factorisation: a bounded wait on the tensor cores or on a TMA load ran out "
                                         "(the update matrices are incomplete)");
        }
        float milliseconds = 0.0f;
        check(cudaEventElapsedTime(&milliseconds, m_start, m_stop), "event time");
        m_factorised = false;
        if (structureError != NO_PIVOT)
            throw Error(STATUS_INVALID_ARGUMENT,
                        "supernodal factorisation: column " + std::to_string(structureError) +
                            " of the matrix has an entry outside the structure of the symbolic factor; build the CSC in "
                            "the order of the symbolic factor, on the graph it was analysed on");

        oosgpu_factor_info result{};
        result.positive = static_cast<std::int64_t>(counters[0]);
        result.negative = static_cast<std::int64_t>(counters[1]);
        result.zero = static_cast<std::int64_t>(counters[2]);
        result.issue_count = static_cast<std::int64_t>(counters[3]);
        result.device_seconds = milliseconds / 1000.0;
        result.largest_ratio = 0.0;
        result.equation_of_largest = -1;
        for (unsigned b = 0; b < summaryBlocks; ++b)
            if (blockEquation[b] != INT_MAX &&
                (result.equation_of_largest < 0 || blockRatio[b] > result.largest_ratio))
            {
                result.largest_ratio = blockRatio[b];
                result.equation_of_largest = blockEquation[b];
            }
        // Issues in elimination order (equation order in positive definite mode).
        const auto issueCount = static_cast<std::size_t>(std::min<std::int64_t>(result.issue_count, ISSUE_CAPACITY));
        if (issueCount > 0)
        {
            std::vector<std::int32_t> issues(issueCount);
            check(cudaMemcpy(issues.data(), m_issues.get(), issueCount * sizeof(std::int32_t), cudaMemcpyDeviceToHost),
                  "download issues");
            std::sort(issues.begin(), issues.end());
            for (std::size_t k = 0; k < std::min<std::size_t>(16, issues.size()); ++k)
                result.issues[k] = issues[k];
        }
        // Zero pivots: a supernode with a failed descendant is not counted (the reference skips it).
        std::vector<char> failedBelow(static_cast<std::size_t>(m_plan.supernodeCount), 0);
        std::vector<std::int32_t> zeroEquations;
        for (std::int32_t s = 0; s < m_plan.supernodeCount; ++s)
        {
            const auto at = static_cast<std::size_t>(s);
            const bool failed = zeroPivot[at] != NO_PIVOT;
            if (failed && failedBelow[at] == 0)
                zeroEquations.push_back(m_plan.fronts[at].first + zeroPivot[at]);
            const std::int32_t p = m_plan.fronts[at].parent;
            if (p >= 0 && (failed || failedBelow[at] != 0))
                failedBelow[static_cast<std::size_t>(p)] = 1;
        }
        result.zero_pivot_count = static_cast<std::int32_t>(zeroEquations.size());
        for (std::size_t k = 0; k < std::min<std::size_t>(16, zeroEquations.size()); ++k)
            result.zero_pivots[k] = zeroEquations[k];
        if (info != nullptr)
            *info = result;
        if (!zeroEquations.empty())
        {
            std::string names;
            for (std::size_t k = 0; k < std::min<std::size_t>(10, zeroEquations.size()); ++k)
                names += "  equation " + std::to_string(zeroEquations[k]) + "\n";
            throw Error(STATUS_SINGULAR, "the stiffness matrix is singular: " + std::to_string(zeroEquations.size()) +
                                             " zero (or not finite) pivots met in the factorisation, a mechanism or an "
                                             "unconstrained DOF at:\n" +
                                             names);
        }
        if (result.issue_count > 0 && bailout >= 0)
            throw Error(STATUS_SINGULAR, "the ratio test flagged " + std::to_string(result.issue_count) +
                                             " pivots (MaxDiagonalRatio " + std::to_string(maxRatio) +
                                             "; the first at equation " + std::to_string(result.issues[0]) + ")");
        if (m_partialLevel >= 0)
            trailingComplement(args, schur);
        m_factorised = true;
    }

    // The checks of a partial factorisation and its launch filter: the last supernode holds the trailing equations
    // (the last `trailing` ones), has no rows below and no other supernode shares its level.
    void preparePartial(std::int32_t dimension, std::int32_t trailing, const oosgpu_factor_options* options)
    {
        const std::int32_t last = m_plan.supernodeCount - 1;
        if (last < 0 || trailing < 0)
            throw Error(STATUS_INVALID_ARGUMENT, "PartialFactor: expected a trailing count in [1, dimension]");
        const device::FrontDesc& f = m_plan.fronts[static_cast<std::size_t>(last)];
        if (f.parent >= 0 || f.r != 0 || f.c != trailing || f.first + f.c != dimension)
            throw Error(STATUS_INVALID_ARGUMENT,
                        "PartialFactor: the symbolic factor's last supernode must be the trailing set (" +
                            std::to_string(trailing) + " equations, ordered last, a root); it has " +
                            std::to_string(f.c) + " columns from equation " + std::to_string(f.first) +
                            "; analyse with the unit's boundary as the trailing nodes");
        const std::int32_t level = m_plan.level[static_cast<std::size_t>(last)];
        if (m_plan.frontsOfLevel[static_cast<std::size_t>(level)].size() != 1)
            throw Error(STATUS_INVALID_ARGUMENT, "PartialFactor: the interior has a part that reaches no boundary "
                                                 "equation (another root beside the trailing supernode)");
        if (options != nullptr && (options->pivoting != 0 || options->precision != 0))
            throw Error(STATUS_INVALID_ARGUMENT,
                        "PartialFactor: the interior of a unit is factorised in positive definite mode, FP64 (a "
                        "delayed pivot would move an interior equation into the boundary); pass pivoting 0");
        m_partialLevel = level;
        m_trailing = trailing;
        m_partialForward.clear();
        m_partialBackward.clear();
        for (const Launch& launch : m_plan.forwardLaunches)
            if (launch.level < level)
                m_partialForward.push_back(launch);
        for (const Launch& launch : m_plan.backwardLaunches)
            if (launch.level < level)
                m_partialBackward.push_back(launch);
    }

    // K* of a partial factorisation: the trailing front assembled from its children's update matrices (at their
    // positions in it, the plan's maps) and the matrix's boundary entries, into `schur` (host).
    void trailingComplement(const device::FactorArgs& args, double* schur)
    {
        const std::int32_t last = m_plan.supernodeCount - 1;
        const device::FrontDesc& f = m_plan.fronts[static_cast<std::size_t>(last)];
        std::vector<device::FrontSource> sources;
        for (std::int32_t q = 0; q < f.childCount; ++q)
        {
            const device::FrontDesc& child =
                m_plan.fronts[static_cast<std::size_t>(m_plan.children[static_cast<std::size_t>(f.childStart + q)])];
            if (child.r > 0)
                sources.push_back({m_updates.get() + child.update, m_relpos.get() + child.rowStart, child.r, 0});
        }
        m_exactSources.upload(sources, m_stream, "partial factor: sources");
        const auto t = static_cast<std::size_t>(m_trailing);
        m_schur.allocate(t * t, "partial factor: K*");
        const device::ExactFront front{last, m_trailing, m_trailing, static_cast<std::int32_t>(sources.size()),
                                       m_exactSources.get(), nullptr};
        device::trailingFront<<<1, 1024, 0, m_stream>>>(args, front, m_schur.get(), m_structureError.get());
        check(cudaGetLastError(), "trailing front launch");
        std::int32_t structureError = 0;
        check(cudaMemcpyAsync(&structureError, m_structureError.get(), sizeof(std::int32_t), cudaMemcpyDeviceToHost,
                              m_stream),
              "download structure check");
        if (schur != nullptr)
            check(cudaMemcpyAsync(schur, m_schur.get(), t * t * sizeof(double), cudaMemcpyDeviceToHost, m_stream),
                  "download K*");
        check(cudaStreamSynchronize(m_stream), "partial factorisation");
        if (structureError != NO_PIVOT)
            throw Error(STATUS_INVALID_ARGUMENT,
                        "supernodal factorisation: column " + std::to_string(structureError) +
                            " of the matrix has an entry outside the structure of the symbolic factor");
        m_isPartial = true;
    }

    // PartialFactor::condenseLoads (condense) and PartialFactor::recover (recover) on host arrays: loads n x columns
    // (ld); condense writes f* = f_b - K_bi K_ii^-1 f_i (trailing x columns, ld ldOut) to `out`; recover replaces the
    // loads by u (its interior u_i = K_ii^-1 (f_i - K_ib u_b), its trailing rows the given u_b, `trailingValues`).
    void partialSolve(double* loads, std::int64_t ld, std::int64_t columns, double* out, std::int64_t ldOut,
                      const double* trailingValues, bool recover)
    {
        check(cudaSetDevice(m_device), "cudaSetDevice");
        if (!m_factorised || !m_isPartial)
            throw Error(STATUS_NOT_FACTORISED, "PartialFactor: no partial factorisation (call factorise_partial)");
        const std::int32_t n = m_plan.dimension;
        const std::int32_t t = m_trailing;
        if (ld < n || columns < 0 || ldOut < t)
            throw Error(STATUS_INVALID_ARGUMENT, "PartialFactor: expected " + std::to_string(n) + " load rows and " +
                                                     std::to_string(t) + " trailing rows (leading dimensions)");
        if (columns == 0)
            return;
        const auto rowsOf = [](std::int64_t k) { return static_cast<std::size_t>(k) * sizeof(double); };
        m_work.allocate(static_cast<std::size_t>(n) * SOLVE_WIDTH, "solve: rows");
        m_updateRows.allocate(updateRowsPerColumn() * SOLVE_WIDTH, "solve: update rows");
        check(cudaStreamSynchronize(m_copyStream), "an unused prefetch");
        m_prefetch = {};
        m_hostB.allocate(static_cast<std::size_t>(n) * static_cast<std::size_t>(columns), "partial factor: loads");
        double* b = m_hostB.get();
        check(cudaMemcpy2DAsync(b, rowsOf(n), loads, rowsOf(ld), rowsOf(n), static_cast<std::size_t>(columns),
                                cudaMemcpyHostToDevice, m_stream),
              "upload loads");
        if (recover)
            check(cudaMemcpy2DAsync(b + (n - t), rowsOf(n), trailingValues, rowsOf(ldOut), rowsOf(t),
                                    static_cast<std::size_t>(columns), cudaMemcpyHostToDevice, m_stream),
                  "upload trailing values");
        const std::int32_t last = m_plan.supernodeCount - 1;
        for (std::int64_t c0 = 0; c0 < columns; c0 += SOLVE_WIDTH)
        {
            const int width = static_cast<int>(std::min<std::int64_t>(SOLVE_WIDTH, columns - c0));
            double* x = m_work.get();
            rowsIn(b, n, static_cast<int>(c0), width, x);
            const SolveView view = solveView();
            const device::SolveArgs args{view.fronts,       m_children.get(), view.rows,       view.relpos,
                                         m_panels.get(),    x,                m_updateRows.get(), width,
                                         view.gatherStart,  view.gatherRows,  nullptr,          n,
                                         m_rowPartials.get(),
                                         m_chainState.get(),
                                         m_chainState.get() + view.plan->chainSlots,
                                         m_chainState.get() + (m_chainState.size() - 1),
                                         m_chainFailed};
            runSweep(args, view, m_partialForward);
            if (recover)
            {
                const std::int64_t items = static_cast<std::int64_t>(n - t) * width;
                device::diagonalSweep<<<blocksFor(std::max<std::int64_t>(items, 1), 256), 256, 0, m_stream>>>(
                    args, m_diagonal.get(), n - t);
                runSweep(args, view, m_partialBackward);
            }
            else
                device::gatherColumns<<<blocksFor(static_cast<std::int64_t>(t) * width, 256), 256, 0, m_stream>>>(
                    args, last);
            check(cudaGetLastError(), "partial solve launch");
            rowsOut(x, static_cast<int>(c0), width, b, n);
        }
        if (recover)
            check(cudaMemcpy2DAsync(loads, rowsOf(ld), b, rowsOf(n), rowsOf(n), static_cast<std::size_t>(columns),
                                    cudaMemcpyDeviceToHost, m_stream),
                  "download solutions");
        else
            check(cudaMemcpy2DAsync(out, rowsOf(ldOut), b + (n - t), rowsOf(n), rowsOf(t),
                                    static_cast<std::size_t>(columns), cudaMemcpyDeviceToHost, m_stream),
                  "download condensed loads");
        check(cudaStreamSynchronize(m_stream), "partial solve");
        checkChains();
    }

    // The indefinite factorisation (the reference's PivotingMode::Indefinite), after the common set-up of factorise():
    // the pivoted launches level by level; at the end of each level the host reads the fronts' status and refactorises
    // by the exact path every front whose block path failed its threshold test, every front that delays pivots to its
    // parent, and every front whose children delayed pivots into it (grown by their columns). Then, without delays,
    // the inertia with 2x2 blocks and the maps of the pivot order; with delays, the same on the structure restated in
    // the order the equations were eliminated.
    void factoriseIndefinite(const device::FactorArgs& args, std::int32_t dimension, oosgpu_factor_info* info)
    {
        const auto count = static_cast<std::size_t>(m_plan.supernodeCount);
        const auto n = static_cast<std::size_t>(dimension);
        m_pivoted = false;
        m_singular = false;
        m_factorised = false;
        m_perm.allocate(n, "indefinite: permutation");
        m_inversePerm.allocate(n, "indefinite: inverse permutation");
        m_subdiagonal.allocate(n, "indefinite: 2x2 subdiagonal");
        m_status.allocate(count, "indefinite: status");
        m_stepPerm.allocate(count * 64, "indefinite: block interchanges");
        m_stepSwapped.allocate(count, "indefinite: block interchanged");
        m_w.allocate(static_cast<std::size_t>(std::max<std::int64_t>(m_plan.wValues, 1)), "indefinite: W");
        if (m_wOffset.get() == nullptr)
            m_wOffset.upload(m_plan.wOffset, m_stream, "indefinite: W offsets");
        m_rowsPivot.allocate(static_cast<std::size_t>(std::max<std::int64_t>(m_plan.rowEntries, 1)), "indefinite: rows");
        m_relposPivot.allocate(static_cast<std::size_t>(std::max<std::int64_t>(m_plan.rowEntries, 1)),
                               "indefinite: positions");
        device::PivotArgs pivots{m_perm.get(),        m_subdiagonal.get(), m_status.get(), m_stepPerm.get(),
                                 m_stepSwapped.get(), m_w.get(),           m_wOffset.get()};
        m_exact.clear();
        m_exact.resize(count);
        m_grown.clear();
        m_delayedPivots = 0;
        m_isRestated = false;
        ++m_structureGeneration;
        device::identityPermutation<<<blocksFor(dimension, 256), 256, 0, m_stream>>>(m_perm.get(), dimension);
        check(cudaMemsetAsync(m_subdiagonal.get(), 0, n * sizeof(double), m_stream), "memset");
        check(cudaMemsetAsync(m_status.get(), 0, count * sizeof(std::int32_t), m_stream), "memset");
        check(cudaMemsetAsync(m_stepSwapped.get(), 0, count * sizeof(std::int32_t), m_stream), "memset");
        std::vector<std::int32_t> status(count);
        std::size_t profiled = 0;
        for (const Launch& launch : m_plan.pivotedLaunches)
        {
            const std::int32_t* list = m_lists.get() + launch.offset;
            const device::TileTask* tiles = m_tiles.get() + launch.offset;
            if (m_profile)
                check(cudaEventRecord(profileEvent(2 * profiled), m_stream), "profile event");
            switch (launch.kind)
            {
            case LaunchKind::SmallFrontsPivoted:
            {
                const std::size_t smem = static_cast<std::size_t>(launch.smemOrder) * (launch.smemOrder + 1) * sizeof(double);
                device::smallFrontsPivoted<<<launch.count, SMALL_THREADS, smem, m_stream>>>(args, pivots, list,
                                                                                            m_structureError.get());
                break;
            }
            case LaunchKind::AssembleFronts:
                device::assembleFronts<<<launch.count, 256, 0, m_stream>>>(args, m_pieces.get() + launch.offset,
                                                                           m_structureError.get());
                break;
            case LaunchKind::PivotedDiagonal:
                device::pivotedDiagonal<<<launch.count, 256, 0, m_stream>>>(args, pivots, list, launch.k0);
                break;
            case LaunchKind::PermuteEarlierRows:
                device::permuteEarlierRows<<<launch.count, 256, 0, m_stream>>>(args, pivots, tiles, launch.k0);
                break;
            case LaunchKind::PanelRowsPivoted:
                device::panelRowsPivotedInverse<<<launch.count, device::TILE_THREADS, device::PANEL_ROWS_PIVOTED_SMEM,
                                                  m_stream>>>(args, pivots, tiles, launch.k0);
                break;
            case LaunchKind::UpdatePivoted:
                device::updatePivoted<<<launch.count, device::TILE_THREADS, 0, m_stream>>>(args, pivots, tiles,
                                                                                          launch.k0);
                break;
            case LaunchKind::LevelEnd:
            {
                check(cudaGetLastError(), "indefinite factorisation launch");
                check(cudaMemcpyAsync(status.data(), m_status.get(), count * sizeof(std::int32_t),
                                      cudaMemcpyDeviceToHost, m_stream),
                      "download status");
                check(cudaStreamSynchronize(m_stream), "indefinite factorisation level");
                for (const std::int32_t s : m_plan.frontsOfLevel[static_cast<std::size_t>(launch.k0)])
                    if ((status[static_cast<std::size_t>(s)] & 3) != 0 || receivesDelayed(s))
                        exactFront(args, s);
                break;
            }
            default:
                throw Error(STATUS_INTERNAL, "indefinite plan: an unexpected launch");
            }
            if (m_profile)
                check(cudaEventRecord(profileEvent(2 * profiled + 1), m_stream), "profile event");
            ++profiled;
        }
        check(cudaGetLastError(), "indefinite factorisation launch");
        if (m_delayedPivots == 0)
        {
            invertDiagonalBlocks(args, true);
            device::inertiaPivoted<<<blocksFor(std::max(dimension, 1), 256), 256, 0, m_stream>>>(
                args, pivots, m_supernodeOfColumn.get(), dimension, m_counters.get());
            device::invertPermutation<<<blocksFor(std::max(dimension, 1), 256), 256, 0, m_stream>>>(
                m_perm.get(), m_inversePerm.get(), dimension);
            device::remapPivotOrder<<<std::max(m_plan.supernodeCount, 1), 128, 0, m_stream>>>(
                m_fronts.get(), m_rows.get(), m_relpos.get(), m_inversePerm.get(), m_rowsPivot.get(),
                m_relposPivot.get(), m_plan.supernodeCount);
        }
        else
            restate(args, pivots);
        check(cudaGetLastError(), "indefinite summary launch");
        check(cudaEventRecord(m_stop, m_stream), "event");
        std::vector<unsigned long long> counters(8);
        std::int32_t structureError = 0;
        check(cudaMemcpyAsync(counters.data(), m_counters.get(), 8 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                              m_stream),
              "download counters");
        check(cudaMemcpyAsync(&structureError, m_structureError.get(), sizeof(std::int32_t), cudaMemcpyDeviceToHost,
                              m_stream),
              "download structure check");
        check(cudaStreamSynchronize(m_stream), "indefinite factorisation");
        m_profileValid = m_profile;
        m_profiledPivoted = m_profile;
        float milliseconds = 0.0f;
        check(cudaEventElapsedTime(&milliseconds, m_start, m_stop), "event time");
        if (structureError != NO_PIVOT)
            throw Error(STATUS_INVALID_ARGUMENT,
                        "supernodal factorisation: column " + std::to_string(structureError) +
                            " of the matrix has an entry outside the structure of the symbolic factor; build the CSC in "
                            "the order of the symbolic factor, on the graph it was analysed on");
        oosgpu_factor_info result{};
        result.positive = static_cast<std::int64_t>(counters[0]);
        result.negative = static_cast<std::int64_t>(counters[1]);
        result.zero = static_cast<std::int64_t>(counters[2]);
        result.two_by_two = static_cast<std::int64_t>(counters[3]);
        result.delayed = m_delayedPivots;
        result.equation_of_largest = -1;
        result.device_seconds = milliseconds / 1000.0;
        if (info != nullptr)
            *info = result;
        m_pivoted = true;
        m_singular = result.zero > 0;
        m_factorised = true;
    }

    // The inverses of the diagonal blocks the solves' 64-column steps apply (into the blocks' upper triangles).
    // The inverses of the diagonal blocks the solves apply: the small fronts' always; the large fronts' only after
    // an indefinite factorisation (in positive definite mode diagonalBlocks has written them already).
    void invertDiagonalBlocks(const device::FactorArgs& args, bool largeFronts)
    {
        for (const Launch& launch : m_plan.inverseLaunches)
            device::invertDiagonal<<<launch.count, 64, 0, m_stream>>>(args, m_tiles.get() + launch.offset);
        if (largeFronts)
            for (const Launch& launch : m_plan.inverseLaunchesLarge)
                device::invertDiagonal<<<launch.count, 64, 0, m_stream>>>(args, m_tiles.get() + launch.offset);
        check(cudaGetLastError(), "diagonal inverse launch");
    }

    // Front s received delayed columns from a child.
    [[nodiscard]] bool receivesDelayed(std::int32_t s) const
    {
        const device::FrontDesc& f = m_plan.fronts[static_cast<std::size_t>(s)];
        for (std::int32_t q = 0; q < f.childCount; ++q)
        {
            const ExactOutcome* x = m_exact[static_cast<std::size_t>(m_plan.children[static_cast<std::size_t>(f.childStart + q)])].get();
            if (x != nullptr && x->delayed() > 0)
                return true;
        }
        return false;
    }

    // A grown panel or update matrix of this factorisation (device memory of its own, freed at the next one).
    double* grownBuffer(std::size_t values, const char* what)
    {
        m_grown.push_back(std::make_unique<DeviceArray<double>>());
        m_grown.back()->allocate(values, what);
        return m_grown.back()->get();
    }

    // The exact path of front s (the reference's eliminatePivoted): its candidates are its c columns and the columns
    // its children delayed (children in increasing order); its sources are its children's update matrices, each row
    // at the front position positionsInFront gives it. Bunch-Kaufman by one block leaves `eliminated` pivots; the
    // candidates left are delayed to the parent (a root front cannot delay: an internal error, as in the reference).
    // A front of its symbolic shape (nothing delayed in or out) keeps its panel, update matrix and pivot order where
    // the batched kernels keep them; a grown front's panel goes to a grown buffer; an update matrix with delayed rows
    // goes to a grown buffer, one without to the front's own place (its order is then r).
    void exactFront(const device::FactorArgs& args, std::int32_t s)
    {
        const device::FrontDesc& f = m_plan.fronts[static_cast<std::size_t>(s)];
        std::vector<std::int32_t> delayedIn;
        for (std::int32_t q = 0; q < f.childCount; ++q)
        {
            const ExactOutcome* x = m_exact[static_cast<std::size_t>(m_plan.children[static_cast<std::size_t>(f.childStart + q)])].get();
            if (x != nullptr && x->delayed() > 0)
                delayedIn.insert(delayedIn.end(), x->equations.begin() + x->eliminated,
                                 x->equations.begin() + x->candidates);
        }
        const auto candidates = static_cast<std::int32_t>(f.c + static_cast<std::int64_t>(delayedIn.size()));
        const std::int32_t order = candidates + f.r;
        const bool symbolicShape = delayedIn.empty();
        // the sources: each child's update matrix and the front positions of its rows
        std::vector<device::FrontSource> sources;
        std::vector<std::int32_t> positions;
        std::vector<std::size_t> positionStart;
        std::int32_t delayedStart = f.c;
        for (std::int32_t q = 0; q < f.childCount; ++q)
        {
            const std::int32_t ch = m_plan.children[static_cast<std::size_t>(f.childStart + q)];
            const device::FrontDesc& cf = m_plan.fronts[static_cast<std::size_t>(ch)];
            const ExactOutcome* x = m_exact[static_cast<std::size_t>(ch)].get();
            const std::int32_t* childRows = x != nullptr ? x->equations.data() + x->eliminated
                                                         : m_plan.rows.data() + cf.rowStart;
            const std::int32_t childOrder = x != nullptr ? x->order - x->eliminated : cf.r;
            const std::int32_t childDelayed = x != nullptr ? x->delayed() : 0;
            if (childOrder == 0)
                continue;
            const std::vector<std::int32_t> p =
                positionsInFront(m_plan, s, candidates, childRows, childOrder, childDelayed, delayedStart);
            delayedStart += childDelayed;
            positionStart.push_back(positions.size());
            positions.insert(positions.end(), p.begin(), p.end());
            sources.push_back({x != nullptr ? x->update : m_updates.get() + cf.update, nullptr, childOrder, 0});
        }
        m_exactPositions.upload(positions, m_stream, "exact front: positions");
        for (std::size_t k = 0; k < sources.size(); ++k)
            sources[k].positions = m_exactPositions.get() + positionStart[k];
        m_exactSources.upload(sources, m_stream, "exact front: sources");
        const std::size_t orderSize = static_cast<std::size_t>(order);
        double* panel = symbolicShape ? m_panels.get() + f.panel
                                      : grownBuffer(orderSize * static_cast<std::size_t>(candidates),
                                                    "indefinite: grown panel");
        m_frontWork.allocate(orderSize * orderSize, "indefinite: exact front");
        m_exactPerm.allocate(static_cast<std::size_t>(std::max(candidates, 1)), "exact front: permutation");
        m_exactSub.allocate(static_cast<std::size_t>(std::max(candidates, 1)), "exact front: subdiagonal");
        m_exactCount.allocate(1, "exact front: eliminated");
        const device::ExactFront front{s, order, candidates, static_cast<std::int32_t>(sources.size()),
                                       m_exactSources.get(), panel};
        device::exactFront<<<1, 1024, 0, m_stream>>>(args, front, m_frontWork.get(), m_exactPerm.get(), m_exactSub.get(),
                                                     m_exactCount.get(), m_structureError.get());
        check(cudaGetLastError(), "exact front launch");
        std::vector<std::int32_t> perm(static_cast<std::size_t>(candidates));
        std::vector<double> sub(static_cast<std::size_t>(candidates));
        std::int32_t eliminated = 0;
        if (candidates > 0)
        {
            check(cudaMemcpyAsync(perm.data(), m_exactPerm.get(), perm.size() * sizeof(std::int32_t),
                                  cudaMemcpyDeviceToHost, m_stream),
                  "download exact front");
            check(cudaMemcpyAsync(sub.data(), m_exactSub.get(), sub.size() * sizeof(double), cudaMemcpyDeviceToHost,
                                  m_stream),
                  "download exact front");
        }
        check(cudaMemcpyAsync(&eliminated, m_exactCount.get(), sizeof(std::int32_t), cudaMemcpyDeviceToHost, m_stream),
              "download exact front");
        check(cudaStreamSynchronize(m_stream), "exact front");
        ++m_exactFronts;
        auto out = std::make_unique<ExactOutcome>();
        out->order = order;
        out->candidates = candidates;
        out->eliminated = eliminated;
        // the equation at each front position: the candidates permuted, then R(s)
        std::vector<std::int32_t> origin(orderSize);
        for (std::int32_t j = 0; j < f.c; ++j)
            origin[static_cast<std::size_t>(j)] = f.first + j;
        std::copy(delayedIn.begin(), delayedIn.end(), origin.begin() + f.c);
        std::copy_n(m_plan.rows.data() + f.rowStart, f.r, origin.begin() + candidates);
        out->equations.resize(orderSize);
        for (std::int32_t k = 0; k < order; ++k)
            out->equations[static_cast<std::size_t>(k)] =
                origin[static_cast<std::size_t>(k < candidates ? perm[static_cast<std::size_t>(k)] : k)];
        out->subdiagonal.assign(sub.begin(), sub.begin() + eliminated);
        // the panel's place from the arena's base, in values (a grown panel lies in an allocation of its own, before
        // or after the arena: the kernels reach it as args.panels + offset)
        out->panel = static_cast<std::int64_t>(reinterpret_cast<std::intptr_t>(panel) -
                                               reinterpret_cast<std::intptr_t>(m_panels.get())) /
                     static_cast<std::int64_t>(sizeof(double));
        if (out->delayed() > 0 && f.parent < 0)
            throw Error(STATUS_INTERNAL, "supernodal factorisation: the root front " + std::to_string(s) + " delayed " +
                                             std::to_string(out->delayed()) + " pivots, which a root front cannot do");
        const std::int32_t updateOrder = order - eliminated;
        const bool keepsShape = symbolicShape && out->delayed() == 0;
        if (updateOrder > 0)
        {
            // Without delays out the update matrix has its symbolic order r (a grown front eliminated its delayed
            // columns too): it goes where the parent's batched assembly reads it.
            double* update = out->delayed() == 0 ? m_updates.get() + f.update
                                                 : grownBuffer(static_cast<std::size_t>(updateOrder) * updateOrder,
                                                               "indefinite: grown update matrix");
            const std::int64_t items = static_cast<std::int64_t>(updateOrder) * updateOrder;
            device::copyTrailing<<<blocksFor(items, 256), 256, 0, m_stream>>>(m_frontWork.get(), order, eliminated,
                                                                            updateOrder, update);
            check(cudaGetLastError(), "exact front update launch");
            out->update = update;
        }
        if (keepsShape && f.c > 0)
        {
            // the front's pivot order where the batched kernels keep it
            std::vector<std::int32_t> pivotOrder(static_cast<std::size_t>(f.c));
            for (std::int32_t j = 0; j < f.c; ++j)
                pivotOrder[static_cast<std::size_t>(j)] = f.first + perm[static_cast<std::size_t>(j)];
            check(cudaMemcpyAsync(m_perm.get() + f.first, pivotOrder.data(), pivotOrder.size() * sizeof(std::int32_t),
                                  cudaMemcpyHostToDevice, m_stream),
                  "upload exact front");
            check(cudaMemcpyAsync(m_subdiagonal.get() + f.first, sub.data(), static_cast<std::size_t>(f.c) * sizeof(double),
                                  cudaMemcpyHostToDevice, m_stream),
                  "upload exact front");
        }
        check(cudaStreamSynchronize(m_stream), "exact front");
        m_delayedPivots += out->delayed();
        m_exact[static_cast<std::size_t>(s)] = std::move(out);
    }

    // After a factorisation that delayed pivots: the structure restated in elimination order (restateDelayed), its
    // solve plan and maps on the device, the diagonal inverses of its panels and the inertia counted on it.
    void restate(const device::FactorArgs& args, const device::PivotArgs& pivots)
    {
        const auto n = static_cast<std::size_t>(m_plan.dimension);
        std::vector<std::int32_t> perm(n);
        std::vector<double> sub(n);
        check(cudaMemcpyAsync(perm.data(), m_perm.get(), n * sizeof(std::int32_t), cudaMemcpyDeviceToHost, m_stream),
              "download pivot order");
        check(cudaMemcpyAsync(sub.data(), m_subdiagonal.get(), n * sizeof(double), cudaMemcpyDeviceToHost, m_stream),
              "download subdiagonals");
        check(cudaStreamSynchronize(m_stream), "download pivot order");
        DelayedStructure d = restateDelayed(m_plan, perm, sub, m_exact);
        Restated& r = m_restated;
        r.plan = std::move(d.plan);
        r.perm = std::move(d.perm);
        r.subdiagonal = std::move(d.subdiagonal);
        r.fronts.upload(r.plan.fronts, m_stream, "restated: fronts");
        r.rows.upload(r.plan.rows, m_stream, "restated: rows");
        r.relpos.upload(r.plan.relpos, m_stream, "restated: positions");
        r.gatherStart.upload(r.plan.gatherStart, m_stream, "restated: gather lists");
        r.gatherRows.upload(r.plan.gatherRows, m_stream, "restated: gather lists");
        r.supernodeOfColumn.upload(r.plan.supernodeOfColumn, m_stream, "restated: columns");
        r.lists.upload(r.plan.lists, m_stream, "restated: lists");
        r.tiles.upload(r.plan.tiles, m_stream, "restated: tiles");
        r.devicePerm.upload(r.perm, m_stream, "restated: pivot order");
        r.deviceSubdiagonal.upload(r.subdiagonal, m_stream, "restated: subdiagonals");
        if (r.plan.rowPartialSlots > m_plan.rowPartialSlots)
            m_rowPartials.allocate(static_cast<std::size_t>(r.plan.rowPartialSlots) * device::TILE * device::TILE,
                                   "solve: split products");
        allocateChains(r.plan);
        device::FactorArgs restatedArgs = args;
        restatedArgs.fronts = r.fronts.get();
        for (const std::vector<Launch>* launches : {&r.plan.inverseLaunches, &r.plan.inverseLaunchesLarge})
            for (const Launch& launch : *launches)
                device::invertDiagonal<<<launch.count, 64, 0, m_stream>>>(restatedArgs, r.tiles.get() + launch.offset);
        device::PivotArgs restatedPivots = pivots;
        restatedPivots.subdiagonal = r.deviceSubdiagonal.get();
        restatedPivots.perm = r.devicePerm.get();
        device::inertiaPivoted<<<blocksFor(std::max(m_plan.dimension, 1), 256), 256, 0, m_stream>>>(
            restatedArgs, restatedPivots, r.supernodeOfColumn.get(), m_plan.dimension, m_counters.get());
        check(cudaGetLastError(), "restated structure launch");
        m_isRestated = true;
    }

    void requireSolvable() const
    {
        if (m_isPartial)
            throw Error(STATUS_INVALID_ARGUMENT, "FactorSolve::solve: a partial factor (its trailing supernode is not "
                                                 "eliminated); use condense and recover");
        if (!m_factorised)
            throw Error(STATUS_NOT_FACTORISED, "FactorSolve: no factor (factorise first, or the last one failed)");
        if (m_singular)
            throw Error(STATUS_SINGULAR, "FactorSolve: the factor has a zero pivot (the shifted matrix is singular); "
                                         "move the shift");
        checkChains();
    }

    void solve(double* b, std::int64_t ld, std::int64_t columns, bool onDevice)
    {
        check(cudaSetDevice(m_device), "cudaSetDevice");
        requireSolvable();
        const std::int32_t n = m_plan.dimension;
        if (ld < n || columns < 0)
            throw Error(STATUS_INVALID_ARGUMENT, "FactorSolve::solve: expected " + std::to_string(n) +
                                                     " rows (leading dimension >= rows), found leading dimension " +
                                                     std::to_string(ld));
        if (columns == 0 || n == 0)
            return;
        m_work.allocate(static_cast<std::size_t>(n) * SOLVE_WIDTH, "solve: rows");
        m_updateRows.allocate(updateRowsPerColumn() * SOLVE_WIDTH,
                              "solve: update rows");
        double* deviceB = b;
        if (!onDevice)
            deviceB = rightHandSides(b, ld, columns, "solve: right-hand sides");
        else
            m_prefetch = {}; // a prefetched host B is dropped by any other solve
        const std::int64_t deviceLd = onDevice ? ld : n;
        check(cudaEventRecord(m_start, m_stream), "event");
        for (std::int64_t c0 = 0; c0 < columns; c0 += SOLVE_WIDTH)
        {
            const int width = static_cast<int>(std::min<std::int64_t>(SOLVE_WIDTH, columns - c0));
            const std::int64_t items = static_cast<std::int64_t>(n) * width;
            (void)items;
            rowsIn(deviceB, deviceLd, static_cast<int>(c0), width, m_work.get());
            sweeps(m_work.get(), width);
            rowsOut(m_work.get(), static_cast<int>(c0), width, deviceB, deviceLd);
            check(cudaGetLastError(), "solve launch");
        }
        check(cudaEventRecord(m_stop, m_stream), "event");
        if (!onDevice)
            check(cudaMemcpy2DAsync(b, static_cast<std::size_t>(ld) * sizeof(double), deviceB,
                                    static_cast<std::size_t>(n) * sizeof(double), static_cast<std::size_t>(n) * sizeof(double),
                                    static_cast<std::size_t>(columns), cudaMemcpyDeviceToHost, m_stream),
                  "download solutions");
        check(cudaStreamSynchronize(m_stream), "solve");
        checkChains();
        float milliseconds = 0.0f;
        check(cudaEventElapsedTime(&milliseconds, m_start, m_stop), "event time");
        m_lastSolveSeconds = milliseconds / 1000.0;
    }

    // A column tile of B (columns [c0, c0 + width), leading dimension ld) into rows of x, in pivot order after an
    // indefinite factorisation, scaled by the solve's scale when one is set (a pencil's S).
    // The structure the solves run on: the plan's, in pivot order after an indefinite factorisation, or the
    // restated one after a factorisation that delayed pivots.
    struct SolveView
    {
        const Plan* plan;
        const device::FrontDesc* fronts;
        const std::int32_t* rows;
        const std::int32_t* relpos;
        const std::int64_t* gatherStart;
        const std::int32_t* gatherRows;
        const std::int32_t* supernodeOfColumn;
        const std::int32_t* lists;
        const device::TileTask* tiles;
        const std::int32_t* perm;
        const double* subdiagonal;
    };
    [[nodiscard]] SolveView solveView() const
    {
        if (m_pivoted && m_isRestated)
        {
            const Restated& r = m_restated;
            return {&r.plan,           r.fronts.get(),     r.rows.get(),  r.relpos.get(),      r.gatherStart.get(),
                    r.gatherRows.get(), r.supernodeOfColumn.get(), r.lists.get(), r.tiles.get(), r.devicePerm.get(),
                    r.deviceSubdiagonal.get()};
        }
        return {&m_plan,
                m_fronts.get(),
                m_pivoted ? m_rowsPivot.get() : m_rows.get(),
                m_pivoted ? m_relposPivot.get() : m_relpos.get(),
                m_gatherStart.get(),
                m_gatherRows.get(),
                m_supernodeOfColumn.get(),
                m_lists.get(),
                m_tiles.get(),
                m_perm.get(),
                m_subdiagonal.get()};
    }
    // The update rows of the forward sweep, per right-hand side.
    [[nodiscard]] std::size_t updateRowsPerColumn() const
    {
        return static_cast<std::size_t>(std::max<std::int64_t>(solveView().plan->rowEntries, 1));
    }

    void rowsIn(const double* b, std::int64_t ld, int c0, int width, double* x)
    {
        const std::int32_t n = m_plan.dimension;
        const std::int64_t items = static_cast<std::int64_t>(n) * width;
        if (m_pivoted)
            device::toRowsPivoted<<<blocksFor(items, 256), 256, 0, m_stream>>>(b, ld, c0, width, n, x,
                                                                               solveView().perm, m_solveScale);
        else
            device::toRows<<<dim3(blocksFor(n, 32), blocksFor(width, 32)), dim3(32, 8), 0, m_stream>>>(
                b, ld, c0, width, n, x, m_solveScale);
    }

    // The rows of x back into the column tile of B.
    void rowsOut(const double* x, int c0, int width, double* b, std::int64_t ld)
    {
        const std::int32_t n = m_plan.dimension;
        const std::int64_t items = static_cast<std::int64_t>(n) * width;
        if (m_pivoted)
            device::fromRowsPivoted<<<blocksFor(items, 256), 256, 0, m_stream>>>(x, c0, width, n, b, ld,
                                                                                 solveView().perm, m_solveScale);
        else
            device::fromRows<<<dim3(blocksFor(n, 32), blocksFor(width, 32)), dim3(32, 8), 0, m_stream>>>(
                x, c0, width, n, b, ld, m_solveScale);
    }

    // The three sweeps on a tile of `width` columns stored by rows (n x width) in x (in pivot order after an indefinite
    // factorisation: the maps of rows in pivot order, 2x2 blocks in the diagonal sweep); the update rows of the forward
    // sweep in `updateRows` (the factor's own when null).
    // replay: run the sweeps as a CUDA graph (captured once per buffers and width) unless the launches are profiled;
    // the solve without allocation runs them one by one.
    void sweeps(double* x, int width, double* updateRows = nullptr, bool replay = true)
    {
        const std::int32_t n = m_plan.dimension;
        const std::int64_t items = static_cast<std::int64_t>(n) * width;
        const SolveView view = solveView();
        device::SolveArgs args{view.fronts,
                               m_children.get(),
                               view.rows,
                               view.relpos,
                               m_panels.get(),
                               x,
                               updateRows != nullptr ? updateRows : m_updateRows.get(),
                               width,
                               view.gatherStart,
                               view.gatherRows,
                               // the plan's gather slots are equations, the restated structure's are positions
                               m_pivoted && !m_isRestated ? view.perm : nullptr,
                               n,
                               m_rowPartials.get(),
                               m_chainState.get(),
                               m_chainState.get() + view.plan->chainSlots,
                               m_chainState.get() + (m_chainState.size() - 1),
                               m_chainFailed};
        const auto launches = [&]
        {
            runSweep(args, view, view.plan->forwardLaunches);
            const std::size_t record =
                beginSolveRecord(DIAGONAL_SWEEP_KIND, static_cast<std::int32_t>(blocksFor(items, 256)), 0);
            if (m_pivoted)
                device::diagonalSweepPivoted<<<blocksFor(items, 256), 256, 0, m_stream>>>(
                    args, view.supernodeOfColumn, view.subdiagonal, n);
            else
                device::diagonalSweep<<<blocksFor(items, 256), 256, 0, m_stream>>>(args, m_diagonal.get(), n);
            endSolveRecord(record);
            runSweep(args, view, view.plan->backwardLaunches);
        };
        m_solveRecords.clear();
        if (m_profile || !replay)
            launches();
        else
            m_sweepGraph.run(m_stream,
                             {keyOf(x), keyOf(args.updates), static_cast<std::uintptr_t>(width),
                              static_cast<std::uintptr_t>(m_pivoted),
                              m_pivoted && m_isRestated ? m_structureGeneration : 0},
                             launches);
        m_solveProfileValid = m_profile;
    }

    // The device this factor lives on.
    [[nodiscard]] int deviceOrdinal() const noexcept { return m_device; }

    // The solve of solve(b, ld, columns, true) with its scratch (the rows of a column tile and the update rows of the
    // forward sweep) in the caller's device memory `scratch` of `capacity` values instead of the factor's own
    // buffers: nothing is allocated. The tile is narrowed to what the scratch holds.
    void solveInScratch(double* b, std::int64_t ld, std::int64_t columns, double* scratch, std::size_t capacity)
    {
        check(cudaSetDevice(m_device), "cudaSetDevice");
        const std::int32_t n = m_plan.dimension;
        const std::size_t perColumn = static_cast<std::size_t>(n) + updateRowsPerColumn();
        if (perColumn > capacity)
            throw Error(STATUS_INVALID_ARGUMENT,
                        "solve without allocation: this factor needs " + std::to_string(perColumn) +
                            " scratch values per right-hand side (equations plus update rows), more than the " +
                            std::to_string(capacity) + " of the fixed scratch; use oosgpu_solve_device");
        requireSolvable();
        if (ld < n || columns < 0)
            throw Error(STATUS_INVALID_ARGUMENT, "FactorSolve::solve: expected " + std::to_string(n) +
                                                     " rows (leading dimension >= rows), found leading dimension " +
                                                     std::to_string(ld));
        if (columns == 0 || n == 0)
            return;
        const int width = static_cast<int>(std::min<std::size_t>(SOLVE_WIDTH, capacity / perColumn));
        double* work = scratch;
        double* updateRows = scratch + static_cast<std::size_t>(n) * static_cast<std::size_t>(width);
        check(cudaEventRecord(m_start, m_stream), "event");
        for (std::int64_t c0 = 0; c0 < columns; c0 += width)
        {
            const int tileWidth = static_cast<int>(std::min<std::int64_t>(width, columns - c0));
            const std::int64_t items = static_cast<std::int64_t>(n) * tileWidth;
            (void)items;
            rowsIn(b, ld, static_cast<int>(c0), tileWidth, work);
            sweeps(work, tileWidth, updateRows, false);
            rowsOut(work, static_cast<int>(c0), tileWidth, b, ld);
            check(cudaGetLastError(), "solve launch");
        }
        check(cudaEventRecord(m_stop, m_stream), "event");
        check(cudaStreamSynchronize(m_stream), "solve");
        checkChains();
        float milliseconds = 0.0f;
        check(cudaEventElapsedTime(&milliseconds, m_start, m_stop), "event time");
        m_lastSolveSeconds = milliseconds / 1000.0;
    }

    // The full symmetric pattern of the factorised matrix (both triangles, rows ascending), for the residuals: built
    // once on the host from the matrix's structure, each term pointing at its value in the lower CSC.
    void ensureFullPattern()
    {
        if (m_fullTerms == m_matrixTerms && m_fullStart.get() != nullptr)
            return;
        const std::int32_t n = m_plan.dimension;
        std::vector<std::int64_t> offsets(static_cast<std::size_t>(n) + 1);
        std::vector<std::int32_t> rows(static_cast<std::size_t>(m_matrixTerms));
        check(cudaMemcpy(offsets.data(), m_matrixOffsets, offsets.size() * sizeof(std::int64_t), cudaMemcpyDeviceToHost),
              "download offsets");
        check(cudaMemcpy(rows.data(), m_matrixRows, rows.size() * sizeof(std::int32_t), cudaMemcpyDeviceToHost),
              "download rows");
        if (m_matrixTerms > INT32_MAX)
            throw Error(STATUS_INVALID_ARGUMENT, "refinement: more than 2^31 matrix terms");
        std::vector<std::int64_t> start(static_cast<std::size_t>(n) + 1, 0);
        for (std::int32_t j = 0; j < n; ++j)
            for (std::int64_t k = offsets[static_cast<std::size_t>(j)]; k < offsets[static_cast<std::size_t>(j) + 1]; ++k)
            {
                const std::int32_t i = rows[static_cast<std::size_t>(k)];
                ++start[static_cast<std::size_t>(i) + 1]; // (i, j) in row i
                if (i != j)
                    ++start[static_cast<std::size_t>(j) + 1]; // (j, i) in row j
            }
        for (std::int32_t i = 0; i < n; ++i)
            start[static_cast<std::size_t>(i) + 1] += start[static_cast<std::size_t>(i)];
        std::vector<std::int32_t> columns(static_cast<std::size_t>(start[static_cast<std::size_t>(n)]));
        std::vector<std::int32_t> source(columns.size());
        std::vector<std::int64_t> next(start.begin(), start.end() - 1);
        // Row i: the terms (i, j), j < i, from the columns j < i in increasing j, then column i's own terms.
        for (std::int32_t j = 0; j < n; ++j)
        {
            for (std::int64_t k = offsets[static_cast<std::size_t>(j)]; k < offsets[static_cast<std::size_t>(j) + 1]; ++k)
            {
                const std::int32_t i = rows[static_cast<std::size_t>(k)];
                if (i == j)
                    continue;
                const auto at = static_cast<std::size_t>(next[static_cast<std::size_t>(i)]++);
                columns[at] = j;
                source[at] = static_cast<std::int32_t>(k);
            }
            for (std::int64_t k = offsets[static_cast<std::size_t>(j)]; k < offsets[static_cast<std::size_t>(j) + 1]; ++k)
            {
                const auto at = static_cast<std::size_t>(next[static_cast<std::size_t>(j)]++);
                columns[at] = rows[static_cast<std::size_t>(k)];
                source[at] = static_cast<std::int32_t>(k);
            }
        }
        // Groups of consecutive rows with the same columns (a node's DOFs), at most RESIDUAL_GROUP rows each.
        std::vector<std::int32_t> groupFirst;
        groupFirst.reserve(static_cast<std::size_t>(n) + 1);
        for (std::int32_t i = 0; i < n;)
        {
            groupFirst.push_back(i);
            const std::int64_t begin = start[static_cast<std::size_t>(i)];
            const std::int64_t length = start[static_cast<std::size_t>(i) + 1] - begin;
            std::int32_t next = i + 1;
            while (next < n && next - i < device::RESIDUAL_GROUP &&
                   start[static_cast<std::size_t>(next) + 1] - start[static_cast<std::size_t>(next)] == length &&
                   std::equal(columns.begin() + begin, columns.begin() + begin + length,
                              columns.begin() + start[static_cast<std::size_t>(next)]))
                ++next;
            i = next;
        }
        groupFirst.push_back(n);
        m_residualGroups = static_cast<std::int32_t>(groupFirst.size()) - 1;
        m_fullStart.upload(start, m_stream, "refinement: pattern");
        m_fullColumns.upload(columns, m_stream, "refinement: pattern");
        m_fullSource.upload(source, m_stream, "refinement: pattern");
        m_groupFirst.upload(groupFirst, m_stream, "refinement: pattern");
        check(cudaStreamSynchronize(m_stream), "refinement pattern");
        m_fullTerms = m_matrixTerms;
    }

    // X = A^-1 B refined in FP64 until every column's normwise backward error ||b - A x||_inf / (||A||_inf ||x||_inf +
    // ||b||_inf) is at most `tolerance` or maxSteps corrections were made; B and X column-major (host or device).
    // Per-column inner products of `vectors` row blocks v_i (stride values apart) with w: out[i * width + c].
    void dotRows(const double* v, std::int64_t stride, int vectors, const double* w, int width, std::vector<double>& out)
    {
        const std::int32_t n = m_plan.dimension;
        const int blocks = std::clamp((n + 1023) / 1024, 1, 592);
        const int rowsPerBlock = (n + blocks - 1) / blocks;
        const std::size_t count = static_cast<std::size_t>(vectors) * static_cast<std::size_t>(width);
        m_gmresPartials.allocate(count * static_cast<std::size_t>(blocks), "refinement: partial sums");
        m_gmresValues.allocate(static_cast<std::size_t>(device::GMRES_MAX_VECTORS) * 64, "refinement: coefficients");
        device::dotRowsPartials<<<blocks, 256, 0, m_stream>>>(v, stride, vectors, w, width, n, rowsPerBlock,
                                                               m_gmresPartials.get());
        device::reducePartials<<<blocksFor(static_cast<std::int64_t>(count), 128), 128, 0, m_stream>>>(
            m_gmresPartials.get(), blocks, static_cast<int>(count), m_gmresValues.get());
        check(cudaGetLastError(), "refinement inner products");
        out.resize(count);
        check(cudaMemcpyAsync(out.data(), m_gmresValues.get(), count * sizeof(double), cudaMemcpyDeviceToHost, m_stream),
              "download inner products");
        check(cudaStreamSynchronize(m_stream), "refinement inner products");
    }

    // Uploads per-column coefficients (vectors x width) for the combination kernels.
    const double* uploadCoefficients(const std::vector<double>& values)
    {
        m_gmresCoefficients.allocate(static_cast<std::size_t>(device::GMRES_MAX_VECTORS) * 64,
                                     "refinement: coefficients");
        check(cudaMemcpyAsync(m_gmresCoefficients.get(), values.data(), values.size() * sizeof(double),
                              cudaMemcpyHostToDevice, m_stream),
              "upload coefficients");
        check(cudaStreamSynchronize(m_stream), "upload coefficients");
        return m_gmresCoefficients.get();
    }

    // One GMRES correction of the tile in x (rows, `width` columns), the residual b - A x in m_rRows: each column's
    // system M^-1 A d = M^-1 r (M^-1 the factor's solve) by GMRES with at most `krylov` vectors, the basis
    // orthogonalised by classical Gram-Schmidt twice, the Hessenberg matrix reduced by Givens rotations on the host;
    // it ends when every column's preconditioned residual has fallen by innerTolerance, then x += V y.
    void gmresCorrection(double* x, int width, int krylov, double innerTolerance)
    {
        const std::int32_t n = m_plan.dimension;
        const std::int64_t items = static_cast<std::int64_t>(n) * width;
        const std::int64_t stride = items;
        const auto w = static_cast<std::size_t>(width);
        const auto m = static_cast<std::size_t>(krylov);
        m_krylov.allocate(static_cast<std::size_t>(krylov + 1) * static_cast<std::size_t>(items), "refinement: Krylov");
        double* basis = m_krylov.get();
        const unsigned elementBlocks = blocksFor(items, 256);
        check(cudaMemcpyAsync(basis, m_rRows.get(), static_cast<std::size_t>(items) * sizeof(double),
                              cudaMemcpyDeviceToDevice, m_stream),
              "copy residual");
        sweeps(basis, width);
        std::vector<double> values;
        dotRows(basis, stride, 1, basis, width, values);
        std::vector<double> beta(w);
        std::vector<double> inverse(w);
        for (std::size_t c = 0; c < w; ++c)
        {
            beta[c] = std::sqrt(std::max(values[c], 0.0));
            inverse[c] = beta[c] > 0.0 ? 1.0 / beta[c] : 0.0;
        }
        device::scaleRowsColumns<<<elementBlocks, 256, 0, m_stream>>>(basis, basis, uploadCoefficients(inverse), width,
                                                                       items);
        // Per column: H (m + 1) x m by columns, the rotations, the rotated right-hand side g.
        std::vector<double> h(w * (m + 1) * m, 0.0);
        std::vector<double> cs(w * m, 0.0);
        std::vector<double> sn(w * m, 0.0);
        std::vector<double> g(w * (m + 1), 0.0);
        const auto H = [&](std::size_t c, std::size_t i, std::size_t j) -> double& { return h[(c * m + j) * (m + 1) + i]; };
        for (std::size_t c = 0; c < w; ++c)
            g[c * (m + 1)] = beta[c];
        std::size_t used = 0;
        constexpr int WARPS = 8;
        const unsigned rowBlocks = std::min<unsigned>(blocksFor(n, WARPS), 148u * 8u);
        for (std::size_t j = 0; j < m; ++j)
        {
            double* vj = basis + static_cast<std::int64_t>(j) * stride;
            double* next = basis + static_cast<std::int64_t>(j + 1) * stride;
            device::multiplyRows<<<rowBlocks, 32 * WARPS, 0, m_stream>>>(m_fullStart.get(), m_fullColumns.get(),
                                                                         m_fullSource.get(), m_matrixValues, vj, next,
                                                                         width, n);
            sweeps(next, width);
            for (int pass = 0; pass < 2; ++pass)
            {
                dotRows(basis, stride, static_cast<int>(j + 1), next, width, values);
                device::subtractRowsCombination<<<elementBlocks, 256, 0, m_stream>>>(
                    next, basis, stride, static_cast<int>(j + 1), uploadCoefficients(values), width, items);
                for (std::size_t i = 0; i <= j; ++i)
                    for (std::size_t c = 0; c < w; ++c)
                        H(c, i, j) += values[i * w + c];
            }
            dotRows(next, stride, 1, next, width, values);
            for (std::size_t c = 0; c < w; ++c)
            {
                const double norm = std::sqrt(std::max(values[c], 0.0));
                H(c, j + 1, j) = norm;
                inverse[c] = norm > 0.0 ? 1.0 / norm : 0.0;
            }
            device::scaleRowsColumns<<<elementBlocks, 256, 0, m_stream>>>(next, next, uploadCoefficients(inverse),
                                                                           width, items);
            used = j + 1;
            double worst = 0.0;
            for (std::size_t c = 0; c < w; ++c)
            {
                for (std::size_t i = 0; i < j; ++i)
                {
                    const double t = cs[c * m + i] * H(c, i, j) + sn[c * m + i] * H(c, i + 1, j);
                    H(c, i + 1, j) = -sn[c * m + i] * H(c, i, j) + cs[c * m + i] * H(c, i + 1, j);
                    H(c, i, j) = t;
                }
                const double a = H(c, j, j);
                const double b = H(c, j + 1, j);
                const double r = std::hypot(a, b);
                cs[c * m + j] = r > 0.0 ? a / r : 1.0;
                sn[c * m + j] = r > 0.0 ? b / r : 0.0;
                H(c, j, j) = r;
                H(c, j + 1, j) = 0.0;
                g[c * (m + 1) + j + 1] = -sn[c * m + j] * g[c * (m + 1) + j];
                g[c * (m + 1) + j] = cs[c * m + j] * g[c * (m + 1) + j];
                if (beta[c] > 0.0)
                    worst = std::max(worst, std::abs(g[c * (m + 1) + j + 1]) / beta[c]);
            }
            if (worst <= innerTolerance)
                break;
        }
        // y from the triangular H, then x += V y.
        std::vector<double> y(used * w, 0.0);
        for (std::size_t c = 0; c < w; ++c)
            for (std::size_t i = used; i-- > 0;)
            {
                double sum = g[c * (m + 1) + i];
                for (std::size_t q = i + 1; q < used; ++q)
                    sum -= H(c, i, q) * y[q * w + c];
                y[i * w + c] = H(c, i, i) != 0.0 ? sum / H(c, i, i) : 0.0;
            }
        device::addRowsCombination<<<elementBlocks, 256, 0, m_stream>>>(x, basis, stride, static_cast<int>(used),
                                                                         uploadCoefficients(y), width, items);
        check(cudaGetLastError(), "GMRES correction");
    }

    void solveRefined(const double* b, std::int64_t ldb, double* x, std::int64_t ldx, std::int64_t columns,
                      bool onDevice, double tolerance, int maxSteps, oosgpu_refine_info* info, int krylov = 0)
    {
        check(cudaSetDevice(m_device), "cudaSetDevice");
        requireSolvable();
        const std::int32_t n = m_plan.dimension;
        if (ldb < n || ldx < n || columns < 0 || maxSteps < 0)
            throw Error(STATUS_INVALID_ARGUMENT, "refinement: leading dimensions below the rows, or negative counts");
        if (krylov < 0 || krylov > device::GMRES_MAX_VECTORS)
            throw Error(STATUS_INVALID_ARGUMENT, "refinement: the Krylov vectors of a GMRES correction must be in [0, " +
                                                     std::to_string(device::GMRES_MAX_VECTORS) + "], found " +
                                                     std::to_string(krylov));
        oosgpu_refine_info result{};
        if (columns == 0 || n == 0)
        {
            if (info != nullptr)
                *info = result;
            return;
        }
        ensureFullPattern();
        const std::size_t tile = static_cast<std::size_t>(n) * SOLVE_WIDTH;
        m_work.allocate(tile, "solve: rows");
        m_bRows.allocate(tile, "refinement: right-hand side rows");
        m_rRows.allocate(tile, "refinement: residual rows");
        m_norms.allocate(384, "refinement: norms");
        m_updateRows.allocate(updateRowsPerColumn() * SOLVE_WIDTH,
                              "solve: update rows");
        const double* deviceB = b;
        double* deviceX = x;
        std::int64_t dLdb = ldb;
        std::int64_t dLdx = ldx;
        if (!onDevice)
        {
            m_hostX.allocate(static_cast<std::size_t>(n) * static_cast<std::size_t>(columns), "refinement: X");
            deviceB = rightHandSides(b, ldb, columns, "refinement: B");
            deviceX = m_hostX.get();
            dLdb = n;
            dLdx = n;
        }
        else
            m_prefetch = {}; // a prefetched host B is dropped by any other solve
        check(cudaEventRecord(m_start, m_stream), "event");
        std::vector<double> norms(384);
        for (std::int64_t c0 = 0; c0 < columns; c0 += SOLVE_WIDTH)
        {
            const int width = static_cast<int>(std::min<std::int64_t>(SOLVE_WIDTH, columns - c0));
            const std::int64_t items = static_cast<std::int64_t>(n) * width;
            rowsIn(deviceB, dLdb, static_cast<int>(c0), width, m_bRows.get());
            check(cudaMemcpyAsync(m_work.get(), m_bRows.get(), static_cast<std::size_t>(items) * sizeof(double),
                                  cudaMemcpyDeviceToDevice, m_stream),
                  "copy right-hand sides");
            sweeps(m_work.get(), width);
            for (int step = 0;; ++step)
            {
                check(cudaMemsetAsync(m_norms.get(), 0, 384 * sizeof(double), m_stream), "memset");
                constexpr int WARPS = 8;
                // A grid of a few blocks per SM: each warp strides over the rows, its norms flushed once.
                const unsigned residualBlocks = std::min<unsigned>(blocksFor(m_residualGroups, WARPS), 148u * 8u);
                device::residualRows<<<residualBlocks, 32 * WARPS, 0, m_stream>>>(
                    m_fullStart.get(), m_fullColumns.get(), m_fullSource.get(), m_groupFirst.get(), m_residualGroups,
                    m_matrixValues, m_bRows.get(), m_work.get(), m_rRows.get(), width, m_norms.get());
                check(cudaMemcpyAsync(norms.data(), m_norms.get(), 384 * sizeof(double), cudaMemcpyDeviceToHost,
                                      m_stream),
                      "download norms");
                check(cudaStreamSynchronize(m_stream), "refinement residual");
                // The normwise backward error of each column decides; the relative residual is reported.
                double worst = 0.0;
                double worstResidual = 0.0;
                const double normA = norms[320];
                for (int c = 0; c < width; ++c)
                {
                    const auto at = static_cast<std::size_t>(c);
                    const double denominator = normA * norms[256 + at] + norms[192 + at];
                    worst = std::max(worst, denominator > 0.0 ? norms[128 + at] / denominator : norms[128 + at]);
                    worstResidual = std::max(worstResidual, norms[64 + at] > 0.0 ? std::sqrt(norms[at] / norms[64 + at])
                                                                                 : std::sqrt(norms[at]));
                }
                if (worst <= tolerance || step >= maxSteps)
                {
                    result.steps = std::max(result.steps, step);
                    result.residual = std::max(result.residual, worstResidual);
                    result.backward_error = std::max(result.backward_error, worst);
                    break;
                }
                if (krylov > 0)
                {
                    gmresCorrection(m_work.get(), width, krylov, GMRES_INNER_TOLERANCE);
                    continue;
                }
                sweeps(m_rRows.get(), width);
                device::addRows<<<blocksFor(items, 256), 256, 0, m_stream>>>(m_work.get(), m_rRows.get(), items);
            }
            rowsOut(m_work.get(), static_cast<int>(c0), width, deviceX, dLdx);
            check(cudaGetLastError(), "refinement launch");
        }
        check(cudaEventRecord(m_stop, m_stream), "event");
        if (!onDevice)
            check(cudaMemcpy2DAsync(x, static_cast<std::size_t>(ldx) * sizeof(double), deviceX,
                                    static_cast<std::size_t>(n) * sizeof(double), static_cast<std::size_t>(n) * sizeof(double),
                                    static_cast<std::size_t>(columns), cudaMemcpyDeviceToHost, m_stream),
                  "download solutions");
        check(cudaStreamSynchronize(m_stream), "refinement");
        float milliseconds = 0.0f;
        check(cudaEventElapsedTime(&milliseconds, m_start, m_stop), "event time");
        result.device_seconds = milliseconds / 1000.0;
        m_lastSolveSeconds = result.device_seconds;
        if (info != nullptr)
            *info = result;
    }

    void panel(std::int32_t s, std::int64_t* eliminated, std::int64_t* rowCount, double* values, std::int32_t* rows,
               double* subdiagonal)
    {
        check(cudaSetDevice(m_device), "cudaSetDevice");
        if (s < 0 || s >= m_plan.supernodeCount)
            throw Error(STATUS_INVALID_ARGUMENT, "panel: supernode out of range");
        if (!m_factorised)
            throw Error(STATUS_NOT_FACTORISED, "panel: no factor");
        // After a factorisation that delayed pivots, the panel of the restated structure: its eliminated columns over
        // its front's rows (eliminated and delayed candidates, then R(s)), as the reference's grown panels.
        const bool restated = m_pivoted && m_isRestated;
        const device::FrontDesc& f = (restated ? m_restated.plan.fronts : m_plan.fronts)[static_cast<std::size_t>(s)];
        const std::int64_t n = f.c + f.r;
        *eliminated = f.c;
        *rowCount = n;
        if (values != nullptr)
        {
            check(cudaMemcpy(values, m_panels.get() + f.panel, static_cast<std::size_t>(n * f.c) * sizeof(double),
                             cudaMemcpyDeviceToHost),
                  "download panel");
            // The strict upper triangle holds the solves' diagonal inverses, not the factor.
            for (std::int64_t j = 0; j < f.c; ++j)
                std::fill_n(values + j * n, j, 0.0);
        }
        // The row equations in pivot order and the 2x2 subdiagonals (positive definite: the natural order, zeros).
        std::vector<std::int32_t> pivotOrder(static_cast<std::size_t>(f.c));
        std::vector<double> sub(static_cast<std::size_t>(f.c), 0.0);
        if (restated)
        {
            for (std::int32_t k = 0; k < f.c; ++k)
            {
                pivotOrder[static_cast<std::size_t>(k)] = m_restated.perm[static_cast<std::size_t>(f.first + k)];
                sub[static_cast<std::size_t>(k)] = m_restated.subdiagonal[static_cast<std::size_t>(f.first + k)];
            }
        }
        else if (m_pivoted && f.c > 0)
        {
            check(cudaMemcpy(pivotOrder.data(), m_perm.get() + f.first, pivotOrder.size() * sizeof(std::int32_t),
                             cudaMemcpyDeviceToHost),
                  "download pivot order");
            check(cudaMemcpy(sub.data(), m_subdiagonal.get() + f.first, sub.size() * sizeof(double),
                             cudaMemcpyDeviceToHost),
                  "download subdiagonals");
        }
        else
            for (std::int32_t k = 0; k < f.c; ++k)
                pivotOrder[static_cast<std::size_t>(k)] = f.first + k;
        if (rows != nullptr)
        {
            std::copy(pivotOrder.begin(), pivotOrder.end(), rows);
            for (std::int32_t k = 0; k < f.r; ++k)
            {
                const std::int32_t row = (restated ? m_restated.plan.rows : m_plan.rows)[static_cast<std::size_t>(f.rowStart + k)];
                rows[f.c + k] = restated ? m_restated.perm[static_cast<std::size_t>(row)] : row;
            }
        }
        if (subdiagonal != nullptr)
            std::copy(sub.begin(), sub.end(), subdiagonal);
    }

    [[nodiscard]] double lastSolveSeconds() const noexcept { return m_lastSolveSeconds; }

    // Profiling: each factorisation launch bracketed by events; after a factorisation, the device time, launches,
    // algorithmic flops and bytes of each launch kind of it.
    void setProfile(bool enable) { m_profile = enable; }

    // The autotuner. Some launch kinds have more than one kernel (Launch::variant): the diagonal blocks by 16-column
    // sub-panels or column by column, the extend-add element-wise or staged in shared memory, the update matrix by
    // 64 x 64 tiles or by TMA-fed 128 x 128 tiles. Which is faster depends
    // on the launch: how many fronts share it, how large they are. On the first positive definite factorisation of
    // this factor (tuning on, FP64), the whole factorisation runs twice per variant, every launch timed by events on
    // the stream; for each launch kind and size class (blocks in the launch: 1, up to 8, up to 148, up to 592, more)
    // the variant with the smaller total time wins, and every launch of that class takes it from then on. Each of
    // those factorisations is a complete, correct one (the variants compute the same factor to rounding); the
    // factorisation that follows, with the chosen variants, is the one the caller gets. Graphs are recorded after
    // the choice.
    // mode 0: the plan's defaults; 1: tune on the next positive definite FP64 factorisation; 2: the alternative
    // kernel of every tunable launch (the staged extend-add, the column-by-column diagonal blocks, the TMA-fed
    // update tiles).
    void setTuning(int mode)
    {
        if (mode < 0 || mode > 2)
            throw Error(STATUS_INVALID_ARGUMENT, "kernel choice: mode must be 0 (defaults), 1 (autotune) or 2 "
                                                 "(alternatives), found " + std::to_string(mode));
        resetVariants();
        m_tuning = mode == 1;
        if (mode == 2)
            for (Launch& launch : m_plan.factorLaunches)
                if (tunable(launch))
                    launch.variant = 1 - defaultVariant(launch);
    }

    struct TuneRecord
    {
        std::int32_t kind = 0;
        std::int32_t sizeClass = 0;
        std::int32_t launches = 0;
        double seconds[2] = {0.0, 0.0};
        std::int32_t chosen = 0;
    };
    [[nodiscard]] const std::vector<TuneRecord>& tuneReport() const noexcept { return m_tuneReport; }

    // The scale every solve applies to its right-hand sides and its solutions (a pencil's S: X <- S A^-1 S B); null
    // for none. Device memory, dimension values, owned by the caller.
    void setSolveScale(const double* scale) { m_solveScale = scale; }

    // Y = A X with A of the last factorisation's structure and the given values (its lower CSC's terms), X and Y
    // column-major device blocks of `width` columns.
    // The device structure (lower CSC offsets and rows) of the matrices later factorisations and symmetric products
    // use, before any factorisation (the pencil's products with a coupled mass).
    void useStructure(const std::int64_t* offsets, const std::int32_t* rows, std::int64_t terms)
    {
        m_matrixOffsets = offsets;
        m_matrixRows = rows;
        m_matrixTerms = terms;
    }

    void multiplySymmetric(const double* values, const double* x, std::int64_t ldx, double* y, std::int64_t ldy,
                           int width)
    {
        check(cudaSetDevice(m_device), "cudaSetDevice");
        if (m_matrixOffsets == nullptr)
            throw Error(STATUS_NOT_FACTORISED, "symmetric product: no matrix structure yet (factorise first)");
        ensureFullPattern();
        const std::int32_t n = m_plan.dimension;
        constexpr int WARPS = 8;
        device::symmetricProduct<<<blocksFor(n, WARPS), 32 * WARPS, 0, m_stream>>>(
            m_fullStart.get(), m_fullColumns.get(), m_fullSource.get(), values, x, ldx, y, ldy, n, width);
        check(cudaGetLastError(), "symmetric product launch");
    }

    [[nodiscard]] std::int64_t exactFronts() const noexcept { return m_exactFronts; }
    void kernelStats(int kinds, double* seconds, std::int64_t* launches, double* flops, double* bytes)
    {
        check(cudaSetDevice(m_device), "cudaSetDevice");
        for (int k = 0; k < kinds; ++k)
        {
            seconds[k] = 0.0;
            launches[k] = 0;
            flops[k] = 0.0;
            bytes[k] = 0.0;
        }
        if (!m_profileValid)
            throw Error(STATUS_NOT_FACTORISED, "kernel statistics: no profiled factorisation");
        const std::vector<Launch>& profiledLaunches = m_profiledPivoted ? m_plan.pivotedLaunches : m_plan.factorLaunches;
        for (std::size_t index = 0; index < profiledLaunches.size(); ++index)
        {
            const Launch& launch = profiledLaunches[index];
            const int kind = static_cast<int>(launch.kind);
            if (kind >= kinds)
                continue;
            float ms = 0.0f;
            check(cudaEventElapsedTime(&ms, m_profileEvents[2 * index], m_profileEvents[2 * index + 1]), "profile time");
            seconds[kind] += ms / 1000.0;
            launches[kind] += 1;
            flops[kind] += launch.flops;
            bytes[kind] += launch.bytes;
        }
    }
    // The launches of the last profiled factorisation (which 0) or solve sweeps (which 1): kind, blocks, first
    // column of the step and device seconds; returns how many there are (at most `capacity` written).
    std::int64_t launchProfile(int which, std::int64_t capacity, std::int32_t* kinds, std::int32_t* counts,
                               std::int32_t* k0, double* seconds)
    {
        check(cudaSetDevice(m_device), "cudaSetDevice");
        check(cudaStreamSynchronize(m_stream), "profile");
        const bool factor = which == 0;
        if (factor ? !m_profileValid : !m_solveProfileValid)
            throw Error(STATUS_NOT_FACTORISED, factor ? "launch profile: no profiled factorisation"
                                                      : "launch profile: no profiled solve");
        const std::vector<Launch>& profiledLaunches = m_profiledPivoted ? m_plan.pivotedLaunches : m_plan.factorLaunches;
        const std::size_t total = factor ? profiledLaunches.size() : m_solveRecords.size();
        for (std::size_t index = 0; index < total && static_cast<std::int64_t>(index) < capacity; ++index)
        {
            float ms = 0.0f;
            if (factor)
            {
                const Launch& launch = profiledLaunches[index];
                kinds[index] = static_cast<std::int32_t>(launch.kind);
                counts[index] = blocksLaunched(launch);
                k0[index] = launch.k0;
                check(cudaEventElapsedTime(&ms, m_profileEvents[2 * index], m_profileEvents[2 * index + 1]),
                      "profile time");
            }
            else
            {
                kinds[index] = m_solveRecords[index].kind;
                counts[index] = m_solveRecords[index].count;
                k0[index] = m_solveRecords[index].k0;
                check(cudaEventElapsedTime(&ms, m_solveEvents[2 * index], m_solveEvents[2 * index + 1]),
                      "profile time");
            }
            seconds[index] = ms / 1000.0;
        }
        return static_cast<std::int64_t>(total);
    }
    [[nodiscard]] std::int64_t factorLaunchCount() const noexcept
    {
        // the plan's launches, the diagonal inverses, the pivot summary and the gathered diagonal
        return static_cast<std::int64_t>(m_plan.factorLaunches.size() + m_plan.inverseLaunches.size()) + 2;
    }
    [[nodiscard]] std::int64_t solveLaunchCount(std::int64_t columns) const noexcept
    {
        const std::int64_t tiles = (columns + SOLVE_WIDTH - 1) / SOLVE_WIDTH;
        const Plan& plan = *solveView().plan;
        return tiles * (static_cast<std::int64_t>(plan.forwardLaunches.size() + plan.backwardLaunches.size()) + 3);
    }

private:
    // The tensor maps of the TMA-fed update-matrix kernel, one per front of Plan::tmaFronts: the front's panel as rows
    // (contiguous, n of them) by its c columns, 16 x 16 boxes, the 128-byte swizzle, zeros outside. Built once per
    // panel arena.
    void buildTensorMaps()
    {
        if (m_plan.tmaFronts.empty() || m_mapsOf == m_panels.get())
            return;
        std::vector<CUtensorMap> maps(m_plan.tmaFronts.size());
        const EncodeTiled encode = tensorMapEncoder();
        for (std::size_t k = 0; k < maps.size(); ++k)
        {
            const device::FrontDesc& f = m_plan.fronts[static_cast<std::size_t>(m_plan.tmaFronts[k])];
            const std::uint64_t n = static_cast<std::uint64_t>(f.c) + static_cast<std::uint64_t>(f.r);
            const cuuint64_t dims[2] = {n, static_cast<cuuint64_t>(f.c)};
            const cuuint64_t strides[1] = {n * sizeof(double)};
            const cuuint32_t box[2] = {16, 16};
            const cuuint32_t elementStrides[2] = {1, 1};
            const CUresult result =
                encode(&maps[k], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, m_panels.get() + f.panel, dims, strides, box,
                       elementStrides, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                       CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            if (result != CUDA_SUCCESS)
                throw Error(STATUS_CUDA, "tensor map of front " + std::to_string(m_plan.tmaFronts[k]) + ": error " +
                                             std::to_string(static_cast<int>(result)));
        }
        m_tensorMaps.upload(maps, m_stream, "factor: tensor maps");
        check(cudaStreamSynchronize(m_stream), "tensor maps");
        m_mapsOf = m_panels.get();
    }

    static bool tunable(const Launch& launch)
    {
        return launch.kind == LaunchKind::DiagonalBlocks ||
               ((launch.kind == LaunchKind::AssembleFronts || launch.kind == LaunchKind::UpdateMatrix) &&
                launch.altCount > 0);
    }

    // The kernel a launch runs untuned: the element-wise extend-add (on the 2 M plate 10.5 ms against the staged
    // one's 23.6), the diagonal blocks by sub-panels, the 64 x 64 update tiles (27.1 ms against the TMA-fed 128 x 128
    // tiles' 38.1).
    static std::int32_t defaultVariant(const Launch&) { return 0; }

    // The blocks a launch runs with its current kernel (some variants run their alternative task range).
    static std::int32_t blocksLaunched(const Launch& launch)
    {
        return launch.variant == 1 && launch.altCount > 0 ? launch.altCount : launch.count;
    }

    static std::int32_t sizeClass(std::int32_t blocks)
    {
        return blocks <= 1 ? 0 : blocks <= 8 ? 1 : blocks <= 148 ? 2 : blocks <= 592 ? 3 : 4;
    }

    // The untuned choices (every tunable launch on variant 0).
    void resetVariants()
    {
        for (Launch& launch : m_plan.factorLaunches)
            if (tunable(launch))
                launch.variant = defaultVariant(launch);
        m_factorGraph.reset();
        m_tuned = false;
        m_tuneReport.clear();
    }

    // The tuner's choices for one structure on one device, kept for the process: a new factor of the same structure
    // (a fresh pencil of the same model) takes them without timing again.
    using TuneKey = std::tuple<int, std::int32_t, std::int32_t, std::int64_t, std::size_t>;
    static std::map<TuneKey, std::vector<TuneRecord>>& tuneCache(std::mutex*& lock)
    {
        static std::mutex mutex;
        static auto* cache = new std::map<TuneKey, std::vector<TuneRecord>>();
        lock = &mutex;
        return *cache;
    }
    [[nodiscard]] TuneKey tuneKey() const
    {
        return {m_device, m_plan.dimension, m_plan.supernodeCount, m_plan.panelValues, m_plan.factorLaunches.size()};
    }

    template <typename Launches> void tune(const Launches& launches)
    {
        constexpr int VARIANTS = 2;
        const std::size_t count = m_plan.factorLaunches.size();
        m_tuneReport.clear();
        if (std::none_of(m_plan.factorLaunches.begin(), m_plan.factorLaunches.end(), tunable))
        {
            m_tuned = true; // nothing to choose
            return;
        }
        {
            std::mutex* lock = nullptr;
            auto& cache = tuneCache(lock);
            const std::lock_guard<std::mutex> guard(*lock);
            const auto known = cache.find(tuneKey());
            if (known != cache.end())
            {
                m_tuneReport = known->second;
                for (Launch& launch : m_plan.factorLaunches)
                    if (tunable(launch))
                        for (const TuneRecord& r : m_tuneReport)
                            if (r.kind == static_cast<std::int32_t>(launch.kind) && r.sizeClass == sizeClass(launch.count))
                                launch.variant = r.chosen;
                m_factorGraph.reset();
                m_tuned = true;
                return;
            }
        }
        std::vector<double> seconds(count * VARIANTS, 0.0);
        // the timing runs launch one by one with events around each launch; the caller's profiling setting comes back
        // whatever happens
        struct Restore
        {
            bool& flag;
            bool value;
            ~Restore() { flag = value; }
        } restore{m_profile, m_profile};
        m_profile = true;
        // Two timed factorisations per variant, each launch keeping its shorter time: the first launch of a kernel in
        // a process also loads its module, which must not count against it.
        constexpr int RUNS = 2;
        std::fill(seconds.begin(), seconds.end(), std::numeric_limits<double>::infinity());
        for (int v = 0; v < VARIANTS; ++v)
        {
            for (Launch& launch : m_plan.factorLaunches)
                if (tunable(launch))
                    launch.variant = v;
            for (int run = 0; run < RUNS; ++run)
            {
                launches();
                check(cudaStreamSynchronize(m_stream), "tuning factorisation");
                for (std::size_t i = 0; i < count; ++i)
                {
                    float ms = 0.0f;
                    check(cudaEventElapsedTime(&ms, profileEvent(2 * i), profileEvent(2 * i + 1)), "tuning time");
                    double& kept = seconds[i * VARIANTS + static_cast<std::size_t>(v)];
                    kept = std::min(kept, ms / 1000.0);
                }
            }
        }
        const auto recordOf = [&](const Launch& launch) -> TuneRecord&
        {
            const std::int32_t kind = static_cast<std::int32_t>(launch.kind);
            const std::int32_t size = sizeClass(launch.count);
            for (TuneRecord& r : m_tuneReport)
                if (r.kind == kind && r.sizeClass == size)
                    return r;
            m_tuneReport.push_back({kind, size, 0, {0.0, 0.0}, 0});
            return m_tuneReport.back();
        };
        for (std::size_t i = 0; i < count; ++i)
        {
            const Launch& launch = m_plan.factorLaunches[i];
            if (!tunable(launch))
                continue;
            TuneRecord& r = recordOf(launch);
            ++r.launches;
            for (int v = 0; v < VARIANTS; ++v)
                r.seconds[v] += seconds[i * VARIANTS + static_cast<std::size_t>(v)];
        }
        for (TuneRecord& r : m_tuneReport)
            r.chosen = r.seconds[1] < r.seconds[0] ? 1 : 0;
        for (Launch& launch : m_plan.factorLaunches)
            if (tunable(launch))
                launch.variant = recordOf(launch).chosen;
        m_factorGraph.reset();
        m_tuned = true;
        std::mutex* lock = nullptr;
        auto& cache = tuneCache(lock);
        const std::lock_guard<std::mutex> guard(*lock);
        cache[tuneKey()] = m_tuneReport;
    }

    // The factor launches in plan order on the main stream, except the side groups (the far part of a finished
    // macro panel's update, Launch::sideGroup), which fork onto the side stream and are waited for where the plan
    // says (Launch::waitGroup) and at the end. A profiled factorisation runs everything on the main stream.
    void runFactorLaunches(const device::FactorArgs& args)
    {
        std::size_t index = 0;
        std::int32_t forkedGroup = -1;
        std::int32_t lastGroup = -1;
        for (const Launch& launch : m_plan.factorLaunches)
        {
            if (m_partialLevel >= 0 && launch.level >= m_partialLevel)
            {
                // a partial factorisation leaves the trailing supernode's level out (its front becomes K*)
                if (m_profile)
                {
                    check(cudaEventRecord(profileEvent(2 * index), m_stream), "profile event");
                    check(cudaEventRecord(profileEvent(2 * index + 1), m_stream), "profile event");
                }
                ++index;
                continue;
            }
            const bool lookahead = !m_profile;
            if (lookahead && launch.waitGroup >= 0)
                check(cudaStreamWaitEvent(m_stream, m_groupDone[launch.waitGroup & 1], 0), "wait for a side group");
            if (m_profile)
                check(cudaEventRecord(profileEvent(2 * index), m_stream), "profile event");
            const std::int32_t mixed = m_mixed ? m_plan.mixedOfFactorLaunch[index] : -1;
            if (mixed >= 0)
            {
                check(cudaGetLastError(), "factorisation launch before the mixed update");
                const Launch& replacement = m_plan.mixedLaunches[static_cast<std::size_t>(mixed)];
                device::updateMatrixMixed<<<replacement.count, 256, device::MIXED_UPDATE_SMEM, m_stream>>>(
                    args, m_tiles.get() + replacement.offset, m_mixedError.get());
                check(cudaGetLastError(), "mixed update launch");
            }
            else if (lookahead && launch.sideGroup >= 0)
            {
                if (launch.sideGroup != forkedGroup)
                {
                    check(cudaEventRecord(m_fork, m_stream), "fork the side stream");
                    check(cudaStreamWaitEvent(m_side, m_fork, 0), "fork the side stream");
                    forkedGroup = launch.sideGroup;
                }
                launchFactor(launch, args, m_side);
                check(cudaEventRecord(m_groupDone[launch.sideGroup & 1], m_side), "side group");
                lastGroup = launch.sideGroup;
            }
            else
                launchFactor(launch, args, m_stream);
            if (m_profile)
                check(cudaEventRecord(profileEvent(2 * index + 1), m_stream), "profile event");
            ++index;
        }
        if (lastGroup >= 0)
            check(cudaStreamWaitEvent(m_stream, m_groupDone[lastGroup & 1], 0), "join the side stream");
        check(cudaGetLastError(), "factorisation launch");
    }

    cudaEvent_t profileEvent(std::size_t k)
    {
        while (m_profileEvents.size() <= k)
        {
            cudaEvent_t e = nullptr;
            check(cudaEventCreate(&e), "cudaEventCreate");
            m_profileEvents.push_back(e);
        }
        return m_profileEvents[k];
    }

    void launchFactor(const Launch& launch, const device::FactorArgs& args, cudaStream_t stream)
    {
        {
            switch (launch.kind)
            {
            case LaunchKind::SmallFronts:
            {
                const std::size_t smem = device::smallFrontSmem(launch.smemOrder);
                device::smallFronts<<<launch.count, SMALL_THREADS, smem, stream>>>(
                    args, m_lists.get() + launch.offset, m_structureError.get());
                break;
            }
            case LaunchKind::AssembleFronts:
                if (launch.variant == 1)
                    device::assembleStaged<<<launch.altCount, device::STAGE_THREADS, device::STAGE_SMEM, stream>>>(
                        args, m_stagedPieces.get() + launch.altOffset, m_structureError.get());
                else
                    device::assembleFronts<<<launch.count, 256, 0, stream>>>(args, m_pieces.get() + launch.offset,
                                                                               m_structureError.get());
                break;
            case LaunchKind::DiagonalBlocks:
                if (launch.variant == 1)
                    device::diagonalBlocksByColumn<<<launch.count, device::DIAGONAL_THREADS, 0, stream>>>(
                        args, m_lists.get() + launch.offset, launch.k0);
                else
                    device::diagonalBlocks<<<launch.count, device::DIAGONAL_THREADS, 0, stream>>>(
                        args, m_lists.get() + launch.offset, launch.k0);
                break;
            case LaunchKind::PanelRows:
                device::panelRowsInverse<<<launch.count, device::TILE_THREADS, device::PANEL_ROWS_INVERSE_SMEM,
                                           stream>>>(args, m_tiles.get() + launch.offset, launch.k0);
                break;
            case LaunchKind::PanelUpdate:
                device::panelUpdate<<<launch.count, device::TILE_THREADS, 0, stream>>>(
                    args, m_tiles.get() + launch.offset, launch.k0);
                break;
            case LaunchKind::UpdateMatrix:
                if (launch.variant == 1)
                    device::updateMatrixTma<<<launch.altCount, device::UPDATE_THREADS, device::UPDATE_TMA_SMEM,
                                              stream>>>(args, m_tiles.get() + launch.altOffset, m_tensorMaps.get(),
                                                        m_mixedError.get());
                else
                    device::updateMatrix<<<launch.count, device::TILE_THREADS, 0, stream>>>(
                        args, m_tiles.get() + launch.offset);
                break;
            default:
                throw Error(STATUS_INTERNAL, "factorisation plan: a solve launch in the factor sequence");
            }
        }
    }

    void runSweep(const device::SolveArgs& args, const SolveView& view, const std::vector<Launch>& launches)
    {
        // the chain launches' tickets and flags start cleared in every sweep
        if (std::any_of(launches.begin(), launches.end(), [](const Launch& l)
                        { return l.kind == LaunchKind::ForwardChain || l.kind == LaunchKind::BackwardChain; }))
            check(cudaMemsetAsync(m_chainState.get(), 0,
                                  (static_cast<std::size_t>(view.plan->chainSlots) +
                                   static_cast<std::size_t>(view.plan->chainFlags)) * sizeof(int),
                                  m_stream),
                  "chain state");
        for (const Launch& launch : launches)
        {
            const std::int32_t* list = view.lists + launch.offset;
            const device::TileTask* tiles = view.tiles + launch.offset;
            const std::size_t smallSmem = device::smallSolveSmem(std::max(launch.smemOrder, 1));
            const std::size_t record = beginSolveRecord(static_cast<std::int32_t>(launch.kind), launch.count, launch.k0);
            switch (launch.kind)
            {
            case LaunchKind::ForwardSmall:
                device::forwardSmall<<<launch.count, device::TILE_THREADS, smallSmem, m_stream>>>(
                    args, list, std::max(launch.smemOrder, 1));
                break;
            case LaunchKind::ForwardGather:
                device::forwardGather<<<launch.count, device::TILE_THREADS, 0, m_stream>>>(args, tiles);
                break;
            case LaunchKind::ForwardChain:
                device::forwardChain<<<launch.count, device::TILE_THREADS, device::CHAIN_SMEM, m_stream>>>(
                    args, tiles, launch.k0);
                break;
            case LaunchKind::BackwardSmall:
                device::backwardSmall<<<launch.count, device::TILE_THREADS, smallSmem, m_stream>>>(
                    args, list, std::max(launch.smemOrder, 1));
                break;
            case LaunchKind::BackwardRows:
                device::backwardRows<<<launch.count, device::TILE_THREADS, 0, m_stream>>>(args, tiles);
                break;
            case LaunchKind::BackwardRowsReduce:
                device::backwardRowsReduce<<<launch.count, device::TILE_THREADS, 0, m_stream>>>(args, tiles);
                break;
            case LaunchKind::BackwardChain:
                device::backwardChain<<<launch.count, device::TILE_THREADS, device::CHAIN_SMEM, m_stream>>>(
                    args, tiles, launch.k0);
                break;
            default:
                throw Error(STATUS_INTERNAL, "solve plan: a factorisation launch in a sweep");
            }
            endSolveRecord(record);
        }
    }

    // Per-launch device times of the last profiled solve's sweeps (its last column tile): events around each launch
    // when profiling is on.
    std::size_t beginSolveRecord(std::int32_t kind, std::int32_t count, std::int32_t k0)
    {
        if (!m_profile)
            return 0;
        const std::size_t index = m_solveRecords.size();
        m_solveRecords.push_back({kind, count, k0});
        while (m_solveEvents.size() < 2 * (index + 1))
        {
            cudaEvent_t e = nullptr;
            check(cudaEventCreate(&e), "profile event");
            m_solveEvents.push_back(e);
        }
        check(cudaEventRecord(m_solveEvents[2 * index], m_stream), "profile event");
        return index;
    }
    void endSolveRecord(std::size_t index)
    {
        if (m_profile)
            check(cudaEventRecord(m_solveEvents[2 * index + 1], m_stream), "profile event");
    }

    Symbolic m_symbolic;
    int m_device = 0;
    Plan m_plan;
    cudaStream_t m_stream = nullptr;
    // the lookahead's side stream, its fork point and the completion of its groups (alternating)
    cudaStream_t m_side = nullptr;
    cudaStream_t m_copyStream = nullptr; // prefetched right-hand sides
    cudaEvent_t m_prefetchDone = nullptr;
    cudaEvent_t m_prefetchStart = nullptr;
    struct Prefetch
    {
        const double* host = nullptr;
        std::int64_t ld = 0;
        std::int64_t columns = 0;
        bool issued = false;
    };
    Prefetch m_prefetch;
    cudaEvent_t m_fork = nullptr;
    cudaEvent_t m_groupDone[2] = {nullptr, nullptr};
    cudaEvent_t m_start = nullptr;
    cudaEvent_t m_stop = nullptr;
    DeviceArray<device::FrontDesc> m_fronts;
    DeviceArray<std::int32_t> m_children;
    DeviceArray<std::int32_t> m_rows;
    DeviceArray<std::int32_t> m_relpos;
    DeviceArray<std::int64_t> m_gatherStart;
    LaunchGraph m_factorGraph;
    LaunchGraph m_sweepGraph;
    DeviceArray<std::int32_t> m_gatherRows;
    DeviceArray<double> m_rowPartials;
    // The chain launches' state: ticket counters and ready flags of the plan's (or the restated plan's) sweeps, then
    // the stop word (last); and the host-mapped word a wait that ran out sets.
    DeviceArray<int> m_chainState;
    int* m_chainFailed = nullptr;
    DeviceArray<std::int32_t> m_supernodeOfColumn;
    DeviceArray<std::int32_t> m_lists;
    DeviceArray<device::TileTask> m_tiles;
    DeviceArray<device::AssemblyTask> m_pieces;
    DeviceArray<device::AssemblyTask> m_stagedPieces;
    DeviceArray<CUtensorMap> m_tensorMaps;
    const double* m_mapsOf = nullptr; // the panel arena the tensor maps describe
    DeviceArray<std::int32_t> m_zeroPivot;
    DeviceArray<unsigned long long> m_counters;
    DeviceArray<std::int32_t> m_issues;
    DeviceArray<double> m_blockRatio;
    DeviceArray<std::int32_t> m_blockEquation;
    DeviceArray<std::int32_t> m_structureError;
    DeviceArray<int> m_mixedError;
    DeviceArray<double> m_krylov;
    DeviceArray<double> m_gmresPartials;
    DeviceArray<double> m_gmresValues;
    DeviceArray<double> m_gmresCoefficients;
    bool m_mixed = false;
    DeviceArray<double> m_panels;
    DeviceArray<double> m_updates;
    DeviceArray<std::int64_t> m_cscOffsets;
    DeviceArray<std::int32_t> m_cscRows;
    DeviceArray<double> m_cscValues;
    DeviceArray<double> m_referenceDiagonal;
    DeviceArray<double> m_work;
    DeviceArray<double> m_updateRows;
    DeviceArray<double> m_hostB;
    // indefinite mode
    DeviceArray<std::int32_t> m_perm;
    DeviceArray<std::int32_t> m_inversePerm;
    DeviceArray<double> m_subdiagonal;
    DeviceArray<std::int32_t> m_status;
    DeviceArray<std::int32_t> m_stepPerm;
    DeviceArray<std::int32_t> m_stepSwapped;
    DeviceArray<double> m_w;
    DeviceArray<std::int64_t> m_wOffset;
    DeviceArray<double> m_frontWork;
    // Delayed pivots: the exact path's outcome of each front it factorised (null elsewhere), the grown panels and
    // update matrices of this factorisation, the exact path's scratch, and the restated structure the solves use when
    // some front delayed.
    std::vector<std::unique_ptr<ExactOutcome>> m_exact;
    std::vector<std::unique_ptr<DeviceArray<double>>> m_grown;
    DeviceArray<device::FrontSource> m_exactSources;
    DeviceArray<std::int32_t> m_exactPositions;
    DeviceArray<std::int32_t> m_exactPerm;
    DeviceArray<double> m_exactSub;
    DeviceArray<std::int32_t> m_exactCount;
    std::int64_t m_delayedPivots = 0;
    struct Restated
    {
        Plan plan;
        std::vector<std::int32_t> perm; // position -> equation (host copy)
        std::vector<double> subdiagonal;
        DeviceArray<device::FrontDesc> fronts;
        DeviceArray<std::int32_t> rows;
        DeviceArray<std::int32_t> relpos;
        DeviceArray<std::int64_t> gatherStart;
        DeviceArray<std::int32_t> gatherRows;
        DeviceArray<std::int32_t> supernodeOfColumn;
        DeviceArray<std::int32_t> lists;
        DeviceArray<device::TileTask> tiles;
        DeviceArray<std::int32_t> devicePerm;
        DeviceArray<double> deviceSubdiagonal;
    };
    Restated m_restated;
    bool m_isRestated = false;
    // Partial factorisation: the trailing supernode's level (-1: a full factorisation), its equations, K* on the
    // device, and the solve launches below that level.
    std::int32_t m_partialLevel = -1;
    std::int32_t m_trailing = 0;
    bool m_isPartial = false;
    DeviceArray<double> m_schur;
    std::vector<Launch> m_partialForward;
    std::vector<Launch> m_partialBackward;
    std::uintptr_t m_structureGeneration = 0;
    DeviceArray<std::int32_t> m_rowsPivot;
    DeviceArray<std::int32_t> m_relposPivot;
    bool m_pivoted = false;
    bool m_singular = false;
    std::int64_t m_exactFronts = 0;
    const double* m_solveScale = nullptr;
    DeviceArray<double> m_hostX;
    DeviceArray<double> m_bRows;
    DeviceArray<double> m_rRows;
    DeviceArray<double> m_norms;
    DeviceArray<std::int64_t> m_fullStart;
    DeviceArray<std::int32_t> m_fullColumns;
    DeviceArray<std::int32_t> m_fullSource;
    DeviceArray<std::int32_t> m_groupFirst;
    DeviceArray<double> m_diagonal; // D of a positive definite factor, contiguous (gatherDiagonal)
    std::int32_t m_residualGroups = 0;
    std::int64_t m_fullTerms = -1;
    const std::int64_t* m_matrixOffsets = nullptr;
    const std::int32_t* m_matrixRows = nullptr;
    const double* m_matrixValues = nullptr;
    std::int64_t m_matrixTerms = 0;
    std::size_t m_smallSmem = 0;
    bool m_factorised = false;
    bool m_profile = false;
    bool m_tuning = true;
    bool m_tuned = false;
    std::vector<TuneRecord> m_tuneReport;
    bool m_profileValid = false;
    bool m_solveProfileValid = false;
    bool m_profiledPivoted = false; // the last profiled factorisation ran the indefinite launches
    struct SolveRecord
    {
        std::int32_t kind;
        std::int32_t count;
        std::int32_t k0;
    };
    // The kind code of the diagonal sweep in a solve's launch profile (after the plan's launch kinds).
    static constexpr std::int32_t DIAGONAL_SWEEP_KIND = static_cast<std::int32_t>(LaunchKind::DiagonalSweep);
    std::vector<SolveRecord> m_solveRecords;
    std::vector<cudaEvent_t> m_solveEvents;
    bool m_annotated = false;
    std::vector<cudaEvent_t> m_profileEvents;
    double m_lastSolveSeconds = 0.0;
};

namespace
{

template <typename F> int guarded(F&& body)
{
    try
    {
        body();
        return STATUS_OK;
    }
    catch (const Error& error)
    {
        g_lastError = error.what();
        return error.status();
    }
    catch (const std::bad_alloc&)
    {
        g_lastError = "host memory exhausted";
        return STATUS_MEMORY_BUDGET;
    }
    catch (const std::exception& error)
    {
        g_lastError = error.what();
        return STATUS_INTERNAL;
    }
}

} // namespace
} // namespace oosgpu

struct oosgpu_symbolic
{
    oosgpu::Symbolic symbolic;
    std::int32_t levels = 0;
    std::int64_t updateValues = 0;
    // The launch plan of the structure, built by the first factor or pencil made on it and copied by the later ones
    // (on the 60^3 block the build takes about half a second; a fresh pencil of the same model then skips it).
    std::mutex planLock;
    std::shared_ptr<const oosgpu::Plan> plan;
};

namespace
{

const oosgpu::Plan* planOf(const oosgpu_symbolic* handle)
{
    auto* s = const_cast<oosgpu_symbolic*>(handle);
    const std::lock_guard<std::mutex> guard(s->planLock);
    if (!s->plan)
        s->plan = std::make_shared<const oosgpu::Plan>(oosgpu::buildPlan(s->symbolic));
    return s->plan.get();
}

} // namespace

struct oosgpu_factor
{
    std::unique_ptr<oosgpu::GpuFactor> factor;
};

namespace oosgpu
{

// The shifted pencil (K, M) on the GPU: the reference's SparsePencil (include/oos/linalg/eigen/SparsePencil.hpp:29-85,
// src/linalg/eigen/SparsePencil.cpp:55-157) behind its ShiftedPencil interface. K and M share one structure (the
// lower CSC of the symbolic factor's order); factorise(sigma) forms S (K - sigma M) S on the device with the scales of
// pencilScaleOf (powers of two near 1/sqrt(K_ii), src/linalg/eigen/PencilScaling.cpp:12-31) and factorises it in
// indefinite mode; solve() gives (K - sigma M)^-1 X = S (S (K - sigma M) S)^-1 S X; multiplyMass() uses the diagonal of
// a lumped mass (every off-diagonal term zero), the full pattern otherwise.
class GpuPencil
{
public:
    // The vibration pencil (K, M) (SparsePencil), or with `buckling` the buckling pencil K phi = lambda B phi of the
    // stiffness and the differential stiffness K_d given as `mass` (BucklingPencil: B = -K_d, held negated, so that
    // the shifted matrix K - sigma B = K + sigma K_d rounds as the reference's combine(1, K, sigma, K_d); the inner
    // product is K's).
    GpuPencil(const Symbolic& symbolic, int device, std::int32_t dimension, const std::int64_t* offsets,
              const std::int32_t* rows, const double* stiffness, const double* mass, bool buckling = false,
              const Plan* prebuilt = nullptr)
        : m_factor(symbolic, device, prebuilt), m_device(device), m_dimension(dimension), m_buckling(buckling)
    {
        const char* name = buckling ? "BucklingPencil" : "SparsePencil";
        if (dimension != symbolic.dofCount)
            throw Error(STATUS_INVALID_ARGUMENT, std::string(name) + ": the matrices have " + std::to_string(dimension) +
                                                     " equations, the symbolic factor " +
                                                     std::to_string(symbolic.dofCount) +
                                                     "; analyse the pattern the matrices were converted on");
        const auto n = static_cast<std::size_t>(dimension);
        m_terms = offsets[dimension];
        std::vector<double> scale(n, 1.0);
        std::vector<double> massDiagonal(n, 0.0);
        std::vector<double> right;
        if (buckling)
        {
            right.resize(static_cast<std::size_t>(m_terms));
            for (std::size_t t = 0; t < right.size(); ++t)
                right[t] = -mass[t];
            mass = right.data();
        }
        m_rayleighBound = INFINITY;
        m_lumped = true;
        for (std::size_t j = 0; j < n; ++j)
        {
            const std::int64_t first = offsets[j];
            const bool hasDiagonal = first < offsets[j + 1] && static_cast<std::size_t>(rows[first]) == j;
            const double k = hasDiagonal ? stiffness[first] : 0.0;
            const double m = hasDiagonal ? mass[first] : 0.0;
            if (buckling)
            {
                // min K_ii / |K_d,ii| over K_d,ii != 0 (finite) and K_ii > 0 (BucklingPencil.cpp:31-44)
                if (m != 0.0 && std::isfinite(m) && k > 0.0)
                    m_rayleighBound = std::min(m_rayleighBound, k / std::abs(m));
            }
            else
            {
                if (!std::isfinite(m) || m < 0.0)
                    throw Error(STATUS_SOLVER, "eigenvalue analysis: the mass matrix has the diagonal term " +
                                                   std::to_string(m) + " at equation " + std::to_string(j) +
                                                   "; the Lanczos method needs a positive semi-definite mass matrix");
                if (m > 0.0 && k > 0.0)
                    m_rayleighBound = std::min(m_rayleighBound, k / m);
            }
            massDiagonal[j] = m;
            // pencilScaleOf: K_ii = f 2^e with f in [0.5, 1): the scale 2^(-(e/2)) leaves a scaled diagonal in [1/4, 2).
            if (k > 0.0 && std::isfinite(k))
            {
                int exponent = 0;
                std::frexp(k, &exponent);
                scale[j] = std::ldexp(1.0, -(exponent / 2));
            }
            for (std::int64_t t = first; t < offsets[j + 1]; ++t)
                if (static_cast<std::size_t>(rows[t]) != j && mass[t] != 0.0)
                    m_lumped = false;
        }
        const cudaStream_t stream = m_factor.stream();
        const auto upload = [&](auto& array, const auto* host, std::size_t count, const char* what)
        {
            array.allocate(count, what);
            check(cudaMemcpyAsync(array.get(), host, count * sizeof(*host), cudaMemcpyHostToDevice, stream), what);
        };
        upload(m_offsets, offsets, n + 1, "pencil: offsets");
        upload(m_rows, rows, static_cast<std::size_t>(m_terms), "pencil: rows");
        upload(m_stiffness, stiffness, static_cast<std::size_t>(m_terms), "pencil: stiffness");
        upload(m_mass, mass, static_cast<std::size_t>(m_terms), "pencil: mass");
        upload(m_massDiagonal, massDiagonal.data(), n, "pencil: mass diagonal");
        upload(m_scale, scale.data(), n, "pencil: scales");
        m_shifted.allocate(static_cast<std::size_t>(m_terms), "pencil: shifted matrix");
        check(cudaStreamSynchronize(stream), "pencil upload");
        m_factor.setSolveScale(m_scale.get());
        m_factor.useStructure(m_offsets.get(), m_rows.get(), m_terms);
    }

    // ShiftedPencil::factorise: the inertia of K - sigma M (a singular factor returned, not refused).
    oosgpu_factor_info factorise(double shift)
    {
        check(cudaSetDevice(m_device), "cudaSetDevice");
        constexpr int WARPS = 8;
        device::shiftedMatrix<<<blocksFor(m_dimension, WARPS), 32 * WARPS, 0, m_factor.stream()>>>(
            m_offsets.get(), m_rows.get(), m_stiffness.get(), m_mass.get(), shift, m_scale.get(), m_shifted.get(),
            m_dimension);
        check(cudaGetLastError(), "shifted matrix launch");
        oosgpu_factor_info info{};
        ++m_factorisations;
        m_shift = shift;
        // Below the spectrum (a vibration pencil at a shift <= 0: K + |sigma| M; a buckling pencil at 0: K) the
        // shifted matrix is positive definite whenever its count can be trusted at all, so it is factorised first
        // without pivots, which a positive definite matrix does not need; a negative or zero pivot sends it to the
        // pivoted factorisation after all. The inertia is the same either way (Sylvester's law).
        if (m_buckling ? shift == 0.0 : shift <= 0.0)
        {
            oosgpu_factor_options definite{1.0e7, -1, nullptr, 0};
            bool accepted = false;
            try
            {
                m_factor.factorise(m_dimension, m_terms, m_offsets.get(), m_rows.get(), m_shifted.get(), true,
                                   &definite, &info);
                accepted = info.negative == 0 && info.zero == 0;
            }
            catch (const Error& e)
            {
                if (e.status() != STATUS_SINGULAR)
                    throw;
            }
            if (accepted)
                return info;
            info = oosgpu_factor_info{};
        }
        oosgpu_factor_options options{1.0e7, -1, nullptr, 1};
        m_factor.factorise(m_dimension, m_terms, m_offsets.get(), m_rows.get(), m_shifted.get(), true, &options, &info);
        return info;
    }

    void solve(double* x, std::int64_t ld, std::int64_t columns) { m_factor.solve(x, ld, columns, true); }

    void multiplyMass(const double* x, std::int64_t ldx, double* y, std::int64_t ldy, std::int64_t columns)
    {
        check(cudaSetDevice(m_device), "cudaSetDevice");
        if (ldx < m_dimension || ldy < m_dimension || columns < 0)
            throw Error(STATUS_INVALID_ARGUMENT, "SparsePencil::multiplyMass: leading dimensions below the rows");
        if (m_lumped)
        {
            const std::int64_t items = static_cast<std::int64_t>(m_dimension) * columns;
            device::diagonalProduct<<<blocksFor(std::max<std::int64_t>(items, 1), 256), 256, 0, m_factor.stream()>>>(
                m_massDiagonal.get(), x, ldx, y, ldy, m_dimension, static_cast<int>(columns));
            check(cudaGetLastError(), "mass product launch");
            return;
        }
        for (std::int64_t c0 = 0; c0 < columns; c0 += 32)
            m_factor.multiplySymmetric(m_mass.get(), x + c0 * ldx, ldx, y + c0 * ldy, ldy,
                                       static_cast<int>(std::min<std::int64_t>(32, columns - c0)));
    }

    // Y <- G X, G the matrix of the inner product: M, or K for a buckling pencil (BucklingPencil::multiplyInnerProduct).
    void multiplyInnerProduct(const double* x, std::int64_t ldx, double* y, std::int64_t ldy, std::int64_t columns)
    {
        if (!m_buckling)
        {
            multiplyMass(x, ldx, y, ldy, columns);
            return;
        }
        check(cudaSetDevice(m_device), "cudaSetDevice");
        if (ldx < m_dimension || ldy < m_dimension || columns < 0)
            throw Error(STATUS_INVALID_ARGUMENT, "BucklingPencil::multiplyInnerProduct: leading dimensions below the rows");
        for (std::int64_t c0 = 0; c0 < columns; c0 += 32)
            m_factor.multiplySymmetric(m_stiffness.get(), x + c0 * ldx, ldx, y + c0 * ldy, ldy,
                                       static_cast<int>(std::min<std::int64_t>(32, columns - c0)));
    }

    [[nodiscard]] bool buckling() const noexcept { return m_buckling; }
    [[nodiscard]] cudaStream_t stream() const noexcept { return m_factor.stream(); }
    [[nodiscard]] double rayleighBound() const noexcept { return m_rayleighBound; }
    [[nodiscard]] bool lumped() const noexcept { return m_lumped; }
    [[nodiscard]] std::int64_t factorisations() const noexcept { return m_factorisations; }
    [[nodiscard]] std::int32_t dimension() const noexcept { return m_dimension; }
    [[nodiscard]] GpuFactor& factor() noexcept { return m_factor; }
    [[nodiscard]] const double* massDiagonal() const noexcept { return m_massDiagonal.get(); }

private:
    GpuFactor m_factor;
    int m_device = 0;
    std::int32_t m_dimension = 0;
    bool m_buckling = false;
    std::int64_t m_terms = 0;
    double m_rayleighBound = 0.0;
    bool m_lumped = true;
    std::int64_t m_factorisations = 0;
    double m_shift = 0.0;
    DeviceArray<std::int64_t> m_offsets;
    DeviceArray<std::int32_t> m_rows;
    DeviceArray<double> m_stiffness;
    DeviceArray<double> m_mass;
    DeviceArray<double> m_massDiagonal;
    DeviceArray<double> m_scale;
    DeviceArray<double> m_shifted;
};

// The GPU pencil behind the eigen solver's PencilPort interface.
class PencilOperations final : public eigen::PencilPort
{
public:
    explicit PencilOperations(GpuPencil& pencil) : m_pencil(pencil) {}

    [[nodiscard]] std::int32_t dimension() const override { return m_pencil.dimension(); }
    eigen::Inertia factorise(double shift) override
    {
        const oosgpu_factor_info info = m_pencil.factorise(shift);
        m_seconds = info.device_seconds;
        return {info.positive, info.negative, info.zero};
    }
    void solve(double* x, std::int64_t ld, std::int64_t columns) override { m_pencil.solve(x, ld, columns); }
    void multiplyMass(const double* x, std::int64_t ldx, double* y, std::int64_t ldy, std::int64_t columns) override
    {
        m_pencil.multiplyMass(x, ldx, y, ldy, columns);
    }
    void multiplyInnerProduct(const double* x, std::int64_t ldx, double* y, std::int64_t ldy,
                              std::int64_t columns) override
    {
        m_pencil.multiplyInnerProduct(x, ldx, y, ldy, columns);
    }
    [[nodiscard]] double diagonalRayleighBound() const override { return m_pencil.rayleighBound(); }
    [[nodiscard]] cudaStream_t stream() const override { return m_pencil.stream(); }
    [[nodiscard]] double lastFactorSeconds() const override { return m_seconds; }

private:
    GpuPencil& m_pencil;
    double m_seconds = 0.0;
};

} // namespace oosgpu

struct oosgpu_pencil
{
    std::unique_ptr<oosgpu::GpuPencil> pencil;
};

struct oosgpu_modes
{
    oosgpu::eigen::ModeResult solution;
};

struct oosgpu_model
{
    oosgpu::Model model;
};

using oosgpu::guarded;

namespace oosgpu
{

int runGuarded(const std::function<void()>& body)
{
    return guarded(body);
}

int factorDevice(const oosgpu_factor* factor)
{
    if (factor == nullptr)
        throw Error(STATUS_INVALID_ARGUMENT, "factor is null");
    return factor->factor->deviceOrdinal();
}

void solveFactorInScratch(oosgpu_factor* factor, double* b, std::int64_t ld, std::int64_t columns, double* scratch,
                          std::size_t capacity)
{
    if (factor == nullptr)
        throw Error(STATUS_INVALID_ARGUMENT, "factor is null");
    factor->factor->solveInScratch(b, ld, columns, scratch, capacity);
}

} // namespace oosgpu

namespace
{

void summarise(oosgpu_symbolic& handle)
{
    handle.symbolic.validate();
    std::vector<std::int32_t> level(static_cast<std::size_t>(handle.symbolic.supernodeCount), 0);
    std::int32_t top = 0;
    std::int64_t update = 0;
    for (std::int32_t s = 0; s < handle.symbolic.supernodeCount; ++s)
    {
        const std::int32_t p = handle.symbolic.parent[static_cast<std::size_t>(s)];
        if (p >= 0)
            level[static_cast<std::size_t>(p)] = std::max(level[static_cast<std::size_t>(p)], level[static_cast<std::size_t>(s)] + 1);
        top = std::max(top, level[static_cast<std::size_t>(s)]);
        const std::int64_t r = handle.symbolic.rowCount(s);
        update += r * r;
    }
    handle.levels = handle.symbolic.supernodeCount == 0 ? 0 : top + 1;
    handle.updateValues = update;
}

void requirePointer(const void* p, const char* what)
{
    if (p == nullptr)
        throw oosgpu::Error(oosgpu::STATUS_INVALID_ARGUMENT, std::string(what) + " is null");
}

} // namespace

extern "C" const char* oosgpu_last_error(void)
{
    return oosgpu::g_lastError.c_str();
}

extern "C" int64_t oosgpu_release_cached_buffers(int device)
{
    return static_cast<int64_t>(oosgpu::eigen::releaseDeviceBuffers(device));
}

extern "C" int oosgpu_device_count(void)
{
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess)
    {
        cudaGetLastError();
        return 0;
    }
    return count;
}

extern "C" int oosgpu_symbolic_create(int32_t dof_count, int32_t supernode_count, const int32_t* first_column,
                                      const int32_t* parent, const int64_t* row_start, const int32_t* rows,
                                      oosgpu_symbolic** out)
{
    return guarded(
        [&]
        {
            requirePointer(out, "out");
            requirePointer(first_column, "first_column");
            requirePointer(parent, "parent");
            requirePointer(row_start, "row_start");
            if (supernode_count < 0)
                throw oosgpu::Error(oosgpu::STATUS_INVALID_ARGUMENT, "negative supernode count");
            auto handle = std::make_unique<oosgpu_symbolic>();
            oosgpu::Symbolic& s = handle->symbolic;
            s.dofCount = dof_count;
            s.supernodeCount = supernode_count;
            s.firstColumn.assign(first_column, first_column + supernode_count + 1);
            s.parent.assign(parent, parent + supernode_count);
            s.rowStart.assign(row_start, row_start + supernode_count + 1);
            if (row_start[supernode_count] > 0)
                requirePointer(rows, "rows");
            s.rows.assign(rows, rows + row_start[supernode_count]);
            summarise(*handle);
            *out = handle.release();
        });
}

extern "C" int oosgpu_symbolic_from_partition(int32_t node_count, const int64_t* offsets, const int32_t* neighbours,
                                              const int32_t* weights, const int32_t* node_at_position,
                                              int32_t supernode_count, const int32_t* first_position,
                                              const int32_t* parent, oosgpu_symbolic** out)
{
    return guarded(
        [&]
        {
            requirePointer(out, "out");
            requirePointer(offsets, "offsets");
            requirePointer(weights, "weights");
            requirePointer(node_at_position, "node_at_position");
            requirePointer(first_position, "first_position");
            requirePointer(parent, "parent");
            auto handle = std::make_unique<oosgpu_symbolic>();
            handle->symbolic = oosgpu::rowStructures(node_count, offsets, neighbours, weights, node_at_position,
                                                     supernode_count, first_position, parent);
            summarise(*handle);
            *out = handle.release();
        });
}

extern "C" int oosgpu_symbolic_sizes(const oosgpu_symbolic* symbolic, int64_t sizes[8], double* flops)
{
    return guarded(
        [&]
        {
            requirePointer(symbolic, "symbolic");
            const oosgpu::Symbolic& s = symbolic->symbolic;
            sizes[0] = s.dofCount;
            sizes[1] = s.supernodeCount;
            sizes[2] = static_cast<int64_t>(s.rows.size());
            sizes[3] = s.panelValueCount();
            sizes[4] = s.factorEntryCount();
            sizes[5] = symbolic->levels;
            sizes[6] = symbolic->updateValues;
            sizes[7] = 0;
            if (flops != nullptr)
                *flops = s.flopCount();
        });
}

extern "C" int oosgpu_symbolic_solve_chains(const oosgpu_symbolic* symbolic, int64_t counts[4])
{
    return guarded(
        [&]
        {
            requirePointer(symbolic, "symbolic");
            requirePointer(counts, "counts");
            const oosgpu::Plan plan = oosgpu::buildPlan(symbolic->symbolic);
            std::int64_t tasks = 0;
            std::int64_t longest = 0;
            for (const auto* launches : {&plan.forwardLaunches, &plan.backwardLaunches})
                for (const oosgpu::Launch& launch : *launches)
                    if (launch.kind == oosgpu::LaunchKind::ForwardChain ||
                        launch.kind == oosgpu::LaunchKind::BackwardChain)
                    {
                        tasks += launch.count;
                        longest = std::max<std::int64_t>(longest, launch.count);
                    }
            counts[0] = plan.chainSlots;
            counts[1] = tasks;
            counts[2] = plan.chainFlags;
            counts[3] = longest;
        });
}

extern "C" int oosgpu_symbolic_rows(const oosgpu_symbolic* symbolic, int64_t* row_start, int32_t* rows)
{
    return guarded(
        [&]
        {
            requirePointer(symbolic, "symbolic");
            const oosgpu::Symbolic& s = symbolic->symbolic;
            std::copy(s.rowStart.begin(), s.rowStart.end(), row_start);
            std::copy(s.rows.begin(), s.rows.end(), rows);
        });
}

extern "C" void oosgpu_symbolic_destroy(oosgpu_symbolic* symbolic)
{
    delete symbolic;
}

extern "C" int oosgpu_factor_create(const oosgpu_symbolic* symbolic, int device, oosgpu_factor** out)
{
    return guarded(
        [&]
        {
            requirePointer(symbolic, "symbolic");
            requirePointer(out, "out");
            auto handle = std::make_unique<oosgpu_factor>();
            handle->factor = std::make_unique<oosgpu::GpuFactor>(symbolic->symbolic, device, planOf(symbolic));
            *out = handle.release();
        });
}

extern "C" void oosgpu_factor_destroy(oosgpu_factor* factor)
{
    delete factor;
}

extern "C" void* oosgpu_factor_stream(oosgpu_factor* factor)
{
    return factor == nullptr ? nullptr : static_cast<void*>(factor->factor->stream());
}

extern "C" int oosgpu_solve_prefetch(oosgpu_factor* factor, const double* b, int64_t ld, int64_t columns,
                                     int32_t deferred)
{
    return guarded(
        [&]
        {
            requirePointer(factor, "factor");
            factor->factor->prefetch(b, ld, columns, deferred != 0);
        });
}

extern "C" int oosgpu_factorise_partial(oosgpu_factor* factor, int32_t dimension, const int64_t* col_offsets,
                                        const int32_t* rows, const double* values, int32_t trailing,
                                        const oosgpu_factor_options* options, double* schur_complement,
                                        oosgpu_factor_info* info)
{
    return guarded(
        [&]
        {
            requirePointer(factor, "factor");
            requirePointer(col_offsets, "col_offsets");
            requirePointer(schur_complement, "schur_complement");
            if (trailing <= 0)
                throw oosgpu::Error(oosgpu::STATUS_INVALID_ARGUMENT, "PartialFactor: expected a trailing count in [1, dimension]");
            factor->factor->factorise(dimension, -1, col_offsets, rows, values, false, options, info, trailing,
                                      schur_complement);
        });
}

extern "C" int oosgpu_partial_condense(oosgpu_factor* factor, const double* loads, int64_t ld, int64_t columns,
                                       double* condensed, int64_t ld_condensed)
{
    return guarded(
        [&]
        {
            requirePointer(factor, "factor");
            requirePointer(loads, "loads");
            requirePointer(condensed, "condensed");
            factor->factor->partialSolve(const_cast<double*>(loads), ld, columns, condensed, ld_condensed, nullptr,
                                         false);
        });
}

extern "C" int oosgpu_partial_recover(oosgpu_factor* factor, double* loads_to_solution, int64_t ld, int64_t columns,
                                      const double* trailing_values, int64_t ld_trailing)
{
    return guarded(
        [&]
        {
            requirePointer(factor, "factor");
            requirePointer(loads_to_solution, "loads_to_solution");
            requirePointer(trailing_values, "trailing_values");
            factor->factor->partialSolve(loads_to_solution, ld, columns, nullptr, ld_trailing, trailing_values, true);
        });
}

extern "C" int oosgpu_factorise(oosgpu_factor* factor, int32_t dimension, const int64_t* col_offsets,
                                const int32_t* rows, const double* values, const oosgpu_factor_options* options,
                                oosgpu_factor_info* info)
{
    return guarded(
        [&]
        {
            requirePointer(factor, "factor");
            requirePointer(col_offsets, "col_offsets");
            factor->factor->factorise(dimension, -1, col_offsets, rows, values, false, options, info);
        });
}

extern "C" int oosgpu_factorise_device(oosgpu_factor* factor, int32_t dimension, int64_t terms,
                                       const int64_t* col_offsets, const int32_t* rows, const double* values,
                                       const oosgpu_factor_options* options, oosgpu_factor_info* info)
{
    return guarded(
        [&]
        {
            requirePointer(factor, "factor");
            requirePointer(col_offsets, "col_offsets");
            factor->factor->factorise(dimension, terms, col_offsets, rows, values, true, options, info);
        });
}

extern "C" int oosgpu_factor_panel(oosgpu_factor* factor, int32_t s, int64_t* eliminated, int64_t* row_count,
                                   double* values, int32_t* rows, double* subdiagonal)
{
    return guarded(
        [&]
        {
            requirePointer(factor, "factor");
            factor->factor->panel(s, eliminated, row_count, values, rows, subdiagonal);
        });
}

extern "C" int oosgpu_solve(oosgpu_factor* factor, double* b, int64_t ld, int64_t columns)
{
    return guarded(
        [&]
        {
            requirePointer(factor, "factor");
            factor->factor->solve(b, ld, columns, false);
        });
}

extern "C" int oosgpu_solve_device(oosgpu_factor* factor, double* b, int64_t ld, int64_t columns)
{
    return guarded(
        [&]
        {
            requirePointer(factor, "factor");
            factor->factor->solve(b, ld, columns, true);
        });
}

extern "C" double oosgpu_last_solve_seconds(oosgpu_factor* factor)
{
    return factor == nullptr ? 0.0 : factor->factor->lastSolveSeconds();
}

extern "C" int oosgpu_model_plate(int32_t nx, int32_t ny, double lx, double ly, double thickness, double young,
                                  double poisson, double pressure, oosgpu_model** out)
{
    return guarded(
        [&]
        {
            requirePointer(out, "out");
            auto handle = std::make_unique<oosgpu_model>();
            handle->model = oosgpu::Model::plate(nx, ny, lx, ly, thickness, young, poisson, pressure);
            *out = handle.release();
        });
}

extern "C" int oosgpu_model_hex(int32_t n, double edge, double young, double poisson, double density,
                                oosgpu_model** out)
{
    return guarded(
        [&]
        {
            requirePointer(out, "out");
            auto handle = std::make_unique<oosgpu_model>();
            handle->model = oosgpu::Model::hexBlock(n, edge, young, poisson, density);
            *out = handle.release();
        });
}

extern "C" int oosgpu_model_stiffened_panel(int32_t n, double lx, double ly, double thickness, double young,
                                            double poisson, int32_t stringers, double blade_height,
                                            double blade_thickness, double pressure, oosgpu_model** out)
{
    return guarded(
        [&]
        {
            requirePointer(out, "out");
            auto handle = std::make_unique<oosgpu_model>();
            handle->model = oosgpu::Model::stiffenedPanel(n, lx, ly, thickness, young, poisson, stringers, blade_height,
                                                          blade_thickness, pressure);
            *out = handle.release();
        });
}

extern "C" int oosgpu_model_wing_box(double span, double chord, double height, double rib_pitch, double h,
                                     const double* thicknesses, double rib_thickness, double young, double poisson,
                                     double density, oosgpu_model** out)
{
    return guarded(
        [&]
        {
            requirePointer(out, "out");
            requirePointer(thicknesses, "thicknesses");
            auto handle = std::make_unique<oosgpu_model>();
            handle->model = oosgpu::Model::wingBox(span, chord, height, rib_pitch, h, thicknesses, rib_thickness, young,
                                                   poisson, density);
            *out = handle.release();
        });
}

extern "C" void oosgpu_model_destroy(oosgpu_model* model)
{
    delete model;
}

extern "C" int oosgpu_model_sizes(const oosgpu_model* model, int64_t sizes[4])
{
    return guarded(
        [&]
        {
            requirePointer(model, "model");
            sizes[0] = model->model.nodeCount();
            sizes[1] = model->model.nodeDofs();
            sizes[2] = static_cast<int64_t>(model->model.neighbours().size());
            sizes[3] = 0;
        });
}

extern "C" int oosgpu_model_graph(const oosgpu_model* model, int64_t* offsets, int32_t* neighbours,
                                  double* coordinates)
{
    return guarded(
        [&]
        {
            requirePointer(model, "model");
            const oosgpu::Model& m = model->model;
            if (offsets != nullptr)
                std::copy(m.offsets().begin(), m.offsets().end(), offsets);
            if (neighbours != nullptr)
                std::copy(m.neighbours().begin(), m.neighbours().end(), neighbours);
            if (coordinates != nullptr)
                std::copy(m.coordinates().begin(), m.coordinates().end(), coordinates);
        });
}

extern "C" int oosgpu_model_csc_terms(const oosgpu_model* model, const int32_t* node_at_position, int64_t* terms)
{
    return guarded(
        [&]
        {
            requirePointer(model, "model");
            requirePointer(node_at_position, "node_at_position");
            *terms = model->model.cscTermCount(node_at_position);
        });
}

extern "C" int oosgpu_model_csc(const oosgpu_model* model, const int32_t* node_at_position, int32_t which,
                                int64_t* col_offsets, int32_t* rows, double* values)
{
    return guarded(
        [&]
        {
            requirePointer(model, "model");
            requirePointer(node_at_position, "node_at_position");
            model->model.toCsc(node_at_position, which, col_offsets, rows, values);
        });
}

extern "C" int oosgpu_model_csc_device(const oosgpu_model* model, const int32_t* node_at_position, int32_t which,
                                       int32_t device, int64_t* col_offsets, int32_t* rows, double* values)
{
    return guarded(
        [&]
        {
            requirePointer(model, "model");
            requirePointer(node_at_position, "node_at_position");
            requirePointer(col_offsets, "col_offsets");
            oosgpu::check(cudaSetDevice(device), "cudaSetDevice");
            model->model.toCscOnDevice(node_at_position, which, col_offsets, rows, values);
        });
}

extern "C" int oosgpu_model_loads(const oosgpu_model* model, const int32_t* node_at_position, int64_t columns,
                                  uint64_t seed_base, int32_t points, double sigma, double* rhs, int64_t ld)
{
    return guarded(
        [&]
        {
            requirePointer(model, "model");
            requirePointer(node_at_position, "node_at_position");
            model->model.loads(node_at_position, columns, seed_base, points, sigma, rhs, ld);
        });
}

extern "C" int oosgpu_factor_profile(oosgpu_factor* factor, int32_t enable)
{
    return guarded(
        [&]
        {
            requirePointer(factor, "factor");
            factor->factor->setProfile(enable != 0);
        });
}

extern "C" int oosgpu_factor_set_tuning(oosgpu_factor* factor, int32_t enable)
{
    return guarded(
        [&]
        {
            requirePointer(factor, "factor");
            factor->factor->setTuning(enable);
        });
}

extern "C" int oosgpu_factor_tuning_report(oosgpu_factor* factor, int64_t capacity, int32_t* kinds,
                                           int32_t* size_classes, int32_t* launches, double* seconds0,
                                           double* seconds1, int32_t* chosen, int64_t* total)
{
    return guarded(
        [&]
        {
            requirePointer(factor, "factor");
            requirePointer(total, "total");
            const auto& report = factor->factor->tuneReport();
            *total = static_cast<int64_t>(report.size());
            for (std::size_t k = 0; k < report.size() && static_cast<int64_t>(k) < capacity; ++k)
            {
                if (kinds != nullptr)
                    kinds[k] = report[k].kind;
                if (size_classes != nullptr)
                    size_classes[k] = report[k].sizeClass;
                if (launches != nullptr)
                    launches[k] = report[k].launches;
                if (seconds0 != nullptr)
                    seconds0[k] = report[k].seconds[0];
                if (seconds1 != nullptr)
                    seconds1[k] = report[k].seconds[1];
                if (chosen != nullptr)
                    chosen[k] = report[k].chosen;
            }
        });
}

extern "C" int oosgpu_factor_kernel_stats(oosgpu_factor* factor, int32_t kinds, double* seconds, int64_t* launches,
                                          double* flops, double* bytes)
{
    return guarded(
        [&]
        {
            requirePointer(factor, "factor");
            factor->factor->kernelStats(kinds, seconds, launches, flops, bytes);
        });
}

extern "C" int oosgpu_factor_launch_profile(oosgpu_factor* factor, int32_t which, int64_t capacity, int32_t* kinds,
                                            int32_t* counts, int32_t* k0, double* seconds, int64_t* total)
{
    return guarded(
        [&]
        {
            requirePointer(factor, "factor");
            requirePointer(total, "total");
            if (which != 0 && which != 1)
                throw oosgpu::Error(oosgpu::STATUS_INVALID_ARGUMENT, "launch profile: which is 0 or 1");
            if (capacity > 0)
            {
                requirePointer(kinds, "kinds");
                requirePointer(counts, "counts");
                requirePointer(k0, "k0");
                requirePointer(seconds, "seconds");
            }
            *total = factor->factor->launchProfile(which, capacity, kinds, counts, k0, seconds);
        });
}

extern "C" int oosgpu_factor_launch_counts(oosgpu_factor* factor, int64_t columns, int64_t counts[2])
{
    return guarded(
        [&]
        {
            requirePointer(factor, "factor");
            counts[0] = factor->factor->factorLaunchCount();
            counts[1] = factor->factor->solveLaunchCount(columns);
        });
}

extern "C" int oosgpu_solve_refined(oosgpu_factor* factor, const double* b, int64_t ldb, double* x, int64_t ldx,
                                    int64_t columns, const oosgpu_refine_options* options, oosgpu_refine_info* info)
{
    return guarded(
        [&]
        {
            requirePointer(factor, "factor");
            const double tolerance = options != nullptr ? options->tolerance : 1.0e-10;
            const int steps = options != nullptr ? options->max_steps : 10;
            const int krylov = options != nullptr ? options->krylov : 0;
            factor->factor->solveRefined(b, ldb, x, ldx, columns, false, tolerance, steps, info, krylov);
        });
}

extern "C" int oosgpu_solve_refined_device(oosgpu_factor* factor, const double* b, int64_t ldb, double* x, int64_t ldx,
                                           int64_t columns, const oosgpu_refine_options* options,
                                           oosgpu_refine_info* info)
{
    return guarded(
        [&]
        {
            requirePointer(factor, "factor");
            const double tolerance = options != nullptr ? options->tolerance : 1.0e-10;
            const int steps = options != nullptr ? options->max_steps : 10;
            const int krylov = options != nullptr ? options->krylov : 0;
            factor->factor->solveRefined(b, ldb, x, ldx, columns, true, tolerance, steps, info, krylov);
        });
}

extern "C" int oosgpu_pencil_create(const oosgpu_symbolic* symbolic, int device, int32_t dimension,
                                    const int64_t* col_offsets, const int32_t* rows, const double* stiffness,
                                    const double* mass, oosgpu_pencil** out)
{
    return guarded(
        [&]
        {
            requirePointer(symbolic, "symbolic");
            requirePointer(col_offsets, "col_offsets");
            requirePointer(rows, "rows");
            requirePointer(stiffness, "stiffness");
            requirePointer(mass, "mass");
            requirePointer(out, "out");
            auto handle = std::make_unique<oosgpu_pencil>();
            handle->pencil = std::make_unique<oosgpu::GpuPencil>(symbolic->symbolic, device, dimension, col_offsets,
                                                                 rows, stiffness, mass, false, planOf(symbolic));
            *out = handle.release();
        });
}

extern "C" int oosgpu_pencil_create_buckling(const oosgpu_symbolic* symbolic, int device, int32_t dimension,
                                             const int64_t* col_offsets, const int32_t* rows, const double* stiffness,
                                             const double* differential, oosgpu_pencil** out)
{
    return guarded(
        [&]
        {
            requirePointer(symbolic, "symbolic");
            requirePointer(col_offsets, "col_offsets");
            requirePointer(rows, "rows");
            requirePointer(stiffness, "stiffness");
            requirePointer(differential, "differential");
            requirePointer(out, "out");
            auto handle = std::make_unique<oosgpu_pencil>();
            handle->pencil = std::make_unique<oosgpu::GpuPencil>(symbolic->symbolic, device, dimension, col_offsets,
                                                                 rows, stiffness, differential, true,
                                                                 planOf(symbolic));
            *out = handle.release();
        });
}

extern "C" void oosgpu_pencil_destroy(oosgpu_pencil* pencil)
{
    delete pencil;
}

extern "C" void* oosgpu_pencil_stream(oosgpu_pencil* pencil)
{
    return pencil == nullptr ? nullptr : static_cast<void*>(pencil->pencil->stream());
}

extern "C" int oosgpu_pencil_factorise(oosgpu_pencil* pencil, double shift, oosgpu_factor_info* info)
{
    return guarded(
        [&]
        {
            requirePointer(pencil, "pencil");
            const oosgpu_factor_info result = pencil->pencil->factorise(shift);
            if (info != nullptr)
                *info = result;
        });
}

extern "C" int oosgpu_pencil_solve_device(oosgpu_pencil* pencil, double* x, int64_t ld, int64_t columns)
{
    return guarded(
        [&]
        {
            requirePointer(pencil, "pencil");
            pencil->pencil->solve(x, ld, columns);
        });
}

extern "C" int oosgpu_pencil_multiply_mass_device(oosgpu_pencil* pencil, const double* x, int64_t ldx, double* y,
                                                  int64_t ldy, int64_t columns)
{
    return guarded(
        [&]
        {
            requirePointer(pencil, "pencil");
            pencil->pencil->multiplyMass(x, ldx, y, ldy, columns);
            oosgpu::check(cudaStreamSynchronize(pencil->pencil->stream()), "mass product");
        });
}

extern "C" int oosgpu_pencil_properties(const oosgpu_pencil* pencil, double* rayleigh_bound, int32_t* lumped,
                                        int64_t* factorisations)
{
    return guarded(
        [&]
        {
            requirePointer(pencil, "pencil");
            if (rayleigh_bound != nullptr)
                *rayleigh_bound = pencil->pencil->rayleighBound();
            if (lumped != nullptr)
                *lumped = pencil->pencil->lumped() ? 1 : 0;
            if (factorisations != nullptr)
                *factorisations = pencil->pencil->factorisations();
        });
}

extern "C" void oosgpu_lanczos_defaults(oosgpu_lanczos_options* options)
{
    if (options == nullptr)
        return;
    const oosgpu::eigen::KrylovSettings defaults;
    options->block_size = static_cast<int64_t>(defaults.block);
    options->modes_per_shift = static_cast<int64_t>(defaults.modesPerShift);
    options->convergence_tolerance = defaults.tolerance;
    options->maximum_shifts = static_cast<int64_t>(defaults.shiftLimit);
    options->maximum_restarts = static_cast<int64_t>(defaults.restartLimit);
    options->seed = defaults.seed;
}

namespace
{

int modesSolve(oosgpu_pencil* pencil, const oosgpu_eigen_request* request, const oosgpu_lanczos_options* options,
               const double* start, int64_t ld, int64_t columns, oosgpu_modes** out)
{
    return guarded(
        [&]
        {
            requirePointer(pencil, "pencil");
            requirePointer(request, "request");
            requirePointer(out, "out");
            *out = nullptr;
            if (request->mode_count < 0)
                throw oosgpu::Error(oosgpu::STATUS_INVALID_ARGUMENT, "eigenvalue request: a negative mode count");
            oosgpu::eigen::ModeRequest eigenRequest;
            eigenRequest.low = request->lower_bound;
            eigenRequest.high = request->upper_bound;
            eigenRequest.count = static_cast<std::size_t>(request->mode_count);
            oosgpu::eigen::KrylovSettings lanczos;
            if (options != nullptr)
            {
                const auto count = [](int64_t value, const char* what)
                {
                    if (value < 0)
                        throw oosgpu::Error(oosgpu::STATUS_INVALID_ARGUMENT,
                                            std::string("BlockLanczos: a negative ") + what);
                    return static_cast<std::size_t>(value);
                };
                lanczos.block = count(options->block_size, "block size");
                lanczos.modesPerShift = count(options->modes_per_shift, "count of modes per shift");
                lanczos.tolerance = options->convergence_tolerance;
                lanczos.shiftLimit = count(options->maximum_shifts, "shift limit");
                lanczos.restartLimit = count(options->maximum_restarts, "restart limit");
                lanczos.seed = options->seed;
            }
            if (start != nullptr)
            {
                const int64_t n = pencil->pencil->factor().plan().dimension;
                if (columns != static_cast<int64_t>(lanczos.block) || ld < n)
                    throw oosgpu::Error(oosgpu::STATUS_INVALID_ARGUMENT,
                                        "learned start: expected a start block of " + std::to_string(n) + " rows (ld >= "
                                        "rows) and the block size's " + std::to_string(lanczos.block) +
                                        " columns, found " + std::to_string(columns) + " columns, ld " +
                                        std::to_string(ld));
            }
            oosgpu::check(cudaSetDevice(pencil->pencil->factor().deviceOrdinal()), "cudaSetDevice");
            oosgpu::PencilOperations operations(*pencil->pencil);
            auto handle = std::make_unique<oosgpu_modes>();
            if (pencil->pencil->buckling())
            {
                if (start != nullptr)
                    throw oosgpu::Error(oosgpu::STATUS_INVALID_ARGUMENT,
                                        "learned start: a buckling pencil takes no start block");
                handle->solution = oosgpu::eigen::solveBuckling(operations, eigenRequest, lanczos);
            }
            else
                handle->solution = oosgpu::eigen::solveModes(operations, eigenRequest, lanczos, start, ld);
            *out = handle.release();
        });
}

} // namespace

extern "C" int oosgpu_modes_solve(oosgpu_pencil* pencil, const oosgpu_eigen_request* request,
                                  const oosgpu_lanczos_options* options, oosgpu_modes** out)
{
    return modesSolve(pencil, request, options, nullptr, 0, 0, out);
}

extern "C" int oosgpu_modes_solve_start(oosgpu_pencil* pencil, const oosgpu_eigen_request* request,
                                        const oosgpu_lanczos_options* options, const double* start, int64_t ld,
                                        int64_t columns, oosgpu_modes** out)
{
    if (start == nullptr)
        return modesSolve(pencil, request, options, nullptr, 0, 0, out);
    return modesSolve(pencil, request, options, start, ld, columns, out);
}

extern "C" int oosgpu_modes_summary(const oosgpu_modes* modes, int64_t counts[6], double seconds[6])
{
    return guarded(
        [&]
        {
            requirePointer(modes, "modes");
            const auto& s = modes->solution;
            if (counts != nullptr)
            {
                counts[0] = static_cast<int64_t>(s.values.size());
                counts[1] = static_cast<int64_t>(s.factorisations);
                counts[2] = static_cast<int64_t>(s.shifts.size());
                counts[3] = static_cast<int64_t>(s.confirmed);
                counts[4] = s.complete ? 1 : 0;
                counts[5] = static_cast<int64_t>(s.blockSteps);
            }
            if (seconds != nullptr)
            {
                seconds[0] = s.seconds;
                seconds[1] = s.factorSeconds;
                seconds[2] = s.factorWallSeconds;
                seconds[3] = s.operatorSeconds;
                seconds[4] = s.orthogonalisationSeconds;
                seconds[5] = s.projectedSeconds;
            }
        });
}

extern "C" int oosgpu_modes_work(const oosgpu_modes* modes, int64_t counts[2], double seconds[7])
{
    return guarded(
        [&]
        {
            requirePointer(modes, "modes");
            const auto& s = modes->solution;
            if (counts != nullptr)
            {
                counts[0] = static_cast<int64_t>(s.hostBlocks);
                counts[1] = static_cast<int64_t>(s.replacementSolves);
            }
            if (seconds != nullptr)
            {
                std::copy(s.orthogonalisationParts.begin(), s.orthogonalisationParts.end(), seconds);
                std::copy(s.outsideParts.begin(), s.outsideParts.end(), seconds + 4);
            }
        });
}

extern "C" int oosgpu_modes_values(const oosgpu_modes* modes, double* eigenvalues, double* residual_bounds)
{
    return guarded(
        [&]
        {
            requirePointer(modes, "modes");
            const auto& s = modes->solution;
            if (eigenvalues != nullptr)
                std::copy(s.values.begin(), s.values.end(), eigenvalues);
            if (residual_bounds != nullptr)
                std::copy(s.residualBounds.begin(), s.residualBounds.end(), residual_bounds);
        });
}

extern "C" int oosgpu_modes_vectors(const oosgpu_modes* modes, double* vectors, int64_t ld)
{
    return guarded(
        [&]
        {
            requirePointer(modes, "modes");
            requirePointer(vectors, "vectors");
            const auto& s = modes->solution;
            if (ld < s.dimension)
                throw oosgpu::Error(oosgpu::STATUS_INVALID_ARGUMENT, "modes: the leading dimension is below the rows");
            if (s.values.empty() || s.dimension == 0)
                return;
            oosgpu::check(cudaMemcpy2D(vectors, static_cast<std::size_t>(ld) * sizeof(double), s.vectors.get(),
                                       static_cast<std::size_t>(s.dimension) * sizeof(double),
                                       static_cast<std::size_t>(s.dimension) * sizeof(double), s.values.size(),
                                       cudaMemcpyDeviceToHost),
                          "download eigenvectors");
        });
}

extern "C" const double* oosgpu_modes_vectors_device(const oosgpu_modes* modes)
{
    return modes == nullptr ? nullptr : modes->solution.vectors.get();
}

extern "C" int oosgpu_modes_shifts(const oosgpu_modes* modes, double* records)
{
    return guarded(
        [&]
        {
            requirePointer(modes, "modes");
            requirePointer(records, "records");
            std::size_t k = 0;
            for (const auto& record : modes->solution.shifts)
            {
                double* out = records + 7 * k++;
                out[0] = record.shift;
                out[1] = static_cast<double>(static_cast<int>(record.role));
                out[2] = static_cast<double>(record.countBelow);
                out[3] = record.ran ? 1.0 : 0.0;
                out[4] = static_cast<double>(record.blockSteps);
                out[5] = static_cast<double>(record.restarts);
                out[6] = static_cast<double>(record.converged);
            }
        });
}

extern "C" void oosgpu_modes_destroy(oosgpu_modes* modes)
{
    delete modes;
}

namespace
{

oosgpu::eigen::Confirmation confirmationFrom(const double v[6])
{
    oosgpu::eigen::Confirmation confirmation;
    confirmation.reach = v[0];
    confirmation.confirmed = static_cast<std::size_t>(v[1]);
    confirmation.hasGap = v[2] != 0.0;
    confirmation.gapLow = v[3];
    confirmation.gapHigh = v[4];
    return confirmation;
}

std::span<const double> valuesOf(const double* values, int64_t count, const char* name)
{
    if (count < 0)
        throw oosgpu::Error(oosgpu::STATUS_INVALID_ARGUMENT, std::string(name) + ": a negative count");
    if (count > 0)
        requirePointer(values, name);
    return {values, static_cast<std::size_t>(count)};
}

} // namespace

extern "C" int oosgpu_symmetric_eigen(const double* a, int64_t p, int64_t ld, double* eigenvalues,
                                      double* eigenvectors)
{
    return guarded(
        [&]
        {
            if (p < 0 || ld < std::max<int64_t>(p, 1))
                throw oosgpu::Error(oosgpu::STATUS_INVALID_ARGUMENT,
                                    "symmetric eigenproblem: expected an order >= 0 and a leading dimension >= it");
            if (p == 0)
                return;
            requirePointer(a, "a");
            requirePointer(eigenvalues, "eigenvalues");
            requirePointer(eigenvectors, "eigenvectors");
            std::vector<double> values;
            std::vector<double> vectors;
            oosgpu::eigen::decomposeSymmetric(a, static_cast<std::size_t>(p), static_cast<std::size_t>(ld), values,
                                              vectors);
            std::copy(values.begin(), values.end(), eigenvalues);
            std::copy(vectors.begin(), vectors.end(), eigenvectors);
        });
}

extern "C" int oosgpu_sturm_verify(int64_t points, const double* shifts, const int64_t* counts, int64_t values,
                                   const double* sorted, double result[6])
{
    return guarded(
        [&]
        {
            requirePointer(result, "result");
            const std::span<const double> shiftSpan = valuesOf(shifts, points, "shifts");
            if (points > 0)
                requirePointer(counts, "counts");
            oosgpu::eigen::CountLedger ledger;
            for (std::size_t k = 0; k < shiftSpan.size(); ++k)
            {
                if (counts[k] < 0)
                    throw oosgpu::Error(oosgpu::STATUS_INVALID_ARGUMENT, "Sturm point: a negative count");
                ledger.record(shiftSpan[k], static_cast<std::size_t>(counts[k]));
            }
            const oosgpu::eigen::Confirmation c = ledger.confirm(valuesOf(sorted, values, "sorted"));
            result[0] = c.reach;
            result[1] = static_cast<double>(c.confirmed);
            result[2] = c.hasGap ? 1.0 : 0.0;
            result[3] = c.gapLow;
            result[4] = c.gapHigh;
            result[5] = static_cast<double>(c.proven) * 1e6 + static_cast<double>(c.found);
        });
}

extern "C" int oosgpu_shift_next(double lower, double upper, int64_t mode_count, double scale,
                                 const double verification[6], int64_t values, const double* sorted,
                                 int64_t ritz_count, const double* ritz, int64_t shift_count,
                                 const double* lanczos_shifts, double* shift, int32_t* purpose)
{
    return guarded(
        [&]
        {
            requirePointer(verification, "verification");
            requirePointer(shift, "shift");
            requirePointer(purpose, "purpose");
            if (mode_count < 0)
                throw oosgpu::Error(oosgpu::STATUS_INVALID_ARGUMENT, "eigenvalue request: a negative mode count");
            oosgpu::eigen::ModeRequest request;
            request.low = lower;
            request.high = upper;
            request.count = static_cast<std::size_t>(mode_count);
            const oosgpu::eigen::ShiftPlanner planner(request, scale);
            const oosgpu::eigen::ShiftPick pick = planner.next(
                confirmationFrom(verification), valuesOf(sorted, values, "sorted"), valuesOf(ritz, ritz_count, "ritz"),
                valuesOf(lanczos_shifts, shift_count, "lanczos shifts"));
            *shift = pick.shift;
            *purpose = static_cast<int32_t>(pick.role);
        });
}
