// Model::toCscOnDevice (declared in host_api.hpp): the stiffness (or the lumped mass on its pattern) of a workload
// model written by the GPU in the compressed-column form toCsc writes on the host, from the model's element list.
// The host uploads what describes the model (the graph, the elements, the element kinds, each node's elements); the
// element matrices, the node blocks and the columns are formed on the device (model_kernels.cu), with the host's
// arithmetic in the host's order: the same values bit for bit.

#include "../device/kernels.cuh"
#include "host_api.hpp"

#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <string>
#include <vector>

namespace oosgpu
{

namespace
{

void check(cudaError_t status, const char* what)
{
    if (status != cudaSuccess)
        throw Error(status == cudaErrorMemoryAllocation ? STATUS_MEMORY_BUDGET : STATUS_CUDA,
                    std::string("device assembly: ") + what + ": " + cudaGetErrorString(status));
}

// A scoped device array, filled from a host vector when given one.
template <typename T> class Scoped
{
public:
    explicit Scoped(std::size_t count) { check(cudaMalloc(&m_data, std::max<std::size_t>(count, 1) * sizeof(T)), "allocation"); }
    explicit Scoped(const std::vector<T>& host, cudaStream_t stream) : Scoped(host.size())
    {
        if (!host.empty())
            check(cudaMemcpyAsync(m_data, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice, stream),
                  "upload");
    }
    Scoped(const Scoped&) = delete;
    Scoped& operator=(const Scoped&) = delete;
    ~Scoped() { cudaFree(m_data); }
    [[nodiscard]] T* get() const noexcept { return m_data; }

private:
    T* m_data = nullptr;
};

unsigned gridFor(std::int64_t items, int threads)
{
    return static_cast<unsigned>(std::max<std::int64_t>((items + threads - 1) / threads, 1));
}

} // namespace

void Model::toCscOnDevice(const std::int32_t* nodeAtPosition, int which, std::int64_t* offsets, std::int32_t* rows,
                          double* values) const
{
    if (which != 0 && which != 1)
        throw Error(STATUS_INVALID_ARGUMENT, "device assembly: which must be 0 (stiffness) or 1 (lumped mass)");
    if (which == 1 && m_lumpedMass.empty())
        throw Error(STATUS_INVALID_ARGUMENT, "device assembly: this model has no lumped mass");
    const std::int32_t nodes = m_nodeCount;
    const int w = m_nodeDofs;
    if (nodes == 0)
    {
        check(cudaMemset(offsets, 0, sizeof(std::int64_t)), "empty model");
        return;
    }
    for (std::int32_t a = 0; a < nodes; ++a)
        if (m_offsets[static_cast<std::size_t>(a) + 1] - m_offsets[static_cast<std::size_t>(a)] > 32)
            throw Error(STATUS_INVALID_ARGUMENT, "device assembly: a node with more than 32 neighbours");
    // each node's elements, in increasing element order (a counting sort of the element list)
    const auto elements = static_cast<std::int64_t>(m_elementKind.size());
    std::vector<std::int64_t> ofNodeStart(static_cast<std::size_t>(nodes) + 1, 0);
    for (std::int64_t e = 0; e < elements; ++e)
        for (std::int64_t t = m_elementStart[static_cast<std::size_t>(e)]; t < m_elementStart[static_cast<std::size_t>(e) + 1]; ++t)
            if (m_elementNodes[static_cast<std::size_t>(t)] >= 0)
                ++ofNodeStart[static_cast<std::size_t>(m_elementNodes[static_cast<std::size_t>(t)]) + 1];
    for (std::int32_t a = 0; a < nodes; ++a)
        ofNodeStart[static_cast<std::size_t>(a) + 1] += ofNodeStart[static_cast<std::size_t>(a)];
    std::vector<std::int32_t> ofNode(static_cast<std::size_t>(ofNodeStart.back()));
    std::vector<std::int64_t> next(ofNodeStart.begin(), ofNodeStart.end() - 1);
    for (std::int64_t e = 0; e < elements; ++e)
        for (std::int64_t t = m_elementStart[static_cast<std::size_t>(e)]; t < m_elementStart[static_cast<std::size_t>(e) + 1]; ++t)
        {
            const std::int32_t a = m_elementNodes[static_cast<std::size_t>(t)];
            if (a >= 0)
                ofNode[static_cast<std::size_t>(next[static_cast<std::size_t>(a)]++)] = static_cast<std::int32_t>(e);
        }
    // the kinds, the given matrices after one another
    std::vector<device::ElementKindDesc> kinds;
    std::vector<double> given;
    for (const ElementKind& k : m_kinds)
    {
        if (k.dofs > 24 || k.dofs < 1)
            throw Error(STATUS_INTERNAL, "device assembly: an element kind beyond 24 DOFs");
        kinds.push_back({k.family, k.orientation, k.dofs, static_cast<int>(given.size()), k.a, k.b, k.thickness,
                         k.young, k.poisson});
        given.insert(given.end(), k.given.begin(), k.given.end());
    }

    cudaStream_t stream = nullptr;
    check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "stream");
    struct StreamGuard
    {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } guard{stream};
    const Scoped<device::ElementKindDesc> dKinds(kinds, stream);
    const Scoped<double> dGiven(given, stream);
    const Scoped<double> dMatrices(kinds.size() * 576);
    const Scoped<std::int64_t> dGraphOffsets(m_offsets, stream);
    const Scoped<std::int32_t> dNeighbours(m_neighbours, stream);
    const Scoped<std::int64_t> dElementStart(m_elementStart, stream);
    const Scoped<std::int32_t> dElementNodes(m_elementNodes, stream);
    const Scoped<std::int32_t> dElementKind(m_elementKind, stream);
    const Scoped<std::int64_t> dOfNodeStart(ofNodeStart, stream);
    const Scoped<std::int32_t> dOfNode(ofNode, stream);
    const std::vector<std::int32_t> order(nodeAtPosition, nodeAtPosition + nodes);
    const Scoped<std::int32_t> dOrder(order, stream);
    const Scoped<std::int32_t> dPosition(static_cast<std::size_t>(nodes));
    const Scoped<double> dMass(which == 1 ? m_lumpedMass : std::vector<double>{}, stream);
    const auto slots = static_cast<std::int64_t>(m_neighbours.size());
    const Scoped<double> dDiagonal(static_cast<std::size_t>(nodes) * w * w);
    const Scoped<double> dOff(static_cast<std::size_t>(std::max<std::int64_t>(slots, 1)) * w * w);
    const Scoped<std::int64_t> dTerms(static_cast<std::size_t>(nodes));
    const Scoped<std::int64_t> dStart(static_cast<std::size_t>(nodes));

    const device::ModelArgs m{nodes,          w,           slots,           dGraphOffsets.get(), dNeighbours.get(),
                              dElementStart.get(), dElementNodes.get(), dElementKind.get(), dOfNodeStart.get(),
                              dOfNode.get(),  dMatrices.get()};
    if (!kinds.empty())
        device::elementMatrices<<<static_cast<unsigned>(kinds.size()), 576, 0, stream>>>(dKinds.get(), dGiven.get(),
                                                                                          dMatrices.get());
    device::nodeBlocks<<<gridFor(nodes + slots, 256), 256, 0, stream>>>(m, dDiagonal.get(), dOff.get());
    device::scatterPositions<<<gridFor(nodes, 256), 256, 0, stream>>>(dOrder.get(), dPosition.get(), nodes);
    device::cscCounts<<<gridFor(nodes, 256), 256, 0, stream>>>(m, dOrder.get(), dPosition.get(), dTerms.get());
    check(cudaGetLastError(), "kernel launch");
    std::size_t scratchBytes = 0;
    check(cub::DeviceScan::ExclusiveSum(nullptr, scratchBytes, dTerms.get(), dStart.get(), nodes, stream), "scan size");
    const Scoped<unsigned char> scratch(scratchBytes);
    check(cub::DeviceScan::ExclusiveSum(scratch.get(), scratchBytes, dTerms.get(), dStart.get(), nodes, stream), "scan");
    device::cscFill<<<gridFor(nodes, 128), 128, 0, stream>>>(m, dOrder.get(), dPosition.get(), dStart.get(),
                                                             dDiagonal.get(), dOff.get(), dMass.get(), which, offsets,
                                                             rows, values);
    check(cudaGetLastError(), "kernel launch");
    check(cudaStreamSynchronize(stream), "assembly");
}

} // namespace oosgpu
