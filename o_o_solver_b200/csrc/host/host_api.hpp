// Host-side C++ types of the library: the workload models, the symbolic structure the factorisation runs on and
// the errors that the C ABI turns into status codes.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace oosgpu
{

// Status codes of the C ABI (include/oos_gpu.h), one per exception class of the reference's boundary.
enum Status : int
{
    STATUS_OK = 0,
    STATUS_INVALID_ARGUMENT = 1, // std::invalid_argument
    STATUS_MEMORY_BUDGET = 2,    // base::MemoryBudgetError
    STATUS_SINGULAR = 3,         // base::SingularityError
    STATUS_CANCELLED = 4,        // base::OperationCancelledError
    STATUS_CUDA = 5,             // a CUDA runtime error
    STATUS_INTERNAL = 6,         // base::InternalError
    STATUS_NOT_FACTORISED = 7,   // std::logic_error: a solve before a factorisation
    STATUS_SOLVER = 8            // base::SolverError (Lanczos: contradicting Sturm counts, no usable shift)
};

// An error carrying its C-ABI status.
class Error : public std::runtime_error
{
public:
    Error(Status status, const std::string& message) : std::runtime_error(message), m_status(status) {}
    [[nodiscard]] Status status() const noexcept { return m_status; }

private:
    Status m_status;
};

// A structured finite-element model: free nodes, their graph, node-block stiffness, lumped mass and loads.
class Model
{
public:
    Model();

    // A flat plate nx by ny rectangular shells of lx by ly, clamped along x = 0.
    [[nodiscard]] static Model plate(std::int32_t nx, std::int32_t ny, double lx, double ly, double thickness,
                                     double young, double poisson, double pressure);
    // A cube of n^3 trilinear hexahedra of edge `edge`, clamped on its base z = 0, lumped mass.
    [[nodiscard]] static Model hexBlock(std::int32_t n, double edge, double young, double poisson, double density);
    // A square skin of n x n shells of lx by ly, clamped along x = 0, stiffened by `stringers` blades along x (on the
    // grid lines y = k ly / (stringers + 1), rounded to the grid), each a Euler-Bernoulli frame element per skin edge
    // on the skin's mid-plane with a blade section of the given height and thickness.
    [[nodiscard]] static Model stiffenedPanel(std::int32_t n, double lx, double ly, double thickness, double young,
                                              double poisson, std::int32_t stringers, double bladeHeight,
                                              double bladeThickness, double pressure);
    // A rectangular wing box of flat shells of size h: skins z = 0 and z = height over chord (x) by span (y), spars
    // x = 0 and x = chord, ribs every ribPitch along the span; clamped at the root y = 0; lumped mass (translations
    // rho t A / 4, rotations rho t^3 A / 48 per node of each element). thicknesses: 24 zone thicknesses (upper skin
    // 8 spanwise zones, lower skin 8, front spar 4, rear spar 4); ribs ribThickness.
    [[nodiscard]] static Model wingBox(double span, double chord, double height, double ribPitch, double h,
                                       const double* thicknesses, double ribThickness, double young, double poisson,
                                       double density);

    [[nodiscard]] std::int32_t nodeCount() const noexcept { return m_nodeCount; }
    [[nodiscard]] int nodeDofs() const noexcept { return m_nodeDofs; }
    [[nodiscard]] const std::vector<std::int64_t>& offsets() const noexcept { return m_offsets; }
    [[nodiscard]] const std::vector<std::int32_t>& neighbours() const noexcept { return m_neighbours; }
    [[nodiscard]] const std::vector<double>& coordinates() const noexcept { return m_coordinates; }
    [[nodiscard]] const std::vector<std::int32_t>& gridIndex() const noexcept { return m_gridIndex; }

    void firstColumns(const std::int32_t* nodeAtPosition, std::int32_t* firstColumnOfPosition) const;
    [[nodiscard]] std::int64_t cscTermCount(const std::int32_t* nodeAtPosition) const;
    void toCsc(const std::int32_t* nodeAtPosition, int which, std::int64_t* offsets, std::int32_t* rows,
               double* values) const;
    void loads(const std::int32_t* nodeAtPosition, std::int64_t columns, std::uint64_t seedBase,
               std::int32_t pointsPerPattern, double sigma, double* rhs, std::int64_t ld) const;
    // toCsc on the GPU (model_kernels.cu): the element matrices computed there, the node blocks assembled there in
    // the host's order (so the same values), the columns written there. offsets (dimension + 1), rows and values
    // (cscTermCount) are device arrays; the call returns when they are written.
    void toCscOnDevice(const std::int32_t* nodeAtPosition, int which, std::int64_t* offsets, std::int32_t* rows,
                       double* values) const;

    // One kind of element matrix: a flat shell (a x b, thickness, E, nu, turned into the global axes by one of three
    // orientations), a trilinear hexahedron (edge, E, nu), or a matrix given by the host (row-major, dofs x dofs).
    struct ElementKind
    {
        int family = 0; // 0 shell, 1 hexahedron, 2 given
        double a = 0.0, b = 0.0, thickness = 0.0, young = 0.0, poisson = 0.0;
        int orientation = 0;
        int dofs = 24;
        std::vector<double> given;
    };

private:
    // The element list the device assembly works from: nodes of element e at m_elementStart[e] (-1 for a clamped
    // node), its kind m_elementKind[e]; kinds in m_kinds.
    int addKind(const ElementKind& kind);
    void recordElement(const std::vector<std::int32_t>& nodes, int kind);
    std::vector<std::int64_t> m_elementStart{0};
    std::vector<std::int32_t> m_elementNodes;
    std::vector<std::int32_t> m_elementKind;
    std::vector<ElementKind> m_kinds;

    void buildGraph(const std::vector<std::vector<std::int32_t>>& elements);
    // Adds an element matrix (nodes.size() x nodeDofs square, row-major) into the node blocks (after clearBlocks).
    void clearBlocks();
    void addElement(const std::vector<std::int32_t>& nodes, const double* elementMatrix);
    void assemble(const std::vector<std::vector<std::int32_t>>& elements, const double* elementMatrix, int nodeDofs);
    [[nodiscard]] std::int64_t slot(std::int32_t node, std::int32_t neighbour) const;

    std::int32_t m_nodeCount = 0;
    int m_nodeDofs = 0;
    std::vector<std::int64_t> m_offsets;
    std::vector<std::int32_t> m_neighbours;
    std::vector<double> m_coordinates;
    std::vector<std::int32_t> m_gridIndex;
    std::vector<std::vector<std::int32_t>> m_elementsOfNode;
    std::vector<double> m_diagonalBlocks;
    std::vector<double> m_offBlocks;
    std::vector<double> m_lumpedMass;
    std::vector<double> m_pressureLoad;
};

// The symbolic structure of a factorisation as the reference's SymbolicFactor exposes it
// (include/oos/linalg/symbolic/SymbolicFactor.hpp:37-126): supernode s owns the DOF columns
// [firstColumn[s], firstColumn[s + 1]), its rows below them are rows[rowStart[s] .. rowStart[s + 1]) ascending, and
// parent[s] is -1 for a root. Children come before their parents.
struct Symbolic
{
    std::int32_t dofCount = 0;
    std::int32_t supernodeCount = 0;
    std::vector<std::int32_t> firstColumn; // supernodeCount + 1
    std::vector<std::int32_t> parent;      // supernodeCount
    std::vector<std::int64_t> rowStart;    // supernodeCount + 1
    std::vector<std::int32_t> rows;

    [[nodiscard]] std::int32_t columnCount(std::int32_t s) const noexcept
    {
        return firstColumn[static_cast<std::size_t>(s) + 1] - firstColumn[static_cast<std::size_t>(s)];
    }
    [[nodiscard]] std::int32_t rowCount(std::int32_t s) const noexcept
    {
        return static_cast<std::int32_t>(rowStart[static_cast<std::size_t>(s) + 1] - rowStart[static_cast<std::size_t>(s)]);
    }

    // Checks the invariants the factorisation relies on; throws Error(STATUS_INVALID_ARGUMENT).
    void validate() const;
    // SymbolicFactor::flopCount (SymbolicFactor.hpp:97-99): per column with m entries below the diagonal,
    // m(m + 1) + 2m.
    [[nodiscard]] double flopCount() const;
    [[nodiscard]] std::int64_t panelValueCount() const;
    [[nodiscard]] std::int64_t factorEntryCount() const;
};

// The row structures of a supernode partition (SymbolicFactor.cpp:227-290): R(s) = (adjacency of the nodes of s
// union R(children)) beyond the last position of s, expanded to DOF rows. nodeAtPosition: the final node order;
// firstPosition: supernodeCount + 1 node positions; parent: per supernode.
Symbolic rowStructures(std::int32_t nodeCount, const std::int64_t* offsets, const std::int32_t* neighbours,
                       const std::int32_t* weights, const std::int32_t* nodeAtPosition, std::int32_t supernodeCount,
                       const std::int32_t* firstPosition, const std::int32_t* parent);

} // namespace oosgpu
