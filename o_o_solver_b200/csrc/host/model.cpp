// Model-side generators of the workloads the solver is measured on: structured meshes of flat-shell quadrilaterals
// (a plate clamped along one edge) and of trilinear hexahedra (a block clamped on its base), their node graphs, their
// stiffness (and lumped mass) as node blocks, and the conversion of those blocks into the lower-triangle compressed
// columns the factorisation takes, in the order of a symbolic factor.
//
// These stand in for the reference's assembly and DOF selection, which lie outside the factorisation's boundary:
// the node graph has the same shape as NodeGraph (src/linalg/ordering/NodeGraph.cpp: sorted, distinct, symmetric
// neighbours), the conversion follows SymmetricCsc::fromBlocks (src/linalg/sparse/SymmetricCsc.cpp:41-200: the kept
// DOFs of a node consecutive in the factor's order, every term of a stored node block kept even when zero, each column
// ascending from its diagonal). The element formulations are this project's own (a rectangular flat shell made of a
// bilinear membrane, MITC4 Mindlin-Reissner bending and a small drilling spring; a fully integrated trilinear hexahedron
// with lumped mass), not the reference's ShellQuad4 and SolidHexa: the factorisation is indifferent to the formulation,
// and the parity of the GPU path is judged on the same matrix given to both.

#include "host_api.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <vector>

namespace oosgpu
{
namespace
{

// 2x2 Gauss points on [-1, 1].
constexpr double GAUSS = 0.57735026918962576451;

// ---------------------------------------------------------------------------------------------------------------
// Rectangular flat shell, 4 nodes x 6 DOFs (u, v, w, rx, ry, rz), element a (x) by b (y). Rotations follow the right
// hand: the slopes are w,x = -ry ... written here with the displacement field u = u0 + z*ry, v = v0 - z*rx.
// ---------------------------------------------------------------------------------------------------------------
constexpr int SHELL_DOFS = 24;
constexpr double NODE_XI[4] = {-1.0, 1.0, 1.0, -1.0};
constexpr double NODE_ETA[4] = {-1.0, -1.0, 1.0, 1.0};

void addBtDB(double* k, int n, const double* b, int rows, const double* d)
{
    // k += B^T D B (b: rows x n row-major, d: rows x rows row-major)
    std::vector<double> db(static_cast<std::size_t>(rows) * n, 0.0);
    for (int r = 0; r < rows; ++r)
        for (int c = 0; c < n; ++c)
        {
            double s = 0.0;
            for (int q = 0; q < rows; ++q)
                s += d[r * rows + q] * b[q * n + c];
            db[static_cast<std::size_t>(r) * n + c] = s;
        }
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
        {
            double s = 0.0;
            for (int r = 0; r < rows; ++r)
                s += b[r * n + i] * db[static_cast<std::size_t>(r) * n + j];
            k[i * n + j] += s;
        }
}

void shellShape(double xi, double eta, double a, double b, double n[4], double dx[4], double dy[4])
{
    for (int i = 0; i < 4; ++i)
    {
        n[i] = 0.25 * (1.0 + xi * NODE_XI[i]) * (1.0 + eta * NODE_ETA[i]);
        dx[i] = 0.25 * NODE_XI[i] * (1.0 + eta * NODE_ETA[i]) * (2.0 / a);
        dy[i] = 0.25 * NODE_ETA[i] * (1.0 + xi * NODE_XI[i]) * (2.0 / b);
    }
}

// The transverse shear strains (gxz, gyz) of the displacement interpolation at (xi, eta), as rows over the 24 DOFs.
void shearRows(double xi, double eta, double a, double b, double* gxz, double* gyz)
{
    double n[4], dx[4], dy[4];
    shellShape(xi, eta, a, b, n, dx, dy);
    std::fill_n(gxz, SHELL_DOFS, 0.0);
    std::fill_n(gyz, SHELL_DOFS, 0.0);
    for (int i = 0; i < 4; ++i)
    {
        gxz[6 * i + 2] = dx[i];
        gxz[6 * i + 4] = n[i];
        gyz[6 * i + 2] = dy[i];
        gyz[6 * i + 3] = -n[i];
    }
}

void shellStiffness(double a, double b, double t, double young, double poisson, double* k)
{
    std::fill_n(k, SHELL_DOFS * SHELL_DOFS, 0.0);
    const double membrane = young * t / (1.0 - poisson * poisson);
    const double bending = young * t * t * t / (12.0 * (1.0 - poisson * poisson));
    const double shear = (5.0 / 6.0) * young / (2.0 * (1.0 + poisson)) * t;
    const double dm[9] = {membrane, membrane * poisson, 0, membrane * poisson, membrane, 0, 0, 0,
                          membrane * (1.0 - poisson) / 2.0};
    const double db[9] = {bending, bending * poisson, 0, bending * poisson, bending, 0, 0, 0,
                          bending * (1.0 - poisson) / 2.0};
    const double ds[4] = {shear, 0, 0, shear};
    const double detJ = a * b / 4.0;
    // MITC4 tying points: gxz at (0, +1) and (0, -1), gyz at (+1, 0) and (-1, 0).
    double gxzA[SHELL_DOFS], gxzC[SHELL_DOFS], gyzD[SHELL_DOFS], gyzB[SHELL_DOFS], unused[SHELL_DOFS];
    shearRows(0.0, 1.0, a, b, gxzA, unused);
    shearRows(0.0, -1.0, a, b, gxzC, unused);
    shearRows(1.0, 0.0, a, b, unused, gyzD);
    shearRows(-1.0, 0.0, a, b, unused, gyzB);
    for (int gx = 0; gx < 2; ++gx)
        for (int gy = 0; gy < 2; ++gy)
        {
            const double xi = gx == 0 ? -GAUSS : GAUSS;
            const double eta = gy == 0 ? -GAUSS : GAUSS;
            double n[4], dx[4], dy[4];
            shellShape(xi, eta, a, b, n, dx, dy);
            double bm[3 * SHELL_DOFS] = {};
            double bb[3 * SHELL_DOFS] = {};
            double bs[2 * SHELL_DOFS] = {};
            for (int i = 0; i < 4; ++i)
            {
                bm[0 * SHELL_DOFS + 6 * i + 0] = dx[i];
                bm[1 * SHELL_DOFS + 6 * i + 1] = dy[i];
                bm[2 * SHELL_DOFS + 6 * i + 0] = dy[i];
                bm[2 * SHELL_DOFS + 6 * i + 1] = dx[i];
                bb[0 * SHELL_DOFS + 6 * i + 4] = dx[i];
                bb[1 * SHELL_DOFS + 6 * i + 3] = -dy[i];
                bb[2 * SHELL_DOFS + 6 * i + 4] = dy[i];
                bb[2 * SHELL_DOFS + 6 * i + 3] = -dx[i];
            }
            for (int c = 0; c < SHELL_DOFS; ++c)
            {
                bs[c] = 0.5 * (1.0 + eta) * gxzA[c] + 0.5 * (1.0 - eta) * gxzC[c];
                bs[SHELL_DOFS + c] = 0.5 * (1.0 + xi) * gyzD[c] + 0.5 * (1.0 - xi) * gyzB[c];
            }
            double w[9];
            for (int q = 0; q < 9; ++q)
                w[q] = dm[q] * detJ;
            addBtDB(k, SHELL_DOFS, bm, 3, w);
            for (int q = 0; q < 9; ++q)
                w[q] = db[q] * detJ;
            addBtDB(k, SHELL_DOFS, bb, 3, w);
            double s[4];
            for (int q = 0; q < 4; ++q)
                s[q] = ds[q] * detJ;
            addBtDB(k, SHELL_DOFS, bs, 2, s);
        }
    // Drilling: a spring on each in-plane rotation, a thousandth of the shear stiffness of the element's area.
    const double drilling = 1.0e-3 * shear * a * b / 4.0;
    for (int i = 0; i < 4; ++i)
        k[(6 * i + 5) * SHELL_DOFS + 6 * i + 5] += drilling;
}

// ---------------------------------------------------------------------------------------------------------------
// Trilinear hexahedron, 8 nodes x 3 DOFs, a cube of edge h, 2x2x2 Gauss.
// ---------------------------------------------------------------------------------------------------------------
constexpr int HEX_DOFS = 24;
constexpr double HX[8] = {-1, 1, 1, -1, -1, 1, 1, -1};
constexpr double HY[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
constexpr double HZ[8] = {-1, -1, -1, -1, 1, 1, 1, 1};

void hexStiffness(double h, double young, double poisson, double* k)
{
    std::fill_n(k, HEX_DOFS * HEX_DOFS, 0.0);
    const double lambda = young * poisson / ((1.0 + poisson) * (1.0 - 2.0 * poisson));
    const double mu = young / (2.0 * (1.0 + poisson));
    double d[36] = {};
    for (int i = 0; i < 3; ++i)
    {
        for (int j = 0; j < 3; ++j)
            d[i * 6 + j] = lambda;
        d[i * 6 + i] = lambda + 2.0 * mu;
        d[(i + 3) * 6 + (i + 3)] = mu;
    }
    const double detJ = h * h * h / 8.0;
    for (int g = 0; g < 8; ++g)
    {
        const double xi = (g & 1) ? GAUSS : -GAUSS;
        const double eta = (g & 2) ? GAUSS : -GAUSS;
        const double zeta = (g & 4) ? GAUSS : -GAUSS;
        double b[6 * HEX_DOFS] = {};
        for (int i = 0; i < 8; ++i)
        {
            const double dx = 0.125 * HX[i] * (1 + eta * HY[i]) * (1 + zeta * HZ[i]) * (2.0 / h);
            const double dy = 0.125 * HY[i] * (1 + xi * HX[i]) * (1 + zeta * HZ[i]) * (2.0 / h);
            const double dz = 0.125 * HZ[i] * (1 + xi * HX[i]) * (1 + eta * HY[i]) * (2.0 / h);
            b[0 * HEX_DOFS + 3 * i + 0] = dx;
            b[1 * HEX_DOFS + 3 * i + 1] = dy;
            b[2 * HEX_DOFS + 3 * i + 2] = dz;
            b[3 * HEX_DOFS + 3 * i + 0] = dy;
            b[3 * HEX_DOFS + 3 * i + 1] = dx;
            b[4 * HEX_DOFS + 3 * i + 1] = dz;
            b[4 * HEX_DOFS + 3 * i + 2] = dy;
            b[5 * HEX_DOFS + 3 * i + 0] = dz;
            b[5 * HEX_DOFS + 3 * i + 2] = dx;
        }
        double w[36];
        for (int q = 0; q < 36; ++q)
            w[q] = d[q] * detJ;
        addBtDB(k, HEX_DOFS, b, 6, w);
    }
}

std::uint64_t splitmix64(std::uint64_t& state)
{
    // Steele, Lea & Flood, "Fast splittable pseudorandom number generators" (OOPSLA 2014).
    std::uint64_t z = (state += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

double uniform01(std::uint64_t& state)
{
    return static_cast<double>(splitmix64(state) >> 11) * 0x1.0p-53;
}

} // namespace

Model::Model() = default;

int Model::addKind(const ElementKind& kind)
{
    m_kinds.push_back(kind);
    return static_cast<int>(m_kinds.size()) - 1;
}

void Model::recordElement(const std::vector<std::int32_t>& nodes, int kind)
{
    m_elementNodes.insert(m_elementNodes.end(), nodes.begin(), nodes.end());
    m_elementStart.push_back(static_cast<std::int64_t>(m_elementNodes.size()));
    m_elementKind.push_back(kind);
}

std::int64_t Model::slot(std::int32_t node, std::int32_t neighbour) const
{
    const auto begin = m_offsets.begin() + m_offsets[static_cast<std::size_t>(node)];
    const auto end = m_offsets.begin() + m_offsets[static_cast<std::size_t>(node) + 1];
    (void)begin;
    (void)end;
    const std::int32_t* first = m_neighbours.data() + m_offsets[static_cast<std::size_t>(node)];
    const std::int32_t* last = m_neighbours.data() + m_offsets[static_cast<std::size_t>(node) + 1];
    const std::int32_t* found = std::lower_bound(first, last, neighbour);
    if (found == last || *found != neighbour)
        return -1;
    return found - m_neighbours.data();
}

void Model::buildGraph(const std::vector<std::vector<std::int32_t>>& elements)
{
    // Node adjacency: two free nodes are adjacent when an element holds both.
    const auto count = static_cast<std::size_t>(m_nodeCount);
    std::vector<std::vector<std::int32_t>> adjacency(count);
    m_elementsOfNode.assign(count, {});
    for (std::size_t e = 0; e < elements.size(); ++e)
    {
        const auto& nodes = elements[e];
        for (const std::int32_t a : nodes)
        {
            if (a < 0)
                continue;
            m_elementsOfNode[static_cast<std::size_t>(a)].push_back(static_cast<std::int32_t>(e));
            for (const std::int32_t b : nodes)
                if (b >= 0 && b != a)
                    adjacency[static_cast<std::size_t>(a)].push_back(b);
        }
    }
    m_offsets.assign(count + 1, 0);
    m_neighbours.clear();
    for (std::size_t a = 0; a < count; ++a)
    {
        auto& list = adjacency[a];
        std::sort(list.begin(), list.end());
        list.erase(std::unique(list.begin(), list.end()), list.end());
        m_neighbours.insert(m_neighbours.end(), list.begin(), list.end());
        m_offsets[a + 1] = static_cast<std::int64_t>(m_neighbours.size());
    }
}

void Model::assemble(const std::vector<std::vector<std::int32_t>>& elements, const double* elementMatrix, int nodeDofs)
{
    // Node blocks: for each node a, its diagonal block then one block per neighbour (CSR order); each block is
    // w x w column-major, rows the DOFs of a, columns those of the other node. Assembled node by node (each node
    // writes its own blocks only).
    const auto w = static_cast<std::size_t>(nodeDofs);
    const std::size_t blockValues = w * w;
    const auto count = static_cast<std::size_t>(m_nodeCount);
    m_diagonalBlocks.assign(count * blockValues, 0.0);
    m_offBlocks.assign(m_neighbours.size() * blockValues, 0.0);
    const int elementDofs = static_cast<int>(elements.empty() ? 0 : elements[0].size()) * nodeDofs;
#pragma omp parallel for schedule(static)
    for (std::int64_t a = 0; a < static_cast<std::int64_t>(count); ++a)
    {
        for (const std::int32_t e : m_elementsOfNode[static_cast<std::size_t>(a)])
        {
            const auto& nodes = elements[static_cast<std::size_t>(e)];
            int local = -1;
            for (std::size_t i = 0; i < nodes.size(); ++i)
                if (nodes[i] == a)
                    local = static_cast<int>(i);
            for (std::size_t j = 0; j < nodes.size(); ++j)
            {
                const std::int32_t b = nodes[j];
                if (b < 0)
                    continue;
                double* block = b == a ? m_diagonalBlocks.data() + static_cast<std::size_t>(a) * blockValues
                                       : m_offBlocks.data() + static_cast<std::size_t>(slot(static_cast<std::int32_t>(a), b)) * blockValues;
                for (std::size_t cc = 0; cc < w; ++cc)
                    for (std::size_t rr = 0; rr < w; ++rr)
                        block[rr + cc * w] +=
                            elementMatrix[(static_cast<std::size_t>(local) * w + rr) * static_cast<std::size_t>(elementDofs) +
                                          j * w + cc];
            }
        }
    }
}

Model Model::plate(std::int32_t nx, std::int32_t ny, double lx, double ly, double thickness, double young,
                   double poisson, double pressure)
{
    if (nx < 1 || ny < 1 || !(lx > 0) || !(ly > 0) || !(thickness > 0) || !(young > 0) || !(poisson > -1.0 && poisson < 0.5))
        throw std::invalid_argument("plate model: expected nx, ny >= 1 and positive dimensions and material");
    Model model;
    model.m_nodeDofs = 6;
    const std::int32_t gridX = nx + 1;
    const std::int32_t gridY = ny + 1;
    // Grid point (ix, iy) is model node iy*gridX + ix; the points of the edge x = 0 are clamped; the free nodes keep
    // the model's order.
    std::vector<std::int32_t> freeOf(static_cast<std::size_t>(gridX) * gridY, -1);
    std::int32_t next = 0;
    for (std::int32_t iy = 0; iy < gridY; ++iy)
        for (std::int32_t ix = 0; ix < gridX; ++ix)
            if (ix > 0)
            {
                freeOf[static_cast<std::size_t>(iy) * gridX + ix] = next++;
                model.m_coordinates.push_back(lx * ix / nx);
                model.m_coordinates.push_back(ly * iy / ny);
                model.m_coordinates.push_back(0.0);
                model.m_gridIndex.push_back(iy * gridX + ix);
            }
    model.m_nodeCount = next;
    std::vector<std::vector<std::int32_t>> elements;
    elements.reserve(static_cast<std::size_t>(nx) * ny);
    for (std::int32_t ey = 0; ey < ny; ++ey)
        for (std::int32_t ex = 0; ex < nx; ++ex)
        {
            const auto at = [&](std::int32_t ix, std::int32_t iy) { return freeOf[static_cast<std::size_t>(iy) * gridX + ix]; };
            elements.push_back({at(ex, ey), at(ex + 1, ey), at(ex + 1, ey + 1), at(ex, ey + 1)});
        }
    model.buildGraph(elements);
    const double a = lx / nx;
    const double b = ly / ny;
    std::vector<double> ke(SHELL_DOFS * SHELL_DOFS);
    shellStiffness(a, b, thickness, young, poisson, ke.data());
    model.assemble(elements, ke.data(), 6);
    ElementKind shell;
    shell.a = a;
    shell.b = b;
    shell.thickness = thickness;
    shell.young = young;
    shell.poisson = poisson;
    const int kind = model.addKind(shell);
    for (const auto& nodes : elements)
        model.recordElement(nodes, kind);
    // The consistent load of a uniform pressure on the bilinear deflection: p*a*b/4 on w at each node.
    model.m_pressureLoad.assign(static_cast<std::size_t>(model.m_nodeCount) * 6, 0.0);
    for (const auto& nodes : elements)
        for (const std::int32_t node : nodes)
            if (node >= 0)
                model.m_pressureLoad[static_cast<std::size_t>(node) * 6 + 2] += pressure * a * b / 4.0;
    return model;
}

void Model::clearBlocks()
{
    const auto w = static_cast<std::size_t>(m_nodeDofs);
    m_diagonalBlocks.assign(static_cast<std::size_t>(m_nodeCount) * w * w, 0.0);
    m_offBlocks.assign(m_neighbours.size() * w * w, 0.0);
}

void Model::addElement(const std::vector<std::int32_t>& nodes, const double* elementMatrix)
{
    const auto w = static_cast<std::size_t>(m_nodeDofs);
    const std::size_t elementDofs = nodes.size() * w;
    for (std::size_t i = 0; i < nodes.size(); ++i)
    {
        const std::int32_t a = nodes[i];
        if (a < 0)
            continue;
        for (std::size_t j = 0; j < nodes.size(); ++j)
        {
            const std::int32_t b = nodes[j];
            if (b < 0)
                continue;
            double* block = b == a ? m_diagonalBlocks.data() + static_cast<std::size_t>(a) * w * w
                                   : m_offBlocks.data() + static_cast<std::size_t>(slot(a, b)) * w * w;
            for (std::size_t cc = 0; cc < w; ++cc)
                for (std::size_t rr = 0; rr < w; ++rr)
                    block[rr + cc * w] += elementMatrix[(i * w + rr) * elementDofs + j * w + cc];
        }
    }
}

Model Model::stiffenedPanel(std::int32_t n, double lx, double ly, double thickness, double young, double poisson,
                            std::int32_t stringers, double bladeHeight, double bladeThickness, double pressure)
{
    if (stringers < 0 || stringers >= n || !(bladeHeight > 0) || !(bladeThickness > 0))
        throw std::invalid_argument("stiffened panel: expected 0 <= stringers < n and a positive blade section");
    Model model = plate(n, n, lx, ly, thickness, young, poisson, pressure);
    // The blades: frame elements between consecutive grid points of their grid line (already neighbours in the skin's
    // graph); grid point (ix, iy) is free node iy * n + ix - 1 for ix >= 1 (plate's order), clamped for ix = 0.
    const double a = lx / n;
    const double area = bladeHeight * bladeThickness;
    const double outOfPlane = bladeThickness * bladeHeight * bladeHeight * bladeHeight / 12.0; // bending in xz (w, ry)
    const double inPlane = bladeHeight * bladeThickness * bladeThickness * bladeThickness / 12.0; // bending in xy
    const double torsion = bladeHeight * bladeThickness * bladeThickness * bladeThickness / 3.0;
    const double shearModulus = young / (2.0 * (1.0 + poisson));
    double ke[12 * 12] = {};
    const auto add = [&](int r, int c, double v) { ke[r * 12 + c] += v; };
    const double L = a;
    // axial (u) and torsion (rx)
    for (const auto& [dof, k] : {std::pair<int, double>{0, young * area / L}, {3, shearModulus * torsion / L}})
    {
        add(dof, dof, k);
        add(dof + 6, dof + 6, k);
        add(dof, dof + 6, -k);
        add(dof + 6, dof, -k);
    }
    // bending: (v, rz) with rz = v' and (w, ry) with ry = -w'
    const auto bend = [&](int d, int r, double ei, double sign)
    {
        const double c = ei / (L * L * L);
        const int idx[4] = {d, r, d + 6, r + 6};
        const double m[4][4] = {{12, 6 * L * sign, -12, 6 * L * sign},
                                {6 * L * sign, 4 * L * L, -6 * L * sign, 2 * L * L},
                                {-12, -6 * L * sign, 12, -6 * L * sign},
                                {6 * L * sign, 2 * L * L, -6 * L * sign, 4 * L * L}};
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j)
                add(idx[i], idx[j], c * m[i][j]);
    };
    bend(1, 5, young * inPlane, 1.0);
    bend(2, 4, young * outOfPlane, -1.0);
    ElementKind frame;
    frame.family = 2;
    frame.dofs = 12;
    frame.given.assign(ke, ke + 12 * 12);
    const int frameKind = model.addKind(frame);
    for (std::int32_t k = 0; k < stringers; ++k)
    {
        const auto iy = static_cast<std::int32_t>(std::lround(static_cast<double>(k + 1) * n / (stringers + 1)));
        for (std::int32_t ix = 0; ix < n; ++ix)
        {
            const std::int32_t first = ix == 0 ? -1 : iy * n + ix - 1;
            const std::int32_t second = iy * n + ix;
            model.addElement({first, second}, ke);
            model.recordElement({first, second}, frameKind);
        }
    }
    return model;
}

Model Model::wingBox(double span, double chord, double height, double ribPitch, double h, const double* thicknesses,
                     double ribThickness, double young, double poisson, double density)
{
    if (!(span > 0) || !(chord > 0) || !(height > 0) || !(ribPitch > 0) || !(h > 0) || thicknesses == nullptr)
        throw std::invalid_argument("wing box: expected positive dimensions and 24 thicknesses");
    const auto nx = static_cast<std::int32_t>(std::lround(chord / h));
    const auto ny = static_cast<std::int32_t>(std::lround(span / h));
    const auto nz = static_cast<std::int32_t>(std::lround(height / h));
    const auto ribEvery = static_cast<std::int32_t>(std::lround(ribPitch / h));
    if (nx < 1 || ny < 1 || nz < 1 || ribEvery < 1 || std::abs(nx * h - chord) > 1e-9 * chord ||
        std::abs(ny * h - span) > 1e-9 * span || std::abs(nz * h - height) > 1e-9 * height)
        throw std::invalid_argument("wing box: the dimensions must be whole multiples of the element size");
    const double hz = height / nz;
    Model model;
    model.m_nodeDofs = 6;
    const auto on = [&](std::int32_t ix, std::int32_t iy, std::int32_t iz)
    { return iz == 0 || iz == nz || ix == 0 || ix == nx || iy % ribEvery == 0; };
    std::vector<std::int32_t> freeOf(static_cast<std::size_t>(nx + 1) * (ny + 1) * (nz + 1), -1);
    const auto index = [&](std::int32_t ix, std::int32_t iy, std::int32_t iz)
    { return (static_cast<std::size_t>(iy) * (nz + 1) + iz) * (nx + 1) + ix; };
    std::int32_t next = 0;
    for (std::int32_t iy = 1; iy <= ny; ++iy) // y = 0 clamped
        for (std::int32_t iz = 0; iz <= nz; ++iz)
            for (std::int32_t ix = 0; ix <= nx; ++ix)
                if (on(ix, iy, iz))
                {
                    freeOf[index(ix, iy, iz)] = next++;
                    model.m_coordinates.push_back(h * ix);
                    model.m_coordinates.push_back(h * iy);
                    model.m_coordinates.push_back(hz * iz);
                    model.m_gridIndex.push_back(static_cast<std::int32_t>(index(ix, iy, iz)));
                }
    model.m_nodeCount = next;
    const auto at = [&](std::int32_t ix, std::int32_t iy, std::int32_t iz) { return freeOf[index(ix, iy, iz)]; };
    // Elements by group: (nodes, group); each group one thickness and one orientation.
    struct Group
    {
        int orientation; // 0: xy plane, 1: yz plane (spars), 2: xz plane (ribs)
        double thickness;
        double a;
        double b;
    };
    std::vector<Group> groups;
    std::vector<std::vector<std::int32_t>> elements;
    std::vector<int> groupOf;
    for (int z = 0; z < 24; ++z)
        if (!(thicknesses[z] > 0))
            throw std::invalid_argument("wing box: the zone thicknesses must be positive");
    for (int z = 0; z < 8; ++z)
        groups.push_back({0, thicknesses[z], h, h}); // upper skin zones 0..7
    for (int z = 0; z < 8; ++z)
        groups.push_back({0, thicknesses[8 + z], h, h}); // lower skin zones 8..15
    for (int z = 0; z < 8; ++z)
        groups.push_back({1, thicknesses[16 + z], h, hz}); // spars: front 16..19, rear 20..23
    groups.push_back({2, ribThickness, h, hz}); // ribs: group 24
    const auto spanZone = [&](std::int32_t ey, int zones) { return std::min(zones - 1, ey * zones / ny); };
    for (std::int32_t ey = 0; ey < ny; ++ey)
        for (std::int32_t ex = 0; ex < nx; ++ex)
        {
            // local x along global x, local y along global y
            elements.push_back({at(ex, ey, nz), at(ex + 1, ey, nz), at(ex + 1, ey + 1, nz), at(ex, ey + 1, nz)});
            groupOf.push_back(spanZone(ey, 8));
            elements.push_back({at(ex, ey, 0), at(ex + 1, ey, 0), at(ex + 1, ey + 1, 0), at(ex, ey + 1, 0)});
            groupOf.push_back(8 + spanZone(ey, 8));
        }
    for (std::int32_t ey = 0; ey < ny; ++ey)
        for (std::int32_t ez = 0; ez < nz; ++ez)
            for (const std::int32_t ix : {0, nx})
            {
                // local x along global y, local y along global z
                elements.push_back({at(ix, ey, ez), at(ix, ey + 1, ez), at(ix, ey + 1, ez + 1), at(ix, ey, ez + 1)});
                groupOf.push_back(16 + (ix == 0 ? 0 : 4) + spanZone(ey, 4));
            }
    for (std::int32_t iy = ribEvery; iy <= ny; iy += ribEvery)
        for (std::int32_t ez = 0; ez < nz; ++ez)
            for (std::int32_t ex = 0; ex < nx; ++ex)
            {
                // local x along global x, local y along global z
                elements.push_back({at(ex, iy, ez), at(ex + 1, iy, ez), at(ex + 1, iy, ez + 1), at(ex, iy, ez + 1)});
                groupOf.push_back(24);
            }
    model.buildGraph(elements);
    model.clearBlocks();
    // Rotation of each orientation: the columns are the local axes in global coordinates.
    const double rotation[3][9] = {{1, 0, 0, 0, 1, 0, 0, 0, 1},   // xy: local (x, y, n) = (x, y, z)
                                   {0, 0, 1, 1, 0, 0, 0, 1, 0},   // yz: local x = y, local y = z, n = x
                                   {1, 0, 0, 0, 0, -1, 0, 1, 0}}; // xz: local x = x, local y = z, n = -y
    std::vector<std::vector<double>> matrices;
    std::vector<int> kindOfGroup;
    for (const Group& g : groups)
    {
        ElementKind shell;
        shell.a = g.a;
        shell.b = g.b;
        shell.thickness = g.thickness;
        shell.young = young;
        shell.poisson = poisson;
        shell.orientation = g.orientation;
        kindOfGroup.push_back(model.addKind(shell));
        std::vector<double> local(SHELL_DOFS * SHELL_DOFS);
        shellStiffness(g.a, g.b, g.thickness, young, poisson, local.data());
        // global = T local T^T with T = blockdiag(R) over the 8 triples of DOFs (R(i, j) = rotation[i * 3 + j])
        const double* r = rotation[g.orientation];
        std::vector<double> tmp(SHELL_DOFS * SHELL_DOFS, 0.0);
        std::vector<double> global(SHELL_DOFS * SHELL_DOFS, 0.0);
        for (int i = 0; i < SHELL_DOFS; ++i)
            for (int j = 0; j < SHELL_DOFS; ++j)
            {
                // tmp = T local: row i of T has R(i % 3, .) on the triple of i
                double sum = 0.0;
                const int base = i / 3 * 3;
                for (int q = 0; q < 3; ++q)
                    sum += r[(i % 3) * 3 + q] * local[(base + q) * SHELL_DOFS + j];
                tmp[i * SHELL_DOFS + j] = sum;
            }
        for (int i = 0; i < SHELL_DOFS; ++i)
            for (int j = 0; j < SHELL_DOFS; ++j)
            {
                double sum = 0.0;
                const int base = j / 3 * 3;
                for (int q = 0; q < 3; ++q)
                    sum += tmp[i * SHELL_DOFS + base + q] * r[(j % 3) * 3 + q];
                global[i * SHELL_DOFS + j] = sum;
            }
        matrices.push_back(std::move(global));
    }
    model.m_lumpedMass.assign(static_cast<std::size_t>(model.m_nodeCount) * 6, 0.0);
    for (std::size_t e = 0; e < elements.size(); ++e)
    {
        const Group& g = groups[static_cast<std::size_t>(groupOf[e])];
        model.addElement(elements[e], matrices[static_cast<std::size_t>(groupOf[e])].data());
        model.recordElement(elements[e], kindOfGroup[static_cast<std::size_t>(groupOf[e])]);
        const double area = g.a * g.b;
        const double translation = density * g.thickness * area / 4.0;
        const double rotary = density * g.thickness * g.thickness * g.thickness * area / 48.0;
        for (const std::int32_t node : elements[e])
            if (node >= 0)
                for (int c = 0; c < 6; ++c)
                    model.m_lumpedMass[static_cast<std::size_t>(node) * 6 + c] += c < 3 ? translation : rotary;
    }
    model.m_pressureLoad.assign(static_cast<std::size_t>(model.m_nodeCount) * 6, 0.0);
    return model;
}

Model Model::hexBlock(std::int32_t n, double edge, double young, double poisson, double density)
{
    if (n < 1 || !(edge > 0) || !(young > 0) || !(poisson > -1.0 && poisson < 0.5) || !(density > 0))
        throw std::invalid_argument("hex model: expected n >= 1 and positive dimensions and material");
    Model model;
    model.m_nodeDofs = 3;
    const std::int32_t g = n + 1;
    std::vector<std::int32_t> freeOf(static_cast<std::size_t>(g) * g * g, -1);
    std::int32_t next = 0;
    for (std::int32_t iz = 0; iz < g; ++iz)
        for (std::int32_t iy = 0; iy < g; ++iy)
            for (std::int32_t ix = 0; ix < g; ++ix)
                if (iz > 0)
                {
                    freeOf[(static_cast<std::size_t>(iz) * g + iy) * g + ix] = next++;
                    model.m_coordinates.push_back(edge * ix / n);
                    model.m_coordinates.push_back(edge * iy / n);
                    model.m_coordinates.push_back(edge * iz / n);
                    model.m_gridIndex.push_back((iz * g + iy) * g + ix);
                }
    model.m_nodeCount = next;
    std::vector<std::vector<std::int32_t>> elements;
    elements.reserve(static_cast<std::size_t>(n) * n * n);
    const auto at = [&](std::int32_t ix, std::int32_t iy, std::int32_t iz)
    { return freeOf[(static_cast<std::size_t>(iz) * g + iy) * g + ix]; };
    for (std::int32_t ez = 0; ez < n; ++ez)
        for (std::int32_t ey = 0; ey < n; ++ey)
            for (std::int32_t ex = 0; ex < n; ++ex)
                elements.push_back({at(ex, ey, ez), at(ex + 1, ey, ez), at(ex + 1, ey + 1, ez), at(ex, ey + 1, ez),
                                    at(ex, ey, ez + 1), at(ex + 1, ey, ez + 1), at(ex + 1, ey + 1, ez + 1),
                                    at(ex, ey + 1, ez + 1)});
    model.buildGraph(elements);
    const double h = edge / n;
    std::vector<double> ke(HEX_DOFS * HEX_DOFS);
    hexStiffness(h, young, poisson, ke.data());
    model.assemble(elements, ke.data(), 3);
    ElementKind solid;
    solid.family = 1;
    solid.a = h;
    solid.young = young;
    solid.poisson = poisson;
    const int kind = model.addKind(solid);
    for (const auto& nodes : elements)
        model.recordElement(nodes, kind);
    // Lumped mass: an eighth of each element's mass at each of its nodes, in every direction.
    model.m_lumpedMass.assign(static_cast<std::size_t>(model.m_nodeCount) * 3, 0.0);
    for (const auto& nodes : elements)
        for (const std::int32_t node : nodes)
            if (node >= 0)
                for (int c = 0; c < 3; ++c)
                    model.m_lumpedMass[static_cast<std::size_t>(node) * 3 + c] += density * h * h * h / 8.0;
    model.m_pressureLoad.assign(static_cast<std::size_t>(model.m_nodeCount) * 3, 0.0);
    return model;
}

void Model::firstColumns(const std::int32_t* nodeAtPosition, std::int32_t* firstColumnOfPosition) const
{
    firstColumnOfPosition[0] = 0;
    for (std::int32_t p = 0; p < m_nodeCount; ++p)
        firstColumnOfPosition[p + 1] = firstColumnOfPosition[p] + m_nodeDofs;
    (void)nodeAtPosition;
}

std::int64_t Model::cscTermCount(const std::int32_t* nodeAtPosition) const
{
    // Per node at position p: its diagonal block's lower triangle, then full blocks for every neighbour at a later
    // position.
    std::vector<std::int32_t> positionOf(static_cast<std::size_t>(m_nodeCount));
    for (std::int32_t p = 0; p < m_nodeCount; ++p)
        positionOf[static_cast<std::size_t>(nodeAtPosition[p])] = p;
    const std::int64_t w = m_nodeDofs;
    std::int64_t terms = 0;
    for (std::int32_t node = 0; node < m_nodeCount; ++node)
    {
        std::int64_t later = 0;
        for (std::int64_t k = m_offsets[static_cast<std::size_t>(node)]; k < m_offsets[static_cast<std::size_t>(node) + 1]; ++k)
            if (positionOf[static_cast<std::size_t>(m_neighbours[static_cast<std::size_t>(k)])] >
                positionOf[static_cast<std::size_t>(node)])
                ++later;
        terms += w * (w + 1) / 2 + later * w * w;
    }
    return terms;
}

void Model::toCsc(const std::int32_t* nodeAtPosition, int which, std::int64_t* offsets, std::int32_t* rows,
                  double* values) const
{
    // which: 0 stiffness, 1 lumped mass (on the stiffness pattern, zeros off the diagonal).
    const std::int32_t count = m_nodeCount;
    const std::int64_t w = m_nodeDofs;
    std::vector<std::int32_t> positionOf(static_cast<std::size_t>(count));
    for (std::int32_t p = 0; p < count; ++p)
        positionOf[static_cast<std::size_t>(nodeAtPosition[p])] = p;
    // Terms per position, then the column offsets.
    std::vector<std::int64_t> later(static_cast<std::size_t>(count));
    for (std::int32_t p = 0; p < count; ++p)
    {
        const std::int32_t node = nodeAtPosition[p];
        std::int64_t laterCount = 0;
        for (std::int64_t k = m_offsets[static_cast<std::size_t>(node)]; k < m_offsets[static_cast<std::size_t>(node) + 1]; ++k)
            if (positionOf[static_cast<std::size_t>(m_neighbours[static_cast<std::size_t>(k)])] > p)
                ++laterCount;
        later[static_cast<std::size_t>(p)] = laterCount;
    }
    offsets[0] = 0;
    for (std::int32_t p = 0; p < count; ++p)
        for (std::int64_t c = 0; c < w; ++c)
        {
            const std::int64_t column = p * w + c;
            offsets[column + 1] = offsets[column] + (w - c) + later[static_cast<std::size_t>(p)] * w;
        }
#pragma omp parallel for schedule(dynamic, 256)
    for (std::int32_t p = 0; p < count; ++p)
    {
        const std::int32_t node = nodeAtPosition[p];
        // The later neighbours sorted by position: their DOFs come in that order.
        std::vector<std::pair<std::int32_t, std::int64_t>> laterNeighbours;
        for (std::int64_t k = m_offsets[static_cast<std::size_t>(node)]; k < m_offsets[static_cast<std::size_t>(node) + 1]; ++k)
        {
            const std::int32_t q = positionOf[static_cast<std::size_t>(m_neighbours[static_cast<std::size_t>(k)])];
            if (q > p)
                laterNeighbours.emplace_back(q, k);
        }
        std::sort(laterNeighbours.begin(), laterNeighbours.end());
        const double* diagonal = m_diagonalBlocks.data() + static_cast<std::size_t>(node) * static_cast<std::size_t>(w * w);
        for (std::int64_t c = 0; c < w; ++c)
        {
            const std::int64_t column = p * w + c;
            std::int64_t at = offsets[column];
            for (std::int64_t r = c; r < w; ++r)
            {
                rows[at] = static_cast<std::int32_t>(p * w + r);
                double value = 0.0;
                if (which == 0)
                    value = diagonal[r + c * w];
                else if (r == c)
                    value = m_lumpedMass[static_cast<std::size_t>(node * w + c)];
                values[at++] = value;
            }
            for (const auto& [q, k] : laterNeighbours)
            {
                // The block (rows of the neighbour, columns of this node): the neighbour's block towards this node,
                // transposed from this node's block towards the neighbour.
                const double* block = m_offBlocks.data() + static_cast<std::size_t>(k) * static_cast<std::size_t>(w * w);
                for (std::int64_t r = 0; r < w; ++r)
                {
                    rows[at] = static_cast<std::int32_t>(static_cast<std::int64_t>(q) * w + r);
                    // block(rr, cc): rows = DOFs of `node`, columns = DOFs of the neighbour; we need K(neighbour r,
                    // node c) = K(node c, neighbour r) = block(c, r).
                    values[at++] = which == 0 ? block[c + r * w] : 0.0;
                }
            }
        }
    }
}

void Model::loads(const std::int32_t* nodeAtPosition, std::int64_t columns, std::uint64_t seedBase,
                  std::int32_t pointsPerPattern, double sigma, double* rhs, std::int64_t ld) const
{
    // Column 0: the pressure; column j >= 1: pointsPerPattern free nodes drawn with splitmix64 seeded seedBase + j,
    // each with a N(0, sigma) force (Box-Muller) on its out-of-plane translation (DOF 2 of a shell node; DOF 2 = z of
    // a solid node).
    const std::int32_t count = m_nodeCount;
    const std::int64_t w = m_nodeDofs;
    std::vector<std::int32_t> positionOf(static_cast<std::size_t>(count));
    for (std::int32_t p = 0; p < count; ++p)
        positionOf[static_cast<std::size_t>(nodeAtPosition[p])] = p;
    for (std::int64_t j = 0; j < columns; ++j)
    {
        double* column = rhs + j * ld;
        std::fill_n(column, count * w, 0.0);
        if (j == 0)
        {
            for (std::int32_t node = 0; node < count; ++node)
                for (std::int64_t c = 0; c < w; ++c)
                    column[positionOf[static_cast<std::size_t>(node)] * w + c] = m_pressureLoad[static_cast<std::size_t>(node * w + c)];
            continue;
        }
        std::uint64_t state = seedBase + static_cast<std::uint64_t>(j);
        for (std::int32_t k = 0; k < pointsPerPattern; ++k)
        {
            const auto node = static_cast<std::int32_t>(splitmix64(state) % static_cast<std::uint64_t>(count));
            const double u1 = 1.0 - uniform01(state);
            const double u2 = uniform01(state);
            const double normal = std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * 3.14159265358979323846 * u2);
            column[positionOf[static_cast<std::size_t>(node)] * w + 2] += sigma * normal;
        }
    }
}

} // namespace oosgpu
