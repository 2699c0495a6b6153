// The workload models' stiffness assembled on the GPU (the role of the reference's StiffnessAssembler and
// SymmetricCsc::fromBlocks, include/oos/assembly/assemble/StiffnessAssembler.hpp:21-33,
// src/linalg/sparse/SymmetricCsc.cpp:41-200, for this project's elements, csrc/host/model.cpp):
//   elementMatrices  one block per kind of element: the flat shell (bilinear membrane, MITC4 bending, drilling
//                    spring; turned into the global axes), the trilinear hexahedron, or a matrix given by the host;
//   nodeBlocks       one thread per node block (a node's diagonal block, or its block towards one neighbour): the terms
//                    of the elements holding both nodes, in increasing element order;
//   cscCounts/Fill   the lower-triangle compressed columns in the equation order of a node order.
// Every element-matrix operation is rounded on its own (__dmul_rn, __dadd_rn, __ddiv_rn: no fused multiply-adds), in
// the host code's order, and every block sums its terms in the host's order, so the matrix is the host's bit for bit.

#include "kernels.cuh"

#include <cstdint>

namespace oosgpu::device
{

namespace
{

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dvd(double a, double b) { return __ddiv_rn(a, b); }

constexpr double GAUSS = 0.57735026918962576451;
__constant__ double NODE_XI[4] = {-1.0, 1.0, 1.0, -1.0};
__constant__ double NODE_ETA[4] = {-1.0, -1.0, 1.0, 1.0};
__constant__ double HX[8] = {-1, 1, 1, -1, -1, 1, 1, -1};
__constant__ double HY[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
__constant__ double HZ[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
// the three orientations of a shell: columns the local axes in global coordinates (R(i, j) = ROTATION[o][3 i + j])
__constant__ double ROTATION[3][9] = {{1, 0, 0, 0, 1, 0, 0, 0, 1}, {0, 0, 1, 1, 0, 0, 0, 1, 0},
                                      {1, 0, 0, 0, 0, -1, 0, 1, 0}};

struct ShellShape
{
    double n[4];
    double dx[4];
    double dy[4];
};

__device__ ShellShape shellShape(double xi, double eta, double a, double b)
{
    ShellShape s;
    for (int i = 0; i < 4; ++i)
    {
        s.n[i] = mul(mul(0.25, add(1.0, mul(xi, NODE_XI[i]))), add(1.0, mul(eta, NODE_ETA[i])));
        s.dx[i] = mul(mul(mul(0.25, NODE_XI[i]), add(1.0, mul(eta, NODE_ETA[i]))), dvd(2.0, a));
        s.dy[i] = mul(mul(mul(0.25, NODE_ETA[i]), add(1.0, mul(xi, NODE_XI[i]))), dvd(2.0, b));
    }
    return s;
}

// Column c (0..23) of the transverse shear rows (gxz, gyz) of the displacement interpolation at (xi, eta).
__device__ void shearColumn(double xi, double eta, double a, double b, int c, double& gxz, double& gyz)
{
    const ShellShape s = shellShape(xi, eta, a, b);
    const int node = c / 6;
    const int dof = c % 6;
    gxz = dof == 2 ? s.dx[node] : (dof == 4 ? s.n[node] : 0.0);
    gyz = dof == 2 ? s.dy[node] : (dof == 3 ? -s.n[node] : 0.0);
}

// Column c of the three strain operators of the shell at a Gauss point: membrane (3 rows), bending (3), shear (2).
__device__ void shellColumn(const ShellShape& s, double xi, double eta, double a, double b, int c, double bm[3],
                            double bb[3], double bs[2])
{
    const int node = c / 6;
    const int dof = c % 6;
    bm[0] = dof == 0 ? s.dx[node] : 0.0;
    bm[1] = dof == 1 ? s.dy[node] : 0.0;
    bm[2] = dof == 0 ? s.dy[node] : (dof == 1 ? s.dx[node] : 0.0);
    bb[0] = dof == 4 ? s.dx[node] : 0.0;
    bb[1] = dof == 3 ? -s.dy[node] : 0.0;
    bb[2] = dof == 4 ? s.dy[node] : (dof == 3 ? -s.dx[node] : 0.0);
    // MITC4: gxz tied at (0, +1) and (0, -1), gyz at (+1, 0) and (-1, 0)
    double gxzA, gxzC, gyzD, gyzB, unused;
    shearColumn(0.0, 1.0, a, b, c, gxzA, unused);
    shearColumn(0.0, -1.0, a, b, c, gxzC, unused);
    shearColumn(1.0, 0.0, a, b, c, unused, gyzD);
    shearColumn(-1.0, 0.0, a, b, c, unused, gyzB);
    bs[0] = add(mul(mul(0.5, add(1.0, eta)), gxzA), mul(mul(0.5, sub(1.0, eta)), gxzC));
    bs[1] = add(mul(mul(0.5, add(1.0, xi)), gyzD), mul(mul(0.5, sub(1.0, xi)), gyzB));
}

// sum_r bi[r] (sum_q d[r][q] bj[q]): one (i, j) term of B^T D B, in the host's order.
template <int ROWS> __device__ double btdb(const double* bi, const double* bj, const double* d)
{
    double s = 0.0;
    for (int r = 0; r < ROWS; ++r)
    {
        double db = 0.0;
        for (int q = 0; q < ROWS; ++q)
            db = add(db, mul(d[r * ROWS + q], bj[q]));
        s = add(s, mul(bi[r], db));
    }
    return s;
}

// Entry (i, j) of the 24 x 24 local shell stiffness.
__device__ double shellEntry(const ElementKindDesc& k, int i, int j)
{
    const double pp = mul(k.poisson, k.poisson);
    const double membrane = dvd(mul(k.young, k.thickness), sub(1.0, pp));
    const double bending = dvd(mul(mul(mul(k.young, k.thickness), k.thickness), k.thickness), mul(12.0, sub(1.0, pp)));
    const double shear = mul(dvd(mul(5.0 / 6.0, k.young), mul(2.0, add(1.0, k.poisson))), k.thickness);
    const double dm[9] = {membrane, mul(membrane, k.poisson), 0, mul(membrane, k.poisson), membrane, 0, 0, 0,
                          dvd(mul(membrane, sub(1.0, k.poisson)), 2.0)};
    const double db[9] = {bending, mul(bending, k.poisson), 0, mul(bending, k.poisson), bending, 0, 0, 0,
                          dvd(mul(bending, sub(1.0, k.poisson)), 2.0)};
    const double ds[4] = {shear, 0, 0, shear};
    const double detJ = dvd(mul(k.a, k.b), 4.0);
    double value = 0.0;
    for (int gx = 0; gx < 2; ++gx)
        for (int gy = 0; gy < 2; ++gy)
        {
            const double xi = gx == 0 ? -GAUSS : GAUSS;
            const double eta = gy == 0 ? -GAUSS : GAUSS;
            const ShellShape s = shellShape(xi, eta, k.a, k.b);
            double bmi[3], bbi[3], bsi[2], bmj[3], bbj[3], bsj[2];
            shellColumn(s, xi, eta, k.a, k.b, i, bmi, bbi, bsi);
            shellColumn(s, xi, eta, k.a, k.b, j, bmj, bbj, bsj);
            double w[9];
            for (int q = 0; q < 9; ++q)
                w[q] = mul(dm[q], detJ);
            value = add(value, btdb<3>(bmi, bmj, w));
            for (int q = 0; q < 9; ++q)
                w[q] = mul(db[q], detJ);
            value = add(value, btdb<3>(bbi, bbj, w));
            double w2[4];
            for (int q = 0; q < 4; ++q)
                w2[q] = mul(ds[q], detJ);
            value = add(value, btdb<2>(bsi, bsj, w2));
        }
    if (i == j && i % 6 == 5) // drilling: a thousandth of the shear stiffness of the element's area
        value = add(value, dvd(mul(mul(mul(1.0e-3, shear), k.a), k.b), 4.0));
    return value;
}

// Column c (0..23) of the hexahedron's strain operator (6 rows) at Gauss point g.
__device__ void hexColumn(double h, int g, int c, double column[6])
{
    const double xi = (g & 1) ? GAUSS : -GAUSS;
    const double eta = (g & 2) ? GAUSS : -GAUSS;
    const double zeta = (g & 4) ? GAUSS : -GAUSS;
    const int i = c / 3;
    const int dof = c % 3;
    const double dx = mul(mul(mul(mul(0.125, HX[i]), add(1.0, mul(eta, HY[i]))), add(1.0, mul(zeta, HZ[i]))), dvd(2.0, h));
    const double dy = mul(mul(mul(mul(0.125, HY[i]), add(1.0, mul(xi, HX[i]))), add(1.0, mul(zeta, HZ[i]))), dvd(2.0, h));
    const double dz = mul(mul(mul(mul(0.125, HZ[i]), add(1.0, mul(xi, HX[i]))), add(1.0, mul(eta, HY[i]))), dvd(2.0, h));
    column[0] = dof == 0 ? dx : 0.0;
    column[1] = dof == 1 ? dy : 0.0;
    column[2] = dof == 2 ? dz : 0.0;
    column[3] = dof == 0 ? dy : (dof == 1 ? dx : 0.0);
    column[4] = dof == 1 ? dz : (dof == 2 ? dy : 0.0);
    column[5] = dof == 0 ? dz : (dof == 2 ? dx : 0.0);
}

__device__ double hexEntry(const ElementKindDesc& k, int i, int j)
{
    const double lambda = dvd(mul(k.young, k.poisson), mul(add(1.0, k.poisson), sub(1.0, mul(2.0, k.poisson))));
    const double mu = dvd(k.young, mul(2.0, add(1.0, k.poisson)));
    double d[36];
    for (int q = 0; q < 36; ++q)
        d[q] = 0.0;
    for (int r = 0; r < 3; ++r)
    {
        for (int c = 0; c < 3; ++c)
            d[r * 6 + c] = lambda;
        d[r * 6 + r] = add(lambda, mul(2.0, mu));
        d[(r + 3) * 6 + (r + 3)] = mu;
    }
    const double detJ = dvd(mul(mul(k.a, k.a), k.a), 8.0);
    double w[36];
    for (int q = 0; q < 36; ++q)
        w[q] = mul(d[q], detJ);
    double value = 0.0;
    for (int g = 0; g < 8; ++g)
    {
        double bi[6], bj[6];
        hexColumn(k.a, g, i, bi);
        hexColumn(k.a, g, j, bj);
        value = add(value, btdb<6>(bi, bj, w));
    }
    return value;
}

} // namespace

// One block of 576 threads per kind: entry (i, j) of its dofs x dofs matrix (row-major) at out + kind * 576. A shell
// of orientation o is T K T^T with T the block diagonal of the rotation over its eight triples of DOFs.
__global__ void __launch_bounds__(576) elementMatrices(const ElementKindDesc* kinds, const double* given, double* out)
{
    __shared__ double local[24 * 24];
    __shared__ double turned[24 * 24];
    const ElementKindDesc k = kinds[blockIdx.x];
    double* matrix = out + static_cast<std::int64_t>(blockIdx.x) * 576;
    const int e = threadIdx.x;
    const int i = e / k.dofs;
    const int j = e % k.dofs;
    const bool inside = e < k.dofs * k.dofs;
    if (k.family == 2)
    {
        if (inside)
            matrix[e] = given[k.givenOffset + e];
        return;
    }
    const double value = inside ? (k.family == 0 ? shellEntry(k, i, j) : hexEntry(k, i, j)) : 0.0;
    if (k.family == 1 || k.orientation == 0)
    {
        if (inside)
            matrix[e] = value;
        return;
    }
    // tmp = T local, then global = tmp T^T (each sum from zero, its three terms in order)
    if (inside)
        local[e] = value;
    __syncthreads();
    const double* r = ROTATION[k.orientation];
    if (inside)
    {
        const int base = i / 3 * 3;
        double sum = 0.0;
        for (int q = 0; q < 3; ++q)
            sum = add(sum, mul(r[(i % 3) * 3 + q], local[(base + q) * 24 + j]));
        turned[e] = sum;
    }
    __syncthreads();
    if (inside)
    {
        const int base = j / 3 * 3;
        double sum = 0.0;
        for (int q = 0; q < 3; ++q)
            sum = add(sum, mul(turned[i * 24 + base + q], r[(j % 3) * 3 + q]));
        matrix[e] = sum;
    }
}

// One thread per node block: blocks [0, nodes) the nodes' diagonal blocks, then one per graph slot (node a's block
// towards neighbour neighbours[k]). Block (a, b) = sum over the elements holding a and b, in increasing element order,
// of their terms; w x w column-major (rows the DOFs of a).
__global__ void nodeBlocks(ModelArgs m, double* diagonalBlocks, double* offBlocks)
{
    const std::int64_t id = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (id >= static_cast<std::int64_t>(m.nodes) + m.slots)
        return;
    const int w = m.nodeDofs;
    std::int32_t a;
    std::int32_t b;
    double* block;
    if (id < m.nodes)
    {
        a = static_cast<std::int32_t>(id);
        b = a;
        block = diagonalBlocks + id * w * w;
    }
    else
    {
        const std::int64_t k = id - m.nodes;
        int lo = 0;
        int hi = m.nodes;
        while (hi - lo > 1) // the node owning slot k: offsets[a] <= k < offsets[a + 1]
        {
            const int mid = (lo + hi) >> 1;
            if (m.graphOffsets[mid] <= k)
                lo = mid;
            else
                hi = mid;
        }
        a = lo;
        b = m.neighbours[k];
        block = offBlocks + k * w * w;
    }
    double sum[36];
    for (int q = 0; q < w * w; ++q)
        sum[q] = 0.0;
    for (std::int64_t t = m.elementsOfNodeStart[a]; t < m.elementsOfNodeStart[a + 1]; ++t)
    {
        const std::int32_t e = m.elementsOfNode[t];
        const std::int64_t first = m.elementStart[e];
        const int count = static_cast<int>(m.elementStart[e + 1] - first);
        int la = -1;
        int lb = -1;
        for (int q = 0; q < count; ++q)
        {
            const std::int32_t node = m.elementNodes[first + q];
            if (node == a)
                la = q;
            if (node == b)
                lb = q;
        }
        if (la < 0 || lb < 0)
            continue;
        const int dofs = count * w;
        const double* matrix = m.matrices + static_cast<std::int64_t>(m.elementKind[e]) * 576;
        for (int cc = 0; cc < w; ++cc)
            for (int rr = 0; rr < w; ++rr)
                sum[rr + cc * w] = add(sum[rr + cc * w], matrix[(la * w + rr) * dofs + lb * w + cc]);
    }
    for (int q = 0; q < w * w; ++q)
        block[q] = sum[q];
}

// Per position p of the node order: the terms of its w columns (its diagonal block's lower part, full blocks towards
// every neighbour at a later position).
__global__ void cscCounts(ModelArgs m, const std::int32_t* nodeAtPosition, const std::int32_t* positionOf,
                          std::int64_t* terms)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= m.nodes)
        return;
    const std::int32_t node = nodeAtPosition[p];
    std::int64_t later = 0;
    for (std::int64_t k = m.graphOffsets[node]; k < m.graphOffsets[node + 1]; ++k)
        later += positionOf[m.neighbours[k]] > p ? 1 : 0;
    const std::int64_t w = m.nodeDofs;
    terms[p] = w * (w + 1) / 2 + later * w * w;
}

// The columns of position p (starting at termStart[p]): column c of the node's DOFs holds rows p w + c .. p w + w - 1
// (its diagonal block), then the w rows of every later neighbour in position order. which 0: the stiffness from the
// node blocks; which 1: the lumped mass on the same pattern (zeros off the diagonal).
__global__ void cscFill(ModelArgs m, const std::int32_t* nodeAtPosition, const std::int32_t* positionOf,
                        const std::int64_t* termStart, const double* diagonalBlocks, const double* offBlocks,
                        const double* lumpedMass, int which, std::int64_t* offsets, std::int32_t* rows, double* values)
{
    constexpr int MAX_NEIGHBOURS = 32;
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= m.nodes)
        return;
    const std::int32_t node = nodeAtPosition[p];
    const int w = m.nodeDofs;
    // the later neighbours, sorted by position (insertion sort of at most MAX_NEIGHBOURS)
    std::int32_t laterPosition[MAX_NEIGHBOURS];
    std::int64_t laterSlot[MAX_NEIGHBOURS];
    int later = 0;
    for (std::int64_t k = m.graphOffsets[node]; k < m.graphOffsets[node + 1]; ++k)
    {
        const std::int32_t q = positionOf[m.neighbours[k]];
        if (q <= p || later == MAX_NEIGHBOURS)
            continue;
        int at = later++;
        while (at > 0 && laterPosition[at - 1] > q)
        {
            laterPosition[at] = laterPosition[at - 1];
            laterSlot[at] = laterSlot[at - 1];
            --at;
        }
        laterPosition[at] = q;
        laterSlot[at] = k;
    }
    std::int64_t at = termStart[p];
    const double* diagonal = diagonalBlocks + static_cast<std::int64_t>(node) * w * w;
    for (int c = 0; c < w; ++c)
    {
        const std::int64_t column = static_cast<std::int64_t>(p) * w + c;
        offsets[column] = at;
        for (int r = c; r < w; ++r)
        {
            rows[at] = static_cast<std::int32_t>(static_cast<std::int64_t>(p) * w + r);
            values[at++] = which == 0 ? diagonal[r + c * w]
                                      : (r == c ? lumpedMass[static_cast<std::int64_t>(node) * w + c] : 0.0);
        }
        for (int t = 0; t < later; ++t)
        {
            // K(neighbour r, node c) = block(node -> neighbour)(c, r)
            const double* block = offBlocks + laterSlot[t] * w * w;
            for (int r = 0; r < w; ++r)
            {
                rows[at] = static_cast<std::int32_t>(static_cast<std::int64_t>(laterPosition[t]) * w + r);
                values[at++] = which == 0 ? block[c + r * w] : 0.0;
            }
        }
    }
    if (p == m.nodes - 1)
        offsets[static_cast<std::int64_t>(m.nodes) * w] = at;
}

__global__ void scatterPositions(const std::int32_t* nodeAtPosition, std::int32_t* positionOf, int nodes)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < nodes)
        positionOf[nodeAtPosition[p]] = p;
}

} // namespace oosgpu::device
