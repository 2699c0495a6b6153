// The symbolic structure the factorisation runs on: its checks, its counts, and the row structures of a supernode
// partition (the last step of the reference's SymbolicFactor::analyse, src/linalg/symbolic/SymbolicFactor.cpp:227-290).

#include "host_api.hpp"

#include <algorithm>
#include <string>

namespace oosgpu
{

void Symbolic::validate() const
{
    const auto fail = [](const std::string& what) { throw Error(STATUS_INVALID_ARGUMENT, "symbolic structure: " + what); };
    if (supernodeCount < 0 || dofCount < 0)
        fail("negative sizes");
    if (firstColumn.size() != static_cast<std::size_t>(supernodeCount) + 1 ||
        parent.size() != static_cast<std::size_t>(supernodeCount) ||
        rowStart.size() != static_cast<std::size_t>(supernodeCount) + 1)
        fail("array sizes do not match the supernode count");
    if (firstColumn[0] != 0 || firstColumn[static_cast<std::size_t>(supernodeCount)] != dofCount)
        fail("the first columns must run from 0 to the DOF count");
    if (rowStart[0] != 0 || rowStart[static_cast<std::size_t>(supernodeCount)] != static_cast<std::int64_t>(rows.size()))
        fail("the row starts must run from 0 to the row count");
    for (std::int32_t s = 0; s < supernodeCount; ++s)
    {
        if (columnCount(s) < 1)
            fail("supernode " + std::to_string(s) + " has no column");
        if (rowStart[static_cast<std::size_t>(s) + 1] < rowStart[static_cast<std::size_t>(s)])
            fail("row starts decrease at supernode " + std::to_string(s));
        const std::int32_t p = parent[static_cast<std::size_t>(s)];
        if (p != -1 && (p <= s || p >= supernodeCount))
            fail("supernode " + std::to_string(s) + " has parent " + std::to_string(p) + " (parents follow children)");
        const std::int32_t end = firstColumn[static_cast<std::size_t>(s) + 1];
        std::int32_t previous = end - 1;
        for (std::int64_t k = rowStart[static_cast<std::size_t>(s)]; k < rowStart[static_cast<std::size_t>(s) + 1]; ++k)
        {
            const std::int32_t row = rows[static_cast<std::size_t>(k)];
            if (row <= previous || row >= dofCount)
                fail("the rows of supernode " + std::to_string(s) + " are not ascending beyond its columns");
            previous = row;
        }
        if (p == -1 && rowCount(s) > 0)
            fail("root supernode " + std::to_string(s) + " has rows below it");
    }
    // The rows of a child lie in the columns and rows of its parent (the extend-add relies on it).
    for (std::int32_t s = 0; s < supernodeCount; ++s)
    {
        const std::int32_t p = parent[static_cast<std::size_t>(s)];
        if (p < 0)
            continue;
        const std::int32_t pFirst = firstColumn[static_cast<std::size_t>(p)];
        const std::int32_t pEnd = firstColumn[static_cast<std::size_t>(p) + 1];
        const std::int32_t* pRows = rows.data() + rowStart[static_cast<std::size_t>(p)];
        const std::int32_t* pRowsEnd = rows.data() + rowStart[static_cast<std::size_t>(p) + 1];
        const std::int32_t* cursor = pRows;
        for (std::int64_t k = rowStart[static_cast<std::size_t>(s)]; k < rowStart[static_cast<std::size_t>(s) + 1]; ++k)
        {
            const std::int32_t row = rows[static_cast<std::size_t>(k)];
            if (row >= pFirst && row < pEnd)
                continue;
            cursor = std::lower_bound(cursor, pRowsEnd, row);
            if (cursor == pRowsEnd || *cursor != row)
                fail("row " + std::to_string(row) + " of supernode " + std::to_string(s) +
                     " is neither a column nor a row of its parent " + std::to_string(p));
        }
    }
}

double Symbolic::flopCount() const
{
    double flops = 0.0;
    for (std::int32_t s = 0; s < supernodeCount; ++s)
    {
        const std::int64_t c = columnCount(s);
        const std::int64_t r = rowCount(s);
        for (std::int64_t m = r; m < r + c; ++m)
            flops += static_cast<double>(m) * static_cast<double>(m + 1) + 2.0 * static_cast<double>(m);
    }
    return flops;
}

std::int64_t Symbolic::panelValueCount() const
{
    std::int64_t values = 0;
    for (std::int32_t s = 0; s < supernodeCount; ++s)
    {
        const std::int64_t c = columnCount(s);
        values += c * (c + rowCount(s));
    }
    return values;
}

std::int64_t Symbolic::factorEntryCount() const
{
    std::int64_t entries = 0;
    for (std::int32_t s = 0; s < supernodeCount; ++s)
    {
        const std::int64_t c = columnCount(s);
        entries += c * (c + 1) / 2 + c * rowCount(s);
    }
    return entries;
}

Symbolic rowStructures(std::int32_t nodeCount, const std::int64_t* offsets, const std::int32_t* neighbours,
                       const std::int32_t* weights, const std::int32_t* nodeAtPosition, std::int32_t supernodeCount,
                       const std::int32_t* firstPosition, const std::int32_t* parent)
{
    if (nodeCount < 0 || supernodeCount < 0 || firstPosition[0] != 0 || firstPosition[supernodeCount] != nodeCount)
        throw Error(STATUS_INVALID_ARGUMENT, "row structures: the supernodes must cover the node positions");
    const auto n = static_cast<std::size_t>(nodeCount);
    std::vector<std::int32_t> positionOf(n, -1);
    for (std::int32_t p = 0; p < nodeCount; ++p)
    {
        const std::int32_t node = nodeAtPosition[p];
        if (node < 0 || node >= nodeCount || positionOf[static_cast<std::size_t>(node)] >= 0)
            throw Error(STATUS_INVALID_ARGUMENT, "row structures: the node order is not a permutation");
        positionOf[static_cast<std::size_t>(node)] = p;
    }
    std::vector<std::int32_t> firstColumnOfPosition(n + 1, 0);
    for (std::int32_t p = 0; p < nodeCount; ++p)
        firstColumnOfPosition[static_cast<std::size_t>(p) + 1] =
            firstColumnOfPosition[static_cast<std::size_t>(p)] + weights[nodeAtPosition[p]];

    Symbolic result;
    result.supernodeCount = supernodeCount;
    result.dofCount = firstColumnOfPosition[n];
    result.firstColumn.resize(static_cast<std::size_t>(supernodeCount) + 1);
    result.parent.assign(parent, parent + supernodeCount);
    for (std::int32_t s = 0; s <= supernodeCount; ++s)
        result.firstColumn[static_cast<std::size_t>(s)] = firstColumnOfPosition[static_cast<std::size_t>(firstPosition[s])];

    // Children lists (increasing), then R(s) at node level, supernode by supernode in increasing order (children
    // first), as marked sets.
    std::vector<std::int32_t> childHead(static_cast<std::size_t>(supernodeCount), -1);
    std::vector<std::int32_t> childNext(static_cast<std::size_t>(supernodeCount), -1);
    for (std::int32_t s = supernodeCount; s-- > 0;)
    {
        const std::int32_t p = parent[s];
        if (p < 0)
            continue;
        if (p <= s || p >= supernodeCount)
            throw Error(STATUS_INVALID_ARGUMENT, "row structures: a parent must follow its child");
        childNext[static_cast<std::size_t>(s)] = childHead[static_cast<std::size_t>(p)];
        childHead[static_cast<std::size_t>(p)] = s;
    }
    std::vector<std::int32_t> marker(n, -1);
    std::vector<std::int64_t> positionStart(static_cast<std::size_t>(supernodeCount) + 1, 0);
    std::vector<std::int32_t> positions;
    result.rowStart.assign(static_cast<std::size_t>(supernodeCount) + 1, 0);
    for (std::int32_t s = 0; s < supernodeCount; ++s)
    {
        const std::int32_t last = firstPosition[s + 1] - 1;
        const std::size_t begin = positions.size();
        const auto add = [&](std::int32_t position)
        {
            if (position <= last || marker[static_cast<std::size_t>(position)] == s)
                return;
            marker[static_cast<std::size_t>(position)] = s;
            positions.push_back(position);
        };
        for (std::int32_t p = firstPosition[s]; p <= last; ++p)
        {
            const std::int32_t node = nodeAtPosition[p];
            for (std::int64_t k = offsets[node]; k < offsets[node + 1]; ++k)
                add(positionOf[static_cast<std::size_t>(neighbours[k])]);
        }
        for (std::int32_t child = childHead[static_cast<std::size_t>(s)]; child >= 0;
             child = childNext[static_cast<std::size_t>(child)])
            for (std::int64_t k = positionStart[static_cast<std::size_t>(child)];
                 k < positionStart[static_cast<std::size_t>(child) + 1]; ++k)
                add(positions[static_cast<std::size_t>(k)]);
        std::sort(positions.begin() + static_cast<std::ptrdiff_t>(begin), positions.end());
        positionStart[static_cast<std::size_t>(s) + 1] = static_cast<std::int64_t>(positions.size());
        for (std::size_t k = begin; k < positions.size(); ++k)
        {
            const std::int32_t position = positions[k];
            for (std::int32_t c = 0; c < weights[nodeAtPosition[position]]; ++c)
                result.rows.push_back(firstColumnOfPosition[static_cast<std::size_t>(position)] + c);
        }
        result.rowStart[static_cast<std::size_t>(s) + 1] = static_cast<std::int64_t>(result.rows.size());
    }
    return result;
}

} // namespace oosgpu
