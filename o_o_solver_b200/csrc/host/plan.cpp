// Builds the GPU plan of a symbolic structure (plan.hpp).

#include "plan.hpp"

#include <algorithm>
#include <cstdint>
#include <string>

namespace oosgpu
{
namespace
{

using device::AssemblyTask;
using device::FrontDesc;
using device::TileTask;

constexpr int BLOCK = 64;
constexpr int PANEL_ROWS = 128;                                     // rows of a pivoted panel-rows task
constexpr int PANEL_ROWS_TASK = device::TILE * device::PANEL_ROW_HALVES; // rows of a panelRowsInverse task

void addList(Plan& plan, std::vector<Launch>& launches, LaunchKind kind, const std::vector<std::int32_t>& list,
             std::int32_t k0 = 0, std::int32_t smemOrder = 0)
{
    if (list.empty())
        return;
    launches.push_back({kind, static_cast<std::int64_t>(plan.lists.size()), static_cast<std::int32_t>(list.size()), k0,
                        smemOrder});
    plan.lists.insert(plan.lists.end(), list.begin(), list.end());
}

void addTiles(Plan& plan, std::vector<Launch>& launches, LaunchKind kind, const std::vector<TileTask>& tiles,
              std::int32_t k0 = 0)
{
    if (tiles.empty())
        return;
    launches.push_back({kind, static_cast<std::int64_t>(plan.tiles.size()), static_cast<std::int32_t>(tiles.size()), k0, 0});
    plan.tiles.insert(plan.tiles.end(), tiles.begin(), tiles.end());
}

// Elements (i, j), i >= j, of a tile of m rows from i0 and n columns from j0 (lower part only when lower).
double lowerElements(std::int64_t i0, std::int64_t j0, std::int64_t m, std::int64_t n, bool lower)
{
    if (!lower)
        return static_cast<double>(m * n);
    double count = 0.0;
    for (std::int64_t jj = 0; jj < n; ++jj)
    {
        const std::int64_t firstRow = std::max<std::int64_t>(0, j0 + jj - i0);
        if (firstRow < m)
            count += static_cast<double>(m - firstRow);
    }
    return count;
}

// The factorisation flops of columns [k0, k1) of a front of order n: per column k, m = n - k - 1 below the diagonal,
// m(m + 1) + 2m (SymbolicFactor::flopCount's count).
double columnFlops(std::int64_t n, std::int64_t k0, std::int64_t k1)
{
    double flops = 0.0;
    for (std::int64_t k = k0; k < k1; ++k)
    {
        const double m = static_cast<double>(n - k - 1);
        flops += m * (m + 1.0) + 2.0 * m;
    }
    return flops;
}

// The forward solve's gather lists of plan.relpos (its transpose, children in increasing order within each slot).
void buildGatherLists(Plan& plan)
{
    const std::int32_t count = plan.supernodeCount;
    if (static_cast<std::int64_t>(plan.rows.size()) > INT32_MAX)
        throw Error(STATUS_INVALID_ARGUMENT, "plan: more than 2^31 row entries");
    const std::size_t slots = static_cast<std::size_t>(plan.dimension) + plan.rows.size();
    plan.gatherStart.assign(slots + 1, 0);
    const auto slotOf = [&](const FrontDesc& p, std::int32_t position)
    {
        return position < p.c ? static_cast<std::size_t>(p.first + position)
                              : static_cast<std::size_t>(plan.dimension) + static_cast<std::size_t>(p.rowStart) +
                                    static_cast<std::size_t>(position - p.c);
    };
    for (std::int32_t s = 0; s < count; ++s)
    {
        const FrontDesc& f = plan.fronts[static_cast<std::size_t>(s)];
        if (f.parent < 0)
            continue;
        const FrontDesc& p = plan.fronts[static_cast<std::size_t>(f.parent)];
        for (std::int64_t k = f.rowStart; k < f.rowStart + f.r; ++k)
            ++plan.gatherStart[slotOf(p, plan.relpos[static_cast<std::size_t>(k)]) + 1];
    }
    for (std::size_t slot = 0; slot < slots; ++slot)
        plan.gatherStart[slot + 1] += plan.gatherStart[slot];
    plan.gatherRows.assign(static_cast<std::size_t>(plan.gatherStart[slots]), 0);
    std::vector<std::int64_t> next(plan.gatherStart.begin(), plan.gatherStart.end() - 1);
    // children of each parent in increasing order: the parent's child list is in that order
    for (std::int32_t s = 0; s < count; ++s)
    {
        const FrontDesc& p = plan.fronts[static_cast<std::size_t>(s)];
        for (std::int32_t q = 0; q < p.childCount; ++q)
        {
            const FrontDesc& ch =
                plan.fronts[static_cast<std::size_t>(plan.children[static_cast<std::size_t>(p.childStart + q)])];
            for (std::int64_t k = ch.rowStart; k < ch.rowStart + ch.r; ++k)
            {
                const std::size_t slot = slotOf(p, plan.relpos[static_cast<std::size_t>(k)]);
                plan.gatherRows[static_cast<std::size_t>(next[slot]++)] = static_cast<std::int32_t>(k);
            }
        }
    }
}

// The chains' progress rests on the order of a chain launch's tasks: every block a task waits on is listed before it
// (forward: a supernode's blocks in increasing order, its update rows after all of them; backward: its blocks from the
// last). Checked on every plan.
void checkChainOrder(const Plan& plan, const std::vector<TileTask>& chain, const std::vector<std::int32_t>& large,
                     const std::vector<std::int32_t>& blocks, bool forward)
{
    std::vector<std::int32_t> listed(large.size(), 0);
    for (const TileTask& task : chain)
    {
        const auto at = std::find(large.begin(), large.end(), task.front);
        if (at == large.end())
            throw Error(STATUS_INTERNAL, "plan: a chain task of a supernode outside its level");
        const auto k = static_cast<std::size_t>(at - large.begin());
        const FrontDesc& f = plan.fronts[static_cast<std::size_t>(task.front)];
        bool inOrder;
        if (task.j0 < 0)
            inOrder = forward && listed[k] == blocks[k] && task.i0 >= f.c && task.i0 < f.c + f.r;
        else
        {
            inOrder = task.j0 == (forward ? listed[k] : blocks[k] - 1 - listed[k]) && task.i0 == task.j0 * BLOCK;
            ++listed[k];
        }
        if (!inOrder)
            throw Error(STATUS_INTERNAL, "plan: a chain task listed before a block it waits on");
    }
}

// The solve launches of one level's supernodes (the forward sweep's into plan.forwardLaunches, the backward sweep's
// into `backward`, emitted later top level first) and the 64-column diagonal blocks whose inverses the solves apply.
void addSolveLevel(Plan& plan, const std::vector<std::int32_t>& members, std::int32_t level,
                   std::vector<Launch>& backward, std::vector<TileTask>& inverseTasks,
                   std::vector<TileTask>& inverseTasksLarge)
{
    const std::size_t forwardBefore = plan.forwardLaunches.size();
    const std::size_t backwardBefore = backward.size();
    // ---- forward sweep ----
    std::vector<std::int32_t> solveSmall;
    std::vector<std::int32_t> solveLarge;
    for (const std::int32_t s : members)
        (plan.fronts[static_cast<std::size_t>(s)].c <= SOLVE_SMALL_COLUMNS ? solveSmall : solveLarge).push_back(s);
    // The small supernodes by width class (at most 16, 32 or SOLVE_SMALL_COLUMNS columns): each launch's shared
    // memory is sized for its widest supernode, so the narrow ones (most of the lowest levels) fit more blocks
    // per SM. The supernodes of one level are independent, so the split changes no result.
    std::vector<std::vector<std::int32_t>> smallClasses(3);
    std::vector<std::int32_t> smallClassColumns(3, 0);
    for (const std::int32_t s : solveSmall)
    {
        const std::int32_t c = plan.fronts[static_cast<std::size_t>(s)].c;
        const std::size_t k = c <= 16 ? 0 : c <= 32 ? 1 : 2;
        smallClasses[k].push_back(s);
        smallClassColumns[k] = std::max(smallClassColumns[k], c);
    }
    for (std::size_t k = 0; k < smallClasses.size(); ++k)
        addList(plan, plan.forwardLaunches, LaunchKind::ForwardSmall, smallClasses[k], 0, smallClassColumns[k]);
    {
        // The children's update rows of the large supernodes, by ranges of GATHER_POSITIONS front positions.
        constexpr std::int32_t GATHER_POSITIONS = 64;
        std::vector<TileTask> ranges;
        for (const std::int32_t s : solveLarge)
        {
            const FrontDesc& f = plan.fronts[static_cast<std::size_t>(s)];
            const std::int32_t n = f.c + f.r;
            for (std::int32_t p0 = 0; p0 < n; p0 += GATHER_POSITIONS)
                ranges.push_back({s, p0, std::min(n, p0 + GATHER_POSITIONS), 0});
        }
        addTiles(plan, plan.forwardLaunches, LaunchKind::ForwardGather, ranges);
    }
    for (const std::int32_t s : members)
    {
        const FrontDesc& f = plan.fronts[static_cast<std::size_t>(s)];
        const bool isLarge = f.c + f.r > SMALL_ORDER; // the factorisation's own split, above
        for (std::int32_t k0 = 0; k0 < f.c; k0 += BLOCK)
            (isLarge ? inverseTasksLarge : inverseTasks).push_back({s, k0, 0, 0});
    }
    // The large supernodes' forward chains, one launch: a task per 64-row block, the blocks of x_F in block order
    // (across the supernodes) before the blocks of the update rows, so that a task waits only on blocks listed before
    // it (TileTask: front, first row, own block or -1, the supernode's first flag).
    std::vector<std::int32_t> chainBlocks(solveLarge.size());
    std::vector<std::int64_t> forwardBase(solveLarge.size());
    std::vector<std::int64_t> backwardBase(solveLarge.size());
    std::int32_t maxBlocks = 0;
    for (std::size_t k = 0; k < solveLarge.size(); ++k)
    {
        const FrontDesc& f = plan.fronts[static_cast<std::size_t>(solveLarge[k])];
        chainBlocks[k] = (f.c + BLOCK - 1) / BLOCK;
        maxBlocks = std::max(maxBlocks, chainBlocks[k]);
        forwardBase[k] = plan.chainFlags;
        backwardBase[k] = plan.chainFlags + chainBlocks[k];
        plan.chainFlags += 2 * static_cast<std::int64_t>(chainBlocks[k]);
    }
    if (plan.chainFlags > INT32_MAX)
        throw Error(STATUS_INVALID_ARGUMENT, "plan: too many 64-column blocks in the large supernodes");
    if (!solveLarge.empty())
    {
        std::vector<TileTask> chain;
        for (std::int32_t b = 0; b < maxBlocks; ++b)
            for (std::size_t k = 0; k < solveLarge.size(); ++k)
                if (b < chainBlocks[k])
                    chain.push_back({solveLarge[k], b * BLOCK, b, static_cast<std::int32_t>(forwardBase[k])});
        for (std::size_t k = 0; k < solveLarge.size(); ++k)
        {
            const FrontDesc& f = plan.fronts[static_cast<std::size_t>(solveLarge[k])];
            for (std::int32_t i0 = f.c; i0 < f.c + f.r; i0 += device::TILE)
                chain.push_back({solveLarge[k], i0, -1, static_cast<std::int32_t>(forwardBase[k])});
        }
        checkChainOrder(plan, chain, solveLarge, chainBlocks, true);
        addTiles(plan, plan.forwardLaunches, LaunchKind::ForwardChain, chain, plan.chainSlots++);
    }

    // ---- backward sweep (collected per level, emitted top level first) ----
    for (std::size_t k = 0; k < smallClasses.size(); ++k)
        addList(plan, backward, LaunchKind::BackwardSmall, smallClasses[k], 0, smallClassColumns[k]);
    // x_F -= L21^T X[R(s)] by 64-column tiles; R(s) longer than SOLVE_ROWS_CHUNK in chunks (task j0: the chunk's
    // first row, k0: its partial's slot, -1 for an unsplit tile), then the partials summed in chunk order.
    std::vector<TileTask> rowTiles;
    std::vector<TileTask> rowSums;
    std::int64_t slots = 0;
    for (const std::int32_t s : solveLarge)
    {
        const FrontDesc& f = plan.fronts[static_cast<std::size_t>(s)];
        if (f.r == 0)
            continue;
        const std::int32_t chunks = (f.r + device::SOLVE_ROWS_CHUNK - 1) / device::SOLVE_ROWS_CHUNK;
        for (std::int32_t i0 = 0; i0 < f.c; i0 += device::TILE)
        {
            if (chunks == 1)
            {
                rowTiles.push_back({s, i0, 0, -1});
                continue;
            }
            rowSums.push_back({s, i0, static_cast<std::int32_t>(slots), chunks});
            for (std::int32_t q = 0; q < chunks; ++q)
                rowTiles.push_back({s, i0, q * device::SOLVE_ROWS_CHUNK, static_cast<std::int32_t>(slots++)});
        }
    }
    if (slots > INT32_MAX)
        throw Error(STATUS_INVALID_ARGUMENT, "plan: too many split backward products in one level");
    plan.rowPartialSlots = std::max(plan.rowPartialSlots, slots);
    addTiles(plan, backward, LaunchKind::BackwardRows, rowTiles);
    addTiles(plan, backward, LaunchKind::BackwardRowsReduce, rowSums);
    // The backward chains, one launch: the blocks of x_F from each supernode's last, by distance from the last.
    if (!solveLarge.empty())
    {
        std::vector<TileTask> chain;
        for (std::int32_t d = 0; d < maxBlocks; ++d)
            for (std::size_t k = 0; k < solveLarge.size(); ++k)
                if (d < chainBlocks[k])
                {
                    const std::int32_t b = chainBlocks[k] - 1 - d;
                    chain.push_back({solveLarge[k], b * BLOCK, b, static_cast<std::int32_t>(backwardBase[k])});
                }
        checkChainOrder(plan, chain, solveLarge, chainBlocks, false);
        addTiles(plan, backward, LaunchKind::BackwardChain, chain, plan.chainSlots++);
    }
    for (std::size_t k = forwardBefore; k < plan.forwardLaunches.size(); ++k)
        plan.forwardLaunches[k].level = level;
    for (std::size_t k = backwardBefore; k < backward.size(); ++k)
        backward[k].level = level;
}

} // namespace

// The algorithmic flops and bytes of every launch of the factorisation (Launch::flops, Launch::bytes).
void annotate(Plan& plan, const std::vector<std::int64_t>& cscTermsOfFront)
{
    constexpr double V = sizeof(double);
    for (Launch& launch : plan.factorLaunches)
    {
        double flops = 0.0;
        double bytes = 0.0;
        const auto front = [&](std::int32_t s) -> const FrontDesc& { return plan.fronts[static_cast<std::size_t>(s)]; };
        const auto childBytes = [&](const FrontDesc& f)
        {
            double b = 0.0;
            for (std::int32_t q = 0; q < f.childCount; ++q)
            {
                const FrontDesc& ch = front(plan.children[static_cast<std::size_t>(f.childStart + q)]);
                b += 3.0 * V * static_cast<double>(ch.r) * (ch.r + 1) / 2.0;
            }
            return b;
        };
        for (std::int32_t k = 0; k < launch.count; ++k)
        {
            const std::size_t at = static_cast<std::size_t>(launch.offset + k);
            switch (launch.kind)
            {
            case LaunchKind::SmallFronts:
            {
                const std::int32_t s = plan.lists[at];
                const FrontDesc& f = front(s);
                const std::int64_t n = f.c + f.r;
                flops += columnFlops(n, 0, f.c);
                // The front's children read, its CSC terms read, its panel and update matrix written.
                bytes += childBytes(f) / 3.0 + 12.0 * static_cast<double>(cscTermsOfFront[static_cast<std::size_t>(s)]) +
                         V * static_cast<double>(n * f.c) + V * static_cast<double>(f.r) * (f.r + 1) / 2.0;
                break;
            }
            case LaunchKind::AssembleFronts:
            {
                // The launch's own range is the element-wise pieces; the accounting follows that range whichever
                // kernel runs it (the staged pieces of the alternative cover the same elements).
                const AssemblyTask& piece = plan.pieces[at];
                const FrontDesc& f = front(piece.front);
                const std::int64_t n = f.c + f.r;
                for (std::int64_t j = piece.j0; j < piece.j1; ++j)
                    bytes += V * static_cast<double>(j < f.c ? n : n - j);
                if (piece.j0 == 0)
                    bytes += childBytes(f) + 12.0 * static_cast<double>(cscTermsOfFront[static_cast<std::size_t>(piece.front)]);
                break;
            }
            case LaunchKind::DiagonalBlocks:
            {
                const FrontDesc& f = front(plan.lists[at]);
                const std::int64_t kb = std::min<std::int64_t>(BLOCK, f.c - launch.k0);
                flops += columnFlops(kb, 0, kb);
                bytes += 2.0 * V * static_cast<double>(kb * (kb + 1) / 2);
                break;
            }
            case LaunchKind::PanelRows:
            {
                const TileTask& t = plan.tiles[at];
                const FrontDesc& f = front(t.front);
                const std::int64_t n = f.c + f.r;
                const std::int64_t kb = std::min<std::int64_t>(BLOCK, f.c - launch.k0);
                const std::int64_t rows = std::min<std::int64_t>(PANEL_ROWS_TASK, n - t.i0);
                flops += static_cast<double>(rows) * static_cast<double>(kb * (kb - 1) + kb);
                bytes += 2.0 * V * static_cast<double>(rows * kb);
                break;
            }
            case LaunchKind::PanelUpdate:
            {
                const TileTask& t = plan.tiles[at];
                const FrontDesc& f = front(t.front);
                const std::int64_t n = f.c + f.r;
                const std::int64_t m = std::min<std::int64_t>(device::TILE, n - t.i0);
                const std::int64_t w = std::min<std::int64_t>(device::TILE, f.c - t.j0);
                const double elements = lowerElements(t.i0, t.j0, m, w, t.i0 == t.j0);
                flops += 2.0 * static_cast<double>(t.k0) * elements;
                bytes += 2.0 * V * elements;
                break;
            }
            case LaunchKind::UpdateMatrix:
            {
                const TileTask& t = plan.tiles[at];
                const FrontDesc& f = front(t.front);
                const std::int64_t m = std::min<std::int64_t>(device::TILE, f.r - t.i0);
                const std::int64_t w = std::min<std::int64_t>(device::TILE, f.r - t.j0);
                const double elements = lowerElements(t.i0, t.j0, m, w, t.i0 == t.j0);
                flops += 2.0 * static_cast<double>(f.c) * elements;
                bytes += 2.0 * V * elements;
                break;
            }
            default:
                break;
            }
        }
        launch.flops = flops;
        launch.bytes = bytes;
    }
}

Plan buildPlan(const Symbolic& symbolic)
{
    Plan plan;
    const std::int32_t count = symbolic.supernodeCount;
    const auto total = static_cast<std::size_t>(count);
    plan.dimension = symbolic.dofCount;
    plan.supernodeCount = count;
    plan.fronts.resize(total);
    plan.rows = symbolic.rows;
    plan.rowEntries = static_cast<std::int64_t>(symbolic.rows.size());
    plan.flops = symbolic.flopCount();
    plan.factorEntries = symbolic.factorEntryCount();

    // Children, in increasing order.
    std::vector<std::int32_t> childCount(total, 0);
    for (std::int32_t s = 0; s < count; ++s)
        if (symbolic.parent[static_cast<std::size_t>(s)] >= 0)
            ++childCount[static_cast<std::size_t>(symbolic.parent[static_cast<std::size_t>(s)])];
    std::vector<std::int32_t> childStart(total + 1, 0);
    for (std::size_t s = 0; s < total; ++s)
        childStart[s + 1] = childStart[s] + childCount[s];
    plan.children.assign(static_cast<std::size_t>(childStart[total]), 0);
    {
        std::vector<std::int32_t> next(childStart.begin(), childStart.end() - 1);
        for (std::int32_t s = 0; s < count; ++s)
        {
            const std::int32_t p = symbolic.parent[static_cast<std::size_t>(s)];
            if (p >= 0)
                plan.children[static_cast<std::size_t>(next[static_cast<std::size_t>(p)]++)] = s;
        }
    }

    // Descriptors: the panels in the reference's layout (supernode s at the sum of c(c + r) before it), the update
    // matrices each its own r x r block.
    std::int64_t panel = 0;
    std::int64_t update = 0;
    for (std::int32_t s = 0; s < count; ++s)
    {
        const auto at = static_cast<std::size_t>(s);
        FrontDesc& f = plan.fronts[at];
        const std::int64_t c = symbolic.columnCount(s);
        const std::int64_t r = symbolic.rowCount(s);
        f.panel = panel;
        f.update = update;
        f.rowStart = symbolic.rowStart[at];
        f.first = symbolic.firstColumn[at];
        f.c = static_cast<std::int32_t>(c);
        f.r = static_cast<std::int32_t>(r);
        f.childStart = childStart[at];
        f.childCount = childCount[at];
        f.parent = symbolic.parent[at];
        panel += c * (c + r);
        update += r * r;
    }
    plan.panelValues = panel;
    plan.updateValues = update;

    // Positions of each supernode's rows in its parent's front (both ascending: a merge).
    plan.relpos.assign(symbolic.rows.size(), 0);
    for (std::int32_t s = 0; s < count; ++s)
    {
        const FrontDesc& f = plan.fronts[static_cast<std::size_t>(s)];
        if (f.parent < 0)
            continue;
        const FrontDesc& p = plan.fronts[static_cast<std::size_t>(f.parent)];
        std::int64_t cursor = p.rowStart;
        const std::int64_t end = p.rowStart + p.r;
        for (std::int64_t k = f.rowStart; k < f.rowStart + f.r; ++k)
        {
            const std::int32_t row = symbolic.rows[static_cast<std::size_t>(k)];
            if (row >= p.first && row < p.first + p.c)
            {
                plan.relpos[static_cast<std::size_t>(k)] = row - p.first;
                continue;
            }
            while (cursor < end && symbolic.rows[static_cast<std::size_t>(cursor)] < row)
                ++cursor;
            if (cursor == end || symbolic.rows[static_cast<std::size_t>(cursor)] != row)
                throw Error(STATUS_INVALID_ARGUMENT, "plan: row " + std::to_string(row) + " of supernode " +
                                                         std::to_string(s) + " is not in its parent's front");
            plan.relpos[static_cast<std::size_t>(k)] = p.c + static_cast<std::int32_t>(cursor - p.rowStart);
        }
    }

    buildGatherLists(plan);

    plan.wOffset.assign(total, 0);
    for (const FrontDesc& f : plan.fronts)
    {
        plan.largestFrontOrder = std::max(plan.largestFrontOrder, f.c + f.r);
        plan.largestColumns = std::max(plan.largestColumns, f.c);
    }
    plan.supernodeOfColumn.assign(static_cast<std::size_t>(plan.dimension), 0);
    for (std::int32_t s = 0; s < count; ++s)
        for (std::int32_t j = symbolic.firstColumn[static_cast<std::size_t>(s)];
             j < symbolic.firstColumn[static_cast<std::size_t>(s) + 1]; ++j)
            plan.supernodeOfColumn[static_cast<std::size_t>(j)] = s;

    // Levels.
    plan.level.assign(total, 0);
    std::int32_t maxLevel = 0;
    for (std::int32_t s = 0; s < count; ++s)
    {
        const std::int32_t p = symbolic.parent[static_cast<std::size_t>(s)];
        if (p >= 0)
            plan.level[static_cast<std::size_t>(p)] =
                std::max(plan.level[static_cast<std::size_t>(p)], plan.level[static_cast<std::size_t>(s)] + 1);
        maxLevel = std::max(maxLevel, plan.level[static_cast<std::size_t>(s)]);
    }
    plan.levelCount = count == 0 ? 0 : maxLevel + 1;
    std::vector<std::vector<std::int32_t>> byLevel(static_cast<std::size_t>(plan.levelCount));
    for (std::int32_t s = 0; s < count; ++s)
        byLevel[static_cast<std::size_t>(plan.level[static_cast<std::size_t>(s)])].push_back(s);

    std::vector<std::vector<Launch>> backwardByLevel(static_cast<std::size_t>(plan.levelCount));
    std::vector<TileTask> inverseTasks;      // the blocks of the small fronts (smallFronts inverts none)
    std::vector<TileTask> inverseTasksLarge; // those of the large fronts (diagonalBlocks inverts them itself)
    for (std::int32_t level = 0; level < plan.levelCount; ++level)
    {
        const auto& members = byLevel[static_cast<std::size_t>(level)];
        const std::size_t factorBefore = plan.factorLaunches.size();
        // ---- factorisation ----
        // Small fronts in three classes of order (shared memory per block follows the class's largest front).
        std::vector<std::int32_t> small64;
        std::vector<std::int32_t> small96;
        std::vector<std::int32_t> small128;
        std::vector<std::int32_t> large;
        std::int32_t order64 = 0;
        std::int32_t order96 = 0;
        std::int32_t order128 = 0;
        for (const std::int32_t s : members)
        {
            const FrontDesc& f = plan.fronts[static_cast<std::size_t>(s)];
            const std::int32_t n = f.c + f.r;
            if (n <= SMALL_ORDER_LOW)
            {
                small64.push_back(s);
                order64 = std::max(order64, n);
            }
            else if (n <= SMALL_ORDER_MIDDLE)
            {
                small96.push_back(s);
                order96 = std::max(order96, n);
            }
            else if (n <= SMALL_ORDER)
            {
                small128.push_back(s);
                order128 = std::max(order128, n);
            }
            else
                large.push_back(s);
        }
        plan.largestSmallOrder = std::max({plan.largestSmallOrder, order64, order96, order128});
        addList(plan, plan.factorLaunches, LaunchKind::SmallFronts, small64, 0, order64);
        addList(plan, plan.factorLaunches, LaunchKind::SmallFronts, small96, 0, order96);
        addList(plan, plan.factorLaunches, LaunchKind::SmallFronts, small128, 0, order128);
        Launch elementwiseAssembly{LaunchKind::AssembleFronts, 0, 0, 0, 0};
        if (!large.empty())
        {
            std::vector<AssemblyTask> pieces;
            std::int32_t maxColumns = 0;
            for (const std::int32_t s : large)
            {
                const FrontDesc& f = plan.fronts[static_cast<std::size_t>(s)];
                const std::int32_t n = f.c + f.r;
                maxColumns = std::max(maxColumns, f.c);
                std::int64_t values = 0;
                std::int32_t start = 0;
                for (std::int32_t p = 0; p < n; ++p)
                {
                    values += n - p;
                    if (values >= ASSEMBLY_PIECE_VALUES || p + 1 == n)
                    {
                        pieces.push_back({s, start, p + 1, 0});
                        start = p + 1;
                        values = 0;
                    }
                }
            }
            // The indefinite sequence assembles element-wise (its launch is kept for it below); the positive definite
            // one by pieces staged in shared memory: bands of STAGE_COLUMNS columns that stop at the panel's edge, each
            // cut into STAGE_ROWS positions (a panel band from row 0, its zeros above the diagonal included; an update
            // band from its diagonal).
            elementwiseAssembly = Launch{LaunchKind::AssembleFronts, static_cast<std::int64_t>(plan.pieces.size()),
                                         static_cast<std::int32_t>(pieces.size()), 0, 0};
            plan.pieces.insert(plan.pieces.end(), pieces.begin(), pieces.end());
            std::vector<AssemblyTask> staged;
            for (const std::int32_t s : large)
            {
                const FrontDesc& f = plan.fronts[static_cast<std::size_t>(s)];
                const std::int32_t n = f.c + f.r;
                for (std::int32_t j0 = 0; j0 < n;)
                {
                    const std::int32_t j1 = std::min(j0 + device::STAGE_COLUMNS, j0 < f.c ? f.c : n);
                    for (std::int32_t i0 = j0 < f.c ? 0 : j0; i0 < n; i0 += device::STAGE_ROWS)
                        staged.push_back({s, j0, j1, i0});
                    j0 = j1;
                }
            }
            Launch assembly = elementwiseAssembly; // variant 1: the staged pieces (altOffset, altCount)
            assembly.altOffset = static_cast<std::int64_t>(plan.stagedPieces.size());
            assembly.altCount = static_cast<std::int32_t>(staged.size());
            plan.factorLaunches.push_back(assembly);
            plan.stagedPieces.insert(plan.stagedPieces.end(), staged.begin(), staged.end());
            // Two-level blocking: the 64-column steps update the trailing columns of their PANEL_MACRO-column macro
            // panel only (K = 64); after a macro panel's last step, its columns update every later column of the panel
            // at once (K = PANEL_MACRO), a quarter of the passes over the trailing panel. Lookahead: that update is
            // split into the next macro panel's columns (the main stream, before its steps) and the columns beyond
            // (a side group, which runs while the next macro panel's steps run; the next split waits for it, since its
            // near part covers columns the side group updates). The two streams touch disjoint columns, and every
            // element still receives its macro panels' terms in order.
            std::int32_t levelLastGroup = -1;
            for (std::int32_t k0 = 0; k0 < maxColumns; k0 += BLOCK)
            {
                std::vector<std::int32_t> diagonal;
                std::vector<TileTask> rowTasks;
                std::vector<TileTask> updateTiles;
                std::vector<TileTask> macroTiles;
                std::vector<TileTask> farTiles;
                const std::int32_t macroStart = k0 / device::PANEL_MACRO * device::PANEL_MACRO;
                for (const std::int32_t s : large)
                {
                    const FrontDesc& f = plan.fronts[static_cast<std::size_t>(s)];
                    if (f.c <= k0)
                        continue;
                    const std::int32_t n = f.c + f.r;
                    const std::int32_t kb = std::min(BLOCK, f.c - k0);
                    const std::int32_t macroEnd = std::min(macroStart + device::PANEL_MACRO, f.c);
                    diagonal.push_back(s);
                    for (std::int32_t i0 = k0 + kb; i0 < n; i0 += PANEL_ROWS_TASK)
                        rowTasks.push_back({s, i0, 0, 0});
                    const std::int32_t origin = k0 + BLOCK;
                    for (std::int32_t j0 = origin; j0 < macroEnd; j0 += device::TILE)
                        for (std::int32_t i0 = j0; i0 < n; i0 += device::TILE)
                            updateTiles.push_back({s, i0, j0, BLOCK});
                    if (origin >= macroEnd)
                        for (std::int32_t j0 = macroEnd; j0 < f.c; j0 += device::TILE)
                            for (std::int32_t i0 = j0; i0 < n; i0 += device::TILE)
                                (j0 < macroEnd + device::PANEL_MACRO ? macroTiles : farTiles)
                                    .push_back({s, i0, j0, macroEnd - macroStart});
                }
                addList(plan, plan.factorLaunches, LaunchKind::DiagonalBlocks, diagonal, k0);
                addTiles(plan, plan.factorLaunches, LaunchKind::PanelRows, rowTasks, k0);
                addTiles(plan, plan.factorLaunches, LaunchKind::PanelUpdate, updateTiles, k0);
                const std::int32_t previousGroup = plan.sideGroups - 1;
                if (!farTiles.empty())
                {
                    addTiles(plan, plan.factorLaunches, LaunchKind::PanelUpdate, farTiles, macroStart);
                    plan.factorLaunches.back().sideGroup = plan.sideGroups;
                    levelLastGroup = plan.sideGroups++;
                }
                if (!macroTiles.empty())
                {
                    addTiles(plan, plan.factorLaunches, LaunchKind::PanelUpdate, macroTiles, macroStart);
                    if (previousGroup >= 0)
                        plan.factorLaunches.back().waitGroup = previousGroup;
                }
            }
            std::vector<TileTask> schur;
            for (const std::int32_t s : large)
            {
                const FrontDesc& f = plan.fronts[static_cast<std::size_t>(s)];
                for (std::int32_t j0 = 0; j0 < f.r; j0 += device::TILE)
                    for (std::int32_t i0 = j0; i0 < f.r; i0 += device::TILE)
                        schur.push_back({s, i0, j0, 0});
            }
            // The longest products first (a tile's work grows with the front's columns).
            std::stable_sort(schur.begin(), schur.end(), [&](const TileTask& x, const TileTask& y)
                             { return plan.fronts[static_cast<std::size_t>(x.front)].c >
                                      plan.fronts[static_cast<std::size_t>(y.front)].c; });
            const std::size_t at = plan.factorLaunches.size();
            addTiles(plan, plan.factorLaunches, LaunchKind::UpdateMatrix, schur);
            if (levelLastGroup >= 0 && plan.factorLaunches.size() > at)
                plan.factorLaunches.back().waitGroup = levelLastGroup;
            // The TMA-fed kernel's 128 x 128 tiles (variant 1, the launch's alternative range), when every front of
            // the launch can be read by a tensor map: a panel that starts on a 16-byte boundary, an even order (its
            // stride a multiple of 16 bytes) and an even c, so that every box's first row, c + i0 + 16 b, is even (a
            // TMA copy's contiguous coordinate times 8 bytes must be a multiple of 16). Each tile carries its front's
            // tensor map index in k0.
            bool tmaFed = !schur.empty();
            for (const std::int32_t s : large)
            {
                const FrontDesc& f = plan.fronts[static_cast<std::size_t>(s)];
                if (f.r > 0 && (f.c % 2 != 0 || f.r % 2 != 0 || f.panel % 2 != 0))
                    tmaFed = false;
            }
            if (tmaFed && plan.factorLaunches.size() > at)
            {
                std::vector<TileTask> wide;
                for (const std::int32_t s : large)
                {
                    const FrontDesc& f = plan.fronts[static_cast<std::size_t>(s)];
                    if (f.r == 0)
                        continue;
                    const auto map = static_cast<std::int32_t>(plan.tmaFronts.size());
                    plan.tmaFronts.push_back(s);
                    for (std::int32_t j0 = 0; j0 < f.r; j0 += device::UPDATE_TILE)
                        for (std::int32_t i0 = j0; i0 < f.r; i0 += device::UPDATE_TILE)
                            wide.push_back({s, i0, j0, map});
                }
                std::stable_sort(wide.begin(), wide.end(), [&](const TileTask& x, const TileTask& y)
                                 { return plan.fronts[static_cast<std::size_t>(x.front)].c >
                                          plan.fronts[static_cast<std::size_t>(y.front)].c; });
                Launch& update = plan.factorLaunches.back();
                update.altOffset = static_cast<std::int64_t>(plan.tiles.size());
                update.altCount = static_cast<std::int32_t>(wide.size());
                plan.tiles.insert(plan.tiles.end(), wide.begin(), wide.end());
            }
            // The same update matrices by 128 x 128 tiles, for the mixed-precision form.
            std::vector<TileTask> mixed;
            for (const std::int32_t s : large)
            {
                const FrontDesc& f = plan.fronts[static_cast<std::size_t>(s)];
                for (std::int32_t j0 = 0; j0 < f.r; j0 += device::MIXED_TILE)
                    for (std::int32_t i0 = j0; i0 < f.r; i0 += device::MIXED_TILE)
                        mixed.push_back({s, i0, j0, 0});
            }
            std::stable_sort(mixed.begin(), mixed.end(), [&](const TileTask& x, const TileTask& y)
                             { return plan.fronts[static_cast<std::size_t>(x.front)].c >
                                      plan.fronts[static_cast<std::size_t>(y.front)].c; });
            if (!schur.empty() && !mixed.empty())
            {
                plan.mixedOfFactorLaunch.resize(plan.factorLaunches.size(), -1);
                plan.mixedOfFactorLaunch[at] = static_cast<std::int32_t>(plan.mixedLaunches.size());
                addTiles(plan, plan.mixedLaunches, LaunchKind::UpdateMatrixMixed, mixed);
            }
        }

        // ---- factorisation, indefinite mode ----
        plan.frontsOfLevel.push_back(members);
        plan.largeFrontsOfLevel.push_back(large);
        addList(plan, plan.pivotedLaunches, LaunchKind::SmallFrontsPivoted, small64, 0, order64);
        addList(plan, plan.pivotedLaunches, LaunchKind::SmallFrontsPivoted, small96, 0, order96);
        addList(plan, plan.pivotedLaunches, LaunchKind::SmallFrontsPivoted, small128, 0, order128);
        if (!large.empty())
        {
            plan.pivotedLaunches.push_back(elementwiseAssembly);
            std::int64_t w = 0;
            std::int32_t maxColumns = 0;
            for (const std::int32_t s : large)
            {
                const FrontDesc& f = plan.fronts[static_cast<std::size_t>(s)];
                plan.wOffset[static_cast<std::size_t>(s)] = w;
                w += static_cast<std::int64_t>(f.c + f.r) * std::min(f.c, device::PANEL_MACRO);
                maxColumns = std::max(maxColumns, f.c);
            }
            plan.wValues = std::max(plan.wValues, w);
            // Two-level blocking as in positive definite mode: a step updates the later columns of its macro panel
            // (K = the step's columns, its slice of W); a finished macro panel updates the rest of the front, the panel's
            // columns and the update matrix's (K = the macro panel's columns, all its W slices). The interchanges of a
            // step stay inside its diagonal block, so they never touch the rows a finished macro panel's update reads.
            for (std::int32_t k0 = 0; k0 < maxColumns; k0 += BLOCK)
            {
                std::vector<std::int32_t> diagonal;
                std::vector<TileTask> earlier;
                std::vector<TileTask> rowTasks;
                std::vector<TileTask> trailing;
                std::vector<TileTask> macroTrailing;
                const std::int32_t macroStart = k0 / device::PANEL_MACRO * device::PANEL_MACRO;
                for (const std::int32_t s : large)
                {
                    const FrontDesc& f = plan.fronts[static_cast<std::size_t>(s)];
                    if (f.c <= k0)
                        continue;
                    const std::int32_t n = f.c + f.r;
                    const std::int32_t kb = std::min(BLOCK, f.c - k0);
                    const std::int32_t macroEnd = std::min(macroStart + device::PANEL_MACRO, f.c);
                    diagonal.push_back(s);
                    for (std::int32_t q = 0; q < k0; q += BLOCK)
                        earlier.push_back({s, q, 0, 0});
                    for (std::int32_t i0 = k0 + kb; i0 < n; i0 += PANEL_ROWS)
                        rowTasks.push_back({s, i0, 0, 0});
                    for (std::int32_t j0 = k0 + kb; j0 < macroEnd; j0 += device::TILE)
                        for (std::int32_t i0 = j0; i0 < n; i0 += device::TILE)
                            trailing.push_back({s, i0, j0, kb});
                    if (k0 + kb < macroEnd)
                        continue;
                    // The rest of the front after the macro panel: the panel's columns, then the update matrix's, in
                    // tiles of 64 that never straddle column c.
                    for (std::int32_t j0 = macroEnd; j0 < n;)
                    {
                        const std::int32_t width = j0 < f.c ? std::min(device::TILE, f.c - j0) : device::TILE;
                        for (std::int32_t i0 = j0; i0 < n; i0 += device::TILE)
                            macroTrailing.push_back({s, i0, j0, macroEnd - macroStart});
                        j0 += width;
                    }
                }
                addList(plan, plan.pivotedLaunches, LaunchKind::PivotedDiagonal, diagonal, k0);
                addTiles(plan, plan.pivotedLaunches, LaunchKind::PermuteEarlierRows, earlier, k0);
                addTiles(plan, plan.pivotedLaunches, LaunchKind::PanelRowsPivoted, rowTasks, k0);
                addTiles(plan, plan.pivotedLaunches, LaunchKind::UpdatePivoted, trailing, k0);
                addTiles(plan, plan.pivotedLaunches, LaunchKind::UpdatePivoted, macroTrailing, macroStart);
            }
        }
        plan.pivotedLaunches.push_back({LaunchKind::LevelEnd, 0, 0, level, 0});

        for (std::size_t k = factorBefore; k < plan.factorLaunches.size(); ++k)
            plan.factorLaunches[k].level = level;
        addSolveLevel(plan, members, level, backwardByLevel[static_cast<std::size_t>(level)], inverseTasks,
                      inverseTasksLarge);
    }
    for (std::int32_t level = plan.levelCount; level-- > 0;)
    {
        const auto& launches = backwardByLevel[static_cast<std::size_t>(level)];
        plan.backwardLaunches.insert(plan.backwardLaunches.end(), launches.begin(), launches.end());
    }
    addTiles(plan, plan.inverseLaunches, LaunchKind::InvertDiagonal, inverseTasks);
    addTiles(plan, plan.inverseLaunchesLarge, LaunchKind::InvertDiagonal, inverseTasksLarge);
    plan.mixedOfFactorLaunch.resize(plan.factorLaunches.size(), -1);
    return plan;
}

Plan buildSolvePlan(std::int32_t dimension, std::vector<FrontDesc> fronts, std::vector<std::int32_t> children,
                    std::vector<std::int32_t> rows, std::vector<std::int32_t> relpos, const std::vector<std::int32_t>& level)
{
    Plan plan;
    plan.dimension = dimension;
    plan.supernodeCount = static_cast<std::int32_t>(fronts.size());
    plan.fronts = std::move(fronts);
    plan.children = std::move(children);
    plan.rows = std::move(rows);
    plan.relpos = std::move(relpos);
    plan.rowEntries = static_cast<std::int64_t>(plan.rows.size());
    plan.level = level;
    buildGatherLists(plan);
    plan.supernodeOfColumn.assign(static_cast<std::size_t>(dimension), 0);
    std::int32_t maxLevel = -1;
    for (std::int32_t s = 0; s < plan.supernodeCount; ++s)
    {
        const FrontDesc& f = plan.fronts[static_cast<std::size_t>(s)];
        if (f.first < 0 || f.c < 0 || f.first + f.c > dimension)
            throw Error(STATUS_INTERNAL, "solve plan: supernode " + std::to_string(s) + " outside the equations");
        for (std::int32_t j = f.first; j < f.first + f.c; ++j)
            plan.supernodeOfColumn[static_cast<std::size_t>(j)] = s;
        plan.largestFrontOrder = std::max(plan.largestFrontOrder, f.c + f.r);
        plan.largestColumns = std::max(plan.largestColumns, f.c);
        maxLevel = std::max(maxLevel, level[static_cast<std::size_t>(s)]);
    }
    plan.levelCount = maxLevel + 1;
    std::vector<std::vector<std::int32_t>> byLevel(static_cast<std::size_t>(plan.levelCount));
    for (std::int32_t s = 0; s < plan.supernodeCount; ++s)
        byLevel[static_cast<std::size_t>(level[static_cast<std::size_t>(s)])].push_back(s);
    std::vector<std::vector<Launch>> backwardByLevel(static_cast<std::size_t>(plan.levelCount));
    std::vector<TileTask> inverseTasks;
    std::vector<TileTask> inverseTasksLarge;
    for (std::int32_t lv = 0; lv < plan.levelCount; ++lv)
        addSolveLevel(plan, byLevel[static_cast<std::size_t>(lv)], lv, backwardByLevel[static_cast<std::size_t>(lv)],
                      inverseTasks, inverseTasksLarge);
    for (std::int32_t lv = plan.levelCount; lv-- > 0;)
    {
        const auto& launches = backwardByLevel[static_cast<std::size_t>(lv)];
        plan.backwardLaunches.insert(plan.backwardLaunches.end(), launches.begin(), launches.end());
    }
    addTiles(plan, plan.inverseLaunches, LaunchKind::InvertDiagonal, inverseTasks);
    addTiles(plan, plan.inverseLaunchesLarge, LaunchKind::InvertDiagonal, inverseTasksLarge);
    return plan;
}

} // namespace oosgpu
