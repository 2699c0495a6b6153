// Delayed pivots: the front positions of a child's update rows and the restated structure of a factor whose fronts
// delayed pivots (delayed.hpp).

#include "delayed.hpp"

#include "host_api.hpp"

#include <algorithm>
#include <string>

namespace oosgpu
{

std::vector<std::int32_t> positionsInFront(const Plan& plan, std::int32_t s, std::int32_t candidates,
                                           const std::int32_t* childRows, std::int32_t childOrder,
                                           std::int32_t childDelayed, std::int32_t delayedStart)
{
    const device::FrontDesc& f = plan.fronts[static_cast<std::size_t>(s)];
    const std::int32_t* rows = plan.rows.data() + f.rowStart;
    std::vector<std::int32_t> positions(static_cast<std::size_t>(childOrder));
    for (std::int32_t i = 0; i < childOrder; ++i)
    {
        const std::int32_t equation = childRows[i];
        std::int32_t position = -1;
        if (i < childDelayed)
            position = delayedStart + i;
        else if (equation >= f.first && equation < f.first + f.c)
            position = equation - f.first;
        else
        {
            const std::int32_t* at = std::lower_bound(rows, rows + f.r, equation);
            if (at != rows + f.r && *at == equation)
                position = candidates + static_cast<std::int32_t>(at - rows);
        }
        if (position < 0)
            throw Error(STATUS_INTERNAL, "delayed pivots: equation " + std::to_string(equation) +
                                             " of a child's update matrix is not in the front of supernode " +
                                             std::to_string(s));
        positions[static_cast<std::size_t>(i)] = position;
    }
    return positions;
}

namespace
{

// One supernode's front after the factorisation, from the exact path or from the device's pivot order.
struct FrontView
{
    std::int32_t order = 0;
    std::int32_t eliminated = 0;
    const std::int32_t* equations = nullptr;
    const double* subdiagonal = nullptr;
    std::int64_t panel = 0;
};

} // namespace

DelayedStructure restateDelayed(const Plan& plan, const std::vector<std::int32_t>& perm,
                                const std::vector<double>& subdiagonal,
                                const std::vector<std::unique_ptr<ExactOutcome>>& exact)
{
    const std::int32_t count = plan.supernodeCount;
    const std::int32_t n = plan.dimension;
    // the equations of the fronts the exact path left alone: their columns in the device's pivot order, then R(s)
    std::vector<std::int32_t> staticEquations;
    std::vector<std::int64_t> staticStart(static_cast<std::size_t>(count) + 1, 0);
    for (std::int32_t s = 0; s < count; ++s)
    {
        const device::FrontDesc& f = plan.fronts[static_cast<std::size_t>(s)];
        staticStart[static_cast<std::size_t>(s) + 1] =
            staticStart[static_cast<std::size_t>(s)] + (exact[static_cast<std::size_t>(s)] ? 0 : f.c + f.r);
    }
    staticEquations.resize(static_cast<std::size_t>(staticStart.back()));
    std::vector<FrontView> views(static_cast<std::size_t>(count));
    DelayedStructure out;
    for (std::int32_t s = 0; s < count; ++s)
    {
        const device::FrontDesc& f = plan.fronts[static_cast<std::size_t>(s)];
        FrontView& v = views[static_cast<std::size_t>(s)];
        if (const ExactOutcome* x = exact[static_cast<std::size_t>(s)].get())
        {
            v = {x->order, x->eliminated, x->equations.data(), x->subdiagonal.data(), x->panel};
            out.delayedPivots += x->delayed();
            continue;
        }
        std::int32_t* e = staticEquations.data() + staticStart[static_cast<std::size_t>(s)];
        std::copy_n(perm.data() + f.first, f.c, e);
        std::copy_n(plan.rows.data() + f.rowStart, f.r, e + f.c);
        v = {f.c + f.r, f.c, e, subdiagonal.data() + f.first, f.panel};
    }
    // the position where each equation is eliminated
    std::vector<std::int32_t> positionOf(static_cast<std::size_t>(n), -1);
    std::vector<std::int32_t> first(static_cast<std::size_t>(count), 0);
    out.perm.assign(static_cast<std::size_t>(n), 0);
    out.subdiagonal.assign(static_cast<std::size_t>(n), 0.0);
    std::int32_t position = 0;
    for (std::int32_t s = 0; s < count; ++s)
    {
        const FrontView& v = views[static_cast<std::size_t>(s)];
        first[static_cast<std::size_t>(s)] = position;
        for (std::int32_t k = 0; k < v.eliminated; ++k)
        {
            const std::int32_t equation = v.equations[k];
            if (equation < 0 || equation >= n || positionOf[static_cast<std::size_t>(equation)] >= 0 || position >= n)
                throw Error(STATUS_INTERNAL, "delayed pivots: equation " + std::to_string(equation) +
                                                 " eliminated twice or out of range (supernode " + std::to_string(s) +
                                                 ")");
            positionOf[static_cast<std::size_t>(equation)] = position;
            out.perm[static_cast<std::size_t>(position)] = equation;
            out.subdiagonal[static_cast<std::size_t>(position)] = v.subdiagonal[k];
            ++position;
        }
    }
    if (position != n)
        throw Error(STATUS_INTERNAL, "delayed pivots: " + std::to_string(n - position) + " equations never eliminated");
    // the restated supernodes: rows by their elimination positions, places in the parent's front
    std::vector<device::FrontDesc> fronts(plan.fronts);
    std::vector<std::int32_t> rows;
    std::vector<std::int32_t> relpos;
    std::vector<std::int32_t> placeInParent(static_cast<std::size_t>(n), -1);
    std::vector<std::int64_t> rowStart(static_cast<std::size_t>(count), 0);
    for (std::int32_t s = 0; s < count; ++s)
    {
        const FrontView& v = views[static_cast<std::size_t>(s)];
        device::FrontDesc& f = fronts[static_cast<std::size_t>(s)];
        f.first = first[static_cast<std::size_t>(s)];
        f.c = v.eliminated;
        f.r = v.order - v.eliminated;
        f.panel = v.panel;
        f.update = 0;
        f.rowStart = static_cast<std::int64_t>(rows.size());
        rowStart[static_cast<std::size_t>(s)] = f.rowStart;
        for (std::int32_t k = v.eliminated; k < v.order; ++k)
            rows.push_back(positionOf[static_cast<std::size_t>(v.equations[k])]);
    }
    relpos.assign(rows.size(), 0);
    for (std::int32_t p = 0; p < count; ++p)
    {
        const device::FrontDesc& pf = plan.fronts[static_cast<std::size_t>(p)];
        if (pf.childCount == 0)
            continue;
        const FrontView& pv = views[static_cast<std::size_t>(p)];
        for (std::int32_t k = 0; k < pv.order; ++k)
            placeInParent[static_cast<std::size_t>(pv.equations[k])] = k;
        for (std::int32_t q = 0; q < pf.childCount; ++q)
        {
            const std::int32_t ch = plan.children[static_cast<std::size_t>(pf.childStart + q)];
            const FrontView& cv = views[static_cast<std::size_t>(ch)];
            for (std::int32_t k = cv.eliminated; k < cv.order; ++k)
            {
                const std::int32_t place = placeInParent[static_cast<std::size_t>(cv.equations[k])];
                if (place < 0)
                    throw Error(STATUS_INTERNAL, "delayed pivots: a row of supernode " + std::to_string(ch) +
                                                     " is not in its parent's front");
                relpos[static_cast<std::size_t>(rowStart[static_cast<std::size_t>(ch)] + (k - cv.eliminated))] = place;
            }
        }
        for (std::int32_t k = 0; k < pv.order; ++k)
            placeInParent[static_cast<std::size_t>(pv.equations[k])] = -1;
    }
    out.plan = buildSolvePlan(n, std::move(fronts), plan.children, std::move(rows), std::move(relpos), plan.level);
    return out;
}

} // namespace oosgpu
