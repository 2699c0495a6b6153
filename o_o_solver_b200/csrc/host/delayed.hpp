// Delayed pivots of the indefinite factorisation (the reference's grown fronts, MultifrontalDriver.cpp:346-436 and
// FrontAssembly.cpp:32-57): what the exact path leaves for a front, the front positions of a child's update rows in
// its parent's front, and the structure of a factor whose fronts delayed pivots, restated for the solves.
#pragma once

#include "plan.hpp"

#include <cstdint>
#include <memory>
#include <vector>

namespace oosgpu
{

// What the exact path left for one front.
struct ExactOutcome
{
    std::int32_t order = 0;      // its candidates, then its rows R(s)
    std::int32_t candidates = 0; // its c columns, then the columns its children delayed
    std::int32_t eliminated = 0;
    std::vector<std::int32_t> equations; // the equation at each front position, candidates in pivot order
    std::vector<double> subdiagonal;     // e_k of a 2x2 pivot at its first position, 0 elsewhere (eliminated entries)
    std::int64_t panel = 0;              // the panel (order x eliminated, leading dimension order), from the arena
    const double* update = nullptr;      // its update matrix: (order - eliminated)^2 values, lower, column-major
    [[nodiscard]] std::int32_t delayed() const noexcept { return candidates - eliminated; }
};

// The front positions of the rows of a child's update matrix in front s (order: c columns, `delayedIn` delayed
// columns, then R(s)): the child's delayed columns (its first `childDelayed` rows) at delayedStart onwards, its other
// rows at their column of s or after the candidates at their row of R(s). Throws when a row is in neither.
std::vector<std::int32_t> positionsInFront(const Plan& plan, std::int32_t s, std::int32_t candidates,
                                           const std::int32_t* childRows, std::int32_t childOrder,
                                           std::int32_t childDelayed, std::int32_t delayedStart);

// A factor whose fronts delayed pivots, restated in the order its equations were eliminated: supernode s eliminates
// positions [first, first + eliminated) (the supernodes in order), its panel keeps its rows in its front's order
// (eliminated candidates, delayed candidates, R(s)), each row known by the position where its equation is eliminated
// and by its place in the parent's front. The solve plan over it, the equation at each position and the 2x2
// subdiagonals by position.
struct DelayedStructure
{
    Plan plan;
    std::vector<std::int32_t> perm;
    std::vector<double> subdiagonal;
    std::int64_t delayedPivots = 0;
};

// perm / subdiagonal: the device's pivot order of the fronts the exact path left alone (each permuting its own
// columns); exact[s]: the outcome of each front the exact path factorised (null elsewhere).
DelayedStructure restateDelayed(const Plan& plan, const std::vector<std::int32_t>& perm,
                                const std::vector<double>& subdiagonal,
                                const std::vector<std::unique_ptr<ExactOutcome>>& exact);

} // namespace oosgpu
