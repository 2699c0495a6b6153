// The plan of a factorisation on the GPU, built once per symbolic structure on the host (the counterpart of the
// reference's FactorSchedule and SolvePlan, src/linalg/supernodal/FactorSchedule.cpp:24-120, SolvePlan.cpp:59): the
// front descriptors, the positions of every child's rows in its parent's front, the levels of the supernode tree
// (a supernode's level is one more than its highest child's: the fronts of one level are independent), and for
// each level the batched launches of the factorisation and of the sweeps.
#pragma once

#include "../device/common.cuh"
#include "host_api.hpp"

#include <cstdint>
#include <vector>

namespace oosgpu
{

// Fronts whose order is at most SMALL_ORDER are factorised whole in shared memory, one block each.
constexpr int SMALL_ORDER_LOW = 64;
constexpr int SMALL_ORDER_MIDDLE = 96;
constexpr int SMALL_ORDER = 128;
// The columns of a large front's assembly piece: about this many elements of its lower triangle. Smaller pieces
// measured faster (2 M plate: 2^16 10.6 ms, 2^14 9.2 ms, 2^13 9.0 ms a factorisation), as expected if a piece's
// target lines stay in L2 between its clear and its children's additions; no DRAM counters were taken for it.
constexpr std::int64_t ASSEMBLY_PIECE_VALUES = std::int64_t{1} << 13;
// Supernodes with at most this many columns are swept by one block.
constexpr int SOLVE_SMALL_COLUMNS = 64;

enum class LaunchKind : int
{
    SmallFronts,
    AssembleFronts,
    DiagonalBlocks,
    PanelRows,
    PanelUpdate,
    UpdateMatrix,
    ForwardSmall,
    ForwardGather,
    // the large supernodes of a level in one launch of dataflow tasks, one per 64-row block (k0: the launch's ticket
    // counter): the forward sweep's blocks of x_F and of the update rows, the backward sweep's blocks of x_F
    ForwardChain,
    BackwardSmall,
    BackwardRows,
    BackwardChain,
    // indefinite mode
    SmallFrontsPivoted,
    PivotedDiagonal,
    PermuteEarlierRows,
    PanelRowsPivoted,
    UpdatePivoted,
    LevelEnd, // the host checks the level's fronts (k0: the level) and runs the exact path where needed
    // after a factorisation: the inverses of the unit lower diagonal blocks the solves apply
    InvertDiagonal,
    // mixed precision: the update matrices by 128 x 128 tiles on tcgen05 (3xTF32), in place of UpdateMatrix
    UpdateMatrixMixed,
    // the sums of the split products of BackwardRows (supernodes with more than SOLVE_ROWS_CHUNK rows)
    BackwardRowsReduce,
    // the diagonal sweep between the two sweeps (not a plan launch; named in the solves' launch records)
    DiagonalSweep
};

// One batched launch: `count` items from `offset` in the array of its kind (front lists: int32; tiles: TileTask;
// assembly pieces: AssemblyTask); k0 the step's first column; smemOrder the largest front order of a small batch.
struct Launch
{
    LaunchKind kind;
    std::int64_t offset;
    std::int32_t count;
    std::int32_t k0;
    std::int32_t smemOrder;
    // Algorithmic work of the launch (the roofline's numerator): useful flops (the multiply-adds of the lower
    // triangles a launch updates, twice) and the bytes it must move at least.
    double flops = 0.0;
    double bytes = 0.0;
    // Lookahead (positive definite factorisation): sideGroup >= 0 runs the launch on the side stream, after all the
    // launches before it in the list on the main stream (a group's first launch forks the side stream off there);
    // waitGroup >= 0 makes the launch wait until side group waitGroup has finished. Groups count up from 0.
    std::int32_t sideGroup = -1;
    std::int32_t waitGroup = -1;
    // Which kernel runs a launch of this kind, where there are several (AssembleFronts: 0 element-wise on
    // Plan::pieces, 1 staged in shared memory on Plan::stagedPieces; DiagonalBlocks: 0 by 16-column sub-panels,
    // 1 column by column; UpdateMatrix: 0 64 x 64 tiles by cp.async, 1 128 x 128 tiles by TMA).
    std::int32_t variant = 0;
    // The task range of variant 1 where it reads another task array than variant 0 (AssembleFronts: the staged
    // pieces in Plan::stagedPieces; UpdateMatrix: the 128 x 128 tiles of the TMA-fed kernel in Plan::tiles); the
    // launch's own range (offset, count) is variant 0's.
    std::int64_t altOffset = 0;
    std::int32_t altCount = 0;
    // The level of the supernodes the launch works on (factorisation and solve launches): a partial factorisation
    // runs the levels below its trailing supernode's.
    std::int32_t level = -1;
};

constexpr int LAUNCH_KIND_COUNT = 14;

struct Plan
{
    std::int32_t dimension = 0;
    std::int32_t supernodeCount = 0;
    std::int32_t levelCount = 0;
    std::vector<device::FrontDesc> fronts;
    std::vector<std::int32_t> children;
    std::vector<std::int32_t> rows;
    std::vector<std::int32_t> relpos;
    // The forward solve's gather lists: for each slot (a supernode's column position p < c: slot first + p; an update
    // row k of R(s): slot dimension + rowStart + k) the update rows of the children that land there, children in
    // increasing order: gatherRows[gatherStart[slot] .. gatherStart[slot + 1]) (indexes into the row arrays).
    std::vector<std::int64_t> gatherStart;
    std::vector<std::int32_t> gatherRows;
    std::vector<std::int32_t> supernodeOfColumn;
    std::vector<std::int32_t> level;
    std::int64_t panelValues = 0;
    std::int64_t updateValues = 0;
    std::int64_t rowEntries = 0;
    // Partial products of the split BackwardRows tiles one level needs at most (each 64 x 64 values).
    std::int64_t rowPartialSlots = 0;
    // The chain launches' ticket counters (one per launch) and ready flags (one per 64-column block of a large
    // supernode and sweep direction), reset before each sweep.
    std::int32_t chainSlots = 0;
    std::int64_t chainFlags = 0;
    std::int32_t largestSmallOrder = 0;
    double flops = 0.0;
    std::int64_t factorEntries = 0;

    // Task arrays (uploaded once) and the launch sequences that index them.
    std::vector<std::int32_t> lists;
    std::vector<device::TileTask> tiles;
    std::vector<device::AssemblyTask> pieces;
    // The fronts whose update matrices the TMA-fed kernel can take, in the order of their tensor maps.
    std::vector<std::int32_t> tmaFronts;
    // The staged extend-add's pieces (AssemblyTask.pad: the piece's first front position).
    std::vector<device::AssemblyTask> stagedPieces;
    std::vector<Launch> factorLaunches;
    std::vector<Launch> forwardLaunches;
    std::vector<Launch> backwardLaunches;
    // The 64-column diagonal blocks (front, k0) of every supernode, inverted after each factorisation into the blocks'
    // upper triangles (the solves apply the inverses).
    // The diagonal inverses after a factorisation: of the small fronts' blocks, and of the large fronts' blocks
    // (which diagonalBlocks writes itself; the indefinite path recomputes them).
    std::vector<Launch> inverseLaunches;
    std::vector<Launch> inverseLaunchesLarge;
    // Mixed precision: for each factorisation launch, the index of the launch that replaces it (-1: none).
    std::vector<Launch> mixedLaunches;
    std::vector<std::int32_t> mixedOfFactorLaunch;
    // The side groups of the factor launches (Launch::sideGroup): 0 .. sideGroups - 1.
    std::int32_t sideGroups = 0;

    // Indefinite mode: the launches (assembly shared with the positive definite sequence), the large fronts of each
    // level, and each large front's W buffer (n x min(c, PANEL_MACRO) values at wOffset: the W = L D columns of its
    // current macro panel; the fronts of one level apart, the levels sharing the buffer).
    std::vector<Launch> pivotedLaunches;
    std::vector<std::vector<std::int32_t>> largeFrontsOfLevel;
    std::vector<std::vector<std::int32_t>> frontsOfLevel;
    std::vector<std::int64_t> wOffset;
    std::int64_t wValues = 0;
    std::int32_t largestFrontOrder = 0;
    std::int32_t largestColumns = 0;
};

// Builds the plan of a validated symbolic structure.
Plan buildPlan(const Symbolic& symbolic);

// The solve part of a plan (the gather lists, the columns' supernodes, the forward and backward sweeps' launches and
// the diagonal blocks to invert) over a structure given directly: supernode s owns the equations [first, first + c)
// of the solve's order, its panel (c + r rows, ld c + r) at fronts[s].panel, its r rows below at rows[rowStart ..]
// (equations of the solve's order) and their positions in the parent's front at relpos[rowStart ..] (< c of the
// parent: its column; else c + its row). `level`: each supernode's level (a parent above its children).
Plan buildSolvePlan(std::int32_t dimension, std::vector<device::FrontDesc> fronts, std::vector<std::int32_t> children,
                    std::vector<std::int32_t> rows, std::vector<std::int32_t> relpos, const std::vector<std::int32_t>& level);

// Sets the algorithmic flops and bytes of every factorisation launch; cscTermsOfFront: the matrix terms in each
// supernode's columns.
void annotate(Plan& plan, const std::vector<std::int64_t>& cscTermsOfFront);

} // namespace oosgpu
