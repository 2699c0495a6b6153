// Shift-invert block Lanczos over a GPU pencil: the types of the request and the answer, the ledger of proven
// eigenvalue counts, the shift planner, the dense symmetric eigensolver of the projected problems, and the entry
// point solveModes (krylov.cu).
//
// The division of labour: everything that scales with the model (the Krylov basis, the blocks, the eigenvectors, every
// product over the rows) lives in HBM and runs as kernels on the pencil's stream; the host keeps the handful of numbers
// that steer the method (the projected matrix, the counts, the shifts) and reads them back once per block step.
//
// The behaviour is the reference's BlockLanczos::solve (src/linalg/eigen/BlockLanczos.cpp:87-244) to the Sturm point:
// the same shifts are factorised for the same reasons, so every inertia count is the reference's. The rules that make
// it so (the rigid-body floor, the descent factor, the clearance around roots already found, the moves off a singular
// shift, the seeds of the random blocks) are stated here as constants; the code that applies them is this project's.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <cstddef>
#include <cstdint>
#include <limits>
#include <memory>
#include <span>
#include <vector>

namespace oosgpu::eigen
{

// Counts of positive, negative and zero pivots of one factorisation of K - sigma M. `negative` is the number of
// eigenvalues below sigma (Sylvester); zero > 0 marks a singular shift.
struct Inertia
{
    std::int64_t positive = 0;
    std::int64_t negative = 0;
    std::int64_t zero = 0;
};

// The operations the solver needs from a pencil (the role of the reference's ShiftedPencil plug-in,
// include/oos/linalg/eigen/ShiftedPencil.hpp:55-88). Blocks are device arrays, column-major, on stream().
class PencilPort
{
public:
    virtual ~PencilPort() = default;
    [[nodiscard]] virtual std::int32_t dimension() const = 0;
    // Factorises K - shift M; a singular shift is reported in the inertia, not thrown.
    virtual Inertia factorise(double shift) = 0;
    // X <- (K - shift M)^-1 X with the last factorisation.
    virtual void solve(double* x, std::int64_t ld, std::int64_t columns) = 0;
    // Y <- M X (Y distinct from X): the right-hand matrix of the pencil (the mass of a vibration problem, B = -K_d of
    // a buckling problem).
    virtual void multiplyMass(const double* x, std::int64_t ldx, double* y, std::int64_t ldy, std::int64_t columns) = 0;
    // Y <- G X, G the matrix of the inner product the operator is self-adjoint in (M for vibration, K for buckling).
    virtual void multiplyInnerProduct(const double* x, std::int64_t ldx, double* y, std::int64_t ldy,
                                      std::int64_t columns) = 0;
    // An estimate of the pencil's scale (max K_ii / M_ii over the DOFs with mass), the unit of the shift rules.
    [[nodiscard]] virtual double diagonalRayleighBound() const = 0;
    [[nodiscard]] virtual cudaStream_t stream() const = 0;
    [[nodiscard]] virtual double lastFactorSeconds() const = 0;
};

// What is wanted: the eigenvalues in [low, high), at most `count` of them (count 0: all of them, which needs a finite
// high end). low <= 0 (or -inf) means "from the lowest".
struct ModeRequest
{
    double low = -std::numeric_limits<double>::infinity();
    double high = std::numeric_limits<double>::infinity();
    std::size_t count = 0;

    [[nodiscard]] bool fromLowest() const noexcept { return !(low > 0.0); }
    [[nodiscard]] bool bounded() const noexcept { return high < std::numeric_limits<double>::infinity(); }
};

// How the Krylov runs are shaped (the reference's LanczosOptions, with its defaults).
struct KrylovSettings
{
    std::size_t block = 7;            // vectors per block step
    std::size_t modesPerShift = 40;   // pairs a run aims at
    double tolerance = 1.0e-10;       // a pair converges when its residual <= tolerance * |theta|
    std::size_t shiftLimit = 40;      // factorisations allowed
    std::size_t restartLimit = 20;    // thick restarts per run
    std::uint64_t seed = 0x6E61737472616E5FULL;
};

// Why a shift was factorised. The codes are part of the C ABI (oosgpu_modes_shifts).
enum class ShiftRole : int
{
    Floor = 0,   // below the lowest eigenvalue (the request starts from the lowest)
    Low = 1,     // the low end of the request
    High = 2,    // the high end of the request
    Advance = 3, // beyond what is confirmed, to find more
    Gap = 4      // inside an interval where eigenvalues are missing
};

// One factorisation of the solve, in order.
struct ShiftLog
{
    double shift = 0.0;
    ShiftRole role = ShiftRole::Advance;
    std::size_t countBelow = 0;
    bool ran = false; // a Krylov run followed at this shift
    std::size_t blockSteps = 0;
    std::size_t restarts = 0;
    std::size_t converged = 0;
};

// Device buffers of the eigen solves come from a process-wide cache of freed buffers (per device and size), so that
// the solves after the first allocate and free nothing: cudaFree synchronises the device, and freeing a solve's
// workspace was measured at up to 1.1 s on a B200 holding a large factor.
double* takeDeviceBuffer(std::size_t bytes, const char* what);
void giveDeviceBuffer(double* p, std::size_t bytes, int device) noexcept;
// Frees every idle buffer of the cache (device -1: of every device); returns the bytes freed.
std::size_t releaseDeviceBuffers(int device) noexcept;

struct DeviceFree
{
    std::size_t bytes = 0;
    int device = 0;
    void operator()(double* p) const noexcept;
};

// The answer: eigenvalues ascending, their M-normalised eigenvectors (device, dimension x values.size()), the residual
// bound of each pair, the factorisations made, and how much of it the counts confirm.
struct ModeResult
{
    std::vector<double> values;
    std::unique_ptr<double, DeviceFree> vectors;
    std::int64_t dimension = 0;
    std::vector<double> residualBounds;
    std::vector<ShiftLog> shifts;
    std::size_t factorisations = 0;
    std::size_t confirmed = 0;
    bool complete = false;
    // Wall seconds of the solve; device seconds of its factorisations; wall seconds of the factorisations, of the
    // operator (solves and mass products), of the M-orthogonalisation, and of the projected problems.
    double seconds = 0.0;
    double factorSeconds = 0.0;
    double factorWallSeconds = 0.0;
    double operatorSeconds = 0.0;
    double orthogonalisationSeconds = 0.0;
    double projectedSeconds = 0.0;
    std::size_t blockSteps = 0;
    // Blocks that met a dependent column and were orthonormalised column by column on the host, and the one-column
    // operator applications that replaced dependent columns.
    std::size_t hostBlocks = 0;
    std::size_t replacementSolves = 0;
    // orthogonalisationSeconds by part: start blocks, block steps, thick restarts, harvests.
    std::array<double, 4> orthogonalisationParts{};
    // Wall seconds outside the phases: the workspace's set-up, the answer's gathering, the workspace's release.
    std::array<double, 3> outsideParts{};
};

// ---- proven counts --------------------------------------------------------------------------------------------------

// `below` eigenvalues lie strictly below `shift`: the negative pivots of one factorisation.
struct CountPoint
{
    double shift = 0.0;
    std::size_t below = 0;
};

// What the proven counts say about a set of eigenvalues found. Walking the points upward, each interval between two
// neighbouring points must hold exactly the difference of their counts; `reach` is the highest point up to which every
// interval did (the lowest point when none did), `confirmed` how many found values those intervals hold. The first
// interval that does not is the gap.
struct Confirmation
{
    double reach = 0.0;
    std::size_t confirmed = 0;
    bool hasGap = false;
    double gapLow = 0.0;
    double gapHigh = 0.0;
    std::size_t proven = 0; // eigenvalues the gap holds by the counts
    std::size_t found = 0;  // eigenvalues found in it
};

// The proven counts, kept sorted by shift. A count that contradicts the others (more eigenvalues below a lower shift
// than below a higher one, or two counts at one shift) is refused: the factorisations cannot be trusted.
class CountLedger
{
public:
    void record(double shift, std::size_t below);
    [[nodiscard]] std::size_t countAt(double shift) const;
    [[nodiscard]] const std::vector<CountPoint>& points() const noexcept { return m_points; }
    [[nodiscard]] Confirmation confirm(std::span<const double> sortedValues) const;

private:
    std::vector<CountPoint> m_points;
};

// ---- where to factorise next ----------------------------------------------------------------------------------------

// The rules of the reference's shift strategy (src/linalg/eigen/ShiftStrategy.cpp:29-193; constants
// include/oos/linalg/eigen/ShiftStrategy.hpp:66-80), which fix every shift and so every Sturm point. Lengths are
// relative to the pencil's scale s (diagonalRayleighBound).
namespace rules
{
constexpr double FLOOR_FRACTION = 1.0e-6;      // the first floor shift: -1e-6 s (below the rigid-body roots)
constexpr double DESCENT = 100.0;              // a floor with roots below it moves down 100-fold
constexpr std::size_t DESCENT_LIMIT = 8;       // ... at most this often
constexpr double CLEARANCE = 1.0e-8;           // relative distance kept from every root found
constexpr std::size_t CLEARANCE_PASSES = 64;
constexpr double STRIDE = 0.5;                 // a blind step: half the span confirmed so far
constexpr double NUDGE = 1.0e-6;               // relative move off a singular shift, per attempt
constexpr std::size_t NUDGE_LIMIT = 3;
constexpr double REUSE_TOLERANCE = 1.0e-3;     // a shift this close (relatively) to a used one counts as used
} // namespace rules

struct ShiftPick
{
    double shift = 0.0;
    ShiftRole role = ShiftRole::Advance;
};

class ShiftPlanner
{
public:
    ShiftPlanner(const ModeRequest& request, double scale);

    [[nodiscard]] double scale() const noexcept { return m_scale; }
    // The first factorisation of a solve.
    [[nodiscard]] ShiftPick opening() const noexcept;
    // The next floor below `shift`, which had eigenvalues under it.
    [[nodiscard]] double deeper(double shift) const noexcept;
    // The attempt-th try near `shift` after a singular factorisation there.
    [[nodiscard]] double nudge(double shift, bool upward, std::size_t attempt) const noexcept;
    // The request is met by what the counts confirm.
    [[nodiscard]] bool satisfied(const Confirmation& confirmation) const noexcept;
    // Which of the sorted values answer the request: [first, first + count).
    struct Window
    {
        std::size_t first = 0;
        std::size_t count = 0;
    };
    [[nodiscard]] Window window(std::span<const double> sortedValues, double lowPoint, double highPoint) const noexcept;
    // Where to factorise next, from the confirmation, the values found, the estimates the last run left (sorted) and
    // the shifts that had a run.
    [[nodiscard]] ShiftPick next(const Confirmation& confirmation, std::span<const double> sortedValues,
                                 std::span<const double> estimates, std::span<const double> usedShifts) const;
    // `shift` moved above every found value it comes too close to.
    [[nodiscard]] double clearOf(double shift, std::span<const double> sortedValues) const noexcept;

private:
    [[nodiscard]] double margin(double value, double shift) const noexcept;
    [[nodiscard]] bool alreadyUsed(double shift, std::span<const double> usedShifts) const noexcept;

    ModeRequest m_request;
    double m_scale = 1.0;
};

// ---- dense symmetric eigenproblem -------------------------------------------------------------------------------------

// Eigenvalues (ascending) and eigenvectors (columns, each signed so that its first largest component is positive) of
// the symmetric p x p matrix whose lower triangle `a` holds (column-major, leading dimension ld): Householder
// tridiagonalisation and implicit QL with Wilkinson's shift (Golub & Van Loan, Matrix Computations, 4th ed., 8.3).
// Throws a SolverError when an eigenvalue needs more than 60 sweeps or a term is not finite.
void decomposeSymmetric(const double* a, std::size_t p, std::size_t ld, std::vector<double>& values,
                        std::vector<double>& vectors);

// ---- the solve ----------------------------------------------------------------------------------------------------------

// The block size, basis width and pairs per run for a request on a pencil of `dimension` equations (the reference's
// BlockLanczos::shapeFor, BlockLanczos.cpp:53-67: a basis of 2 * pairs + 3 blocks, rounded up to whole blocks).
struct KrylovShape
{
    std::size_t block = 0;
    std::size_t basis = 0;
    std::size_t pairs = 0;
};
KrylovShape shapeFor(const KrylovSettings& settings, std::size_t dimension, const ModeRequest& request) noexcept;

// Refuses settings out of range (an invalid-argument Error).
void validate(const KrylovSettings& settings);

// The eigenpairs of `request`. `start` (device, dimension x block, leading dimension startLd) replaces the first run's
// random start block (a learned start); later runs start from random blocks.
ModeResult solveModes(PencilPort& pencil, const ModeRequest& request, const KrylovSettings& settings,
                      const double* start = nullptr, std::int64_t startLd = 0);
// The load factors of a buckling pencil (K phi = lambda B phi, B = -K_d; PencilPort: multiplyMass gives B X,
// multiplyInnerProduct K X) nearest 0 of either sign in the request's range [low, high), at most `count` of them
// (the reference's BlockLanczos::solveBuckling, src/linalg/eigen/BlockLanczosBuckling.cpp): values by increasing
// magnitude, the positive first on a tie.
ModeResult solveBuckling(PencilPort& pencil, const ModeRequest& request, const KrylovSettings& settings);

} // namespace oosgpu::eigen
