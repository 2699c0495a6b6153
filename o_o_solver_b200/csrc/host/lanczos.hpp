// The block shift-invert Lanczos eigenvalue solver over a shifted pencil whose factorisations, solves and mass
// products run on the GPU: the reference's BlockLanczos::solve (src/linalg/eigen/BlockLanczos.cpp:84-246) with its
// LanczosRun (src/linalg/eigen/LanczosRun.cpp), MassOrthogonalizer, EigenvectorStore, ShiftStrategy and SturmCheck.
// The Lanczos basis, the blocks and the eigenvectors live in device memory; the projected problem, the Sturm walk and
// the shift strategy are host logic (a few hundred values).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <limits>
#include <memory>
#include <span>
#include <vector>

namespace oosgpu::eigen
{

struct Inertia
{
    std::int64_t positive = 0;
    std::int64_t negative = 0;
    std::int64_t zero = 0;
};

// The ShiftedPencil plug-in (include/oos/linalg/eigen/ShiftedPencil.hpp:55-88) with device blocks: column-major,
// `ld` apart, on the pencil's stream.
class ShiftedPencil
{
public:
    virtual ~ShiftedPencil() = default;
    [[nodiscard]] virtual std::int32_t dimension() const = 0;
    // The inertia of K - shift M (zero > 0: singular, returned, not refused).
    virtual Inertia factorise(double shift) = 0;
    // X <- (K - shift M)^-1 X with the last factor.
    virtual void solve(double* x, std::int64_t ld, std::int64_t columns) = 0;
    // Y <- M X, distinct storage.
    virtual void multiplyMass(const double* x, std::int64_t ldx, double* y, std::int64_t ldy, std::int64_t columns) = 0;
    [[nodiscard]] virtual double diagonalRayleighBound() const = 0;
    [[nodiscard]] virtual cudaStream_t stream() const = 0;
    // The device seconds of the last factorisation (reports).
    [[nodiscard]] virtual double lastFactorSeconds() const = 0;
};

// EigenRequest (include/oos/linalg/eigen/EigenRequest.hpp:21-35).
struct EigenRequest
{
    double lowerBound = -std::numeric_limits<double>::infinity();
    double upperBound = std::numeric_limits<double>::infinity();
    std::size_t modeCount = 0;

    [[nodiscard]] bool startsFromLowest() const noexcept { return !(lowerBound > 0.0); }
    [[nodiscard]] bool hasUpperBound() const noexcept { return upperBound < std::numeric_limits<double>::infinity(); }
};

// LanczosOptions (include/oos/linalg/eigen/BlockLanczos.hpp:21-64), the settings that shape the method.
struct LanczosOptions
{
    std::size_t blockSize = 7;
    std::size_t modesPerShift = 40;
    double convergenceTolerance = 1.0e-10;
    std::size_t maximumShifts = 40;
    std::size_t maximumRestarts = 20;
    std::uint64_t seed = 0x6E61737472616E5FULL;
};

// ShiftPurpose (include/oos/linalg/eigen/ShiftStrategy.hpp:14-27).
enum class ShiftPurpose : int
{
    LowestBound = 0,
    LowerBound = 1,
    UpperBound = 2,
    Advance = 3,
    FillGap = 4
};

struct ShiftRecord
{
    double shift = 0.0;
    ShiftPurpose purpose = ShiftPurpose::Advance;
    std::size_t sturmCount = 0;
    bool hasLanczosRun = false;
    std::size_t blockSteps = 0;
    std::size_t restarts = 0;
    std::size_t convergedCount = 0;
};

struct DeviceFree
{
    void operator()(double* p) const noexcept;
};

// EigenSolution (BlockLanczos.hpp:81-100); the eigenvectors are a device matrix dimension x eigenvalues.size().
struct EigenSolution
{
    std::vector<double> eigenvalues;
    std::unique_ptr<double, DeviceFree> eigenvectors;
    std::int64_t dimension = 0;
    std::vector<double> residualBounds;
    std::vector<ShiftRecord> shifts;
    std::size_t factorisationCount = 0;
    std::size_t verifiedCount = 0;
    bool isComplete = false;
    // Wall seconds of the solve, and the device seconds of its factorisations.
    double seconds = 0.0;
    double factorSeconds = 0.0;
    // Wall seconds of the factorisations (with their host work), of the operator Op = (K - sigma M)^-1 M (the solves
    // and the mass products), of the M-orthogonalisation, and of the projected problem (host).
    double factorWallSeconds = 0.0;
    double operatorSeconds = 0.0;
    double orthogonalisationSeconds = 0.0;
    double projectedSeconds = 0.0;
    std::size_t blockSteps = 0;
};

// SturmCheck (include/oos/linalg/eigen/SturmCheck.hpp:14-70, src/linalg/eigen/SturmCheck.cpp).
struct SturmPoint
{
    double shift = 0.0;
    std::size_t countBelow = 0;
};

struct SturmMismatch
{
    double lower = 0.0;
    double upper = 0.0;
    std::size_t expectedCount = 0;
    std::size_t foundCount = 0;
};

struct SturmVerification
{
    double verifiedUpTo = 0.0;
    std::size_t verifiedCount = 0;
    bool hasMismatch = false;
    SturmMismatch mismatch;
};

class SturmCheck
{
public:
    void addPoint(SturmPoint point);
    [[nodiscard]] const std::vector<SturmPoint>& points() const noexcept { return m_points; }
    [[nodiscard]] std::size_t countBelow(double shift) const;
    [[nodiscard]] SturmVerification verify(std::span<const double> sortedEigenvalues) const;

private:
    std::vector<SturmPoint> m_points;
};

struct ShiftChoice
{
    double shift = 0.0;
    ShiftPurpose purpose = ShiftPurpose::Advance;
};

// ShiftStrategy (include/oos/linalg/eigen/ShiftStrategy.hpp:29-128, src/linalg/eigen/ShiftStrategy.cpp).
class ShiftStrategy
{
public:
    static constexpr double RIGID_SHIFT_FRACTION = 1.0e-6;
    static constexpr double DESCENT_FACTOR = 100.0;
    static constexpr std::size_t MAX_DESCENTS = 8;
    static constexpr double SHIFT_CLEARANCE = 1.0e-8;
    static constexpr double STEP_FRACTION = 0.5;
    static constexpr double SINGULAR_SHIFT_MOVE = 1.0e-6;

    ShiftStrategy(const EigenRequest& request, double scale);

    [[nodiscard]] double scale() const noexcept { return m_scale; }
    [[nodiscard]] ShiftChoice firstShift() const noexcept;
    [[nodiscard]] double descend(double shift) const noexcept;
    [[nodiscard]] double moveOffEigenvalue(double shift, bool isUpward, std::size_t attempt) const noexcept;
    [[nodiscard]] bool isComplete(const SturmVerification& verification) const noexcept;

    struct Selection
    {
        std::size_t first = 0;
        std::size_t count = 0;
    };
    [[nodiscard]] Selection select(std::span<const double> sortedEigenvalues, double lowerPoint,
                                   double upperPoint) const noexcept;
    [[nodiscard]] ShiftChoice nextShift(const SturmVerification& verification,
                                        std::span<const double> sortedEigenvalues,
                                        std::span<const double> ritzEstimates,
                                        std::span<const double> lanczosShifts) const;
    [[nodiscard]] double clear(double shift, std::span<const double> sortedEigenvalues) const noexcept;

private:
    [[nodiscard]] double clearanceAt(double value, double shift) const noexcept;
    [[nodiscard]] bool isNearShift(double shift, std::span<const double> lanczosShifts) const noexcept;

    EigenRequest m_request;
    double m_scale = 1.0;
};

// The eigenvalues (increasing) and eigenvectors (columns, each signed so that its component of largest magnitude,
// the first such, is positive) of a symmetric p x p matrix given by its lower triangle, column-major with leading
// dimension ld: Householder reduction to tridiagonal form and the implicit QL method with Wilkinson's shift
// (Golub & Van Loan, Matrix Computations, 4th ed., §8.3). Throws SolverError when an eigenvalue needs more than 60
// sweeps.
void decomposeSymmetric(const double* a, std::size_t p, std::size_t ld, std::vector<double>& values,
                        std::vector<double>& vectors);

// BlockLanczos::shapeFor (BlockLanczos.cpp:56-72).
struct BasisShape
{
    std::size_t blockSize = 0;
    std::size_t basisColumns = 0;
    std::size_t modesPerShift = 0;
};
BasisShape shapeFor(const LanczosOptions& options, std::size_t dimension, const EigenRequest& request) noexcept;

// Throws std::invalid_argument (as an Error of status INVALID_ARGUMENT) for settings out of range
// (BlockLanczos::BlockLanczos, BlockLanczos.cpp:32-48).
void validate(const LanczosOptions& options);

// BlockLanczos::solve.
// startBlock: the first run's start block (device, dimension x blockSize, leading dimension startLd) given by the
// caller in place of the random one (a learned start); the later runs start from random blocks.
EigenSolution solveModes(ShiftedPencil& pencil, const EigenRequest& request, const LanczosOptions& options,
                         const double* startBlock = nullptr, std::int64_t startLd = 0);

} // namespace oosgpu::eigen
