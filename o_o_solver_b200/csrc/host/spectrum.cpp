// The host side of the eigen solve that is independent of the GPU (declared in spectrum.hpp): the ledger of proven
// counts, the shift planner, the dense symmetric eigensolver of the projected problems, and the basis shape.

#include "spectrum.hpp"

#include "host_api.hpp"

#include <algorithm>
#include <map>
#include <mutex>
#include <cmath>
#include <string>

namespace oosgpu::eigen
{

namespace
{

constexpr double INFINITE = std::numeric_limits<double>::infinity();
constexpr double EPSILON = std::numeric_limits<double>::epsilon();
constexpr int MAX_QL_SWEEPS = 60;
constexpr double LARGEST_TOLERANCE = 1.0e-2;

std::string text(double value)
{
    return std::to_string(value);
}

// How many of the sorted values lie strictly below x.
std::size_t foundBelow(std::span<const double> sortedValues, double x)
{
    return static_cast<std::size_t>(std::lower_bound(sortedValues.begin(), sortedValues.end(), x) -
                                    sortedValues.begin());
}

// sqrt(a^2 + b^2) by scaling with the larger magnitude (no overflow for finite inputs).
double hypotenuse(double a, double b)
{
    a = std::abs(a);
    b = std::abs(b);
    const double big = std::max(a, b);
    if (big == 0.0)
        return 0.0;
    const double small = std::min(a, b) / big;
    return big * std::sqrt(1.0 + small * small);
}

} // namespace

namespace
{

// Freed buffers kept for reuse, at most CACHE_LIMIT bytes in all; beyond that a buffer is freed at once.
constexpr std::size_t CACHE_LIMIT = std::size_t{4} << 30;

struct BufferCache
{
    std::mutex lock;
    std::multimap<std::pair<int, std::size_t>, double*> idle;
    std::size_t idleBytes = 0;
};

BufferCache& bufferCache()
{
    static BufferCache* cache = new BufferCache(); // never destroyed: the context's teardown frees the buffers
    return *cache;
}

} // namespace

double* takeDeviceBuffer(std::size_t bytes, const char* what)
{
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess)
        throw Error(STATUS_CUDA, std::string(what) + ": no current device");
    BufferCache& cache = bufferCache();
    {
        const std::lock_guard<std::mutex> guard(cache.lock);
        const auto found = cache.idle.find({device, bytes});
        if (found != cache.idle.end())
        {
            double* p = found->second;
            cache.idle.erase(found);
            cache.idleBytes -= bytes;
            return p;
        }
    }
    void* p = nullptr;
    cudaError_t status = cudaMalloc(&p, bytes);
    if (status == cudaErrorMemoryAllocation)
    {
        // give this device's idle buffers back and try once more
        (void)cudaGetLastError();
        const std::lock_guard<std::mutex> guard(cache.lock);
        for (auto it = cache.idle.begin(); it != cache.idle.end();)
            if (it->first.first == device)
            {
                cudaFree(it->second);
                cache.idleBytes -= it->first.second;
                it = cache.idle.erase(it);
            }
            else
                ++it;
        status = cudaMalloc(&p, bytes);
    }
    if (status != cudaSuccess)
        throw Error(status == cudaErrorMemoryAllocation ? STATUS_MEMORY_BUDGET : STATUS_CUDA,
                    std::string(what) + ": " + cudaGetErrorString(status));
    return static_cast<double*>(p);
}

void giveDeviceBuffer(double* p, std::size_t bytes, int device) noexcept
{
    if (p == nullptr)
        return;
    BufferCache& cache = bufferCache();
    {
        const std::lock_guard<std::mutex> guard(cache.lock);
        if (cache.idleBytes + bytes <= CACHE_LIMIT)
        {
            cache.idle.insert({{device, bytes}, p});
            cache.idleBytes += bytes;
            return;
        }
    }
    cudaFree(p);
}

std::size_t releaseDeviceBuffers(int device) noexcept
{
    BufferCache& cache = bufferCache();
    const std::lock_guard<std::mutex> guard(cache.lock);
    std::size_t freed = 0;
    int current = 0;
    cudaGetDevice(&current);
    for (auto it = cache.idle.begin(); it != cache.idle.end();)
        if (device < 0 || it->first.first == device)
        {
            cudaSetDevice(it->first.first);
            cudaFree(it->second);
            freed += it->first.second;
            cache.idleBytes -= it->first.second;
            it = cache.idle.erase(it);
        }
        else
            ++it;
    cudaSetDevice(current);
    return freed;
}

void DeviceFree::operator()(double* p) const noexcept
{
    giveDeviceBuffer(p, bytes, device);
}

// ---- CountLedger ----------------------------------------------------------------------------------------------------

void CountLedger::record(double shift, std::size_t below)
{
    const auto at = std::lower_bound(m_points.begin(), m_points.end(), shift,
                                     [](const CountPoint& p, double s) { return p.shift < s; });
    const bool repeat = at != m_points.end() && at->shift == shift;
    // Counts must not decrease upward: what lies below a lower shift lies below a higher one too.
    const CountPoint* conflict = nullptr;
    if (repeat)
    {
        if (at->below != below)
            conflict = &*at;
    }
    else if (at != m_points.end() && at->below < below)
        conflict = &*at;
    else if (at != m_points.begin() && std::prev(at)->below > below)
        conflict = &*std::prev(at);
    if (conflict != nullptr)
        throw Error(STATUS_SOLVER,
                    "eigenvalue analysis: two factorisations disagree: " + std::to_string(below) +
                        " eigenvalues below " + text(shift) + ", but " + std::to_string(conflict->below) + " below " +
                        text(conflict->shift) + ". The factorisations of K - sigma*M cannot be trusted there (a "
                        "pencil close to singular, or a mass matrix that is not positive semi-definite): look for "
                        "mechanisms without mass and for negative masses");
    if (!repeat)
        m_points.insert(at, {shift, below});
}

std::size_t CountLedger::countAt(double shift) const
{
    const auto at = std::find_if(m_points.begin(), m_points.end(), [&](const CountPoint& p) { return p.shift == shift; });
    if (at == m_points.end())
        throw Error(STATUS_INVALID_ARGUMENT, "count ledger: no factorisation at the shift " + text(shift));
    return at->below;
}

Confirmation CountLedger::confirm(std::span<const double> sortedValues) const
{
    if (m_points.empty())
        throw Error(STATUS_INVALID_ARGUMENT, "count ledger: no Sturm point yet; factorise at a shift first");
    Confirmation result;
    result.reach = m_points.front().shift;
    std::size_t lowIndex = foundBelow(sortedValues, m_points.front().shift);
    for (std::size_t k = 1; k < m_points.size(); ++k)
    {
        const std::size_t highIndex = foundBelow(sortedValues, m_points[k].shift);
        const std::size_t found = highIndex - lowIndex;
        const std::size_t proven = m_points[k].below - m_points[k - 1].below;
        if (found != proven)
        {
            result.hasGap = true;
            result.gapLow = m_points[k - 1].shift;
            result.gapHigh = m_points[k].shift;
            result.proven = proven;
            result.found = found;
            break;
        }
        result.reach = m_points[k].shift;
        result.confirmed += found;
        lowIndex = highIndex;
    }
    return result;
}

// ---- ShiftPlanner ---------------------------------------------------------------------------------------------------

ShiftPlanner::ShiftPlanner(const ModeRequest& request, double scale) : m_request(request)
{
    if (request.count == 0 && !request.bounded())
        throw Error(STATUS_INVALID_ARGUMENT, "eigenvalue request: neither a mode count nor an upper bound; ask for a "
                                             "number of modes, or bound the range from above");
    if (request.bounded() && !request.fromLowest() && !(request.high > request.low))
        throw Error(STATUS_INVALID_ARGUMENT, "eigenvalue request: the upper bound " + text(request.high) +
                                                 " must be above the lower bound " + text(request.low));
    if (request.bounded() && request.fromLowest() && !(request.high > 0.0))
        throw Error(STATUS_INVALID_ARGUMENT, "eigenvalue request: the upper bound " + text(request.high) +
                                                 " must be above 0");
    m_scale = std::isfinite(scale) && scale > 0.0 ? scale : 1.0;
}

ShiftPick ShiftPlanner::opening() const noexcept
{
    if (m_request.fromLowest())
        return {-rules::FLOOR_FRACTION * m_scale, ShiftRole::Floor};
    return {m_request.low, ShiftRole::Low};
}

double ShiftPlanner::deeper(double shift) const noexcept
{
    if (shift < 0.0)
        return shift * rules::DESCENT;
    return -rules::FLOOR_FRACTION * m_scale;
}

double ShiftPlanner::nudge(double shift, bool upward, std::size_t attempt) const noexcept
{
    const double unit = std::max(std::abs(shift), rules::FLOOR_FRACTION * m_scale);
    const double step = rules::NUDGE * static_cast<double>(attempt) * unit;
    return upward ? shift + step : shift - step;
}

bool ShiftPlanner::satisfied(const Confirmation& confirmation) const noexcept
{
    const bool enough = m_request.count > 0 && confirmation.confirmed >= m_request.count;
    const bool covered = m_request.bounded() && confirmation.reach >= m_request.high;
    return enough || covered;
}

ShiftPlanner::Window ShiftPlanner::window(std::span<const double> sortedValues, double lowPoint,
                                          double highPoint) const noexcept
{
    Window w;
    w.first = foundBelow(sortedValues, lowPoint);
    w.count = std::max(foundBelow(sortedValues, highPoint), w.first) - w.first;
    if (m_request.count > 0 && w.count > m_request.count)
        w.count = m_request.count;
    return w;
}

double ShiftPlanner::margin(double value, double shift) const noexcept
{
    return rules::CLEARANCE * std::max({std::abs(value), std::abs(shift), rules::FLOOR_FRACTION * m_scale});
}

double ShiftPlanner::clearOf(double shift, std::span<const double> sortedValues) const noexcept
{
    // A shift on top of a found root would factorise a nearly singular matrix: step over each root it nears, and
    // repeat while a step lands next to another root.
    for (std::size_t pass = 0; pass < rules::CLEARANCE_PASSES; ++pass)
    {
        bool moved = false;
        for (const double root : sortedValues)
        {
            const double keep = margin(root, shift);
            if (std::abs(shift - root) < keep)
            {
                shift = root + keep;
                moved = true;
            }
        }
        if (!moved)
            break;
    }
    return shift;
}

bool ShiftPlanner::alreadyUsed(double shift, std::span<const double> usedShifts) const noexcept
{
    for (const double used : usedShifts)
    {
        const double unit = std::max({std::abs(used), std::abs(shift), rules::FLOOR_FRACTION * m_scale});
        if (std::abs(shift - used) <= rules::REUSE_TOLERANCE * unit)
            return true;
    }
    return false;
}

ShiftPick ShiftPlanner::next(const Confirmation& confirmation, std::span<const double> sortedValues,
                             std::span<const double> estimates, std::span<const double> usedShifts) const
{
    // The interval still open: from the confirmed reach to the top of the gap (or upward without end).
    const double from = confirmation.reach;
    const double to = confirmation.hasGap ? confirmation.gapHigh : INFINITE;
    const ShiftRole role = confirmation.hasGap ? ShiftRole::Gap : ShiftRole::Advance;
    const std::size_t firstInside = foundBelow(sortedValues, from);
    const std::size_t endInside = std::max(foundBelow(sortedValues, to), firstInside);
    const std::span<const double> inside = sortedValues.subspan(firstInside, endInside - firstInside);
    // The lowest estimate strictly above x that still lies inside the interval.
    const auto estimateAbove = [&](double x)
    {
        const auto it = std::upper_bound(estimates.begin(), estimates.end(), x);
        return it != estimates.end() && *it < to ? *it : INFINITE;
    };

    // 1. A gap: an estimate the last run left inside it marks a missing root; go there unless a run was there already.
    if (confirmation.hasGap)
        for (const double estimate : estimates)
            if (estimate > from && estimate < to && !alreadyUsed(estimate, usedShifts))
                return {clearOf(estimate, sortedValues), role};

    // 2. Otherwise beyond the highest root found in the interval (or its low end): halfway to the next estimate above
    //    it, else a blind step of half the span covered, kept below the middle of what remains of a closed interval.
    double proposal = 0.0;
    if (!inside.empty())
    {
        const double top = inside.back();
        const double estimate = estimateAbove(top + margin(top, top));
        if (estimate < INFINITE)
            proposal = 0.5 * (top + estimate);
        else
        {
            proposal = top + rules::STRIDE * std::max(top - from, rules::FLOOR_FRACTION * m_scale);
            if (to < INFINITE)
                proposal = std::min(proposal, 0.5 * (top + to));
        }
    }
    else
    {
        const double estimate = estimateAbove(from);
        if (estimate < INFINITE)
            proposal = estimate;
        else if (to < INFINITE)
            proposal = 0.5 * (from + to);
        else
            proposal = from + std::max(std::abs(from), m_scale);
    }

    // 3. A proposal next to a shift that already had a run would learn nothing new: split the widest stretch between
    //    the interval's ends and the roots found in it instead (its middle, or its first quarter if that was used).
    if (alreadyUsed(proposal, usedShifts))
    {
        std::vector<double> marks;
        marks.reserve(inside.size() + 2);
        marks.push_back(from);
        marks.insert(marks.end(), inside.begin(), inside.end());
        const double last = marks.back();
        marks.push_back(to < INFINITE ? to : last + std::max(last - from, m_scale));
        std::size_t widest = 0;
        for (std::size_t k = 1; k + 1 < marks.size(); ++k)
            if (marks[k + 1] - marks[k] > marks[widest + 1] - marks[widest])
                widest = k;
        const double lo = marks[widest];
        const double hi = marks[widest + 1];
        proposal = 0.5 * (lo + hi);
        if (alreadyUsed(proposal, usedShifts))
            proposal = lo + 0.25 * (hi - lo);
    }
    return {clearOf(proposal, sortedValues), role};
}

// ---- the projected problem ------------------------------------------------------------------------------------------

void decomposeSymmetric(const double* a, std::size_t p, std::size_t ld, std::vector<double>& values,
                        std::vector<double>& vectors)
{
    values.assign(p, 0.0);
    vectors.assign(p * p, 0.0);
    if (p == 0)
        return;
    std::vector<double> m(p * p);
    for (std::size_t j = 0; j < p; ++j)
        for (std::size_t i = j; i < p; ++i)
        {
            if (!std::isfinite(a[i + j * ld]))
                throw Error(STATUS_SOLVER, "symmetric eigenproblem: the term (" + std::to_string(i) + ", " +
                                               std::to_string(j) + ") of the matrix is not finite");
            m[i + j * p] = a[i + j * ld];
            m[j + i * p] = a[i + j * ld];
        }
    std::vector<double>& z = vectors;
    for (std::size_t i = 0; i < p; ++i)
        z[i + i * p] = 1.0;
    // Householder reduction: step k zeroes rows k+2.. of column k with H = I - beta v v^T on rows and columns k+1..;
    // the trailing block becomes H B H = B - v w^T - w v^T (u = beta B v, w = u - (beta/2)(v^T u) v), and Z <- Z H.
    std::vector<double> v(p);
    std::vector<double> u(p);
    for (std::size_t k = 0; k + 2 < p; ++k)
    {
        double scale = 0.0;
        for (std::size_t i = k + 1; i < p; ++i)
            scale = std::max(scale, std::abs(m[i + k * p]));
        if (scale == 0.0)
            continue;
        double sigma = 0.0;
        for (std::size_t i = k + 1; i < p; ++i)
        {
            v[i] = m[i + k * p] / scale;
            sigma += v[i] * v[i];
        }
        double alpha = std::sqrt(sigma);
        if (v[k + 1] > 0.0)
            alpha = -alpha;
        v[k + 1] -= alpha;
        double vv = 0.0;
        for (std::size_t i = k + 1; i < p; ++i)
            vv += v[i] * v[i];
        if (vv == 0.0)
            continue;
        const double beta = 2.0 / vv;
        double vu = 0.0;
        for (std::size_t i = k + 1; i < p; ++i)
        {
            double sum = 0.0;
            for (std::size_t j = k + 1; j < p; ++j)
                sum += m[i + j * p] * v[j];
            u[i] = beta * sum;
            vu += v[i] * u[i];
        }
        const double half = 0.5 * beta * vu;
        for (std::size_t i = k + 1; i < p; ++i)
            u[i] -= half * v[i];
        for (std::size_t j = k + 1; j < p; ++j)
            for (std::size_t i = k + 1; i < p; ++i)
                m[i + j * p] -= v[i] * u[j] + u[i] * v[j];
        m[(k + 1) + k * p] = alpha * scale;
        m[k + (k + 1) * p] = alpha * scale;
        for (std::size_t i = k + 2; i < p; ++i)
        {
            m[i + k * p] = 0.0;
            m[k + i * p] = 0.0;
        }
        for (std::size_t r = 0; r < p; ++r)
        {
            double sum = 0.0;
            for (std::size_t i = k + 1; i < p; ++i)
                sum += z[r + i * p] * v[i];
            sum *= beta;
            for (std::size_t i = k + 1; i < p; ++i)
                z[r + i * p] -= sum * v[i];
        }
    }
    std::vector<double>& d = values;
    std::vector<double> e(p, 0.0); // e[i] couples i and i + 1
    for (std::size_t i = 0; i < p; ++i)
    {
        d[i] = m[i + i * p];
        if (i + 1 < p)
            e[i] = m[(i + 1) + i * p];
    }
    // Implicit QL with Wilkinson's shift: a chase of plane rotations from the bottom of the unreduced block [l, mm].
    for (std::size_t l = 0; l < p; ++l)
    {
        int sweeps = 0;
        while (true)
        {
            std::size_t mm = l;
            for (; mm + 1 < p; ++mm)
            {
                const double dd = std::abs(d[mm]) + std::abs(d[mm + 1]);
                if (std::abs(e[mm]) <= EPSILON * dd)
                    break;
            }
            if (mm == l)
                break;
            if (++sweeps > MAX_QL_SWEEPS)
                throw Error(STATUS_SOLVER, "eigenvalue analysis: the projected eigenproblem did not converge in " +
                                               std::to_string(MAX_QL_SWEEPS) + " QL sweeps");
            double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
            double r = hypotenuse(g, 1.0);
            g = d[mm] - d[l] + e[l] / (g + (g >= 0.0 ? r : -r));
            double s = 1.0;
            double c = 1.0;
            double shiftSum = 0.0;
            bool isSplit = false;
            for (std::size_t i = mm; i-- > l;)
            {
                const double f = s * e[i];
                const double bb = c * e[i];
                r = hypotenuse(f, g);
                e[i + 1] = r;
                if (r == 0.0)
                {
                    d[i + 1] -= shiftSum;
                    e[mm] = 0.0;
                    isSplit = true;
                    break;
                }
                s = f / r;
                c = g / r;
                g = d[i + 1] - shiftSum;
                r = (d[i] - g) * s + 2.0 * c * bb;
                shiftSum = s * r;
                d[i + 1] = g + shiftSum;
                g = c * r - bb;
                for (std::size_t k = 0; k < p; ++k)
                {
                    const double zf = z[k + (i + 1) * p];
                    z[k + (i + 1) * p] = s * z[k + i * p] + c * zf;
                    z[k + i * p] = c * z[k + i * p] - s * zf;
                }
            }
            if (isSplit)
                continue;
            d[l] -= shiftSum;
            e[l] = g;
            e[mm] = 0.0;
        }
    }
    // Increasing order (the first minimum each time), each vector signed by its largest component.
    for (std::size_t i = 0; i + 1 < p; ++i)
    {
        std::size_t k = i;
        for (std::size_t j = i + 1; j < p; ++j)
            if (d[j] < d[k])
                k = j;
        if (k != i)
        {
            std::swap(d[i], d[k]);
            for (std::size_t r = 0; r < p; ++r)
                std::swap(z[r + i * p], z[r + k * p]);
        }
    }
    for (std::size_t j = 0; j < p; ++j)
    {
        std::size_t largest = 0;
        for (std::size_t r = 1; r < p; ++r)
            if (std::abs(z[r + j * p]) > std::abs(z[largest + j * p]))
                largest = r;
        if (z[largest + j * p] < 0.0)
            for (std::size_t r = 0; r < p; ++r)
                z[r + j * p] = -z[r + j * p];
    }
}

// ---- shape and settings -------------------------------------------------------------------------------------------

void validate(const KrylovSettings& settings)
{
    if (settings.block == 0 || settings.modesPerShift == 0)
        throw Error(STATUS_INVALID_ARGUMENT, "BlockLanczos: the block size (" + std::to_string(settings.block) +
                                                 ") and the modes per shift (" +
                                                 std::to_string(settings.modesPerShift) + ") must be at least 1");
    if (!(settings.tolerance > 0.0 && settings.tolerance <= LARGEST_TOLERANCE))
        throw Error(STATUS_INVALID_ARGUMENT, "BlockLanczos: the convergence tolerance must lie in (0, 1e-2], found " +
                                                 text(settings.tolerance));
    if (settings.shiftLimit == 0 || settings.restartLimit == 0)
        throw Error(STATUS_INVALID_ARGUMENT, "BlockLanczos: allow at least one shift and one restart");
}

KrylovShape shapeFor(const KrylovSettings& settings, std::size_t dimension, const ModeRequest& request) noexcept
{
    KrylovShape shape;
    if (dimension == 0)
        return shape;
    // At least three blocks must fit in the space, so a block is at most a third of the dimension.
    shape.block = std::max<std::size_t>(1, std::min(settings.block, dimension / 3));
    shape.pairs = request.count > 0 ? std::min(settings.modesPerShift, request.count) : settings.modesPerShift;
    const std::size_t wanted = (2 * shape.pairs + 3 * shape.block + shape.block - 1) / shape.block * shape.block;
    const std::size_t room = std::max(dimension / shape.block * shape.block, std::min<std::size_t>(dimension, 3));
    shape.basis = std::min(wanted, room);
    return shape;
}

} // namespace oosgpu::eigen
