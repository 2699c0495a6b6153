// The indefinite multifrontal LDL^T on the GPU (the reference's PivotingMode::Indefinite: the shifted matrices of the
// eigenvalue solver), and the pieces of the solves that follow its pivots.
//
// - bunchKaufman: the reference's Bunch-Kaufman pivoting restricted to a front's candidate columns
//   (src/linalg/kernels/reference/DenseBlockKernels.cpp:448-580, LAPACK dsytf2, lower): 1x1 and 2x2 pivots with
//   alpha = (1 + sqrt 17) / 8, a candidate whose column maximum lies outside the candidates taken as a 1x1 pivot when
//   |a_kk| >= 0.01 colmax and delayed otherwise, ties of the maxima to the first index. It runs on a whole small front
//   in shared memory (smallFrontsPivoted), on a large front's diagonal block (pivotedDiagonal), and on a whole front
//   in global memory (exactFront, the exact path of a front the block path refuses, or that delays, or grows).
//   The candidates its passes cannot pivot are delayed to the parent front, as the reference delays them
//   (MultifrontalDriver.cpp:346-436): a front that delays is refactorised by the exact path (exactFront), which
//   leaves the delayed candidates in its update matrix; its parent is assembled with them as extra candidate columns
//   (a grown front) by the exact path too.
// - large fronts, per 64-column block: Bunch-Kaufman inside the diagonal block (its columns are all candidates and its
//   rows the only ones searched), then the rows below solved against it (L = A L11^-T D^-1, 2x2 blocks by the dsytf2
//   formula) with an a-posteriori threshold test |l_ij| <= 1/u, u = 0.01 (the reference's delay threshold), and the
//   trailing front updated by tile products C -= L W^T with W = L D. A front whose test fails is refactorised by the
//   exact path. The pivots may differ from the reference's, the inertia may not (Sylvester's law): every Sturm count
//   is the reference's.
// - the pivot order: without delays every supernode permutes only its own columns, so the factor is P A P^T = L D L^T
//   with P a permutation within each supernode's columns; the solves run in pivot order on the same kernels, with the
//   maps of rows remapped (remapPivotOrder) and 2x2 blocks in the diagonal sweep. With delays the host restates the
//   structure in the order the equations were eliminated (each supernode's eliminated columns, its delayed candidates
//   among its rows) and the same solve kernels run on that.

#include "assembly.cuh"
#include "kernels.cuh"

#include <cstdint>

namespace oosgpu::device
{

namespace
{

constexpr double BK_ALPHA = 0.6403882032022076;  // (1 + sqrt(17)) / 8
constexpr double DELAY_THRESHOLD = 0.01;          // the reference's DELAYED_PIVOT_THRESHOLD
constexpr double GROWTH_LIMIT = 1.0 / DELAY_THRESHOLD;

// The column maximum |a(i, k)| over i in (k, n) and its first row, on the whole block (ties to the first index).
// scratchValue / scratchIndex: one slot per warp.
template <typename At>
__device__ void columnMax(At at, int k, int n, double* scratchValue, int* scratchIndex, double& best, int& where)
{
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int warps = blockDim.x >> 5;
    double value = 0.0;
    int index = k;
    for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x)
    {
        const double v = fabs(at(i, k));
        if (v > value)
        {
            value = v;
            index = i;
        }
    }
    for (int offset = 16; offset > 0; offset >>= 1)
    {
        const double v = __shfl_xor_sync(0xffffffffu, value, offset);
        const int idx = __shfl_xor_sync(0xffffffffu, index, offset);
        if (v > value || (v == value && idx < index))
        {
            value = v;
            index = idx;
        }
    }
    if (lane == 0)
    {
        scratchValue[warp] = value;
        scratchIndex[warp] = index;
    }
    __syncthreads();
    best = 0.0;
    where = k;
    for (int w = 0; w < warps; ++w)
        if (scratchValue[w] > best || (scratchValue[w] == best && scratchIndex[w] < where && scratchValue[w] > 0.0))
        {
            best = scratchValue[w];
            where = scratchIndex[w];
        }
    __syncthreads();
}

// max |a(imax, j)| over j in [k, imax) and |a(i, imax)| over i in (imax, n).
template <typename At>
__device__ double rowMax(At at, int k, int imax, int n, double* scratchValue)
{
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int warps = blockDim.x >> 5;
    double value = 0.0;
    for (int j = k + threadIdx.x; j < imax; j += blockDim.x)
        value = fmax(value, fabs(at(imax, j)));
    for (int i = imax + 1 + threadIdx.x; i < n; i += blockDim.x)
        value = fmax(value, fabs(at(i, imax)));
    for (int offset = 16; offset > 0; offset >>= 1)
        value = fmax(value, __shfl_xor_sync(0xffffffffu, value, offset));
    if (lane == 0)
        scratchValue[warp] = value;
    __syncthreads();
    double best = 0.0;
    for (int w = 0; w < warps; ++w)
        best = fmax(best, scratchValue[w]);
    __syncthreads();
    return best;
}

// The symmetric interchange of rows and columns s < t of the lower-stored block: the rows s and t of the columns
// before s, the two diagonal terms, the column s and the row t between them, the columns s and t below t.
template <typename At> __device__ void swapSymmetric(At at, int n, int s, int t)
{
    for (int e = threadIdx.x; e < n; e += blockDim.x)
    {
        if (e < s)
        {
            const double x = at(s, e);
            at(s, e) = at(t, e);
            at(t, e) = x;
        }
        else if (e == s)
        {
            const double x = at(s, s);
            at(s, s) = at(t, t);
            at(t, t) = x;
        }
        else if (e < t)
        {
            const double x = at(e, s);
            at(e, s) = at(t, e);
            at(t, e) = x;
        }
        else if (e > t)
        {
            const double x = at(e, s);
            at(e, s) = at(e, t);
            at(e, t) = x;
        }
    }
    __syncthreads();
}

struct TwoByTwoInverse
{
    double d11;
    double d22;
    double s;
};

// The coefficients of the inverse of a 2 x 2 pivot [[a, b], [b, c]] in LAPACK dsytf2's form (no determinant formed):
// x0 = s (d11 r0 - r1), x1 = s (d22 r1 - r0).
__device__ __forceinline__ TwoByTwoInverse invertTwoByTwo(double a, double b, double c)
{
    const double d11 = c / b;
    const double d22 = a / b;
    const double t = 1.0 / __dsub_rn(__dmul_rn(d11, d22), 1.0);
    return {d11, d22, t / b};
}

// Bunch-Kaufman on the block `at` (n x n lower, the first `candidates` columns the candidates) by the whole thread
// block. perm: the block positions' origins (permuted with the interchanges); subdiagonal: e_k of each 2x2 pivot at its
// first column, 0 elsewhere. A candidate whose column maximum lies outside the untried candidates and whose diagonal is
// below DELAY_THRESHOLD of it is moved behind them and retried in the next pass, as long as a pass eliminates
// something. Returns the columns eliminated; positions [eliminated, candidates) then hold the delayed candidates.
template <typename At>
__device__ int bunchKaufman(At at, int n, int candidates, int* perm, double* subdiagonal, double* scratchValue,
                            int* scratchIndex)
{
    for (int i = threadIdx.x; i < candidates; i += blockDim.x)
    {
        perm[i] = i;
        subdiagonal[i] = 0.0;
    }
    __syncthreads();
    int k = 0;
    int end = candidates;
    int passStart = 0;
    while (true)
    {
        while (k < end)
        {
            const double absakk = fabs(at(k, k));
            double colmax;
            int imax;
            columnMax(at, k, n, scratchValue, scratchIndex, colmax, imax);
            if (absakk == 0.0 && colmax == 0.0)
            {
                k += 1; // a zero column: a zero pivot, L(:, k) = 0
                continue;
            }
            int blockSize = 1;
            int swapWith = k;
            if (absakk < BK_ALPHA * colmax && imax >= end)
            {
                if (absakk < DELAY_THRESHOLD * colmax)
                {
                    --end;
                    if (k != end)
                    {
                        swapSymmetric(at, n, k, end);
                        if (threadIdx.x == 0)
                        {
                            const int x = perm[k];
                            perm[k] = perm[end];
                            perm[end] = x;
                        }
                        __syncthreads();
                    }
                    continue;
                }
            }
            else if (absakk < BK_ALPHA * colmax)
            {
                const double rowmax = rowMax(at, k, imax, n, scratchValue);
                if (absakk >= BK_ALPHA * colmax * (colmax / rowmax))
                    swapWith = k;
                else if (fabs(at(imax, imax)) >= BK_ALPHA * rowmax)
                    swapWith = imax;
                else
                {
                    swapWith = imax;
                    blockSize = 2;
                }
            }
            const int moved = k + blockSize - 1;
            if (swapWith != moved)
            {
                swapSymmetric(at, n, moved, swapWith);
                if (threadIdx.x == 0)
                {
                    const int x = perm[moved];
                    perm[moved] = perm[swapWith];
                    perm[swapWith] = x;
                }
                __syncthreads();
            }
            // Every product and difference rounded on its own (no fused multiply-adds), in the reference family's
            // order: the same bits as its unblocked kernel on the same front.
            if (blockSize == 1)
            {
                const double pivot = at(k, k);
                for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x)
                    at(i, k) = at(i, k) / pivot;
                __syncthreads();
                const int warp = threadIdx.x >> 5;
                const int warps = blockDim.x >> 5;
                const int lane = threadIdx.x & 31;
                for (int j = k + 1 + warp; j < n; j += warps)
                {
                    const double w = __dmul_rn(at(j, k), pivot);
                    for (int i = j + lane; i < n; i += 32)
                        at(i, j) = __dsub_rn(at(i, j), __dmul_rn(at(i, k), w));
                }
                __syncthreads();
            }
            else
            {
                const double d0 = at(k, k);
                const double e = at(k + 1, k);
                const double d1 = at(k + 1, k + 1);
                const TwoByTwoInverse inverse = invertTwoByTwo(d0, e, d1);
                __syncthreads();
                for (int i = k + 2 + threadIdx.x; i < n; i += blockDim.x)
                {
                    const double r0 = at(i, k);
                    const double r1 = at(i, k + 1);
                    at(i, k) = __dmul_rn(inverse.s, __dsub_rn(__dmul_rn(inverse.d11, r0), r1));
                    at(i, k + 1) = __dmul_rn(inverse.s, __dsub_rn(__dmul_rn(inverse.d22, r1), r0));
                }
                if (threadIdx.x == 0)
                {
                    subdiagonal[k] = e;
                    at(k + 1, k) = 0.0;
                }
                __syncthreads();
                const int warp = threadIdx.x >> 5;
                const int warps = blockDim.x >> 5;
                const int lane = threadIdx.x & 31;
                for (int j = k + 2 + warp; j < n; j += warps)
                {
                    const double w0 = __dadd_rn(__dmul_rn(at(j, k), d0), __dmul_rn(at(j, k + 1), e));
                    const double w1 = __dadd_rn(__dmul_rn(at(j, k), e), __dmul_rn(at(j, k + 1), d1));
                    for (int i = j + lane; i < n; i += 32)
                    {
                        double v = at(i, j);
                        v = __dsub_rn(v, __dmul_rn(at(i, k), w0));
                        v = __dsub_rn(v, __dmul_rn(at(i, k + 1), w1));
                        at(i, j) = v;
                    }
                }
                __syncthreads();
            }
            k += blockSize;
        }
        // the delayed candidates get another pass after this one's pivots, as long as a pass eliminates something
        if (end == candidates || k == passStart)
            break;
        passStart = k;
        end = candidates;
    }
    return k;
}

struct SharedAt
{
    double* a;
    int ld;
    __device__ double& operator()(int i, int j) const { return a[i + j * ld]; }
};

struct GlobalAt
{
    double* a;
    std::int64_t ld;
    __device__ double& operator()(int i, int j) const { return a[i + static_cast<std::int64_t>(j) * ld]; }
};

} // namespace

// ------------------------------------------------------------------------------------------------------------------
// Small fronts, indefinite: assembled in shared memory as smallFronts does, then Bunch-Kaufman on the c candidates;
// the panel (pivot order), the 2x2 subdiagonals, the permutation of the supernode's columns and the update matrix
// written out. A front that delays a pivot is flagged (status bit 2, the columns it eliminated from bit 8) and
// refactorised by the exact path, which keeps the delayed candidates.
// ------------------------------------------------------------------------------------------------------------------
__global__ void smallFrontsPivoted(FactorArgs args, PivotArgs pivots, const std::int32_t* list,
                                   std::int32_t* structureError)
{
    extern __shared__ double front[];
    __shared__ double scratchValue[32];
    __shared__ int scratchIndex[32];
    __shared__ int perm[128];
    __shared__ double sub[128];
    const std::int32_t s = list[blockIdx.x];
    const FrontDesc f = args.fronts[s];
    const int n = f.c + f.r;
    const int ld = n + 1;
    assembleFrontBy(
        args, f, [&](int i, int j) -> double& { return front[i + j * ld]; }, structureError);
    const int eliminated = bunchKaufman(SharedAt{front, ld}, n, f.c, perm, sub, scratchValue, scratchIndex);
    if (threadIdx.x == 0 && eliminated < f.c)
        atomicOr(pivots.status + s, 2 | (min(eliminated, 0xfffff) << 8));
    double* panel = args.panels + f.panel;
    for (int e = threadIdx.x; e < n * f.c; e += blockDim.x)
    {
        const int j = e / n;
        const int i = e - j * n;
        panel[e] = i >= j ? front[i + j * ld] : 0.0;
    }
    for (int j = threadIdx.x; j < f.c; j += blockDim.x)
    {
        pivots.perm[f.first + j] = f.first + perm[j];
        pivots.subdiagonal[f.first + j] = sub[j];
    }
    if (f.r > 0)
    {
        double* update = args.updates + f.update;
        for (int e = threadIdx.x; e < f.r * f.r; e += blockDim.x)
        {
            const int j = e / f.r;
            const int i = e - j * f.r;
            if (i >= j)
                update[e] = front[(f.c + i) + (f.c + j) * ld];
        }
    }
}

// ------------------------------------------------------------------------------------------------------------------
// Large fronts, indefinite, step k0: Bunch-Kaufman inside the kb x kb diagonal block. The block's interchanges are
// carried to the supernode's permutation and to the rows of L already computed (columns before k0); the rows below
// the block take them when panelRowsPivotedInverse reads them (pivots.stepPerm).
// ------------------------------------------------------------------------------------------------------------------
__global__ void pivotedDiagonal(FactorArgs args, PivotArgs pivots, const std::int32_t* list, int k0)
{
    constexpr int B = 64;
    constexpr int LD = B + 1;
    __shared__ double a[B * LD];
    __shared__ double scratchValue[32];
    __shared__ int scratchIndex[32];
    __shared__ int perm[B];
    __shared__ double sub[B];
    __shared__ std::int32_t oldOrigin[B];
    __shared__ double products[3 * 16 * 16];
    const std::int32_t s = list[blockIdx.x];
    const FrontDesc f = args.fronts[s];
    const std::int64_t n = f.c + f.r;
    const int kb = min(B, f.c - k0);
    double* block = args.panels + f.panel + k0 + static_cast<std::int64_t>(k0) * n;
    for (int e = threadIdx.x; e < kb * kb; e += blockDim.x)
    {
        const int j = e / kb;
        const int i = e - j * kb;
        copyAsync8(a + i + j * LD, block + i + static_cast<std::int64_t>(j) * n, true);
    }
    commitAsyncCopies();
    waitAsyncCopies<0>();
    __syncthreads();
    // A candidate the block cannot pivot sends the front to the exact path (status bit 1), as a failed growth test.
    const int eliminated = bunchKaufman(SharedAt{a, LD}, kb, kb, perm, sub, scratchValue, scratchIndex);
    if (eliminated < kb && threadIdx.x == 0)
        atomicOr(pivots.status + s, 1);
    for (int e = threadIdx.x; e < kb * kb; e += blockDim.x)
    {
        const int j = e / kb;
        const int i = e - j * kb;
        if (i >= j)
            block[i + static_cast<std::int64_t>(j) * n] = a[i + j * LD];
    }
    for (int j = threadIdx.x; j < kb; j += blockDim.x)
    {
        pivots.stepPerm[static_cast<std::int64_t>(s) * B + j] = perm[j];
        pivots.subdiagonal[f.first + k0 + j] = sub[j];
        oldOrigin[j] = pivots.perm[f.first + k0 + j];
    }
    __syncthreads();
    for (int j = threadIdx.x; j < kb; j += blockDim.x)
        pivots.perm[f.first + k0 + j] = oldOrigin[perm[j]];
    if (threadIdx.x == 0)
    {
        int swapped = 0;
        for (int j = 0; j < kb; ++j)
            swapped |= perm[j] != j;
        pivots.stepSwapped[s] = swapped;
    }
    // L11^-1 (unit lower, zero below each 2x2 pivot) into the block's strict upper triangle, as diagonalBlocks does,
    // by 16 x 16 blocks (the identity beyond kb).
    for (int e = threadIdx.x; e < B * B; e += blockDim.x)
    {
        const int q = e / B;
        const int i = e - q * B;
        if (i >= kb || q >= kb)
            a[i + q * LD] = i == q ? 1.0 : 0.0;
    }
    invertUnitLowerBlocked(a, products);
    for (int e = threadIdx.x; e < kb * kb; e += blockDim.x)
    {
        const int i = e / kb;
        const int j = e - i * kb;
        if (i < j)
            block[i + static_cast<std::int64_t>(j) * n] = a[i + j * LD];
    }
}

// The rows below step k0's diagonal block of an indefinite front, as products with the block's inverse: the row's
// entries in the block's columns read in pivot order, Y = A (L11^-1)^T on the FP64 tensor cores (L11^-1 from the
// block's strict upper triangle), then L = Y D^-1 (2x2 blocks by the dsytf2 formula) written to the panel, W = L D = Y
// to the front's W buffer, and a coefficient above 1/u (or not finite) flags the front (status bit 1). 64-row halves
// of a 128-row task; dynamic shared memory PANEL_ROWS_INVERSE_SMEM bytes plus 64 doubles and 64 ints.
__global__ void __launch_bounds__(TILE_THREADS) panelRowsPivotedInverse(FactorArgs args, PivotArgs pivots,
                                                                        const TileTask* tasks, int k0)
{
    constexpr int B = 64;
    constexpr int LD = TILE + TILE_PAD;
    extern __shared__ double stage[];
    double* sA = stage;       // sA[p * LD + ii] = A(ii, perm p); then Y(ii, jj) at sA[jj * LD + ii]
    double* sB = sA + B * LD; // L11^-1(jj, p) at sB[p * LD + jj], unit diagonal, zero above
    double* sd = sB + B * LD; // d_j
    double* se = sd + B;      // e_j of a 2x2 pivot at its first column
    int* sperm = reinterpret_cast<int*>(se + B);
    const TileTask task = tasks[blockIdx.x];
    const std::int32_t s = task.front;
    const FrontDesc f = args.fronts[s];
    const std::int64_t n = f.c + f.r;
    const int kb = min(B, f.c - k0);
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int wm = (warp >> 1) * 32;
    const int wn = (warp & 1) * 32;
    const double* block = args.panels + f.panel + k0 + static_cast<std::int64_t>(k0) * n;
    for (int e = tid; e < B * B; e += blockDim.x)
    {
        const int jj = e / B;
        const int p = e - jj * B;
        const bool inside = p <= jj && jj < kb;
        copyAsync8(sB + p * LD + jj, inside ? block + p + static_cast<std::int64_t>(jj) * n : block, inside);
    }
    for (int j = tid; j < B; j += blockDim.x)
    {
        se[j] = j < kb ? pivots.subdiagonal[f.first + k0 + j] : 0.0;
        sperm[j] = j < kb ? pivots.stepPerm[static_cast<std::int64_t>(s) * B + j] : j;
    }
    commitAsyncCopies();
    waitAsyncCopies<0>();
    __syncthreads();
    for (int j = tid; j < B; j += blockDim.x)
    {
        sd[j] = j < kb ? sB[j * LD + j] : 1.0;
        sB[j * LD + j] = j < kb ? 1.0 : 0.0;
    }
    bool bad = false;
    for (int half = 0; half < 2; ++half)
    {
        const std::int64_t i0 = task.i0 + half * TILE;
        if (i0 >= n)
            break;
        const int m = static_cast<int>(n - i0 < TILE ? n - i0 : TILE);
        double* rows = args.panels + f.panel + i0 + static_cast<std::int64_t>(k0) * n;
        double* w = pivots.w + pivots.wOffset[s] + i0 + static_cast<std::int64_t>(k0 % PANEL_MACRO) * n;
        for (int e = tid; e < B * TILE; e += blockDim.x)
        {
            const int p = e / TILE;
            const int ii = e - p * TILE;
            const bool inside = p < kb && ii < m;
            copyAsync8(sA + p * LD + ii, inside ? rows + ii + static_cast<std::int64_t>(sperm[p]) * n : rows, inside);
        }
        commitAsyncCopies();
        waitAsyncCopies<0>();
        __syncthreads();
        double acc[4][4][2];
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
            {
                acc[mi][ni][0] = 0.0;
                acc[mi][ni][1] = 0.0;
            }
#pragma unroll 4
        for (int kk = 0; kk < B; kk += 4)
        {
            const int pr = kk + (lane & 3);
            double fa[4];
            double fb[4];
#pragma unroll
            for (int mi = 0; mi < 4; ++mi)
                fa[mi] = sA[pr * LD + wm + mi * 8 + (lane >> 2)];
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
                fb[ni] = sB[pr * LD + wn + ni * 8 + (lane >> 2)];
#pragma unroll
            for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni)
                    dmma8x8x4(acc[mi][ni], fa[mi], fb[ni]);
        }
        __syncthreads();
        // Y into shared memory (over A: every product has read it), column jj at sA[jj * LD].
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                for (int h = 0; h < 2; ++h)
                {
                    const int ii = wm + mi * 8 + (lane >> 2);
                    const int jj = wn + ni * 8 + (lane & 3) * 2 + h;
                    sA[jj * LD + ii] = acc[mi][ni][h];
                }
        __syncthreads();
        // L = Y D^-1 by rows, 1x1 and 2x2 pivots.
        if (tid < m)
        {
            const int ii = tid;
            int j = 0;
            while (j < kb)
            {
                if (j + 1 < kb && se[j] != 0.0)
                {
                    const TwoByTwoInverse inverse = invertTwoByTwo(sd[j], se[j], sd[j + 1]);
                    const double r0 = sA[j * LD + ii];
                    const double r1 = sA[(j + 1) * LD + ii];
                    const double l0 = inverse.s * (inverse.d11 * r0 - r1);
                    const double l1 = inverse.s * (inverse.d22 * r1 - r0);
                    rows[ii + static_cast<std::int64_t>(j) * n] = l0;
                    rows[ii + static_cast<std::int64_t>(j + 1) * n] = l1;
                    w[ii + static_cast<std::int64_t>(j) * n] = r0;
                    w[ii + static_cast<std::int64_t>(j + 1) * n] = r1;
                    bad = bad || !(fabs(l0) <= GROWTH_LIMIT) || !(fabs(l1) <= GROWTH_LIMIT);
                    j += 2;
                }
                else
                {
                    const double r0 = sA[j * LD + ii];
                    const double l = r0 / sd[j];
                    rows[ii + static_cast<std::int64_t>(j) * n] = l;
                    w[ii + static_cast<std::int64_t>(j) * n] = r0;
                    bad = bad || !(fabs(l) <= GROWTH_LIMIT);
                    j += 1;
                }
            }
        }
        __syncthreads();
    }
    if (bad)
        atomicOr(pivots.status + s, 1);
}

// The rows of L already computed (columns before k0) follow the diagonal block's interchanges of step k0: a task
// (front, i0) takes the columns [i0, i0 + 64) of it, a warp per column; nothing to do when the block kept its order.
__global__ void permuteEarlierRows(FactorArgs args, PivotArgs pivots, const TileTask* tasks, int k0)
{
    constexpr int B = 64;
    __shared__ double staged[8][B];
    const TileTask task = tasks[blockIdx.x];
    const std::int32_t s = task.front;
    if (pivots.stepSwapped[s] == 0)
        return;
    const FrontDesc f = args.fronts[s];
    const std::int64_t n = f.c + f.r;
    const int kb = min(B, f.c - k0);
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const std::int32_t* perm = pivots.stepPerm + static_cast<std::int64_t>(s) * B;
    for (int q = task.i0 + warp; q < min(task.i0 + B, k0); q += blockDim.x >> 5)
    {
        double* column = args.panels + f.panel + k0 + static_cast<std::int64_t>(q) * n;
        for (int j = lane; j < kb; j += 32)
            staged[warp][j] = column[j];
        __syncwarp();
        for (int j = lane; j < kb; j += 32)
            column[j] = staged[warp][perm[j]];
        __syncwarp();
    }
}

__global__ void identityPermutation(std::int32_t* perm, int dimension)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < dimension)
        perm[j] = j;
}

// A tile of the trailing front minus L W^T over the K = task.k0 columns from k0 (a step's columns within its macro
// panel, or a finished macro panel's): task (front, i0, j0) a 64 x 64 tile of the front, j0 < c in the panel, j0 >= c
// in the update matrix (tiles never straddle c); W's columns for k0 at slice k0 % PANEL_MACRO of the front's buffer.
__global__ void __launch_bounds__(TILE_THREADS, 5) updatePivoted(FactorArgs args, PivotArgs pivots, const TileTask* tasks,
                                                              int k0)
{
    __shared__ double smem[TILE_SMEM_DOUBLES];
    const TileTask task = tasks[blockIdx.x];
    const FrontDesc f = args.fronts[task.front];
    const std::int64_t n = f.c + f.r;
    double* panel = args.panels + f.panel;
    TileOperands op;
    op.a = panel + task.i0 + static_cast<std::int64_t>(k0) * n;
    op.aRowStride = 1;
    op.aColStride = n;
    op.b = pivots.w + pivots.wOffset[task.front] + task.j0 + static_cast<std::int64_t>(k0 % PANEL_MACRO) * n;
    op.bRowStride = 1;
    op.bColStride = n;
    op.bIndex = nullptr;
    op.d = nullptr;
    op.dStride = 0;
    if (task.j0 < f.c)
    {
        op.c = panel + task.i0 + static_cast<std::int64_t>(task.j0) * n;
        op.cColStride = n;
        op.n = min(TILE, f.c - task.j0);
    }
    else
    {
        op.c = args.updates + f.update + (task.i0 - f.c) + static_cast<std::int64_t>(task.j0 - f.c) * f.r;
        op.cColStride = f.r;
        op.n = min(TILE, static_cast<int>(n) - task.j0);
    }
    op.cRowStride = 1;
    op.m = static_cast<int>(n - task.i0 < TILE ? n - task.i0 : TILE);
    op.k = task.k0;
    op.lower = task.i0 == task.j0;
    op.lowerOffset = 0;
    tileProduct(op, smem);
}

// ------------------------------------------------------------------------------------------------------------------
// The exact path of one front (the reference's eliminatePivoted, MultifrontalDriver.cpp:346-436): a front the block
// path refused, a small front that delays pivots, or a front grown by its children's delayed columns. Assembled whole
// in `work` (order x order, global memory; FrontAssembly.cpp:166-300 with delays): its c columns, then the candidate
// columns its children delayed, then its rows R(s); the matrix's entries of its c columns, then each child's update
// matrix in increasing child order at the front positions the host mapped (a delayed child's rows start with its
// delayed columns, whose positions may lie above another row's: such a term lands in the lower triangle, transposed).
// Then Bunch-Kaufman on the candidates by one block; the panel (order x candidates, pivot order) written to x.panel,
// the permutation of the candidates (front positions), their subdiagonals and the count eliminated to the scratch;
// the update matrix stays in `work`, at [eliminated, order), for copyTrailing.
// ------------------------------------------------------------------------------------------------------------------
// The whole front of x assembled by one block into at(i, j) (i >= j, order x order): cleared, the matrix's entries of
// its c columns (rows in the columns, or in R(s) after the candidates), then each source's update matrix at its rows'
// front positions in increasing source order (a term whose positions are out of order lands transposed).
template <typename At>
__device__ void assembleWholeFront(const FactorArgs& args, const ExactFront& x, At at, std::int32_t* structureError)
{
    const FrontDesc f = args.fronts[x.supernode];
    const int order = x.order;
    const int candidates = x.candidates;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int warps = blockDim.x >> 5;
    for (std::int64_t e = tid; e < static_cast<std::int64_t>(order) * order; e += blockDim.x)
    {
        const int j = static_cast<int>(e / order);
        const int i = static_cast<int>(e - static_cast<std::int64_t>(j) * order);
        if (i >= j)
            at(i, j) = 0.0;
    }
    __syncthreads();
    const std::int32_t* rowsOfFront = args.rows + f.rowStart;
    for (int j = warp; j < f.c; j += warps)
    {
        const std::int32_t column = f.first + j;
        for (std::int64_t k = args.colOffsets[column] + lane; k < args.colOffsets[column + 1]; k += 32)
        {
            const std::int32_t row = args.colRows[k];
            int position = -1;
            if (row >= column && row < f.first + f.c)
                position = row - f.first;
            else if (row >= f.first + f.c)
            {
                int lo = 0;
                int hi = f.r;
                while (lo < hi)
                {
                    const int mid = (lo + hi) >> 1;
                    if (rowsOfFront[mid] < row)
                        lo = mid + 1;
                    else
                        hi = mid;
                }
                if (lo < f.r && rowsOfFront[lo] == row)
                    position = candidates + lo;
            }
            if (position < 0)
            {
                atomicMin(structureError, column);
                continue;
            }
            at(position, j) += args.colValues[k];
        }
    }
    __syncthreads();
    for (int q = 0; q < x.sourceCount; ++q)
    {
        const FrontSource source = x.sources[q];
        for (int jc = warp; jc < source.order; jc += warps)
        {
            const int pj = source.positions[jc];
            const double* column = source.values + static_cast<std::int64_t>(jc) * source.order;
            for (int ic = jc + lane; ic < source.order; ic += 32)
            {
                const int pi = source.positions[ic];
                if (pi >= pj)
                    at(pi, pj) += column[ic];
                else
                    at(pj, pi) += column[ic];
            }
        }
        __syncthreads();
    }
}

__global__ void exactFront(FactorArgs args, ExactFront x, double* work, std::int32_t* perm, double* sub,
                           std::int32_t* eliminated, std::int32_t* structureError)
{
    __shared__ double scratchValue[32];
    __shared__ int scratchIndex[32];
    const int order = x.order;
    const int candidates = x.candidates;
    const std::int64_t ld = order;
    const int tid = threadIdx.x;
    const auto at = [&](int i, int j) -> double& { return work[i + static_cast<std::int64_t>(j) * ld]; };
    assembleWholeFront(args, x, at, structureError);
    const int done = bunchKaufman(GlobalAt{work, ld}, order, candidates, perm, sub, scratchValue, scratchIndex);
    if (tid == 0)
        *eliminated = done;
    for (std::int64_t e = tid; e < static_cast<std::int64_t>(order) * candidates; e += blockDim.x)
    {
        const std::int64_t j = e / order;
        const std::int64_t i = e - j * order;
        x.panel[e] = i >= j ? at(static_cast<int>(i), static_cast<int>(j)) : 0.0;
    }
}

// The trailing front of a partial factorisation (the reference's PartialFactor: the front of the trailing supernode,
// assembled from the matrix's boundary entries and its children's update matrices, is K* itself): assembled whole
// by one block into `schur` (order x order, column-major), then its upper triangle mirrored from the lower.
__global__ void trailingFront(FactorArgs args, ExactFront x, double* schur, std::int32_t* structureError)
{
    const std::int64_t ld = x.order;
    const auto at = [&](int i, int j) -> double& { return schur[i + static_cast<std::int64_t>(j) * ld]; };
    assembleWholeFront(args, x, at, structureError);
    for (std::int64_t e = threadIdx.x; e < ld * ld; e += blockDim.x)
    {
        const std::int64_t j = e / ld;
        const std::int64_t i = e - j * ld;
        if (i < j)
            schur[e] = schur[j + i * ld];
    }
}

// The update matrix an exact front leaves to its parent: the lower triangle of work's trailing block from position
// `from` (count x count, column-major) into `update`.
__global__ void copyTrailing(const double* work, std::int64_t ld, int from, int count, double* update)
{
    const std::int64_t e = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= static_cast<std::int64_t>(count) * count)
        return;
    const std::int64_t j = e / count;
    const std::int64_t i = e - j * count;
    if (i >= j)
        update[e] = work[(from + i) + (from + j) * ld];
}

// ------------------------------------------------------------------------------------------------------------------
// Inertia of D with 2x2 blocks (MultifrontalDriver.cpp:763-790): a 2x2 block by the sign of its determinant (negative:
// one of each; positive: two of the sign of its first term; zero: one zero and one of the sign of its trace), a 1x1
// pivot by its sign. counters: [positive, negative, zero, 2x2 blocks].
// ------------------------------------------------------------------------------------------------------------------
__global__ void inertiaPivoted(FactorArgs args, PivotArgs pivots, const std::int32_t* supernodeOfColumn, int dimension,
                               unsigned long long* counters)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= dimension)
        return;
    const FrontDesc f = args.fronts[supernodeOfColumn[j]];
    const int k = j - f.first;
    const std::int64_t n = f.c + f.r;
    const double* panel = args.panels + f.panel;
    if (k > 0 && pivots.subdiagonal[j - 1] != 0.0)
        return; // the second column of a 2x2 block
    const double pivot = panel[k + k * n];
    if (k + 1 < f.c && pivots.subdiagonal[j] != 0.0)
    {
        const double second = panel[(k + 1) + (k + 1) * n];
        const double e = pivots.subdiagonal[j];
        const double determinant = pivot * second - e * e;
        if (determinant < 0.0)
        {
            atomicAdd(counters + 0, 1ull);
            atomicAdd(counters + 1, 1ull);
        }
        else if (determinant > 0.0)
            atomicAdd(counters + (pivot > 0.0 ? 0 : 1), 2ull);
        else
        {
            atomicAdd(counters + 2, 1ull);
            const double trace = pivot + second;
            atomicAdd(counters + (trace > 0.0 ? 0 : trace < 0.0 ? 1 : 2), 1ull);
        }
        atomicAdd(counters + 3, 1ull);
        return;
    }
    atomicAdd(counters + (pivot > 0.0 ? 0 : pivot < 0.0 ? 1 : 2), 1ull);
}

// ------------------------------------------------------------------------------------------------------------------
// The solves in pivot order.
// ------------------------------------------------------------------------------------------------------------------
// inverse[perm[j]] = j.
__global__ void invertPermutation(const std::int32_t* perm, std::int32_t* inverse, int dimension)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < dimension)
        inverse[perm[j]] = j;
}

// The maps of rows in pivot order: each row of R(s) as its pivot position, each row's position in the parent's front
// with the parent's columns in their pivot order. One block per supernode.
__global__ void remapPivotOrder(const FrontDesc* fronts, const std::int32_t* rows, const std::int32_t* relpos,
                                const std::int32_t* inverse, std::int32_t* rowsPivot, std::int32_t* relposPivot,
                                int supernodes)
{
    const int s = blockIdx.x;
    if (s >= supernodes)
        return;
    const FrontDesc f = fronts[s];
    const FrontDesc* parent = f.parent >= 0 ? fronts + f.parent : nullptr;
    for (int k = threadIdx.x; k < f.r; k += blockDim.x)
    {
        const std::int64_t at = f.rowStart + k;
        rowsPivot[at] = inverse[rows[at]];
        if (parent != nullptr)
        {
            const int position = relpos[at];
            relposPivot[at] = position < parent->c ? inverse[parent->first + position] - parent->first : position;
        }
    }
}

// Column-major B (ld) -> rows of X in pivot order: X[j] = scale[q] B[q], q = perm[j].
__global__ void toRowsPivoted(const double* b, std::int64_t ld, int c0, int width, int dimension, double* x,
                              const std::int32_t* perm, const double* scale)
{
    const std::int64_t e = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= static_cast<std::int64_t>(dimension) * width)
        return;
    const int col = static_cast<int>(e / dimension);
    const int j = static_cast<int>(e - static_cast<std::int64_t>(col) * dimension);
    const int q = perm[j];
    const double s = scale != nullptr ? scale[q] : 1.0;
    x[static_cast<std::int64_t>(j) * width + col] = b[static_cast<std::int64_t>(c0 + col) * ld + q] * s;
}

// Rows of X in pivot order -> column-major B: B[q] = scale[q] X[j] + 0, q = perm[j].
__global__ void fromRowsPivoted(const double* x, int c0, int width, int dimension, double* b, std::int64_t ld,
                                const std::int32_t* perm, const double* scale)
{
    const std::int64_t e = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= static_cast<std::int64_t>(dimension) * width)
        return;
    const int col = static_cast<int>(e / dimension);
    const int j = static_cast<int>(e - static_cast<std::int64_t>(col) * dimension);
    const int q = perm[j];
    const double s = scale != nullptr ? scale[q] : 1.0;
    b[static_cast<std::int64_t>(c0 + col) * ld + q] = x[static_cast<std::int64_t>(j) * width + col] * s + 0.0;
}

// The diagonal sweep with 1x1 and 2x2 pivots: x <- D^-1 x (a 2x2 block by the dsytf2 formula, as the reference's
// block-diagonal solve).
__global__ void diagonalSweepPivoted(SolveArgs a, const std::int32_t* supernodeOfColumn, const double* subdiagonal,
                                     int dimension)
{
    const std::int64_t e = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int w = a.width;
    if (e >= static_cast<std::int64_t>(dimension) * w)
        return;
    const int j = static_cast<int>(e / w);
    const int col = static_cast<int>(e - static_cast<std::int64_t>(j) * w);
    const FrontDesc f = a.fronts[supernodeOfColumn[j]];
    const int k = j - f.first;
    const std::int64_t n = f.c + f.r;
    const double* panel = a.panels + f.panel;
    if (k > 0 && subdiagonal[j - 1] != 0.0)
        return; // solved with its block's first column
    double* x = a.x + static_cast<std::int64_t>(j) * w + col;
    if (k + 1 < f.c && subdiagonal[j] != 0.0)
    {
        const TwoByTwoInverse inverse =
            invertTwoByTwo(panel[k + k * n], subdiagonal[j], panel[(k + 1) + (k + 1) * n]);
        const double r0 = x[0];
        const double r1 = x[w];
        x[0] = __dmul_rn(inverse.s, __dsub_rn(__dmul_rn(inverse.d11, r0), r1));
        x[w] = __dmul_rn(inverse.s, __dsub_rn(__dmul_rn(inverse.d22, r1), r0));
        return;
    }
    x[0] = x[0] / panel[k + k * n];
}

} // namespace oosgpu::device
