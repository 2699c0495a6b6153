// The Schur update of a front's update matrix, U -= L_R D L_R^T (the reference's update of the contribution block,
// DenseKernels::updateSymmetric, src/linalg/dense/DenseKernels.cpp:326, tile subtractProductTile,
// include/oos/linalg/kernels/DenseKernelEntryPoints.hpp:245), FP64 on the tensor cores with its operands brought in by
// the tensor-memory accelerator.
//
// One block of 16 warps per 128 x 128 lower tile of U. The K dimension (the front's c eliminated columns) streams
// through UPDATE_STAGES shared-memory stages of UPDATE_SLICE columns: per stage, one thread issues 16 TMA loads of
// 16 x 16 boxes (the tile's 128 rows of L_R and its 128 columns' rows of L_R, 2 KB each) from the front's tensor map,
// counted on the stage's mbarrier, and 16 threads stage the slice's pivots d_k. Each warp owns a 32 x 32 part of the
// tile: per step of 4 columns, 4 + 4 fragments from shared memory (B scaled by d_k as it is read: W = L D, rounded
// once) and 16 DMMA m8n8k4 products.
//
// Shared-memory layout: a box is 16 rows of 128 bytes (one k column each), stored with the 128-byte swizzle (the
// 16-byte chunk c of row k at chunk c ^ (k mod 8)). A DMMA step's four k-slots are the columns 2t + p (+ 8 q), not
// t: lanes t = 0..3 then read four rows whose XOR patterns spread the fragment over all eight chunks of a row, two
// wavefronts per fragment load, the fewest a 256-byte load can take (the contiguous assignment takes four). The
// products' terms are the same; only the order of the tensor cores' sums changes.
//
// Every wait on an mbarrier is bounded; when one runs out the block records an error, waits (bounded again) for its
// own loads still in flight, and returns, and the host reports it. No load uses cluster multicast; every tensor map
// covers this GPU's own panel arena.

#include "kernels.cuh"
#include "tma.cuh"

#include <cstdint>

namespace oosgpu::device
{

namespace
{

constexpr int UT = UPDATE_TILE;                    // 128
constexpr int BOX = 16;                            // rows (and k columns) of one TMA box
constexpr int BOX_BYTES = BOX * BOX * 8;           // 2 KB
constexpr int OPERAND_BYTES = (UT / BOX) * BOX_BYTES; // 16 KB: one operand's slice
constexpr int STAGE_BYTES = 2 * OPERAND_BYTES;     // 32 KB: A and B

// Byte offset in an operand's slice of row i (0..127) and slice column k (0..15).
__device__ __forceinline__ unsigned swizzled(int i, int k)
{
    const int r = i & (BOX - 1);
    return static_cast<unsigned>((i >> 4) * BOX_BYTES + k * 128 + ((((r >> 1) ^ (k & 7))) << 4) + (r & 1) * 8);
}

__device__ __forceinline__ double sharedLoad(unsigned address)
{
    double v;
    asm volatile("ld.shared.f64 %0, [%1];\n" : "=d"(v) : "r"(address));
    return v;
}

__device__ __forceinline__ void dmma(double (&d)[2], double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

} // namespace

// tasks: the 128 x 128 lower tiles {front, i0, j0, tensor map index}; maps: the fronts' tensor maps (128 bytes each,
// 64-byte aligned), over the panel as rows (contiguous) x columns with 16 x 16 boxes and the 128-byte swizzle; error:
// set to 1 when a wait ran out. Dynamic shared memory: UPDATE_TMA_SMEM bytes.
__global__ void __launch_bounds__(UPDATE_THREADS, 1)
    updateMatrixTma(FactorArgs args, const TileTask* tasks, const void* maps, int* error)
{
    extern __shared__ unsigned char raw[];
    __shared__ std::uint64_t full[UPDATE_STAGES];
    __shared__ double pivots[UPDATE_STAGES][UPDATE_SLICE];
    __shared__ int failed;
    const unsigned base = (sharedAddress(raw) + 1023u) & ~1023u; // the swizzle wants 1024-byte aligned boxes
    const TileTask task = tasks[blockIdx.x];
    const FrontDesc f = args.fronts[task.front];
    const int n = f.c + f.r;
    const void* map = static_cast<const unsigned char*>(maps) + static_cast<std::size_t>(task.k0) * 128;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int wm = (warp >> 2) * 32;
    const int wn = (warp & 3) * 32;
    const int g = lane >> 2;
    const int t = lane & 3;
    const int slices = (f.c + UPDATE_SLICE - 1) / UPDATE_SLICE;
    const double* panel = args.panels + f.panel;
    unsigned lastParity[UPDATE_STAGES] = {};

    if (tid == 0)
    {
        for (int s = 0; s < UPDATE_STAGES; ++s)
            mbarrierInit(&full[s], 1);
        fenceBarrierInit();
        acquireTensorMap(map);
        failed = 0;
    }
    __syncthreads();
    // Slice `slice` into stage `stage`: the loads by thread 0, the pivots by threads 0..15.
    const auto issue = [&](int slice, int stage)
    {
        if (tid == 0)
        {
            const unsigned a = base + static_cast<unsigned>(stage) * STAGE_BYTES;
            fenceProxyAsync(); // the block's reads of this stage (ordered here by the barrier) before the TMA writes
            mbarrierExpectBytes(&full[stage], STAGE_BYTES);
            for (int b = 0; b < UT / BOX; ++b)
            {
                tmaLoad2dShared(a + b * BOX_BYTES, map, f.c + task.i0 + b * BOX, slice * UPDATE_SLICE, &full[stage]);
                tmaLoad2dShared(a + OPERAND_BYTES + b * BOX_BYTES, map, f.c + task.j0 + b * BOX, slice * UPDATE_SLICE,
                                &full[stage]);
            }
            lastParity[stage] = static_cast<unsigned>(slice / UPDATE_STAGES) & 1u;
        }
        if (tid < UPDATE_SLICE)
        {
            const int k = slice * UPDATE_SLICE + tid;
            pivots[stage][tid] = k < f.c ? panel[static_cast<std::int64_t>(k) * (n + 1)] : 0.0;
        }
    };
    for (int s = 0; s < UPDATE_STAGES && s < slices; ++s)
        issue(s, s);
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
    for (int slice = 0; slice < slices; ++slice)
    {
        const int stage = slice % UPDATE_STAGES;
        if (mbarrierWait(&full[stage], static_cast<unsigned>(slice / UPDATE_STAGES) & 1u))
        {
            const unsigned a = base + static_cast<unsigned>(stage) * STAGE_BYTES;
            const unsigned b = a + OPERAND_BYTES;
#pragma unroll
            for (int q = 0; q < 2; ++q)
#pragma unroll
                for (int p = 0; p < 2; ++p)
                {
                    const int kk = 2 * t + p + 8 * q; // this lane's k-slot of the step
                    const double dk = pivots[stage][kk];
                    double fa[4];
                    double fb[4];
#pragma unroll
                    for (int mi = 0; mi < 4; ++mi)
                        fa[mi] = sharedLoad(a + swizzled(wm + mi * 8 + g, kk));
#pragma unroll
                    for (int ni = 0; ni < 4; ++ni)
                        fb[ni] = sharedLoad(b + swizzled(wn + ni * 8 + g, kk)) * dk;
#pragma unroll
                    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                        for (int ni = 0; ni < 4; ++ni)
                            dmma(acc[mi][ni], fa[mi], fb[ni]);
                }
        }
        else
            failed = 1;
        __syncthreads(); // every warp is done with this stage (and has seen `failed`)
        if (failed != 0)
            break;
        if (slice + UPDATE_STAGES < slices)
            issue(slice + UPDATE_STAGES, stage);
    }
    if (failed != 0)
    {
        if (tid == 0)
        {
            atomicExch(error, 1);
            // the loads still in flight land in this block's shared memory: wait for them (bounded) before leaving
            for (int s = 0; s < UPDATE_STAGES && s < slices; ++s)
                mbarrierWait(&full[s], lastParity[s]);
        }
        return;
    }
    double* update = args.updates + f.update;
    const bool diagonalTile = task.i0 == task.j0;
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int h = 0; h < 2; ++h)
            {
                const int ii = task.i0 + wm + mi * 8 + g;
                const int jj = task.j0 + wn + ni * 8 + 2 * t + h;
                if (ii < f.r && jj < f.r && (!diagonalTile || ii >= jj))
                {
                    double* target = update + ii + static_cast<std::int64_t>(jj) * f.r;
                    *target = *target - acc[mi][ni][h];
                }
            }
}

} // namespace oosgpu::device
