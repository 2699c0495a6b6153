// The mixed-precision form of the Schur update (the update matrices of the large fronts): U -= L_R D L_R^T with each
// FP64 operand split into two TF32 parts (x = hi + lo, both rounded to TF32 from x's FP32 value) and the three
// products hi*hi + hi*lo + lo*hi accumulated in FP32 by the fifth-generation tensor cores (tcgen05.mma kind::tf32,
// the accumulator in tensor memory), then subtracted from the FP64 update matrix. About FP32 accuracy: the FP64
// iterative refinement of the solves recovers the rest.
//
// One CTA of eight warps per 128 x 128 tile of an update matrix. The K loop (the front's eliminated columns) runs in
// chunks of 16: every thread loads 8 values of a row of A and of W = L D into registers two chunks ahead, splits them
// and stores them into one of two shared-memory stages in the tensor cores' K-major layout without swizzle (core
// matrices of 8 rows x 16 bytes); one thread issues the chunk's six MMAs and commits them to the stage's mbarrier,
// which the threads wait on before they refill the stage.
// Every wait is bounded: a wait that runs out sets the error flag and the CTA skips its output, frees its tensor
// memory and returns.

#include "kernels.cuh"

#include <cstdint>

namespace oosgpu::device
{

namespace
{

constexpr int MT = 128;                       // tile rows (M) and columns (N)
constexpr int KC = 16;                        // K of one chunk (two MMA k-steps of 8)
constexpr int KSTEP = 8;                      // K of one kind::tf32 MMA
constexpr int OPERAND_BYTES = MT * KC * 4;    // one split part of one operand of one chunk: 8 KB
constexpr int STAGE_BYTES = 4 * OPERAND_BYTES; // A hi, A lo, W hi, W lo
constexpr int KSTEP_BYTES = MT * KSTEP * 4;   // one k-step of one part: 4 KB
constexpr int TMEM_COLUMNS = 128;             // the FP32 accumulator, 128 lanes x 128 columns
// Instruction descriptor of kind::tf32: D F32 (bits 4-5 = 1), A and B TF32 (bits 7-9 = 2, 10-12 = 2), both K-major,
// N >> 3 at bit 17, M >> 4 at bit 24.
constexpr std::uint32_t INSTRUCTION = (1u << 4) | (2u << 7) | (2u << 10) | ((MT >> 3) << 17) | ((MT >> 4) << 24);
constexpr unsigned WAIT_SPINS = 1u << 18;

__device__ __forceinline__ std::uint32_t sharedAddress(const void* p)
{
    return static_cast<std::uint32_t>(__cvta_generic_to_shared(p));
}

// The shared-memory descriptor of a K-major operand without swizzle: start address, the two core matrices along K
// 128 bytes apart (leading byte offset), the 8-row groups 256 bytes apart (stride byte offset), descriptor version 1.
__device__ __forceinline__ std::uint64_t operandDescriptor(std::uint32_t address)
{
    return static_cast<std::uint64_t>((address >> 4) & 0x3FFFu) | (static_cast<std::uint64_t>(128 >> 4) << 16) |
           (static_cast<std::uint64_t>(256 >> 4) << 32) | (1ull << 46);
}

__device__ __forceinline__ void mmaTf32(std::uint32_t tmem, std::uint64_t a, std::uint64_t b, std::uint32_t accumulate)
{
    const std::uint32_t mask[4] = {0, 0, 0, 0}; // no output lane disabled
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
                 "l"(a), "l"(b), "r"(INSTRUCTION), "r"(accumulate), "r"(mask[0]), "r"(mask[1]), "r"(mask[2]),
                 "r"(mask[3]));
}

__device__ __forceinline__ void commitTo(std::uint64_t* barrier)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     sharedAddress(barrier))
                 : "memory");
}

// Waits, at most WAIT_SPINS tries, for the phase of the given parity of an mbarrier to complete.
__device__ __forceinline__ bool waitPhase(std::uint64_t* barrier, std::uint32_t parity)
{
    const std::uint32_t address = sharedAddress(barrier);
    for (unsigned spin = 0; spin < WAIT_SPINS; ++spin)
    {
        std::uint32_t done = 0;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}\n"
                     : "=r"(done)
                     : "r"(address), "r"(parity)
                     : "memory");
        if (done != 0)
            return true;
    }
    return false;
}

__device__ __forceinline__ std::uint32_t toTf32(float x)
{
    std::uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

// x = hi + lo (to about FP32 accuracy): hi the TF32 rounding of x's FP32 value, lo the TF32 rounding of the rest.
__device__ __forceinline__ void splitTf32(double x, std::uint32_t& hi, std::uint32_t& lo)
{
    const float f = static_cast<float>(x);
    hi = toTf32(f);
    lo = toTf32(f - __uint_as_float(hi));
}

// Stores one k-step (8 values) of a row of one operand, split, into a stage's hi and lo parts (K-major, no swizzle).
__device__ __forceinline__ void storeSplitStep(unsigned char* hiPart, unsigned char* loPart, int row, int ks,
                                               const double* v)
{
#pragma unroll
    for (int half = 0; half < 2; ++half)
    {
        std::uint32_t h[4];
        std::uint32_t l[4];
#pragma unroll
        for (int q = 0; q < 4; ++q)
            splitTf32(v[half * 4 + q], h[q], l[q]);
        const int offset = ks * KSTEP_BYTES + (row >> 3) * 256 + half * 128 + (row & 7) * 16;
        *reinterpret_cast<uint4*>(hiPart + offset) = make_uint4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<uint4*>(loPart + offset) = make_uint4(l[0], l[1], l[2], l[3]);
    }
}

} // namespace

// U(i, j) -= sum_{k < c} L(c + i, k) d_k L(c + j, k) for a 128 x 128 tile (i0, j0) of a large front's update matrix
// (lower tiles; a diagonal tile keeps i >= j), 3xTF32 on tcgen05, 256 threads: thread t loads row t % 128 and k-step
// t / 128 of every chunk, two chunks ahead in registers. Dynamic shared memory: MIXED_UPDATE_SMEM bytes.
__global__ void __launch_bounds__(256) updateMatrixMixed(FactorArgs args, const TileTask* tasks, int* error)
{
    extern __shared__ unsigned char dynamicSmem[];
    __shared__ alignas(8) std::uint64_t barriers[2];
    __shared__ std::uint32_t tmemSlot;
    unsigned char* stages = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<std::uintptr_t>(dynamicSmem) + 1023) & ~static_cast<std::uintptr_t>(1023));
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;
    const int row = tid & (MT - 1);
    const int ks = tid >> 7; // the k-step of a chunk this thread loads
    const TileTask task = tasks[blockIdx.x];
    const FrontDesc f = args.fronts[task.front];
    const std::int64_t n = f.c + f.r;
    const double* panel = args.panels + f.panel;
    const double* aRows = panel + f.c + task.i0;
    const double* bRows = panel + f.c + task.j0;
    const int rowsA = min(MT, f.r - task.i0);
    const int rowsB = min(MT, f.r - task.j0);
    const int k = f.c;

    if (tid == 0)
    {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sharedAddress(&barriers[0])) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sharedAddress(&barriers[1])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0)
    {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         sharedAddress(&tmemSlot)),
                     "r"(TMEM_COLUMNS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const std::uint32_t tmem = tmemSlot;

    // Two register sets: chunk q is in set q % 2, loaded two chunks before it is stored.
    double a[2][KSTEP];
    double w[2][KSTEP];
    const auto load = [&](int set, int chunk)
    {
        const int kbase = chunk * KC + ks * KSTEP;
#pragma unroll
        for (int q = 0; q < KSTEP; ++q)
        {
            const int kk = kbase + q;
            const bool inK = kk < k;
            a[set][q] = inK && row < rowsA ? aRows[row + static_cast<std::int64_t>(kk) * n] : 0.0;
            w[set][q] = inK && row < rowsB ? bRows[row + static_cast<std::int64_t>(kk) * n] *
                                                 panel[kk + static_cast<std::int64_t>(kk) * n]
                                           : 0.0;
        }
    };

    const int chunks = (k + KC - 1) / KC;
    bool ok = true;
    int committed = 0; // chunks whose MMAs are committed (the same count in every thread)
    const auto step = [&](int q, int set) -> bool
    {
        const int stage = q & 1;
        unsigned char* base = stages + stage * STAGE_BYTES;
        if (q >= 2)
            ok = waitPhase(&barriers[stage], static_cast<std::uint32_t>(((q >> 1) - 1) & 1));
        if (__syncthreads_and(ok ? 1 : 0) == 0)
        {
            ok = false;
            return false;
        }
        storeSplitStep(base, base + OPERAND_BYTES, row, ks, a[set]);
        storeSplitStep(base + 2 * OPERAND_BYTES, base + 3 * OPERAND_BYTES, row, ks, w[set]);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0)
        {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int s = 0; s < KC / KSTEP; ++s)
            {
                const std::uint32_t at = sharedAddress(base) + s * KSTEP_BYTES;
                const std::uint64_t aHi = operandDescriptor(at);
                const std::uint64_t aLo = operandDescriptor(at + OPERAND_BYTES);
                const std::uint64_t wHi = operandDescriptor(at + 2 * OPERAND_BYTES);
                const std::uint64_t wLo = operandDescriptor(at + 3 * OPERAND_BYTES);
                mmaTf32(tmem, aLo, wHi, q > 0 || s > 0 ? 1u : 0u);
                mmaTf32(tmem, aHi, wLo, 1u);
                mmaTf32(tmem, aHi, wHi, 1u);
            }
            commitTo(&barriers[stage]);
        }
        ++committed;
        return true;
    };

    load(0, 0);
    if (chunks > 1)
        load(1, 1);
    for (int q = 0; q < chunks; q += 2)
    {
        if (!step(q, 0))
            break;
        if (q + 2 < chunks)
            load(0, q + 2);
        if (q + 1 < chunks)
        {
            if (!step(q + 1, 1))
                break;
            if (q + 3 < chunks)
                load(1, q + 3);
        }
    }
    // The last commit covers every MMA issued before it (after a failed wait too, bounded, before the memory goes).
    if (committed > 0)
    {
        const int last = committed - 1;
        const bool done = waitPhase(&barriers[last & 1], static_cast<std::uint32_t>((last >> 1) & 1));
        ok = ok && done;
    }
    const bool allOk = __syncthreads_and(ok ? 1 : 0) != 0;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (allOk)
    {
        // Warp w: the rows of its lane quarter (w % 4), the columns of its half (w / 4).
        const int outRow = (warp & 3) * 32 + lane;
        const int colBase = (warp >> 2) * (MT / 2);
        double* c = args.updates + f.update;
        const std::int64_t ld = f.r;
        const bool diagonal = task.i0 == task.j0;
#pragma unroll 1
        for (int col0 = colBase; col0 < colBase + MT / 2; col0 += 16)
        {
            std::uint32_t v[16];
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
                         "%12, %13, %14, %15}, [%16];"
                         : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                           "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                           "=r"(v[14]), "=r"(v[15])
                         : "r"(tmem + (static_cast<std::uint32_t>((warp & 3) * 32) << 16) +
                               static_cast<std::uint32_t>(col0)));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (outRow < rowsA)
            {
#pragma unroll
                for (int q = 0; q < 16; ++q)
                {
                    const int col = col0 + q;
                    if (col < rowsB && (!diagonal || outRow >= col))
                    {
                        double* target = c + (task.i0 + outRow) + static_cast<std::int64_t>(task.j0 + col) * ld;
                        *target = *target - static_cast<double>(__uint_as_float(v[q]));
                    }
                }
            }
        }
    }
    else if (tid == 0)
    {
        atomicExch(error, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLUMNS)
                     : "memory");
}

} // namespace oosgpu::device
