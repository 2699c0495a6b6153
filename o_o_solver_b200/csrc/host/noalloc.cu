// A solve that allocates no device memory: oosgpu_solve_device_noalloc (include/oos_gpu.h).
//
// Who needs it: a caller that cannot call cudaMalloc once it is running, for instance an application that hands the
// solver a fixed device-memory budget at set-up and forbids allocations afterwards (its own allocator owns the rest of
// the GPU), or a host program that must not let the library grow its device footprint between solves. The ordinary
// solve (oosgpu_solve_device) allocates its scratch on its first call and keeps it with the factor; this one takes
// its scratch from a fixed array that is part of the library image instead.
//
// The scratch: NOALLOC_SCRATCH_VALUES doubles (16 MiB) in the file-scope device array below. Every GPU that loads the
// library holds that array until the process exits. In host code `g_noallocScratch` is only a host-side stand-in for
// the array, not a device address: it is never passed to a kernel. Its device address is taken once per device with
// cudaGetSymbolAddress, with that device current, on the first call of the entry point on that device; that first
// call therefore does this set-up, and should come before any stream capture. Under CUDA's lazy module loading (the
// default), that lookup is also when this file's module, and with it the array, is loaded onto the device, and the
// first solve loads the solve kernels: the first call takes device memory, later calls take none. A call with zero
// columns does the set-up alone. The cached address belongs to the device's primary context: like every factor
// handle, it does not survive a cudaDeviceReset.
//
// Sharing: every call on a device uses the same array and leaves its contents behind; the solve writes every scratch
// value before it reads it (the column tile's rows are copied in; each supernode's update rows are written whole by
// its own forward step before its parent gathers them), so nothing carries over. Two calls whose work overlaps on the GPU (on two streams, or from two
// threads) race on the array: issue them one after the other.
//
// The limit: a factor needs (equations + update rows of its supernodes) scratch values per right-hand side; the
// column tile is narrowed to what the array holds, and a factor that needs more than the whole array for one column is
// refused with OOSGPU_INVALID_ARGUMENT (use oosgpu_solve_device then).

#include "factor_internal.hpp"
#include "host_api.hpp"

#include <cuda_runtime.h>

#include <cstddef>
#include <mutex>
#include <string>

namespace
{

constexpr std::size_t NOALLOC_SCRATCH_VALUES = std::size_t{1} << 21; // 2 Mi doubles = 16 MiB
constexpr int MAX_DEVICES = 64;

__device__ __align__(256) double g_noallocScratch[NOALLOC_SCRATCH_VALUES];

std::mutex g_setupMutex;
double* g_scratchOfDevice[MAX_DEVICES] = {};

// The device address of the scratch on `device`, which is current: looked up on the first call on that device.
double* scratchOn(int device)
{
    if (device < 0 || device >= MAX_DEVICES)
        throw oosgpu::Error(oosgpu::STATUS_INVALID_ARGUMENT,
                            "solve without allocation: device " + std::to_string(device) + " out of range");
    const std::lock_guard<std::mutex> lock(g_setupMutex);
    if (g_scratchOfDevice[device] == nullptr)
    {
        void* address = nullptr;
        const cudaError_t status = cudaGetSymbolAddress(&address, g_noallocScratch);
        if (status != cudaSuccess || address == nullptr)
            throw oosgpu::Error(oosgpu::STATUS_CUDA, std::string("solve without allocation: cudaGetSymbolAddress: ") +
                                                         cudaGetErrorString(status));
        g_scratchOfDevice[device] = static_cast<double*>(address);
    }
    return g_scratchOfDevice[device];
}

} // namespace

extern "C" int oosgpu_solve_device_noalloc(oosgpu_factor* factor, double* b, int64_t ld, int64_t columns)
{
    return oosgpu::runGuarded(
        [&]
        {
            const int device = oosgpu::factorDevice(factor);
            const cudaError_t status = cudaSetDevice(device);
            if (status != cudaSuccess)
                throw oosgpu::Error(oosgpu::STATUS_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(status));
            double* scratch = scratchOn(device);
            oosgpu::solveFactorInScratch(factor, b, ld, columns, scratch, NOALLOC_SCRATCH_VALUES);
        });
}
