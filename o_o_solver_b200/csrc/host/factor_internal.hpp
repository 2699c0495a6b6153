// Internal entry points of the factor handle shared between the library's translation units.
#pragma once

#include "oos_gpu.h"

#include <cstddef>
#include <cstdint>
#include <functional>

namespace oosgpu
{

// Runs `body`, turning the library's exceptions into a C-ABI status and the last-error message.
int runGuarded(const std::function<void()>& body);
// The CUDA device a factor handle lives on.
int factorDevice(const oosgpu_factor* factor);
// The device-memory solve of a factor with its scratch in `scratch` (capacity values), allocating nothing.
void solveFactorInScratch(oosgpu_factor* factor, double* b, std::int64_t ld, std::int64_t columns, double* scratch,
                          std::size_t capacity);

} // namespace oosgpu
