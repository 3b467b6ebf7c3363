// The action with its projector scratch in a fixed device array (noalloc.cu).
#pragma once

#include "device.cuh"

namespace a43g {

size_t noalloc_capacity();                                      // bytes of the fixed array
size_t noalloc_required(DevicePlan const &dp, size_t real_bytes); // bytes a plan needs
// device address of the fixed array on the current device (looked up once per device)
bool noalloc_scratch_address(void **address);
// y = (H - E S) x with no device allocation; false (error set) if the plan needs more scratch
template <typename T>
bool action_noalloc(DevicePlan &dp, T *y, T const *x, uint16_t const *colIndex, cudaStream_t st);

} // namespace a43g
