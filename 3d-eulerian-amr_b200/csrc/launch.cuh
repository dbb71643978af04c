// Kernel launch with a per-thread tally of launches: every kernel of this
// library goes through launch_k, so the tally counts exactly the kernels this
// thread issued (or recorded into a graph under stream capture).
#pragma once

#include <cuda_runtime.h>

#include <utility>

#include "amr_internal.h"

namespace amr {

template <typename... KArgs, typename... Args>
inline void launch_k(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args&&... args) {
    ++g_launch_tally;
    kernel<<<grid, block, smem, s>>>(std::forward<Args>(args)...);
}

}  // namespace amr
