// warp.cuh -- sums over the lanes of a thread group inside a warp.
#pragma once

#include <cstdint>

namespace arp {

// Sum of v over the LANES consecutive lanes (LANES a power of two, at most
// 32) that share one item: a butterfly of shuffles, the same order on every
// lane, so the result is deterministic and identical on all of them.
template <int LANES>
__device__ __forceinline__ float group_sum(float v) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t mask = (LANES == 32 ? 0xFFFFFFFFu : ((1u << LANES) - 1u)) << (lane & ~(uint32_t)(LANES - 1));
#pragma unroll
    for (int o = LANES / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o, LANES);
    return v;
}

}  // namespace arp
