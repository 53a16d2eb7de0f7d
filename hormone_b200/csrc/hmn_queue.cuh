// hmn_queue.cuh -- how the CTAs of a persistent batch launch share out the
// work list of (simulation, tile) items.
//
// Static: CTA b takes items b, b + grid, b + 2 grid, ... (no shared state).
// Dynamic: CTAs take the next item from a counter in global memory, so a CTA
// that finishes early (an edge tile, a CTA with its SM to itself) takes more.
// The counter pair {next item, CTAs finished} resets itself: the last CTA to
// finish sets both back to zero, after every CTA's last fetch has returned,
// so the next launch on the stream (a CUDA graph replays them in order)
// starts from zero with no memset node.  Nothing waits on another CTA.
//
// Either way every item is processed exactly once by one CTA with the same
// device function, so the order changes which CTA computes a tile and when,
// never the bits it writes.
#pragma once

#include <cuda_runtime.h>

namespace hmn {

// body(item) processes one item and ends with __syncthreads() (the batch
// stage kernels' tile loop body) or returns without touching shared memory.
// The split is a template parameter, so the static loop is exactly the
// plain strided loop (the kernels run at 96 registers or fewer, where an
// extra live value costs spills).
template <bool DYN, class F>
__device__ __forceinline__ void for_each_item(int nitems, int* queue, F&& body) {
  if constexpr (!DYN) {
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) body(it);
  } else {
    __shared__ int next;
    if (threadIdx.x == 0) next = atomicAdd(queue, 1);
    __syncthreads();
    int it = next;
    while (it < nitems) {
      __syncthreads();  // every thread has read `next`
      int ahead = 0;
      if (threadIdx.x == 0) ahead = atomicAdd(queue, 1);  // its latency hides behind the tile
      body(it);
      if (threadIdx.x == 0) next = ahead;
      __syncthreads();
      it = next;
    }
    if (threadIdx.x == 0) {
      __threadfence();
      if (atomicAdd(queue + 1, 1) == (int)gridDim.x - 1) {
        atomicExch(queue, 0);
        atomicExch(queue + 1, 0);
      }
    }
  }
}

}  // namespace hmn
