// batch.cuh — the launches of one kernel for many objects (or scenes) as a single launch.
//
// Each kernel of the pipeline is written as a __device__ body over an argument struct, its block index and its block
// count. The per-object launch runs the body with blockIdx.x and gridDim.x; a batched launch runs the blocks of many
// items back to back: item i owns blocks [starts[i], starts[i + 1]) of the grid, each with the block count the
// per-object launch would have used. A block finds its item by binary search over `starts` and runs the item's body,
// so every item computes exactly what its own launch would have computed; only the number of launches changes.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace bvhg {

// The item owning grid block b: the last i with starts[i] <= b (starts ascending, starts[0] = 0).
__device__ __forceinline__ int batch_item_of(const uint32_t *__restrict__ starts, int n, uint32_t b)
{
  int lo = 0, hi = n - 1;
  while ( lo < hi )
  {
    const int mid = ( lo + hi + 1 ) >> 1;
    if ( __ldg( starts + mid ) <= b ) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// One launch over the blocks of all items: items[i] are item i's arguments.
template< typename Args, void ( *Body )( const Args &, uint32_t, uint32_t ), int THREADS, int MIN_BLOCKS >
__global__ void __launch_bounds__( THREADS, MIN_BLOCKS ) k_batched(const Args *__restrict__ items,
                                                                   const uint32_t *__restrict__ starts, int nitems)
{
  __shared__ int s_item;
  if ( threadIdx.x == 0 ) s_item = batch_item_of( starts, nitems, blockIdx.x );
  __syncthreads();
  const int i = s_item;
  const uint32_t b0 = __ldg( starts + i );
  const Args a = items[i];
  Body( a, blockIdx.x - b0, __ldg( starts + i + 1 ) - b0 );
}

// One per-object launch of a body.
template< typename Args, void ( *Body )( const Args &, uint32_t, uint32_t ), int THREADS, int MIN_BLOCKS >
__global__ void __launch_bounds__( THREADS, MIN_BLOCKS ) k_single(const Args a)
{
  Body( a, blockIdx.x, gridDim.x );
}

// Host side: a batched launch description (item arguments and block starts on the device, built when a batch graph
// is captured).
struct batch_launch
{
  const void *items = nullptr;     // device array of the kernel's argument structs
  const uint32_t *starts = nullptr;  // device array of nitems + 1 block starts
  int nitems = 0;
  uint32_t blocks = 0;             // starts[nitems]
};

}  // namespace bvhg
