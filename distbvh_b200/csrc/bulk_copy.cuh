// bulk_copy.cuh — one-dimensional TMA bulk copies (global -> shared) completing on shared-memory mbarriers, and
// the bounded waits on them. Both addresses of a copy are 16-byte aligned and its size is a multiple of 16.
#pragma once

#include <cstdint>

namespace bvhg {

// Shared-memory address of a pointer into shared memory (PTX operand form).
__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
  return static_cast< uint32_t >( __cvta_generic_to_shared( p ) );
}

// 16 bytes global -> shared without a register round trip (cached in L1 as well); both addresses 16-byte aligned.
__device__ __forceinline__ void cp_async16(void *dst, const void *src)
{
  asm volatile( "cp.async.ca.shared.global [%0], [%1], 16;" ::"r"( smem_addr( dst ) ), "l"( src ) : "memory" );
}

// 4 or 8 bytes global -> shared without a register round trip; both addresses aligned to the size.
template< int BYTES >
__device__ __forceinline__ void cp_async_small(void *dst, const void *src)
{
  static_assert( BYTES == 4 || BYTES == 8, "cp.async.ca copies 4, 8 or 16 bytes" );
  asm volatile( "cp.async.ca.shared.global [%0], [%1], %2;" ::"r"( smem_addr( dst ) ), "l"( src ), "n"( BYTES ) : "memory" );
}

// Waits for all of this thread's cp_async16 / cp_async_small copies (a __syncwarp / __syncthreads then publishes them to the others).
__device__ __forceinline__ void cp_async_wait_all()
{
  asm volatile( "cp.async.wait_all;" ::: "memory" );
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
  asm volatile( "mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"( smem_addr( bar ) ), "r"( count ) : "memory" );
}

// Makes the barrier initialisation visible to the async proxy (before the first copy that completes on it).
__device__ __forceinline__ void mbar_init_fence()
{
  asm volatile( "fence.mbarrier_init.release.cluster;" ::: "memory" );
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
  asm volatile( "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"( smem_addr( bar ) ), "r"( bytes )
                : "memory" );
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t phase)
{
  uint32_t ok;
  asm volatile( "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                : "=r"( ok )
                : "r"( smem_addr( bar ) ), "r"( phase )
                : "memory" );
  return ok != 0;
}

// Polls the barrier for the given phase at most `limit` times; true when the phase completed.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t phase, uint32_t limit)
{
  for ( uint32_t k = 0; k <= limit; ++k )
    if ( mbar_try_wait( bar, phase ) ) return true;
  return false;
}

// Orders this thread's earlier generic-proxy accesses to shared memory before later async-proxy writes (a buffer
// that was read is refilled by a bulk copy).
__device__ __forceinline__ void fence_proxy_async_smem()
{
  asm volatile( "fence.proxy.async.shared::cta;" ::: "memory" );
}

// One-dimensional bulk copy global -> shared (TMA), completing on an mbarrier.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
  asm volatile( "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                  smem_addr( dst ) ),
                "l"( src ), "r"( bytes ), "r"( smem_addr( bar ) )
                : "memory" );
}

}  // namespace bvhg
