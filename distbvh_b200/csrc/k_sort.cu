// k_sort.cu — stable LSD radix sort of (63-bit Morton key, u32 element index) pairs.
//
// Replaces radix_sorter<T, Idx> (src/bvh/util/sort.hpp:75-144), which makes 8*sizeof(T) one-bit passes of
// three kernels each (flag map, exclusive scan, split scatter). A stable sort's output is unique, so any digit
// width yields the reference's permutation; BITS = 1 is the reference's one-bit-per-pass schedule, BITS = 8 the
// fast one. Bit 63 of a morton64 key is always zero (hash.hpp:100-103), so ceil(63 / BITS) passes cover it.
//
// One kernel per pass, onesweep style: all digit histograms come from the key kernel (one read of the keys);
// each block takes a tile of 4096 keys in launch order from an atomic tile counter, ranks them with warp-level
// match (stable within the tile), publishes its per-digit counts, resolves its global offsets by decoupled
// look-back over the preceding tiles' status words, reorders the tile in shared memory and writes contiguous
// digit runs. Every look-back wait is bounded: past spin_limit polls the block records BVHG_ERR_TIMEOUT and
// goes on with a garbage offset (the host reports the error; no thread waits forever).
#include "bvhg_internal.cuh"

#include <atomic>

namespace bvhg {
namespace {

constexpr uint32_t kFlagAggregate = 1u << 30;
constexpr uint32_t kFlagPrefix = 2u << 30;
constexpr uint32_t kValueMask = ( 1u << 30 ) - 1;
constexpr int kWarps = kSortThreads / 32;
constexpr int kLookback = 8;  // predecessor status words fetched per look-back step

// Exclusive scan of one value per thread over a 256-thread block.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t x, uint32_t *s_warp)
{
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t inc = x;
#pragma unroll
  for ( int o = 1; o < 32; o <<= 1 )
  {
    const uint32_t y = __shfl_up_sync( 0xffffffffu, inc, o );
    if ( lane >= o ) inc += y;
  }
  if ( lane == 31 ) s_warp[w] = inc;
  __syncthreads();
  uint32_t wpre = 0;
#pragma unroll
  for ( int k = 0; k < kWarps; ++k )
    if ( k < w ) wpre += s_warp[k];
  __syncthreads();
  return wpre + inc - x;
}

template< int BITS >
__global__ void __launch_bounds__( kSortThreads, 3 ) k_onesweep(const uint64_t *__restrict__ keys_in,
                                                           const uint32_t *__restrict__ vals_in,
                                                           uint64_t *__restrict__ keys_out,
                                                           uint32_t *__restrict__ vals_out, uint64_t n64, int pass,
                                                           const uint32_t *__restrict__ hist, uint32_t *status,
                                                           obj_scalars *sc, uint32_t spin_limit, int stall)
{
  constexpr int RADIX = 1 << BITS;
  constexpr uint32_t MASK = RADIX - 1;
  extern __shared__ uint64_t s_keys[];  // kSortTile keys, then kSortTile vals, then kSortTile digits
  uint32_t *s_vals = reinterpret_cast< uint32_t * >( s_keys + kSortTile );
  uint8_t *s_dig = reinterpret_cast< uint8_t * >( s_vals + kSortTile );
  __shared__ uint32_t s_whist[kWarps][RADIX];
  __shared__ uint32_t s_gbase[RADIX];
  __shared__ uint32_t s_lstart[RADIX];
  __shared__ uint32_t s_scan[kWarps];
  __shared__ int s_tile;

  const uint32_t n = static_cast< uint32_t >( n64 );  // n < 2^30
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int shift = pass * BITS;
  // digits never straddle the two 32-bit halves of a key (BITS divides 32)
  const bool high = shift >= 32;
  const int sh = shift & 31;
  auto digit = [&](uint64_t key) -> uint32_t {
    const uint32_t w = high ? static_cast< uint32_t >( key >> 32 ) : static_cast< uint32_t >( key );
    return ( w >> sh ) & MASK;
  };
  if ( tid == 0 ) s_tile = static_cast< int >( atomicAdd( &sc->sort_tile_counter[pass], 1u ) );
  for ( int k = tid; k < kWarps * RADIX; k += kSortThreads ) ( &s_whist[0][0] )[k] = 0;
  __syncthreads();
  const uint32_t tile = static_cast< uint32_t >( s_tile );
  const uint32_t tile_base = tile * kSortTile;
  const uint32_t wbase = tile_base + static_cast< uint32_t >( warp ) * ( kSortItems * 32 );

  // Keys stay in registers through ranking; values are only loaded at scatter time (fewer live registers,
  // three blocks per SM). Ranks within the warp are < 512 and kept two per register.
  uint64_t k[kSortItems];
  uint32_t rk[kSortItems / 2];
#pragma unroll
  for ( int j = 0; j < kSortItems; ++j )
  {
    const uint32_t idx = wbase + j * 32 + lane;
    k[j] = idx < n ? keys_in[idx] : 0ull;
  }
  // Stable warp-level ranking: the lanes holding one digit meet by match; their leader takes the group's slots
  // with one shared-memory atomic (a warp's atomics on one address retire in program order, so earlier items
  // rank first) and hands the base back by shuffle.
  const unsigned lt_mask = ( 1u << lane ) - 1u;
#pragma unroll
  for ( int j = 0; j < kSortItems; ++j )
  {
    const bool valid = ( wbase + j * 32 + lane ) < n;
    const uint32_t d = valid ? digit( k[j] ) : RADIX;
    const unsigned peers = __match_any_sync( 0xffffffffu, d );
    const int leader = __ffs( peers ) - 1;
    uint32_t base = 0;
    if ( valid && lane == leader ) base = atomicAdd( &s_whist[warp][d], static_cast< uint32_t >( __popc( peers ) ) );
    base = __shfl_sync( 0xffffffffu, base, leader );
    const uint32_t rank = base + static_cast< uint32_t >( __popc( peers & lt_mask ) );
    if ( j & 1 ) rk[j >> 1] |= rank << 16;
    else rk[j >> 1] = rank;
  }
  __syncthreads();

  // Per digit: exclusive prefix over warps (in place) and the tile total.
  uint32_t total = 0;
  if ( tid < RADIX )
  {
#pragma unroll
    for ( int w = 0; w < kWarps; ++w )
    {
      const uint32_t c = s_whist[w][tid];
      s_whist[w][tid] = total;
      total += c;
    }
    volatile uint32_t *st = status + static_cast< size_t >( tile ) * RADIX;
    st[tid] = ( tile == 0 ? kFlagPrefix : kFlagAggregate ) | total;
  }
  const uint32_t g = ( tid < RADIX ) ? hist[tid] : 0u;
  const uint32_t gexcl = block_exclusive_scan( g, s_scan );
  const uint32_t lexcl = block_exclusive_scan( tid < RADIX ? total : 0u, s_scan );

  if ( tid < RADIX )
  {
    uint32_t excl = 0;
    if ( tile > 0 )
    {
      const volatile uint32_t *vs = reinterpret_cast< const volatile uint32_t * >( status );
      uint32_t spins = 0;
      if ( stall )
      {
        // Test hook: poll the spare status row after the last tile, which no block ever publishes.
        while ( ( vs[static_cast< uint64_t >( gridDim.x ) * RADIX + tid] & ~kValueMask ) == 0 )
        {
          if ( ++spins > spin_limit )
          {
            atomicCAS( &sc->error, 0, kErrTimeout );
            __threadfence();
            break;
          }
          __nanosleep( 32 );
        }
      } else {
        // Look back over a window of kLookback predecessors per step: their status words are fetched together
        // (independent loads in flight) and consumed nearest first until an inclusive prefix is found.
        int p = static_cast< int >( tile ) - 1;
        bool done = false;
        while ( !done )
        {
          uint32_t w[kLookback];
#pragma unroll
          for ( int q = 0; q < kLookback; ++q ) w[q] = ( p - q >= 0 ) ? vs[static_cast< size_t >( p - q ) * RADIX + tid] : kFlagPrefix;
          int consumed = 0;
#pragma unroll
          for ( int q = 0; q < kLookback; ++q )
          {
            if ( done || consumed < q ) break;  // stop at the first word that was not ready
            const uint32_t flag = w[q] & ~kValueMask;
            if ( flag == 0 ) break;
            excl += w[q] & kValueMask;
            consumed = q + 1;
            if ( flag == kFlagPrefix ) done = true;
          }
          if ( done ) break;
          p -= consumed;
          if ( consumed == 0 )
          {
            if ( ++spins > spin_limit )
            {
              atomicCAS( &sc->error, 0, kErrTimeout );
              __threadfence();
              break;
            }
            __nanosleep( 32 );
          }
        }
      }
      reinterpret_cast< volatile uint32_t * >( status )[static_cast< size_t >( tile ) * RADIX + tid] =
        kFlagPrefix | ( ( excl + total ) & kValueMask );
    }
    s_gbase[tid] = gexcl + excl - lexcl;
    s_lstart[tid] = lexcl;
  }
  // A block that timed out published a garbage prefix (so that no successor waits forever) and raised the
  // object's error word before doing so; every block that could have read such a prefix sees the word here and
  // writes nothing.
  __shared__ int s_err;
  __syncthreads();
  if ( tid == 0 )
  {
    __threadfence();
    s_err = *reinterpret_cast< volatile int * >( &sc->error ) == kErrTimeout;
  }
  __syncthreads();
  if ( s_err ) return;

#pragma unroll
  for ( int j = 0; j < kSortItems; ++j )
  {
    const uint32_t idx = wbase + j * 32 + lane;
    if ( idx < n )
    {
      const uint32_t d = digit( k[j] );
      const uint32_t rank = ( rk[j >> 1] >> ( ( j & 1 ) * 16 ) ) & 0xffffu;
      const uint32_t pos = s_lstart[d] + s_whist[warp][d] + rank;
      s_keys[pos] = k[j];
      s_dig[pos] = static_cast< uint8_t >( d );
      s_vals[pos] = vals_in ? vals_in[idx] : idx;
    }
  }
  __syncthreads();

  const uint32_t cnt = min( static_cast< uint32_t >( kSortTile ), n - tile_base );
  for ( uint32_t i = tid; i < cnt; i += kSortThreads )
  {
    const uint32_t gp = s_gbase[s_dig[i]] + i;
    if ( gp < n )
    {
      keys_out[gp] = s_keys[i];
      vals_out[gp] = s_vals[i];
    }
  }
}

template< int BITS >
cudaError_t launch_os_t(const uint64_t *keys_in, const uint32_t *vals_in, uint64_t *keys_out, uint32_t *vals_out,
                        uint64_t n, int pass, const uint32_t *hist, uint32_t *status, obj_scalars *sc,
                        uint32_t spin_limit, int stall, cudaStream_t s)
{
  constexpr int RADIX = 1 << BITS;
  const size_t smem = static_cast< size_t >( kSortTile ) * ( sizeof( uint64_t ) + sizeof( uint32_t ) + 1 );
  // The attribute is per device: set it once for each device this process launches on.
  static std::atomic< unsigned long long > configured{ 0 };
  int dev = 0;
  cudaError_t e = cudaGetDevice( &dev );
  if ( e != cudaSuccess ) return e;
  const unsigned long long bit = 1ull << ( dev & 63 );
  if ( !( configured.load() & bit ) )
  {
    e = cudaFuncSetAttribute( k_onesweep< BITS >, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              static_cast< int >( smem ) );
    if ( e != cudaSuccess ) return e;
    configured.fetch_or( bit );
  }
  const uint64_t tiles = ( n + kSortTile - 1 ) / kSortTile;
  k_onesweep< BITS ><<< static_cast< unsigned >( tiles ), kSortThreads, smem, s >>>(
    keys_in, vals_in, keys_out, vals_out, n, pass, hist + static_cast< size_t >( pass ) * RADIX,
    status + static_cast< size_t >( pass ) * ( tiles + 1 ) * RADIX, sc, spin_limit, stall );
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_onesweep(int bits, const uint64_t *keys_in, const uint32_t *vals_in, uint64_t *keys_out,
                            uint32_t *vals_out, uint64_t n, int pass, const uint32_t *hist, uint32_t *status,
                            obj_scalars *sc, uint32_t spin_limit, int stall, cudaStream_t s)
{
  switch ( bits )
  {
    case 1: return launch_os_t< 1 >( keys_in, vals_in, keys_out, vals_out, n, pass, hist, status, sc, spin_limit, stall, s );
    case 2: return launch_os_t< 2 >( keys_in, vals_in, keys_out, vals_out, n, pass, hist, status, sc, spin_limit, stall, s );
    case 4: return launch_os_t< 4 >( keys_in, vals_in, keys_out, vals_out, n, pass, hist, status, sc, spin_limit, stall, s );
    case 8: return launch_os_t< 8 >( keys_in, vals_in, keys_out, vals_out, n, pass, hist, status, sc, spin_limit, stall, s );
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace bvhg
