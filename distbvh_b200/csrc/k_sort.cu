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
#include "bulk_copy.cuh"
#include "bvhg_internal.cuh"

#include <atomic>

namespace bvhg {
int device_sm_count();
namespace {

constexpr uint32_t kFlagAggregate = 1u << 30;
constexpr uint32_t kFlagPrefix = 2u << 30;
constexpr uint32_t kValueMask = ( 1u << 30 ) - 1;
constexpr int kWarps = kSortThreads / 32;
constexpr int kLookback = 8;  // predecessor status words fetched per look-back step

// Exclusive scan of one value per thread over the block.
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

// Persistent radix pass. A block keeps taking tiles from the pass's tile counter; while it ranks, resolves and
// writes one tile, the next one is already streaming into the other half of its double-buffered shared memory
// (TMA bulk copies on an mbarrier). Per tile: keys and indices to registers, stable warp-level ranking (the lanes
// holding one digit meet by match; their leader takes the group's slots with one shared-memory atomic, which
// retire in program order within the warp, and hands the base back by shuffle), per-digit tile counts published
// for the decoupled look-back, the tile reordered in the shared buffer it came from, contiguous digit runs
// written out. Every wait is bounded (look-back polls and mbarrier waits); on a timeout the block raises the
// object's error word and stops, and blocks that may have read a garbage prefix write only inside the output.
template< int BITS >
__device__ void onesweep_body(const sort_pass_args &a, uint32_t, uint32_t)
{
  const uint64_t *__restrict__ keys_in = a.keys_in;
  const uint32_t *__restrict__ vals_in = a.vals_in;
  uint64_t *__restrict__ keys_out = a.keys_out;
  uint32_t *__restrict__ vals_out = a.vals_out;
  const uint64_t n64 = a.n;
  const int pass = a.pass;
  const uint32_t *__restrict__ hist = a.hist;
  uint32_t *status = a.status;
  obj_scalars *sc = a.sc;
  const uint32_t spin_limit = a.spin_limit;
  const int stall = a.stall;
  const int use_tma = a.use_tma;
  constexpr int RADIX = 1 << BITS;
  constexpr uint32_t MASK = RADIX - 1;
  extern __shared__ __align__( 128 ) unsigned char s_raw[];  // 2 stages of [kSortTile keys][kSortTile indices]
  __shared__ __align__( 8 ) uint64_t s_mbar[2];
  __shared__ uint32_t s_whist[kWarps / 2][RADIX];  // warp 2p: low 16 bits, warp 2p + 1: high 16 bits
  __shared__ uint32_t s_gbase[RADIX];
  __shared__ uint32_t s_lstart[RADIX];
  __shared__ uint32_t s_scan[kWarps];
  __shared__ int s_next, s_err;

  const uint32_t n = static_cast< uint32_t >( n64 );  // n < 2^30
  const uint32_t tiles = ( n + kSortTile - 1 ) / kSortTile;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int shift = pass * BITS;
  // digits never straddle the two 32-bit halves of a key (BITS divides 32)
  const bool high = shift >= 32;
  const int sh = shift & 31;
  auto digit = [&](uint64_t key) -> uint32_t {
    const uint32_t w = high ? static_cast< uint32_t >( key >> 32 ) : static_cast< uint32_t >( key );
    return ( w >> sh ) & MASK;
  };
  auto stage_keys = [&](int st) { return reinterpret_cast< uint64_t * >( s_raw + st * kSortTile * 12 ); };
  auto stage_vals = [&](int st) { return reinterpret_cast< uint32_t * >( s_raw + st * kSortTile * 12 + kSortTile * 8 ); };

  // global exclusive offsets of the digits (the same for every tile of the pass)
  const uint32_t gexcl = block_exclusive_scan( ( tid < RADIX ) ? hist[tid] : 0u, s_scan );
  if ( tid == 0 )
  {
    mbar_init( &s_mbar[0], 1 );
    mbar_init( &s_mbar[1], 1 );
    mbar_init_fence();
    s_next = static_cast< int >( atomicAdd( &sc->sort_tile_counter[pass], 1u ) );
    s_err = 0;
  }
  for ( int q = tid; q < ( kWarps / 2 ) * RADIX; q += kSortThreads ) ( &s_whist[0][0] )[q] = 0;
  __syncthreads();
  uint32_t tile = static_cast< uint32_t >( s_next );
  // a tile goes through the bulk copy when it is full and the arrays are 16-byte aligned
  auto tma_tile = [&](uint32_t t) { return use_tma && ( t + 1 ) * kSortTile <= n; };
  auto issue = [&](uint32_t t, int st) {
    const uint32_t bytes = kSortTile * 8 + ( vals_in ? kSortTile * 4 : 0 );
    mbar_expect_tx( &s_mbar[st], bytes );
    bulk_load( stage_keys( st ), keys_in + static_cast< size_t >( t ) * kSortTile, kSortTile * 8, &s_mbar[st] );
    if ( vals_in )
      bulk_load( stage_vals( st ), vals_in + static_cast< size_t >( t ) * kSortTile, kSortTile * 4, &s_mbar[st] );
  };
  if ( tid == 0 && tile < tiles && tma_tile( tile ) ) issue( tile, 0 );
  uint32_t phases = 0u;  // bit s: parity of stage s's mbarrier phase to wait for
  int st = 0;
  const unsigned lt_mask = ( 1u << lane ) - 1u;

  while ( tile < tiles )
  {
    const uint32_t tile_base = tile * kSortTile;
    const uint32_t cnt = min( static_cast< uint32_t >( kSortTile ), n - tile_base );
    const bool bulk = tma_tile( tile );
    uint64_t *sk = stage_keys( st );
    uint32_t *sv = stage_vals( st );
    if ( bulk )
    {
      uint32_t spins = 0;
      bool ok = true;
      const uint32_t ph = ( phases >> st ) & 1u;
      while ( !mbar_try_wait( &s_mbar[st], ph ) )
        if ( ++spins > spin_limit )
        {
          ok = false;
          break;
        }
      phases ^= 1u << st;
      if ( __syncthreads_or( !ok ) )
      {
        // the copy did not complete in time: give it one more bounded wait, raise the error and stop
        if ( tid == 0 )
        {
          for ( uint32_t k = 0; k < spin_limit && !mbar_try_wait( &s_mbar[st], ph ); ++k ) {}
          atomicCAS( &sc->error, 0, kErrTimeout );
        }
        return;
      }
    }
    // keys and indices of the tile to registers, warp-striped (item j of lane l: local 512 w + 32 j + l)
    uint64_t k[kSortItems];
    uint32_t v[kSortItems];
    uint32_t rk[kSortItems / 2];
    const uint32_t wl = static_cast< uint32_t >( warp ) * ( kSortItems * 32 );
#pragma unroll
    for ( int j = 0; j < kSortItems; ++j )
    {
      const uint32_t li = wl + j * 32 + lane;
      const bool valid = li < cnt;
      if ( bulk )
      {
        k[j] = sk[li];
        v[j] = vals_in ? sv[li] : tile_base + li;
      } else {
        k[j] = valid ? keys_in[tile_base + li] : 0ull;
        v[j] = valid ? ( vals_in ? vals_in[tile_base + li] : tile_base + li ) : 0u;
      }
    }
    const int wrow = warp >> 1, wsh = ( warp & 1 ) * 16;  // s_whist is zero here (cleared before the first tile
                                                         // and during the previous tile's write-out)
#pragma unroll
    for ( int j = 0; j < kSortItems; ++j )
    {
      const bool valid = ( wl + j * 32 + lane ) < cnt;
      const uint32_t d = valid ? digit( k[j] ) : RADIX;
      const unsigned peers = __match_any_sync( 0xffffffffu, d );
      const int leader = __ffs( peers ) - 1;
      uint32_t base = 0;
      if ( valid && lane == leader )
        base = ( atomicAdd( &s_whist[wrow][d], static_cast< uint32_t >( __popc( peers ) ) << wsh ) >> wsh ) & 0xffffu;
      base = __shfl_sync( 0xffffffffu, base, leader );
      const uint32_t rank = base + static_cast< uint32_t >( __popc( peers & lt_mask ) );
      if ( j & 1 ) rk[j >> 1] |= rank << 16;
      else rk[j >> 1] = rank;
    }
    __syncthreads();

    // per digit: exclusive prefix over warps (in place) and the tile total, published for the look-back
    uint32_t total = 0;
    if ( tid < RADIX )
    {
#pragma unroll
      for ( int w = 0; w < kWarps / 2; ++w )
      {
        const uint32_t c = s_whist[w][tid];
        const uint32_t lo = total;
        total += c & 0xffffu;
        s_whist[w][tid] = lo | ( total << 16 );
        total += c >> 16;
      }
      reinterpret_cast< volatile uint32_t * >( status )[static_cast< size_t >( tile ) * RADIX + tid] =
        ( tile == 0 ? kFlagPrefix : kFlagAggregate ) | total;
    }
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
          while ( ( vs[static_cast< size_t >( tiles ) * RADIX + tid] & ~kValueMask ) == 0 )
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
          // a window of kLookback predecessors per step, fetched together and consumed nearest first
          int p = static_cast< int >( tile ) - 1;
          bool done = false;
          while ( !done )
          {
            uint32_t w[kLookback];
#pragma unroll
            for ( int q = 0; q < kLookback; ++q )
              w[q] = ( p - q >= 0 ) ? vs[static_cast< size_t >( p - q ) * RADIX + tid] : kFlagPrefix;
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
    __syncthreads();
    // reorder the tile into its own stage buffer (its data now lives in registers)
#pragma unroll
    for ( int j = 0; j < kSortItems; ++j )
    {
      if ( ( wl + j * 32 + lane ) < cnt )
      {
        const uint32_t d = digit( k[j] );
        const uint32_t rank = ( rk[j >> 1] >> ( ( j & 1 ) * 16 ) ) & 0xffffu;
        const uint32_t pos = s_lstart[d] + ( ( s_whist[wrow][d] >> wsh ) & 0xffffu ) + rank;
        sk[pos] = k[j];
        sv[pos] = v[j];
      }
    }
    __syncthreads();
    // While the tile is written out, thread 0 claims the next tile, reads the error word and starts the next copy
    // into the other stage (drained by the previous iteration's write-out). Claiming here, not before the reorder,
    // keeps a claimed tile's wait for its block short: every successor's look-back waits for that tile's counts.
    // A block that timed out published a garbage prefix (so that no successor waits forever) and raised the
    // object's error word. A block that sees the error stops after this tile (no copy is then in flight); a block
    // that read a garbage prefix writes only inside [0, n) (the bound on every output position below), and the
    // host reports the error for the whole sort.
    if ( tid == 0 )
    {
      const uint32_t nx = atomicAdd( &sc->sort_tile_counter[pass], 1u );
      const bool err = *reinterpret_cast< volatile int * >( &sc->error ) == kErrTimeout;
      s_next = static_cast< int >( nx );
      s_err = err;
      if ( !err && nx < tiles && tma_tile( nx ) )
      {
        fence_proxy_async_smem();
        issue( nx, st ^ 1 );
      }
    }
    // the warp histograms were last read by the reorder above: clear them for the next tile
    for ( int q = tid; q < ( kWarps / 2 ) * RADIX; q += kSortThreads ) ( &s_whist[0][0] )[q] = 0;
    for ( uint32_t i = tid; i < cnt; i += kSortThreads )
    {
      const uint64_t key = sk[i];
      const uint32_t gp = s_gbase[digit( key )] + i;
      if ( gp < n )
      {
        keys_out[gp] = key;
        vals_out[gp] = sv[i];
      }
    }
    __syncthreads();  // the stage is drained: the next iteration may refill it
    if ( s_err ) return;
    st ^= 1;
    tile = static_cast< uint32_t >( s_next );
  }
}

// The attribute is per device and per kernel: set it once for each device this process launches on.
template< int BITS >
cudaError_t onesweep_setup()
{
  static std::atomic< unsigned long long > configured{ 0 };
  int dev = 0;
  cudaError_t e = cudaGetDevice( &dev );
  if ( e != cudaSuccess ) return e;
  const unsigned long long bit = 1ull << ( dev & 63 );
  if ( configured.load() & bit ) return cudaSuccess;
  const int smem = static_cast< int >( 2 * kSortTile * ( sizeof( uint64_t ) + sizeof( uint32_t ) ) );
  e = cudaFuncSetAttribute( k_single< sort_pass_args, onesweep_body< BITS >, kSortThreads, 2 >,
                            cudaFuncAttributeMaxDynamicSharedMemorySize, smem );
  if ( e != cudaSuccess ) return e;
  e = cudaFuncSetAttribute( k_batched< sort_pass_args, onesweep_body< BITS >, kSortThreads, 2 >,
                            cudaFuncAttributeMaxDynamicSharedMemorySize, smem );
  if ( e != cudaSuccess ) return e;
  configured.fetch_or( bit );
  return cudaSuccess;
}

constexpr size_t kOnesweepSmem = static_cast< size_t >( 2 ) * kSortTile * ( sizeof( uint64_t ) + sizeof( uint32_t ) );

// persistent: two blocks per SM (shared memory for two 48 KB stages each), never more blocks than tiles
uint32_t os_grid(uint64_t n)
{
  const uint64_t tiles = ( n + kSortTile - 1 ) / kSortTile;
  const uint64_t cap = static_cast< uint64_t >( device_sm_count() ) * 2;
  return static_cast< uint32_t >( tiles < cap ? tiles : cap );
}

template< int BITS >
cudaError_t launch_os_t(const sort_pass_args &a, cudaStream_t s)
{
  cudaError_t e = onesweep_setup< BITS >();
  if ( e != cudaSuccess ) return e;
  k_single< sort_pass_args, onesweep_body< BITS >, kSortThreads, 2 ><<< os_grid( a.n ), kSortThreads, kOnesweepSmem, s >>>( a );
  return cudaGetLastError();
}

template< int BITS >
cudaError_t launch_os_batch_t(const batch_launch &b, cudaStream_t s)
{
  cudaError_t e = onesweep_setup< BITS >();
  if ( e != cudaSuccess ) return e;
  k_batched< sort_pass_args, onesweep_body< BITS >, kSortThreads, 2 ><<< b.blocks, kSortThreads, kOnesweepSmem, s >>>(
    static_cast< const sort_pass_args * >( b.items ), b.starts, b.nitems );
  return cudaGetLastError();
}

// Low-half fix-up after the radix passes over the high key half (bits 32..62). Those passes leave the keys stably
// ordered by their high 32 bits: every run of equal high halves is in original-index order. Placing each element
// of a run at the run's start plus its rank by (full key, position) -- a stable sort of the run by the low half --
// then gives the stable order of the full keys. One thread per element, out of place (in -> out), so that no
// thread reads what another writes. Runs are found by scanning neighbours (cache hits: a warp reads contiguous
// keys). A run longer than kFixRun is listed and sorted from `in` to `out` by runs_body (sort_run_block); no thread
// of the fix-up writes its elements.
constexpr int kFixRun = 32;
constexpr int kFixThreads = 512;
constexpr int kFixWarps = kFixThreads / 32;
constexpr int kRunSmem = 2048;

// Stable sort by the low key half of the run [s, s + L) of equal high halves, by one block of kFixThreads threads,
// from (src keys, src vals) into (dst keys, dst vals). Up to kRunSmem elements: a bitonic network in shared memory
// over the distinct composite keys (low half << 32 | position in the run), whose order is the stable order. Longer:
// the run is copied to dst, then four stable 8-bit LSD passes over the low half ping-pong between dst and src (src
// is scratch then: nothing reads it after the radix passes but this block, and the high halves every neighbour
// scan compares stay in place), ending in dst; per pass, 512 elements at a time are ranked by warp match in
// element order and placed at the digit's running offset.
__device__ void sort_run_block(uint64_t *__restrict__ skeys, uint32_t *__restrict__ svals, uint64_t *__restrict__ dkeys,
                               uint32_t *__restrict__ dvals, uint32_t s, uint32_t L, unsigned char *s_raw,
                               uint32_t *s_scan)
{
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const unsigned lt_mask = ( 1u << lane ) - 1u;
  const uint64_t hi_bits = skeys[s] & 0xffffffff00000000ull;
  if ( L <= kRunSmem )
  {
    uint64_t *c = reinterpret_cast< uint64_t * >( s_raw );
    uint32_t *v = reinterpret_cast< uint32_t * >( s_raw + kRunSmem * 8 );
    uint32_t P = 1;
    while ( P < L ) P <<= 1;
    for ( uint32_t j = tid; j < P; j += kFixThreads )
    {
      if ( j < L )
      {
        c[j] = ( ( skeys[s + j] & 0xffffffffull ) << 32 ) | j;
        v[j] = svals[s + j];
      } else {
        c[j] = ~0ull;
      }
    }
    __syncthreads();
    for ( uint32_t k = 2; k <= P; k <<= 1 )
      for ( uint32_t j = k >> 1; j > 0; j >>= 1 )
      {
        for ( uint32_t t = tid; t < P; t += kFixThreads )
        {
          const uint32_t u = t ^ j;
          if ( u > t )
          {
            const uint64_t a = c[t], b = c[u];
            if ( ( a > b ) == ( ( t & k ) == 0 ) )
            {
              c[t] = b;
              c[u] = a;
            }
          }
        }
        __syncthreads();
      }
    for ( uint32_t j = tid; j < L; j += kFixThreads )
    {
      const uint64_t x = c[j];
      dkeys[s + j] = hi_bits | ( x >> 32 );
      dvals[s + j] = v[x & 0xffffffffull];
    }
    __syncthreads();
    return;
  }
  uint32_t( *cnt )[256] = reinterpret_cast< uint32_t( * )[256] >( s_raw );  // [kFixWarps][256]
  uint32_t *run_off = reinterpret_cast< uint32_t * >( s_raw + kFixWarps * 256 * 4 );
  uint32_t *tot = run_off + 256;
  uint32_t( *hist )[256] = reinterpret_cast< uint32_t( * )[256] >( tot + 256 );  // [4][256]
  for ( int q = tid; q < kFixWarps * 256; q += kFixThreads ) ( &cnt[0][0] )[q] = 0;
  for ( int q = tid; q < 4 * 256; q += kFixThreads ) ( &hist[0][0] )[q] = 0;
  for ( uint32_t j = tid; j < L; j += kFixThreads )
  {
    dkeys[s + j] = skeys[s + j];
    dvals[s + j] = svals[s + j];
  }
  __syncthreads();
  for ( uint32_t j = tid; j < L; j += kFixThreads )
  {
    const uint32_t low = static_cast< uint32_t >( dkeys[s + j] );
#pragma unroll
    for ( int p = 0; p < 4; ++p ) atomicAdd( &hist[p][( low >> ( 8 * p ) ) & 255u], 1u );
  }
  __syncthreads();
  uint64_t *sk = dkeys, *dk = skeys;
  uint32_t *sv = dvals, *dv = svals;
  for ( int p = 0; p < 4; ++p )
  {
    const uint32_t x = tid < 256 ? hist[p][tid] : 0u;
    const uint32_t ex = block_exclusive_scan( x, s_scan );
    if ( tid < 256 ) run_off[tid] = ex;
    __syncthreads();
    for ( uint32_t base = 0; base < L; base += kFixThreads )
    {
      const uint32_t j = base + tid;
      const bool valid = j < L;
      const uint64_t key = valid ? sk[s + j] : 0ull;
      const uint32_t val = valid ? sv[s + j] : 0u;
      const uint32_t d = valid ? ( static_cast< uint32_t >( key ) >> ( 8 * p ) ) & 255u : 256u;
      const unsigned peers = __match_any_sync( 0xffffffffu, d );
      const uint32_t rank = __popc( peers & lt_mask );
      if ( valid && lane == __ffs( peers ) - 1 ) cnt[warp][d] = __popc( peers );
      __syncthreads();
      if ( tid < 256 )
      {
        uint32_t t = 0;
#pragma unroll
        for ( int w = 0; w < kFixWarps; ++w )
        {
          const uint32_t c = cnt[w][tid];
          cnt[w][tid] = t;
          t += c;
        }
        tot[tid] = t;
      }
      __syncthreads();
      if ( valid )
      {
        const uint32_t pos = run_off[d] + cnt[warp][d] + rank;
        dk[s + pos] = key;
        dv[s + pos] = val;
      }
      __syncthreads();
      if ( tid < 256 )
      {
        run_off[tid] += tot[tid];
#pragma unroll
        for ( int w = 0; w < kFixWarps; ++w ) cnt[w][tid] = 0;
      }
      __syncthreads();
    }
    uint64_t *tk = sk;
    sk = dk;
    dk = tk;
    uint32_t *tv = sv;
    sv = dv;
    dv = tv;
  }
}

// The fix-up proper: one lean thread per element. A run longer than kFixRun is left in place and its first element
// listed (runs[], count in sc->long_runs) for runs_body.
__device__ void fixup_body(const fixup_args &a, uint32_t bid, uint32_t)
{
  const uint64_t *__restrict__ keys_in = a.keys_in;
  const uint32_t *__restrict__ vals_in = a.vals_in;
  uint64_t *__restrict__ keys_out = a.keys_out;
  uint32_t *__restrict__ vals_out = a.vals_out;
  const uint32_t n = static_cast< uint32_t >( a.n );
  const uint32_t i = bid * blockDim.x + threadIdx.x;
  if ( i >= n ) return;
  const uint64_t ki = keys_in[i];
  const uint32_t hi = static_cast< uint32_t >( ki >> 32 );
  uint32_t s = i, e = i;
  bool limit = false;
  while ( s > 0 && static_cast< uint32_t >( __ldg( keys_in + s - 1 ) >> 32 ) == hi )
  {
    --s;
    if ( i - s >= kFixRun )
    {
      limit = true;
      break;
    }
  }
  while ( !limit && e + 1 < n && static_cast< uint32_t >( __ldg( keys_in + e + 1 ) >> 32 ) == hi )
  {
    ++e;
    if ( e - i >= kFixRun )
    {
      limit = true;
      break;
    }
  }
  if ( limit || e - s + 1 > kFixRun )
  {
    // s == i only at the run's first element (the backward scan stops before its limit there); a run has more
    // than kFixRun elements, so at most n / 33 runs are listed
    if ( s == i ) a.runs[atomicAdd( &a.sc->long_runs, 1u )] = i;
    return;
  }
  uint32_t pos = i;
  if ( e > s )
  {
    uint32_t rank = 0;
    for ( uint32_t j = s; j <= e; ++j )
    {
      const uint64_t kj = __ldg( keys_in + j );
      rank += ( kj < ki || ( kj == ki && j < i ) ) ? 1u : 0u;
    }
    pos = s + rank;
  }
  keys_out[pos] = ki;
  vals_out[pos] = vals_in[i];
}

// The long runs the fix-up listed, by a few blocks: block r takes runs r, r + grid, ... (sort_run_block, from the
// pass output into the fix-up output). Exits at once when none was listed.
constexpr uint32_t kRunBlocks = 8;

__device__ void runs_body(const fixup_args &a, uint32_t bid, uint32_t nblk)
{
  __shared__ __align__( 16 ) unsigned char s_raw[kRunSmem * 12];
  __shared__ uint32_t s_scan[kFixWarps];
  __shared__ uint32_t s_start, s_len;
  const uint32_t n = static_cast< uint32_t >( a.n );
  const uint32_t nruns = *reinterpret_cast< const volatile unsigned int * >( &a.sc->long_runs );
  for ( uint32_t r = bid; r < nruns; r += nblk )
  {
    if ( threadIdx.x == 0 )
    {
      const uint32_t s = a.runs[r];
      const uint32_t hi = static_cast< uint32_t >( a.keys_in[s] >> 32 );
      uint32_t lo = s + 1, up = n;  // first index past s whose high half differs
      while ( lo < up )
      {
        const uint32_t mid = lo + ( up - lo ) / 2;
        if ( static_cast< uint32_t >( a.keys_in[mid] >> 32 ) == hi ) lo = mid + 1;
        else up = mid;
      }
      s_start = s;
      s_len = lo - s;
    }
    __syncthreads();
    sort_run_block( const_cast< uint64_t * >( a.keys_in ), const_cast< uint32_t * >( a.vals_in ), a.keys_out,
                    a.vals_out, s_start, s_len, s_raw, s_scan );
    __syncthreads();  // the next run reuses shared memory and the run bounds
  }
}

}  // namespace

uint32_t sort_fixup_blocks(uint64_t n) { return static_cast< uint32_t >( ( n + 255 ) / 256 ); }

uint32_t sort_runs_blocks(uint64_t n)
{
  if ( n <= static_cast< uint64_t >( kFixRun ) ) return 0;  // no run can be long
  const uint64_t most = long_run_capacity( n );
  return static_cast< uint32_t >( most < kRunBlocks ? most : kRunBlocks );
}

cudaError_t launch_sort_fixup(const uint64_t *keys_in, const uint32_t *vals_in, uint64_t *keys_out,
                              uint32_t *vals_out, uint64_t n, uint32_t *runs, obj_scalars *sc, cudaStream_t s)
{
  if ( n == 0 ) return cudaSuccess;
  const fixup_args a{ keys_in, vals_in, keys_out, vals_out, n, runs, sc };
  k_single< fixup_args, fixup_body, 256, 8 ><<< sort_fixup_blocks( n ), 256, 0, s >>>( a );
  if ( const uint32_t rb = sort_runs_blocks( n ) ) k_single< fixup_args, runs_body, kFixThreads, 1 ><<< rb, kFixThreads, 0, s >>>( a );
  return cudaGetLastError();
}

cudaError_t launch_sort_fixup_batch(const batch_launch &b, cudaStream_t s)
{
  if ( !b.nitems ) return cudaSuccess;
  k_batched< fixup_args, fixup_body, 256, 8 ><<< b.blocks, 256, 0, s >>>( static_cast< const fixup_args * >( b.items ),
                                                                        b.starts, b.nitems );
  return cudaGetLastError();
}

cudaError_t launch_sort_runs_batch(const batch_launch &b, cudaStream_t s)
{
  if ( !b.nitems ) return cudaSuccess;
  k_batched< fixup_args, runs_body, kFixThreads, 1 ><<< b.blocks, kFixThreads, 0, s >>>(
    static_cast< const fixup_args * >( b.items ), b.starts, b.nitems );
  return cudaGetLastError();
}

sort_pass_args onesweep_args(int bits, const uint64_t *keys_in, const uint32_t *vals_in, uint64_t *keys_out,
                             uint32_t *vals_out, uint64_t n, int pass, const uint32_t *hist, uint32_t *status,
                             obj_scalars *sc, uint32_t spin_limit, int stall)
{
  const uint64_t radix = 1ull << bits;
  const uint64_t tiles = ( n + kSortTile - 1 ) / kSortTile;
  const int use_tma = ( ( reinterpret_cast< uintptr_t >( keys_in ) | reinterpret_cast< uintptr_t >( vals_in ) ) & 15 ) == 0;
  return sort_pass_args{ keys_in, vals_in, keys_out, vals_out, n, pass, hist + static_cast< size_t >( pass ) * radix,
                         status + static_cast< size_t >( pass ) * ( tiles + 1 ) * radix, sc, spin_limit, stall, use_tma };
}

uint32_t onesweep_blocks(uint64_t n) { return os_grid( n ); }

cudaError_t launch_onesweep(int bits, const uint64_t *keys_in, const uint32_t *vals_in, uint64_t *keys_out,
                            uint32_t *vals_out, uint64_t n, int pass, const uint32_t *hist, uint32_t *status,
                            obj_scalars *sc, uint32_t spin_limit, int stall, cudaStream_t s)
{
  const sort_pass_args a = onesweep_args( bits, keys_in, vals_in, keys_out, vals_out, n, pass, hist, status, sc,
                                          spin_limit, stall );
  switch ( bits )
  {
    case 1: return launch_os_t< 1 >( a, s );
    case 2: return launch_os_t< 2 >( a, s );
    case 4: return launch_os_t< 4 >( a, s );
    case 8: return launch_os_t< 8 >( a, s );
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_onesweep_batch(int bits, const batch_launch &b, cudaStream_t s)
{
  if ( !b.nitems ) return cudaSuccess;
  switch ( bits )
  {
    case 1: return launch_os_batch_t< 1 >( b, s );
    case 2: return launch_os_batch_t< 2 >( b, s );
    case 4: return launch_os_batch_t< 4 >( b, s );
    case 8: return launch_os_batch_t< 8 >( b, s );
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace bvhg
