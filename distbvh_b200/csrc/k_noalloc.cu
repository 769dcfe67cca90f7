// k_noalloc.cu — a stable radix sort of 64-bit keys that allocates no memory.
//
// Some callers cannot call cudaMalloc: a host that has handed all device memory to its own pool allocator (as
// solid-mechanics codes and frameworks with caching allocators commonly do, so a cudaMalloc beside the pool fails
// or fragments it), a step loop that runs under a fixed device-memory budget, or a library boundary that forbids
// the callee from owning device memory. For them bvhg_radix_sort_noalloc sorts caller-owned device keys into
// caller-owned outputs and takes every byte of scratch (digit histograms, look-back status words, tile counters,
// the ping-pong key/index buffer) from one file-scope static device array of fixed size. The sort itself is the
// library's radix pass kernel (k_sort.cu), unchanged, over all 8 digits of the keys.
//
// The array exists on every GPU that loads this library, for the life of the process. Its device address is
// resolved once per device, on the first call made with that device current (cudaGetSymbolAddress); make that
// first call before any stream capture. The cached address belongs to the CUDA context it was resolved in: after
// cudaDeviceReset on a device, the library must not be called on that device again in the same process. All
// calls share the array and it keeps the last call's contents: each call clears the parts that must start at
// zero, and calls that overlap on the GPU (different streams, or different host threads) race on it. A call waits
// for its stream before it returns (it reads back the sort's error word).
#include "../../include/bvhg.h"
#include "bvhg_internal.cuh"

#include <atomic>
#include <mutex>

namespace bvhg {
namespace {

constexpr uint64_t kNoAllocMaxKeys = 1ull << 20;  // 1,048,576 keys
constexpr int kNoAllocBits = 8;
constexpr int kNoAllocRadix = 1 << kNoAllocBits;
constexpr int kNoAllocPasses = ( kKeyBits + kNoAllocBits - 1 ) / kNoAllocBits;
constexpr uint64_t kNoAllocTiles = ( kNoAllocMaxKeys + kSortTile - 1 ) / kSortTile;

constexpr size_t align256(size_t x) { return ( x + 255 ) & ~size_t( 255 ); }
constexpr size_t kOffHist = align256( sizeof( obj_scalars ) );
constexpr size_t kOffStatus = align256( kOffHist + size_t( kNoAllocPasses ) * kNoAllocRadix * 4 );
constexpr size_t kStatusBytes = size_t( kNoAllocPasses ) * ( kNoAllocTiles + 1 ) * kNoAllocRadix * 4;
constexpr size_t kOffKeys = align256( kOffStatus + kStatusBytes );
constexpr size_t kOffVals = align256( kOffKeys + kNoAllocMaxKeys * 8 );
constexpr size_t kScratchBytes = align256( kOffVals + kNoAllocMaxKeys * 4 );  // about 14 MB

// In host code this name is a stand-in, not a device address: kernels get the address cudaGetSymbolAddress
// returns for the current device.
static __device__ __align__( 256 ) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_addr_mutex;
void *g_addr[64] = {};

// Device address of the scratch array on the current device (resolved once per device).
cudaError_t scratch_address(void **out)
{
  int dev = 0;
  cudaError_t e = cudaGetDevice( &dev );
  if ( e != cudaSuccess ) return e;
  if ( dev < 0 || dev >= 64 ) return cudaErrorInvalidDevice;
  std::lock_guard< std::mutex > lock( g_addr_mutex );
  if ( !g_addr[dev] )
  {
    void *p = nullptr;
    e = cudaGetSymbolAddress( &p, g_noalloc_scratch );
    if ( e != cudaSuccess ) return e;
    g_addr[dev] = p;
  }
  *out = g_addr[dev];
  return cudaSuccess;
}

// Digit histograms of every pass, straight from the keys (warp-uniform digits take one atomic).
__global__ void __launch_bounds__( 256 ) k_hist_keys(const uint64_t *__restrict__ keys, uint64_t n,
                                                   uint32_t *__restrict__ hist)
{
  __shared__ uint32_t s_hist[kNoAllocPasses * kNoAllocRadix];
  for ( int k = threadIdx.x; k < kNoAllocPasses * kNoAllocRadix; k += 256 ) s_hist[k] = 0;
  __syncthreads();
  const unsigned lane = threadIdx.x & 31;
  const uint64_t stride = static_cast< uint64_t >( gridDim.x ) * 256;
  for ( uint64_t w0 = static_cast< uint64_t >( blockIdx.x ) * 256 + ( threadIdx.x & ~31u ); w0 < n; w0 += stride )
  {
    const uint64_t i = w0 + lane;
    const bool valid = i < n;
    const uint64_t key = valid ? keys[i] : 0ull;
    const unsigned vmask = __ballot_sync( 0xffffffffu, valid );
#pragma unroll
    for ( int p = 0; p < kNoAllocPasses; ++p )
    {
      const unsigned d = static_cast< unsigned >( ( key >> ( p * kNoAllocBits ) ) & ( kNoAllocRadix - 1 ) );
      const unsigned d0 = __shfl_sync( 0xffffffffu, d, 0 );
      if ( __all_sync( 0xffffffffu, d == d0 || !valid ) && vmask == 0xffffffffu )
      {
        if ( lane == 0 ) atomicAdd( &s_hist[p * kNoAllocRadix + d0], 32u );
      } else if ( valid ) {
        atomicAdd( &s_hist[p * kNoAllocRadix + d], 1u );
      }
    }
  }
  __syncthreads();
  for ( int k = threadIdx.x; k < kNoAllocPasses * kNoAllocRadix; k += 256 )
    if ( s_hist[k] ) atomicAdd( &hist[k], s_hist[k] );
}

}  // namespace
}  // namespace bvhg

using namespace bvhg;

extern "C" bvhg_status bvhg_radix_sort_noalloc(const uint64_t *keys_in, uint64_t *keys_out, uint32_t *perm_out,
                                               uint64_t n, void *stream)
{
  if ( n > kNoAllocMaxKeys ) return BVHG_ERR_ARG;  // beyond the scratch array's capacity
  if ( n == 0 ) return BVHG_OK;
  if ( !keys_in || !keys_out || !perm_out ) return BVHG_ERR_ARG;
  if ( keys_in == keys_out ) return BVHG_ERR_ARG;
  cudaStream_t s = static_cast< cudaStream_t >( stream );
  void *base = nullptr;
  if ( scratch_address( &base ) != cudaSuccess ) return BVHG_ERR_CUDA;
  unsigned char *b = static_cast< unsigned char * >( base );
  obj_scalars *sc = reinterpret_cast< obj_scalars * >( b );
  uint32_t *hist = reinterpret_cast< uint32_t * >( b + kOffHist );
  uint32_t *status = reinterpret_cast< uint32_t * >( b + kOffStatus );
  uint64_t *tmp_keys = reinterpret_cast< uint64_t * >( b + kOffKeys );
  uint32_t *tmp_vals = reinterpret_cast< uint32_t * >( b + kOffVals );
  const uint64_t tiles = ( n + kSortTile - 1 ) / kSortTile;
  // what must start at zero: tile counters and the error word, the histograms, this size's status words
  if ( cudaMemsetAsync( sc, 0, sizeof( obj_scalars ), s ) != cudaSuccess ) return BVHG_ERR_CUDA;
  if ( cudaMemsetAsync( hist, 0, size_t( kNoAllocPasses ) * kNoAllocRadix * 4, s ) != cudaSuccess ) return BVHG_ERR_CUDA;
  if ( cudaMemsetAsync( status, 0, size_t( kNoAllocPasses ) * ( tiles + 1 ) * kNoAllocRadix * 4, s ) != cudaSuccess )
    return BVHG_ERR_CUDA;
  const uint64_t blocks = ( n + 255 ) / 256;
  k_hist_keys<<< static_cast< unsigned >( blocks < 148 * 8 ? blocks : 148 * 8 ), 256, 0, s >>>( keys_in, n, hist );
  if ( cudaGetLastError() != cudaSuccess ) return BVHG_ERR_CUDA;
  // even passes write the scratch buffer, odd passes the caller's outputs: the last (odd) pass ends there
  static_assert( kNoAllocPasses % 2 == 0, "the final pass must write the caller's outputs" );
  const uint64_t *kin = keys_in;
  const uint32_t *vin = nullptr;
  for ( int p = 0; p < kNoAllocPasses; ++p )
  {
    uint64_t *kout = ( p & 1 ) ? keys_out : tmp_keys;
    uint32_t *vout = ( p & 1 ) ? perm_out : tmp_vals;
    if ( launch_onesweep( kNoAllocBits, kin, vin, kout, vout, n, p, hist, status, sc, 1u << 22, 0, s ) != cudaSuccess )
      return BVHG_ERR_CUDA;
    kin = kout;
    vin = vout;
  }
  int err = 0;
  if ( cudaMemcpyAsync( &err, &sc->error, sizeof( int ), cudaMemcpyDeviceToHost, s ) != cudaSuccess ) return BVHG_ERR_CUDA;
  if ( cudaStreamSynchronize( s ) != cudaSuccess ) return BVHG_ERR_CUDA;
  return err == kErrTimeout ? BVHG_ERR_TIMEOUT : ( err ? BVHG_ERR_CUDA : BVHG_OK );
}
