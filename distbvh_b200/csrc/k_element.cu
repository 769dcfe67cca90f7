// k_element.cu — per-element kernels: centroids + Morton bounds (K1), Morton keys + radix digit histograms (K2).
//
// K1 follows compute_bounds(min_inv_diag_bounds) (src/bvh/contact_entity.hpp:67-80, 136-148): the min over
// elements of each cardinal slab min and the max of each cardinal slab max, computed from the element's FP64
// slabs exactly as kdop_base::from_vertices builds them (kdop.hpp:238-264). The element centroid is the mean of
// its vertices, accumulated from zero and divided by the vertex count (tests/TestCommon.hpp:62-65).
// K2 follows morton_impl (contact_entity.hpp:104-118) with quantize64 (hash.hpp:177-198) and morton64
// (hash.hpp:72-103): q = u64(((c - min) * inv) * 2^21) & 0x1fffff per axis; key = z<<2 | y<<1 | x interleave.
#include "bulk_copy.cuh"
#include "bvhg_internal.cuh"
#include "kdop_math.cuh"

#include <cfloat>

namespace bvhg {
namespace {

constexpr int kElemThreads = 256;
constexpr int kKeyUnroll = 4;  // elements per thread per step of the key kernel

// Exact min/max block reduction of 6 doubles, then one order-preserving 64-bit atomic per value.
__device__ __forceinline__ void reduce_bounds(double mn[3], double mx[3], bool bad, obj_scalars *sc)
{
  __shared__ double s_red[6][kElemThreads / 32];
  __shared__ int s_bad;
  if ( threadIdx.x == 0 ) s_bad = 0;
  for ( int c = 0; c < 3; ++c )
  {
    for ( int o = 16; o > 0; o >>= 1 )
    {
      const double a = __shfl_xor_sync( 0xffffffffu, mn[c], o );
      const double b = __shfl_xor_sync( 0xffffffffu, mx[c], o );
      mn[c] = ( a < mn[c] ) ? a : mn[c];
      mx[c] = ( b > mx[c] ) ? b : mx[c];
    }
  }
  __syncthreads();
  if ( bad ) s_bad = 1;
  const int w = threadIdx.x >> 5;
  if ( ( threadIdx.x & 31 ) == 0 )
  {
    for ( int c = 0; c < 3; ++c )
    {
      s_red[c][w] = mn[c];
      s_red[3 + c][w] = mx[c];
    }
  }
  __syncthreads();
  if ( threadIdx.x < 6 )
  {
    const int c = threadIdx.x;
    double v = s_red[c][0];
    for ( int k = 1; k < kElemThreads / 32; ++k )
    {
      const double x = s_red[c][k];
      if ( c < 3 ) v = ( x < v ) ? x : v;
      else v = ( x > v ) ? x : v;
    }
    if ( c < 3 ) atomicMin( &sc->bounds_enc[c], ord_encode( v ) );
    else atomicMax( &sc->bounds_enc[c], ord_encode( v ) );
  }
  if ( threadIdx.x == 0 && s_bad ) atomicCAS( &sc->error, 0, kErrArg );
}

// One element (its V vertices at p, in shared memory): centroid to cx/cy/cz[i], cardinal slabs into the running
// min/max, non-finite coordinates into bad.
template< int K >
__device__ __forceinline__ void element_centroid_bounds(const double *p, int V, double eps, uint64_t i,
                                                        double *__restrict__ cx, double *__restrict__ cy,
                                                        double *__restrict__ cz, double mn[3], double mx[3], bool &bad)
{
  double sx = 0.0, sy = 0.0, sz = 0.0;
  for ( int v = 0; v < V; ++v )
  {
    const double x = p[3 * v], y = p[3 * v + 1], z = p[3 * v + 2];
    bad |= !( isfinite( x ) && isfinite( y ) && isfinite( z ) );
    sx = __dadd_rn( sx, x );
    sy = __dadd_rn( sy, y );
    sz = __dadd_rn( sz, z );
  }
  const double dv = static_cast< double >( V );
  cx[i] = __ddiv_rn( sx, dv );
  cy[i] = __ddiv_rn( sy, dv );
  cz[i] = __ddiv_rn( sz, dv );
#pragma unroll
  for ( int a = 0; a < 3; ++a )
  {
    double lo, hi;
    slab64< K >( p, V, a, eps, lo, hi );
    mn[a] = ( lo < mn[a] ) ? lo : mn[a];
    mx[a] = ( hi > mx[a] ) ? hi : mx[a];
  }
}

// K1. Each block stages a tile of 256 elements (256 * V * 24 bytes, contiguous) into shared memory with
// coalesced 16-byte loads, then each thread reduces its own element. Grid-stride over tiles.
template< int K, int VT >
__global__ void __launch_bounds__( kElemThreads ) k_centroid_bounds(const double *__restrict__ verts, uint32_t Vrt,
                                                                  uint64_t n, double eps, double *__restrict__ cx,
                                                                  double *__restrict__ cy, double *__restrict__ cz,
                                                                  obj_scalars *__restrict__ sc)
{
  extern __shared__ double s_v[];
  const int V = VT > 0 ? VT : static_cast< int >( Vrt );
  const int per = V * 3;
  const double inf = __longlong_as_double( 0x7ff0000000000000LL );
  double mn[3] = { inf, inf, inf };  // identity of min
  double mx[3] = { -inf, -inf, -inf };
  bool bad = false;
  for ( uint64_t t0 = static_cast< uint64_t >( blockIdx.x ) * kElemThreads; t0 < n;
        t0 += static_cast< uint64_t >( gridDim.x ) * kElemThreads )
  {
    const int cnt = static_cast< int >( min( static_cast< uint64_t >( kElemThreads ), n - t0 ) );
    const double *src = verts + t0 * per;
    const int total = cnt * per;
    __syncthreads();
    if ( ( reinterpret_cast< uintptr_t >( src ) & 15 ) == 0 )
    {
      const int n2 = total >> 1;
      const double2 *src2 = reinterpret_cast< const double2 * >( src );
      double2 *dst2 = reinterpret_cast< double2 * >( s_v );
      for ( int k = threadIdx.x; k < n2; k += kElemThreads ) dst2[k] = __ldcs( src2 + k );
      if ( ( total & 1 ) && threadIdx.x == 0 ) s_v[total - 1] = __ldcs( src + total - 1 );
    } else {
      for ( int k = threadIdx.x; k < total; k += kElemThreads ) s_v[k] = __ldcs( src + k );
    }
    __syncthreads();
    if ( static_cast< int >( threadIdx.x ) < cnt )
      element_centroid_bounds< K >( s_v + threadIdx.x * per, V, eps, t0 + threadIdx.x, cx, cy, cz, mn, mx, bad );
  }
  reduce_bounds( mn, mx, bad, sc );
}

// K1 for a fixed vertex count, persistent and double-buffered: block b takes tiles b, b + G, b + 2G, ... (G = the
// grid); while it reduces one tile from shared memory, the bulk copy (TMA) of its next tile streams into the other
// stage. Full tiles (256 elements, 256 * VT * 24 bytes, 16-byte aligned) go through the bulk copy; the last,
// partial tile through plain loads. Every wait on a copy is bounded: past spin_limit polls the block raises the
// object's error word, waits (bounded) for its copies in flight and stops.
template< int K, int VT >
__global__ void __launch_bounds__( kElemThreads, VT == 8 ? 2 : 3 ) k_centroid_bounds_tma(const double *__restrict__ verts, uint64_t n,
                                                                      double eps, double *__restrict__ cx,
                                                                      double *__restrict__ cy, double *__restrict__ cz,
                                                                      obj_scalars *__restrict__ sc, uint32_t spin_limit)
{
  constexpr int per = VT * 3;
  constexpr uint32_t kTileD = kElemThreads * per;  // doubles per tile
  extern __shared__ __align__( 128 ) double s_stage[];  // 2 stages of kTileD doubles
  __shared__ __align__( 8 ) uint64_t s_mbar[2];
  const double inf = __longlong_as_double( 0x7ff0000000000000LL );
  double mn[3] = { inf, inf, inf };
  double mx[3] = { -inf, -inf, -inf };
  bool bad = false;
  const uint64_t tiles = ( n + kElemThreads - 1 ) / kElemThreads;
  const uint64_t full = n / kElemThreads;  // tiles that are bulk-copied
  const uint64_t G = gridDim.x;
  const int tid = threadIdx.x;
  auto issue = [&](uint64_t t, int st) {
    mbar_expect_tx( &s_mbar[st], kTileD * 8 );
    bulk_load( s_stage + st * kTileD, verts + t * kTileD, kTileD * 8, &s_mbar[st] );
  };
  uint32_t pend = 0;  // thread 0: bit s set while stage s has a copy in flight
  if ( tid == 0 )
  {
    mbar_init( &s_mbar[0], 1 );
    mbar_init( &s_mbar[1], 1 );
    mbar_init_fence();
    if ( blockIdx.x < full )
    {
      issue( blockIdx.x, 0 );
      pend |= 1u;
    }
    if ( blockIdx.x + G < full )
    {
      issue( blockIdx.x + G, 1 );
      pend |= 2u;
    }
  }
  __syncthreads();
  uint32_t phases = 0;  // bit s: parity of stage s's next completion
  int st = 0;
  for ( uint64_t t = blockIdx.x; t < tiles; t += G, st ^= 1 )
  {
    double *sv = s_stage + st * kTileD;
    const int cnt = static_cast< int >( min( static_cast< uint64_t >( kElemThreads ), n - t * kElemThreads ) );
    if ( t < full )
    {
      const uint32_t ph = ( phases >> st ) & 1u;
      const bool ok = mbar_wait_bounded( &s_mbar[st], ph, spin_limit );
      phases ^= 1u << st;
      if ( tid == 0 && ok ) pend &= ~( 1u << st );
      if ( __syncthreads_or( !ok ) )
      {
        if ( tid == 0 )
        {
          atomicCAS( &sc->error, 0, kErrTimeout );
          // the shared memory stays allocated until the copies in flight have landed (or the wait gives up)
          for ( int s2 = 0; s2 < 2; ++s2 )
            if ( pend & ( 1u << s2 ) )
              mbar_wait_bounded( &s_mbar[s2], ( ( phases >> s2 ) & 1u ) ^ ( s2 == st ? 1u : 0u ), spin_limit );
        }
        return;
      }
    } else {
      const double *src = verts + t * kTileD;
      for ( int k = tid; k < cnt * per; k += kElemThreads ) sv[k] = __ldcs( src + k );
      __syncthreads();
    }
    if ( tid < cnt ) element_centroid_bounds< K >( sv + tid * per, VT, eps, t * kElemThreads + tid, cx, cy, cz, mn, mx, bad );
    __syncthreads();  // the stage was read by every thread: it may be refilled
    if ( tid == 0 && t + 2 * G < full )
    {
      fence_proxy_async_smem();
      issue( t + 2 * G, st );
      pend |= 1u << st;
    }
  }
  reduce_bounds( mn, mx, bad, sc );
}

__device__ __forceinline__ uint64_t expand64(uint64_t v)
{
  v = ( v * 0x1000001ull ) & 0xfff000000fffull;
  v = ( v * 0x1001ull ) & 0xfc003f000fc003full;
  v = ( v * 0x41ull ) & 0x01c0e070381c0e07ull;
  v = ( v * 0x11ull ) & 0x10c86432190c8643ull;
  v = ( v * 0x5ull ) & 0x1249249249249249ull;
  return v;
}

// static_cast<uint64_t>(double) with the x86-64 truncating semantics the reference is built with: values below
// 2^63 convert through the signed path, so (-1, 0) -> 0 and NaN -> 0 after the 21-bit mask.
__device__ __forceinline__ uint64_t quant21(double c, double mn, double inv)
{
  const double norm = __dmul_rn( __dsub_rn( c, mn ), inv );
  const double scaled = __dmul_rn( norm, 2097152.0 );
  return static_cast< uint64_t >( static_cast< long long >( scaled ) ) & 0x1fffffull;
}

// K2. Morton key of every element, written in original order, plus the digit histogram of every radix pass that
// runs, those over the high key half (warp-aggregated shared-memory counters, one global atomic per nonzero bin
// per block).
template< int BITS >
__global__ void __launch_bounds__( kElemThreads ) k_keys_hist(const double *__restrict__ cx,
                                                            const double *__restrict__ cy,
                                                            const double *__restrict__ cz, uint64_t n,
                                                            obj_scalars *__restrict__ sc, uint64_t *__restrict__ keys,
                                                            uint32_t *__restrict__ hist)
{
  constexpr int RADIX = 1 << BITS;
  constexpr int PASSES = ( kKeyBits + BITS - 1 ) / BITS;
  constexpr int FIRST = 32 / BITS;  // only the passes over the high key half run (the fix-up sorts the low half)
  constexpr int NH = PASSES - FIRST;
  __shared__ uint32_t s_hist[NH * RADIX];
  __shared__ double s_min[3], s_inv[3];
  for ( int k = threadIdx.x; k < NH * RADIX; k += kElemThreads ) s_hist[k] = 0;
  if ( threadIdx.x < 3 )
  {
    const int c = threadIdx.x;
    const double mn = ord_decode( sc->bounds_enc[c] );
    const double mx = ord_decode( sc->bounds_enc[3 + c] );
    const double width = __dsub_rn( mx, mn );
    const double inv = __ddiv_rn( 1.0, width );
    s_min[c] = mn;
    s_inv[c] = inv;
    if ( blockIdx.x == 0 )
    {
      sc->min3[c] = mn;
      sc->inv3[c] = inv;
    }
  }
  __syncthreads();
  const double m0 = s_min[0], m1 = s_min[1], m2 = s_min[2];
  const double i0 = s_inv[0], i1 = s_inv[1], i2 = s_inv[2];
  const unsigned lane = threadIdx.x & 31;
  // Each warp takes runs of kKeyUnroll * 32 consecutive elements (element w0 + 32 u + lane in step u): the loads of
  // all steps are issued before the first key is formed, which keeps kKeyUnroll loads per thread in flight.
  constexpr int U = kKeyUnroll;
  const uint64_t stride = static_cast< uint64_t >( gridDim.x ) * kElemThreads * U;
  const uint64_t base = static_cast< uint64_t >( blockIdx.x ) * kElemThreads * U;
  // Every warp runs the same number of iterations so that the warp-wide match below sees all 32 lanes.
  for ( uint64_t w0 = base + ( threadIdx.x & ~31u ) * U; w0 < n; w0 += stride )
  {
    double vx[U], vy[U], vz[U];
#pragma unroll
    for ( int u = 0; u < U; ++u )
    {
      const uint64_t i = w0 + 32 * u + lane;
      vx[u] = i < n ? cx[i] : 0.0;
      vy[u] = i < n ? cy[i] : 0.0;
      vz[u] = i < n ? cz[i] : 0.0;
    }
#pragma unroll
    for ( int u = 0; u < U; ++u )
    {
      const uint64_t i = w0 + 32 * u + lane;
      const bool valid = i < n;
      uint64_t key = 0;
      if ( valid )
      {
        const uint64_t qx = quant21( vx[u], m0, i0 );
        const uint64_t qy = quant21( vy[u], m1, i1 );
        const uint64_t qz = quant21( vz[u], m2, i2 );
        key = ( expand64( qz ) << 2 ) | ( expand64( qy ) << 1 ) | expand64( qx );
        keys[i] = key;
      }
      const unsigned vmask = __ballot_sync( 0xffffffffu, valid );
#pragma unroll
      for ( int p = FIRST; p < PASSES; ++p )
      {
        const unsigned d = static_cast< unsigned >( ( key >> ( p * BITS ) ) & ( RADIX - 1 ) );
        // Spatially coherent warps share their high digits: one atomic for a uniform warp, else one per lane.
        const unsigned d0 = __shfl_sync( 0xffffffffu, d, 0 );
        if ( __all_sync( 0xffffffffu, d == d0 || !valid ) && vmask == 0xffffffffu )
        {
          if ( lane == 0 ) atomicAdd( &s_hist[( p - FIRST ) * RADIX + d0], 32u );
        } else if ( valid ) {
          atomicAdd( &s_hist[( p - FIRST ) * RADIX + d], 1u );
        }
      }
    }
  }
  __syncthreads();
  for ( int k = threadIdx.x; k < NH * RADIX; k += kElemThreads )
    if ( s_hist[k] ) atomicAdd( &hist[FIRST * RADIX + k], s_hist[k] );
}

int sm_count()
{
  static int cached = 0;
  if ( !cached )
  {
    int dev = 0;
    cudaGetDevice( &dev );
    cudaDeviceGetAttribute( &cached, cudaDevAttrMultiProcessorCount, dev );
    if ( cached <= 0 ) cached = 148;
  }
  return cached;
}

template< int K, int VT >
cudaError_t launch_cb_t(const double *verts, uint32_t V, uint64_t n, double eps, double *cx, double *cy, double *cz,
                        obj_scalars *sc, uint32_t spin_limit, cudaStream_t s)
{
  if constexpr ( VT > 0 )
  {
    if ( ( reinterpret_cast< uintptr_t >( verts ) & 15 ) == 0 )
    {
      const size_t smem2 = static_cast< size_t >( 2 ) * kElemThreads * VT * 3 * sizeof( double );
      // per device: the shared-memory opt-in and the resident blocks per SM of the persistent grid
      static int per_sm[64] = {};
      int dev = 0;
      cudaError_t e = cudaGetDevice( &dev );
      if ( e != cudaSuccess ) return e;
      if ( dev < 0 || dev >= 64 ) return cudaErrorInvalidDevice;
      if ( !per_sm[dev] )
      {
        e = cudaFuncSetAttribute( k_centroid_bounds_tma< K, VT >, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast< int >( smem2 ) );
        if ( e != cudaSuccess ) return e;
        int b = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor( &b, k_centroid_bounds_tma< K, VT >, kElemThreads, smem2 );
        if ( e != cudaSuccess ) return e;
        per_sm[dev] = b > 0 ? b : 1;
      }
      const uint64_t tiles = ( n + kElemThreads - 1 ) / kElemThreads;
      const uint64_t cap = static_cast< uint64_t >( sm_count() ) * per_sm[dev];
      const unsigned grid = static_cast< unsigned >( tiles < cap ? ( tiles ? tiles : 1 ) : cap );
      k_centroid_bounds_tma< K, VT ><<< grid, kElemThreads, smem2, s >>>( verts, n, eps, cx, cy, cz, sc, spin_limit );
      return cudaGetLastError();
    }
  }
  const size_t smem = static_cast< size_t >( kElemThreads ) * V * 3 * sizeof( double );
  // Static shared memory counts against the same 48 KB default: opt in whenever the tile is large.
  if ( smem >= 40 * 1024 )
  {
    cudaError_t e = cudaFuncSetAttribute( k_centroid_bounds< K, VT >, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          static_cast< int >( smem ) );
    if ( e != cudaSuccess ) return e;
  }
  const uint64_t tiles = ( n + kElemThreads - 1 ) / kElemThreads;
  const uint64_t cap = static_cast< uint64_t >( sm_count() ) * 8;
  const unsigned grid = static_cast< unsigned >( tiles < cap ? ( tiles ? tiles : 1 ) : cap );
  k_centroid_bounds< K, VT ><<< grid, kElemThreads, smem, s >>>( verts, V, n, eps, cx, cy, cz, sc );
  return cudaGetLastError();
}

template< int K >
cudaError_t launch_cb_k(const double *verts, uint32_t V, uint64_t n, double eps, double *cx, double *cy, double *cz,
                        obj_scalars *sc, uint32_t spin_limit, cudaStream_t s)
{
  switch ( V )
  {
    case 3: return launch_cb_t< K, 3 >( verts, V, n, eps, cx, cy, cz, sc, spin_limit, s );
    case 4: return launch_cb_t< K, 4 >( verts, V, n, eps, cx, cy, cz, sc, spin_limit, s );
    case 8: return launch_cb_t< K, 8 >( verts, V, n, eps, cx, cy, cz, sc, spin_limit, s );
    default: return launch_cb_t< K, 0 >( verts, V, n, eps, cx, cy, cz, sc, spin_limit, s );
  }
}

template< int BITS >
cudaError_t launch_kh_t(const double *cx, const double *cy, const double *cz, uint64_t n, obj_scalars *sc,
                        uint64_t *keys, uint32_t *hist, cudaStream_t s)
{
  const uint64_t blocks = ( n + kElemThreads * kKeyUnroll - 1 ) / ( kElemThreads * kKeyUnroll );
  const uint64_t cap = static_cast< uint64_t >( sm_count() ) * 8;
  const unsigned grid = static_cast< unsigned >( blocks < cap ? ( blocks ? blocks : 1 ) : cap );
  k_keys_hist< BITS ><<< grid, kElemThreads, 0, s >>>( cx, cy, cz, n, sc, keys, hist );
  return cudaGetLastError();
}

}  // namespace

int device_sm_count() { return sm_count(); }

namespace {

// The reset state of a rebuild in one launch: the object's scalars (zero, Morton-bound minima at the largest
// encoding), the digit histograms, the look-back words of the passes that run, the climb's exchange slots (-1).
__global__ void k_obj_init(obj_scalars *sc, uint32_t *hist, uint64_t hist_words, uint32_t *status,
                           uint64_t status_words, int *exch, uint64_t exch_words)
{
  const uint64_t stride = static_cast< uint64_t >( gridDim.x ) * blockDim.x;
  const uint64_t t = static_cast< uint64_t >( blockIdx.x ) * blockDim.x + threadIdx.x;
  constexpr uint64_t sc_words = sizeof( obj_scalars ) / 4;
  for ( uint64_t i = t; i < sc_words; i += stride ) reinterpret_cast< uint32_t * >( sc )[i] = 0u;
  for ( uint64_t i = t; i < hist_words; i += stride ) hist[i] = 0u;
  for ( uint64_t i = t; i < status_words; i += stride ) status[i] = 0u;
  for ( uint64_t i = t; i < exch_words; i += stride ) exch[i] = -1;
  // the minima start at the largest encoding (written after the zeroing by the same thread)
  for ( uint64_t i = t; i < sc_words; i += stride )
  {
    const uint64_t byte = i * 4;
    if ( byte < 3 * sizeof( unsigned long long ) ) reinterpret_cast< uint32_t * >( sc )[i] = 0xffffffffu;
  }
}

}  // namespace

cudaError_t launch_obj_init(obj_scalars *sc, uint32_t *hist, uint64_t hist_words, uint32_t *status,
                            uint64_t status_words, int *exch, uint64_t exch_words, cudaStream_t s)
{
  uint64_t most = sizeof( obj_scalars ) / 4;
  if ( hist_words > most ) most = hist_words;
  if ( status_words > most ) most = status_words;
  if ( exch_words > most ) most = exch_words;
  const uint64_t blocks = ( most + 255 ) / 256;
  const uint64_t cap = static_cast< uint64_t >( sm_count() ) * 4;
  k_obj_init<<< static_cast< unsigned >( blocks < cap ? blocks : cap ), 256, 0, s >>>( sc, hist, hist_words, status,
                                                                                     status_words, exch, exch_words );
  return cudaGetLastError();
}

cudaError_t launch_centroid_bounds(int K, const double *verts, uint32_t V, uint64_t n, double eps, double *cx,
                                   double *cy, double *cz, obj_scalars *sc, uint32_t spin_limit, cudaStream_t s)
{
  switch ( K )
  {
    case 6: return launch_cb_k< 6 >( verts, V, n, eps, cx, cy, cz, sc, spin_limit, s );
    case 18: return launch_cb_k< 18 >( verts, V, n, eps, cx, cy, cz, sc, spin_limit, s );
    case 26: return launch_cb_k< 26 >( verts, V, n, eps, cx, cy, cz, sc, spin_limit, s );
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_keys_hist(int bits, const double *cx, const double *cy, const double *cz, uint64_t n,
                             obj_scalars *sc, uint64_t *keys, uint32_t *hist, cudaStream_t s)
{
  switch ( bits )
  {
    case 1: return launch_kh_t< 1 >( cx, cy, cz, n, sc, keys, hist, s );
    case 2: return launch_kh_t< 2 >( cx, cy, cz, n, sc, keys, hist, s );
    case 4: return launch_kh_t< 4 >( cx, cy, cz, n, sc, keys, hist, s );
    case 8: return launch_kh_t< 8 >( cx, cy, cz, n, sc, keys, hist, s );
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace bvhg
