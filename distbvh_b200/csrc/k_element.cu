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
__device__ void cb_body(const cb_args &args, uint32_t bid, uint32_t nblk)
{
  const double *__restrict__ verts = args.verts;
  const uint64_t n = args.n;
  const double eps = args.eps;
  double *__restrict__ cx = args.cx;
  double *__restrict__ cy = args.cy;
  double *__restrict__ cz = args.cz;
  obj_scalars *__restrict__ sc = args.sc;
  extern __shared__ double s_v[];
  const int V = VT > 0 ? VT : static_cast< int >( args.V );
  const int per = V * 3;
  const double inf = __longlong_as_double( 0x7ff0000000000000LL );
  double mn[3] = { inf, inf, inf };  // identity of min
  double mx[3] = { -inf, -inf, -inf };
  bool bad = false;
  for ( uint64_t t0 = static_cast< uint64_t >( bid ) * kElemThreads; t0 < n;
        t0 += static_cast< uint64_t >( nblk ) * kElemThreads )
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
__device__ void cb_tma_body(const cb_args &args, uint32_t bid, uint32_t nblk)
{
  const double *__restrict__ verts = args.verts;
  const uint64_t n = args.n;
  const double eps = args.eps;
  double *__restrict__ cx = args.cx;
  double *__restrict__ cy = args.cy;
  double *__restrict__ cz = args.cz;
  obj_scalars *__restrict__ sc = args.sc;
  const uint32_t spin_limit = args.spin_limit;
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
  const uint64_t G = nblk;
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
    if ( bid < full )
    {
      issue( bid, 0 );
      pend |= 1u;
    }
    if ( bid + G < full )
    {
      issue( bid + G, 1 );
      pend |= 2u;
    }
  }
  __syncthreads();
  uint32_t phases = 0;  // bit s: parity of stage s's next completion
  int st = 0;
  for ( uint64_t t = bid; t < tiles; t += G, st ^= 1 )
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
__device__ void kh_body(const kh_args &args, uint32_t bid, uint32_t nblk)
{
  const double *__restrict__ cx = args.cx;
  const double *__restrict__ cy = args.cy;
  const double *__restrict__ cz = args.cz;
  const uint64_t n = args.n;
  obj_scalars *__restrict__ sc = args.sc;
  uint64_t *__restrict__ keys = args.keys;
  uint32_t *__restrict__ hist = args.hist;
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
    if ( bid == 0 )
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
  const uint64_t stride = static_cast< uint64_t >( nblk ) * kElemThreads * U;
  const uint64_t base = static_cast< uint64_t >( bid ) * kElemThreads * U;
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
constexpr int kCbTmaMinBlocks = VT == 8 ? 2 : 3;

// Shared memory of the centroid/bounds kernels: two TMA stages of 256 elements, or one plain tile.
size_t cb_smem(uint32_t V, bool tma)
{
  return static_cast< size_t >( tma ? 2 : 1 ) * kElemThreads * V * 3 * sizeof( double );
}

// Per device: the shared-memory opt-in of both launch forms of the TMA kernel and its resident blocks per SM.
template< int K, int VT >
cudaError_t cb_tma_setup(int *per_sm_out)
{
  static int per_sm[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice( &dev );
  if ( e != cudaSuccess ) return e;
  if ( dev < 0 || dev >= 64 ) return cudaErrorInvalidDevice;
  if ( !per_sm[dev] )
  {
    const int smem2 = static_cast< int >( cb_smem( VT, true ) );
    constexpr int MB = kCbTmaMinBlocks< K, VT >;
    e = cudaFuncSetAttribute( k_single< cb_args, cb_tma_body< K, VT >, kElemThreads, MB >,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, smem2 );
    if ( e != cudaSuccess ) return e;
    e = cudaFuncSetAttribute( k_batched< cb_args, cb_tma_body< K, VT >, kElemThreads, MB >,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, smem2 );
    if ( e != cudaSuccess ) return e;
    int b = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor( &b, k_single< cb_args, cb_tma_body< K, VT >, kElemThreads, MB >,
                                                       kElemThreads, smem2 );
    if ( e != cudaSuccess ) return e;
    per_sm[dev] = b > 0 ? b : 1;
  }
  *per_sm_out = per_sm[dev];
  return cudaSuccess;
}

template< int K, int VT >
cudaError_t cb_plain_setup(uint32_t V)
{
  const size_t smem = cb_smem( V, false );
  // Static shared memory counts against the same 48 KB default: opt in whenever the tile is large.
  if ( smem < 40 * 1024 ) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute( k_single< cb_args, cb_body< K, VT >, kElemThreads, 4 >,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast< int >( smem ) );
  if ( e != cudaSuccess ) return e;
  return cudaFuncSetAttribute( k_batched< cb_args, cb_body< K, VT >, kElemThreads, 4 >,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast< int >( smem ) );
}

// Blocks of one object's centroid/bounds launch.
uint32_t cb_grid(uint64_t n, bool tma, int per_sm)
{
  const uint64_t tiles = ( n + kElemThreads - 1 ) / kElemThreads;
  const uint64_t cap = static_cast< uint64_t >( sm_count() ) * ( tma ? per_sm : 8 );
  return static_cast< uint32_t >( tiles < cap ? ( tiles ? tiles : 1 ) : cap );
}

template< int K, int VT >
cudaError_t launch_cb_t(const cb_args &a, cudaStream_t s)
{
  if constexpr ( VT > 0 )
  {
    if ( ( reinterpret_cast< uintptr_t >( a.verts ) & 15 ) == 0 )
    {
      int per_sm = 1;
      cudaError_t e = cb_tma_setup< K, VT >( &per_sm );
      if ( e != cudaSuccess ) return e;
      k_single< cb_args, cb_tma_body< K, VT >, kElemThreads, kCbTmaMinBlocks< K, VT > >
        <<< cb_grid( a.n, true, per_sm ), kElemThreads, cb_smem( VT, true ), s >>>( a );
      return cudaGetLastError();
    }
  }
  cudaError_t e = cb_plain_setup< K, VT >( a.V );
  if ( e != cudaSuccess ) return e;
  k_single< cb_args, cb_body< K, VT >, kElemThreads, 4 ><<< cb_grid( a.n, false, 0 ), kElemThreads, cb_smem( a.V, false ), s >>>( a );
  return cudaGetLastError();
}

// Batched: every item's verts 16-byte aligned and VT > 0 for the TMA form (tma), one V for all items.
template< int K, int VT >
cudaError_t launch_cb_batch_t(uint32_t V, bool tma, const batch_launch &b, cudaStream_t s)
{
  const cb_args *items = static_cast< const cb_args * >( b.items );
  if constexpr ( VT > 0 )
  {
    if ( tma )
    {
      int per_sm = 1;
      cudaError_t e = cb_tma_setup< K, VT >( &per_sm );
      if ( e != cudaSuccess ) return e;
      k_batched< cb_args, cb_tma_body< K, VT >, kElemThreads, kCbTmaMinBlocks< K, VT > >
        <<< b.blocks, kElemThreads, cb_smem( VT, true ), s >>>( items, b.starts, b.nitems );
      return cudaGetLastError();
    }
  }
  cudaError_t e = cb_plain_setup< K, VT >( V );
  if ( e != cudaSuccess ) return e;
  k_batched< cb_args, cb_body< K, VT >, kElemThreads, 4 ><<< b.blocks, kElemThreads, cb_smem( V, false ), s >>>(
    items, b.starts, b.nitems );
  return cudaGetLastError();
}

template< int K >
cudaError_t launch_cb_k(const cb_args &a, cudaStream_t s)
{
  switch ( a.V )
  {
    case 3: return launch_cb_t< K, 3 >( a, s );
    case 4: return launch_cb_t< K, 4 >( a, s );
    case 8: return launch_cb_t< K, 8 >( a, s );
    default: return launch_cb_t< K, 0 >( a, s );
  }
}

template< int K >
cudaError_t launch_cb_batch_k(uint32_t V, bool tma, const batch_launch &b, cudaStream_t s)
{
  switch ( V )
  {
    case 3: return launch_cb_batch_t< K, 3 >( V, tma, b, s );
    case 4: return launch_cb_batch_t< K, 4 >( V, tma, b, s );
    case 8: return launch_cb_batch_t< K, 8 >( V, tma, b, s );
    default: return launch_cb_batch_t< K, 0 >( V, false, b, s );
  }
}

uint32_t kh_grid(uint64_t n)
{
  const uint64_t blocks = ( n + kElemThreads * kKeyUnroll - 1 ) / ( kElemThreads * kKeyUnroll );
  const uint64_t cap = static_cast< uint64_t >( sm_count() ) * 8;
  return static_cast< uint32_t >( blocks < cap ? ( blocks ? blocks : 1 ) : cap );
}

template< int BITS >
cudaError_t launch_kh_t(const kh_args &a, cudaStream_t s)
{
  k_single< kh_args, kh_body< BITS >, kElemThreads, 1 ><<< kh_grid( a.n ), kElemThreads, 0, s >>>( a );
  return cudaGetLastError();
}

template< int BITS >
cudaError_t launch_kh_batch_t(const batch_launch &b, cudaStream_t s)
{
  k_batched< kh_args, kh_body< BITS >, kElemThreads, 1 ><<< b.blocks, kElemThreads, 0, s >>>(
    static_cast< const kh_args * >( b.items ), b.starts, b.nitems );
  return cudaGetLastError();
}

}  // namespace

int device_sm_count() { return sm_count(); }

namespace {

// The reset state of a rebuild in one launch: the object's scalars (zero, Morton-bound minima at the largest
// encoding), the digit histograms, the look-back words of the passes that run, the climb's exchange slots (-1).
__device__ void init_body(const init_args &a, uint32_t bid, uint32_t nblk)
{
  const uint64_t stride = static_cast< uint64_t >( nblk ) * blockDim.x;
  const uint64_t t = static_cast< uint64_t >( bid ) * blockDim.x + threadIdx.x;
  const uint64_t sc_words = a.sc ? sizeof( obj_scalars ) / 4 : 0;  // no scalars: only the exchange slots (refit)
  for ( uint64_t i = t; i < sc_words; i += stride ) reinterpret_cast< uint32_t * >( a.sc )[i] = 0u;
  for ( uint64_t i = t; i < a.hist_words; i += stride ) a.hist[i] = 0u;
  for ( uint64_t i = t; i < a.status_words; i += stride ) a.status[i] = 0u;
  for ( uint64_t i = t; i < a.exch_words; i += stride ) a.exch[i] = -1;
  // the minima start at the largest encoding (written after the zeroing by the same thread)
  for ( uint64_t i = t; i < sc_words; i += stride )
  {
    const uint64_t byte = i * 4;
    if ( byte < 3 * sizeof( unsigned long long ) ) reinterpret_cast< uint32_t * >( a.sc )[i] = 0xffffffffu;
  }
}

uint32_t init_blocks(const init_args &a)
{
  uint64_t most = sizeof( obj_scalars ) / 4;
  if ( a.hist_words > most ) most = a.hist_words;
  if ( a.status_words > most ) most = a.status_words;
  if ( a.exch_words > most ) most = a.exch_words;
  const uint64_t blocks = ( most + 255 ) / 256;
  const uint64_t cap = static_cast< uint64_t >( sm_count() ) * 4;
  return static_cast< uint32_t >( blocks < cap ? blocks : cap );
}

}  // namespace

cudaError_t launch_obj_init(obj_scalars *sc, uint32_t *hist, uint64_t hist_words, uint32_t *status,
                            uint64_t status_words, int *exch, uint64_t exch_words, cudaStream_t s)
{
  const init_args a{ sc, hist, hist_words, status, status_words, exch, exch_words };
  k_single< init_args, init_body, 256, 1 ><<< init_blocks( a ), 256, 0, s >>>( a );
  return cudaGetLastError();
}

uint32_t obj_init_blocks(const init_args &a) { return init_blocks( a ); }

cudaError_t launch_obj_init_batch(const batch_launch &b, cudaStream_t s)
{
  if ( !b.nitems ) return cudaSuccess;
  k_batched< init_args, init_body, 256, 1 ><<< b.blocks, 256, 0, s >>>( static_cast< const init_args * >( b.items ),
                                                                      b.starts, b.nitems );
  return cudaGetLastError();
}

cudaError_t launch_centroid_bounds(int K, const double *verts, uint32_t V, uint64_t n, double eps, double *cx,
                                   double *cy, double *cz, obj_scalars *sc, uint32_t spin_limit, cudaStream_t s)
{
  const cb_args a{ verts, V, n, eps, cx, cy, cz, sc, spin_limit };
  switch ( K )
  {
    case 6: return launch_cb_k< 6 >( a, s );
    case 18: return launch_cb_k< 18 >( a, s );
    case 26: return launch_cb_k< 26 >( a, s );
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t centroid_bounds_blocks(int K, uint32_t V, uint64_t n, bool tma, uint32_t *blocks)
{
  int per_sm = 0;
  if ( tma )
  {
    cudaError_t e = cudaSuccess;
    switch ( K * 100 + static_cast< int >( V ) )
    {
      case 603: e = cb_tma_setup< 6, 3 >( &per_sm ); break;
      case 604: e = cb_tma_setup< 6, 4 >( &per_sm ); break;
      case 608: e = cb_tma_setup< 6, 8 >( &per_sm ); break;
      case 1803: e = cb_tma_setup< 18, 3 >( &per_sm ); break;
      case 1804: e = cb_tma_setup< 18, 4 >( &per_sm ); break;
      case 1808: e = cb_tma_setup< 18, 8 >( &per_sm ); break;
      case 2603: e = cb_tma_setup< 26, 3 >( &per_sm ); break;
      case 2604: e = cb_tma_setup< 26, 4 >( &per_sm ); break;
      case 2608: e = cb_tma_setup< 26, 8 >( &per_sm ); break;
      default: return cudaErrorInvalidValue;
    }
    if ( e != cudaSuccess ) return e;
  }
  *blocks = cb_grid( n, tma, per_sm );
  return cudaSuccess;
}

cudaError_t launch_centroid_bounds_batch(int K, uint32_t V, bool tma, const batch_launch &b, cudaStream_t s)
{
  if ( !b.nitems ) return cudaSuccess;
  switch ( K )
  {
    case 6: return launch_cb_batch_k< 6 >( V, tma, b, s );
    case 18: return launch_cb_batch_k< 18 >( V, tma, b, s );
    case 26: return launch_cb_batch_k< 26 >( V, tma, b, s );
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_keys_hist(int bits, const double *cx, const double *cy, const double *cz, uint64_t n,
                             obj_scalars *sc, uint64_t *keys, uint32_t *hist, cudaStream_t s)
{
  const kh_args a{ cx, cy, cz, n, sc, keys, hist };
  switch ( bits )
  {
    case 1: return launch_kh_t< 1 >( a, s );
    case 2: return launch_kh_t< 2 >( a, s );
    case 4: return launch_kh_t< 4 >( a, s );
    case 8: return launch_kh_t< 8 >( a, s );
    default: return cudaErrorInvalidValue;
  }
}

uint32_t keys_hist_blocks(uint64_t n) { return kh_grid( n ); }

cudaError_t launch_keys_hist_batch(int bits, const batch_launch &b, cudaStream_t s)
{
  if ( !b.nitems ) return cudaSuccess;
  switch ( bits )
  {
    case 1: return launch_kh_batch_t< 1 >( b, s );
    case 2: return launch_kh_batch_t< 2 >( b, s );
    case 4: return launch_kh_batch_t< 4 >( b, s );
    case 8: return launch_kh_batch_t< 8 >( b, s );
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace bvhg
