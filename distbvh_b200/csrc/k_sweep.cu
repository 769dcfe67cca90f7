// k_sweep.cu — sort-and-sweep candidate generation between two objects.
//
// Follows sort_and_sweep_local (src/bvh/narrowphase/kokkos.hpp:164-248) with the two objects as the two patches,
// and max_variant_axis (kokkos.hpp:125-160) for the sweep axis when the caller gives none:
// - the global range on the axis is the union of both objects' slab extents there (the K1 bounds of each object:
//   min of the cardinal slab minima, max of the maxima);
// - B's slab minima on the axis become u32 keys (min - global_min) * (UINT32_MAX / (global_max - global_min)),
//   truncated; a stable LSD radix sort of (key, index) over the four bytes of the key (the radix pass of k_sort.cu);
// - every element of A sweeps B in key order: it skips B elements whose scaled maximum lies below its minimum key,
//   stops at the first B key above its maximum key, and emits the B elements that overlap it strictly on every
//   slab. The emitted set is the exact pair set S(A, B) for any axis.
// Here each A element sweeps only the key window [its minimum key - W, its maximum key], W = the largest
// (scaled maximum - key) over B: every B element below the window has a scaled maximum below A's minimum key and is
// one the reference's loop skips, so the window emits the same pairs.
// A degenerate axis (global_max == global_min) gives every key 0 here; the reference's factor is then infinite and
// its keys 0 as well (NaN converts to 0), with the same outcome: no element is skipped or stops a sweep.
#include "bvhg_internal.cuh"
#include "kdop_math.cuh"

namespace bvhg {
int device_sm_count();
namespace {

constexpr int kSweepThreads = 256;
constexpr int kAxisBlocks = 512;  // partial sums of the axis choice (a fixed grid: a fixed summation order)

struct sweep_params
{
  int axis;
  int pad;
  double gmin;
  double fac;
  unsigned long long wmax_enc;  // order-preserving encoding of W
};

// u32 of a scaled value as the reference's conversion yields it for every value this path produces (truncation;
// NaN and values outside the signed 64-bit range give 0).
__device__ __forceinline__ uint32_t key32(double x)
{
  if ( !( x < 9223372036854775808.0 ) || !( x >= -9223372036854775808.0 ) ) return 0u;
  return static_cast< uint32_t >( static_cast< unsigned long long >( __double2ll_rz( x ) ) );
}

__device__ __forceinline__ double scaled(double v, const sweep_params &p)
{
  return __dmul_rn( __dsub_rn( v, p.gmin ), p.fac );
}

// Partial sums of the centroids and their squares over A then B (block b: a grid-stride range), fixed order.
__global__ void __launch_bounds__( kSweepThreads ) k_axis_partial(const double *__restrict__ ax,
                                                                  const double *__restrict__ ay,
                                                                  const double *__restrict__ az, uint64_t na,
                                                                  const double *__restrict__ bx,
                                                                  const double *__restrict__ by,
                                                                  const double *__restrict__ bz, uint64_t nb,
                                                                  double *__restrict__ partial)
{
  __shared__ double s_red[6][kSweepThreads];
  double s[6] = { 0, 0, 0, 0, 0, 0 };
  const uint64_t n = na + nb;
  for ( uint64_t i = static_cast< uint64_t >( blockIdx.x ) * kSweepThreads + threadIdx.x; i < n;
        i += static_cast< uint64_t >( gridDim.x ) * kSweepThreads )
  {
    const double x = i < na ? ax[i] : bx[i - na];
    const double y = i < na ? ay[i] : by[i - na];
    const double z = i < na ? az[i] : bz[i - na];
    s[0] = __dadd_rn( s[0], x );
    s[1] = __dadd_rn( s[1], y );
    s[2] = __dadd_rn( s[2], z );
    s[3] = __dadd_rn( s[3], __dmul_rn( x, x ) );
    s[4] = __dadd_rn( s[4], __dmul_rn( y, y ) );
    s[5] = __dadd_rn( s[5], __dmul_rn( z, z ) );
  }
  for ( int k = 0; k < 6; ++k ) s_red[k][threadIdx.x] = s[k];
  __syncthreads();
  for ( int h = kSweepThreads / 2; h > 0; h >>= 1 )
  {
    if ( static_cast< int >( threadIdx.x ) < h )
      for ( int k = 0; k < 6; ++k ) s_red[k][threadIdx.x] = __dadd_rn( s_red[k][threadIdx.x], s_red[k][threadIdx.x + h] );
    __syncthreads();
  }
  if ( threadIdx.x < 6 ) partial[blockIdx.x * 6 + threadIdx.x] = s_red[threadIdx.x][0];
}

// The axis (given, or of largest centroid variance), the global range on it and the scale factor.
__global__ void k_sweep_setup(const double *__restrict__ partial, int nblocks, uint64_t n, int axis_in,
                              const obj_scalars *__restrict__ sa, const obj_scalars *__restrict__ sb,
                              sweep_params *__restrict__ p)
{
  if ( threadIdx.x != 0 ) return;
  int axis = axis_in;
  if ( axis < 0 )
  {
    double s[6] = { 0, 0, 0, 0, 0, 0 };
    for ( int b = 0; b < nblocks; ++b )
      for ( int k = 0; k < 6; ++k ) s[k] = __dadd_rn( s[k], partial[b * 6 + k] );
    double var[3];
    for ( int k = 0; k < 3; ++k )
      var[k] = __dsub_rn( s[3 + k], __ddiv_rn( __dmul_rn( s[k], s[k] ), static_cast< double >( n ) ) );
    axis = 0;
    if ( var[1] > var[0] ) axis = 1;
    if ( var[2] > var[axis] ) axis = 2;
  }
  const double amin = ord_decode( sa->bounds_enc[axis] ), amax = ord_decode( sa->bounds_enc[3 + axis] );
  const double bmin = ord_decode( sb->bounds_enc[axis] ), bmax = ord_decode( sb->bounds_enc[3 + axis] );
  const double gmin = bmin < amin ? bmin : amin;
  const double gmax = amax < bmax ? bmax : amax;
  p->axis = axis;
  p->gmin = gmin;
  p->fac = gmax > gmin ? __ddiv_rn( 4294967295.0, __dsub_rn( gmax, gmin ) ) : 0.0;
  p->wmax_enc = ord_encode( 0.0 );
}

// B: element slab rows (original order), u32 keys of the slab minima on the axis, the byte histograms of the four
// radix passes, and W = max (scaled maximum - key).
template< int K, int VT >
__global__ void __launch_bounds__( kSweepThreads ) k_sweep_keys(const double *__restrict__ verts, uint32_t Vrt,
                                                                uint64_t n, double eps,
                                                                const sweep_params *pp, double *__restrict__ rows,
                                                                uint64_t *__restrict__ keys, uint32_t *__restrict__ hist,
                                                                sweep_params *pw)  // pp and pw: the same struct
{
  constexpr int D = K / 2;
  __shared__ uint32_t s_hist[4 * 256];
  __shared__ double s_w[kSweepThreads / 32];
  for ( int k = threadIdx.x; k < 4 * 256; k += kSweepThreads ) s_hist[k] = 0;
  const sweep_params p = *pp;
  __syncthreads();
  const uint64_t i = static_cast< uint64_t >( blockIdx.x ) * kSweepThreads + threadIdx.x;
  double w = 0.0;
  if ( i < n )
  {
    double lo[D], hi[D];
    leaf_slabs< K, double, VT >( verts, Vrt, static_cast< uint32_t >( i ), eps, 0.f, lo, hi );
    double *row = rows + i * 2 * D;
#pragma unroll
    for ( int a = 0; a < D; ++a )
    {
      row[2 * a] = lo[a];
      row[2 * a + 1] = hi[a];
    }
    const double mn = p.axis == 0 ? lo[0] : ( p.axis == 1 ? lo[1] : lo[2] );
    const double mx = p.axis == 0 ? hi[0] : ( p.axis == 1 ? hi[1] : hi[2] );
    const uint32_t key = key32( scaled( mn, p ) );
    keys[i] = key;
    w = __dsub_rn( scaled( mx, p ), static_cast< double >( key ) );
    for ( int q = 0; q < 4; ++q ) atomicAdd( &s_hist[q * 256 + ( ( key >> ( 8 * q ) ) & 255u )], 1u );
  }
  for ( int o = 16; o > 0; o >>= 1 )
  {
    const double x = __shfl_xor_sync( 0xffffffffu, w, o );
    w = x > w ? x : w;
  }
  if ( ( threadIdx.x & 31 ) == 0 ) s_w[threadIdx.x >> 5] = w;
  __syncthreads();
  for ( int k = threadIdx.x; k < 4 * 256; k += kSweepThreads )
    if ( s_hist[k] ) atomicAdd( &hist[k], s_hist[k] );
  if ( threadIdx.x == 0 )
  {
    double m = s_w[0];
    for ( int k = 1; k < kSweepThreads / 32; ++k ) m = s_w[k] > m ? s_w[k] : m;
    atomicMax( &pw->wmax_enc, ord_encode( m ) );
  }
}

// B in key order: its slab rows and its scaled maxima on the axis (the sweeps read both sequentially).
template< int K >
__global__ void __launch_bounds__( kSweepThreads ) k_sweep_gather(const double *__restrict__ rows,
                                                                  const uint32_t *__restrict__ svals, uint64_t n,
                                                                  const sweep_params *__restrict__ pp,
                                                                  double *__restrict__ srows,
                                                                  double *__restrict__ sbmax)
{
  constexpr int C = K;  // 2 D values per row
  const sweep_params p = *pp;
  for ( uint64_t k = static_cast< uint64_t >( blockIdx.x ) * kSweepThreads + threadIdx.x; k < n * C;
        k += static_cast< uint64_t >( gridDim.x ) * kSweepThreads )
  {
    const uint64_t j = k / C;
    const int c = static_cast< int >( k - j * C );
    const double v = __ldg( rows + static_cast< uint64_t >( __ldg( svals + j ) ) * C + c );
    srows[k] = v;
    if ( c == 2 * p.axis + 1 ) sbmax[j] = scaled( v, p );
  }
}

// First index in [0, n) whose key is >= v (lower) or > v (upper).
__device__ __forceinline__ uint64_t key_bound(const uint64_t *__restrict__ keys, uint64_t n, uint64_t v, bool upper)
{
  uint64_t lo = 0, hi = n;
  while ( lo < hi )
  {
    const uint64_t mid = ( lo + hi ) >> 1;
    const uint64_t k = __ldg( keys + mid );
    if ( upper ? k <= v : k < v ) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// A: one warp per element (A in its Morton order, warps grid-stride over it). All lanes form the element's slabs
// and window (the same values; the loads are broadcasts), then scan the window 32 keys at a time: lane l tests
// key j0 + l + 32 k, so every load of the scaled maxima and of the rows is coalesced across the warp.
template< int K, int VT >
__global__ void __launch_bounds__( kSweepThreads ) k_sweep(const double *__restrict__ verts, uint32_t Vrt, uint64_t na,
                                                           double eps, const sweep_params *__restrict__ pp,
                                                           const uint32_t *__restrict__ aperm,
                                                           const uint64_t *__restrict__ skeys,
                                                           const uint32_t *__restrict__ svals,
                                                           const double *__restrict__ srows,
                                                           const double *__restrict__ sbmax, uint64_t nb,
                                                           const obj_scalars *__restrict__ ssc, uint2 *__restrict__ pairs,
                                                           uint64_t cap, pair_scalars *__restrict__ ps)
{
  constexpr int D = K / 2;
  if ( *reinterpret_cast< const volatile int * >( &ssc->error ) == kErrTimeout ) return;  // keys not sorted
  const sweep_params p = *pp;
  const double W = ord_decode( p.wmax_enc );
  const uint64_t wq = W < 8589934592.0 ? static_cast< uint64_t >( ceil( W ) ) : 8589934592ull;  // >= every key span
  const unsigned lane = threadIdx.x & 31u;
  const uint64_t nwarps = static_cast< uint64_t >( gridDim.x ) * ( kSweepThreads / 32 );
  for ( uint64_t t = ( static_cast< uint64_t >( blockIdx.x ) * kSweepThreads + threadIdx.x ) >> 5; t < na; t += nwarps )
  {
    const uint32_t i = __ldg( aperm + t );
    double lo[D], hi[D];
    leaf_slabs< K, double, VT >( verts, Vrt, i, eps, 0.f, lo, hi );
    const double mn = p.axis == 0 ? lo[0] : ( p.axis == 1 ? lo[1] : lo[2] );
    const double mx = p.axis == 0 ? hi[0] : ( p.axis == 1 ? hi[1] : hi[2] );
    const uint32_t amin = key32( scaled( mn, p ) );
    const uint32_t amax = key32( scaled( mx, p ) );
    const uint64_t start = amin > wq ? amin - wq : 0;
    const uint64_t j0 = key_bound( skeys, nb, start, false );
    const uint64_t j1 = key_bound( skeys, nb, amax, true );
    const double amin_d = static_cast< double >( amin );
    for ( uint64_t j = j0 + lane; j < j1; j += 32 )
    {
      if ( __ldg( sbmax + j ) < amin_d ) continue;
      const double *row = srows + j * 2 * D;
      bool o = true;
#pragma unroll
      for ( int a = 0; a < D; ++a )
      {
        if ( !o ) break;
        o = lo[a] < __ldg( row + 2 * a + 1 ) && __ldg( row + 2 * a ) < hi[a];
      }
      if ( o )
      {
        const unsigned long long pos = atomicAdd( &ps->count, 1ull );
        if ( pos < cap ) pairs[pos] = make_uint2( i, __ldg( svals + j ) );
      }
    }
  }
}

template< int K, int VT >
void sweep_kernels(const sweep_launch &x, cudaError_t &e, bool keys_phase)
{
  const sweep_params *pp = static_cast< const sweep_params * >( x.params );
  if ( keys_phase )
  {
    const unsigned grid = static_cast< unsigned >( ( x.nb + kSweepThreads - 1 ) / kSweepThreads );
    k_sweep_keys< K, VT ><<< grid, kSweepThreads, 0, x.s >>>( x.bverts, x.bV, x.nb, x.eps, pp, x.rows, x.keys, x.hist,
                                                             static_cast< sweep_params * >( x.params ) );
  } else {
    // warps grid-stride over A: at most 16 resident blocks' worth per SM, never more warps than elements
    const uint64_t want = ( x.na + kSweepThreads / 32 - 1 ) / ( kSweepThreads / 32 );
    const uint64_t cap = static_cast< uint64_t >( device_sm_count() ) * 16;
    const unsigned grid = static_cast< unsigned >( want < cap ? want : cap );
    const unsigned ggrid = static_cast< unsigned >( device_sm_count() ) * 8;
    k_sweep_gather< K ><<< ggrid, kSweepThreads, 0, x.s >>>( x.rows, x.svals, x.nb, pp, x.srows, x.sbmax );
    e = cudaGetLastError();
    if ( e != cudaSuccess ) return;
    k_sweep< K, VT ><<< grid, kSweepThreads, 0, x.s >>>( x.averts, x.aV, x.na, x.eps, pp, x.aperm, x.skeys, x.svals,
                                                        x.srows, x.sbmax, x.nb, x.sc, x.pairs, x.cap, x.ps );
  }
  e = cudaGetLastError();
}

template< int K >
void sweep_v(const sweep_launch &x, cudaError_t &e, bool keys_phase)
{
  const uint32_t V = keys_phase ? x.bV : x.aV;
  switch ( V )
  {
    case 3: sweep_kernels< K, 3 >( x, e, keys_phase ); break;
    case 4: sweep_kernels< K, 4 >( x, e, keys_phase ); break;
    case 8: sweep_kernels< K, 8 >( x, e, keys_phase ); break;
    default: sweep_kernels< K, 0 >( x, e, keys_phase ); break;
  }
}

cudaError_t sweep_phase(const sweep_launch &x, bool keys_phase)
{
  cudaError_t e = cudaErrorInvalidValue;
  switch ( x.K )
  {
    case 6: sweep_v< 6 >( x, e, keys_phase ); break;
    case 18: sweep_v< 18 >( x, e, keys_phase ); break;
    case 26: sweep_v< 26 >( x, e, keys_phase ); break;
    default: break;
  }
  return e;
}

}  // namespace

size_t sweep_params_bytes() { return sizeof( sweep_params ); }
size_t sweep_partial_bytes() { return static_cast< size_t >( kAxisBlocks ) * 6 * sizeof( double ); }

int sweep_axis_read(const void *params_host_copy) { return static_cast< const sweep_params * >( params_host_copy )->axis; }

cudaError_t launch_sweep_setup(const sweep_launch &x, int axis)
{
  if ( axis < 0 )
  {
    k_axis_partial<<< kAxisBlocks, kSweepThreads, 0, x.s >>>( x.acx, x.acy, x.acz, x.na, x.bcx, x.bcy, x.bcz, x.nb,
                                                             x.partial );
    cudaError_t e = cudaGetLastError();
    if ( e != cudaSuccess ) return e;
  }
  k_sweep_setup<<< 1, 32, 0, x.s >>>( x.partial, kAxisBlocks, x.na + x.nb, axis, x.asc, x.bsc,
                                      static_cast< sweep_params * >( x.params ) );
  return cudaGetLastError();
}

cudaError_t launch_sweep_keys(const sweep_launch &x) { return sweep_phase( x, true ); }
cudaError_t launch_sweep(const sweep_launch &x) { return sweep_phase( x, false ); }

}  // namespace bvhg
