// k_cluster.cu — the reference's Morton clustering of an object into patches, and the grouping of exact element
// pairs by patch pair, on the device.
//
// morton_cluster (src/bvh/split/cluster.hpp:89-179) orders the elements stably by their 32-bit Morton hash, takes
// the split depth of every neighbouring pair (31 - floor(log2(h_i ^ h_{i+1})), or all ones for equal hashes), sorts
// the positions by depth (stably: ties keep position order) and cuts at the first od_factor - 1 of them, in
// position order; patch k then spans positions [split[k - 1], split[k]) of that order
// (src/bvh/collision_object.cpp:134-141). Here:
//   - The 32-bit hash of an element is its 63-bit Morton key shifted right by 33 (quantize32 keeps the top 10 of
//     the 21 bits per axis that quantize64 keeps, and the interleave puts them at bits 33..62). The build's sorted
//     keys are ordered by hash already; only equal-hash runs need their elements in index order (k_cluster_fix for
//     runs of up to 32, k_cluster_runs beyond).
//   - A depth is one of 33 values (0..31 and "equal"), so the selection needs no sort: a histogram of the depths
//     gives the threshold depth t and how many positions of depth t to take (the first ones in position order);
//     a stable block-scan compaction then writes the chosen positions in order.
// Every kernel is a bounded loop; nothing waits on another block.
#include "bvhg_internal.cuh"
#include "kdop_math.cuh"

namespace bvhg {
int device_sm_count();
namespace {

constexpr int kClThreads = 512;
constexpr int kClItems = 8;
constexpr int kClTile = kClThreads * kClItems;  // positions per block of the depth kernels
constexpr int kClRun = 32;                      // equal-hash runs ranked in place up to this length
constexpr int kClRunSmem = 2048;                // longer runs sorted in shared memory up to this length
constexpr int kDepthBins = 33;                  // depths 0..31, then "equal hashes"

__device__ __forceinline__ uint32_t hash_of(uint64_t key) { return static_cast< uint32_t >( key >> 33 ); }

// Depth of the split between positions i and i + 1 (bin 32 stands for the reference's all-ones value).
__device__ __forceinline__ uint32_t depth_at(const uint64_t *__restrict__ keys, uint32_t i)
{
  const uint32_t m = hash_of( __ldg( keys + i ) ) ^ hash_of( __ldg( keys + i + 1 ) );
  return m ? static_cast< uint32_t >( __clz( m ) ) : 32u;
}

// Exclusive scan of one value per thread over a block of kClThreads threads.
__device__ __forceinline__ uint32_t cl_block_scan(uint32_t x, uint32_t *s_warp, uint32_t *total)
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
  uint32_t pre = 0, tot = 0;
#pragma unroll
  for ( int k = 0; k < kClThreads / 32; ++k )
  {
    const uint32_t v = s_warp[k];
    if ( k < w ) pre += v;
    tot += v;
  }
  __syncthreads();
  if ( total ) *total = tot;
  return pre + inc - x;
}

// Elements of each run of equal hashes in index order (out of place): a run of up to kClRun elements is ranked
// from the neighbours; a longer one is copied in order and its first position listed for k_cluster_runs.
__global__ void __launch_bounds__( 256 ) k_cluster_fix(const uint64_t *__restrict__ keys,
                                                       const uint32_t *__restrict__ perm, uint32_t n,
                                                       uint32_t *__restrict__ order, uint32_t *__restrict__ runs,
                                                       cluster_scalars *cs)
{
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if ( i >= n ) return;
  const uint32_t h = hash_of( keys[i] );
  const uint32_t v = perm[i];
  uint32_t s = i, e = i;
  bool limit = false;
  while ( s > 0 && hash_of( __ldg( keys + s - 1 ) ) == h )
  {
    --s;
    if ( i - s >= kClRun )
    {
      limit = true;
      break;
    }
  }
  while ( !limit && e + 1 < n && hash_of( __ldg( keys + e + 1 ) ) == h )
  {
    ++e;
    if ( e - i >= kClRun )
    {
      limit = true;
      break;
    }
  }
  uint32_t pos = i;
  if ( limit || e - s + 1 > kClRun )
  {
    if ( s == i ) runs[atomicAdd( &cs->runs, 1u )] = i;
  } else if ( e > s ) {
    uint32_t rank = 0;
    for ( uint32_t j = s; j <= e; ++j ) rank += __ldg( perm + j ) < v ? 1u : 0u;
    pos = s + rank;
  }
  order[pos] = v;
}

// Sorts the element indices of every listed run (in place in `order`, `tmp` as scratch): a bitonic network in
// shared memory up to kClRunSmem elements, four stable 8-bit LSD passes beyond (ending back in `order`).
__global__ void __launch_bounds__( kClThreads ) k_cluster_runs(const uint64_t *__restrict__ keys, uint32_t n,
                                                               uint32_t *__restrict__ order, uint32_t *__restrict__ tmp,
                                                               const uint32_t *__restrict__ runs,
                                                               const cluster_scalars *cs)
{
  constexpr int W = kClThreads / 32;
  __shared__ __align__( 16 ) uint32_t s_raw[W * 256 + 3 * 256 + 4 * 256];  // >= kClRunSmem words as well
  __shared__ uint32_t s_warp[W];
  __shared__ uint32_t s_start, s_len;
  static_assert( W * 256 + 3 * 256 + 4 * 256 >= kClRunSmem, "shared memory too small for the bitonic runs" );
  const uint32_t nruns = *reinterpret_cast< const volatile unsigned int * >( &cs->runs );
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const unsigned lt_mask = ( 1u << lane ) - 1u;
  for ( uint32_t r = blockIdx.x; r < nruns; r += gridDim.x )
  {
    if ( tid == 0 )
    {
      const uint32_t s = runs[r];
      const uint32_t h = hash_of( keys[s] );
      uint32_t lo = s + 1, up = n;
      while ( lo < up )
      {
        const uint32_t mid = lo + ( up - lo ) / 2;
        if ( hash_of( keys[mid] ) == h ) lo = mid + 1;
        else up = mid;
      }
      s_start = s;
      s_len = lo - s;
    }
    __syncthreads();
    const uint32_t s = s_start, L = s_len;
    if ( L <= kClRunSmem )
    {
      uint32_t *c = s_raw;
      uint32_t P = 1;
      while ( P < L ) P <<= 1;
      for ( uint32_t j = tid; j < P; j += kClThreads ) c[j] = j < L ? order[s + j] : 0xffffffffu;
      __syncthreads();
      for ( uint32_t k = 2; k <= P; k <<= 1 )
        for ( uint32_t j = k >> 1; j > 0; j >>= 1 )
        {
          for ( uint32_t t = tid; t < P; t += kClThreads )
          {
            const uint32_t u = t ^ j;
            if ( u > t )
            {
              const uint32_t a = c[t], b = c[u];
              if ( ( a > b ) == ( ( t & k ) == 0 ) )
              {
                c[t] = b;
                c[u] = a;
              }
            }
          }
          __syncthreads();
        }
      for ( uint32_t j = tid; j < L; j += kClThreads ) order[s + j] = c[j];
    } else {
      uint32_t( *cnt )[256] = reinterpret_cast< uint32_t( * )[256] >( s_raw );
      uint32_t *run_off = s_raw + W * 256, *tot = run_off + 256, *unused = tot + 256;
      uint32_t( *hist )[256] = reinterpret_cast< uint32_t( * )[256] >( unused + 256 );
      for ( int q = tid; q < W * 256; q += kClThreads ) ( &cnt[0][0] )[q] = 0;
      for ( int q = tid; q < 4 * 256; q += kClThreads ) ( &hist[0][0] )[q] = 0;
      __syncthreads();
      for ( uint32_t j = tid; j < L; j += kClThreads )
      {
        const uint32_t v = order[s + j];
#pragma unroll
        for ( int p = 0; p < 4; ++p ) atomicAdd( &hist[p][( v >> ( 8 * p ) ) & 255u], 1u );
      }
      __syncthreads();
      uint32_t *src = order, *dst = tmp;
      for ( int p = 0; p < 4; ++p )
      {
        const uint32_t ex = cl_block_scan( tid < 256 ? hist[p][tid] : 0u, s_warp, nullptr );
        if ( tid < 256 ) run_off[tid] = ex;
        __syncthreads();
        for ( uint32_t base = 0; base < L; base += kClThreads )
        {
          const uint32_t j = base + tid;
          const bool valid = j < L;
          const uint32_t v = valid ? src[s + j] : 0u;
          const uint32_t d = valid ? ( v >> ( 8 * p ) ) & 255u : 256u;
          const unsigned peers = __match_any_sync( 0xffffffffu, d );
          const uint32_t rank = __popc( peers & lt_mask );
          if ( valid && lane == __ffs( peers ) - 1 ) cnt[warp][d] = __popc( peers );
          __syncthreads();
          if ( tid < 256 )
          {
            uint32_t t = 0;
#pragma unroll
            for ( int w = 0; w < W; ++w )
            {
              const uint32_t cv = cnt[w][tid];
              cnt[w][tid] = t;
              t += cv;
            }
            tot[tid] = t;
          }
          __syncthreads();
          if ( valid ) dst[s + run_off[d] + cnt[warp][d] + rank] = v;
          __syncthreads();
          if ( tid < 256 )
          {
            run_off[tid] += tot[tid];
#pragma unroll
            for ( int w = 0; w < W; ++w ) cnt[w][tid] = 0;
          }
          __syncthreads();
        }
        uint32_t *t2 = src;
        src = dst;
        dst = t2;
      }
    }
    __syncthreads();
  }
}

// Per block of kClTile positions i < n - 1: the histogram of the split depths (row b of bhist, kDepthBins words).
__global__ void __launch_bounds__( kClThreads ) k_cluster_depths(const uint64_t *__restrict__ keys, uint32_t n,
                                                                 uint32_t *__restrict__ bhist)
{
  __shared__ uint32_t s_h[kDepthBins];
  if ( threadIdx.x < kDepthBins ) s_h[threadIdx.x] = 0;
  __syncthreads();
  const uint32_t b0 = blockIdx.x * kClTile;
  for ( uint32_t k = threadIdx.x; k < kClTile; k += kClThreads )
  {
    const uint32_t i = b0 + k;
    if ( i + 1 < n ) atomicAdd( &s_h[depth_at( keys, i )], 1u );
  }
  __syncthreads();
  if ( threadIdx.x < kDepthBins ) bhist[blockIdx.x * kDepthBins + threadIdx.x] = s_h[threadIdx.x];
}

// One block: the threshold depth t, how many positions of depth t are taken (need), and per block of positions the
// number of chosen positions before it (bbase[2 b]) and of depth-t positions before it (bbase[2 b + 1]).
__global__ void __launch_bounds__( kClThreads ) k_cluster_select(const uint32_t *__restrict__ bhist, uint32_t nblocks,
                                                                 uint32_t take, uint32_t *__restrict__ bbase,
                                                                 cluster_scalars *cs)
{
  __shared__ uint32_t s_h[kDepthBins];
  __shared__ uint32_t s_warp[kClThreads / 32];
  __shared__ uint32_t s_t, s_need;
  if ( threadIdx.x < kDepthBins ) s_h[threadIdx.x] = 0;
  __syncthreads();
  for ( uint32_t b = threadIdx.x; b < nblocks; b += kClThreads )
    for ( int d = 0; d < kDepthBins; ++d )
    {
      const uint32_t c = bhist[b * kDepthBins + d];
      if ( c ) atomicAdd( &s_h[d], c );
    }
  __syncthreads();
  if ( threadIdx.x == 0 )
  {
    uint32_t cum = 0, t = kDepthBins - 1, need = 0;
    for ( int d = 0; d < kDepthBins; ++d )
    {
      if ( cum + s_h[d] >= take )
      {
        t = static_cast< uint32_t >( d );
        need = take - cum;
        break;
      }
      cum += s_h[d];
    }
    s_t = t;
    s_need = need;
    cs->t = t;
    cs->need = need;
  }
  __syncthreads();
  const uint32_t t = s_t, need = s_need;
  uint32_t chosen_before = 0, eq_before = 0;
  for ( uint32_t b0 = 0; b0 < nblocks; b0 += kClThreads )
  {
    const uint32_t b = b0 + threadIdx.x;
    uint32_t lt = 0, eq = 0;
    if ( b < nblocks )
    {
      for ( uint32_t d = 0; d < t; ++d ) lt += bhist[b * kDepthBins + d];
      eq = bhist[b * kDepthBins + t];
    }
    uint32_t eq_tot = 0;
    const uint32_t eq_ex = cl_block_scan( eq, s_warp, &eq_tot ) + eq_before;
    // depth-t positions of this block that are taken: those whose rank among all depth-t positions is below need
    const uint32_t ties = eq_ex >= need ? 0u : min( eq, need - eq_ex );
    uint32_t ch_tot = 0;
    const uint32_t ch_ex = cl_block_scan( lt + ties, s_warp, &ch_tot ) + chosen_before;
    if ( b < nblocks )
    {
      bbase[2 * b] = ch_ex;
      bbase[2 * b + 1] = eq_ex;
    }
    chosen_before += ch_tot;
    eq_before += eq_tot;
  }
}

// Per block of positions: the chosen split positions (depth < t, or depth t among the first `need` of them), written
// in position order to splits[bbase[2 b] + their rank in the block].
__global__ void __launch_bounds__( kClThreads ) k_cluster_emit(const uint64_t *__restrict__ keys, uint32_t n,
                                                               const uint32_t *__restrict__ bbase,
                                                               const cluster_scalars *cs, uint32_t *__restrict__ splits)
{
  __shared__ uint32_t s_warp[kClThreads / 32];
  const uint32_t t = cs->t, need = cs->need;
  const uint32_t i0 = blockIdx.x * kClTile + threadIdx.x * kClItems;
  uint32_t d[kClItems];
  uint32_t eq = 0;
#pragma unroll
  for ( int k = 0; k < kClItems; ++k )
  {
    const uint32_t i = i0 + k;
    d[k] = i + 1 < n ? depth_at( keys, i ) : 0xffffffffu;
    eq += d[k] == t ? 1u : 0u;
  }
  uint32_t eq_rank = cl_block_scan( eq, s_warp, nullptr ) + bbase[2 * blockIdx.x + 1];
  uint32_t chosen = 0;
  uint32_t pick = 0;  // bit k: position i0 + k is a split
#pragma unroll
  for ( int k = 0; k < kClItems; ++k )
  {
    bool c = d[k] < t;
    if ( d[k] == t )
    {
      c = eq_rank < need;
      ++eq_rank;
    }
    if ( c )
    {
      pick |= 1u << k;
      ++chosen;
    }
  }
  uint32_t pos = cl_block_scan( chosen, s_warp, nullptr ) + bbase[2 * blockIdx.x];
#pragma unroll
  for ( int k = 0; k < kClItems; ++k )
    if ( ( pick >> k ) & 1u ) splits[pos++] = i0 + k;
}

// Patch boundaries: bounds[0] = 0, bounds[k] = split k - 1 (positions past the chosen ones: n - 1, as the
// reference fills splits it cannot choose), bounds[P] = n; and the inverse of the order (rank of every element).
__global__ void k_cluster_bounds(const uint32_t *__restrict__ splits, uint32_t take, uint32_t patches, uint32_t n,
                                 uint64_t *__restrict__ bounds)
{
  for ( uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k <= patches; k += gridDim.x * blockDim.x )
  {
    uint64_t v;
    if ( k == 0 ) v = 0;
    else if ( k == patches ) v = n;
    else v = k - 1 < take ? splits[k - 1] : ( n > 0 ? n - 1 : 0 );
    bounds[k] = v;
  }
}

__global__ void k_cluster_rank(const uint32_t *__restrict__ order, uint32_t n, uint32_t *__restrict__ rank)
{
  for ( uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x ) rank[order[r]] = r;
}

// ---- element pairs grouped by patch pair -----------------------------------------------------------------------

// Patch of a position: the last k with bounds[k] <= r (bounds ascending, bounds[0] = 0).
__device__ __forceinline__ uint32_t patch_of(const uint64_t *__restrict__ bounds, uint32_t patches, uint32_t r)
{
  uint32_t lo = 0, hi = patches - 1;
  while ( lo < hi )
  {
    const uint32_t mid = ( lo + hi + 1 ) >> 1;
    if ( __ldg( bounds + mid ) <= r ) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__global__ void k_group_count(const uint2 *__restrict__ pairs, uint64_t np, group_launch g,
                              uint32_t *__restrict__ bin_count)
{
  for ( uint64_t p = static_cast< uint64_t >( blockIdx.x ) * blockDim.x + threadIdx.x; p < np;
        p += static_cast< uint64_t >( gridDim.x ) * blockDim.x )
  {
    const uint2 c = pairs[p];
    const uint32_t pa = patch_of( g.bounds_a, g.patches_a, __ldg( g.rank_a + c.x ) );
    const uint32_t pb = patch_of( g.bounds_b, g.patches_b, __ldg( g.rank_b + c.y ) );
    atomicAdd( bin_count + static_cast< uint64_t >( pa ) * g.patches_b + pb, 1u );
  }
}

// One block: exclusive offsets of the bins (in bin order) into bin_off, and the table of non-empty bins as
// (patch a, patch b, first pair, pair count) rows; the number of rows in cs->groups.
__global__ void __launch_bounds__( kClThreads ) k_group_scan(const uint32_t *__restrict__ bin_count, uint64_t bins,
                                                             uint32_t patches_b, uint32_t *__restrict__ bin_off,
                                                             uint32_t *__restrict__ groups, uint64_t group_cap,
                                                             cluster_scalars *cs)
{
  __shared__ uint32_t s_warp[kClThreads / 32];
  uint32_t off = 0, rows = 0;
  for ( uint64_t b0 = 0; b0 < bins; b0 += kClThreads )
  {
    const uint64_t b = b0 + threadIdx.x;
    const uint32_t c = b < bins ? bin_count[b] : 0u;
    uint32_t tot = 0, rtot = 0;
    const uint32_t ex = cl_block_scan( c, s_warp, &tot ) + off;
    const uint32_t rex = cl_block_scan( c ? 1u : 0u, s_warp, &rtot ) + rows;
    if ( b < bins )
    {
      bin_off[b] = ex;
      if ( c && rex < group_cap )
      {
        groups[4 * static_cast< uint64_t >( rex )] = static_cast< uint32_t >( b / patches_b );
        groups[4 * static_cast< uint64_t >( rex ) + 1] = static_cast< uint32_t >( b % patches_b );
        groups[4 * static_cast< uint64_t >( rex ) + 2] = ex;
        groups[4 * static_cast< uint64_t >( rex ) + 3] = c;
      }
    }
    off += tot;
    rows += rtot;
  }
  if ( threadIdx.x == 0 ) cs->groups = rows;
}

// Every pair to its bin's slot: (index in patch a, index in patch b); the order within a bin is unspecified.
__global__ void k_group_scatter(const uint2 *__restrict__ pairs, uint64_t np, group_launch g,
                                uint32_t *__restrict__ bin_fill, const uint32_t *__restrict__ bin_off,
                                uint32_t *__restrict__ out)
{
  for ( uint64_t p = static_cast< uint64_t >( blockIdx.x ) * blockDim.x + threadIdx.x; p < np;
        p += static_cast< uint64_t >( gridDim.x ) * blockDim.x )
  {
    const uint2 c = pairs[p];
    const uint32_t ra = __ldg( g.rank_a + c.x ), rb = __ldg( g.rank_b + c.y );
    const uint32_t pa = patch_of( g.bounds_a, g.patches_a, ra );
    const uint32_t pb = patch_of( g.bounds_b, g.patches_b, rb );
    const uint64_t bin = static_cast< uint64_t >( pa ) * g.patches_b + pb;
    const uint64_t slot = static_cast< uint64_t >( __ldg( bin_off + bin ) ) + atomicAdd( bin_fill + bin, 1u );
    out[2 * slot] = ra - static_cast< uint32_t >( __ldg( g.bounds_a + pa ) );
    out[2 * slot + 1] = rb - static_cast< uint32_t >( __ldg( g.bounds_b + pb ) );
  }
}

// ---- patch k-DOPs ----------------------------------------------------------------------------------------------

// Patch boxes: the union of the FP64 slabs (kdop_base::from_vertices, src/bvh/kdop.hpp:238-264) of every element of
// each patch, as the reference's patch snapshot unions its elements' k-DOPs (make_snapshot,
// src/bvh/snapshot.hpp:139-149). One thread per position of the patch order; a warp whose positions all lie in one
// patch reduces in registers and updates the patch's order-preserving encodings once per slab, other warps per lane.
template< int K, int VT >
__global__ void __launch_bounds__( 256 ) k_patch_kdops(const double *__restrict__ verts, uint32_t Vrt, uint32_t n,
                                                       double eps, const uint32_t *__restrict__ order,
                                                       const uint64_t *__restrict__ bounds, uint32_t patches,
                                                       unsigned long long *__restrict__ enc)
{
  constexpr int D = K / 2;
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned lane = threadIdx.x & 31u;
  const bool valid = r < n;
  const uint32_t p = valid ? patch_of( bounds, patches, r ) : 0xffffffffu;
  const uint32_t p0 = __shfl_sync( 0xffffffffu, p, 0 );
  const bool uniform = __all_sync( 0xffffffffu, valid && p == p0 );
  double lo[D], hi[D];
  if ( valid ) leaf_slabs< K, double, VT >( verts, Vrt, __ldg( order + r ), eps, 0.f, lo, hi );
#pragma unroll
  for ( int a = 0; a < D; ++a )
  {
    unsigned long long emin = valid ? ord_encode( lo[a] ) : ~0ull, emax = valid ? ord_encode( hi[a] ) : 0ull;
    if ( uniform )
    {
#pragma unroll
      for ( int o = 16; o > 0; o >>= 1 )
      {
        const unsigned long long om = __shfl_xor_sync( 0xffffffffu, emin, o );
        const unsigned long long oM = __shfl_xor_sync( 0xffffffffu, emax, o );
        emin = om < emin ? om : emin;
        emax = oM > emax ? oM : emax;
      }
      if ( lane == 0 )
      {
        atomicMin( enc + ( static_cast< size_t >( p0 ) * D + a ) * 2, emin );
        atomicMax( enc + ( static_cast< size_t >( p0 ) * D + a ) * 2 + 1, emax );
      }
    } else if ( valid ) {
      atomicMin( enc + ( static_cast< size_t >( p ) * D + a ) * 2, emin );
      atomicMax( enc + ( static_cast< size_t >( p ) * D + a ) * 2 + 1, emax );
    }
  }
}

__global__ void k_patch_kdops_init(unsigned long long *enc, uint64_t words)
{
  for ( uint64_t i = static_cast< uint64_t >( blockIdx.x ) * blockDim.x + threadIdx.x; i < words;
        i += static_cast< uint64_t >( gridDim.x ) * blockDim.x )
    enc[i] = ( i & 1 ) ? 0ull : ~0ull;
}

// Decoded boxes; an empty patch gets (+inf, -inf) on every slab.
__global__ void k_patch_kdops_decode(const unsigned long long *__restrict__ enc, uint64_t words, double *__restrict__ out)
{
  for ( uint64_t i = static_cast< uint64_t >( blockIdx.x ) * blockDim.x + threadIdx.x; i < words;
        i += static_cast< uint64_t >( gridDim.x ) * blockDim.x )
  {
    const unsigned long long e = enc[i];
    const bool untouched = ( i & 1 ) ? e == 0ull : e == ~0ull;
    out[i] = untouched ? ( ( i & 1 ) ? -__longlong_as_double( 0x7ff0000000000000LL ) : __longlong_as_double( 0x7ff0000000000000LL ) )
                       : ord_decode( e );
  }
}

unsigned grid_for(uint64_t work, unsigned threads, unsigned per_sm)
{
  const uint64_t blocks = ( work + threads - 1 ) / threads;
  const uint64_t cap = static_cast< uint64_t >( device_sm_count() ) * per_sm;
  return static_cast< unsigned >( blocks < cap ? ( blocks ? blocks : 1 ) : cap );
}

}  // namespace

size_t cluster_block_count(uint64_t n) { return static_cast< size_t >( ( n + kClTile - 1 ) / kClTile ); }

cudaError_t launch_cluster(const cluster_launch &x)
{
  if ( x.n == 0 )
  {
    k_cluster_bounds<<< 1, 256, 0, x.s >>>( x.splits, 0, x.patches, 0, x.bounds );
    return cudaGetLastError();
  }
  const uint32_t n = static_cast< uint32_t >( x.n );
  cudaError_t e = cudaMemsetAsync( x.cs, 0, sizeof( cluster_scalars ), x.s );
  if ( e != cudaSuccess ) return e;
  k_cluster_fix<<< ( n + 255 ) / 256, 256, 0, x.s >>>( x.keys, x.perm, n, x.order, x.runs, x.cs );
  if ( n > static_cast< uint32_t >( kClRun ) )
  {
    const uint64_t most = n / ( kClRun + 1 ) + 1;
    const uint64_t cap = static_cast< uint64_t >( device_sm_count() );
    k_cluster_runs<<< static_cast< unsigned >( most < cap ? most : cap ), kClThreads, 0, x.s >>>( x.keys, n, x.order, x.tmp,
                                                                                                 x.runs, x.cs );
  }
  const uint32_t take = x.patches - 1 < n - 1 ? x.patches - 1 : n - 1;
  if ( take > 0 )
  {
    const uint32_t nb = static_cast< uint32_t >( cluster_block_count( n ) );
    k_cluster_depths<<< nb, kClThreads, 0, x.s >>>( x.keys, n, x.bhist );
    k_cluster_select<<< 1, kClThreads, 0, x.s >>>( x.bhist, nb, take, x.bbase, x.cs );
    k_cluster_emit<<< nb, kClThreads, 0, x.s >>>( x.keys, n, x.bbase, x.cs, x.splits );
  }
  k_cluster_bounds<<< 1, 256, 0, x.s >>>( x.splits, take, x.patches, n, x.bounds );
  k_cluster_rank<<< grid_for( n, 256, 8 ), 256, 0, x.s >>>( x.order, n, x.rank );
  return cudaGetLastError();
}

cudaError_t launch_patch_kdops(int K, const double *verts, uint32_t V, uint64_t n, double eps, const uint32_t *order,
                               const uint64_t *bounds, uint32_t patches, unsigned long long *enc, double *out,
                               cudaStream_t s)
{
  const uint64_t words = static_cast< uint64_t >( patches ) * K;
  k_patch_kdops_init<<< grid_for( words, 256, 4 ), 256, 0, s >>>( enc, words );
  if ( n > 0 )
  {
    const unsigned grid = static_cast< unsigned >( ( n + 255 ) / 256 );
    const uint32_t n32 = static_cast< uint32_t >( n );
#define BVHG_PK( KK, VV ) k_patch_kdops< KK, VV ><<< grid, 256, 0, s >>>( verts, V, n32, eps, order, bounds, patches, enc )
    if ( K == 6 ) { if ( V == 3 ) BVHG_PK( 6, 3 ); else if ( V == 4 ) BVHG_PK( 6, 4 ); else if ( V == 8 ) BVHG_PK( 6, 8 ); else BVHG_PK( 6, 0 ); }
    else if ( K == 18 ) { if ( V == 3 ) BVHG_PK( 18, 3 ); else if ( V == 4 ) BVHG_PK( 18, 4 ); else if ( V == 8 ) BVHG_PK( 18, 8 ); else BVHG_PK( 18, 0 ); }
    else if ( K == 26 ) { if ( V == 3 ) BVHG_PK( 26, 3 ); else if ( V == 4 ) BVHG_PK( 26, 4 ); else if ( V == 8 ) BVHG_PK( 26, 8 ); else BVHG_PK( 26, 0 ); }
    else return cudaErrorInvalidValue;
#undef BVHG_PK
  }
  k_patch_kdops_decode<<< grid_for( words, 256, 4 ), 256, 0, s >>>( enc, words, out );
  return cudaGetLastError();
}

cudaError_t launch_group_pairs(const uint2 *pairs, uint64_t np, const group_launch &g, uint32_t *bin_count,
                               uint32_t *bin_off, uint32_t *groups, uint64_t group_cap, uint32_t *out,
                               cluster_scalars *cs, cudaStream_t s)
{
  const uint64_t bins = static_cast< uint64_t >( g.patches_a ) * g.patches_b;
  cudaError_t e = cudaMemsetAsync( bin_count, 0, bins * sizeof( uint32_t ), s );
  if ( e != cudaSuccess ) return e;
  const unsigned grid = grid_for( np, 256, 8 );
  if ( np ) k_group_count<<< grid, 256, 0, s >>>( pairs, np, g, bin_count );
  k_group_scan<<< 1, kClThreads, 0, s >>>( bin_count, bins, g.patches_b, bin_off, groups, group_cap, cs );
  e = cudaMemsetAsync( bin_count, 0, bins * sizeof( uint32_t ), s );  // reused as the fill counters
  if ( e != cudaSuccess ) return e;
  if ( np ) k_group_scatter<<< grid, 256, 0, s >>>( pairs, np, g, bin_count, bin_off, out );
  return cudaGetLastError();
}

}  // namespace bvhg
