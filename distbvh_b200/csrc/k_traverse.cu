// k_traverse.cu — tree traversal emitting candidate element pairs (K6), FP64 recheck (K7), gid output.
//
// The reference finds pairs with a 4-way simultaneous recursion over two trees (get_overlapping_indices,
// src/bvh/collision_query.hpp:293-329) or a per-entity descent (query_tree, collision_query.hpp:166-213), both
// pruning on the strict all-slab overlap (kdop.hpp:120-125, 538-549). Here a warp walks the other object's tree
// for a packet of 32 consecutive query ranks (Morton order: spatially coherent), one query per lane, with a stack
// of (node, lane mask) entries: both children of a node are tested from one row holding their slabs (one 32-byte
// FP64 / 16-byte FP32 sector per slab, loaded a chunk of slabs at a time), and a child is entered with the mask of
// the lanes that overlap it. At a leaf bucket each lane of the mask tests its query against the bucket's
// elements. Overlaps are emitted as (query element, tree element) local indices: through one warp-aggregated
// reservation per bucket visit in sparse contact, through a per-warp buffer in shared memory in dense contact;
// pairs beyond capacity are counted but not stored, so the host can grow the buffer and retry. In sparse contact
// the grid is persistent and culls 32 packets per warp step against the target root before walking the
// survivors; in dense contact it is one warp per packet. The FP64 recheck of the precision form reads both
// elements' vertices per candidate and decides the overlap by comparison-only projections (kdop_math.cuh).
//
// Self-collision (self_collision_set, collision_query.hpp:331-368): the query of rank i only visits subtrees
// holding ranks > i (internal node k splits its bucket range [l, r] into [l, k] and [k + 1, r]) and tests only
// bucket elements of rank > i, so every unordered pair is found once and no element is paired with itself.
#include <cstddef>

#include "bulk_copy.cuh"
#include "bvhg_internal.cuh"
#include "kdop_math.cuh"

namespace bvhg {
int device_sm_count();
namespace {

constexpr int kTravThreads = 128;
constexpr int kStack = 96;  // radix tree over 96-bit (key, rank) pairs: at most 95 internal levels

template< typename T >
struct slab_pair;

// Both children's (min, max) of one slab.
template<>
struct slab_pair< double >
{
  double min0, max0, min1, max1;
  __device__ static slab_pair load(const double *p)
  {
    const double2 a = __ldg( reinterpret_cast< const double2 * >( p ) );
    const double2 b = __ldg( reinterpret_cast< const double2 * >( p ) + 1 );
    return { a.x, a.y, b.x, b.y };
  }
};

template<>
struct slab_pair< float >
{
  float min0, max0, min1, max1;
  __device__ static slab_pair load(const float *p)
  {
    const float4 a = __ldg( reinterpret_cast< const float4 * >( p ) );
    return { a.x, a.y, a.z, a.w };
  }
};

// Axes of a node row loaded together in the walk (a chunk of loads in flight per round trip; bounded by registers).
template< int K, typename T >
constexpr int kNodeChunk = ( K / 2 ) <= 4 ? K / 2 : ( sizeof( T ) == 4 ? ( K / 2 + 1 ) / 2 : 5 );

// Resident blocks per SM of the single-node walk, which computes the element slabs it tests (128 registers).
constexpr int kTravBlocksPerSM = 4;

// Slots for k outputs of each calling lane, one atomic per group of converged lanes: the lanes' exclusive prefix of
// k is formed from one ballot per bit of k (k < 64), the lowest lane reserves the group's total.
__device__ __forceinline__ unsigned long long warp_reserve(unsigned k, unsigned long long *counter)
{
  const unsigned active = __activemask();
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lt = ( 1u << lane ) - 1u;
  unsigned pre = 0, tot = 0;
#pragma unroll
  for ( int bit = 0; bit < 6; ++bit )
  {
    const unsigned bal = __ballot_sync( active, ( k >> bit ) & 1u );
    pre += static_cast< unsigned >( __popc( bal & lt ) ) << bit;
    tot += static_cast< unsigned >( __popc( bal ) ) << bit;
  }
  const int leader = __ffs( active ) - 1;
  unsigned long long base = 0;
  if ( static_cast< int >( lane ) == leader && tot ) base = atomicAdd( counter, static_cast< unsigned long long >( tot ) );
  base = __shfl_sync( active, base, leader );
  return base + pre;
}

// Slabs of element e straight into a shared-memory row (C = 2 D values: min, max per slab): the same FP64 slabs
// (slab by slab, so that only the vertices stay in registers), or the same FP32 enclosures, that slabs_body
// unites into the bucket boxes.
template< int K, typename T, int VT >
__device__ __forceinline__ void slabs_to_row(const double *__restrict__ verts, uint32_t Vrt, uint32_t e, double eps,
                                             float eps_hi, T *row)
{
  constexpr int D = K / 2;
  if constexpr ( VT > 0 )
  {
    double p[VT * 3];
    const double *src = verts + static_cast< size_t >( e ) * VT * 3;
#pragma unroll
    for ( int k = 0; k < VT * 3; ++k ) p[k] = __ldg( src + k );
    if constexpr ( sizeof( T ) == 8 )
    {
#pragma unroll
      for ( int a = 0; a < D; ++a )
      {
        double l, h;
        slab64< K >( p, VT, a, eps, l, h );
        row[2 * a] = l;
        row[2 * a + 1] = h;
      }
    } else {
      float lo[D], hi[D];
      slabs32_all< K, VT >( p, eps_hi, lo, hi );
#pragma unroll
      for ( int a = 0; a < D; ++a )
      {
        row[2 * a] = lo[a];
        row[2 * a + 1] = hi[a];
      }
    }
  } else {
    T lo[D], hi[D];
    leaf_slabs< K, T, 0 >( verts, Vrt, e, eps, eps_hi, lo, hi );
#pragma unroll
    for ( int a = 0; a < D; ++a )
    {
      row[2 * a] = lo[a];
      row[2 * a + 1] = hi[a];
    }
  }
}

// Everything one query packet needs besides the tree (see traverse_body).
template< typename T >
struct trav_args
{
  const T *qwarp;
  const double *qverts;
  uint32_t qV;
  const T *qrows;    // query element slabs in rank order (stored variant only)
  const uint32_t *qperm;
  uint32_t nq;
  const int2 *child;
  const T *nbox;
  const int2 *range;
  const double *tverts;
  uint32_t tV;
  const T *tcache;   // element slabs of the target in rank order (stored variant only)
  const uint32_t *tperm;
  const obj_scalars *tsc;
  uint32_t nt;
  int self;
  double eps;
  float eps_hi;
  uint2 *pairs;
  uint64_t cap;
  pair_scalars *ps;
  int dense_stack;  // stack bound of the batched dense walk (kDenseStack, lower under a test hook)
};

// The typed view of a scene's traversal item.
template< typename T >
__device__ __forceinline__ trav_args< T > typed(const trav_item &it)
{
  trav_args< T > x;
  x.qwarp = static_cast< const T * >( it.qwarp );
  x.qverts = it.qverts;
  x.qV = it.qV;
  x.qrows = static_cast< const T * >( it.qrows );
  x.qperm = it.qperm;
  x.nq = it.nq;
  x.child = it.child;
  x.nbox = static_cast< const T * >( it.nbox );
  x.range = it.range;
  x.tverts = it.tverts;
  x.tV = it.tV;
  x.tcache = static_cast< const T * >( it.tcache );
  x.tperm = it.tperm;
  x.tsc = it.tsc;
  x.nt = it.nt;
  x.self = it.self;
  x.eps = it.eps;
  x.eps_hi = it.eps_hi;
  x.pairs = it.pairs;
  x.cap = it.cap;
  x.ps = it.ps;
  x.dense_stack = it.dense_stack;
  return x;
}

// Target leaf bucket bb for the lanes in `mine`: the warp first computes the bucket's element slabs into its cache
// (lane j: element of rank 8 bb + j), then every lane of the mask tests its query against them (ranks above its own
// in self-collision). Hits go out through one warp-aggregated reservation. Called by the whole warp.
template< int K, typename T, int VT >
__device__ __forceinline__ void test_bucket(const trav_args< T > &x, const T *qlo, const T *qhi, uint32_t qe, int bb,
                                            int skip, bool mine, T *cache, unsigned lane)
{
  constexpr int D = K / 2;
  const int t0 = kLeafSize * bb;
  const int cnt = min( kLeafSize, static_cast< int >( x.nt ) - t0 );
  // The bucket's element slabs, computed from the vertices into the warp's shared-memory cache by lanes 0..7
  // (sparse contact: a bucket is tested by few packets, so nothing is kept).
  if ( static_cast< int >( lane ) < cnt )
    slabs_to_row< K, T, VT >( x.tverts, x.tV, __ldg( x.tperm + t0 + lane ), x.eps, x.eps_hi, cache + lane * 2 * D );
  __syncwarp();
  const T *rows = cache;
  if ( mine )
  {
    const int r0 = max( t0, skip + 1 );
    unsigned hits = 0;
    for ( int r = r0; r < t0 + cnt; ++r )
    {
      const T *eb = rows + ( r - t0 ) * 2 * D;
      bool o = true;
#pragma unroll
      for ( int a = 0; a < D; ++a )
      {
        if ( !o ) break;
        o = qlo[a] < eb[2 * a + 1] && eb[2 * a] < qhi[a];
      }
      if ( o ) hits |= 1u << ( r - t0 );
    }
    unsigned long long pos = warp_reserve( static_cast< unsigned >( __popc( hits ) ), &x.ps->count );
    for ( ; hits; hits &= hits - 1, ++pos )
      if ( pos < x.cap ) x.pairs[pos] = make_uint2( qe, __ldg( x.tperm + t0 + __ffs( hits ) - 1 ) );
  }
  __syncwarp();  // the cache is refilled by the next leaf
}

// One packet: the union box of ranks pk*32 .. pk*32 + 31 against the target root, then the walk (see traverse_body).
template< int K, typename T, int VT >
__device__ __forceinline__ void traverse_packet(const trav_args< T > &x, const uint32_t i, const unsigned lane,
                                                int2 *stack, T *cache, const T *rb)
{
  constexpr int D = K / 2;
  constexpr int D0 = D < 4 ? D : 4;
  // 1. The packet's union box against the target's root box, first four slabs first (uniform per warp).
  {
    const T *wb = x.qwarp + static_cast< size_t >( i >> 5 ) * D * 2;
    bool o = true;
#pragma unroll
    for ( int a = 0; a < D0; ++a ) o = o && ( __ldg( wb + 2 * a ) < rb[2 * a + 1] && rb[2 * a] < __ldg( wb + 2 * a + 1 ) );
    if ( !o ) return;
#pragma unroll
    for ( int a = D0; a < D; ++a ) o = o && ( __ldg( wb + 2 * a ) < rb[2 * a + 1] && rb[2 * a] < __ldg( wb + 2 * a + 1 ) );
    if ( !o ) return;
  }
  // 2. Each lane's own slabs, from its element's vertices, against the root box.
  const bool valid = i < x.nq;
  const uint32_t qe = valid ? __ldg( x.qperm + i ) : 0u;
  T qlo[D], qhi[D];
  bool in_root = valid;
  if ( valid ) leaf_slabs< K, T, VT >( x.qverts, x.qV, qe, x.eps, x.eps_hi, qlo, qhi );
#pragma unroll
  for ( int a = 0; a < D; ++a )
  {
    if ( !valid )
    {
      qlo[a] = T( 0 );
      qhi[a] = T( 0 );
    }
    in_root = in_root && ( qlo[a] < rb[2 * a + 1] && rb[2 * a] < qhi[a] );
  }
  unsigned mask = __ballot_sync( 0xffffffffu, in_root );
  if ( !mask ) return;
  const int skip = x.self ? static_cast< int >( i ) : -1;  // self-collision: only ranks above the query's
  const int root = x.tsc->root;
  if ( root < 0 )
  {
    test_bucket< K, T, VT >( x, qlo, qhi, qe, ~root, skip, in_root, cache, lane );
    return;
  }
  int sp = 0;
  int node = root;
  while ( true )
  {
    const bool me = ( mask >> lane ) & 1u;
    const int2 c = __ldg( x.child + node );
    const T *nb = x.nbox + static_cast< size_t >( node ) * D * 4;
    bool o0 = me, o1 = me;
    if ( x.self )
    {
      // left child covers buckets [l, node], right child [node + 1, r]; skip subtrees whose last rank <= i
      o0 = o0 && kLeafSize * node + kLeafSize - 1 > static_cast< int >( i );
      o1 = o1 && min( kLeafSize * __ldg( &x.range[node].y ) + kLeafSize - 1, static_cast< int >( x.nt ) - 1 ) >
                   static_cast< int >( i );
    }
    // The node row's slabs in chunks of kNodeChunk axes: a chunk's loads (one sector per axis) are all in flight
    // before its tests, and the warp stops between chunks once no lane overlaps either child.
#pragma unroll
    for ( int a0 = 0; a0 < D; a0 += kNodeChunk< K, T > )
    {
      if ( a0 > 0 && !__any_sync( 0xffffffffu, o0 || o1 ) ) break;
      slab_pair< T > sl[kNodeChunk< K, T >];
#pragma unroll
      for ( int j = 0; j < kNodeChunk< K, T >; ++j )
        if ( a0 + j < D ) sl[j] = slab_pair< T >::load( nb + ( a0 + j ) * 4 );
#pragma unroll
      for ( int j = 0; j < kNodeChunk< K, T >; ++j )
      {
        if ( a0 + j >= D ) break;
        o0 = o0 && ( qlo[a0 + j] < sl[j].max0 && sl[j].min0 < qhi[a0 + j] );
        o1 = o1 && ( qlo[a0 + j] < sl[j].max1 && sl[j].min1 < qhi[a0 + j] );
      }
    }
    const unsigned m0 = __ballot_sync( 0xffffffffu, o0 );
    const unsigned m1 = __ballot_sync( 0xffffffffu, o1 );
    int next = -1;
    unsigned nmask = 0;
    if ( m0 )
    {
      if ( c.x < 0 ) test_bucket< K, T, VT >( x, qlo, qhi, qe, ~c.x, skip, o0, cache, lane );
      else
      {
        next = c.x;
        nmask = m0;
      }
    }
    if ( m1 )
    {
      if ( c.y < 0 ) test_bucket< K, T, VT >( x, qlo, qhi, qe, ~c.y, skip, o1, cache, lane );
      else if ( next < 0 )
      {
        next = c.y;
        nmask = m1;
      } else {
        if ( sp == kStack )
        {
          if ( lane == 0 ) atomicCAS( &x.ps->error, 0, kErrOverflowStack );
          return;
        }
        if ( lane == 0 ) stack[sp] = make_int2( c.y, static_cast< int >( m1 ) );
        ++sp;
      }
    }
    if ( next < 0 )
    {
      if ( sp == 0 ) break;
      __syncwarp();
      const int2 e = stack[--sp];
      next = e.x;
      nmask = static_cast< unsigned >( e.y );
    }
    __syncwarp();
    node = next;
    mask = nmask;
  }
}

// One warp per group of 32 query ranks (a packet), lane = query element. The warp walks the target tree once for
// its packet: every lane tests its own element's slabs (computed from its vertices) against both children of the
// current node (the node row is read once for the warp, a broadcast), and a child is entered with the mask of the
// lanes that overlap it (a lane that misses a node misses all of its descendants). Stack entries are (node, lane
// mask), in shared memory. At a leaf bucket the lanes of the mask test their element against the bucket's element
// slabs, computed once by the warp from the vertices into a shared cache.
template< int K, typename T, int VT >
__device__ void traverse_body(const trav_item &item, uint32_t, uint32_t)
{
  const trav_args< T > x = typed< T >( item );
  const obj_scalars *__restrict__ qsc = item.qsc;
  constexpr int D = K / 2;
  constexpr int D0 = D < 4 ? D : 4;
  constexpr int WPB = kTravThreads / 32;
  __shared__ int2 s_stack[WPB][kStack];                          // (node, lane mask)
  __shared__ __align__( 16 ) T s_cache[WPB][kLeafSize * 2 * D];  // slabs of the leaf bucket being tested
  const unsigned lane = threadIdx.x & 31u;
  int2 *stack = s_stack[threadIdx.x >> 5];
  T *cache = s_cache[threadIdx.x >> 5];
  // No tree exists after a failed sort of either object.
  if ( *reinterpret_cast< const volatile int * >( &x.tsc->error ) == kErrTimeout ||
       *reinterpret_cast< const volatile int * >( &qsc->error ) == kErrTimeout )
    return;
  const T *rb = reinterpret_cast< const T * >( x.tsc->root_box );
  // 0. Root against root: objects far apart (most pairs of a batch) end here for the whole grid.
  {
    const T *qr = reinterpret_cast< const T * >( qsc->root_box );
    bool o = true;
#pragma unroll
    for ( int a = 0; a < D0; ++a ) o = o && ( qr[2 * a] < rb[2 * a + 1] && rb[2 * a] < qr[2 * a + 1] );
    if ( !o ) return;
  }
  const uint32_t packets = ( x.nq + 31 ) / 32;
  // Packets (32 query ranks) in a persistent grid. A warp takes chunks from the pair counters'
  // packet dispenser; chunk c holds the packets c, c + C, c + 2C, ... (C chunks), so a contact region (consecutive
  // Morton ranks) is spread over many chunks. Lane j tests the union box of the chunk's packet j against the target
  // root (one load per lane for the packets far from the target), then the warp walks the survivors one after the
  // other.
  const uint32_t chunks = ( packets + 31 ) / 32;
  while ( true )
  {
    uint32_t c = 0;
    if ( lane == 0 ) c = atomicAdd( &x.ps->packet_next, 1u );
    c = __shfl_sync( 0xffffffffu, c, 0 );
    if ( c >= chunks ) break;
    const uint64_t pk = c + static_cast< uint64_t >( lane ) * chunks;
    bool o = false;
    if ( pk < packets )
    {
      const T *wb = x.qwarp + pk * D * 2;
      o = true;
#pragma unroll
      for ( int a = 0; a < D; ++a ) o = o && ( __ldg( wb + 2 * a ) < rb[2 * a + 1] && rb[2 * a] < __ldg( wb + 2 * a + 1 ) );
    }
    for ( unsigned m = __ballot_sync( 0xffffffffu, o ); m; m &= m - 1 )
    {
      const uint32_t p = c + static_cast< uint32_t >( __ffs( m ) - 1 ) * chunks;
      traverse_packet< K, T, VT >( x, p * 32 + lane, lane, stack, cache, rb );
    }
  }
}

// ---- dense contact: both objects' element slabs stored ----------------------------------------------------------
//
// In dense contact a packet's walk visits a few hundred internal nodes and tens of leaf buckets, each shared by only
// a fraction of the packet's 32 queries. Two changes over the walk of traverse_packet:
//   - Nodes in batches. Each step pops up to kDenseBatch (4 or 6) (node, lane mask) entries from the stack; the
//     warp copies their rows (both children's slabs) into shared memory with one round of 16-byte asynchronous
//     copies, and every lane tests its query against the children of each popped node whose mask holds it, from
//     shared memory. One global round trip serves the whole batch instead of one per chunk of slabs per node.
//   - Leaves in batches. The walk only queues (bucket, lane mask) entries; a flush spreads all (query, element)
//     tests of the queued entries over the warp's lanes, 32 at a time, with every query's slabs staged in shared
//     memory and the target elements' stored rows read from global memory. A lane finds the entry of its test from
//     two warp votes per round and reads it from the lane that holds it. Hits collect in a per-warp buffer in
//     shared memory (one ballot per 32 tests); a full buffer leaves through one atomic reservation and coalesced
//     stores, so a warp pays an atomic's round trip per 33-64 pairs instead of per round of tests with a hit.
// The stack grows by at most kDenseBatch entries per step, so its depth bound is kDenseStack; a walk that would pass
// it raises kErrOverflowStack, and the host then runs the pair search again with the single-node walk (whose stack
// is bounded by the tree depth).
constexpr int kLeafQueue = 32;  // queued (bucket, mask) entries per warp
constexpr int kPairBuf = 64;    // buffered pairs per warp: drained once more than 32 are held

// A (min, max) pair: from global memory (read-only path) or from shared memory, as one vector load.
__device__ __forceinline__ void load_pair(const double *p, double &lo, double &hi)
{
  const double2 v = __ldg( reinterpret_cast< const double2 * >( p ) );
  lo = v.x;
  hi = v.y;
}
__device__ __forceinline__ void load_pair(const float *p, float &lo, float &hi)
{
  const float2 v = __ldg( reinterpret_cast< const float2 * >( p ) );
  lo = v.x;
  hi = v.y;
}
__device__ __forceinline__ void shared_pair(const double *p, double &lo, double &hi)
{
  const double2 v = *reinterpret_cast< const double2 * >( p );
  lo = v.x;
  hi = v.y;
}
__device__ __forceinline__ void shared_pair(const float *p, float &lo, float &hi)
{
  const float2 v = *reinterpret_cast< const float2 * >( p );
  lo = v.x;
  hi = v.y;
}
// Nodes popped per step: 6 for 26-DOP FP64 rows (measured 6% faster there, at 4 resident blocks per SM instead of
// 5), 4 otherwise (6 measured 1-6% slower for the other k-DOPs and the FP32 rows).
template< int K, typename T >
constexpr int kDenseBatch = ( K == 26 && sizeof( T ) == 8 ) ? 6 : 4;
constexpr int kDenseStack = 256;

template< int K, typename T >
struct dense_smem
{
  // every array starts on a 16-byte boundary: rows[] receives 16-byte asynchronous copies, and q[] and rows[] are
  // read as 8- or 16-byte (min, max) pairs
  alignas( 16 ) T q[32][K];                  // query slabs of the packet, (min, max) per slab
  alignas( 16 ) T rows[kDenseBatch< K, T >][2 * K];  // node rows of the batch: [slab][child][min, max]
  alignas( 16 ) uint32_t qe[32];             // query element indices
  alignas( 16 ) int2 stack[kDenseStack];     // (node, lane mask)
  alignas( 16 ) int2 leaf[kLeafQueue];       // (bucket, lane mask)
  alignas( 16 ) uint2 out[kPairBuf];         // pairs found and not yet written
};

template< int K, typename T >
constexpr bool dense_smem_aligned()
{
  using S = dense_smem< K, T >;
  return offsetof( S, q ) % 16 == 0 && offsetof( S, rows ) % 16 == 0 && sizeof( S ) % 16 == 0 &&
         ( 2 * K * sizeof( T ) ) % 16 == 0;  // node rows: whole 16-byte pieces
}
static_assert( dense_smem_aligned< 6, double >() && dense_smem_aligned< 18, double >() &&
                 dense_smem_aligned< 26, double >() && dense_smem_aligned< 6, float >() &&
                 dense_smem_aligned< 18, float >() && dense_smem_aligned< 26, float >(),
               "dense walk shared memory must keep 16-byte alignment" );

// Writes the warp's buffered pairs: one atomic reservation for all of them, then coalesced stores (a count past
// the capacity is still counted, so the host learns the size it needs).
template< int K, typename T >
__device__ __forceinline__ void drain_pairs(const trav_args< T > &x, dense_smem< K, T > &sm, uint32_t &nout,
                                            unsigned lane)
{
  __syncwarp();
  unsigned long long base = 0;
  if ( lane == 0 && nout ) base = atomicAdd( &x.ps->count, static_cast< unsigned long long >( nout ) );
  base = __shfl_sync( 0xffffffffu, base, 0 );
  for ( uint32_t j = lane; j < nout; j += 32 )
    if ( base + j < x.cap ) x.pairs[base + j] = sm.out[j];
  __syncwarp();
  nout = 0;
}

// Tests every (query, element) pair of the queued entries; i0 = the packet's first query rank. Hits are appended to
// the warp's pair buffer (nout pairs held).
template< int K, typename T >
__device__ __forceinline__ void flush_leaves(const trav_args< T > &x, dense_smem< K, T > &sm, int nleaf, uint32_t i0,
                                             unsigned lane, uint32_t &nout)
{
  constexpr int D = K / 2;
  __syncwarp();
  const int2 ent = static_cast< int >( lane ) < nleaf ? sm.leaf[lane] : make_int2( 0, 0 );
  const uint32_t c = 8u * static_cast< uint32_t >( __popc( static_cast< unsigned >( ent.y ) ) );
  uint32_t inc = c;
#pragma unroll
  for ( int o = 1; o < 32; o <<= 1 )
  {
    const uint32_t y = __shfl_up_sync( 0xffffffffu, inc, o );
    if ( lane >= static_cast< unsigned >( o ) ) inc += y;
  }
  const uint32_t total = __shfl_sync( 0xffffffffu, inc, 31 );
  const bool is_entry = static_cast< int >( lane ) < nleaf;
  const uint32_t mypre = inc - c;
  __syncwarp();
  const unsigned lt = ( 1u << lane ) - 1u;
  for ( uint32_t base = 0; base < total; base += 32 )
  {
    const uint32_t g = base + lane;
    bool hit = false;
    uint32_t q = 0, r = 0;
    // the entry of test g: the last entry whose prefix is <= g, from the entries that start before this round and
    // the starts inside it (entries have distinct prefixes: every entry holds at least 8 tests)
    const unsigned before = __ballot_sync( 0xffffffffu, is_entry && mypre < base );
    const unsigned inround = ( is_entry && mypre >= base && mypre - base < 32u ) ? ( 1u << ( mypre - base ) ) : 0u;
    const unsigned starts = __reduce_or_sync( 0xffffffffu, inround );
    int lo = __popc( before ) + __popc( starts & ( ( 2u << lane ) - 1u ) ) - 1;
    lo = lo < 0 ? 0 : lo;
    const uint32_t lpre = __shfl_sync( 0xffffffffu, mypre, lo );
    const int enx = __shfl_sync( 0xffffffffu, ent.x, lo ), eny = __shfl_sync( 0xffffffffu, ent.y, lo );
    if ( g < total )
    {
      const uint32_t rr = g - lpre;
      const int2 en = make_int2( enx, eny );
      unsigned m = static_cast< unsigned >( en.y );
      for ( uint32_t k = rr >> 3; k > 0; --k ) m &= m - 1;  // the (rr / 8)-th query of the entry's mask
      q = static_cast< uint32_t >( __ffs( m ) - 1 );
      r = static_cast< uint32_t >( en.x ) * kLeafSize + ( rr & 7u );
      if ( r < x.nt && ( !x.self || r > i0 + q ) )
      {
        // a chunk of slabs of the element (global) and of the query (shared) is loaded before it is tested
        const T *er = x.tcache + static_cast< size_t >( r >> 3 ) * ( kLeafSize * K ) + 2 * ( r & 7u );
        const T *qr = sm.q[q];
        hit = true;
#pragma unroll
        for ( int a0 = 0; a0 < D; a0 += kNodeChunk< K, T > )
        {
          if ( !hit ) break;
          T ev[2 * kNodeChunk< K, T >], qv[2 * kNodeChunk< K, T >];
#pragma unroll
          for ( int j = 0; j < kNodeChunk< K, T >; ++j )
          {
            if ( a0 + j >= D ) break;
            load_pair( er + 2 * kLeafSize * ( a0 + j ), ev[2 * j], ev[2 * j + 1] );
            shared_pair( qr + 2 * ( a0 + j ), qv[2 * j], qv[2 * j + 1] );
          }
#pragma unroll
          for ( int j = 0; j < kNodeChunk< K, T >; ++j )
          {
            if ( a0 + j >= D ) break;
            hit = hit && qv[2 * j] < ev[2 * j + 1] && ev[2 * j] < qv[2 * j + 1];
          }
        }
      }
    }
    const unsigned bal = __ballot_sync( 0xffffffffu, hit );
    if ( bal )
    {
      if ( hit ) sm.out[nout + static_cast< unsigned >( __popc( bal & lt ) )] = make_uint2( sm.qe[q], __ldg( x.tperm + r ) );
      nout += static_cast< uint32_t >( __popc( bal ) );
      if ( nout > kPairBuf - 32 ) drain_pairs< K, T >( x, sm, nout, lane );
    }
  }
  __syncwarp();
}

// One packet in dense contact (see above). Returns false when the stack bound was reached (error raised).
template< int K, typename T >
__device__ __forceinline__ void traverse_packet_stored(const trav_args< T > &x, const uint32_t i0, const unsigned lane,
                                                       dense_smem< K, T > &sm, const T *rb)
{
  constexpr int D = K / 2;
  constexpr int D0 = D < 4 ? D : 4;
  constexpr int R16 = 2 * K * static_cast< int >( sizeof( T ) ) / 16;  // 16-byte pieces of a node row
  const uint32_t i = i0 + lane;
  {
    const T *wb = x.qwarp + static_cast< size_t >( i0 >> 5 ) * K;
    bool o = true;
#pragma unroll
    for ( int a = 0; a < D0; ++a ) o = o && ( __ldg( wb + 2 * a ) < rb[2 * a + 1] && rb[2 * a] < __ldg( wb + 2 * a + 1 ) );
    if ( !o ) return;
#pragma unroll
    for ( int a = D0; a < D; ++a ) o = o && ( __ldg( wb + 2 * a ) < rb[2 * a + 1] && rb[2 * a] < __ldg( wb + 2 * a + 1 ) );
    if ( !o ) return;
  }
  const bool valid = i < x.nq;
  T qlo[D], qhi[D];
  bool in_root = valid;
  {
    const uint32_t iv = valid ? i : 0u;
    const T *qs = x.qrows + static_cast< size_t >( iv >> 3 ) * ( kLeafSize * K ) + 2 * ( iv & 7u );
#pragma unroll
    for ( int a = 0; a < D; ++a )
    {
      load_pair( qs + 2 * kLeafSize * a, qlo[a], qhi[a] );
      if ( !valid )
      {
        qlo[a] = T( 0 );
        qhi[a] = T( 0 );
      }
      sm.q[lane][2 * a] = qlo[a];
      sm.q[lane][2 * a + 1] = qhi[a];
      in_root = in_root && ( qlo[a] < rb[2 * a + 1] && rb[2 * a] < qhi[a] );
    }
  }
  sm.qe[lane] = valid ? __ldg( x.qperm + i ) : 0u;
  const unsigned mask = __ballot_sync( 0xffffffffu, in_root );
  if ( !mask ) return;
  const int root = x.tsc->root;
  int nleaf = 0;
  uint32_t nout = 0;
  if ( root < 0 )
  {
    if ( lane == 0 ) sm.leaf[0] = make_int2( ~root, static_cast< int >( mask ) );
    flush_leaves< K, T >( x, sm, 1, i0, lane, nout );
    drain_pairs< K, T >( x, sm, nout, lane );
    return;
  }
  if ( lane == 0 ) sm.stack[0] = make_int2( root, static_cast< int >( mask ) );
  int sp = 1;
  while ( sp > 0 )
  {
    __syncwarp();
    const int nb = sp < kDenseBatch< K, T > ? sp : kDenseBatch< K, T >;
    sp -= nb;
    // the batch's node rows into shared memory (one round of asynchronous copies), their links into registers
    for ( int t = static_cast< int >( lane ); t < nb * R16; t += 32 )
    {
      const int k = t / R16, piece = t - k * R16;
      const int node = sm.stack[sp + k].x;
      cp_async16( reinterpret_cast< char * >( sm.rows[k] ) + 16 * piece,
                  reinterpret_cast< const char * >( x.nbox + static_cast< size_t >( node ) * 2 * K ) + 16 * piece );
    }
    int2 links = make_int2( 0, 0 ), span = make_int2( 0, 0 );
    if ( static_cast< int >( lane ) < nb )
    {
      const int node = sm.stack[sp + lane].x;
      links = __ldg( x.child + node );
      if ( x.self ) span = make_int2( node, __ldg( &x.range[node].y ) );
    }
    unsigned emask[kDenseBatch< K, T >];
#pragma unroll
    for ( int k = 0; k < kDenseBatch< K, T >; ++k ) emask[k] = k < nb ? static_cast< unsigned >( sm.stack[sp + k].y ) : 0u;
    cp_async_wait_all();
    __syncwarp();
    unsigned m0[kDenseBatch< K, T >], m1[kDenseBatch< K, T >];
#pragma unroll
    for ( int k = 0; k < kDenseBatch< K, T >; ++k )
    {
      if ( k >= nb ) break;
      bool o0 = ( emask[k] >> lane ) & 1u, o1 = o0;
      if ( x.self )
      {
        // left child covers buckets [l, node], right child [node + 1, r]: skip subtrees whose last rank <= i
        const int node = __shfl_sync( 0xffffffffu, span.x, k ), last = __shfl_sync( 0xffffffffu, span.y, k );
        o0 = o0 && kLeafSize * node + kLeafSize - 1 > static_cast< int >( i );
        o1 = o1 && min( kLeafSize * last + kLeafSize - 1, static_cast< int >( x.nt ) - 1 ) > static_cast< int >( i );
      }
      // a chunk of slabs of the row is read from shared memory before it is tested
      const T *row = sm.rows[k];
#pragma unroll
      for ( int a0 = 0; a0 < D; a0 += kNodeChunk< K, T > )
      {
        if ( !( o0 || o1 ) ) break;
        T v[4 * kNodeChunk< K, T >];
#pragma unroll
        for ( int j = 0; j < kNodeChunk< K, T >; ++j )
        {
          if ( a0 + j >= D ) break;
          shared_pair( row + 4 * ( a0 + j ), v[4 * j], v[4 * j + 1] );
          shared_pair( row + 4 * ( a0 + j ) + 2, v[4 * j + 2], v[4 * j + 3] );
        }
#pragma unroll
        for ( int j = 0; j < kNodeChunk< K, T >; ++j )
        {
          if ( a0 + j >= D ) break;
          o0 = o0 && ( qlo[a0 + j] < v[4 * j + 1] && v[4 * j] < qhi[a0 + j] );
          o1 = o1 && ( qlo[a0 + j] < v[4 * j + 3] && v[4 * j + 2] < qhi[a0 + j] );
        }
      }
      m0[k] = __ballot_sync( 0xffffffffu, o0 );
      m1[k] = __ballot_sync( 0xffffffffu, o1 );
    }
    // children: buckets to the leaf queue, internal nodes onto the stack (warp-uniform; lane 0 writes)
#pragma unroll
    for ( int k = 0; k < kDenseBatch< K, T >; ++k )
    {
      if ( k >= nb ) break;
      const int cx = __shfl_sync( 0xffffffffu, links.x, k ), cy = __shfl_sync( 0xffffffffu, links.y, k );
#pragma unroll
      for ( int side = 0; side < 2; ++side )
      {
        const unsigned m = side ? m1[k] : m0[k];
        const int ch = side ? cy : cx;
        if ( !m ) continue;
        if ( ch < 0 )
        {
          if ( lane == 0 ) sm.leaf[nleaf] = make_int2( ~ch, static_cast< int >( m ) );
          ++nleaf;
        } else {
          if ( sp >= x.dense_stack )
          {
            if ( lane == 0 ) atomicCAS( &x.ps->error, 0, kErrOverflowStack );
            drain_pairs< K, T >( x, sm, nout, lane );
            return;
          }
          if ( lane == 0 ) sm.stack[sp] = make_int2( ch, static_cast< int >( m ) );
          ++sp;
        }
      }
    }
    if ( nleaf > kLeafQueue - 2 * kDenseBatch< K, T > )
    {
      flush_leaves< K, T >( x, sm, nleaf, i0, lane, nout );
      nleaf = 0;
    }
  }
  if ( nleaf > 0 ) flush_leaves< K, T >( x, sm, nleaf, i0, lane, nout );
  drain_pairs< K, T >( x, sm, nout, lane );
}

// Resident blocks per SM of the dense walk: as many as its shared memory allows (228 KB per SM, 1 KB of it reserved
// per block), at most kDenseBlockCap; the register budget follows from it. 18-DOP FP64 rows run at 5 blocks (96
// registers, no spills): at 6 they were squeezed into 80 registers with spills, and the walk was 16% slower.
template< int K, typename T >
constexpr int kDenseBlockCap = ( K == 18 && sizeof( T ) == 8 ) ? 5 : 6;
template< int K, typename T >
constexpr int kDenseBlocksBySmem =
  ( 228 * 1024 ) / ( ( kTravThreads / 32 ) * static_cast< int >( sizeof( dense_smem< K, T > ) ) + 1024 );
template< int K, typename T >
constexpr int kDenseBlocksPerSM =
  kDenseBlocksBySmem< K, T > < kDenseBlockCap< K, T > ? kDenseBlocksBySmem< K, T > : kDenseBlockCap< K, T >;

// Dense contact: one warp per packet of 32 query ranks (the hardware balances the walks).
template< int K, typename T >
__device__ void stored_body(const trav_item &item, uint32_t bid, uint32_t)
{
  const trav_args< T > x = typed< T >( item );
  const obj_scalars *__restrict__ qsc = item.qsc;
  constexpr int D = K / 2;
  constexpr int D0 = D < 4 ? D : 4;
  constexpr int WPB = kTravThreads / 32;
  __shared__ __align__( 16 ) dense_smem< K, T > s_dense[WPB];
  const unsigned lane = threadIdx.x & 31u;
  if ( *reinterpret_cast< const volatile int * >( &x.tsc->error ) == kErrTimeout ||
       *reinterpret_cast< const volatile int * >( &qsc->error ) == kErrTimeout )
    return;
  const T *rb = reinterpret_cast< const T * >( x.tsc->root_box );
  {
    const T *qr = reinterpret_cast< const T * >( qsc->root_box );
    bool o = true;
#pragma unroll
    for ( int a = 0; a < D0; ++a ) o = o && ( qr[2 * a] < rb[2 * a + 1] && rb[2 * a] < qr[2 * a + 1] );
    if ( !o ) return;
  }
  const uint32_t packets = ( x.nq + 31 ) / 32;
  const uint32_t pk = ( bid * blockDim.x + threadIdx.x ) >> 5;
  if ( pk < packets ) traverse_packet_stored< K, T >( x, pk * 32, lane, s_dense[threadIdx.x >> 5], rb );
}

// One scene's item and grid. Dense contact: one warp per packet. Sparse: a persistent grid of at most the resident
// blocks (4 per SM), one warp per chunk of 32 packets at most.
template< int K, typename T >
void trav_item_t(tree_view q, tree_view t, bool self, bool dense, double eps, uint2 *pairs, uint64_t cap,
                 pair_scalars *ps, int dense_stack_limit, trav_item *it, uint32_t *blocks, bool *dense_out)
{
  it->qwarp = q.warp_box;
  it->qverts = q.verts;
  it->qV = q.V;
  it->qrows = q.elem_cache;
  it->qperm = q.perm;
  it->nq = static_cast< uint32_t >( q.n );
  it->child = t.child;
  it->nbox = t.node_box;
  it->range = t.range;
  it->tverts = t.verts;
  it->tV = t.V;
  it->tcache = t.elem_cache;
  it->tperm = t.perm;
  it->tsc = t.sc;
  it->nt = static_cast< uint32_t >( t.n );
  it->self = self ? 1 : 0;
  it->eps = eps;
  it->eps_hi = f32_round_up( eps );
  it->pairs = pairs;
  it->cap = cap;
  it->ps = ps;
  it->dense_stack = dense_stack_limit > 0 && dense_stack_limit < kDenseStack ? dense_stack_limit : kDenseStack;
  it->qsc = q.sc;
  constexpr uint64_t kWarps = kTravThreads / 32;
  const uint64_t packets = ( q.n + 31 ) / 32;
  const uint64_t chunks = ( packets + 31 ) / 32;
  const uint64_t resident = static_cast< uint64_t >( device_sm_count() ) * kTravBlocksPerSM;
  dense = dense && q.stored && t.stored;
  uint64_t b = dense ? ( packets + kWarps - 1 ) / kWarps : ( chunks + kWarps - 1 ) / kWarps;
  if ( !dense && b > resident ) b = resident;
  *blocks = static_cast< uint32_t >( b < ( 1ull << 30 ) ? ( b ? b : 1 ) : ( 1ull << 30 ) );
  *dense_out = dense;
}

template< int K, typename T >
cudaError_t launch_trav_t(tree_view q, tree_view t, bool self, bool dense, double eps, uint2 *pairs, uint64_t cap,
                          pair_scalars *ps, cudaStream_t s, int dense_stack_limit)
{
  trav_item it;
  uint32_t grid = 0;
  trav_item_t< K, T >( q, t, self, dense, eps, pairs, cap, ps, dense_stack_limit, &it, &grid, &dense );
  // both objects' element slabs stored (dense contact): the batched walk that only reads them; else the one that
  // computes the slabs it tests from the vertices (unrolled when both objects have the same vertex count)
  if ( dense )
  {
    k_single< trav_item, stored_body< K, T >, kTravThreads, kDenseBlocksPerSM< K, T > ><<< grid, kTravThreads, 0, s >>>( it );
    return cudaGetLastError();
  }
  const uint32_t V = q.V == t.V ? q.V : 0;
  switch ( V )
  {
    case 3: k_single< trav_item, traverse_body< K, T, 3 >, kTravThreads, kTravBlocksPerSM ><<< grid, kTravThreads, 0, s >>>( it ); break;
    case 4: k_single< trav_item, traverse_body< K, T, 4 >, kTravThreads, kTravBlocksPerSM ><<< grid, kTravThreads, 0, s >>>( it ); break;
    case 8: k_single< trav_item, traverse_body< K, T, 8 >, kTravThreads, kTravBlocksPerSM ><<< grid, kTravThreads, 0, s >>>( it ); break;
    default: k_single< trav_item, traverse_body< K, T, 0 >, kTravThreads, kTravBlocksPerSM ><<< grid, kTravThreads, 0, s >>>( it ); break;
  }
  return cudaGetLastError();
}

template< int K, typename T >
cudaError_t launch_trav_batch_t(bool dense, uint32_t V, const batch_launch &b, cudaStream_t s)
{
  const trav_item *items = static_cast< const trav_item * >( b.items );
  if ( dense )
  {
    k_batched< trav_item, stored_body< K, T >, kTravThreads, kDenseBlocksPerSM< K, T > ><<< b.blocks, kTravThreads, 0, s >>>(
      items, b.starts, b.nitems );
    return cudaGetLastError();
  }
  switch ( V )
  {
    case 3: k_batched< trav_item, traverse_body< K, T, 3 >, kTravThreads, kTravBlocksPerSM ><<< b.blocks, kTravThreads, 0, s >>>( items, b.starts, b.nitems ); break;
    case 4: k_batched< trav_item, traverse_body< K, T, 4 >, kTravThreads, kTravBlocksPerSM ><<< b.blocks, kTravThreads, 0, s >>>( items, b.starts, b.nitems ); break;
    case 8: k_batched< trav_item, traverse_body< K, T, 8 >, kTravThreads, kTravBlocksPerSM ><<< b.blocks, kTravThreads, 0, s >>>( items, b.starts, b.nitems ); break;
    default: k_batched< trav_item, traverse_body< K, T, 0 >, kTravThreads, kTravBlocksPerSM ><<< b.blocks, kTravThreads, 0, s >>>( items, b.starts, b.nitems ); break;
  }
  return cudaGetLastError();
}

// The vertices of one element into registers: 16-byte loads when every element starts on a 16-byte boundary (an
// even vertex count, 48 bytes per vertex pair, and a 16-byte aligned array), else 8-byte loads. Half the load
// instructions of the recheck for tetrahedra and hexahedra (tet lattice: 1.88 -> 1.65 ms at 18-DOP).
template< int V >
__device__ __forceinline__ void load_verts(const double *p, bool vec16, double *x)
{
  if constexpr ( V % 2 == 0 )
  {
    if ( vec16 )
    {
#pragma unroll
      for ( int k = 0; k < V * 3; k += 2 )
      {
        const double2 t = __ldg( reinterpret_cast< const double2 * >( p + k ) );
        x[k] = t.x;
        x[k + 1] = t.y;
      }
      return;
    }
  }
#pragma unroll
  for ( int k = 0; k < V * 3; ++k ) x[k] = __ldg( p + k );
}

constexpr int kRecheckThreads = 256;
constexpr int kRecheckBuf = 128;  // buffered pairs per warp: drained once more than 96 are held

// K7: FP64 overlap of both elements from their vertices. With both vertex counts known at compile time, the
// comparison-only projections of overlap64 (shared products, no products by 0 or 1, one epsilon shift per slab);
// otherwise slab64 slab by slab with early exit. Both give the outcome of comparing the FP64 slabs.
template< int K, int VA, int VB >
__device__ void recheck_body(const recheck_args &args, uint32_t bid, uint32_t nblk)
{
  const double *__restrict__ va = args.va;
  const uint32_t Var = args.Va;
  const double *__restrict__ vb = args.vb;
  const uint32_t Vbr = args.Vb;
  const double eps = args.eps;
  const uint2 *__restrict__ cand = args.cand;
  const uint64_t cand_cap = args.cand_cap;
  uint2 *out = args.out;
  const uint64_t cap = args.cap;
  pair_scalars *ps = args.ps;
  constexpr int D = K / 2;
  // The candidate count is read on the device: no host round trip between traversal and recheck.
  const uint64_t ncand = min( static_cast< uint64_t >( *reinterpret_cast< volatile unsigned long long * >( &ps->count ) ),
                              cand_cap );
  const int Va = VA > 0 ? VA : static_cast< int >( Var );
  const int Vb = VB > 0 ? VB : static_cast< int >( Vbr );
  const bool vec16 = ( ( reinterpret_cast< uintptr_t >( va ) | reinterpret_cast< uintptr_t >( vb ) ) & 15 ) == 0;
  // Confirmed pairs collect in a per-warp buffer in shared memory and leave through one atomic reservation per
  // 97-128 pairs, with coalesced stores (one same-address atomic per 32 candidates made the kernel wait on the
  // counter's round trip).
  __shared__ uint2 s_out[kRecheckThreads / 32][kRecheckBuf];
  const unsigned lane = threadIdx.x & 31u, lt = ( 1u << lane ) - 1u;
  uint2 *wout = s_out[threadIdx.x >> 5];
  uint32_t nout = 0;
  auto drain = [&]() {
    __syncwarp();
    unsigned long long base = 0;
    if ( lane == 0 && nout ) base = atomicAdd( &ps->count2, static_cast< unsigned long long >( nout ) );
    base = __shfl_sync( 0xffffffffu, base, 0 );
    for ( uint32_t j = lane; j < nout; j += 32 )
      if ( base + j < cap ) out[base + j] = wout[j];
    __syncwarp();
    nout = 0;
  };
  // warp-uniform trips: lane l of a warp takes candidate p0 + l
  for ( uint64_t p0 = static_cast< uint64_t >( bid ) * blockDim.x + ( threadIdx.x & ~31u ); p0 < ncand;
        p0 += static_cast< uint64_t >( nblk ) * blockDim.x )
  {
    const uint64_t p = p0 + lane;
    const bool valid = p < ncand;
    const uint2 c = valid ? __ldg( cand + p ) : make_uint2( 0u, 0u );
    bool ok = valid;
    const double *pa = va + static_cast< size_t >( c.x ) * Va * 3;
    const double *pb = vb + static_cast< size_t >( c.y ) * Vb * 3;
    double xa[VA > 0 ? VA * 3 : 24], xb[VB > 0 ? VB * 3 : 24];
    if constexpr ( VA > 0 && VB > 0 )
    {
      if ( valid )
      {
        load_verts< VA >( pa, vec16, xa );
        load_verts< VB >( pb, vec16, xb );
        ok = overlap64< K, VA, VB >( xa, xb, eps );
      }
    } else {
      (void)xa;
      (void)xb;
#pragma unroll
      for ( int a = 0; a < D; ++a )
      {
        if ( !ok ) break;
        double alo = 0, ahi = 0, blo = 0, bhi = 0;
        for ( int v = 0; v < Va; ++v )
        {
          const double q[3] = { __ldg( pa + 3 * v ), __ldg( pa + 3 * v + 1 ), __ldg( pa + 3 * v + 2 ) };
          double l, h;
          slab64< K >( q, 1, a, eps, l, h );
          alo = v ? std_min( alo, l ) : l;
          ahi = v ? std_max( ahi, h ) : h;
        }
        for ( int v = 0; v < Vb; ++v )
        {
          const double q[3] = { __ldg( pb + 3 * v ), __ldg( pb + 3 * v + 1 ), __ldg( pb + 3 * v + 2 ) };
          double l, h;
          slab64< K >( q, 1, a, eps, l, h );
          blo = v ? std_min( blo, l ) : l;
          bhi = v ? std_max( bhi, h ) : h;
        }
        ok = alo < bhi && blo < ahi;
      }
    }
    const unsigned bal = __ballot_sync( 0xffffffffu, ok );
    if ( ok ) wout[nout + static_cast< unsigned >( __popc( bal & lt ) )] = c;
    nout += static_cast< uint32_t >( __popc( bal ) );
    if ( nout > kRecheckBuf - 32 ) drain();
  }
  drain();
}

// grid-stride over the candidates (their count is read on the device): at most 4 blocks per SM
uint32_t recheck_grid(uint64_t ncand)
{
  const uint64_t blocks = ( ncand + kRecheckThreads - 1 ) / kRecheckThreads;
  const uint64_t capb = static_cast< uint64_t >( device_sm_count() ) * 4;
  return static_cast< uint32_t >( blocks < capb ? ( blocks ? blocks : 1 ) : capb );
}

template< int K >
cudaError_t recheck_k(const recheck_args &a, cudaStream_t s)
{
  const uint32_t grid = recheck_grid( a.cand_cap );
  if ( a.Va == 3 && a.Vb == 3 ) k_single< recheck_args, recheck_body< K, 3, 3 >, kRecheckThreads, 2 ><<< grid, kRecheckThreads, 0, s >>>( a );
  else if ( a.Va == 4 && a.Vb == 4 ) k_single< recheck_args, recheck_body< K, 4, 4 >, kRecheckThreads, 2 ><<< grid, kRecheckThreads, 0, s >>>( a );
  else if ( a.Va == 8 && a.Vb == 8 ) k_single< recheck_args, recheck_body< K, 8, 8 >, kRecheckThreads, 2 ><<< grid, kRecheckThreads, 0, s >>>( a );
  else k_single< recheck_args, recheck_body< K, 0, 0 >, kRecheckThreads, 2 ><<< grid, kRecheckThreads, 0, s >>>( a );
  return cudaGetLastError();
}

template< int K >
cudaError_t recheck_batch_k(uint32_t V, const batch_launch &b, cudaStream_t s)
{
  const recheck_args *it = static_cast< const recheck_args * >( b.items );
  if ( V == 3 ) k_batched< recheck_args, recheck_body< K, 3, 3 >, kRecheckThreads, 2 ><<< b.blocks, kRecheckThreads, 0, s >>>( it, b.starts, b.nitems );
  else if ( V == 4 ) k_batched< recheck_args, recheck_body< K, 4, 4 >, kRecheckThreads, 2 ><<< b.blocks, kRecheckThreads, 0, s >>>( it, b.starts, b.nitems );
  else if ( V == 8 ) k_batched< recheck_args, recheck_body< K, 8, 8 >, kRecheckThreads, 2 ><<< b.blocks, kRecheckThreads, 0, s >>>( it, b.starts, b.nitems );
  else k_batched< recheck_args, recheck_body< K, 0, 0 >, kRecheckThreads, 2 ><<< b.blocks, kRecheckThreads, 0, s >>>( it, b.starts, b.nitems );
  return cudaGetLastError();
}

__global__ void k_gid_pairs(const uint2 *__restrict__ pairs, uint64_t count, const uint64_t *__restrict__ gid_a,
                            const uint64_t *__restrict__ gid_b, int normalize, uint64_t *__restrict__ out)
{
  for ( uint64_t p = static_cast< uint64_t >( blockIdx.x ) * blockDim.x + threadIdx.x; p < count;
        p += static_cast< uint64_t >( gridDim.x ) * blockDim.x )
  {
    uint2 c = pairs[p];
    if ( normalize && c.x > c.y ) c = make_uint2( c.y, c.x );
    const uint64_t a = gid_a ? __ldg( gid_a + c.x ) : c.x;
    const uint64_t b = gid_b ? __ldg( gid_b + c.y ) : c.y;
    reinterpret_cast< ulonglong2 * >( out )[p] = make_ulonglong2( a, b );
  }
}

// k_gid_pairs with the count read on the device (at most cap): for launches whose count is unknown when they are
// enqueued (batched scenes in a CUDA graph).
__device__ void gid_dev_body(const gid_args &a, uint32_t bid, uint32_t nblk)
{
  const uint64_t n = min( static_cast< uint64_t >( *reinterpret_cast< const volatile unsigned long long * >( a.count ) ),
                          a.cap );
  for ( uint64_t p = static_cast< uint64_t >( bid ) * blockDim.x + threadIdx.x; p < n;
        p += static_cast< uint64_t >( nblk ) * blockDim.x )
  {
    uint2 c = a.pairs[p];
    if ( a.normalize && c.x > c.y ) c = make_uint2( c.y, c.x );
    const uint64_t ga = a.gid_a ? __ldg( a.gid_a + c.x ) : c.x;
    const uint64_t gb = a.gid_b ? __ldg( a.gid_b + c.y ) : c.y;
    reinterpret_cast< ulonglong2 * >( a.out )[p] = make_ulonglong2( ga, gb );
  }
}

// dst[i] = *src[i]: the error words of many objects in one copy.
__global__ void k_gather_words(const int *const *__restrict__ src, int n, int *__restrict__ dst)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if ( i < n ) dst[i] = *reinterpret_cast< const volatile int * >( src[i] );
}

}  // namespace

uint32_t gid_pairs_dev_blocks(uint64_t cap)
{
  const uint64_t blocks = ( cap + 255 ) / 256;
  return static_cast< uint32_t >( blocks < 148 * 2 ? ( blocks ? blocks : 1 ) : 148 * 2 );
}

cudaError_t launch_gid_pairs_dev(const uint2 *pairs, const unsigned long long *count, uint64_t cap,
                                 const uint64_t *gid_a, const uint64_t *gid_b, bool normalize, uint64_t *out,
                                 cudaStream_t s)
{
  if ( cap == 0 ) return cudaSuccess;
  const gid_args a{ pairs, count, cap, gid_a, gid_b, normalize ? 1 : 0, out };
  k_single< gid_args, gid_dev_body, 256, 1 ><<< gid_pairs_dev_blocks( cap ), 256, 0, s >>>( a );
  return cudaGetLastError();
}

cudaError_t launch_gid_pairs_dev_batch(const batch_launch &b, cudaStream_t s)
{
  if ( !b.nitems ) return cudaSuccess;
  k_batched< gid_args, gid_dev_body, 256, 1 ><<< b.blocks, 256, 0, s >>>( static_cast< const gid_args * >( b.items ),
                                                                        b.starts, b.nitems );
  return cudaGetLastError();
}

cudaError_t launch_gather_words(const int *const *src, int n, int *dst, cudaStream_t s)
{
  if ( n == 0 ) return cudaSuccess;
  k_gather_words<<< ( n + 255 ) / 256, 256, 0, s >>>( src, n, dst );
  return cudaGetLastError();
}

cudaError_t launch_traverse(int K, bool fp32, tree_view q, tree_view t, bool self, bool dense, double eps, uint2 *pairs,
                            uint64_t cap, pair_scalars *ps, cudaStream_t s, int dense_stack_limit)
{
  switch ( K )
  {
    case 6: return fp32 ? launch_trav_t< 6, float >( q, t, self, dense, eps, pairs, cap, ps, s, dense_stack_limit )
                        : launch_trav_t< 6, double >( q, t, self, dense, eps, pairs, cap, ps, s, dense_stack_limit );
    case 18: return fp32 ? launch_trav_t< 18, float >( q, t, self, dense, eps, pairs, cap, ps, s, dense_stack_limit )
                         : launch_trav_t< 18, double >( q, t, self, dense, eps, pairs, cap, ps, s, dense_stack_limit );
    case 26: return fp32 ? launch_trav_t< 26, float >( q, t, self, dense, eps, pairs, cap, ps, s, dense_stack_limit )
                         : launch_trav_t< 26, double >( q, t, self, dense, eps, pairs, cap, ps, s, dense_stack_limit );
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_recheck(int K, const double *verts_a, uint32_t Va, const double *verts_b, uint32_t Vb, double eps,
                           const uint2 *cand, uint64_t ncand, uint2 *out, uint64_t cap, pair_scalars *ps,
                           cudaStream_t s)
{
  const recheck_args a{ verts_a, Va, verts_b, Vb, eps, cand, ncand, out, cap, ps };
  switch ( K )
  {
    case 6: return recheck_k< 6 >( a, s );
    case 18: return recheck_k< 18 >( a, s );
    case 26: return recheck_k< 26 >( a, s );
    default: return cudaErrorInvalidValue;
  }
}

uint32_t recheck_blocks(uint64_t ncand) { return recheck_grid( ncand ); }

cudaError_t launch_recheck_batch(int K, uint32_t V, const batch_launch &b, cudaStream_t s)
{
  if ( !b.nitems ) return cudaSuccess;
  switch ( K )
  {
    case 6: return recheck_batch_k< 6 >( V, b, s );
    case 18: return recheck_batch_k< 18 >( V, b, s );
    case 26: return recheck_batch_k< 26 >( V, b, s );
    default: return cudaErrorInvalidValue;
  }
}

void traverse_item(int K, bool fp32, tree_view q, tree_view t, bool self, bool dense, double eps, uint2 *pairs,
                   uint64_t cap, pair_scalars *ps, int dense_stack_limit, trav_item *item, uint32_t *blocks,
                   bool *dense_out)
{
  // the item's fields do not depend on K or the slab type; only the grid depends on K through nothing either
  if ( fp32 ) trav_item_t< 18, float >( q, t, self, dense, eps, pairs, cap, ps, dense_stack_limit, item, blocks, dense_out );
  else trav_item_t< 18, double >( q, t, self, dense, eps, pairs, cap, ps, dense_stack_limit, item, blocks, dense_out );
  (void)K;
}

cudaError_t launch_traverse_batch(int K, bool fp32, bool dense, uint32_t V, const batch_launch &b, cudaStream_t s)
{
  if ( !b.nitems ) return cudaSuccess;
  switch ( K )
  {
    case 6: return fp32 ? launch_trav_batch_t< 6, float >( dense, V, b, s ) : launch_trav_batch_t< 6, double >( dense, V, b, s );
    case 18: return fp32 ? launch_trav_batch_t< 18, float >( dense, V, b, s ) : launch_trav_batch_t< 18, double >( dense, V, b, s );
    case 26: return fp32 ? launch_trav_batch_t< 26, float >( dense, V, b, s ) : launch_trav_batch_t< 26, double >( dense, V, b, s );
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_gid_pairs(const uint2 *pairs, uint64_t count, const uint64_t *gid_a, const uint64_t *gid_b,
                             bool normalize, uint64_t *out, cudaStream_t s)
{
  if ( count == 0 ) return cudaSuccess;
  const uint64_t blocks = ( count + 255 ) / 256;
  const unsigned grid = static_cast< unsigned >( blocks < 148 * 8 ? blocks : 148 * 8 );
  k_gid_pairs<<< grid, 256, 0, s >>>( pairs, count, gid_a, gid_b, normalize ? 1 : 0, out );
  return cudaGetLastError();
}

}  // namespace bvhg
