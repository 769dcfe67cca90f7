// k_tree.cu — element slabs, LBVH build and bottom-up k-DOP refit (K4 + K5).
//
// The reference builds its element trees on the host, top-down (top_down_builder, src/bvh/bvh_build.hpp:55-139,
// mean split on the longest axis) or with a serial Morton bottom-up builder (bvh_build.hpp:145-296), one element
// per leaf, node k-DOP = union of the subtree (bvh_build.hpp:109-124; kdop merge, kdop.hpp:558-569). The pair set
// of a strict-overlap traversal does not depend on the tree shape, so here the leaves are buckets of kLeafSize
// consecutive Morton ranks (the traversal tests a bucket's elements one by one) and the tree over the buckets is
// the radix tree of the bucket-boundary keys, built bottom-up agglomeratively (Apetrei): a subtree [l, r] joins
// the neighbour across its more similar boundary.
//
// No thread ever waits. Nodes whose two children close inside a block of 128 buckets are merged in shared memory
// (warp rounds, then block rounds) and written out coalesced; the rest use a global exchange slot per node: the
// first arrival's slab stores are ordered before its acq_rel atomic exchange, and the second arrival, which sees
// the slot taken with an acquire load (or learns it from its own exchange), reads them through L2 after it. The
// refit keeps the topology and splits the same way: the nodes inside a block in barrier-separated rounds over
// shared memory, then the block's local roots climb through the crossing nodes with the same exchange.
#include "bvhg_internal.cuh"
#include "bulk_copy.cuh"
#include "kdop_math.cuh"

namespace bvhg {

namespace {

constexpr int kBuildThreads = 128;


// Dissimilarity of ranks j and j + 1: 33 + highest differing key bit when the keys differ, else
// 1 + highest differing bit of the ranks. Larger = more different.
__device__ __forceinline__ int delta(const uint64_t *__restrict__ keys, int j)
{
  const uint64_t x = __ldg( keys + j ) ^ __ldg( keys + j + 1 );
  if ( x ) return 96 - __clzll( static_cast< long long >( x ) );
  return 32 - __clz( j ^ ( j + 1 ) );
}

// Exchange with acquire-release semantics at GPU scope (orders this thread's earlier stores before the exchange
// and its later loads after it).
__device__ __forceinline__ int atomic_exch_acq_rel(int *p, int v)
{
  int old;
  asm volatile( "atom.acq_rel.gpu.global.exch.b32 %0, [%1], %2;" : "=r"( old ) : "l"( p ), "r"( v ) : "memory" );
  return old;
}

// Load with acquire semantics at GPU scope (later loads are ordered after it).
__device__ __forceinline__ int ld_acquire(const int *p)
{
  int v;
  asm volatile( "ld.acquire.gpu.global.b32 %0, [%1];" : "=r"( v ) : "l"( p ) : "memory" );
  return v;
}

template< typename T >
struct box_io;

template<>
struct box_io< double >
{
  __device__ static void store2(double *p, double lo, double hi) { *reinterpret_cast< double2 * >( p ) = make_double2( lo, hi ); }
  __device__ static void store4(double *p, double a, double b, double c, double d)
  {
    reinterpret_cast< double2 * >( p )[0] = make_double2( a, b );
    reinterpret_cast< double2 * >( p )[1] = make_double2( c, d );
  }
  __device__ static void load2(const double *p, double &lo, double &hi)
  {
    const double2 v = *reinterpret_cast< const double2 * >( p );
    lo = v.x;
    hi = v.y;
  }
  __device__ static void load2_cg(const double *p, double &lo, double &hi)
  {
    const double2 v = __ldcg( reinterpret_cast< const double2 * >( p ) );
    lo = v.x;
    hi = v.y;
  }
  __device__ static double mn(double a, double b) { return ( b < a ) ? b : a; }
  __device__ static double mx(double a, double b) { return ( a < b ) ? b : a; }
};

template<>
struct box_io< float >
{
  __device__ static void store2(float *p, float lo, float hi) { *reinterpret_cast< float2 * >( p ) = make_float2( lo, hi ); }
  __device__ static void store4(float *p, float a, float b, float c, float d)
  {
    *reinterpret_cast< float4 * >( p ) = make_float4( a, b, c, d );
  }
  __device__ static void load2(const float *p, float &lo, float &hi)
  {
    const float2 v = *reinterpret_cast< const float2 * >( p );
    lo = v.x;
    hi = v.y;
  }
  __device__ static void load2_cg(const float *p, float &lo, float &hi)
  {
    const float2 v = __ldcg( reinterpret_cast< const float2 * >( p ) );
    lo = v.x;
    hi = v.y;
  }
  __device__ static float mn(float a, float b) { return fminf( a, b ); }
  __device__ static float mx(float a, float b) { return fmaxf( a, b ); }
};

// The root's slabs, for the traversal's first test.
template< typename T, size_t D >
__device__ __forceinline__ void store_root(obj_scalars *sc, const T ( &lo )[D], const T ( &hi )[D])
{
  T *rb = reinterpret_cast< T * >( sc->root_box );
#pragma unroll
  for ( size_t a = 0; a < D; ++a )
  {
    rb[2 * a] = lo[a];
    rb[2 * a + 1] = hi[a];
  }
}

// Dissimilarity from two adjacent keys (see delta()).
__device__ __forceinline__ int delta_of(uint64_t a, uint64_t b, int j)
{
  const uint64_t x = a ^ b;
  if ( x ) return 96 - __clzll( static_cast< long long >( x ) );
  return 32 - __clz( j ^ ( j + 1 ) );
}

// Dissimilarity of leaf buckets b and b + 1: the element dissimilarity across the bucket boundary, ties broken by
// position, so that the values are distinct and the agglomerative rule builds a well-defined binary tree (the
// Cartesian tree of these values, i.e. the radix tree of the boundary keys).
__device__ __forceinline__ long long bdelta(const uint64_t *__restrict__ keys, int b)
{
  return ( static_cast< long long >( delta( keys, kLeafSize * b + kLeafSize - 1 ) ) << 32 ) | static_cast< unsigned >( b );
}

// The same value from the per-boundary byte the block-local build stored (bdel[b] = the element dissimilarity
// across boundary b): the climb reads one byte of a small, cache-resident array instead of two keys.
__device__ __forceinline__ long long cdelta(const uint8_t *__restrict__ bdel, int b)
{
  return ( static_cast< long long >( __ldg( bdel + b ) ) << 32 ) | static_cast< unsigned >( b );
}

constexpr int kSlabThreads = 128;  // ranks per block of the element slab kernel

// Element slabs in rank order, one thread per rank (the element perm[r] of rank r), staged in shared memory (padded
// to C + 1 components against bank conflicts); per block of 128 ranks, the unions of its 16 leaf buckets and its 4
// query groups of 32 ranks are written out coalesced: bucket_box row b and warp_box row g each hold the C = 2 D
// values (min, max) per slab. The element slabs themselves go to elem_rows (slab-major per leaf bucket: rank
// r = 8 b + j, slab a at elem_rows[b * 8 C + 16 a + 2 j + {0 min, 1 max}]) only when given (objects in dense
// contact, whose traversals test most buckets); otherwise the traversal computes the few it tests from the
// vertices. A one-bucket object also gets its root box here. A rank whose index is not an element index marks a failed sort.
template< int K, int VT >
constexpr int kSlabMinBlocks = ( VT == 3 && K <= 18 ) ? 8 : ( VT == 8 ? 3 : 4 );

template< int K, typename T, int VT >
__device__ void slabs_body(const slabs_args &args, uint32_t bid, uint32_t)
{
  const double *__restrict__ verts = args.verts;
  const uint32_t Vrt = args.V;
  const int n = static_cast< int >( args.n );
  const double eps = args.eps;
  const float eps_hi = args.eps_hi;
  const uint32_t *__restrict__ vals = args.vals;
  T *__restrict__ bucket_box = static_cast< T * >( args.bucket_box );
  T *__restrict__ warp_box = static_cast< T * >( args.warp_box );
  T *__restrict__ elem_rows = static_cast< T * >( args.elem_rows );
  obj_scalars *sc = args.sc;
  constexpr int D = K / 2;
  constexpr int C = 2 * D;
  constexpr int P = C + 1;
  constexpr int G = 32 / kLeafSize;  // buckets per query group
  using io = box_io< T >;
  __shared__ T s_el[kSlabThreads * P];
  __shared__ T s_bk[( kSlabThreads / kLeafSize ) * P];
  if ( *reinterpret_cast< volatile int * >( &sc->error ) == kErrTimeout ) return;  // no valid permutation
  const int tid = threadIdx.x;
  const int r0 = static_cast< int >( bid ) * kSlabThreads;
  const int rows = min( kSlabThreads, n - r0 );
  if ( tid < rows )
  {
    const uint32_t e = __ldg( vals + r0 + tid );
    T lo[D], hi[D];
    if ( e < static_cast< uint32_t >( n ) )
    {
      leaf_slabs< K, T, VT >( verts, Vrt, e, eps, eps_hi, lo, hi );
    } else {
      atomicCAS( &sc->error, 0, kErrTimeout );
      const T inf = static_cast< T >( __longlong_as_double( 0x7ff0000000000000LL ) );
#pragma unroll
      for ( int a = 0; a < D; ++a )
      {
        lo[a] = inf;
        hi[a] = -inf;
      }
    }
#pragma unroll
    for ( int a = 0; a < D; ++a )
    {
      s_el[tid * P + 2 * a] = lo[a];
      s_el[tid * P + 2 * a + 1] = hi[a];
    }
  }
  __syncthreads();
  if ( elem_rows )
  {
    // slab-major per leaf bucket: [bucket][slab][element j < 8][min, max], so the 8 elements' values of one slab are
    // contiguous (the dense traversal reads them 8 lanes at a time)
    T *eb = elem_rows + static_cast< size_t >( r0 ) * C;
    const int nbk = ( rows + kLeafSize - 1 ) / kLeafSize;
    for ( int k = tid; k < nbk * kLeafSize * C; k += kSlabThreads )
    {
      const int lb = k / ( kLeafSize * C ), rem = k - lb * ( kLeafSize * C );
      const int a = rem / ( 2 * kLeafSize ), j = ( rem >> 1 ) & ( kLeafSize - 1 ), side = rem & 1;
      const int q = lb * kLeafSize + j;
      if ( q < rows ) eb[k] = s_el[q * P + 2 * a + side];
    }
  }
  // bucket unions (ranks in order, as the serial union of the reference merges them)
  const int nb = ( rows + kLeafSize - 1 ) / kLeafSize;
  T *bb = bucket_box + static_cast< size_t >( r0 / kLeafSize ) * C;
  for ( int k = tid; k < nb * C; k += kSlabThreads )
  {
    const int q = k / C, c = k - q * C;
    const int j1 = min( kLeafSize, rows - q * kLeafSize );
    T v = s_el[q * kLeafSize * P + c];
    for ( int j = 1; j < j1; ++j )
    {
      const T x = s_el[( q * kLeafSize + j ) * P + c];
      v = ( c & 1 ) ? io::mx( v, x ) : io::mn( v, x );
    }
    s_bk[q * P + c] = v;
    bb[k] = v;
  }
  __syncthreads();
  // query-group unions
  const int ng = ( nb + G - 1 ) / G;
  T *wb = warp_box + static_cast< size_t >( r0 / 32 ) * C;
  for ( int k = tid; k < ng * C; k += kSlabThreads )
  {
    const int g = k / C, c = k - g * C;
    const int j1 = min( G, nb - g * G );
    T v = s_bk[g * G * P + c];
    for ( int j = 1; j < j1; ++j )
    {
      const T x = s_bk[( g * G + j ) * P + c];
      v = ( c & 1 ) ? io::mx( v, x ) : io::mn( v, x );
    }
    wb[k] = v;
  }
  if ( n <= kLeafSize )
  {
    // one bucket: it is the tree
    T *rb = reinterpret_cast< T * >( sc->root_box );
    if ( tid < C ) rb[tid] = s_bk[tid];
    if ( tid == 0 ) sc->root = ~0;
  }
}

// Phase 1 (one thread per leaf bucket b, blocks of 128 consecutive buckets).
//
// a. The block loads its 128 bucket boxes (slabs_body wrote them) into a shared box table, one row per bucket
//    (C = 2 D components, padded to C + 1 against bank conflicts). A subtree's box lives in the row of its first
//    bucket: merging two subtrees writes the parent's node_box row (both children's slabs, with the lanes of a
//    warp acting as slab components) straight to global memory and leaves the union in the left child's row.
// b. Warp rounds (topology in registers): every lane holding an unfinished subtree [l, r] (in buckets) picks its
//    parent from the dissimilarities just outside the range; two lanes meeting on one parent are its children.
// c. Block rounds: the warps' remaining subtrees meet through shared tables indexed by the first and the last
//    bucket of each subtree (a left child with parent r looks for a subtree starting at r + 1 that targets the
//    same parent as right child; a right child with parent l - 1 for one ending at l - 1).
// d. Subtrees still unfinished publish their box into their parent's slot and are queued for phase 2 as
//    (parent * 2 + side, l, r, node).
// e. Coalesced write-out of the topology of every node closed in the block (child, range, parent).
template< int K, typename T >
__device__ void build_leaf_body(const tree_args &args, uint32_t bid, uint32_t)
{
  const int n = static_cast< int >( args.n );
  const uint64_t *__restrict__ keys = args.keys;
  uint8_t *__restrict__ bdel = args.bdel;
  const T *__restrict__ bucket_box = static_cast< const T * >( args.bucket_box );
  T *__restrict__ node_box = static_cast< T * >( args.node_box );
  int *__restrict__ child = reinterpret_cast< int * >( args.child );
  int2 *__restrict__ range = args.range;
  int *__restrict__ parent = args.parent;
  int4 *__restrict__ queue = args.queue;
  obj_scalars *sc = args.sc;
  constexpr int D = K / 2;
  constexpr int C = 2 * D;
  constexpr int W = kBuildThreads / 32;
  using io = box_io< T >;
  extern __shared__ unsigned char s_raw[];
  T *s_box = reinterpret_cast< T * >( s_raw );  // [kBuildThreads][C + 1]
  __shared__ int2 s_child[kBuildThreads];       // closed node p - bbase: global child encodings
  __shared__ int2 s_rng[kBuildThreads];         // closed node p - bbase: bucket range (x < 0: not closed here)
  __shared__ int s_pnode[kBuildThreads];        // parent entry of node p - bbase, -1 when not closed here
  __shared__ int s_pleaf[kBuildThreads];        // parent entry of bucket bbase + k
  __shared__ short s_start[kBuildThreads], s_end[kBuildThreads];
  __shared__ int s_par[kBuildThreads], s_r[kBuildThreads], s_ref[kBuildThreads], s_gn[kBuildThreads];
  __shared__ long long s_delta[kBuildThreads + 1];  // dissimilarity of buckets (bbase - 1 + k, bbase + k)
  __shared__ int4 s_pairs[kBuildThreads / 2];
  __shared__ int s_npairs, s_root_ref;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int b = static_cast< int >( bid * blockDim.x ) + tid;
  const int wbase = b - lane, bbase = b - tid;
  const int m = ( n + kLeafSize - 1 ) / kLeafSize;  // buckets
  auto box = [&](int ref, int c) -> T & { return s_box[ref * ( C + 1 ) + c]; };
  // Merge rows rl (left child) and rr (right child) of node p: the node's row of both children's slabs to global
  // memory, their union into row rl. Called by a whole warp; lanes < C each handle one component.
  auto merge = [&](int p, int rl, int rr) {
    if ( lane < C )
    {
      const T x = box( rl, lane ), y = box( rr, lane );
      T *row = node_box + static_cast< size_t >( p ) * D * 4 + ( lane >> 1 ) * 4 + ( lane & 1 );
      row[0] = x;
      row[2] = y;
      box( rl, lane ) = ( lane & 1 ) ? io::mx( x, y ) : io::mn( x, y );
    }
  };
  // A failed sort leaves no valid permutation: build nothing (the host reports the object's error word). A
  // one-bucket object got its root from the slab kernel.
  if ( *reinterpret_cast< volatile int * >( &sc->error ) == kErrTimeout || m == 1 ) return;  // uniform
  bool active = b < m;

  // a. the block's bucket boxes into the table (coalesced rows), by asynchronous copies: every copy of the thread is
  // in flight at once, and it waits for them before the barrier below
  {
    const int rows = min( kBuildThreads, m - bbase );
    const T *src = bucket_box + static_cast< size_t >( bbase ) * C;
    for ( int k = tid; k < rows * C; k += kBuildThreads )
    {
      const int row = k / C;
      cp_async_small< sizeof( T ) >( &box( row, k - row * C ), src + k );
    }
  }
  const long long dself = ( b + 1 < m ) ? bdelta( keys, b ) : 0ll;
  if ( b + 1 < m ) bdel[b] = static_cast< uint8_t >( dself >> 32 );  // for the climb: one byte per boundary
  long long dleft = 0;
  if ( lane == 0 && wbase >= 1 && wbase < m ) dleft = bdelta( keys, wbase - 1 );
  dleft = __shfl_sync( 0xffffffffu, dleft, 0 );
  s_pnode[tid] = -1;
  s_pleaf[tid] = -1;
  s_rng[tid] = make_int2( -1, -1 );
  s_start[tid] = -1;
  s_end[tid] = -1;
  s_delta[tid + 1] = dself;
  if ( tid == 0 )
  {
    s_npairs = 0;
    s_root_ref = -1;
    s_delta[0] = ( bbase >= 1 && bbase < m ) ? bdelta( keys, bbase - 1 ) : 0ll;
  }
  cp_async_wait_all();
  __syncthreads();  // the returns above are uniform over the grid

  int l = b, r = b;
  int gnode = ~b;       // child encoding of the subtree this lane holds (bucket: ~bucket)
  int ref = tid;        // its box row in the table (the row of its first bucket)
  int selfp = -1 - tid; // its parent entry: bucket (-1 - k) or closed node (p - bbase)
  int par = 0, side = 0;
  auto set_parent = [&](int entry) {
    if ( selfp < 0 ) s_pleaf[-1 - selfp] = entry;
    else s_pnode[selfp] = entry;
  };

  // b. warp rounds
  while ( true )
  {
    const long long d_r = __shfl_sync( 0xffffffffu, dself, ( r - wbase ) & 31 );
    const long long d_lm1 = __shfl_sync( 0xffffffffu, dself, ( l - 1 - wbase ) & 31 );
    if ( active )
    {
      bool left_child;
      if ( l == 0 ) left_child = true;
      else if ( r == m - 1 ) left_child = false;
      else left_child = d_r < ( l == wbase ? dleft : d_lm1 );
      par = left_child ? r : l - 1;
      side = left_child ? 0 : 1;
    }
    const unsigned peers = __match_any_sync( 0xffffffffu, active ? par : -2 - lane );
    const bool paired = active && __popc( peers ) == 2;
    const unsigned lefts = __ballot_sync( 0xffffffffu, paired && side == 0 );
    if ( !lefts ) break;
    const int src = paired ? __ffs( peers & ~( 1u << lane ) ) - 1 : lane;
    const int sref = __shfl_sync( 0xffffffffu, ref, src );
    const int sgnode = __shfl_sync( 0xffffffffu, gnode, src );
    const int sr = __shfl_sync( 0xffffffffu, r, src );
    if ( paired ) set_parent( 2 * par + side );
    if ( paired && side == 0 )
    {
      const int q = par - bbase;
      s_child[q] = make_int2( gnode, sgnode );
      s_rng[q] = make_int2( l, sr );
    }
    for ( unsigned mm = lefts; mm; mm &= mm - 1 )
    {
      const int L = __ffs( mm ) - 1;
      merge( __shfl_sync( 0xffffffffu, par, L ), __shfl_sync( 0xffffffffu, ref, L ),
             __shfl_sync( 0xffffffffu, sref, L ) );
    }
    __syncwarp();
    if ( paired )
    {
      if ( side == 0 )
      {
        r = sr;
        gnode = par;
        selfp = par - bbase;
        if ( l == 0 && r == m - 1 )
        {
          sc->root = par;
          s_root_ref = ref;
          active = false;
        }
      } else {
        active = false;
      }
    }
  }
  __syncthreads();

  // c. block rounds
  while ( true )
  {
    if ( active )
    {
      s_start[l - bbase] = static_cast< short >( tid );
      s_end[r - bbase] = static_cast< short >( tid );
      s_par[tid] = 2 * par + side;
      s_r[tid] = r;
      s_ref[tid] = ref;
      s_gn[tid] = gnode;
    }
    __syncthreads();
    int partner = -1;
    if ( active )
    {
      if ( side == 0 )
      {
        const int q = r + 1;
        if ( q < bbase + kBuildThreads && q < m )
        {
          const int c = s_start[q - bbase];
          if ( c >= 0 && s_par[c] == 2 * par + 1 ) partner = c;
        }
      } else {
        const int q = l - 1;
        if ( q >= bbase )
        {
          const int c = s_end[q - bbase];
          if ( c >= 0 && s_par[c] == 2 * par ) partner = c;
        }
      }
    }
    const bool paired = partner >= 0;
    if ( paired ) set_parent( 2 * par + side );
    if ( paired && side == 0 ) s_pairs[atomicAdd( &s_npairs, 1 )] = make_int4( tid, partner, par, 0 );
    const int any = __syncthreads_or( paired );
    if ( !any ) break;
    const int np = s_npairs;
    // closed nodes (warp w takes pairs w, w + W, ...)
    for ( int k = warp; k < np; k += W )
    {
      const int4 pr = s_pairs[k];
      merge( pr.z, s_ref[pr.x], s_ref[pr.y] );
      if ( lane == 0 ) s_child[pr.z - bbase] = make_int2( s_gn[pr.x], s_gn[pr.y] );
    }
    const int r2 = ( paired && side == 0 ) ? s_r[partner] : r;
    __syncthreads();
    if ( active )
    {
      s_start[l - bbase] = -1;
      s_end[r - bbase] = -1;
    }
    if ( paired )
    {
      if ( side == 0 )
      {
        r = r2;
        s_rng[par - bbase] = make_int2( l, r );
        gnode = par;
        selfp = par - bbase;
        if ( l == 0 && r == m - 1 )
        {
          sc->root = par;
          s_root_ref = ref;
          active = false;
        } else {
          bool left_child;
          if ( l == 0 ) left_child = true;
          else if ( r == m - 1 ) left_child = false;
          else left_child = s_delta[r - bbase + 1] < s_delta[l - bbase];
          par = left_child ? r : l - 1;
          side = left_child ? 0 : 1;
        }
      } else {
        active = false;
      }
    }
    if ( tid == 0 ) s_npairs = 0;
    __syncthreads();
  }
  // the root's box, when the whole tree closed inside this block
  if ( s_root_ref >= 0 && warp == 0 && lane < C ) reinterpret_cast< T * >( sc->root_box )[lane] = box( s_root_ref, lane );

  // d. unfinished subtrees: publish their box into the parent's slot and queue them for phase 2
  const unsigned waiting = __ballot_sync( 0xffffffffu, active );
  for ( unsigned mm = waiting; mm; mm &= mm - 1 )
  {
    const int j = __ffs( mm ) - 1;
    const int p = __shfl_sync( 0xffffffffu, par, j );
    const int sd = __shfl_sync( 0xffffffffu, side, j );
    const int rf = __shfl_sync( 0xffffffffu, ref, j );
    if ( lane < C )
      node_box[static_cast< size_t >( p ) * D * 4 + ( lane >> 1 ) * 4 + sd * 2 + ( lane & 1 )] = box( rf, lane );
  }
  if ( waiting )
  {
    unsigned base = 0;
    if ( lane == 0 ) base = atomicAdd( &sc->climb_count, static_cast< unsigned >( __popc( waiting ) ) );
    base = __shfl_sync( 0xffffffffu, base, 0 );
    if ( active )
    {
      child[2 * par + side] = gnode;
      parent[selfp < 0 ? b : m + bbase + selfp] = 2 * par + side;
      queue[base + __popc( waiting & ( ( 1u << lane ) - 1u ) )] = make_int4( 2 * par + side, l, r, gnode );
    }
  }

  // e. topology of the nodes closed in this block (their node_box rows were written at merge time)
  const int nclosed = min( kBuildThreads, m - 1 - bbase );  // internal nodes bbase .. bbase + nclosed - 1
  if ( tid < nclosed && s_rng[tid].x >= 0 )
  {
    reinterpret_cast< int2 * >( child )[bbase + tid] = s_child[tid];
    range[bbase + tid] = s_rng[tid];
    if ( s_pnode[tid] >= 0 ) parent[m + bbase + tid] = s_pnode[tid];
  }
  if ( b < m && s_pleaf[tid] >= 0 ) parent[b] = s_pleaf[tid];
}

// Phase 2 (dense, one thread per queued subtree): the agglomerative climb with a global exchange slot per node.
// The first arrival at a node leaves; the second merges and climbs on. The first arrival publishes through an
// acq_rel atomic exchange that orders its slab stores before it; the second arrival's slab loads (through L2)
// are ordered after its acquire load or exchange. Slabs written by phase 1 are visible here (kernel boundary).
template< int K, typename T >
__device__ void climb_body(const tree_args &args, uint32_t bid, uint32_t nblk)
{
  const int n = static_cast< int >( args.n );
  const uint8_t *__restrict__ bdel = args.bdel;
  T *node_box = static_cast< T * >( args.node_box );
  int *child = reinterpret_cast< int * >( args.child );
  int2 *__restrict__ range = args.range;
  int *__restrict__ parent = args.parent;
  int *exch = args.exch;
  const int4 *__restrict__ queue = args.queue;
  obj_scalars *sc = args.sc;
  constexpr int D = K / 2;
  using io = box_io< T >;
  if ( *reinterpret_cast< volatile int * >( &sc->error ) == kErrTimeout ) return;
  const int m = ( n + kLeafSize - 1 ) / kLeafSize;
  const unsigned count = *reinterpret_cast< volatile unsigned * >( &sc->climb_count );
  // A first arrival publishes the end of its range the sibling needs (its first bucket as a left child, its last as
  // a right one) together with that end's boundary dissimilarity, packed as (end << 7 | byte) while bucket indices
  // fit 24 bits: the second arrival then chooses the next parent without loading bdel.
  const bool packed = m < ( 1 << 24 );
  for ( unsigned q = bid * blockDim.x + threadIdx.x; q < count; q += nblk * blockDim.x )
  {
    const int4 w = queue[q];
    int par = w.x >> 1, side = w.x & 1, l = w.y, r = w.z;
    T lo[D], hi[D];
    {
      const T *pb = node_box + static_cast< size_t >( par ) * D * 4;
#pragma unroll
      for ( int a = 0; a < D; ++a ) io::load2_cg( pb + a * 4 + side * 2, lo[a], hi[a] );
    }
    int dl = l > 0 ? __ldg( bdel + l - 1 ) : 0;      // dissimilarity across the range's left boundary
    int dr = r < m - 1 ? __ldg( bdel + r ) : 0;      // and across its right boundary
    // A sibling that already arrived is seen with one acquire load (its slab stores were released by its
    // exchange); only when the slot looks empty does this thread publish through the exchange itself, whose
    // release also covers its own slab stores. The next level's acquire load is issued before the sibling's slabs
    // are merged, so the two round trips of a level overlap.
    int other = ld_acquire( exch + par );
    while ( true )
    {
      if ( other < 0 )
      {
        const int end = side == 0 ? l : r, dend = side == 0 ? dl : dr;
        other = atomic_exch_acq_rel( exch + par, packed ? ( end << 7 ) | dend : end );
        if ( other < 0 ) break;  // first arrival: the sibling's thread finishes this node
      }
      const int oend = packed ? other >> 7 : other;
      if ( side == 0 )
      {
        r = oend;
        dr = packed ? ( other & 127 ) : ( r < m - 1 ? __ldg( bdel + r ) : 0 );
      } else {
        l = oend;
        dl = packed ? ( other & 127 ) : ( l > 0 ? __ldg( bdel + l - 1 ) : 0 );
      }
      const T *pb = node_box + static_cast< size_t >( par ) * D * 4 + ( 1 - side ) * 2;
      T sl[D], sh[D];
#pragma unroll
      for ( int a = 0; a < D; ++a ) io::load2_cg( pb + a * 4, sl[a], sh[a] );
      range[par] = make_int2( l, r );
      if ( l == 0 && r == m - 1 )
      {
#pragma unroll
        for ( int a = 0; a < D; ++a )
        {
          lo[a] = io::mn( lo[a], sl[a] );
          hi[a] = io::mx( hi[a], sh[a] );
        }
        sc->root = par;
        store_root( sc, lo, hi );
        break;
      }
      const int node = par;
      // cdelta(r) against cdelta(l - 1): (byte << 32 | boundary index)
      const bool left_child = l == 0 || ( r != m - 1 && ( ( static_cast< long long >( dr ) << 32 ) | r ) <
                                                            ( ( static_cast< long long >( dl ) << 32 ) | ( l - 1 ) ) );
      par = left_child ? r : l - 1;
      side = left_child ? 0 : 1;
      other = ld_acquire( exch + par );
#pragma unroll
      for ( int a = 0; a < D; ++a )
      {
        lo[a] = io::mn( lo[a], sl[a] );
        hi[a] = io::mx( hi[a], sh[a] );
      }
      T *qb = node_box + static_cast< size_t >( par ) * D * 4 + side * 2;
#pragma unroll
      for ( int a = 0; a < D; ++a ) io::store2( qb + a * 4, lo[a], hi[a] );
      child[2 * par + side] = node;
      parent[m + node] = 2 * par + side;
    }
  }
}

// The climb of one subtree root whose parent node crosses the block: publishes the subtree's slabs in its parent's
// slot and meets the sibling through the node's exchange word (the protocol of the build's climb); the second
// arrival merges and goes on. lo/hi hold the subtree's slabs, ps its parent entry (2 * node + side).
template< int K, typename T >
__device__ __forceinline__ void refit_climb_global(T *node_box, const int *__restrict__ parent, int *exch,
                                                   obj_scalars *__restrict__ sc, int m, int root, int ps, T *row)
{
  constexpr int D = K / 2;
  using io = box_io< T >;
  int par = ps >> 1, side = ps & 1;
  // FP64 form. The subtree's slabs stay in its shared-memory row (registers hold only the sibling's slabs in
  // flight). The next level's parent link and this level's exchange word are read ahead: the acquire load of a level
  // is issued before the previous level's sibling slabs are merged, so the two round trips overlap.
  int nxt = par == root ? 0 : __ldg( parent + m + par );
  int other = ld_acquire( exch + par );
  while ( true )
  {
    T *pb = node_box + static_cast< size_t >( par ) * D * 4;
#pragma unroll
    for ( int a = 0; a < D; ++a ) io::store2( pb + a * 4 + side * 2, row[2 * a], row[2 * a + 1] );
    if ( other < 0 )
    {
      // the exchange's release covers the slab stores above
      other = atomic_exch_acq_rel( exch + par, 1 );
      if ( other < 0 ) return;  // first arrival: the sibling's thread finishes this node
    }
    // the sibling's slabs are read through L2, since another SM may have written them
    T sl[D], sh[D];
#pragma unroll
    for ( int a = 0; a < D; ++a ) io::load2_cg( pb + a * 4 + ( 1 - side ) * 2, sl[a], sh[a] );
    const bool at_root = par == root;
    if ( !at_root )
    {
      par = nxt >> 1;
      side = nxt & 1;
      nxt = par == root ? 0 : __ldg( parent + m + par );
      other = ld_acquire( exch + par );
    }
#pragma unroll
    for ( int a = 0; a < D; ++a )
    {
      row[2 * a] = io::mn( row[2 * a], sl[a] );
      row[2 * a + 1] = io::mx( row[2 * a + 1], sh[a] );
    }
    if ( at_root )
    {
      T lo[D], hi[D];
#pragma unroll
      for ( int a = 0; a < D; ++a )
      {
        lo[a] = row[2 * a];
        hi[a] = row[2 * a + 1];
      }
      store_root( sc, lo, hi );
      return;
    }
  }
}

// The same climb with the subtree's slabs in registers and no read-ahead of the exchange word (the FP32 form: there
// the read-ahead measured slower).
template< int K, typename T >
__device__ __forceinline__ void refit_climb_global_regs(T *node_box, const int *__restrict__ parent, int *exch,
                                                   obj_scalars *__restrict__ sc, int m, int root, int ps,
                                                   T ( &lo )[K / 2], T ( &hi )[K / 2])
{
  constexpr int D = K / 2;
  using io = box_io< T >;
  while ( true )
  {
    const int par = ps >> 1, side = ps & 1;
    // the next level's parent link is read before this level's exchange (it does not depend on it)
    const int next = par == root ? 0 : __ldg( parent + m + par );
    T *pb = node_box + static_cast< size_t >( par ) * D * 4;
#pragma unroll
    for ( int a = 0; a < D; ++a ) io::store2( pb + a * 4 + side * 2, lo[a], hi[a] );
    // a sibling that already arrived is seen with one acquire load; its slabs are read through L2, since another
    // SM may have written them
    int other = ld_acquire( exch + par );
    if ( other < 0 )
    {
      other = atomic_exch_acq_rel( exch + par, 1 );
      if ( other < 0 ) return;  // first arrival: the sibling's thread finishes this node
    }
#pragma unroll
    for ( int a = 0; a < D; ++a )
    {
      T sl, sh;
      io::load2_cg( pb + a * 4 + ( 1 - side ) * 2, sl, sh );
      lo[a] = io::mn( lo[a], sl );
      hi[a] = io::mx( hi[a], sh );
    }
    if ( par == root )
    {
      store_root( sc, lo, hi );
      return;
    }
    ps = next;
  }
}

// Refit: new slabs for every node of an unchanged topology. Block `bid` owns buckets [B0, B0 + blockDim.x) and the
// window of internal nodes with the same indices. Internal node k splits its bucket range [l, r] at k (l <= k < r),
// so every node whose range lies inside the block's buckets (a local node) is in the window. The local nodes are
// refit in rounds over shared memory: a subtree [l, r] keeps its slabs in row l - B0 of s_tab (its first bucket's
// row), and in each round every local node whose children are done merges their rows, writes both children's
// slabs to its node_box row and leaves the union in its row. Barriers separate the rounds, so no exchange word,
// atomic or fence is used inside the block. Then every local root (a bucket or local node whose parent crosses the
// block) climbs through the crossing nodes with the global exchange.
template< int K, typename T >
__device__ void refit_body(const tree_args &args, uint32_t bid, uint32_t)
{
  const int n = static_cast< int >( args.n );
  const T *__restrict__ bucket_box = static_cast< const T * >( args.bucket_box );
  T *node_box = static_cast< T * >( args.node_box );
  const int2 *__restrict__ child = args.child;
  const int *__restrict__ parent = args.parent;
  const int2 *__restrict__ range = args.range;
  int *exch = args.exch;
  obj_scalars *__restrict__ sc = args.sc;
  constexpr int D = K / 2;
  constexpr int C = 2 * D;
  using io = box_io< T >;
  static_assert( ( C * sizeof( T ) ) % 8 == 0, "rows of slab pairs" );
  __shared__ alignas( 16 ) T s_tab[kBuildThreads * C];  // bucket rows (contiguous, as in bucket_box), then subtrees
  __shared__ int2 s_child[kBuildThreads];
  __shared__ int2 s_rng[kBuildThreads];
  __shared__ int s_up[kBuildThreads];
  __shared__ unsigned char s_done[kBuildThreads];
  __shared__ int s_list[kBuildThreads];
  __shared__ int s_wcnt[kBuildThreads / 32];
  const int B0 = static_cast< int >( bid * blockDim.x );
  const int tid = static_cast< int >( threadIdx.x );
  const int m = ( n + kLeafSize - 1 ) / kLeafSize;
  // a one-bucket object's root box came from the slab kernel; a failed sort leaves nothing to refit (both uniform)
  if ( m == 1 || *reinterpret_cast< volatile int * >( &sc->error ) == kErrTimeout ) return;
  const int rows = min( static_cast< int >( blockDim.x ), m - B0 );
  const int nodes_here = min( static_cast< int >( blockDim.x ), m - 1 - B0 );  // internal nodes of the window
  {
    // the block's bucket rows: 16-byte asynchronous copies (the block's first row starts on a 16-byte boundary:
    // B0 * C * sizeof(T) is a multiple of 128 * 8), the last few bytes of a ragged block by plain loads
    const int bytes = rows * C * static_cast< int >( sizeof( T ) );
    const unsigned char *src = reinterpret_cast< const unsigned char * >( bucket_box + static_cast< size_t >( B0 ) * C );
    unsigned char *dst = reinterpret_cast< unsigned char * >( s_tab );
    for ( int o = tid * 16; o + 16 <= bytes; o += blockDim.x * 16 ) cp_async16( dst + o, src + o );
    const int tail = bytes & ~15;
    for ( int o = tail + tid * static_cast< int >( sizeof( T ) ); o < bytes; o += blockDim.x * sizeof( T ) )
      *reinterpret_cast< T * >( dst + o ) = *reinterpret_cast< const T * >( src + o );
  }
  if ( tid < nodes_here )
  {
    s_child[tid] = __ldg( child + B0 + tid );
    s_rng[tid] = __ldg( range + B0 + tid );
    s_up[tid] = __ldg( parent + m + B0 + tid );
  }
  const int root = sc->root;
  int pb_entry = tid < rows ? __ldg( parent + B0 + tid ) : 0;  // this thread's bucket's parent entry
  cp_async_wait_all();
  __syncthreads();
  auto is_local = [&](int node) {
    if ( node < B0 || node - B0 >= nodes_here ) return false;
    const int2 rg = s_rng[node - B0];
    return rg.x >= B0 && rg.y < B0 + static_cast< int >( blockDim.x );
  };
  const bool mine = is_local( B0 + tid );  // this thread owns node B0 + tid, refit in the rounds
  bool pending = mine;
  s_done[tid] = 0;
  // rounds: the nodes whose children are buckets or done nodes are listed, then merged by groups of D lanes (lane
  // a: axis a of both children, so a node's node_box row is written by one coalesced store per group); barriers
  // order one round's rows and flags before the next round's reads
  constexpr int G = 32 / D;  // node groups per warp
  const int lane = tid & 31, warp = tid >> 5, nwarps = static_cast< int >( blockDim.x ) >> 5;
  while ( __syncthreads_or( pending ) )
  {
    bool ready = false;
    if ( pending )
    {
      const int2 c = s_child[tid];
      ready = ( c.x < 0 || s_done[c.x - B0] ) && ( c.y < 0 || s_done[c.y - B0] );
    }
    const unsigned bal = __ballot_sync( 0xffffffffu, ready );
    if ( lane == 0 ) s_wcnt[warp] = __popc( bal );
    __syncthreads();
    int off = 0, total = 0;
    for ( int w = 0; w < nwarps; ++w )
    {
      const int c = s_wcnt[w];
      off += w < warp ? c : 0;
      total += c;
    }
    if ( ready ) s_list[off + __popc( bal & ( ( 1u << lane ) - 1u ) )] = tid;
    __syncthreads();
    if ( lane < G * D )
    {
      const int a = lane % D;
      for ( int e = warp * G + lane / D; e < total; e += nwarps * G )
      {
        const int q = s_list[e];
        const int node = B0 + q;
        T *L = s_tab + ( s_rng[q].x - B0 ) * C;  // the left child's row (its range starts at the node's)
        const T *R = s_tab + ( node + 1 - B0 ) * C;  // the right child's row
        T ll, lh, rlo, rhi;
        io::load2( L + 2 * a, ll, lh );
        io::load2( R + 2 * a, rlo, rhi );
        io::store4( node_box + static_cast< size_t >( node ) * D * 4 + a * 4, ll, lh, rlo, rhi );
        io::store2( L + 2 * a, io::mn( ll, rlo ), io::mx( lh, rhi ) );
      }
    }
    __syncthreads();
    if ( ready )
    {
      if ( B0 + tid == root )
      {
        const T *L = s_tab + ( s_rng[tid].x - B0 ) * C;
        T lo[D], hi[D];
#pragma unroll
        for ( int a = 0; a < D; ++a ) io::load2( L + 2 * a, lo[a], hi[a] );
        store_root( sc, lo, hi );
      }
      s_done[tid] = 1;
      pending = false;
    }
  }
  // local roots climb through the crossing nodes: this thread's bucket when its parent is not local, and its node
  // when it is local and its parent is not
  // (each local root's row belongs to its climbing thread alone)
  auto climb_from = [&](int ps, int row) {
    if constexpr ( sizeof( T ) == 8 )
    {
      refit_climb_global< K, T >( node_box, parent, exch, sc, m, root, ps, s_tab + row * C );
    } else {
      T lo[D], hi[D];
#pragma unroll
      for ( int a = 0; a < D; ++a ) io::load2( s_tab + row * C + 2 * a, lo[a], hi[a] );
      refit_climb_global_regs< K, T >( node_box, parent, exch, sc, m, root, ps, lo, hi );
    }
  };
  if ( tid < rows && !is_local( pb_entry >> 1 ) ) climb_from( pb_entry, tid );
  if ( mine && B0 + tid != root && !is_local( s_up[tid] >> 1 ) ) climb_from( s_up[tid], s_rng[tid].x - B0 );
}

uint32_t slab_grid(uint64_t n) { return static_cast< uint32_t >( ( n + kSlabThreads - 1 ) / kSlabThreads ); }

template< int K, typename T, int VT >
cudaError_t launch_slabs_t(const slabs_args &a, cudaStream_t s)
{
  k_single< slabs_args, slabs_body< K, T, VT >, kSlabThreads, kSlabMinBlocks< K, VT > ><<< slab_grid( a.n ), kSlabThreads, 0, s >>>( a );
  return cudaGetLastError();
}

template< int K, typename T, int VT >
cudaError_t launch_slabs_batch_t(const batch_launch &b, cudaStream_t s)
{
  k_batched< slabs_args, slabs_body< K, T, VT >, kSlabThreads, kSlabMinBlocks< K, VT > ><<< b.blocks, kSlabThreads, 0, s >>>(
    static_cast< const slabs_args * >( b.items ), b.starts, b.nitems );
  return cudaGetLastError();
}

template< int K, typename T >
cudaError_t slabs_v(const slabs_args &a, cudaStream_t s)
{
  switch ( a.V )
  {
    case 3: return launch_slabs_t< K, T, 3 >( a, s );
    case 4: return launch_slabs_t< K, T, 4 >( a, s );
    case 8: return launch_slabs_t< K, T, 8 >( a, s );
    default: return launch_slabs_t< K, T, 0 >( a, s );
  }
}

template< int K, typename T >
cudaError_t slabs_batch_v(uint32_t V, const batch_launch &b, cudaStream_t s)
{
  switch ( V )
  {
    case 3: return launch_slabs_batch_t< K, T, 3 >( b, s );
    case 4: return launch_slabs_batch_t< K, T, 4 >( b, s );
    case 8: return launch_slabs_batch_t< K, T, 8 >( b, s );
    default: return launch_slabs_batch_t< K, T, 0 >( b, s );
  }
}

uint32_t build_grid(uint64_t n)
{
  const uint64_t m = ( n + kLeafSize - 1 ) / kLeafSize;
  return m <= 1 ? 0u : static_cast< uint32_t >( ( m + kBuildThreads - 1 ) / kBuildThreads );
}

template< int K, typename T >
constexpr size_t kBuildSmem = static_cast< size_t >( kBuildThreads ) * ( 2 * ( K / 2 ) + 1 ) * sizeof( T );  // [rows][C + 1]

template< int K, typename T >
cudaError_t build_setup()
{
  cudaError_t e = cudaFuncSetAttribute( k_single< tree_args, build_leaf_body< K, T >, kBuildThreads, 8 >,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast< int >( kBuildSmem< K, T > ) );
  if ( e != cudaSuccess ) return e;
  return cudaFuncSetAttribute( k_batched< tree_args, build_leaf_body< K, T >, kBuildThreads, 8 >,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast< int >( kBuildSmem< K, T > ) );
}

template< int K, typename T >
cudaError_t launch_build_t(const tree_args &a, cudaStream_t s)
{
  const uint32_t grid = build_grid( a.n );
  if ( !grid ) return cudaSuccess;  // the slab kernel stored a one-bucket object's root
  const cudaError_t e = build_setup< K, T >();
  if ( e != cudaSuccess ) return e;
  k_single< tree_args, build_leaf_body< K, T >, kBuildThreads, 8 ><<< grid, kBuildThreads, kBuildSmem< K, T >, s >>>( a );
  return cudaGetLastError();
}

template< int K, typename T >
cudaError_t launch_build_batch_t(const batch_launch &b, cudaStream_t s)
{
  const cudaError_t e = build_setup< K, T >();
  if ( e != cudaSuccess ) return e;
  k_batched< tree_args, build_leaf_body< K, T >, kBuildThreads, 8 ><<< b.blocks, kBuildThreads, kBuildSmem< K, T >, s >>>(
    static_cast< const tree_args * >( b.items ), b.starts, b.nitems );
  return cudaGetLastError();
}

// The queue length is known only on the device: a grid-stride grid sized for the usual fraction.
uint32_t climb_grid(uint64_t n)
{
  const uint64_t m = ( n + kLeafSize - 1 ) / kLeafSize;
  const uint64_t want = ( m / 8 + 127 ) / 128;
  return static_cast< uint32_t >( want < 148 * 16 ? ( want ? want : 1 ) : 148 * 16 );
}

template< int K, typename T >
cudaError_t launch_climb_t(const tree_args &a, cudaStream_t s)
{
  k_single< tree_args, climb_body< K, T >, 128, 4 ><<< climb_grid( a.n ), 128, 0, s >>>( a );
  return cudaGetLastError();
}

template< int K, typename T >
cudaError_t launch_climb_batch_t(const batch_launch &b, cudaStream_t s)
{
  k_batched< tree_args, climb_body< K, T >, 128, 4 ><<< b.blocks, 128, 0, s >>>( static_cast< const tree_args * >( b.items ),
                                                                               b.starts, b.nitems );
  return cudaGetLastError();
}

uint32_t refit_grid(uint64_t n)
{
  const uint64_t m = ( n + kLeafSize - 1 ) / kLeafSize;
  return m <= 1 ? 0u : static_cast< uint32_t >( ( m + kBuildThreads - 1 ) / kBuildThreads );
}

template< int K, typename T >
cudaError_t launch_refit_t(const tree_args &a, cudaStream_t s)
{
  const uint32_t grid = refit_grid( a.n );
  if ( !grid ) return cudaSuccess;
  k_single< tree_args, refit_body< K, T >, kBuildThreads, 7 ><<< grid, kBuildThreads, 0, s >>>( a );
  return cudaGetLastError();
}

template< int K, typename T >
cudaError_t launch_refit_batch_t(const batch_launch &b, cudaStream_t s)
{
  k_batched< tree_args, refit_body< K, T >, kBuildThreads, 7 ><<< b.blocks, kBuildThreads, 0, s >>>(
    static_cast< const tree_args * >( b.items ), b.starts, b.nitems );
  return cudaGetLastError();
}

// Original-order slabs (parity probe).
template< int K, typename T, int VT >
__global__ void k_probe_kdops(const double *__restrict__ verts, uint32_t Vrt, uint64_t n, double eps, float eps_hi,
                              T *__restrict__ out)
{
  constexpr int D = K / 2;
  const uint64_t i = static_cast< uint64_t >( blockIdx.x ) * blockDim.x + threadIdx.x;
  if ( i >= n ) return;
  T lo[D], hi[D];
  leaf_slabs< K, T, VT >( verts, Vrt, static_cast< uint32_t >( i ), eps, eps_hi, lo, hi );
  for ( int a = 0; a < D; ++a )
  {
    out[( i * D + a ) * 2] = lo[a];
    out[( i * D + a ) * 2 + 1] = hi[a];
  }
}

template< int K, typename T >
cudaError_t probe_v(const double *verts, uint32_t V, uint64_t n, double eps, void *out, cudaStream_t s)
{
  const float eps_hi = f32_round_up( eps );
  const unsigned grid = static_cast< unsigned >( ( n + 255 ) / 256 );
  if ( V == 3 ) k_probe_kdops< K, T, 3 ><<< grid, 256, 0, s >>>( verts, V, n, eps, eps_hi, static_cast< T * >( out ) );
  else if ( V == 4 ) k_probe_kdops< K, T, 4 ><<< grid, 256, 0, s >>>( verts, V, n, eps, eps_hi, static_cast< T * >( out ) );
  else if ( V == 8 ) k_probe_kdops< K, T, 8 ><<< grid, 256, 0, s >>>( verts, V, n, eps, eps_hi, static_cast< T * >( out ) );
  else k_probe_kdops< K, T, 0 ><<< grid, 256, 0, s >>>( verts, V, n, eps, eps_hi, static_cast< T * >( out ) );
  return cudaGetLastError();
}

}  // namespace

#define BVHG_BY_K( CALL_F, CALL_D )                                                                                    \
  switch ( K )                                                                                                         \
  {                                                                                                                    \
    case 6: return fp32 ? CALL_F( 6 ) : CALL_D( 6 );                                                                   \
    case 18: return fp32 ? CALL_F( 18 ) : CALL_D( 18 );                                                                \
    case 26: return fp32 ? CALL_F( 26 ) : CALL_D( 26 );                                                                \
    default: return cudaErrorInvalidValue;                                                                             \
  }

cudaError_t launch_slabs(int K, bool fp32, const double *verts, uint32_t V, uint64_t n, double eps,
                         const uint32_t *vals, void *bucket_box, void *warp_box, void *elem_rows, obj_scalars *sc,
                         cudaStream_t s)
{
  const slabs_args a{ verts, V, n, eps, f32_round_up( eps ), vals, bucket_box, warp_box, elem_rows, sc };
#define F( KK ) slabs_v< KK, float >( a, s )
#define D( KK ) slabs_v< KK, double >( a, s )
  BVHG_BY_K( F, D )
#undef F
#undef D
}

uint32_t slabs_blocks(uint64_t n) { return slab_grid( n ); }

cudaError_t launch_slabs_batch(int K, bool fp32, uint32_t V, const batch_launch &b, cudaStream_t s)
{
  if ( !b.nitems ) return cudaSuccess;
#define F( KK ) slabs_batch_v< KK, float >( V, b, s )
#define D( KK ) slabs_batch_v< KK, double >( V, b, s )
  BVHG_BY_K( F, D )
#undef F
#undef D
}

cudaError_t launch_build(int K, bool fp32, uint64_t n, const uint64_t *keys, uint8_t *bdel, const void *bucket_box,
                         void *node_box, int2 *child, int2 *range, int *parent, int4 *queue, obj_scalars *sc,
                         cudaStream_t s)
{
  const tree_args a{ n, keys, bdel, bucket_box, node_box, child, range, parent, nullptr, queue, sc };
#define F( KK ) launch_build_t< KK, float >( a, s )
#define D( KK ) launch_build_t< KK, double >( a, s )
  BVHG_BY_K( F, D )
#undef F
#undef D
}

uint32_t build_blocks(uint64_t n) { return build_grid( n ); }

cudaError_t launch_build_batch(int K, bool fp32, const batch_launch &b, cudaStream_t s)
{
  if ( !b.nitems ) return cudaSuccess;
#define F( KK ) launch_build_batch_t< KK, float >( b, s )
#define D( KK ) launch_build_batch_t< KK, double >( b, s )
  BVHG_BY_K( F, D )
#undef F
#undef D
}

cudaError_t launch_climb(int K, bool fp32, uint64_t n, const uint8_t *bdel, void *node_box, int2 *child, int2 *range,
                         int *parent, int *exch, const int4 *queue, obj_scalars *sc, cudaStream_t s)
{
  const tree_args a{ n, nullptr, const_cast< uint8_t * >( bdel ), nullptr, node_box, child, range, parent, exch,
                     const_cast< int4 * >( queue ), sc };
#define F( KK ) launch_climb_t< KK, float >( a, s )
#define D( KK ) launch_climb_t< KK, double >( a, s )
  BVHG_BY_K( F, D )
#undef F
#undef D
}

uint32_t climb_blocks(uint64_t n) { return climb_grid( n ); }

cudaError_t launch_climb_batch(int K, bool fp32, const batch_launch &b, cudaStream_t s)
{
  if ( !b.nitems ) return cudaSuccess;
#define F( KK ) launch_climb_batch_t< KK, float >( b, s )
#define D( KK ) launch_climb_batch_t< KK, double >( b, s )
  BVHG_BY_K( F, D )
#undef F
#undef D
}

cudaError_t launch_refit(int K, bool fp32, uint64_t n, const void *bucket_box, void *node_box, const int2 *child,
                         const int2 *range, const int *parent, int *exch, obj_scalars *sc, cudaStream_t s)
{
  const tree_args a{ n, nullptr, nullptr, bucket_box, node_box, const_cast< int2 * >( child ), const_cast< int2 * >( range ),
                     const_cast< int * >( parent ), exch, nullptr, sc };
#define F( KK ) launch_refit_t< KK, float >( a, s )
#define D( KK ) launch_refit_t< KK, double >( a, s )
  BVHG_BY_K( F, D )
#undef F
#undef D
}

uint32_t refit_blocks(uint64_t n) { return refit_grid( n ); }

cudaError_t launch_refit_batch(int K, bool fp32, const batch_launch &b, cudaStream_t s)
{
  if ( !b.nitems ) return cudaSuccess;
#define F( KK ) launch_refit_batch_t< KK, float >( b, s )
#define D( KK ) launch_refit_batch_t< KK, double >( b, s )
  BVHG_BY_K( F, D )
#undef F
#undef D
}

#undef BVHG_BY_K

cudaError_t launch_probe_kdops(int K, bool fp32, const double *verts, uint32_t V, uint64_t n, double eps, void *out,
                               cudaStream_t s)
{
  switch ( K )
  {
    case 6: return fp32 ? probe_v< 6, float >( verts, V, n, eps, out, s ) : probe_v< 6, double >( verts, V, n, eps, out, s );
    case 18: return fp32 ? probe_v< 18, float >( verts, V, n, eps, out, s ) : probe_v< 18, double >( verts, V, n, eps, out, s );
    case 26: return fp32 ? probe_v< 26, float >( verts, V, n, eps, out, s ) : probe_v< 26, double >( verts, V, n, eps, out, s );
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace bvhg
