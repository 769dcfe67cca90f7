// bvh_oracle.cpp — CPU restatement of distBVH's per-rank element broadphase arithmetic.
//
// TEST INFRASTRUCTURE ONLY. This file is the parity checker for the CUDA path in distbvh_b200/csrc.
// Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load it; the product library never
// links, calls or falls back to it.
//
// Parity pinning: tests/test_oracle_golden.py checks every function here against the known answers in the
// reference's own unit tests (tests/hash_test.cpp, tests/sort_test.cpp, tests/UtilTest.cpp,
// tests/KDopTest.cpp, tests/CollisionTest.cpp, tests/snapshot_test.cpp) and, when oracle/_ref was built
// from the reference headers, against the reference code itself on seeded random inputs.
//
// Build flags matter for bit-exactness: -O2 -ffp-contract=off and no -ffast-math, so that every FP64
// product and sum is rounded separately, exactly as written in the reference source (the reference's
// Release build adds -ffast-math, CMakeLists.txt:65; the intended arithmetic is the source order).
//
// Element layout used throughout: xyz[(i * V + v) * 3 + c] is coordinate c of vertex v of element i.
// k-DOP layout: slabs[(i * D + a) * 2 + {0: min, 1: max}] for axis a < D = K / 2.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <numeric>
#include <vector>

namespace {

constexpr double kOverRoot2 = 0.7071067811865475;   // kdop.hpp:608 and kdop.hpp:659 (as a double literal)
constexpr double kOverRoot3 = 0.5773502691896258;   // kdop.hpp:660

struct vec3 { double x, y, z; };

// The first K/2 normals of dop_6 (kdop.hpp:583-587), dop_18 (kdop.hpp:613-624) and dop_26 (kdop.hpp:662-677).
// Only the first K/2 entries of each table are ever read (from_vertices loops over num_axis = K/2).
int normal_table(int K, vec3 *out)
{
  const double r = kOverRoot2, s = kOverRoot3;
  const vec3 card[3] = { { 1., 0., 0. }, { 0., 1., 0. }, { 0., 0., 1. } };
  const vec3 edges[6] = { { r, r, 0. }, { r, 0., r }, { 0., r, r }, { r, -r, 0. }, { r, 0., -r }, { 0., r, -r } };
  const vec3 corners[4] = { { s, s, s }, { s, -s, s }, { s, s, -s }, { s, -s, -s } };
  int n = 0;
  for ( auto &c : card ) out[n++] = c;
  if ( K == 6 ) return n;
  if ( K == 18 )
  {
    for ( auto &e : edges ) out[n++] = e;
    return n;
  }
  if ( K == 26 )
  {
    for ( auto &c : corners ) out[n++] = c;
    for ( auto &e : edges ) out[n++] = e;
    return n;
  }
  return -1;
}

// kdop.hpp:223-227: _v[0] * ax[0] + _v[1] * ax[1] + _v[2] * ax[2], evaluated left to right.
inline double project(const double *v, const vec3 &a)
{
  double t0 = v[0] * a.x;
  double t1 = v[1] * a.y;
  double t2 = v[2] * a.z;
  return ( t0 + t1 ) + t2;
}

// std::min / std::max as libstdc++ defines them: min(a, b) = (b < a) ? b : a, max(a, b) = (a < b) ? b : a.
inline double std_min(double a, double b) { return ( b < a ) ? b : a; }
inline double std_max(double a, double b) { return ( a < b ) ? b : a; }

// hash.hpp:72-81 (expand64) and hash.hpp:100-103 (morton64).
inline std::uint64_t expand64(std::uint64_t v)
{
  v = ( v * 0x1000001u ) & 0xfff000000fffu;
  v = ( v * 0x1001u ) & 0xfc003f000fc003fu;
  v = ( v * 0x41u ) & 0x01c0e070381c0e07u;
  v = ( v * 0x11u ) & 0x10c86432190c8643u;
  v = ( v * 0x5u ) & 0x1249249249249249u;
  return v;
}

inline std::uint32_t expand32(std::uint32_t v)
{
  v = ( v * 0x00010001u ) & 0xff0000ffu;
  v = ( v * 0x00000101u ) & 0x0f00f00fu;
  v = ( v * 0x00000011u ) & 0xc30c30c3u;
  v = ( v * 0x00000005u ) & 0x49249249u;
  return v;
}

// Truncating FP64 -> u64 conversion as x86-64 gcc emits it for static_cast<std::uint64_t>(double):
// values below 2^63 take the signed truncating path (so (-1, 0) -> 0), NaN -> 0x8000000000000000.
// Only the low 21 bits survive the mask in quantize64, where both give the same answer as the GPU's
// saturating cvt.rzi.u64.f64 for every value the pipeline can produce.
inline std::uint64_t to_u64(double x)
{
  if ( std::isnan( x ) ) return 0x8000000000000000ull;
  if ( x < 9223372036854775808.0 )
    return static_cast< std::uint64_t >( static_cast< std::int64_t >( x ) );
  return static_cast< std::uint64_t >( static_cast< std::int64_t >( x - 9223372036854775808.0 ) ) ^ 0x8000000000000000ull;
}

struct kdop_view
{
  const double *s;   // D (min, max) pairs
  int D;
};

// kdop.hpp:120-125 + kdop.hpp:538-549: strict overlap on every slab.
inline bool overlap(const double *a, const double *b, int D)
{
  for ( int k = 0; k < D; ++k )
  {
    if ( !( a[2 * k] < b[2 * k + 1] && b[2 * k] < a[2 * k + 1] ) )
      return false;
  }
  return true;
}

}  // namespace

extern "C" {

int orc_version() { return 1; }

// Normal table (first K/2 normals). Returns the count or -1 for an unsupported K.
int orc_normals(int K, double *out3)
{
  vec3 n[13];
  int c = normal_table( K, n );
  for ( int i = 0; i < c; ++i )
  {
    out3[3 * i + 0] = n[i].x;
    out3[3 * i + 1] = n[i].y;
    out3[3 * i + 2] = n[i].z;
  }
  return c;
}

double orc_project(const double *v, const double *axis)
{
  vec3 a{ axis[0], axis[1], axis[2] };
  return project( v, a );
}

// kdop_base::from_vertices, kdop.hpp:238-264, for n elements of V vertices each.
int orc_kdops(const double *xyz, std::uint32_t V, std::uint64_t n, int K, double eps, double *out)
{
  vec3 nt[13];
  const int D = normal_table( K, nt );
  if ( D < 0 || V == 0 ) return -1;
  for ( std::uint64_t i = 0; i < n; ++i )
  {
    const double *verts = xyz + i * V * 3;
    double *o = out + i * D * 2;
    for ( int a = 0; a < D; ++a )
    {
      double proj = project( verts, nt[a] );
      double mn = proj - eps;
      double mx = proj + eps;
      for ( std::uint32_t v = 1; v < V; ++v )
      {
        proj = project( verts + 3 * v, nt[a] );
        mn = std_min( mn, proj - eps );
        mx = std_max( mx, proj + eps );
      }
      o[2 * a] = mn;
      o[2 * a + 1] = mx;
    }
  }
  return D;
}

// Element centroid as the reference test element computes it: accumulate from zeros, then a true division by
// the vertex count (tests/TestCommon.hpp:62-65; m::vec division is component-wise '/',
// math/ops/vec_arithmetic_ops.hpp:238-252).
void orc_centroids(const double *xyz, std::uint32_t V, std::uint64_t n, double *out)
{
  const double cnt = static_cast< double >( V );
  for ( std::uint64_t i = 0; i < n; ++i )
  {
    const double *verts = xyz + i * V * 3;
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for ( std::uint32_t v = 0; v < V; ++v )
    {
      sx = sx + verts[3 * v + 0];
      sy = sy + verts[3 * v + 1];
      sz = sz + verts[3 * v + 2];
    }
    out[3 * i + 0] = sx / cnt;
    out[3 * i + 1] = sy / cnt;
    out[3 * i + 2] = sz / cnt;
  }
}

// compute_bounds(min_inv_diag_bounds), contact_entity.hpp:67-80 (reduction body), 136-148 (1/(max-min)).
// The reduction is written with serial semantics: the reference's join (contact_entity.hpp:90) drops the
// source partial max, which only matters for a partitioned multithreaded reduction. min/max are exact, so
// any order of the reduction gives these bits. Kokkos::min/max: (a < b ? a : b), (a > b ? a : b).
// Initial values are the reduction identity: +max and lowest.
void orc_morton_bounds(const double *slabs, std::uint64_t n, int K, double *min3, double *inv3)
{
  const int D = K / 2;
  double mn[3], mx[3];
  for ( int c = 0; c < 3; ++c )
  {
    mn[c] = std::numeric_limits< double >::max();
    mx[c] = std::numeric_limits< double >::lowest();
  }
  for ( std::uint64_t i = 0; i < n; ++i )
  {
    const double *s = slabs + i * D * 2;
    for ( int c = 0; c < 3; ++c )
    {
      const double cmin = s[2 * c], cmax = s[2 * c + 1];
      mn[c] = ( cmin < mn[c] ) ? cmin : mn[c];
      mx[c] = ( cmax > mx[c] ) ? cmax : mx[c];
    }
  }
  for ( int c = 0; c < 3; ++c )
  {
    const double width = mx[c] - mn[c];
    min3[c] = mn[c];
    inv3[c] = 1.0 / width;
  }
}

// quantize64, hash.hpp:177-198: q = u64(((p - min) * inv) * 2097152) & 0x1fffff per axis.
void orc_quantize64(const double *p, const double *min3, const double *inv3, std::uint64_t *q3)
{
  for ( int c = 0; c < 3; ++c )
  {
    const double norm = ( p[c] - min3[c] ) * inv3[c];
    const double scaled = norm * 2097152.0;
    q3[c] = to_u64( scaled ) & 0x1fffffull;
  }
}

// quantize32, hash.hpp:146-167 (10 bits per axis).
void orc_quantize32(const double *p, const double *min3, const double *inv3, std::uint32_t *q3)
{
  for ( int c = 0; c < 3; ++c )
  {
    const double norm = ( p[c] - min3[c] ) * inv3[c];
    const double scaled = norm * 1024.0;
    q3[c] = static_cast< std::uint32_t >( to_u64( scaled ) ) & 0x3ffu;
  }
}

std::uint64_t orc_morton64(std::uint64_t x, std::uint64_t y, std::uint64_t z)
{
  return ( expand64( z ) << 2u ) | ( expand64( y ) << 1u ) | expand64( x );
}

// hash.hpp:106-110 (32-bit morton, additions instead of ors: the fields never overlap).
std::uint32_t orc_morton32(std::uint32_t x, std::uint32_t y, std::uint32_t z)
{
  return ( expand32( z ) << 2 ) + ( expand32( y ) << 1 ) + expand32( x );
}

// morton_impl, contact_entity.hpp:104-118 with T = u64: key = morton(quantize64(centroid, min, inv)).
void orc_morton_keys(const double *centroids, std::uint64_t n, const double *min3, const double *inv3,
                     std::uint64_t *keys)
{
  for ( std::uint64_t i = 0; i < n; ++i )
  {
    std::uint64_t q[3];
    orc_quantize64( centroids + 3 * i, min3, inv3, q );
    keys[i] = orc_morton64( q[0], q[1], q[2] );
  }
}

// prefix_sum, util/prefix_sum.hpp:41-54: exclusive scan in place.
void orc_exclusive_scan_i64(std::int64_t *v, std::uint64_t n)
{
  std::int64_t acc = 0;
  for ( std::uint64_t i = 0; i < n; ++i )
  {
    const std::int64_t x = v[i];
    v[i] = acc;
    acc += x;
  }
}

}  // extern "C"

// radix_sorter::operator() + step, util/sort.hpp:98-136: one bit per pass, all 8*sizeof(key) passes, each
// pass a flag map, an exclusive scan of the zero-flags and a stable split scatter of key and index.
template< typename Key >
static void radix_sort_1bit(Key *keys, std::uint64_t *idx, std::uint64_t n, unsigned passes)
{
  if ( n == 0 ) return;
  std::vector< Key > ks( n );
  std::vector< std::uint64_t > is( n );
  std::vector< Key > bits( n ), scan( n );
  Key *src_k = keys, *dst_k = ks.data();
  std::uint64_t *src_i = idx, *dst_i = is.data();
  for ( unsigned p = 0; p < passes; ++p )
  {
    for ( std::uint64_t i = 0; i < n; ++i )
    {
      const Key h = src_k[i] >> p;
      bits[i] = ~h & 0x1;
      scan[i] = bits[i];
    }
    Key acc = 0;
    for ( std::uint64_t i = 0; i < n; ++i )
    {
      const Key x = scan[i];
      scan[i] = acc;
      acc += x;
    }
    const Key total = scan[n - 1] + bits[n - 1];
    for ( std::uint64_t i = 0; i < n; ++i )
    {
      const Key t = static_cast< Key >( i ) - scan[i] + total;
      const Key new_idx = bits[i] ? scan[i] : t;
      dst_i[new_idx] = src_i[i];
      dst_k[new_idx] = src_k[i];
    }
    std::swap( src_k, dst_k );
    std::swap( src_i, dst_i );
  }
  if ( src_k != keys )
  {
    std::memcpy( keys, src_k, n * sizeof( Key ) );
    std::memcpy( idx, src_i, n * sizeof( std::uint64_t ) );
  }
}

extern "C" {

void orc_radix_sort_1bit_u64(std::uint64_t *keys, std::uint64_t *idx, std::uint64_t n)
{
  radix_sort_1bit< std::uint64_t >( keys, idx, n, 64 );
}

void orc_radix_sort_1bit_u32(std::uint32_t *keys, std::uint64_t *idx, std::uint64_t n)
{
  radix_sort_1bit< std::uint32_t >( keys, idx, n, 32 );
}

// The permutation a stable sort of (key, original index) yields: unique, so equal to the 1-bit radix
// sorter's output for any input. perm[r] = original index of the element of rank r.
void orc_stable_sort_perm_u64(const std::uint64_t *keys, std::uint64_t n, std::uint32_t *perm)
{
  std::vector< std::uint32_t > p( n );
  std::iota( p.begin(), p.end(), 0u );
  std::stable_sort( p.begin(), p.end(), [keys](std::uint32_t a, std::uint32_t b) { return keys[a] < keys[b]; } );
  std::memcpy( perm, p.data(), n * sizeof( std::uint32_t ) );
}

int orc_overlap(const double *a, const double *b, int K)
{
  return overlap( a, b, K / 2 ) ? 1 : 0;
}

// Pair set S(A, B) by brute force: every (i, j) with strict overlap on every slab. Pairs are local indices
// (i into A, j into B), written as out[2p], out[2p+1] while p < cap. Returns |S|.
std::int64_t orc_pairs_brute(const double *sa, std::uint64_t na, const double *sb, std::uint64_t nb, int K,
                             std::uint32_t *out, std::uint64_t cap)
{
  const int D = K / 2;
  std::int64_t cnt = 0;
  for ( std::uint64_t i = 0; i < na; ++i )
    for ( std::uint64_t j = 0; j < nb; ++j )
      if ( overlap( sa + i * D * 2, sb + j * D * 2, D ) )
      {
        if ( static_cast< std::uint64_t >( cnt ) < cap )
        {
          out[2 * cnt] = static_cast< std::uint32_t >( i );
          out[2 * cnt + 1] = static_cast< std::uint32_t >( j );
        }
        ++cnt;
      }
  return cnt;
}

// Self pair set by brute force: i < j.
std::int64_t orc_self_pairs_brute(const double *s, std::uint64_t n, int K, std::uint32_t *out, std::uint64_t cap)
{
  const int D = K / 2;
  std::int64_t cnt = 0;
  for ( std::uint64_t i = 0; i < n; ++i )
    for ( std::uint64_t j = i + 1; j < n; ++j )
      if ( overlap( s + i * D * 2, s + j * D * 2, D ) )
      {
        if ( static_cast< std::uint64_t >( cnt ) < cap )
        {
          out[2 * cnt] = static_cast< std::uint32_t >( i );
          out[2 * cnt + 1] = static_cast< std::uint32_t >( j );
        }
        ++cnt;
      }
  return cnt;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------------------
// Top-down tree (the reference's tree shape) and tree-vs-tree traversal with the intended pair orientation.
// ---------------------------------------------------------------------------------------------------------

namespace {

struct td_node
{
  std::vector< double > kd;     // D (min, max)
  std::int64_t child[2] = { -1, -1 };
  std::uint64_t begin = 0, end = 0;
};

struct td_tree
{
  int D = 0;
  std::vector< td_node > nodes;           // preorder, root at 0
  std::vector< std::uint32_t > leaf_elem; // element (local index) at each leaf position
};

// Union k-DOP over a range of elements (kdop.hpp:174-200 with m::min/m::max).
void union_range(const double *slabs, int D, const std::uint32_t *el, std::uint64_t b, std::uint64_t e,
                 std::vector< double > &out)
{
  out.assign( 2 * D, 0.0 );
  const double *f = slabs + static_cast< std::uint64_t >( el[b] ) * D * 2;
  for ( int a = 0; a < D; ++a )
  {
    double mn = f[2 * a], mx = f[2 * a + 1];
    for ( std::uint64_t i = b + 1; i < e; ++i )
    {
      const double *s = slabs + static_cast< std::uint64_t >( el[i] ) * D * 2;
      mn = ( s[2 * a] < mn ) ? s[2 * a] : mn;
      mx = ( s[2 * a + 1] > mx ) ? s[2 * a + 1] : mx;
    }
    out[2 * a] = mn;
    out[2 * a + 1] = mx;
  }
}

// longest_axis, kdop.hpp:354-362: the first axis of largest (max - min).
int longest_axis(const std::vector< double > &kd, int D)
{
  int best = 0;
  for ( int a = 1; a < D; ++a )
    if ( ( kd[2 * best + 1] - kd[2 * best] ) < ( kd[2 * a + 1] - kd[2 * a] ) )
      best = a;
  return best;
}

// top_down_builder::build, bvh_build.hpp:80-133, with split::mean (split/mean.hpp:47-65) and
// split_in_place (split/split.hpp:54-75): mean projected centroid, std::partition, middle fallback.
void td_build(td_tree &t, const double *slabs, const double *cent, const vec3 *nt, std::uint64_t node,
              std::uint64_t b, std::uint64_t e)
{
  const int D = t.D;
  t.nodes[node].begin = b;
  t.nodes[node].end = e;
  if ( e - b <= 1 ) return;
  const int axis = longest_axis( t.nodes[node].kd, D );
  std::uint32_t *first = t.leaf_elem.data() + b;
  std::uint32_t *last = t.leaf_elem.data() + e;
  double sum = 0.0;
  for ( auto *p = first; p != last; ++p ) sum = sum + project( cent + 3 * static_cast< std::uint64_t >( *p ), nt[axis] );
  const double split_pt = sum / static_cast< double >( e - b );
  std::uint32_t *mid = std::partition( first, last, [&](std::uint32_t el) {
    return project( cent + 3 * static_cast< std::uint64_t >( el ), nt[axis] ) < split_pt;
  } );
  if ( mid == first || mid == last ) mid = first + ( e - b ) / 2;
  const std::uint64_t m = b + static_cast< std::uint64_t >( mid - first );
  // left child
  {
    td_node ln;
    union_range( slabs, D, t.leaf_elem.data(), b, m, ln.kd );
    const std::uint64_t li = t.nodes.size();
    t.nodes.push_back( std::move( ln ) );
    t.nodes[node].child[0] = static_cast< std::int64_t >( li );
    td_build( t, slabs, cent, nt, li, b, m );
  }
  {
    td_node rn;
    union_range( slabs, D, t.leaf_elem.data(), m, e, rn.kd );
    const std::uint64_t ri = t.nodes.size();
    t.nodes.push_back( std::move( rn ) );
    t.nodes[node].child[1] = static_cast< std::int64_t >( ri );
    td_build( t, slabs, cent, nt, ri, m, e );
  }
}

void td_make(td_tree &t, const double *slabs, const double *cent, std::uint64_t n, int K)
{
  vec3 nt[13];
  t.D = normal_table( K, nt );
  t.nodes.clear();
  t.leaf_elem.resize( n );
  std::iota( t.leaf_elem.begin(), t.leaf_elem.end(), 0u );
  if ( n == 0 ) return;
  t.nodes.reserve( 2 * n );
  td_node root;
  union_range( slabs, t.D, t.leaf_elem.data(), 0, n, root.kd );
  t.nodes.push_back( std::move( root ) );
  td_build( t, slabs, cent, nt, 0, 0, n );
}

struct pair_sink
{
  std::uint32_t *out;
  std::uint64_t cap;
  std::int64_t cnt = 0;
  void emit(std::uint32_t a, std::uint32_t b)
  {
    if ( static_cast< std::uint64_t >( cnt ) < cap )
    {
      out[2 * cnt] = a;
      out[2 * cnt + 1] = b;
    }
    ++cnt;
  }
};

bool is_leaf(const td_node &n) { return n.child[0] < 0 && n.child[1] < 0; }

// get_overlapping_indices, collision_query.hpp:293-329, emitting (left element, right element): the
// reference's leaf loop indexes _right_leafs with the left range and vice versa (collision_query.hpp:310-312);
// its pair count is right, its ids are not, so the intended orientation is restated here.
void td_overlap(const td_tree &L, const td_tree &R, std::int64_t li, std::int64_t ri, pair_sink &sink)
{
  if ( li < 0 || ri < 0 ) return;
  const td_node &l = L.nodes[li];
  const td_node &r = R.nodes[ri];
  if ( !overlap( l.kd.data(), r.kd.data(), L.D ) ) return;
  if ( is_leaf( l ) )
  {
    if ( is_leaf( r ) )
    {
      for ( std::uint64_t i = l.begin; i < l.end; ++i )
        for ( std::uint64_t j = r.begin; j < r.end; ++j )
          sink.emit( L.leaf_elem[i], R.leaf_elem[j] );
    } else {
      td_overlap( L, R, li, r.child[0], sink );
      td_overlap( L, R, li, r.child[1], sink );
    }
  } else if ( is_leaf( r ) ) {
    td_overlap( L, R, l.child[0], ri, sink );
    td_overlap( L, R, l.child[1], ri, sink );
  } else {
    td_overlap( L, R, l.child[0], r.child[0], sink );
    td_overlap( L, R, l.child[0], r.child[1], sink );
    td_overlap( L, R, l.child[1], r.child[0], sink );
    td_overlap( L, R, l.child[1], r.child[1], sink );
  }
}

// get_self_colliding_indices, collision_query.hpp:331-368 (one element per leaf, so the leaf loop emits none).
void td_self(const td_tree &T, std::int64_t ni, pair_sink &sink)
{
  if ( ni < 0 ) return;
  const td_node &n = T.nodes[ni];
  if ( is_leaf( n ) ) return;
  td_self( T, n.child[0], sink );
  td_self( T, n.child[1], sink );
  if ( n.child[0] >= 0 && n.child[1] >= 0 ) td_overlap( T, T, n.child[0], n.child[1], sink );
}

}  // namespace

extern "C" {

// potential_collision_set over two top-down trees built from the given per-element slabs and centroids.
// Pairs are (local index into A, local index into B). Returns |S|.
std::int64_t orc_pairs_tree(const double *sa, const double *ca, std::uint64_t na,
                            const double *sb, const double *cb, std::uint64_t nb, int K,
                            std::uint32_t *out, std::uint64_t cap)
{
  td_tree A, B;
  td_make( A, sa, ca, na, K );
  td_make( B, sb, cb, nb, K );
  pair_sink sink{ out, cap };
  if ( na && nb ) td_overlap( A, B, 0, 0, sink );
  return sink.cnt;
}

// self_collision_set over one top-down tree. Pairs are normalised to (min index, max index).
std::int64_t orc_self_pairs_tree(const double *s, const double *c, std::uint64_t n, int K,
                                 std::uint32_t *out, std::uint64_t cap)
{
  td_tree T;
  td_make( T, s, c, n, K );
  pair_sink sink{ out, cap };
  if ( n ) td_self( T, 0, sink );
  const std::uint64_t m = std::min< std::uint64_t >( static_cast< std::uint64_t >( sink.cnt ), cap );
  for ( std::uint64_t p = 0; p < m; ++p )
    if ( out[2 * p] > out[2 * p + 1] ) std::swap( out[2 * p], out[2 * p + 1] );
  return sink.cnt;
}

// max_variant_axis (src/bvh/narrowphase/kokkos.hpp:125-160): the cardinal axis of largest variance of the
// centroids of A and B together, var = sum(c^2) - sum(c)^2 / N, sums in element order (A then B); ties keep the
// lower axis (0, then 1 only when strictly larger, then 2 only when strictly larger than the kept one).
int orc_max_variant_axis(const double *ca, std::uint64_t na, const double *cb, std::uint64_t nb)
{
  double s[3] = { 0, 0, 0 }, s2[3] = { 0, 0, 0 };
  for ( std::uint64_t i = 0; i < na + nb; ++i )
  {
    const double *c = i < na ? ca + 3 * i : cb + 3 * ( i - na );
    for ( int k = 0; k < 3; ++k )
    {
      s[k] += c[k];
      s2[k] += c[k] * c[k];
    }
  }
  double var[3];
  for ( int k = 0; k < 3; ++k ) var[k] = s2[k] - s[k] * s[k] / static_cast< double >( na + nb );
  int axis = 0;
  if ( var[1] > var[0] ) axis = 1;
  if ( var[2] > var[axis] ) axis = 2;
  return axis;
}

// sort_and_sweep_local (src/bvh/narrowphase/kokkos.hpp:164-248) with A and B as the two patches:
// - the global range on the axis is the union of both sets' slab extents there (the patches' k-DOPs);
// - B's slab minima become u32 keys, (min - global_min) * (UINT32_MAX / (global_max - global_min)), converted as
//   x86-64 gcc converts a double to u32 (truncation of the signed 64-bit value, NaN -> 0);
// - a stable sort of (key, index) (the reference's radix_sorter);
// - for every element of A, B in key order: skip while the scaled B maximum is below A's minimum key, stop at the
//   first B key above A's maximum key, emit the pairs that overlap strictly on every slab.
// Pairs are (index into A, index into B). Returns the pair count.
namespace {
inline std::uint32_t to_u32(double x)
{
  if ( std::isnan( x ) || !( x < 9223372036854775808.0 ) || x < -9223372036854775808.0 ) return 0u;
  return static_cast< std::uint32_t >( static_cast< std::uint64_t >( static_cast< std::int64_t >( x ) ) );
}
}  // namespace

std::int64_t orc_sort_and_sweep(const double *sa, std::uint64_t na, const double *sb, std::uint64_t nb, int K,
                                int axis, std::uint32_t *out, std::uint64_t cap)
{
  const int D = K / 2;
  if ( na == 0 || nb == 0 ) return 0;
  double gmin = std::numeric_limits< double >::infinity(), gmax = -gmin;
  for ( std::uint64_t i = 0; i < na; ++i )
  {
    gmin = std::min( gmin, sa[i * 2 * D + 2 * axis] );
    gmax = std::max( gmax, sa[i * 2 * D + 2 * axis + 1] );
  }
  for ( std::uint64_t j = 0; j < nb; ++j )
  {
    gmin = std::min( gmin, sb[j * 2 * D + 2 * axis] );
    gmax = std::max( gmax, sb[j * 2 * D + 2 * axis + 1] );
  }
  const double fac = static_cast< double >( std::numeric_limits< std::uint32_t >::max() ) / ( gmax - gmin );
  std::vector< std::uint32_t > key( nb );
  std::vector< std::uint32_t > idx( nb );
  for ( std::uint64_t j = 0; j < nb; ++j )
  {
    key[j] = to_u32( ( sb[j * 2 * D + 2 * axis] - gmin ) * fac );
    idx[j] = static_cast< std::uint32_t >( j );
  }
  std::stable_sort( idx.begin(), idx.end(), [&](std::uint32_t x, std::uint32_t y) { return key[x] < key[y]; } );
  std::int64_t cnt = 0;
  for ( std::uint64_t i = 0; i < na; ++i )
  {
    const double *ak = sa + i * 2 * D;
    const std::uint32_t amin = to_u32( ( ak[2 * axis] - gmin ) * fac );
    const std::uint32_t amax = to_u32( ( ak[2 * axis + 1] - gmin ) * fac );
    for ( std::uint64_t r = 0; r < nb; ++r )
    {
      const std::uint32_t j = idx[r];
      const double *bk = sb + static_cast< std::uint64_t >( j ) * 2 * D;
      const std::uint32_t bmin = key[j];
      const double bmax = ( bk[2 * axis + 1] - gmin ) * fac;
      if ( bmax < amin ) continue;
      if ( bmin > amax ) break;
      if ( overlap( ak, bk, D ) )
      {
        if ( static_cast< std::uint64_t >( cnt ) < cap )
        {
          out[2 * cnt] = static_cast< std::uint32_t >( i );
          out[2 * cnt + 1] = j;
        }
        ++cnt;
      }
    }
  }
  return cnt;
}

// Node count of the top-down tree (TreeTest.cpp:49-90 checks 2n - 1 for one element per leaf).
std::int64_t orc_tree_node_count(const double *s, const double *c, std::uint64_t n, int K)
{
  td_tree T;
  td_make( T, s, c, n, K );
  return static_cast< std::int64_t >( T.nodes.size() );
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------------------
// Whole-path CPU baseline (OpenMP): the reference's algorithms for each stage, on all host threads.
//   kdop_base::from_vertices per element (kdop.hpp:238-264), centroid, compute_bounds (contact_entity.hpp:136-148),
//   morton keys (contact_entity.hpp:104-118), radix_sorter one bit per pass with a parallel map, an exclusive
//   scan (prefix_sum.hpp:41-54) and a split scatter (util/sort.hpp:117-136), top_down_builder
//   (bvh_build.hpp:80-133, serial as in the reference) and query_tree (collision_query.hpp:166-213) for every
//   element of A against B's tree, in parallel over A's elements.
// ---------------------------------------------------------------------------------------------------------
#include <chrono>
#include <omp.h>

namespace {

template< typename Key >
void radix_sort_1bit_omp(std::vector< Key > &keys, std::vector< std::uint64_t > &idx, unsigned passes)
{
  const std::int64_t n = static_cast< std::int64_t >( keys.size() );
  if ( n == 0 ) return;
  std::vector< Key > ks( n ), bits( n ), scan( n );
  std::vector< std::uint64_t > is( n );
  const int T = omp_get_max_threads();
  std::vector< Key > part( T + 1 );
  for ( unsigned p = 0; p < passes; ++p )
  {
#pragma omp parallel
    {
      const int t = omp_get_thread_num();
      const std::int64_t b = n * t / T, e = n * ( t + 1 ) / T;
      Key acc = 0;
      for ( std::int64_t i = b; i < e; ++i )
      {
        bits[i] = ~( keys[i] >> p ) & 0x1;
        acc += bits[i];
      }
      part[t + 1] = acc;
#pragma omp barrier
#pragma omp single
      {
        part[0] = 0;
        for ( int k = 1; k <= T; ++k ) part[k] += part[k - 1];
      }
      Key run = part[t];
      for ( std::int64_t i = b; i < e; ++i )
      {
        scan[i] = run;
        run += bits[i];
      }
#pragma omp barrier
      const Key total = scan[n - 1] + bits[n - 1];
      for ( std::int64_t i = b; i < e; ++i )
      {
        const Key tt = static_cast< Key >( i ) - scan[i] + total;
        const Key ni = bits[i] ? scan[i] : tt;
        is[ni] = idx[i];
        ks[ni] = keys[i];
      }
    }
    keys.swap( ks );
    idx.swap( is );
  }
}

void query_node(const td_tree &T, std::int64_t ni, const double *q, int D, std::uint32_t qe,
                std::vector< std::uint32_t > &out)
{
  // query_node_impl: !node || !overlap -> return; leaf -> emit range; else left, right
  if ( ni < 0 ) return;
  const td_node &n = T.nodes[ni];
  if ( !overlap( q, n.kd.data(), D ) ) return;
  if ( is_leaf( n ) )
  {
    for ( std::uint64_t i = n.begin; i < n.end; ++i )
    {
      out.push_back( qe );
      out.push_back( T.leaf_elem[i] );
    }
  } else {
    query_node( T, n.child[0], q, D, qe, out );
    query_node( T, n.child[1], q, D, qe, out );
  }
}

double now_s()
{
  return std::chrono::duration< double >( std::chrono::steady_clock::now().time_since_epoch() ).count();
}

}  // namespace

extern "C" {

// Runs the whole path for objects A and B with `threads` OpenMP threads (0 = all). stage_s[7] receives the
// seconds of: slabs+centroids, bounds, keys, sort, tree build, traversal (pair list included), total. The pair
// list (index in A, index in B), in no particular order, goes to pairs[2p], pairs[2p + 1] for p < cap when pairs
// is given. Returns |S(A, B)|.
std::int64_t orc_pipeline(const double *xa, std::uint64_t na, const double *xb, std::uint64_t nb, std::uint32_t V,
                          int K, double eps, int threads, double *stage_s, std::uint32_t *pairs, std::uint64_t cap)
{
  if ( threads > 0 ) omp_set_num_threads( threads );
  const int D = K / 2;
  const double t0 = now_s();
  std::vector< double > sa( na * D * 2 ), sb( nb * D * 2 ), ca( na * 3 ), cb( nb * 3 );
#pragma omp parallel for schedule(static)
  for ( std::int64_t i = 0; i < static_cast< std::int64_t >( na ); ++i )
  {
    orc_kdops( xa + i * V * 3, V, 1, K, eps, sa.data() + i * D * 2 );
    orc_centroids( xa + i * V * 3, V, 1, ca.data() + i * 3 );
  }
#pragma omp parallel for schedule(static)
  for ( std::int64_t i = 0; i < static_cast< std::int64_t >( nb ); ++i )
  {
    orc_kdops( xb + i * V * 3, V, 1, K, eps, sb.data() + i * D * 2 );
    orc_centroids( xb + i * V * 3, V, 1, cb.data() + i * 3 );
  }
  const double t1 = now_s();
  double mna[3], inva[3], mnb[3], invb[3];
  orc_morton_bounds( sa.data(), na, K, mna, inva );
  orc_morton_bounds( sb.data(), nb, K, mnb, invb );
  const double t2 = now_s();
  std::vector< std::uint64_t > ka( na ), kb( nb );
#pragma omp parallel for schedule(static)
  for ( std::int64_t i = 0; i < static_cast< std::int64_t >( na ); ++i ) orc_morton_keys( ca.data() + 3 * i, 1, mna, inva, &ka[i] );
#pragma omp parallel for schedule(static)
  for ( std::int64_t i = 0; i < static_cast< std::int64_t >( nb ); ++i ) orc_morton_keys( cb.data() + 3 * i, 1, mnb, invb, &kb[i] );
  const double t3 = now_s();
  std::vector< std::uint64_t > ia( na ), ib( nb );
  std::iota( ia.begin(), ia.end(), 0ull );
  std::iota( ib.begin(), ib.end(), 0ull );
  radix_sort_1bit_omp( ka, ia, 64 );
  radix_sort_1bit_omp( kb, ib, 64 );
  const double t4 = now_s();
  td_tree TB;
  td_make( TB, sb.data(), cb.data(), nb, K );
  const double t5 = now_s();
  // every thread keeps the pairs it finds (the path's output is the pair list, not only its size)
  std::vector< std::vector< std::uint32_t > > found( omp_get_max_threads() );
  if ( na && nb )
  {
#pragma omp parallel
    {
      std::vector< std::uint32_t > &mine = found[omp_get_thread_num()];
      std::vector< std::uint32_t > out;
#pragma omp for schedule(dynamic, 1024)
      for ( std::int64_t r = 0; r < static_cast< std::int64_t >( na ); ++r )
      {
        // queries in the sorted (Morton) order of A, as the clustered element order of the reference
        const std::uint32_t e = static_cast< std::uint32_t >( ia[r] );
        out.clear();
        query_node( TB, 0, sa.data() + static_cast< std::uint64_t >( e ) * D * 2, D, e, out );
        mine.insert( mine.end(), out.begin(), out.end() );
      }
    }
  }
  const double t6 = now_s();
  std::int64_t total = 0;
  for ( const auto &f : found )
  {
    if ( pairs )
      for ( std::size_t j = 0; j + 1 < f.size(); j += 2 )
      {
        const std::uint64_t p = static_cast< std::uint64_t >( total ) + j / 2;
        if ( p < cap )
        {
          pairs[2 * p] = f[j];
          pairs[2 * p + 1] = f[j + 1];
        }
      }
    total += static_cast< std::int64_t >( f.size() / 2 );
  }
  if ( stage_s )
  {
    stage_s[0] = t1 - t0;
    stage_s[1] = t2 - t1;
    stage_s[2] = t3 - t2;
    stage_s[3] = t4 - t3;
    stage_s[4] = t5 - t4;
    stage_s[5] = t6 - t5;
    stage_s[6] = t6 - t0;
  }
  return total;
}

// morton_cluster (src/bvh/split/cluster.hpp:89-179) with its hashes from morton_impl over the 32-bit type
// (src/bvh/contact_entity.hpp:104-118: morton32(quantize32(centroid, min, inv_diag)), hash.hpp:106-110, 148-166):
// the element indices stably sorted by hash; the depth of every neighbouring pair, 31 - floor(log2(h_i ^ h_{i+1}))
// or all ones for equal hashes (cluster.hpp:143-151); the positions stably sorted by depth; the first `patches` - 1
// of them, in position order, are the splits, and positions that cannot be chosen hold n - 1 (cluster.hpp:109-116,
// 156-169). order_out receives the n element indices in hash order, bounds_out the patches + 1 patch boundaries
// [0, splits..., n] (set_entity_data_impl, src/bvh/collision_object.cpp:134-141).
void orc_morton_cluster(const double *centroids, std::uint64_t n, const double *min3, const double *inv3,
                        std::uint32_t patches, std::uint32_t *order_out, std::uint64_t *bounds_out)
{
  const std::uint64_t nsplit = patches > 0 ? patches - 1 : 0;
  std::vector< std::uint64_t > splits( nsplit, 0 );
  std::vector< std::uint32_t > hash( n ), idx( n );
  for ( std::uint64_t i = 0; i < n; ++i )
  {
    std::uint32_t q[3];
    orc_quantize32( centroids + 3 * i, min3, inv3, q );
    hash[i] = orc_morton32( q[0], q[1], q[2] );
  }
  std::iota( idx.begin(), idx.end(), 0u );
  std::stable_sort( idx.begin(), idx.end(), [&hash](std::uint32_t a, std::uint32_t b) { return hash[a] < hash[b]; } );
  if ( n > 0 )
  {
    const std::uint64_t max_idx = n - 1;
    if ( nsplit > max_idx ) std::fill( splits.begin(), splits.end(), max_idx );
    std::vector< std::uint32_t > depth( n - 1 ), pos( n - 1 );
    for ( std::uint64_t i = 0; i + 1 < n; ++i )
    {
      const std::uint32_t mask = hash[idx[i]] ^ hash[idx[i + 1]];
      depth[i] = mask ? 31u - static_cast< std::uint32_t >( 31 - __builtin_clz( mask ) ) : 0xffffffffu;
      pos[i] = static_cast< std::uint32_t >( i );
    }
    std::stable_sort( pos.begin(), pos.end(), [&depth](std::uint32_t a, std::uint32_t b) { return depth[a] < depth[b]; } );
    const std::uint64_t take = std::min< std::uint64_t >( nsplit, n - 1 );
    std::vector< std::uint32_t > chosen( pos.begin(), pos.begin() + take );
    std::sort( chosen.begin(), chosen.end() );
    for ( std::uint64_t k = 0; k < take; ++k ) splits[k] = chosen[k];
  }
  if ( order_out ) std::memcpy( order_out, idx.data(), n * sizeof( std::uint32_t ) );
  if ( bounds_out && patches > 0 )
  {
    bounds_out[0] = 0;
    for ( std::uint64_t k = 1; k < patches; ++k ) bounds_out[k] = splits[k - 1];
    bounds_out[patches] = n;
  }
}

int orc_max_threads() { return omp_get_max_threads(); }

}  // extern "C"
