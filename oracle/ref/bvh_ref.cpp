// Cross-check driver for the oracle: the reference's own element-broadphase code behind a C ABI. Its headers are
// included read-only from the reference's source tree (src/bvh/...), built by oracle/ref_build.sh with the serial
// Kokkos stand-in of oracle/ref/shim into oracle/_ref/. Test scaffolding only: the tests compare the oracle's
// restatement with these functions; nothing of the product links them.
//
// The reference's element trees hold bphase_kdop snapshots (src/bvh/types.hpp:46-50): a 26-DOP by default, a
// 6-DOP when built with BVH_BROADPHASE_6_DOP (the second build of this file). 18-DOP slabs come from the
// reference's projection with dop_18's normal table (its from_vertices cannot compile for dop_18, whose normals
// are a data member, src/bvh/kdop.hpp:610), and 18-DOP pairs from its strict overlap test by brute force.
#include <bvh/collision_query.hpp>
#include <bvh/contact_entity.hpp>
#include <bvh/hash.hpp>
#include <bvh/kdop.hpp>
#include <bvh/narrowphase/kokkos.hpp>
#include <bvh/snapshot.hpp>
#include <bvh/split/cluster.hpp>
#include <bvh/tree_build.hpp>
#include <bvh/util/sort.hpp>

#include <cstdint>
#include <vector>

namespace
{
using vec3 = bvh::m::vec3d;

// An element as the reference's tests build one (tests/TestCommon.hpp:60-75): vertices, the k-DOP from
// kdop_base::from_vertices, centroid = accumulate from zero / count, its index as global id.
struct ref_element
{
  std::vector< vec3 > verts;
  bvh::bphase_kdop bounds;
  std::size_t gid = 0;

  const bvh::bphase_kdop &kdop() const { return bounds; }
  vec3 centroid() const
  {
    return std::accumulate( verts.begin(), verts.end(), vec3::zeros() ) / static_cast< double >( verts.size() );
  }
  std::size_t global_id() const { return gid; }
};

std::vector< ref_element > make_elements(const double *xyz, uint64_t n, int V, double eps)
{
  std::vector< ref_element > el( n );
  for ( uint64_t e = 0; e < n; ++e )
  {
    el[e].verts.resize( V );
    for ( int v = 0; v < V; ++v )
      el[e].verts[v] = vec3( xyz[( e * V + v ) * 3], xyz[( e * V + v ) * 3 + 1], xyz[( e * V + v ) * 3 + 2] );
    el[e].bounds = bvh::bphase_kdop::from_vertices( el[e].verts.begin(), el[e].verts.end(), eps );
    el[e].gid = e;
  }
  return el;
}

template< typename Kdop >
void store(const Kdop &k, double *out)
{
  for ( int a = 0; a < Kdop::num_axis; ++a )
  {
    out[2 * a] = k.extents[a].min;
    out[2 * a + 1] = k.extents[a].max;
  }
}

// 18-DOP of one element: the loop of kdop_base::from_vertices (src/bvh/kdop.hpp:238-264) over dop_18's table.
bvh::dop_18d dop18_of(const vec3 *v, int V, double eps)
{
  bvh::dop_18d ret;
  for ( int i = 0; i < bvh::dop_18d::num_axis; ++i )
  {
    double proj = bvh::dop_18d::project( v[0], bvh::dop_18d::normals[i] );
    ret.extents[i].min = proj - eps;
    ret.extents[i].max = proj + eps;
    for ( int k = 1; k < V; ++k )
    {
      proj = bvh::dop_18d::project( v[k], bvh::dop_18d::normals[i] );
      ret.extents[i].min = std::min( ret.extents[i].min, proj - eps );
      ret.extents[i].max = std::max( ret.extents[i].max, proj + eps );
    }
  }
  return ret;
}

std::vector< bvh::dop_18d > dops18(const double *xyz, uint64_t n, int V, double eps)
{
  std::vector< bvh::dop_18d > d( n );
  std::vector< vec3 > v( V );
  for ( uint64_t e = 0; e < n; ++e )
  {
    for ( int k = 0; k < V; ++k ) v[k] = vec3( xyz[( e * V + k ) * 3], xyz[( e * V + k ) * 3 + 1], xyz[( e * V + k ) * 3 + 2] );
    d[e] = dop18_of( v.data(), V, eps );
  }
  return d;
}

uint64_t emit(const std::vector< std::pair< std::size_t, std::size_t > > &p, uint64_t *out, uint64_t cap)
{
  for ( uint64_t i = 0; i < p.size() && i < cap; ++i )
  {
    out[2 * i] = p[i].first;
    out[2 * i + 1] = p[i].second;
  }
  return p.size();
}
}  // namespace

extern "C" {

// K of the k-DOP in this build's element trees (26, or 6 with BVH_BROADPHASE_6_DOP).
int ref_tree_k() { return bvh::bphase_kdop::num_axis * 2; }

// Element slabs [n][K/2][min, max] for K = 6, 18 or 26.
int ref_kdops(const double *xyz, uint64_t n, int V, int K, double eps, double *out)
{
  std::vector< vec3 > v( V );
  for ( uint64_t e = 0; e < n; ++e )
  {
    for ( int k = 0; k < V; ++k ) v[k] = vec3( xyz[( e * V + k ) * 3], xyz[( e * V + k ) * 3 + 1], xyz[( e * V + k ) * 3 + 2] );
    if ( K == 6 ) store( bvh::dop_6d::from_vertices( v.begin(), v.end(), eps ), out + e * 6 );
    else if ( K == 26 ) store( bvh::dop_26d::from_vertices( v.begin(), v.end(), eps ), out + e * 26 );
    else if ( K == 18 ) store( dop18_of( v.data(), V, eps ), out + e * 18 );
    else return 1;
  }
  return 0;
}

// Centroids as TestCommon.hpp's Element computes them.
void ref_centroids(const double *xyz, uint64_t n, int V, double *out)
{
  auto el = make_elements( xyz, n, V, 0.0 );
  for ( uint64_t e = 0; e < n; ++e )
  {
    const vec3 c = el[e].centroid();
    out[3 * e] = c[0];
    out[3 * e + 1] = c[1];
    out[3 * e + 2] = c[2];
  }
}

// Morton bounds (compute_bounds over the elements' tree k-DOPs, src/bvh/contact_entity.hpp:136-148) and the
// 64-bit Morton code of each centroid (morton_impl, :104-118: quantize64 then morton).
void ref_morton(const double *xyz, uint64_t n, int V, double eps, double *min3, double *inv3, uint64_t *keys)
{
  auto el = make_elements( xyz, n, V, eps );
  bvh::view< const ref_element * > ev( el.data(), n );
  bvh::single_view< bvh::min_inv_diag_bounds > b( "bounds" );
  bvh::compute_bounds( ev, b );
  for ( int i = 0; i < 3; ++i )
  {
    min3[i] = b().min[i];
    inv3[i] = b().inv_diag[i];
  }
  bvh::view< bvh::morton64_t * > codes( "codes", n );
  bvh::morton( ev, b, codes );
  for ( uint64_t e = 0; e < n; ++e ) keys[e] = codes( e );
}

uint64_t ref_morton64(uint64_t x, uint64_t y, uint64_t z) { return bvh::morton( x, y, z ); }

// Element trees (build_snapshot_tree_top_down, src/bvh/tree_build.hpp:176-185) and potential_collision_set
// (src/bvh/collision_query.hpp:370-379): returns the pair count; the first cap pairs as the reference emits them.
uint64_t ref_tree_pairs(const double *xa, uint64_t na, const double *xb, uint64_t nb, int V, double eps,
                        uint64_t *out, uint64_t cap)
{
  auto a = make_elements( xa, na, V, eps );
  auto b = make_elements( xb, nb, V, eps );
  auto ta = bvh::build_snapshot_tree_top_down( a );
  auto tb = bvh::build_snapshot_tree_top_down( b );
  return emit( bvh::potential_collision_set( ta, tb ).pairs, out, cap );
}

// self_collision_set (src/bvh/collision_query.hpp:355-363) over one element tree.
uint64_t ref_self_pairs(const double *x, uint64_t n, int V, double eps, uint64_t *out, uint64_t cap)
{
  auto a = make_elements( x, n, V, eps );
  auto t = bvh::build_snapshot_tree_top_down( a );
  return emit( bvh::self_collision_set( t ).pairs, out, cap );
}

// 18-DOP pairs (i, j) by brute force with the reference's strict overlap (src/bvh/kdop.hpp:538-549).
uint64_t ref_brute_pairs18(const double *xa, uint64_t na, const double *xb, uint64_t nb, int V, double eps,
                           uint64_t *out, uint64_t cap)
{
  auto a = dops18( xa, na, V, eps );
  auto b = dops18( xb, nb, V, eps );
  uint64_t cnt = 0;
  for ( uint64_t i = 0; i < na; ++i )
    for ( uint64_t j = 0; j < nb; ++j )
      if ( bvh::overlap( a[i], b[j] ) )
      {
        if ( cnt < cap )
        {
          out[2 * cnt] = i;
          out[2 * cnt + 1] = j;
        }
        ++cnt;
      }
  return cnt;
}

// The reference's stable 1-bit radix sort (src/bvh/util/sort.hpp:75-144) of n 64-bit keys with their indices.
void ref_radix_sort_u64(const uint64_t *keys, uint64_t n, uint64_t *sorted, uint64_t *perm)
{
  bvh::radix_sorter< uint64_t, std::size_t > sorter( n );
  bvh::view< uint64_t * > h( "keys", n );
  bvh::view< std::size_t * > idx( "indices", n );
  for ( uint64_t i = 0; i < n; ++i )
  {
    h( i ) = keys[i];
    idx( i ) = i;
  }
  sorter( h, idx );
  for ( uint64_t i = 0; i < n; ++i )
  {
    sorted[i] = h( i );
    perm[i] = idx( i );
  }
}

// Morton clustering of the elements into `clusters` patches (morton_cluster, src/bvh/split/cluster.hpp:89-179, as
// set_entity_data_clustering uses it, src/bvh/collision_object.hpp:89-131): order[r] = element of rank r, splits
// (clusters - 1 values) = the patch boundaries in that order (patch k = ranks [splits[k-1], splits[k])).
void ref_cluster(const double *xyz, uint64_t n, int V, uint64_t clusters, uint64_t *order, uint64_t *splits)
{
  auto el = make_elements( xyz, n, V, 0.0 );
  bvh::morton_cluster mc( n );
  bvh::view< const ref_element * > ev( el.data(), n );
  bvh::view< std::size_t * > idx( "indices", n );
  for ( uint64_t i = 0; i < n; ++i ) idx( i ) = i;
  bvh::view< std::size_t * > sp( "splits", clusters > 0 ? clusters - 1 : 0 );
  mc( ev, idx, sp );
  for ( uint64_t i = 0; i < n; ++i ) order[i] = idx( i );
  for ( uint64_t k = 0; k + 1 < clusters; ++k ) splits[k] = sp( k );
}

// sort_and_sweep_local (src/bvh/narrowphase/kokkos.hpp:164-248) with each element set as one patch (the patch's
// k-DOP is the union of its elements', patch.hpp), axis = max_variant_axis (kokkos.hpp:125-160) when axis < 0.
// Returns the pair count; the first cap pairs (index in A, index in B) in the order the functor sees them.
uint64_t ref_sort_and_sweep(const double *xa, uint64_t na, const double *xb, uint64_t nb, int V, double eps,
                            int axis, int *axis_used, uint64_t *out, uint64_t cap)
{
  auto a = make_elements( xa, na, V, eps );
  auto b = make_elements( xb, nb, V, eps );
  using elem_view = Kokkos::View< ref_element *, Kokkos::HostSpace, Kokkos::MemoryTraits< Kokkos::Unmanaged > >;
  elem_view va( a.data(), a.size() ), vb( b.data(), b.size() );
  bvh::patch<> pa( 0, bvh::span< const ref_element >( a.data(), a.size() ) );
  bvh::patch<> pb( 1, bvh::span< const ref_element >( b.data(), b.size() ) );
  const int ax = axis >= 0 ? axis : bvh::max_variant_axis( va, vb );
  if ( axis_used ) *axis_used = ax;
  uint64_t cnt = 0;
  bvh::sort_and_sweep_local( pa, va, pb, vb, ax, [&]( const ref_element &e, const ref_element &f ) {
    if ( cnt < cap )
    {
      out[2 * cnt] = e.gid;
      out[2 * cnt + 1] = f.gid;
    }
    ++cnt;
  } );
  return cnt;
}
}
