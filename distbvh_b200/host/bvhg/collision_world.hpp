// collision_world.hpp — vt-free, single-rank host mirror of distBVH's collision_world / collision_object API over
// the C ABI of libbvhg.so (include/bvhg.h). Header-only C++17; link with -lbvhg.
//
// It keeps the reference's L5 signatures (src/bvh/collision_world.hpp:54-114, src/bvh/collision_object.hpp:55-283):
//
//   bvhg::collision_world world( od_factor );
//   auto &a = world.create_collision_object();
//   a.set_entity_data( elements, bvhg::split_algorithm::clustering );  // span / vector of the caller's element type
//   a.init_broadphase();
//   world.set_narrowphase_functor< Element >( functor );                 // narrowphase_result_pair( bc_a, bc_b )
//   world.start_iteration(); a.broadphase( b ); world.finish_iteration();
//   a.for_each_result< R >( []( const R & ) { ... } );
//
// Differences, each forced by the single-rank, element-exact design:
//   - The element type supplies vertices instead of a k-DOP: `e.vertices()` (or a free get_entity_vertices(e))
//     returning a contiguous range of 3-vectors indexable as v[0..2], and `e.global_id()` (or
//     get_entity_global_id(e)). The library computes the k-DOP exactly as kdop_base::from_vertices
//     (src/bvh/kdop.hpp:238-264) with world_config::k (26 by default: the reference's bphase_kdop).
//   - Patches: an object's elements are split into od_factor patches exactly as the reference's Morton clustering
//     splits them (morton_cluster, src/bvh/split/cluster.hpp:89-179; every split algorithm uses it here), on the
//     device (bvhg_cluster). The functor is called once for every patch pair that holds at least one overlapping
//     element pair (the reference calls it for every pair of overlapping patch k-DOPs, a superset), with both
//     patches' elements as spans in the reference's order and, in addition, the exact element pairs of that patch
//     pair (broadphase_collision::candidates, indices into the two spans; grouped by patch pair on the device,
//     bvhg_patch_pairs; unordered within a patch pair). A functor that only reports overlapping elements gives
//     the same results.
//   - The element bytes handed to the functor are copies made at init_broadphase (the reference ships copies to
//     the narrowphase rank too); the caller's array is read only during set_entity_data.
//   - Errors throw bvhg::error (the reference asserts and terminates).
#ifndef BVHG_HOST_COLLISION_WORLD_HPP
#define BVHG_HOST_COLLISION_WORLD_HPP

#include "../../../include/bvhg.h"

#include <algorithm>
#include <array>
#include <cfloat>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

namespace bvhg
{
class error : public std::runtime_error
{
public:
  error(bvhg_status s, const std::string &what) : std::runtime_error( what ), status( s ) {}
  bvhg_status status;
};

// Same enumerators as src/bvh/types.hpp:52-57; all three order patches by Morton rank here.
enum class split_algorithm
{
  geom_axis,
  ml_geom_axis,
  clustering
};

struct world_config
{
  int k = 26;                                  // 6, 18 or 26
  bvhg_precision precision = BVHG_PLAIN_FP64;  // or BVHG_FILTER_FP32 (same pair set)
  double epsilon = 0.0;                        // slab inflation
  int device = 0;
  void *stream = nullptr;                      // cudaStream_t; NULL = one the library owns
};

template< typename T >
class span
{
public:
  span() = default;
  span(T *p, std::size_t n) : m_p( p ), m_n( n ) {}
  template< typename C >
  span(C &c) : m_p( c.data() ), m_n( c.size() )
  {}
  T *data() const { return m_p; }
  std::size_t size() const { return m_n; }
  T &operator[](std::size_t i) const { return m_p[i]; }
  T *begin() const { return m_p; }
  T *end() const { return m_p + m_n; }

private:
  T *m_p = nullptr;
  std::size_t m_n = 0;
};

class collision_object;

// A patch of an object (src/bvh/patch.hpp:55-123): its global id, element count, k-DOP (the union of its elements'
// slabs: kdop()[2 a] the minimum and kdop()[2 a + 1] the maximum of slab a) and centroid (the mean of its
// elements' centroids, summed in the patch's element order as std::accumulate does there). An empty patch has the
// default k-DOP of the reference (every slab [DBL_MAX, lowest]) and centroid (0, 0, 0).
class patch
{
public:
  patch() = default;
  patch(std::size_t id, std::size_t size, std::vector< double > kdop, std::array< double, 3 > centroid)
      : m_global_id( id ), m_size( size ), m_kdop( std::move( kdop ) ), m_centroid( centroid )
  {}
  std::size_t global_id() const noexcept { return m_global_id; }
  const std::vector< double > &kdop() const noexcept { return m_kdop; }
  const std::array< double, 3 > &centroid() const noexcept { return m_centroid; }
  bool empty() const noexcept { return m_size == 0; }
  std::size_t size() const noexcept { return m_size; }

private:
  std::size_t m_global_id = static_cast< std::size_t >( -1 );
  std::size_t m_size = 0;
  std::vector< double > m_kdop;
  std::array< double, 3 > m_centroid{};
};

// The tree over an object's non-empty patches that for_each_tree hands out (the snapshot_tree of
// src/bvh/collision_object.hpp:59, built top-down as src/bvh/bvh_build.hpp:55-139 builds it: split at the mean
// centroid along the longest cardinal axis of the node's k-DOP, halves when one side would be empty). nodes()[0] is
// the root; a leaf holds one patch (index into patches()); count() is the number of leaves.
class snapshot_tree
{
public:
  struct node
  {
    std::vector< double > kdop;  // union of the patches below, as patch::kdop()
    int child[2] = { -1, -1 };   // node indices, -1 at a leaf
    std::size_t patch = 0;       // a leaf's index into patches()
    bool leaf() const noexcept { return child[0] < 0; }
  };
  std::size_t count() const noexcept { return m_patches.size(); }
  bool empty() const noexcept { return m_nodes.empty(); }
  const node *root() const noexcept { return m_nodes.empty() ? nullptr : &m_nodes[0]; }
  const std::vector< node > &nodes() const noexcept { return m_nodes; }
  const std::vector< patch > &patches() const noexcept { return m_patches; }

  explicit snapshot_tree(std::vector< patch > non_empty, int k) : m_patches( std::move( non_empty ) )
  {
    if ( m_patches.empty() ) return;
    std::vector< std::size_t > idx( m_patches.size() );
    for ( std::size_t i = 0; i < idx.size(); ++i ) idx[i] = i;
    m_nodes.reserve( 2 * idx.size() );
    build( idx, 0, idx.size(), k );
  }

private:
  // node over idx[lo, hi); returns its index
  int build(std::vector< std::size_t > &idx, std::size_t lo, std::size_t hi, int k)
  {
    const int me = static_cast< int >( m_nodes.size() );
    m_nodes.emplace_back();
    std::vector< double > box( m_patches[idx[lo]].kdop() );
    for ( std::size_t i = lo + 1; i < hi; ++i )
      for ( int a = 0; a < k / 2; ++a )
      {
        box[2 * a] = std::min( box[2 * a], m_patches[idx[i]].kdop()[2 * a] );
        box[2 * a + 1] = std::max( box[2 * a + 1], m_patches[idx[i]].kdop()[2 * a + 1] );
      }
    m_nodes[me].kdop = box;
    if ( hi - lo == 1 )
    {
      m_nodes[me].patch = idx[lo];
      return me;
    }
    // the first three slabs are the cardinal axes in every k-DOP of the library
    int axis = 0;
    for ( int a = 1; a < 3; ++a )
      if ( box[2 * a + 1] - box[2 * a] > box[2 * axis + 1] - box[2 * axis] ) axis = a;
    double mean = 0.0;
    for ( std::size_t i = lo; i < hi; ++i ) mean += m_patches[idx[i]].centroid()[axis];
    mean /= static_cast< double >( hi - lo );
    auto mid = std::partition( idx.begin() + static_cast< std::ptrdiff_t >( lo ), idx.begin() + static_cast< std::ptrdiff_t >( hi ),
                               [&](std::size_t i) { return m_patches[i].centroid()[axis] < mean; } );
    std::size_t m = static_cast< std::size_t >( mid - idx.begin() );
    if ( m == lo || m == hi ) m = lo + ( hi - lo ) / 2;
    const int l = build( idx, lo, m, k );
    const int r = build( idx, m, hi, k );
    m_nodes[me].child[0] = l;
    m_nodes[me].child[1] = r;
    return me;
  }

  std::vector< patch > m_patches;
  std::vector< node > m_nodes;
};

// src/bvh/collision_query.hpp:50-64, plus the exact element pairs of the patch pair.
template< typename T >
struct broadphase_collision
{
  collision_object &object;
  const patch &meta;
  std::size_t patch_id;
  span< const T > elements;
  span< const std::pair< uint32_t, uint32_t > > candidates;  // (index in this span, index in the other span)
};

// src/bvh/collision_query.hpp:66-128: a byte buffer of fixed-stride records.
class narrowphase_result
{
public:
  narrowphase_result() = default;
  explicit narrowphase_result(std::size_t stride) : m_stride( stride ) {}
  void *allocate(std::size_t n)
  {
    m_n += n;
    const std::size_t at = m_data.size();
    m_data.resize( at + n * m_stride, 0 );
    return m_data.data() + at;
  }
  void append_data(const void *p, std::size_t n)
  {
    std::memcpy( allocate( n ), p, n * m_stride );
  }
  void *at(std::size_t i) { return m_data.data() + i * m_stride; }
  const void *at(std::size_t i) const { return m_data.data() + i * m_stride; }
  std::size_t stride() const noexcept { return m_stride; }
  std::size_t size() const noexcept { return m_n; }

private:
  std::vector< unsigned char > m_data;
  std::size_t m_stride = 0;
  std::size_t m_n = 0;
};

template< typename T >
class typed_narrowphase_result : public narrowphase_result
{
public:
  typed_narrowphase_result() : narrowphase_result( sizeof( T ) ) {}
  template< typename... Args >
  T &emplace_back(Args &&...args)
  {
    return *( new ( allocate( 1 ) ) T( std::forward< Args >( args )... ) );
  }
  T &operator[](std::size_t i) { return *static_cast< T * >( at( i ) ); }
};

struct narrowphase_result_pair
{
  narrowphase_result a;
  narrowphase_result b;
};

namespace detail
{
inline void check(bvhg_ctx *ctx, bvhg_status s, const char *what)
{
  if ( s != BVHG_OK )
    throw error( s, std::string( what ) + ": " + bvhg_status_string( s ) + ( ctx ? std::string( " (" ) + bvhg_last_error( ctx ) + ")" : "" ) );
}

template< typename E >
auto vertices_of(const E &e, int) -> decltype( get_entity_vertices( e ) )
{
  return get_entity_vertices( e );
}
template< typename E >
auto vertices_of(const E &e, long) -> decltype( e.vertices() )
{
  return e.vertices();
}
template< typename E >
auto global_id_of(const E &e, int) -> decltype( get_entity_global_id( e ) )
{
  return get_entity_global_id( e );
}
template< typename E >
auto global_id_of(const E &e, long) -> decltype( e.global_id() )
{
  return e.global_id();
}

// Type-erased element storage of one object (the functor's spans point into it).
struct element_store
{
  std::vector< unsigned char > bytes;  // elements in Morton rank order
  std::size_t size = 0;
  std::size_t elem_size = 0;
  const void *type = nullptr;  // identity of T
};

template< typename T >
const void *type_id()
{
  static const char id = 0;
  return &id;
}
}  // namespace detail

class collision_world;

class collision_object
{
public:
  collision_object(const collision_object &) = delete;
  collision_object &operator=(const collision_object &) = delete;

  // collision_object::set_entity_data (src/bvh/collision_object.hpp:69-84). Reads the elements now: vertices and
  // global ids go to the library, the element values are kept for the narrowphase functor.
  template< typename T >
  void set_entity_data(span< const T > data, split_algorithm = split_algorithm::clustering)
  {
    // element bytes are copied and handed to the functor as span<const T>, as the reference ships them
    static_assert( std::is_trivially_copyable< T >::value, "element types must be trivially copyable" );
    const std::size_t n = data.size();
    std::vector< double > xyz;
    std::vector< uint64_t > gid( n );
    uint32_t V = 0;
    for ( std::size_t i = 0; i < n; ++i )
    {
      const auto &verts = detail::vertices_of( data[i], 0 );
      const uint32_t vi = static_cast< uint32_t >( std::end( verts ) - std::begin( verts ) );
      if ( i == 0 )
      {
        V = vi;
        xyz.reserve( n * V * 3 );
      }
      if ( vi != V ) throw error( BVHG_ERR_ARG, "set_entity_data: every element needs the same vertex count" );
      for ( const auto &v : verts )
        for ( int c = 0; c < 3; ++c ) xyz.push_back( static_cast< double >( v[c] ) );
      gid[i] = static_cast< uint64_t >( detail::global_id_of( data[i], 0 ) );
    }
    m_gid = gid;
    m_n = n;
    detail::check( ctx(), bvhg_set_elements( ctx(), m_obj, n ? xyz.data() : nullptr, n ? V : 3, nullptr, n, BVHG_MEM_HOST ),
                   "set_entity_data" );
    m_elems.size = n;
    m_elems.elem_size = sizeof( T );
    m_elems.type = detail::type_id< T >();
    m_src = std::vector< unsigned char >( reinterpret_cast< const unsigned char * >( data.data() ),
                                          reinterpret_cast< const unsigned char * >( data.data() + n ) );
    m_built = false;
  }
  template< typename T >
  void set_entity_data(const std::vector< T > &data, split_algorithm alg = split_algorithm::clustering)
  {
    set_entity_data( span< const T >( data.data(), data.size() ), alg );
  }

  // collision_object::init_broadphase (src/bvh/collision_object.cpp:148): bounds, Morton keys, sort, tree.
  void init_broadphase();

  // collision_object::broadphase (src/bvh/collision_object.cpp:248-299): the exact element pairs with `other`,
  // then the narrowphase functor for every patch pair holding one; results go to both objects.
  void broadphase(collision_object &other);

  // collision_object::for_each_result (src/bvh/collision_object.hpp:178-187).
  template< typename R, typename F >
  void for_each_result(F &&f) const
  {
    for ( const auto &r : m_results )
      for ( std::size_t i = 0; i < r.size(); ++i ) f( *static_cast< const R * >( r.at( i ) ) );
  }

  // The exact element pairs (global ids) of the last broadphase with `other`.
  const std::vector< std::pair< uint64_t, uint64_t > > &last_pairs() const { return m_last_pairs; }

  // collision_object::local_patches (src/bvh/collision_object.hpp:189): this object's od_factor patches (after
  // init_broadphase), global ids id() * od_factor + p.
  const std::vector< patch > &local_patches() const noexcept { return m_patches; }

  // collision_object::for_each_tree (src/bvh/collision_object.hpp:164-168): f(const snapshot_tree &) with the tree
  // over this object's non-empty patches (one rank: the reference's tree spans every rank's patches).
  template< typename F >
  void for_each_tree(F &&f) const
  {
    std::vector< patch > non_empty;
    for ( const auto &p : m_patches )
      if ( !p.empty() ) non_empty.push_back( p );
    const snapshot_tree tree( std::move( non_empty ), world_k() );
    f( tree );
  }

  // Global ids of each patch's elements, in the patch order (after init_broadphase).
  std::vector< std::vector< uint64_t > > patch_global_ids() const
  {
    std::vector< std::vector< uint64_t > > out( num_patches() );
    for ( std::size_t p = 0; p < out.size(); ++p )
      for ( std::size_t r = m_pbeg[p]; r < m_pbeg[p + 1]; ++r ) out[p].push_back( m_gid[m_order[r]] );
    return out;
  }

  // collision_object::end_phase (src/bvh/collision_object.cpp:400-403) closes a vt phase of the object's task
  // chains; one rank with no chains has nothing to close. The results and patches stay as they are.
  void end_phase() noexcept {}

  std::size_t id() const noexcept { return m_id; }
  int overdecomposition_factor() const noexcept;
  std::size_t num_patches() const noexcept;

  ~collision_object()
  {
    if ( ctx() ) bvhg_object_destroy( ctx(), m_obj );
  }

private:
  friend class collision_world;
  collision_object(collision_world &w, std::size_t id);
  bvhg_ctx *ctx() const;

  // where patch p starts in the patch order (m_pbeg has od_factor + 1 entries)
  std::size_t patch_begin(std::size_t p) const { return m_pbeg[p]; }

  collision_world &m_world;
  std::size_t m_id;
  int32_t m_obj = -1;
  std::size_t m_n = 0;
  bool m_built = false;
  std::vector< uint64_t > m_gid;
  std::vector< unsigned char > m_src;  // the caller's elements, original order
  detail::element_store m_elems;       // patch order (after init_broadphase)
  std::vector< uint32_t > m_order;     // element index of every position of the patch order
  std::vector< std::size_t > m_pbeg;   // patch p = positions [m_pbeg[p], m_pbeg[p + 1])
  std::vector< narrowphase_result > m_results;
  std::vector< std::pair< uint64_t, uint64_t > > m_last_pairs;
  std::vector< patch > m_patches;      // local_patches()
  int world_k() const;
};

class collision_world
{
public:
  template< typename T >
  using narrowphase_functor =
    std::function< narrowphase_result_pair( const broadphase_collision< T > &, const broadphase_collision< T > & ) >;

  // collision_world( od_factor, world_config ) (src/bvh/collision_world.cpp:45-74); od_factor is a power of two.
  explicit collision_world(std::size_t od_factor, const world_config &cfg = {}) : m_od( od_factor ), m_cfg( cfg )
  {
    if ( od_factor == 0 || ( od_factor & ( od_factor - 1 ) ) ) throw error( BVHG_ERR_ARG, "od_factor must be a power of two" );
    bvhg_config c;
    bvhg_config_default( &c );
    c.k = cfg.k;
    c.precision = cfg.precision;
    c.epsilon = cfg.epsilon;
    c.device = cfg.device;
    c.stream = cfg.stream;
    bvhg_ctx *ctx = nullptr;
    detail::check( nullptr, bvhg_create( &ctx, &c ), "collision_world" );
    m_ctx.reset( ctx );
  }
  collision_world(const collision_world &) = delete;
  collision_world &operator=(const collision_world &) = delete;
  ~collision_world()
  {
    m_objects.clear();  // objects release their library handles before the context goes
  }

  collision_object &create_collision_object()
  {
    m_objects.emplace_back( new collision_object( *this, m_objects.size() ) );
    return *m_objects.back();
  }
  std::size_t num_collision_objects() const noexcept { return m_objects.size(); }
  std::size_t overdecomposition_factor() const noexcept { return m_od; }

  // collision_world::set_narrowphase_functor<T> (src/bvh/collision_world.hpp:58-94).
  template< typename T >
  void set_narrowphase_functor(narrowphase_functor< T > fun)
  {
    m_functor_type = detail::type_id< T >();
    m_functor = [fun](collision_object &oa, const patch &ma, const void *ea, std::size_t na, collision_object &ob,
                      const patch &mb, const void *eb, std::size_t nb,
                      span< const std::pair< uint32_t, uint32_t > > cand) {
      broadphase_collision< T > a{ oa, ma, ma.global_id(), span< const T >( static_cast< const T * >( ea ), na ), cand };
      broadphase_collision< T > b{ ob, mb, mb.global_id(), span< const T >( static_cast< const T * >( eb ), nb ), cand };
      return fun( a, b );
    };
  }

  // Iteration bracketing (src/bvh/collision_world.cpp:108-133): results of the previous iteration are dropped.
  void start_iteration()
  {
    for ( auto &o : m_objects ) o->m_results.clear();
  }
  void finish_iteration() { detail::check( ctx(), bvhg_synchronize( ctx() ), "finish_iteration" ); }

  bvhg_ctx *ctx() const { return m_ctx.get(); }
  const world_config &config() const { return m_cfg; }

private:
  friend class collision_object;
  struct ctx_deleter
  {
    void operator()(bvhg_ctx *c) const { bvhg_destroy( c ); }
  };
  std::size_t m_od;
  world_config m_cfg;
  std::unique_ptr< bvhg_ctx, ctx_deleter > m_ctx;
  std::vector< std::unique_ptr< collision_object > > m_objects;
  const void *m_functor_type = nullptr;
  std::function< narrowphase_result_pair( collision_object &, const patch &, const void *, std::size_t,
                                          collision_object &, const patch &, const void *, std::size_t,
                                          span< const std::pair< uint32_t, uint32_t > > ) >
    m_functor;
};

inline collision_object::collision_object(collision_world &w, std::size_t id) : m_world( w ), m_id( id )
{
  detail::check( ctx(), bvhg_object_create( ctx(), &m_obj ), "create_collision_object" );
}

inline bvhg_ctx *collision_object::ctx() const { return m_world.ctx(); }
inline int collision_object::overdecomposition_factor() const noexcept { return static_cast< int >( m_world.m_od ); }
inline std::size_t collision_object::num_patches() const noexcept { return m_world.m_od; }
inline int collision_object::world_k() const { return m_world.m_cfg.k; }

inline void collision_object::init_broadphase()
{
  detail::check( ctx(), bvhg_build( ctx(), m_obj, BVHG_REBUILD ), "init_broadphase" );
  // patches by the reference's Morton clustering, cut on the device (bvhg_cluster): only the patch bounds and the
  // element order come back
  const std::size_t P = m_world.m_od;
  std::vector< uint64_t > bounds( P + 1 );
  std::vector< uint32_t > order( m_n );
  detail::check( ctx(), bvhg_cluster( ctx(), m_obj, static_cast< uint32_t >( P ), bounds.data(), m_n ? order.data() : nullptr,
                                      BVHG_MEM_HOST ),
                 "init_broadphase" );
  m_pbeg.assign( bounds.begin(), bounds.end() );
  m_order = order;
  m_elems.bytes.assign( m_n * m_elems.elem_size, 0 );
  for ( std::size_t r = 0; r < m_n; ++r )
    std::memcpy( m_elems.bytes.data() + r * m_elems.elem_size, m_src.data() + order[r] * m_elems.elem_size,
                 m_elems.elem_size );
  // the patches' k-DOPs from the device (bvhg_patch_kdops), their centroids from the elements' (the library's
  // centroids are the reference's bit for bit), summed in patch order
  const int D = m_world.m_cfg.k / 2;
  std::vector< double > boxes( P * D * 2 );
  detail::check( ctx(), bvhg_patch_kdops( ctx(), m_obj, boxes.data(), BVHG_MEM_HOST ), "init_broadphase" );
  std::vector< double > cent( 3 * std::max< std::size_t >( m_n, 1 ) );
  if ( m_n ) detail::check( ctx(), bvhg_get_centroids( ctx(), m_obj, cent.data() ), "init_broadphase" );
  m_patches.clear();
  for ( std::size_t p = 0; p < P; ++p )
  {
    const std::size_t size = m_pbeg[p + 1] - m_pbeg[p];
    std::vector< double > box( boxes.begin() + static_cast< std::ptrdiff_t >( p * D * 2 ),
                               boxes.begin() + static_cast< std::ptrdiff_t >( ( p + 1 ) * D * 2 ) );
    std::array< double, 3 > c{ 0.0, 0.0, 0.0 };
    if ( size == 0 )
    {
      for ( int a = 0; a < D; ++a )
      {
        box[2 * a] = DBL_MAX;
        box[2 * a + 1] = -DBL_MAX;
      }
    } else {
      for ( std::size_t r = m_pbeg[p]; r < m_pbeg[p + 1]; ++r )
        for ( int a = 0; a < 3; ++a ) c[a] += cent[3 * order[r] + a];
      for ( int a = 0; a < 3; ++a ) c[a] /= static_cast< double >( size );
    }
    m_patches.emplace_back( m_id * P + p, size, std::move( box ), c );
  }
  m_built = true;
}

inline void collision_object::broadphase(collision_object &other)
{
  if ( !m_built || !other.m_built ) throw error( BVHG_ERR_STATE, "broadphase before init_broadphase" );
  // the exact element pairs, grouped by patch pair on the device (bvhg_patch_pairs): rows (patch here, patch there,
  // first pair, pair count) and pairs (position in this patch, position in the other patch)
  std::vector< uint32_t > groups( 4 * 64 ), pairs( 2 * 4096 );
  uint64_t ngroups = 0, npairs = 0;
  bvhg_status s = bvhg_patch_pairs( ctx(), m_obj, other.m_obj, groups.data(), groups.size() / 4, &ngroups, pairs.data(),
                                    pairs.size() / 2, &npairs, BVHG_MEM_HOST );
  if ( s == BVHG_ERR_OVERFLOW )
  {
    groups.resize( 4 * ngroups );
    pairs.resize( 2 * npairs );
    s = bvhg_patch_pairs( ctx(), m_obj, other.m_obj, groups.data(), ngroups, &ngroups, pairs.data(), npairs, &npairs,
                          BVHG_MEM_HOST );
  }
  detail::check( ctx(), s, "broadphase" );
  m_last_pairs.resize( npairs );
  for ( uint64_t g = 0; g < ngroups; ++g )
  {
    const std::size_t pa = groups[4 * g], pb = groups[4 * g + 1], first = groups[4 * g + 2], cnt = groups[4 * g + 3];
    for ( std::size_t q = first; q < first + cnt; ++q )
      m_last_pairs[q] = { m_gid[m_order[patch_begin( pa ) + pairs[2 * q]]],
                          other.m_gid[other.m_order[other.patch_begin( pb ) + pairs[2 * q + 1]]] };
  }
  if ( !m_world.m_functor ) return;
  if ( m_world.m_functor_type != m_elems.type || m_world.m_functor_type != other.m_elems.type )
    throw error( BVHG_ERR_ARG, "narrowphase functor element type differs from the objects' element type" );
  std::vector< std::pair< uint32_t, uint32_t > > cand;
  for ( uint64_t g = 0; g < ngroups; ++g )
  {
    const std::size_t pa = groups[4 * g], pb = groups[4 * g + 1], first = groups[4 * g + 2], cnt = groups[4 * g + 3];
    cand.resize( cnt );
    for ( std::size_t q = 0; q < cnt; ++q ) cand[q] = { pairs[2 * ( first + q )], pairs[2 * ( first + q ) + 1] };
    const std::size_t a0 = patch_begin( pa ), a1 = patch_begin( pa + 1 );
    const std::size_t b0 = other.patch_begin( pb ), b1 = other.patch_begin( pb + 1 );
    narrowphase_result_pair res = m_world.m_functor(
      *this, m_patches[pa], m_elems.bytes.data() + a0 * m_elems.elem_size, a1 - a0, other, other.m_patches[pb],
      other.m_elems.bytes.data() + b0 * other.m_elems.elem_size, b1 - b0,
      span< const std::pair< uint32_t, uint32_t > >( cand.data(), cand.size() ) );
    if ( res.a.size() ) m_results.push_back( std::move( res.a ) );
    if ( res.b.size() ) other.m_results.push_back( std::move( res.b ) );
  }
}
}  // namespace bvhg

#endif  // BVHG_HOST_COLLISION_WORLD_HPP
