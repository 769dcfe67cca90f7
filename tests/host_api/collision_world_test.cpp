// Drives the C++ host mirror of collision_world / collision_object (distbvh_b200/host/bvhg/collision_world.hpp)
// the way the reference's collision_object test drives its API (tests/collision_object_test.cpp:395-430): two
// objects, a narrowphase functor that records (patch a, element a, patch b, element b) for every candidate, the
// results read back with for_each_result. Reads two element files (n, then n * 9 doubles of triangle vertices)
// and prints "pairs <count>" followed by the recorded element gid pairs, one per line.
#include "bvhg/collision_world.hpp"

#include <algorithm>
#include <array>
#include <cfloat>
#include <cstdio>
#include <string>
#include <vector>

namespace
{
struct tri_element
{
  std::array< std::array< double, 3 >, 3 > v;
  std::size_t gid;
  const std::array< std::array< double, 3 >, 3 > &vertices() const { return v; }
  std::size_t global_id() const { return gid; }
};

struct detailed_result
{
  std::size_t patch_a, elem_a, patch_b, elem_b;
};

std::vector< tri_element > read_elements(const char *path, std::size_t gid_base)
{
  std::FILE *f = std::fopen( path, "rb" );
  if ( !f ) throw std::runtime_error( "cannot open input" );
  uint64_t n = 0;
  if ( std::fread( &n, 8, 1, f ) != 1 ) throw std::runtime_error( "bad input" );
  std::vector< double > xyz( n * 9 );
  if ( std::fread( xyz.data(), 8, xyz.size(), f ) != xyz.size() ) throw std::runtime_error( "bad input" );
  std::fclose( f );
  std::vector< tri_element > el( n );
  for ( uint64_t i = 0; i < n; ++i )
  {
    for ( int v = 0; v < 3; ++v )
      for ( int c = 0; c < 3; ++c ) el[i].v[v][c] = xyz[i * 9 + v * 3 + c];
    el[i].gid = gid_base + i;
  }
  return el;
}
}  // namespace

// "empty <od>": an object without elements (the reference's set_empty_data section,
// tests/collision_object_test.cpp:207-240): od empty patches with the default k-DOP, an empty tree.
int empty_object(std::size_t od)
{
  bvhg::collision_world world( od );
  auto &obj = world.create_collision_object();
  obj.set_entity_data( std::vector< tri_element >{}, bvhg::split_algorithm::clustering );
  obj.init_broadphase();
  if ( obj.local_patches().size() != od ) return 4;
  for ( const auto &p : obj.local_patches() )
  {
    if ( !p.empty() || p.size() != 0 ) return 5;
    for ( std::size_t a = 0; a < p.kdop().size(); a += 2 )
      if ( p.kdop()[a] != DBL_MAX || p.kdop()[a + 1] != -DBL_MAX ) return 6;
  }
  std::size_t count = 1;
  obj.for_each_tree( [&](const bvhg::snapshot_tree &t) { count = t.count() + ( t.empty() ? 0 : 1 ); } );
  std::printf( "empty %zu\n", count );
  return count == 0 ? 0 : 7;
}

int main(int argc, char **argv)
{
  if ( argc == 3 && std::string( argv[1] ) == "empty" ) return empty_object( static_cast< std::size_t >( std::atoi( argv[2] ) ) );
  if ( argc < 5 ) return 2;
  const std::size_t od = static_cast< std::size_t >( std::atoi( argv[3] ) );
  bvhg::world_config cfg;
  cfg.k = std::atoi( argv[4] );
  auto ea = read_elements( argv[1], 0 );
  auto eb = read_elements( argv[2], 1000000 );

  bvhg::collision_world world( od, cfg );
  auto &obj = world.create_collision_object();
  auto &obj2 = world.create_collision_object();
  obj.set_entity_data( ea, bvhg::split_algorithm::clustering );
  obj.init_broadphase();
  obj2.set_entity_data( eb, bvhg::split_algorithm::clustering );
  obj2.init_broadphase();

  std::size_t calls = 0;
  world.set_narrowphase_functor< tri_element >(
    [&](const bvhg::broadphase_collision< tri_element > &a, const bvhg::broadphase_collision< tri_element > &b) {
      ++calls;
      bvhg::narrowphase_result_pair res;
      res.a = bvhg::narrowphase_result( sizeof( detailed_result ) );
      res.b = bvhg::narrowphase_result( sizeof( detailed_result ) );
      auto &ra = static_cast< bvhg::typed_narrowphase_result< detailed_result > & >( res.a );
      if ( a.object.id() != 0 || b.object.id() != 1 ) throw std::runtime_error( "object ids" );
      // the functor's patches are the objects' own (local_patches), with their elements
      if ( &a.meta != &a.object.local_patches()[a.meta.global_id() % od] || a.meta.size() != a.elements.size() ||
           &b.meta != &b.object.local_patches()[b.meta.global_id() % od] || b.meta.size() != b.elements.size() )
        throw std::runtime_error( "patch metadata" );
      for ( const auto &c : a.candidates )
        ra.emplace_back( detailed_result{ a.meta.global_id(), a.elements[c.first].global_id(), b.meta.global_id(),
                                          b.elements[c.second].global_id() } );
      return res;
    } );

  world.start_iteration();
  obj.broadphase( obj2 );
  world.finish_iteration();

  std::vector< std::pair< std::size_t, std::size_t > > got;
  obj.for_each_result< detailed_result >( [&](const detailed_result &r) {
    if ( r.patch_a / od != 0 || r.patch_b / od != 1 ) throw std::runtime_error( "patch ids" );
    got.emplace_back( r.elem_a, r.elem_b );
  } );
  std::sort( got.begin(), got.end() );
  if ( got.size() != obj.last_pairs().size() ) return 3;
  std::printf( "pairs %zu calls %zu\n", got.size(), calls );
  for ( const auto &p : got ) std::printf( "%zu %zu\n", p.first, p.second );
  // the first object's patches (local_patches) and the tree over them (for_each_tree), as in the reference's
  // collision_object init test (tests/collision_object_test.cpp:136-170): exact values in hexadecimal floats
  for ( const auto &p : obj.local_patches() )
  {
    std::printf( "patch %zu %zu", p.global_id(), p.size() );
    for ( double v : p.kdop() ) std::printf( " %a", v );
    for ( double v : p.centroid() ) std::printf( " %a", v );
    std::printf( "\n" );
  }
  obj.for_each_tree( [](const bvhg::snapshot_tree &t) {
    std::size_t leaves = 0;
    for ( const auto &n : t.nodes() ) leaves += n.leaf() ? 1 : 0;
    std::printf( "tree %zu %zu %zu\n", t.count(), t.nodes().size(), leaves );
  } );
  obj.end_phase();
  obj2.end_phase();
  return 0;
}
