// The collision_world mirror's Morton clustering (bvhg::detail::morton_cluster) on keys and a permutation read from
// a file (n, then n sorted 63-bit keys, then n element indices): prints the patch boundaries and the element order.
// Needs no GPU: the test computes the keys with the oracle.
#include "bvhg/collision_world.hpp"

#include <cstdio>
#include <cstdlib>
#include <vector>

int main(int argc, char **argv)
{
  if ( argc < 3 ) return 2;
  std::FILE *f = std::fopen( argv[1], "rb" );
  if ( !f ) return 2;
  uint64_t n = 0;
  if ( std::fread( &n, 8, 1, f ) != 1 ) return 2;
  std::vector< uint64_t > keys( n );
  std::vector< uint32_t > order( n );
  if ( std::fread( keys.data(), 8, n, f ) != n || std::fread( order.data(), 4, n, f ) != n ) return 2;
  std::fclose( f );
  const auto pbeg = bvhg::detail::morton_cluster( keys, order, std::strtoull( argv[2], nullptr, 10 ) );
  for ( std::size_t b : pbeg ) std::printf( "%zu ", b );
  std::printf( "\n" );
  for ( uint32_t e : order ) std::printf( "%u ", e );
  std::printf( "\n" );
  return 0;
}
