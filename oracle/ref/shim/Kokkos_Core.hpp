// Serial stand-in for the subset of Kokkos that the reference's element-broadphase headers use, so that those
// headers (included read-only from the reference's own source tree) compile and run on one host thread for the
// oracle's cross-check. Test scaffolding only: nothing of the product includes it.
#pragma once
#include <algorithm>
#include <bit>
#include <cstddef>
#include <cstdint>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

#define KOKKOS_INLINE_FUNCTION inline
#define KOKKOS_FORCEINLINE_FUNCTION inline
#define KOKKOS_FUNCTION
#define KOKKOS_LAMBDA [=]

namespace Kokkos
{
struct LayoutRight
{};
struct HostSpace
{
  using array_layout = LayoutRight;
  using memory_space = HostSpace;
};
struct Serial
{
  using array_layout = LayoutRight;
  using memory_space = HostSpace;
  using execution_space = Serial;
};
using DefaultExecutionSpace = Serial;
using DefaultHostExecutionSpace = Serial;
using OpenMP = Serial;

enum MemoryTraitsFlags : unsigned { Unmanaged = 1 };
template< unsigned >
struct MemoryTraits
{};

// One-dimensional views: owning (shared storage, like Kokkos' reference-counted views) or wrapping a pointer.
template< class DataType, class... Props >
class View
{
public:
  using value_type = std::remove_pointer_t< DataType >;
  using non_const_value_type = std::remove_const_t< value_type >;
  using pointer_type = value_type *;
  using HostMirror = View;
  using size_type = std::size_t;

  View() = default;
  // rank 1 (DataType = T*) holds n values; rank 0 (DataType = T) one value, read as v()
  explicit View(const std::string &, std::size_t n = 0)
  {
    const std::size_t count = std::is_pointer_v< DataType > ? n : 1;
    m_store = std::make_shared< std::vector< non_const_value_type > >( count );
    m_ptr = m_store->data();
    m_size = count;
  }
  View(pointer_type p, std::size_t n) : m_ptr( p ), m_size( n ) {}
  template< class... P2 >
  View(const View< std::remove_const_t< DataType >, P2... > &o) : m_ptr( o.data() ), m_size( o.size() )
  {}

  value_type &operator()() const { return m_ptr[0]; }
  value_type &operator()(std::size_t i) const { return m_ptr[i]; }
  value_type &operator[](std::size_t i) const { return m_ptr[i]; }
  pointer_type data() const { return m_ptr; }
  std::size_t size() const { return m_size; }
  std::size_t extent(int) const { return m_size; }
  std::size_t span() const { return m_size; }

  void resize_storage(std::size_t n)
  {
    if ( !m_store ) m_store = std::make_shared< std::vector< non_const_value_type > >();
    m_store->resize( n );
    m_ptr = m_store->data();
    m_size = n;
  }

private:
  std::shared_ptr< std::vector< non_const_value_type > > m_store;
  pointer_type m_ptr = nullptr;
  std::size_t m_size = 0;
};

// Two-dimensional views with a static second extent (DataType = T*[N]): element (i, j) at i * N + j.
template< class T, std::size_t N, class... Props >
class View< T *[N], Props... >
{
public:
  using value_type = T;
  using size_type = std::size_t;

  View() = default;
  explicit View(const std::string &, std::size_t n = 0)
      : m_store( std::make_shared< std::vector< std::remove_const_t< T > > >( n * N ) ), m_rows( n )
  {}
  T &operator()(std::size_t i, std::size_t j) const { return ( *m_store )[i * N + j]; }
  T *data() const { return m_store ? m_store->data() : nullptr; }
  std::size_t size() const { return m_rows * N; }
  std::size_t extent(int d) const { return d == 0 ? m_rows : N; }

private:
  std::shared_ptr< std::vector< std::remove_const_t< T > > > m_store;
  std::size_t m_rows = 0;
};

inline void fence() {}

template< class V >
void resize(V &v, std::size_t n)
{
  v.resize_storage( n );
}
template< class V >
V create_mirror_view(const V &v)
{
  return v;
}
template< class V, class T >
std::enable_if_t< std::is_arithmetic_v< T > > deep_copy(const V &v, const T &x)
{
  for ( std::size_t i = 0; i < v.size(); ++i ) v( i ) = x;
}
template< class A, class B >
std::enable_if_t< !std::is_arithmetic_v< B > > deep_copy(const A &dst, const B &src)
{
  for ( std::size_t i = 0; i < dst.size(); ++i ) dst( i ) = src( i );
}

template< class... >
struct RangePolicy
{
  std::size_t b, e;
  RangePolicy(std::size_t b_, std::size_t e_) : b( b_ ), e( e_ ) {}
};

template< class F, class... P >
void parallel_for(const RangePolicy< P... > &p, const F &f)
{
  for ( std::size_t i = p.b; i < p.e; ++i ) f( static_cast< int >( i ) );
}

namespace detail
{
template< class M >
struct scan_value;
template< class C, class R, class A0, class A1, class A2 >
struct scan_value< R ( C::* )( A0, A1, A2 ) const >
{
  using type = std::remove_cv_t< std::remove_reference_t< A1 > >;
};
}  // namespace detail

// One host thread: the scan functor sees every index once, in order, with final = true.
template< class F >
void parallel_scan(std::size_t n, const F &f)
{
  typename detail::scan_value< decltype( &F::operator() ) >::type acc{};
  for ( std::size_t i = 0; i < n; ++i ) f( static_cast< int >( i ), acc, true );
}

template< class F >
void parallel_for(std::size_t n, const F &f)
{
  for ( std::size_t i = 0; i < n; ++i ) f( static_cast< int >( i ) );
}
template< class F >
void parallel_for(const std::string &, std::size_t n, const F &f)
{
  parallel_for( n, f );
}
namespace detail
{
template< class F, class = void >
struct has_value_type : std::false_type
{};
template< class F >
struct has_value_type< F, std::void_t< typename F::value_type > > : std::true_type
{};
template< class R, class = void >
struct is_view : std::false_type
{};
template< class R >
struct is_view< R, std::void_t< decltype( std::declval< R & >().data() ) > > : std::true_type
{};
}  // namespace detail

// One host thread: a reducer functor (value_type, init, operator()) accumulates into one init'd value, as a
// serial Kokkos backend does (join is never needed); a plain lambda sums into a zero-initialised value.
template< class F, class R >
void parallel_reduce(std::size_t n, const F &f, R &&result)
{
  using RR = std::remove_cv_t< std::remove_reference_t< R > >;
  if constexpr ( detail::has_value_type< F >::value )
  {
    using VT = typename F::value_type;
    if constexpr ( std::is_array_v< VT > && std::extent_v< VT > == 0 )
    {
      // array reducer (value_type = T[], F::value_count entries), result an array of as many
      F g = f;  // Kokkos runs a copy of the functor (its init need not be const)
      std::vector< std::remove_extent_t< VT > > acc( F::value_count );
      g.init( acc.data() );
      for ( std::size_t i = 0; i < n; ++i ) g( i, acc.data() );
      for ( std::size_t k = 0; k < F::value_count; ++k ) result[k] = acc[k];
    } else {
      VT acc;
      f.init( acc );
      for ( std::size_t i = 0; i < n; ++i ) f( i, acc );
      if constexpr ( detail::is_view< RR >::value ) result() = acc;
      else result = acc;
    }
  } else {
    RR acc{};
    for ( std::size_t i = 0; i < n; ++i ) f( static_cast< int >( i ), acc );
    result = acc;
  }
}
template< class F, class R >
void parallel_reduce(const std::string &, std::size_t n, const F &f, R &&result)
{
  parallel_reduce( n, f, std::forward< R >( result ) );
}

template< class T >
constexpr int countl_zero(T x) noexcept
{
  return std::countl_zero( x );
}
template< class T >
constexpr const T &min(const T &a, const T &b)
{
  return std::min( a, b );
}
template< class T >
constexpr const T &max(const T &a, const T &b)
{
  return std::max( a, b );
}

namespace Impl
{
template< class T >
constexpr int int_log2(T x)
{
  return static_cast< int >( sizeof( T ) * 8 - 1 ) - std::countl_zero( x );
}
}  // namespace Impl
}  // namespace Kokkos
