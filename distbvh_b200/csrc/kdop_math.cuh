// kdop_math.cuh — k-DOP slab arithmetic on the device.
//
// FP64 slabs follow kdop_base::from_vertices (src/bvh/kdop.hpp:238-264) bit for bit: every projection is
// ((v0 * n0) + (v1 * n1)) + (v2 * n2) (kdop.hpp:223-227) with each product and sum rounded separately
// (__dmul_rn / __dadd_rn stop nvcc from contracting them into FMAs), then proj - eps / proj + eps, then
// std::min / std::max over the vertices.
//
// FP32 slabs (precision form) enclose the FP64 slabs: lo32 <= lo64 and hi32 >= hi64 for every element and
// slab, computed with FP32 directed rounding only (interval products and sums, then a widening by an explicit
// bound on the FP64 evaluation error). Strict overlap then carries over: a64.min < b64.max implies
// a32.min <= a64.min < b64.max <= b32.max, so the FP32 candidate set is a superset of the FP64 pair set.
#pragma once

#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

namespace bvhg {

// epsilon rounded up to FP32 (host side): the FP32 enclosure's inflation.
inline float f32_round_up(double x)
{
  if ( x == 0.0 ) return 0.f;
  float f = static_cast< float >( x );
  if ( static_cast< double >( f ) < x ) f = nextafterf( f, INFINITY );
  return f;
}

constexpr double kOverRoot2 = 0.7071067811865475;  // dop_18::over_root_2, dop_26::one_over_root_2 (kdop.hpp:608,659)
constexpr double kOverRoot3 = 0.5773502691896258;  // dop_26::one_over_root_3 (kdop.hpp:660)

// Component c of normal a of the K-DOP (the first K/2 normals: kdop.hpp:583-587, 613-624, 662-677).
template< int K >
__host__ __device__ constexpr double normal_comp(int a, int c)
{
  if ( a < 3 ) return a == c ? 1.0 : 0.0;
  if ( K == 18 || ( K == 26 && a >= 7 ) )
  {
    const int e = ( K == 18 ) ? a - 3 : a - 7;  // edge normals
    // (r,r,0) (r,0,r) (0,r,r) (r,-r,0) (r,0,-r) (0,r,-r)
    const int zero_c = ( e % 3 == 0 ) ? 2 : ( ( e % 3 == 1 ) ? 1 : 0 );
    if ( c == zero_c ) return 0.0;
    const bool second = ( c == ( e % 3 == 2 ? 2 : ( e % 3 == 0 ? 1 : 2 ) ) );
    if ( e >= 3 && second ) return -kOverRoot2;
    return kOverRoot2;
  }
  // K == 26 corners, a in [3, 7): (s,s,s) (s,-s,s) (s,s,-s) (s,-s,-s)
  const int cidx = a - 3;
  if ( c == 0 ) return kOverRoot3;
  if ( c == 1 ) return ( cidx & 1 ) ? -kOverRoot3 : kOverRoot3;
  return ( cidx & 2 ) ? -kOverRoot3 : kOverRoot3;
}

// FP64 projection exactly as kdop.hpp:226 evaluates it (no FMA contraction).
template< int K >
__device__ __forceinline__ double project64(const double v0, const double v1, const double v2, const int a)
{
  const double t0 = __dmul_rn( v0, normal_comp< K >( a, 0 ) );
  const double t1 = __dmul_rn( v1, normal_comp< K >( a, 1 ) );
  const double t2 = __dmul_rn( v2, normal_comp< K >( a, 2 ) );
  return __dadd_rn( __dadd_rn( t0, t1 ), t2 );
}

// std::min / std::max (libstdc++): min(a, b) = (b < a) ? b : a; max(a, b) = (a < b) ? b : a.
__device__ __forceinline__ double std_min(double a, double b) { return ( b < a ) ? b : a; }
__device__ __forceinline__ double std_max(double a, double b) { return ( a < b ) ? b : a; }

// Slab a of one element from its V vertices (vertex v at p[3 v + c]), FP64, as from_vertices.
template< int K >
__device__ __forceinline__ void slab64(const double *p, int V, int a, double eps, double &mn, double &mx)
{
  double proj = project64< K >( p[0], p[1], p[2], a );
  mn = __dsub_rn( proj, eps );
  mx = __dadd_rn( proj, eps );
  for ( int v = 1; v < V; ++v )
  {
    proj = project64< K >( p[3 * v], p[3 * v + 1], p[3 * v + 2], a );
    mn = std_min( mn, __dsub_rn( proj, eps ) );
    mx = std_max( mx, __dadd_rn( proj, eps ) );
  }
}

// ---- FP64 overlap outcome (no slab bits) ---------------------------------------------------------------
//
// The recheck of the precision form needs the outcome of the strict overlap test, not the slab bits. The
// projections below equal project64's in value; they may differ only in the sign of a zero, which no comparison
// sees. A product by 0 is a zero that the sums absorb (t + (+-0) == t), a product by 1 is the coordinate, a
// product by -c is -(v * c) exactly, and each product v_k * c shared by several normals is rounded once. The
// epsilon shift is monotone under round-to-nearest, so min over vertices of (p - eps) == (min p) - eps, and it is
// applied once per slab. Per tetrahedron at K = 26 this is 72 FP64 operations for the projections instead of 260.

// Projections of one vertex onto the normals of group G: 0 = the axes (normals 0..2), 1 = the edge normals
// (r,r,0) (r,0,r) (0,r,r) (r,-r,0) (r,0,-r) (0,r,-r), 2 = the corner normals (s,s,s) (s,-s,s) (s,s,-s) (s,-s,-s),
// in normal_comp's order within the group.
template< int G >
__device__ __forceinline__ void project_group(const double v0, const double v1, const double v2, double *p)
{
  if constexpr ( G == 0 )
  {
    p[0] = v0;
    p[1] = v1;
    p[2] = v2;
  } else if constexpr ( G == 1 ) {
    const double m0 = __dmul_rn( v0, kOverRoot2 ), m1 = __dmul_rn( v1, kOverRoot2 ), m2 = __dmul_rn( v2, kOverRoot2 );
    p[0] = __dadd_rn( m0, m1 );
    p[1] = __dadd_rn( m0, m2 );
    p[2] = __dadd_rn( m1, m2 );
    p[3] = __dsub_rn( m0, m1 );
    p[4] = __dsub_rn( m0, m2 );
    p[5] = __dsub_rn( m1, m2 );
  } else {
    const double c0 = __dmul_rn( v0, kOverRoot3 ), c1 = __dmul_rn( v1, kOverRoot3 ), c2 = __dmul_rn( v2, kOverRoot3 );
    const double s = __dadd_rn( c0, c1 ), d = __dsub_rn( c0, c1 );
    p[0] = __dadd_rn( s, c2 );
    p[1] = __dadd_rn( d, c2 );
    p[2] = __dsub_rn( s, c2 );
    p[3] = __dsub_rn( d, c2 );
  }
}

template< int G >
constexpr int group_size = G == 0 ? 3 : ( G == 1 ? 6 : 4 );

// Strict overlap of two elements (V* vertices each at x*[3 v + c]) over the slabs of group G, with the same
// outcome as comparing slab64's values.
template< int G, int VA, int VB >
__device__ __forceinline__ bool group_overlap64(const double *xa, const double *xb, double eps)
{
  constexpr int N = group_size< G >;
  double alo[N], ahi[N], blo[N], bhi[N];
#pragma unroll
  for ( int v = 0; v < VA; ++v )
  {
    double p[N];
    project_group< G >( xa[3 * v], xa[3 * v + 1], xa[3 * v + 2], p );
#pragma unroll
    for ( int k = 0; k < N; ++k )
    {
      alo[k] = v ? fmin( alo[k], p[k] ) : p[k];
      ahi[k] = v ? fmax( ahi[k], p[k] ) : p[k];
    }
  }
#pragma unroll
  for ( int v = 0; v < VB; ++v )
  {
    double p[N];
    project_group< G >( xb[3 * v], xb[3 * v + 1], xb[3 * v + 2], p );
#pragma unroll
    for ( int k = 0; k < N; ++k )
    {
      blo[k] = v ? fmin( blo[k], p[k] ) : p[k];
      bhi[k] = v ? fmax( bhi[k], p[k] ) : p[k];
    }
  }
  bool ok = true;
#pragma unroll
  for ( int k = 0; k < N; ++k )
    ok = ok && __dsub_rn( alo[k], eps ) < __dadd_rn( bhi[k], eps ) && __dsub_rn( blo[k], eps ) < __dadd_rn( ahi[k], eps );
  return ok;
}

// Strict overlap of two elements over all K/2 slabs (the FP64 pair-set test), group by group.
template< int K, int VA, int VB >
__device__ __forceinline__ bool overlap64(const double *xa, const double *xb, double eps)
{
  bool ok = group_overlap64< 0, VA, VB >( xa, xb, eps );
  if constexpr ( K >= 18 )
    if ( ok ) ok = group_overlap64< 1, VA, VB >( xa, xb, eps );
  if constexpr ( K == 26 )
    if ( ok ) ok = group_overlap64< 2, VA, VB >( xa, xb, eps );
  return ok;
}

// ---- FP32 enclosure ------------------------------------------------------------------------------------

// Error bound constant: the FP64 value of ((t0 + t1) + t2), t_k = fl(v_k n_k), differs from the exact sum by
// at most gamma_3 * sum |v_k n_k| with gamma_3 = 3u / (1 - 3u), u = 2^-53; 2^-51 > gamma_3.
constexpr float kTwoPowM51 = 4.44089209850062616169452667236328125e-16f;  // 2^-51, exact in FP32
constexpr float kTwoPowM52 = 2.220446049250313080847263336181640625e-16f; // 2^-52, exact in FP32

// Product interval of an FP32 interval [alo, ahi] (both roundings of one FP64 value, so they never straddle 0)
// with the FP32 interval [nlo, nhi] of a nonzero constant of known sign.
__device__ __forceinline__ void mul_interval(float alo, float ahi, float nlo, float nhi, bool npos, float &lo,
                                             float &hi)
{
  if ( npos )
  {
    lo = __fmul_rd( alo, alo >= 0.f ? nlo : nhi );
    hi = __fmul_ru( ahi, ahi >= 0.f ? nhi : nlo );
  } else {
    lo = __fmul_rd( ahi, ahi >= 0.f ? nlo : nhi );
    hi = __fmul_ru( alo, alo >= 0.f ? nhi : nlo );
  }
}

// FP32 enclosures of the two irrational normal magnitudes: lo = the largest float <= c, hi = the smallest
// float >= c (hex literals; bvhg_debug_normal_interval exposes them so a CPU test checks the bracketing).
constexpr float kOverRoot2Lo = 0x1.6a09e6p-1f;
constexpr float kOverRoot2Hi = 0x1.6a09e8p-1f;
constexpr float kOverRoot3Lo = 0x1.279a74p-1f;
constexpr float kOverRoot3Hi = 0x1.279a76p-1f;

// FP32 interval [lo, hi] of normal component (a, c).
template< int K >
__host__ __device__ constexpr float normal_lo(int a, int c)
{
  const double v = normal_comp< K >( a, c );
  if ( v == kOverRoot2 ) return kOverRoot2Lo;
  if ( v == -kOverRoot2 ) return -kOverRoot2Hi;
  if ( v == kOverRoot3 ) return kOverRoot3Lo;
  if ( v == -kOverRoot3 ) return -kOverRoot3Hi;
  return static_cast< float >( v );  // 0, 1, -1: exact
}

template< int K >
__host__ __device__ constexpr float normal_hi(int a, int c)
{
  const double v = normal_comp< K >( a, c );
  if ( v == kOverRoot2 ) return kOverRoot2Hi;
  if ( v == -kOverRoot2 ) return -kOverRoot2Lo;
  if ( v == kOverRoot3 ) return kOverRoot3Hi;
  if ( v == -kOverRoot3 ) return -kOverRoot3Lo;
  return static_cast< float >( v );
}

// FP32 enclosure of slab a of one element: lo <= the FP64 slab min and hi >= the FP64 slab max that slab64
// computes for the same vertices and epsilon. eps_hi is epsilon rounded up to FP32 (0 when epsilon is 0).
template< int K >
__device__ __forceinline__ void slab32(const double *p, int V, int a, float eps_hi, float &lo, float &hi)
{
  const double n0 = normal_comp< K >( a, 0 ), n1 = normal_comp< K >( a, 1 ), n2 = normal_comp< K >( a, 2 );
  const int nz = ( n0 != 0.0 ) + ( n1 != 0.0 ) + ( n2 != 0.0 );
  // A single unit component: the FP64 projection is the coordinate itself, exactly.
  const bool exact = ( nz == 1 ) && ( n0 == 1.0 || n0 == -1.0 || n1 == 1.0 || n1 == -1.0 || n2 == 1.0 || n2 == -1.0 );
  const float inf = __int_as_float( 0x7f800000 );
  lo = inf;
  hi = -inf;
  for ( int v = 0; v < V; ++v )
  {
    float slo = 0.f, shi = 0.f, mag = 0.f;
    bool first = true;
#pragma unroll
    for ( int c = 0; c < 3; ++c )
    {
      const double nc = normal_comp< K >( a, c );
      if ( nc == 0.0 ) continue;
      const double x = p[3 * v + c];
      const float xlo = __double2float_rd( x ), xhi = __double2float_ru( x );
      float tlo, thi;
      if ( nc == 1.0 )
      {
        tlo = xlo;
        thi = xhi;
      } else if ( nc == -1.0 ) {
        tlo = -xhi;
        thi = -xlo;
      } else {
        mul_interval( xlo, xhi, normal_lo< K >( a, c ), normal_hi< K >( a, c ), nc > 0.0, tlo, thi );
      }
      const float tmag = fmaxf( fabsf( tlo ), fabsf( thi ) );
      if ( first )
      {
        slo = tlo;
        shi = thi;
        mag = tmag;
        first = false;
      } else {
        slo = __fadd_rd( slo, tlo );
        shi = __fadd_ru( shi, thi );
        mag = __fadd_ru( mag, tmag );
      }
    }
    if ( !exact )
    {
      const float e = __fmul_ru( mag, kTwoPowM51 );
      slo = __fsub_rd( slo, e );
      shi = __fadd_ru( shi, e );
    }
    if ( eps_hi != 0.f )
    {
      const float m2 = __fadd_ru( fmaxf( fabsf( slo ), fabsf( shi ) ), eps_hi );
      const float e2 = __fmul_ru( m2, kTwoPowM52 );
      slo = __fsub_rd( __fsub_rd( slo, eps_hi ), e2 );
      shi = __fadd_ru( __fadd_ru( shi, eps_hi ), e2 );
    }
    lo = fminf( lo, slo );
    hi = fmaxf( hi, shi );
  }
}

// All K/2 FP32 enclosures of one element with V vertices, bit for bit the values slab32 gives slab by slab, with
// the shared work done once per vertex: each coordinate is rounded down and up once, and the product interval of a
// coordinate by a normal magnitude is formed once for all normals that use it (a component -c gives the negated
// interval exactly, because directed rounding is symmetric under negation: rd(-z) = -ru(z)). Sums, magnitudes,
// the widening and the epsilon step run in slab32's order.
template< int K, int V >
__device__ __forceinline__ void slabs32_all(const double *p, float eps_hi, float *lo, float *hi)
{
  constexpr int D = K / 2;
  const float inf = __int_as_float( 0x7f800000 );
#pragma unroll
  for ( int a = 0; a < D; ++a )
  {
    lo[a] = inf;
    hi[a] = -inf;
  }
  // widening by the FP64 evaluation error (not for the axes, whose projection is the coordinate), the epsilon
  // step, and the running min / max over the vertices: slab32's tail
  auto finish = [&](int a, float slo, float shi, float mag, bool exact) {
    if ( !exact )
    {
      const float e = __fmul_ru( mag, kTwoPowM51 );
      slo = __fsub_rd( slo, e );
      shi = __fadd_ru( shi, e );
    }
    if ( eps_hi != 0.f )
    {
      const float m2 = __fadd_ru( fmaxf( fabsf( slo ), fabsf( shi ) ), eps_hi );
      const float e2 = __fmul_ru( m2, kTwoPowM52 );
      slo = __fsub_rd( __fsub_rd( slo, eps_hi ), e2 );
      shi = __fadd_ru( __fadd_ru( shi, eps_hi ), e2 );
    }
    lo[a] = fminf( lo[a], slo );
    hi[a] = fmaxf( hi[a], shi );
  };
#pragma unroll
  for ( int v = 0; v < V; ++v )
  {
    float xl[3], xh[3];
#pragma unroll
    for ( int c = 0; c < 3; ++c )
    {
      xl[c] = __double2float_rd( p[3 * v + c] );
      xh[c] = __double2float_ru( p[3 * v + c] );
    }
#pragma unroll
    for ( int c = 0; c < 3; ++c ) finish( c, xl[c], xh[c], 0.f, true );
    if constexpr ( K == 26 )
    {
      // corners (s,s,s) (s,-s,s) (s,s,-s) (s,-s,-s): normals 3..6
      float tl[3], th[3];
#pragma unroll
      for ( int c = 0; c < 3; ++c ) mul_interval( xl[c], xh[c], kOverRoot3Lo, kOverRoot3Hi, true, tl[c], th[c] );
      const float mag = __fadd_ru( __fadd_ru( fmaxf( fabsf( tl[0] ), fabsf( th[0] ) ), fmaxf( fabsf( tl[1] ), fabsf( th[1] ) ) ),
                                   fmaxf( fabsf( tl[2] ), fabsf( th[2] ) ) );
#pragma unroll
      for ( int q = 0; q < 4; ++q )
      {
        const float l1 = ( q & 1 ) ? -th[1] : tl[1], h1 = ( q & 1 ) ? -tl[1] : th[1];
        const float l2 = ( q & 2 ) ? -th[2] : tl[2], h2 = ( q & 2 ) ? -tl[2] : th[2];
        finish( 3 + q, __fadd_rd( __fadd_rd( tl[0], l1 ), l2 ), __fadd_ru( __fadd_ru( th[0], h1 ), h2 ), mag, false );
      }
    }
    if constexpr ( K >= 18 )
    {
      // edges (r,r,0) (r,0,r) (0,r,r) (r,-r,0) (r,0,-r) (0,r,-r): normals 3..8 (K = 18) or 7..12 (K = 26)
      constexpr int E = K == 18 ? 3 : 7;
      float tl[3], th[3], tm[3];
#pragma unroll
      for ( int c = 0; c < 3; ++c )
      {
        mul_interval( xl[c], xh[c], kOverRoot2Lo, kOverRoot2Hi, true, tl[c], th[c] );
        tm[c] = fmaxf( fabsf( tl[c] ), fabsf( th[c] ) );
      }
#pragma unroll
      for ( int e = 0; e < 6; ++e )
      {
        const int c1 = ( e % 3 == 2 ) ? 1 : 0, c2 = ( e % 3 == 0 ) ? 1 : 2;
        const bool neg = e >= 3;
        const float l2 = neg ? -th[c2] : tl[c2], h2 = neg ? -tl[c2] : th[c2];
        finish( E + e, __fadd_rd( tl[c1], l2 ), __fadd_ru( th[c1], h2 ), __fadd_ru( tm[c1], tm[c2] ), false );
      }
    }
  }
}

// Slabs of element e (gathered vertices) into lo/hi.
template< int K, typename T, int VT >
__device__ __forceinline__ void leaf_slabs(const double *__restrict__ verts, uint32_t Vrt, uint32_t e, double eps,
                                           float eps_hi, T *lo, T *hi)
{
  constexpr int D = K / 2;
  constexpr int VMAX = VT > 0 ? VT : 32;
  const int V = VT > 0 ? VT : static_cast< int >( Vrt );
  double p[VT > 0 ? VT * 3 : 3];
  const double *src = verts + static_cast< size_t >( e ) * V * 3;
  if constexpr ( VT > 0 )
  {
#pragma unroll
    for ( int k = 0; k < VT * 3; ++k ) p[k] = __ldg( src + k );
    if constexpr ( sizeof( T ) == 8 )
    {
#pragma unroll
      for ( int a = 0; a < D; ++a )
      {
        double l, h;
        slab64< K >( p, VT, a, eps, l, h );
        lo[a] = l;
        hi[a] = h;
      }
    } else {
      slabs32_all< K, VT >( p, eps_hi, lo, hi );
    }
  } else {
    (void)VMAX;
    (void)p;
    // Generic vertex count: one vertex at a time, slab by slab (vertices re-read from L1).
#pragma unroll
    for ( int a = 0; a < D; ++a )
    {
      if constexpr ( sizeof( T ) == 8 )
      {
        double l = 0, h = 0;
        for ( int v = 0; v < V; ++v )
        {
          const double q[3] = { __ldg( src + 3 * v ), __ldg( src + 3 * v + 1 ), __ldg( src + 3 * v + 2 ) };
          double vl, vh;
          slab64< K >( q, 1, a, eps, vl, vh );
          if ( v == 0 )
          {
            l = vl;
            h = vh;
          } else {
            l = std_min( l, vl );
            h = std_max( h, vh );
          }
        }
        lo[a] = l;
        hi[a] = h;
      } else {
        float l = 0, h = 0;
        for ( int v = 0; v < V; ++v )
        {
          const double q[3] = { __ldg( src + 3 * v ), __ldg( src + 3 * v + 1 ), __ldg( src + 3 * v + 2 ) };
          float vl, vh;
          slab32< K >( q, 1, a, eps_hi, vl, vh );
          if ( v == 0 )
          {
            l = vl;
            h = vh;
          } else {
            l = fminf( l, vl );
            h = fmaxf( h, vh );
          }
        }
        lo[a] = l;
        hi[a] = h;
      }
    }
  }
}

}  // namespace bvhg
