// bvhg_api.cu — the C ABI declared in include/bvhg.h: contexts, objects and the per-object pipeline
// K1 (centroids + Morton bounds) -> K2 (keys + digit histograms) -> K3 (radix passes) -> K4/K5 (leaf slabs, LBVH
// build, refit) and the pairwise K6 (traversal) -> K7 (FP64 recheck, precision form) -> gid output.
#include "../../include/bvhg.h"
#include "bvhg_internal.cuh"
#include "kdop_math.cuh"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

namespace bvhg {
cudaError_t launch_gid_pairs(const uint2 *pairs, uint64_t count, const uint64_t *gid_a, const uint64_t *gid_b,
                             bool normalize, uint64_t *out, cudaStream_t s);
int device_sm_count();
}  // namespace bvhg

using namespace bvhg;

namespace {

constexpr uint32_t kDefaultSpinLimit = 1u << 22;
constexpr uint64_t kMaxElements = ( 1ull << 30 ) - 1;  // 30-bit radix status counters, int32 node links

struct dev_buf
{
  void *p = nullptr;
  size_t bytes = 0;
  dev_buf() = default;
  dev_buf(const dev_buf &) = delete;
  dev_buf &operator=(const dev_buf &) = delete;
  ~dev_buf()
  {
    if ( p ) cudaFree( p );
  }
  cudaError_t reserve(size_t b)
  {
    if ( b <= bytes ) return cudaSuccess;
    if ( p ) cudaFree( p );
    p = nullptr;
    bytes = 0;
    size_t want = b < 256 ? 256 : b;
    cudaError_t e = cudaMalloc( &p, want );
    if ( e != cudaSuccess )
    {
      p = nullptr;
      return e;
    }
    bytes = want;
    return cudaSuccess;
  }
  template< typename T >
  T *as() const { return static_cast< T * >( p ); }
};

struct object
{
  uint64_t n = 0;
  uint32_t V = 0;
  const double *verts = nullptr;  // in use (owned copy or borrowed device pointer)
  const uint64_t *gid = nullptr;
  bool has_data = false;
  bool built = false;  // slabs current for the present vertex data
  bool topo = false;   // a rebuild's topology exists for the present n and V (refit allowed)
  bool fresh = false;  // a rebuild ran since the last set_elements: bounds and centroids match the vertices
  int sort_result_alt = 0;  // sorted keys/vals ended in the *_alt buffers
  // Dense contact (a broadphase of this object found pairs for a sizable fraction of the elements): its next builds
  // store every element's slabs, which its traversals then only read; in sparse contact they compute the few they
  // test from the vertices instead of storing all of them.
  bool store_slabs = false;
  bool stored = false;  // the last build stored them
  // The batched dense walk reached its stack bound on this object's tree: its traversals use the single-node walk
  // until the element count changes.
  bool dense_ok = true;
  // Patches (bvhg_cluster): valid until the next set_elements or rebuild.
  bool clustered = false;
  uint32_t cl_patches = 0;
  dev_buf cl_order, cl_rank, cl_tmp, cl_runs, cl_bhist, cl_bbase, cl_splits, cl_bounds, cl_scal, cl_enc, cl_boxes;
  dev_buf verts_own, gid_own;
  dev_buf cx, cy, cz;
  dev_buf keys, keys_alt, vals, vals_alt;
  dev_buf hist, status, runs;
  dev_buf warp_box, bucket_box, node_box, child, range, parent, exch, bdel, queue, elem_cache;
  dev_buf scal;  // obj_scalars
  // Each object's build runs on its own stream, forked from and joined back into the context stream with
  // events, so two objects' builds overlap (one's latency-bound tree climb beside the other's streaming kernels).
  // The largest object builds on a high-priority stream: its chain is the longest, and the others' kernels fill
  // the SMs its latency-bound phases leave idle.
  cudaStream_t st = nullptr, st_hi = nullptr;
  cudaEvent_t done = nullptr;
  bool pending = false;
  ~object()
  {
    if ( st ) cudaStreamSynchronize( st );
    if ( st_hi ) cudaStreamSynchronize( st_hi );
    if ( done ) cudaEventDestroy( done );
    if ( st ) cudaStreamDestroy( st );
    if ( st_hi ) cudaStreamDestroy( st_hi );
  }
  obj_scalars *sc() const { return scal.as< obj_scalars >(); }
  const uint64_t *sorted_keys() const { return sort_result_alt ? keys_alt.as< uint64_t >() : keys.as< uint64_t >(); }
  const uint32_t *sorted_vals() const { return sort_result_alt ? vals_alt.as< uint32_t >() : vals.as< uint32_t >(); }
};

// Batching form: every object and scene of a batch as one CUDA graph (builds and traversals spread over lanes of
// concurrent streams, no host round trip between scenes), captured once per batch layout and replayed.
// Device tables (item arguments, block starts) of a fused batch graph's batched launches.
using launch_tables = std::vector< std::unique_ptr< dev_buf > >;

struct batch_graph
{
  std::vector< uint64_t > key;  // layout the graph was captured for
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::shared_ptr< launch_tables > tables;  // read by the graph's kernels (fused form)
};

struct batch_state
{
  // The last few captured layouts (a time-stepped loop alternates REBUILD and REFIT graphs of the same bodies).
  std::vector< batch_graph > graphs;
  std::vector< uint64_t > key;  // layout of the graph in use
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::shared_ptr< launch_tables > tables;
  // groups > 0: the fused form (one batched launch per pipeline stage for each of `groups` groups of objects, on
  // `lanes` streams); groups == 0: the laned form, per-object launches on `lanes` streams. bvhg_batch_autotune picks
  // both.
  int groups = 16;
  int lanes = 16;
  std::vector< cudaStream_t > lane;
  std::vector< cudaEvent_t > obj_done, lane_done;
  cudaEvent_t fork = nullptr;
  dev_buf cand, exact, out, ps, err_src, err_words;
  std::vector< uint64_t > cap, off;  // per scene: pair capacity and offset into cand / exact / out
  pair_scalars *host_ps = nullptr;
  int *host_err = nullptr;
  size_t host_scenes = 0, host_objs = 0;
  // Makes the cached graph of `k` current; false when none matches.
  bool select(const std::vector< uint64_t > &k)
  {
    for ( auto &g : graphs )
      if ( g.key == k )
      {
        key = g.key;
        graph = g.graph;
        exec = g.exec;
        tables = g.tables;
        return true;
      }
    return false;
  }
  // Caches the graph just captured (graph, exec, key), dropping the oldest beyond four.
  void keep()
  {
    if ( graphs.size() >= 4 )
    {
      cudaGraphExecDestroy( graphs.front().exec );
      cudaGraphDestroy( graphs.front().graph );
      graphs.erase( graphs.begin() );
    }
    graphs.push_back( { key, graph, exec, tables } );
  }
  void drop_graph()
  {
    for ( auto &g : graphs )
    {
      cudaGraphExecDestroy( g.exec );
      cudaGraphDestroy( g.graph );
    }
    graphs.clear();
    exec = nullptr;
    graph = nullptr;
    tables.reset();
    key.clear();
  }
  ~batch_state()
  {
    drop_graph();
    for ( auto st : lane ) cudaStreamDestroy( st );
    for ( auto e : obj_done ) cudaEventDestroy( e );
    for ( auto e : lane_done ) cudaEventDestroy( e );
    if ( fork ) cudaEventDestroy( fork );
    if ( host_ps ) cudaFreeHost( host_ps );
    if ( host_err ) cudaFreeHost( host_err );
  }
};

struct timed_stage
{
  int stage;
  cudaEvent_t start, stop;
};

}  // namespace

struct bvhg_ctx
{
  bvhg_config cfg{};
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  uint32_t spin_limit = kDefaultSpinLimit;
  int stall_sort = 0;  // test hook: radix look-back polls a status row nobody publishes
  int dense_stack = 0;  // test hook: lower stack bound of the batched dense walk (0 = its own)
  std::vector< std::unique_ptr< object > > objs;
  cudaEvent_t fork_evt = nullptr;
  std::string err;
  // sort-and-sweep scratch
  dev_buf sw_keys, sw_vals, sw_rows, sw_srows, sw_sbmax, sw_hist, sw_status, sw_sc, sw_params, sw_partial;
  // pairs
  dev_buf pairs, pairs2, pairs_out, pscal;
  // element pairs grouped by patch pair
  dev_buf grp_count, grp_off, grp_rows, grp_pairs, grp_scal;
  uint64_t pair_cap = 0, pair2_cap = 0;
  pair_scalars *host_ps = nullptr;  // pinned: pair counters + the two objects' error words after a broadphase
  int *host_err = nullptr;          // pinned [2]
  obj_scalars *init_template = nullptr;  // pinned, constant: the reset state of an object's scalars
  uint64_t last_candidates = 0;
  // timing
  std::vector< timed_stage > pending;
  std::vector< cudaEvent_t > event_pool;
  double stage_ms[BVHG_NUM_STAGES] = {};
  uint64_t stage_launches[BVHG_NUM_STAGES] = {};
  uint64_t launches = 0;
  std::unique_ptr< batch_state > batch;
};

namespace {

bvhg_status fail(bvhg_ctx *ctx, bvhg_status st, const std::string &msg)
{
  if ( ctx ) ctx->err = msg;
  return st;
}

bvhg_status cuda_fail(bvhg_ctx *ctx, cudaError_t e, const char *where)
{
  std::string m = std::string( where ) + ": " + cudaGetErrorString( e );
  return fail( ctx, e == cudaErrorMemoryAllocation ? BVHG_ERR_NOMEM : BVHG_ERR_CUDA, m );
}

#define BVHG_CUDA(ctx, call)                                                                                          \
  do                                                                                                                  \
  {                                                                                                                   \
    cudaError_t e_ = ( call );                                                                                        \
    if ( e_ != cudaSuccess ) return cuda_fail( ( ctx ), e_, #call );                                                  \
  } while ( 0 )

cudaEvent_t take_event(bvhg_ctx *ctx)
{
  if ( !ctx->event_pool.empty() )
  {
    cudaEvent_t e = ctx->event_pool.back();
    ctx->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate( &e );
  return e;
}

struct stage_scope
{
  bvhg_ctx *ctx;
  int stage;
  cudaEvent_t start = nullptr;
  stage_scope(bvhg_ctx *c, int s) : ctx( c ), stage( s )
  {
    if ( ctx->cfg.flags & BVHG_FLAG_STAGE_TIMING )
    {
      start = take_event( ctx );
      cudaEventRecord( start, ctx->stream );
    }
  }
  void launched(uint64_t k = 1)
  {
    ctx->launches += k;
    ctx->stage_launches[stage] += k;
  }
  ~stage_scope()
  {
    if ( start )
    {
      cudaEvent_t stop = take_event( ctx );
      cudaEventRecord( stop, ctx->stream );
      ctx->pending.push_back( { stage, start, stop } );
    }
  }
};

void collect_timing(bvhg_ctx *ctx)
{
  for ( auto &t : ctx->pending )
  {
    float ms = 0.f;
    if ( cudaEventSynchronize( t.stop ) == cudaSuccess && cudaEventElapsedTime( &ms, t.start, t.stop ) == cudaSuccess )
      ctx->stage_ms[t.stage] += ms;
    ctx->event_pool.push_back( t.start );
    ctx->event_pool.push_back( t.stop );
  }
  ctx->pending.clear();
}

// The stream an object's build runs on: its own, ordered after everything already on the context stream.
// With stage timing the context stream itself (stages then never overlap and their times are per kernel).
cudaError_t fork_object(bvhg_ctx *ctx, object &o, cudaStream_t *out)
{
  if ( ctx->cfg.flags & BVHG_FLAG_STAGE_TIMING )
  {
    *out = ctx->stream;
    return cudaSuccess;
  }
  bool largest = true;
  for ( const auto &p : ctx->objs )
    if ( p && p.get() != &o && p->n > o.n ) largest = false;
  cudaError_t e = cudaSuccess;
  cudaStream_t *sp = largest ? &o.st_hi : &o.st;
  if ( !*sp )
  {
    int least = 0, greatest = 0;
    e = cudaDeviceGetStreamPriorityRange( &least, &greatest );
    if ( e == cudaSuccess ) e = cudaStreamCreateWithPriority( sp, cudaStreamNonBlocking, largest ? greatest : least );
  }
  if ( e == cudaSuccess && !o.done ) e = cudaEventCreateWithFlags( &o.done, cudaEventDisableTiming );
  if ( e == cudaSuccess && !ctx->fork_evt ) e = cudaEventCreateWithFlags( &ctx->fork_evt, cudaEventDisableTiming );
  if ( e == cudaSuccess ) e = cudaEventRecord( ctx->fork_evt, ctx->stream );
  if ( e == cudaSuccess ) e = cudaStreamWaitEvent( *sp, ctx->fork_evt, 0 );
  *out = *sp;
  return e;
}

// Orders the context stream after the object's last build.
void join_object(bvhg_ctx *ctx, object &o)
{
  if ( o.pending )
  {
    cudaStreamWaitEvent( ctx->stream, o.done, 0 );
    o.pending = false;
  }
}

bool valid_obj(bvhg_ctx *ctx, int32_t obj)
{
  return ctx && obj >= 0 && static_cast< size_t >( obj ) < ctx->objs.size() && ctx->objs[obj];
}

size_t slab_bytes(const bvhg_ctx *ctx) { return ctx->cfg.precision == BVHG_FILTER_FP32 ? 4 : 8; }

bvhg_status object_error(bvhg_ctx *ctx, int err)
{
  if ( err == kErrArg ) return fail( ctx, BVHG_ERR_ARG, "non-finite vertex coordinate in element data" );
  if ( err == kErrTimeout ) return fail( ctx, BVHG_ERR_TIMEOUT, "radix sort look-back exceeded the spin limit" );
  if ( err ) return fail( ctx, BVHG_ERR_CUDA, "device error " + std::to_string( err ) );
  return BVHG_OK;
}

// Reads an object's device error word in stream order (synchronizes the stream).
bvhg_status check_scalar_errors(bvhg_ctx *ctx, const object &o)
{
  BVHG_CUDA( ctx, cudaMemcpyAsync( ctx->host_err, &o.sc()->error, sizeof( int ), cudaMemcpyDeviceToHost, ctx->stream ) );
  BVHG_CUDA( ctx, cudaStreamSynchronize( ctx->stream ) );
  return object_error( ctx, ctx->host_err[0] );
}

bvhg_status do_build_on(bvhg_ctx *ctx, object &o, int mode, cudaStream_t s);

// Device buffers of an object's rebuild for its present element count (no allocation when they suffice).
bvhg_status reserve_object(bvhg_ctx *ctx, object &o)
{
  const uint64_t n = o.n;
  const int D = ctx->cfg.k / 2;
  const size_t sb = slab_bytes( ctx );
  const int bits = ctx->cfg.sort_digit_bits;
  const int passes = sort_passes( bits );
  const uint64_t radix = 1ull << bits;
  const uint64_t tiles = ( n + kSortTile - 1 ) / kSortTile;
  BVHG_CUDA( ctx, o.scal.reserve( sizeof( obj_scalars ) ) );
  BVHG_CUDA( ctx, o.cx.reserve( n * 8 ) );
  BVHG_CUDA( ctx, o.cy.reserve( n * 8 ) );
  BVHG_CUDA( ctx, o.cz.reserve( n * 8 ) );
  BVHG_CUDA( ctx, o.keys.reserve( n * 8 ) );
  BVHG_CUDA( ctx, o.keys_alt.reserve( n * 8 ) );
  BVHG_CUDA( ctx, o.vals.reserve( n * 4 ) );
  BVHG_CUDA( ctx, o.vals_alt.reserve( n * 4 ) );
  BVHG_CUDA( ctx, o.hist.reserve( passes * radix * 4 ) );
  BVHG_CUDA( ctx, o.status.reserve( passes * ( tiles + 1 ) * radix * 4 ) );
  BVHG_CUDA( ctx, o.runs.reserve( long_run_capacity( n ) * 4 ) );
  const uint64_t m = ( n + kLeafSize - 1 ) / kLeafSize;  // leaf buckets
  BVHG_CUDA( ctx, o.warp_box.reserve( ( ( n + 31 ) / 32 ) * D * 2 * sb ) );
  BVHG_CUDA( ctx, o.bucket_box.reserve( m * D * 2 * sb ) );
  BVHG_CUDA( ctx, o.elem_cache.reserve( m * kLeafSize * D * 2 * sb ) );  // whole buckets (slab-major tiles)
  BVHG_CUDA( ctx, o.node_box.reserve( ( m - 1 ) * D * 4 * sb + 16 ) );
  BVHG_CUDA( ctx, o.child.reserve( ( m - 1 ) * 8 + 8 ) );
  BVHG_CUDA( ctx, o.range.reserve( ( m - 1 ) * 8 + 8 ) );
  BVHG_CUDA( ctx, o.parent.reserve( ( 2 * m ) * 4 ) );
  BVHG_CUDA( ctx, o.exch.reserve( m * 4 ) );
  BVHG_CUDA( ctx, o.bdel.reserve( m ) );
  BVHG_CUDA( ctx, o.queue.reserve( m * 16 ) );
  return BVHG_OK;
}


bvhg_status do_build(bvhg_ctx *ctx, object &o, int mode)
{
  const uint64_t n = o.n;
  const int K = ctx->cfg.k;
  const bool fp32 = ctx->cfg.precision == BVHG_FILTER_FP32;
  const int D = K / 2;
  if ( n == 0 )
  {
    o.built = true;
    o.fresh = true;
    return BVHG_OK;
  }
  cudaStream_t s = nullptr;
  BVHG_CUDA( ctx, fork_object( ctx, o, &s ) );
  if ( s != ctx->stream )
  {
    // recorded when this call returns, whatever path it takes
    struct recorder
    {
      object &o;
      cudaStream_t s;
      ~recorder()
      {
        cudaEventRecord( o.done, s );
        o.pending = true;
      }
    } rec{ o, s };
    return do_build_on( ctx, o, mode, s );
  }
  return do_build_on( ctx, o, mode, s );
}

bvhg_status do_build_on(bvhg_ctx *ctx, object &o, int mode, cudaStream_t s)
{
  const uint64_t n = o.n;
  const int K = ctx->cfg.k;
  const bool fp32 = ctx->cfg.precision == BVHG_FILTER_FP32;
  const int D = K / 2;
  const size_t sb = slab_bytes( ctx );
  if ( mode == BVHG_REFIT )
  {
    if ( !o.topo ) return fail( ctx, BVHG_ERR_STATE, "refit without a rebuild of this element count" );
    const uint64_t m = ( n + kLeafSize - 1 ) / kLeafSize;
    {
      stage_scope st( ctx, BVHG_STAGE_SLABS );
      BVHG_CUDA( ctx, launch_slabs( K, fp32, o.verts, o.V, n, ctx->cfg.epsilon, o.sorted_vals(),
                                    o.bucket_box.p, o.warp_box.p, o.store_slabs ? o.elem_cache.p : nullptr,
                                    o.sc(), s ) );
      o.stored = o.store_slabs;
      st.launched();
    }
    if ( m > 1 )
    {
      stage_scope st( ctx, BVHG_STAGE_BUILD );
      BVHG_CUDA( ctx, cudaMemsetAsync( o.exch.p, 0xff, ( m - 1 ) * sizeof( int ), s ) );
      BVHG_CUDA( ctx, launch_refit( K, fp32, n, o.bucket_box.p, o.node_box.p, o.child.as< int2 >(), o.range.as< int2 >(),
                                    o.parent.as< int >(), o.exch.as< int >(), o.sc(), s ) );
      st.launched();
    }
    o.built = true;
    o.fresh = false;  // a refit keeps the last rebuild's bounds and centroids
    return BVHG_OK;
  }
  const int bits = ctx->cfg.sort_digit_bits;
  const int passes = sort_passes( bits );
  const uint64_t radix = 1ull << bits;
  const uint64_t tiles = ( n + kSortTile - 1 ) / kSortTile;
  const uint64_t m = ( n + kLeafSize - 1 ) / kLeafSize;  // leaf buckets
  {
    const bvhg_status rs = reserve_object( ctx, o );
    if ( rs != BVHG_OK ) return rs;
  }
  o.clustered = false;  // a rebuild recomputes the keys and their order
  {
    stage_scope st( ctx, BVHG_STAGE_BOUNDS );
    {
      // one launch resets the scalars, histograms, the look-back words of the passes that run and the exchange
      const size_t first_words = static_cast< size_t >( sort_first_pass( bits ) ) * ( tiles + 1 ) * radix;
      BVHG_CUDA( ctx, launch_obj_init( o.sc(), o.hist.as< uint32_t >(), passes * radix,
                                       o.status.as< uint32_t >() + first_words,
                                       passes * ( tiles + 1 ) * radix - first_words, o.exch.as< int >(),
                                       m > 1 ? m - 1 : 0, s ) );
      st.launched();
    }
    BVHG_CUDA( ctx, launch_centroid_bounds( K, o.verts, o.V, n, ctx->cfg.epsilon, o.cx.as< double >(),
                                            o.cy.as< double >(), o.cz.as< double >(), o.sc(), ctx->spin_limit, s ) );
    st.launched();
  }
  {
    stage_scope st( ctx, BVHG_STAGE_KEYS );
    BVHG_CUDA( ctx, launch_keys_hist( bits, o.cx.as< double >(), o.cy.as< double >(), o.cz.as< double >(), n, o.sc(),
                                      o.keys.as< uint64_t >(), o.hist.as< uint32_t >(), s ) );
    st.launched();
  }
  uint64_t *kin = o.keys.as< uint64_t >(), *kout = o.keys_alt.as< uint64_t >();
  uint32_t *vin = nullptr, *vout = o.vals_alt.as< uint32_t >();
  {
    stage_scope st( ctx, BVHG_STAGE_SORT );
    // Radix passes over the high key half only; the fix-up then sorts each run of equal high halves by the low
    // half (runs are a handful of elements for meshes: 2^31 cells of the Morton grid).
    uint32_t *vother = o.vals.as< uint32_t >();
    const int first = sort_first_pass( bits );
    for ( int p = first; p < passes; ++p )
    {
      BVHG_CUDA( ctx, launch_onesweep( bits, kin, vin, kout, vout, n, p, o.hist.as< uint32_t >(),
                                       o.status.as< uint32_t >(), o.sc(), ctx->spin_limit, ctx->stall_sort, s ) );
      st.launched();
      std::swap( kin, kout );
      uint32_t *next_out = vin ? vin : vother;
      vin = vout;
      vout = next_out;
    }
  }
  {
    // the fix-up reads the last pass's output and writes the other buffers
    stage_scope st( ctx, BVHG_STAGE_FIXUP );
    BVHG_CUDA( ctx, launch_sort_fixup( kin, vin, kout, vout, n, o.runs.as< uint32_t >(), o.sc(), s ) );
    st.launched();
    if ( sort_runs_blocks( n ) ) st.launched();
    o.sort_result_alt = ( kout == o.keys_alt.as< uint64_t >() ) ? 1 : 0;
  }
  {
    stage_scope st( ctx, BVHG_STAGE_SLABS );
    BVHG_CUDA( ctx, launch_slabs( K, fp32, o.verts, o.V, n, ctx->cfg.epsilon, o.sorted_vals(),
                                  o.bucket_box.p, o.warp_box.p, o.store_slabs ? o.elem_cache.p : nullptr,
                                  o.sc(), s ) );
    o.stored = o.store_slabs;
    st.launched();
  }
  if ( m > 1 )
  {
    stage_scope st( ctx, BVHG_STAGE_BUILD );
    BVHG_CUDA( ctx, launch_build( K, fp32, n, o.sorted_keys(), o.bdel.as< uint8_t >(), o.bucket_box.p, o.node_box.p,
                                  o.child.as< int2 >(), o.range.as< int2 >(), o.parent.as< int >(),
                                  o.queue.as< int4 >(), o.sc(), s ) );
    st.launched();
  }
  if ( m > 1 )
  {
    stage_scope st( ctx, BVHG_STAGE_CLIMB );
    BVHG_CUDA( ctx, launch_climb( K, fp32, n, o.bdel.as< uint8_t >(), o.node_box.p, o.child.as< int2 >(),
                                  o.range.as< int2 >(), o.parent.as< int >(), o.exch.as< int >(),
                                  o.queue.as< int4 >(), o.sc(), s ) );
    st.launched();
  }
  o.built = true;
  o.topo = true;
  o.fresh = true;
  return BVHG_OK;
}

tree_view view_of(const object &o)
{
  tree_view v;
  v.node_box = o.node_box.p;
  v.child = o.child.as< int2 >();
  v.range = o.range.as< int2 >();
  v.warp_box = o.warp_box.p;
  v.verts = o.verts;
  v.V = o.V;
  v.elem_cache = o.elem_cache.p;
  v.stored = o.stored;
  v.perm = o.sorted_vals();
  v.n = o.n;
  v.sc = o.sc();
  return v;
}

// Runs traversal (+ recheck) until both buffers were large enough; returns the final local pair buffer and count.
// One host synchronization per attempt: the pair counters and both objects' error words come back together.
bvhg_status find_pairs(bvhg_ctx *ctx, object &a, object &b, bool self, const uint2 **out_pairs, uint64_t *out_count)
{
  const int K = ctx->cfg.k;
  const bool fp32 = ctx->cfg.precision == BVHG_FILTER_FP32;
  cudaStream_t s = ctx->stream;
  BVHG_CUDA( ctx, ctx->pscal.reserve( sizeof( pair_scalars ) ) );
  if ( ctx->pair_cap == 0 )
  {
    ctx->pair_cap = 1u << 20;
    BVHG_CUDA( ctx, ctx->pairs.reserve( ctx->pair_cap * sizeof( uint2 ) ) );
  }
  if ( fp32 && ctx->pair2_cap == 0 )
  {
    ctx->pair2_cap = 1u << 20;
    BVHG_CUDA( ctx, ctx->pairs2.reserve( ctx->pair2_cap * sizeof( uint2 ) ) );
  }
  pair_scalars *ps = ctx->pscal.as< pair_scalars >();
  for ( int attempt = 0; attempt < 4; ++attempt )
  {
    BVHG_CUDA( ctx, cudaMemsetAsync( ps, 0, sizeof( pair_scalars ), s ) );
    const bool dense = a.dense_ok && b.dense_ok;
    {
      stage_scope st( ctx, BVHG_STAGE_TRAVERSE );
      BVHG_CUDA( ctx, launch_traverse( K, fp32, view_of( a ), view_of( b ), self, dense, ctx->cfg.epsilon,
                                       ctx->pairs.as< uint2 >(), ctx->pair_cap, ps, s, ctx->dense_stack ) );
      st.launched();
    }
    if ( fp32 )
    {
      stage_scope st( ctx, BVHG_STAGE_RECHECK );
      BVHG_CUDA( ctx, launch_recheck( K, a.verts, a.V, b.verts, b.V, ctx->cfg.epsilon, ctx->pairs.as< uint2 >(),
                                      ctx->pair_cap, ctx->pairs2.as< uint2 >(), ctx->pair2_cap, ps, s ) );
      st.launched();
    }
    BVHG_CUDA( ctx, cudaMemcpyAsync( ctx->host_ps, ps, sizeof( pair_scalars ), cudaMemcpyDeviceToHost, s ) );
    BVHG_CUDA( ctx, cudaMemcpyAsync( ctx->host_err, &a.sc()->error, sizeof( int ), cudaMemcpyDeviceToHost, s ) );
    BVHG_CUDA( ctx, cudaMemcpyAsync( ctx->host_err + 1, &b.sc()->error, sizeof( int ), cudaMemcpyDeviceToHost, s ) );
    BVHG_CUDA( ctx, cudaStreamSynchronize( s ) );
    bvhg_status st = object_error( ctx, ctx->host_err[0] );
    if ( st == BVHG_OK ) st = object_error( ctx, ctx->host_err[1] );
    if ( st != BVHG_OK ) return st;
    if ( ctx->host_ps->error == kErrOverflowStack && dense && a.stored && b.stored )
    {
      // the batched dense walk reached its stack bound: search again with the single-node walk
      a.dense_ok = false;
      b.dense_ok = false;
      continue;
    }
    if ( ctx->host_ps->error ) return fail( ctx, BVHG_ERR_CUDA, "traversal stack overflow" );
    const uint64_t ncand = ctx->host_ps->count;
    ctx->last_candidates = ncand;
    if ( ncand > ctx->pair_cap )
    {
      ctx->pair_cap = ncand + ncand / 8;
      BVHG_CUDA( ctx, ctx->pairs.reserve( ctx->pair_cap * sizeof( uint2 ) ) );
      continue;
    }
    if ( !fp32 )
    {
      *out_pairs = ctx->pairs.as< uint2 >();
      *out_count = ncand;
      return BVHG_OK;
    }
    const uint64_t nexact = ctx->host_ps->count2;
    if ( nexact > ctx->pair2_cap )
    {
      ctx->pair2_cap = nexact + nexact / 8;
      BVHG_CUDA( ctx, ctx->pairs2.reserve( ctx->pair2_cap * sizeof( uint2 ) ) );
      continue;
    }
    *out_pairs = ctx->pairs2.as< uint2 >();
    *out_count = nexact;
    return BVHG_OK;
  }
  return fail( ctx, BVHG_ERR_CUDA, "pair buffer did not converge" );
}

// Contact density decides whether the objects' next builds store their element slabs (see object::store_slabs):
// candidate pairs for at least 2% of the elements involved.
void note_density(object &a, object &b, bool self, uint64_t candidates)
{
  const uint64_t elems = self ? a.n : a.n + b.n;
  const bool dense = candidates * 50 >= elems && candidates > 0;
  a.store_slabs = dense;
  b.store_slabs = dense;
}

bvhg_status emit_pairs(bvhg_ctx *ctx, const object &a, const object &b, bool self, const uint2 *pairs, uint64_t np,
                       uint64_t *out, uint64_t capacity, uint64_t *count, int32_t mem)
{
  cudaStream_t s = ctx->stream;
  *count = np;
  const uint64_t nw = np < capacity ? np : capacity;
  if ( nw > 0 && out )
  {
    stage_scope st( ctx, BVHG_STAGE_OUTPUT );
    uint64_t *dst = out;
    if ( mem == BVHG_MEM_HOST )
    {
      BVHG_CUDA( ctx, ctx->pairs_out.reserve( nw * 16 ) );
      dst = ctx->pairs_out.as< uint64_t >();
    }
    BVHG_CUDA( ctx, launch_gid_pairs( pairs, nw, a.gid, b.gid, self, dst, s ) );
    st.launched();
    if ( mem == BVHG_MEM_HOST )
      BVHG_CUDA( ctx, cudaMemcpyAsync( out, dst, nw * 16, cudaMemcpyDeviceToHost, s ) );
  }
  BVHG_CUDA( ctx, cudaStreamSynchronize( s ) );
  if ( np > capacity ) return fail( ctx, BVHG_ERR_OVERFLOW, "pair buffer too small: " + std::to_string( np ) + " pairs" );
  return BVHG_OK;
}


// ---- batching form ---------------------------------------------------------------------------------------------

struct batch_args
{
  uint32_t nscenes;
  const int32_t *a, *b;
  int mode;
};

// Captures the graph of one batch: all unique objects' builds, then every scene's traversal (+ recheck) and gid
// mapping into its own slot of the batch buffers, then the gather of the objects' error words.
bvhg_status capture_batch(bvhg_ctx *ctx, batch_state &B, const batch_args &x, const std::vector< int32_t > &uniq,
                          const std::vector< int > &slot)
{
  const int K = ctx->cfg.k;
  const bool fp32 = ctx->cfg.precision == BVHG_FILTER_FP32;
  const int L = B.lanes;
  while ( static_cast< int >( B.lane.size() ) < L )
  {
    cudaStream_t st = nullptr;
    BVHG_CUDA( ctx, cudaStreamCreateWithFlags( &st, cudaStreamNonBlocking ) );
    B.lane.push_back( st );
    cudaEvent_t e = nullptr;
    BVHG_CUDA( ctx, cudaEventCreateWithFlags( &e, cudaEventDisableTiming ) );
    B.lane_done.push_back( e );
  }
  while ( B.obj_done.size() < uniq.size() )
  {
    cudaEvent_t e = nullptr;
    BVHG_CUDA( ctx, cudaEventCreateWithFlags( &e, cudaEventDisableTiming ) );
    B.obj_done.push_back( e );
  }
  if ( !B.fork ) BVHG_CUDA( ctx, cudaEventCreateWithFlags( &B.fork, cudaEventDisableTiming ) );
  B.graph = nullptr;
  B.exec = nullptr;
  const uint32_t flags = ctx->cfg.flags;
  ctx->cfg.flags &= ~BVHG_FLAG_STAGE_TIMING;  // no timing events inside a graph
  cudaStream_t s = ctx->stream;
  BVHG_CUDA( ctx, cudaStreamBeginCapture( s, cudaStreamCaptureModeRelaxed ) );
  auto body = [&]() -> bvhg_status {
    pair_scalars *ps = B.ps.as< pair_scalars >();
    BVHG_CUDA( ctx, cudaMemsetAsync( ps, 0, x.nscenes * sizeof( pair_scalars ), s ) );
    BVHG_CUDA( ctx, cudaEventRecord( B.fork, s ) );
    for ( int l = 0; l < L; ++l ) BVHG_CUDA( ctx, cudaStreamWaitEvent( B.lane[l], B.fork, 0 ) );
    for ( size_t i = 0; i < uniq.size(); ++i )
    {
      object &o = *ctx->objs[uniq[i]];
      cudaStream_t ls = B.lane[i % L];
      if ( o.n > 0 )
      {
        const bvhg_status st = do_build_on( ctx, o, x.mode, ls );
        if ( st != BVHG_OK ) return st;
      } else {
        o.built = true;
      }
      BVHG_CUDA( ctx, cudaEventRecord( B.obj_done[i], ls ) );
    }
    for ( uint32_t sc = 0; sc < x.nscenes; ++sc )
    {
      cudaStream_t ls = B.lane[sc % L];
      object &oa = *ctx->objs[x.a[sc]];
      object &ob = *ctx->objs[x.b[sc]];
      BVHG_CUDA( ctx, cudaStreamWaitEvent( ls, B.obj_done[slot[x.a[sc]]], 0 ) );
      BVHG_CUDA( ctx, cudaStreamWaitEvent( ls, B.obj_done[slot[x.b[sc]]], 0 ) );
      const bool self = x.a[sc] == x.b[sc];
      if ( oa.n == 0 || ob.n == 0 || ( self && oa.n < 2 ) ) continue;
      uint2 *cand = B.cand.as< uint2 >() + B.off[sc];
      BVHG_CUDA( ctx, launch_traverse( K, fp32, view_of( oa ), view_of( ob ), self, oa.dense_ok && ob.dense_ok,
                                       ctx->cfg.epsilon, cand, B.cap[sc], ps + sc, ls, ctx->dense_stack ) );
      const uint2 *fin = cand;
      const unsigned long long *cnt = &ps[sc].count;
      if ( fp32 )
      {
        uint2 *ex = B.exact.as< uint2 >() + B.off[sc];
        BVHG_CUDA( ctx, launch_recheck( K, oa.verts, oa.V, ob.verts, ob.V, ctx->cfg.epsilon, cand, B.cap[sc], ex,
                                        B.cap[sc], ps + sc, ls ) );
        fin = ex;
        cnt = &ps[sc].count2;
      }
      BVHG_CUDA( ctx, launch_gid_pairs_dev( fin, cnt, B.cap[sc], oa.gid, ob.gid, self,
                                            B.out.as< uint64_t >() + 2 * B.off[sc], ls ) );
      ctx->launches += fp32 ? 3 : 2;
    }
    for ( int l = 0; l < L; ++l )
    {
      BVHG_CUDA( ctx, cudaEventRecord( B.lane_done[l], B.lane[l] ) );
      BVHG_CUDA( ctx, cudaStreamWaitEvent( s, B.lane_done[l], 0 ) );
    }
    BVHG_CUDA( ctx, launch_gather_words( B.err_src.as< const int *const >(), static_cast< int >( uniq.size() ),
                                         B.err_words.as< int >(), s ) );
    return BVHG_OK;
  };
  const bvhg_status st = body();
  ctx->cfg.flags = flags;
  cudaGraph_t g = nullptr;
  const cudaError_t ce = cudaStreamEndCapture( s, &g );
  if ( st != BVHG_OK )
  {
    if ( g ) cudaGraphDestroy( g );
    return st;
  }
  if ( ce != cudaSuccess ) return cuda_fail( ctx, ce, "cudaStreamEndCapture" );
  B.graph = g;
  BVHG_CUDA( ctx, cudaGraphInstantiate( &B.exec, B.graph, 0 ) );
  return BVHG_OK;
}

// One batched launch's tables on the device (before capture: a synchronous upload).
template< typename A >
bvhg_status make_launch(bvhg_ctx *ctx, launch_tables &keep, const std::vector< A > &items,
                        const std::vector< uint32_t > &blocks, batch_launch *out)
{
  *out = batch_launch{};
  if ( items.empty() ) return BVHG_OK;
  std::vector< uint32_t > starts( items.size() + 1, 0 );
  for ( size_t i = 0; i < items.size(); ++i ) starts[i + 1] = starts[i] + blocks[i];
  keep.emplace_back( new dev_buf );
  dev_buf &bi = *keep.back();
  BVHG_CUDA( ctx, bi.reserve( items.size() * sizeof( A ) ) );
  BVHG_CUDA( ctx, cudaMemcpy( bi.p, items.data(), items.size() * sizeof( A ), cudaMemcpyHostToDevice ) );
  keep.emplace_back( new dev_buf );
  dev_buf &bs = *keep.back();
  BVHG_CUDA( ctx, bs.reserve( starts.size() * sizeof( uint32_t ) ) );
  BVHG_CUDA( ctx, cudaMemcpy( bs.p, starts.data(), starts.size() * sizeof( uint32_t ), cudaMemcpyHostToDevice ) );
  out->items = bi.p;
  out->starts = bs.as< uint32_t >();
  out->nitems = static_cast< int >( items.size() );
  out->blocks = starts.back();
  return BVHG_OK;
}

// The vertex count shared by every non-empty object of the batch, or 0 when they differ (the laned form then runs).
uint32_t batch_vertex_count(bvhg_ctx *ctx, const std::vector< int32_t > &uniq)
{
  uint32_t V = 0;
  for ( int32_t o : uniq )
  {
    const object &ob = *ctx->objs[o];
    if ( ob.n == 0 ) continue;
    if ( V == 0 ) V = ob.V;
    else if ( V != ob.V ) return 0;
  }
  return V ? V : 3;
}

// The batched launches of one group of a fused batch: its objects' pipeline stages and its scenes' traversal,
// recheck and gid mapping (items and blocks per launch; uploaded by make_launch before capture).
struct fused_group
{
  std::vector< init_args > init;
  std::vector< cb_args > cb;
  std::vector< kh_args > kh;
  std::vector< std::vector< sort_pass_args > > pass;
  std::vector< fixup_args > fix, runs;
  std::vector< slabs_args > slabs;
  std::vector< tree_args > tree;  // objects with more than one bucket (build + climb, or refit)
  std::vector< uint32_t > b_init, b_cb, b_kh, b_fix, b_runs, b_slabs, b_build, b_climb, b_refit;
  std::vector< std::vector< uint32_t > > b_pass;
  std::vector< trav_item > dense, sparse;
  std::vector< recheck_args > recheck;
  std::vector< gid_args > gid;
  std::vector< uint32_t > b_dense, b_sparse, b_recheck, b_gid;
  std::vector< int > needs;  // other groups whose objects this group's scenes read
  batch_launch l_init, l_cb, l_kh, l_fix, l_runs, l_slabs, l_build, l_climb, l_refit, l_dense, l_sparse, l_recheck, l_gid;
  std::vector< batch_launch > l_pass;
};

// Fused form of a batch: the objects are split into `groups` groups of about equal element counts (in first-use
// order, so a scene's two objects mostly share a group); each group runs every pipeline stage of its objects as one
// batched launch per stage (batch.cuh), then the traversal, recheck and gid mapping of the scenes whose later object
// is in the group, on one of `lanes` streams. Groups small enough for their objects' working sets to stay in L2
// between stages run faster than one group over the whole batch; the autotuner picks the group count. The
// per-object computation, its buffers and its host-side state are those of do_build_on; only the launches change.
bvhg_status capture_batch_fused(bvhg_ctx *ctx, batch_state &B, const batch_args &x, const std::vector< int32_t > &uniq,
                                uint32_t V, int groups, int lanes)
{
  const int K = ctx->cfg.k;
  const bool fp32 = ctx->cfg.precision == BVHG_FILTER_FP32;
  const int bits = ctx->cfg.sort_digit_bits;
  const int passes = sort_passes( bits );
  const int first = sort_first_pass( bits );
  const uint64_t radix = 1ull << bits;
  const double eps = ctx->cfg.epsilon;
  auto tables = std::make_shared< launch_tables >();
  // objects to groups by cumulative element count
  uint64_t total = 0;
  for ( int32_t oi : uniq ) total += ctx->objs[oi]->n;
  const int G = std::max( 1, std::min< int >( groups, static_cast< int >( uniq.size() ) ) );
  std::vector< int > group_of( ctx->objs.size(), 0 );
  {
    uint64_t acc = 0;
    for ( int32_t oi : uniq )
    {
      const int g = total ? static_cast< int >( std::min< uint64_t >( G - 1, ( acc * G ) / total ) ) : 0;
      group_of[oi] = g;
      acc += ctx->objs[oi]->n;
    }
  }
  std::vector< fused_group > grp( G );
  for ( auto &fg : grp )
  {
    fg.pass.resize( passes );
    fg.b_pass.resize( passes );
    fg.l_pass.resize( passes );
  }
  bool tma = V == 3 || V == 4 || V == 8;
  for ( int32_t oi : uniq )
    if ( ctx->objs[oi]->n && ( reinterpret_cast< uintptr_t >( ctx->objs[oi]->verts ) & 15 ) ) tma = false;
  for ( int32_t oi : uniq )
  {
    object &o = *ctx->objs[oi];
    fused_group &fg = grp[group_of[oi]];
    if ( o.n == 0 )
    {
      o.built = true;
      o.fresh = x.mode == BVHG_REBUILD;
      continue;
    }
    const uint64_t n = o.n;
    const uint64_t m = ( n + kLeafSize - 1 ) / kLeafSize;
    const uint64_t tiles = ( n + kSortTile - 1 ) / kSortTile;
    if ( x.mode == BVHG_REBUILD )
    {
      const size_t first_words = static_cast< size_t >( first ) * ( tiles + 1 ) * radix;
      const init_args ia{ o.sc(), o.hist.as< uint32_t >(), passes * radix, o.status.as< uint32_t >() + first_words,
                          passes * ( tiles + 1 ) * radix - first_words, o.exch.as< int >(), m > 1 ? m - 1 : 0 };
      fg.init.push_back( ia );
      fg.b_init.push_back( obj_init_blocks( ia ) );
      fg.cb.push_back( cb_args{ o.verts, o.V, n, eps, o.cx.as< double >(), o.cy.as< double >(), o.cz.as< double >(),
                                o.sc(), ctx->spin_limit } );
      uint32_t cbb = 0;
      BVHG_CUDA( ctx, centroid_bounds_blocks( K, V, n, tma, &cbb ) );
      fg.b_cb.push_back( cbb );
      fg.kh.push_back( kh_args{ o.cx.as< double >(), o.cy.as< double >(), o.cz.as< double >(), n, o.sc(),
                                o.keys.as< uint64_t >(), o.hist.as< uint32_t >() } );
      fg.b_kh.push_back( keys_hist_blocks( n ) );
      uint64_t *kin = o.keys.as< uint64_t >(), *kout = o.keys_alt.as< uint64_t >();
      uint32_t *vin = nullptr, *vout = o.vals_alt.as< uint32_t >();
      uint32_t *vother = o.vals.as< uint32_t >();
      for ( int p = first; p < passes; ++p )
      {
        fg.pass[p].push_back( onesweep_args( bits, kin, vin, kout, vout, n, p, o.hist.as< uint32_t >(),
                                             o.status.as< uint32_t >(), o.sc(), ctx->spin_limit, ctx->stall_sort ) );
        fg.b_pass[p].push_back( onesweep_blocks( n ) );
        std::swap( kin, kout );
        uint32_t *next_out = vin ? vin : vother;
        vin = vout;
        vout = next_out;
      }
      const fixup_args fa{ kin, vin, kout, vout, n, o.runs.as< uint32_t >(), o.sc() };
      fg.fix.push_back( fa );
      fg.b_fix.push_back( sort_fixup_blocks( n ) );
      if ( const uint32_t rb = sort_runs_blocks( n ) )
      {
        fg.runs.push_back( fa );
        fg.b_runs.push_back( rb );
      }
      o.sort_result_alt = ( kout == o.keys_alt.as< uint64_t >() ) ? 1 : 0;
    } else if ( m > 1 ) {
      // refit: only the exchange slots start over
      const init_args ia{ nullptr, nullptr, 0, nullptr, 0, o.exch.as< int >(), m - 1 };
      fg.init.push_back( ia );
      fg.b_init.push_back( obj_init_blocks( ia ) );
    }
    fg.slabs.push_back( slabs_args{ o.verts, o.V, n, eps, f32_round_up( eps ), o.sorted_vals(), o.bucket_box.p,
                                    o.warp_box.p, o.store_slabs ? o.elem_cache.p : nullptr, o.sc() } );
    fg.b_slabs.push_back( slabs_blocks( n ) );
    o.stored = o.store_slabs;
    if ( m > 1 )
    {
      fg.tree.push_back( tree_args{ n, o.sorted_keys(), o.bdel.as< uint8_t >(), o.bucket_box.p, o.node_box.p,
                                    o.child.as< int2 >(), o.range.as< int2 >(), o.parent.as< int >(), o.exch.as< int >(),
                                    o.queue.as< int4 >(), o.sc() } );
      fg.b_build.push_back( build_blocks( n ) );
      fg.b_climb.push_back( climb_blocks( n ) );
      fg.b_refit.push_back( refit_blocks( n ) );
    }
    o.built = true;
    if ( x.mode == BVHG_REBUILD )
    {
      o.topo = true;
      o.fresh = true;
      o.clustered = false;
    } else {
      o.fresh = false;
    }
  }
  // scenes (after the objects' host state above: the views read which buffers hold the sorted order and slabs), in
  // the group of their later object
  pair_scalars *ps = B.ps.as< pair_scalars >();
  for ( uint32_t sc = 0; sc < x.nscenes; ++sc )
  {
    object &oa = *ctx->objs[x.a[sc]];
    object &ob = *ctx->objs[x.b[sc]];
    const bool self = x.a[sc] == x.b[sc];
    if ( oa.n == 0 || ob.n == 0 || ( self && oa.n < 2 ) ) continue;
    const int ga = group_of[x.a[sc]], gb = group_of[x.b[sc]];
    fused_group &fg = grp[std::max( ga, gb )];
    const int other = std::min( ga, gb );
    if ( other != std::max( ga, gb ) && std::find( fg.needs.begin(), fg.needs.end(), other ) == fg.needs.end() )
      fg.needs.push_back( other );
    uint2 *cand = B.cand.as< uint2 >() + B.off[sc];
    trav_item ti;
    uint32_t tb = 0;
    bool dense = false;
    traverse_item( K, fp32, view_of( oa ), view_of( ob ), self, oa.dense_ok && ob.dense_ok, eps, cand, B.cap[sc],
                   ps + sc, ctx->dense_stack, &ti, &tb, &dense );
    ( dense ? fg.dense : fg.sparse ).push_back( ti );
    ( dense ? fg.b_dense : fg.b_sparse ).push_back( tb );
    const uint2 *fin = cand;
    const unsigned long long *cnt = &ps[sc].count;
    if ( fp32 )
    {
      uint2 *ex = B.exact.as< uint2 >() + B.off[sc];
      fg.recheck.push_back( recheck_args{ oa.verts, oa.V, ob.verts, ob.V, eps, cand, B.cap[sc], ex, B.cap[sc], ps + sc } );
      fg.b_recheck.push_back( recheck_blocks( B.cap[sc] ) );
      fin = ex;
      cnt = &ps[sc].count2;
    }
    fg.gid.push_back( gid_args{ fin, cnt, B.cap[sc], oa.gid, ob.gid, self ? 1 : 0, B.out.as< uint64_t >() + 2 * B.off[sc] } );
    fg.b_gid.push_back( gid_pairs_dev_blocks( B.cap[sc] ) );
  }
  // the tables on the device
  for ( auto &fg : grp )
  {
    bvhg_status st = make_launch( ctx, *tables, fg.init, fg.b_init, &fg.l_init );
    if ( st == BVHG_OK && x.mode == BVHG_REBUILD )
    {
      if ( st == BVHG_OK ) st = make_launch( ctx, *tables, fg.cb, fg.b_cb, &fg.l_cb );
      if ( st == BVHG_OK ) st = make_launch( ctx, *tables, fg.kh, fg.b_kh, &fg.l_kh );
      for ( int p = first; p < passes && st == BVHG_OK; ++p )
        st = make_launch( ctx, *tables, fg.pass[p], fg.b_pass[p], &fg.l_pass[p] );
      if ( st == BVHG_OK ) st = make_launch( ctx, *tables, fg.fix, fg.b_fix, &fg.l_fix );
      if ( st == BVHG_OK ) st = make_launch( ctx, *tables, fg.runs, fg.b_runs, &fg.l_runs );
      if ( st == BVHG_OK ) st = make_launch( ctx, *tables, fg.tree, fg.b_build, &fg.l_build );
      if ( st == BVHG_OK ) st = make_launch( ctx, *tables, fg.tree, fg.b_climb, &fg.l_climb );
    } else if ( st == BVHG_OK ) {
      st = make_launch( ctx, *tables, fg.tree, fg.b_refit, &fg.l_refit );
    }
    if ( st == BVHG_OK ) st = make_launch( ctx, *tables, fg.slabs, fg.b_slabs, &fg.l_slabs );
    if ( st == BVHG_OK ) st = make_launch( ctx, *tables, fg.dense, fg.b_dense, &fg.l_dense );
    if ( st == BVHG_OK ) st = make_launch( ctx, *tables, fg.sparse, fg.b_sparse, &fg.l_sparse );
    if ( st == BVHG_OK ) st = make_launch( ctx, *tables, fg.recheck, fg.b_recheck, &fg.l_recheck );
    if ( st == BVHG_OK ) st = make_launch( ctx, *tables, fg.gid, fg.b_gid, &fg.l_gid );
    if ( st != BVHG_OK ) return st;
  }
  // streams and events
  const int L = std::max( 1, std::min( lanes, G ) );
  while ( static_cast< int >( B.lane.size() ) < L )
  {
    cudaStream_t st = nullptr;
    BVHG_CUDA( ctx, cudaStreamCreateWithFlags( &st, cudaStreamNonBlocking ) );
    B.lane.push_back( st );
    cudaEvent_t e = nullptr;
    BVHG_CUDA( ctx, cudaEventCreateWithFlags( &e, cudaEventDisableTiming ) );
    B.lane_done.push_back( e );
  }
  while ( B.obj_done.size() < static_cast< size_t >( G ) )
  {
    cudaEvent_t e = nullptr;
    BVHG_CUDA( ctx, cudaEventCreateWithFlags( &e, cudaEventDisableTiming ) );
    B.obj_done.push_back( e );
  }
  if ( !B.fork ) BVHG_CUDA( ctx, cudaEventCreateWithFlags( &B.fork, cudaEventDisableTiming ) );
  B.graph = nullptr;
  B.exec = nullptr;
  cudaStream_t s = ctx->stream;
  BVHG_CUDA( ctx, cudaStreamBeginCapture( s, cudaStreamCaptureModeRelaxed ) );
  auto body = [&]() -> bvhg_status {
    BVHG_CUDA( ctx, cudaMemsetAsync( ps, 0, x.nscenes * sizeof( pair_scalars ), s ) );
    BVHG_CUDA( ctx, cudaEventRecord( B.fork, s ) );
    for ( int l = 0; l < L; ++l ) BVHG_CUDA( ctx, cudaStreamWaitEvent( B.lane[l], B.fork, 0 ) );
    // builds, group by group on its lane
    for ( int g = 0; g < G; ++g )
    {
      fused_group &fg = grp[g];
      cudaStream_t ls = B.lane[g % L];
      BVHG_CUDA( ctx, launch_obj_init_batch( fg.l_init, ls ) );
      if ( x.mode == BVHG_REBUILD )
      {
        BVHG_CUDA( ctx, launch_centroid_bounds_batch( K, V, tma, fg.l_cb, ls ) );
        BVHG_CUDA( ctx, launch_keys_hist_batch( bits, fg.l_kh, ls ) );
        for ( int p = first; p < passes; ++p ) BVHG_CUDA( ctx, launch_onesweep_batch( bits, fg.l_pass[p], ls ) );
        BVHG_CUDA( ctx, launch_sort_fixup_batch( fg.l_fix, ls ) );
        BVHG_CUDA( ctx, launch_sort_runs_batch( fg.l_runs, ls ) );
        BVHG_CUDA( ctx, launch_slabs_batch( K, fp32, V, fg.l_slabs, ls ) );
        BVHG_CUDA( ctx, launch_build_batch( K, fp32, fg.l_build, ls ) );
        BVHG_CUDA( ctx, launch_climb_batch( K, fp32, fg.l_climb, ls ) );
      } else {
        BVHG_CUDA( ctx, launch_slabs_batch( K, fp32, V, fg.l_slabs, ls ) );
        BVHG_CUDA( ctx, launch_refit_batch( K, fp32, fg.l_refit, ls ) );
      }
      BVHG_CUDA( ctx, cudaEventRecord( B.obj_done[g], ls ) );
      ctx->launches += x.mode == BVHG_REBUILD ? 9 + ( passes - first ) : 3;
    }
    // scenes, group by group after the builds they read
    for ( int g = 0; g < G; ++g )
    {
      fused_group &fg = grp[g];
      cudaStream_t ls = B.lane[g % L];
      for ( int o : fg.needs )
        if ( o % L != g % L ) BVHG_CUDA( ctx, cudaStreamWaitEvent( ls, B.obj_done[o], 0 ) );
      BVHG_CUDA( ctx, launch_traverse_batch( K, fp32, true, V, fg.l_dense, ls ) );
      BVHG_CUDA( ctx, launch_traverse_batch( K, fp32, false, V, fg.l_sparse, ls ) );
      if ( fp32 ) BVHG_CUDA( ctx, launch_recheck_batch( K, V, fg.l_recheck, ls ) );
      BVHG_CUDA( ctx, launch_gid_pairs_dev_batch( fg.l_gid, ls ) );
      ctx->launches += fp32 ? 4 : 3;
    }
    for ( int l = 0; l < L; ++l )
    {
      BVHG_CUDA( ctx, cudaEventRecord( B.lane_done[l], B.lane[l] ) );
      BVHG_CUDA( ctx, cudaStreamWaitEvent( s, B.lane_done[l], 0 ) );
    }
    BVHG_CUDA( ctx, launch_gather_words( B.err_src.as< const int *const >(), static_cast< int >( uniq.size() ),
                                         B.err_words.as< int >(), s ) );
    return BVHG_OK;
  };
  bvhg_status st = body();
  cudaGraph_t gph = nullptr;
  const cudaError_t ce = cudaStreamEndCapture( s, &gph );
  if ( st != BVHG_OK )
  {
    if ( gph ) cudaGraphDestroy( gph );
    return st;
  }
  if ( ce != cudaSuccess ) return cuda_fail( ctx, ce, "cudaStreamEndCapture" );
  B.graph = gph;
  BVHG_CUDA( ctx, cudaGraphInstantiate( &B.exec, B.graph, 0 ) );
  B.tables = tables;
  return BVHG_OK;
}

// Runs a batch: returns the per-scene exact counts in `counts` (host) and leaves scene sc's pairs in
// B.out[2 * B.off[sc] ...]. Grows per-scene capacities and recaptures until every scene fits.
bvhg_status run_batch(bvhg_ctx *ctx, const batch_args &x, uint64_t *counts)
{
  if ( !ctx->batch ) ctx->batch = std::make_unique< batch_state >();
  batch_state &B = *ctx->batch;
  const bool fp32 = ctx->cfg.precision == BVHG_FILTER_FP32;
  // unique objects in first-use order
  std::vector< int32_t > uniq;
  std::vector< int > slot( ctx->objs.size(), -1 );
  for ( uint32_t sc = 0; sc < x.nscenes; ++sc )
    for ( int32_t o : { x.a[sc], x.b[sc] } )
    {
      if ( !valid_obj( ctx, o ) ) return fail( ctx, BVHG_ERR_ARG, "invalid object in batch" );
      object &ob = *ctx->objs[o];
      if ( !ob.has_data ) return fail( ctx, BVHG_ERR_STATE, "batch object without element data" );
      if ( x.mode == BVHG_REFIT && ob.n > 0 && !ob.topo ) return fail( ctx, BVHG_ERR_STATE, "refit without a rebuild" );
      if ( slot[o] < 0 )
      {
        slot[o] = static_cast< int >( uniq.size() );
        uniq.push_back( o );
      }
    }
  for ( int32_t o : uniq )
  {
    object &ob = *ctx->objs[o];
    join_object( ctx, ob );
    if ( ob.n > 0 && x.mode == BVHG_REBUILD )
    {
      const bvhg_status rs = reserve_object( ctx, ob );
      if ( rs != BVHG_OK ) return rs;
    }
  }
  // per-scene capacities: the last run's if the batch has the same scenes, else an estimate
  const bool same_scenes = B.cap.size() == x.nscenes && B.key.size() > 3 && B.key[1] == x.nscenes;
  if ( !same_scenes )
  {
    B.cap.assign( x.nscenes, 0 );
    for ( uint32_t sc = 0; sc < x.nscenes; ++sc )
      B.cap[sc] = 1024 + 2 * ( ctx->objs[x.a[sc]]->n + ctx->objs[x.b[sc]]->n );
  }
  for ( int attempt = 0; attempt < 4; ++attempt )
  {
    B.off.assign( x.nscenes, 0 );
    uint64_t total = 0;
    for ( uint32_t sc = 0; sc < x.nscenes; ++sc )
    {
      B.off[sc] = total;
      total += B.cap[sc];
    }
    BVHG_CUDA( ctx, B.cand.reserve( total * sizeof( uint2 ) ) );
    if ( fp32 ) BVHG_CUDA( ctx, B.exact.reserve( total * sizeof( uint2 ) ) );
    BVHG_CUDA( ctx, B.out.reserve( total * 16 ) );
    BVHG_CUDA( ctx, B.ps.reserve( x.nscenes * sizeof( pair_scalars ) ) );
    BVHG_CUDA( ctx, B.err_words.reserve( uniq.size() * sizeof( int ) ) );
    BVHG_CUDA( ctx, B.err_src.reserve( uniq.size() * sizeof( void * ) ) );
    if ( B.host_scenes < x.nscenes )
    {
      if ( B.host_ps ) cudaFreeHost( B.host_ps );
      B.host_ps = nullptr;
      BVHG_CUDA( ctx, cudaMallocHost( reinterpret_cast< void ** >( &B.host_ps ), x.nscenes * sizeof( pair_scalars ) ) );
      B.host_scenes = x.nscenes;
    }
    if ( B.host_objs < uniq.size() )
    {
      if ( B.host_err ) cudaFreeHost( B.host_err );
      B.host_err = nullptr;
      BVHG_CUDA( ctx, cudaMallocHost( reinterpret_cast< void ** >( &B.host_err ), uniq.size() * sizeof( int ) ) );
      B.host_objs = uniq.size();
    }
    // graph identity: everything a replay would read from the captured parameters
    std::vector< uint64_t > key{ static_cast< uint64_t >( x.mode ), x.nscenes, static_cast< uint64_t >( B.lanes ),
                                 static_cast< uint64_t >( B.groups ),
                                 reinterpret_cast< uint64_t >( B.cand.p ), reinterpret_cast< uint64_t >( B.out.p ),
                                 reinterpret_cast< uint64_t >( B.exact.p ), reinterpret_cast< uint64_t >( B.ps.p ),
                                 reinterpret_cast< uint64_t >( B.err_src.p ),
                                 reinterpret_cast< uint64_t >( B.err_words.p ) };
    for ( uint32_t sc = 0; sc < x.nscenes; ++sc )
    {
      key.push_back( static_cast< uint64_t >( x.a[sc] ) );
      key.push_back( static_cast< uint64_t >( x.b[sc] ) );
      key.push_back( B.cap[sc] );
    }
    std::vector< const int * > srcs;
    for ( int32_t o : uniq )
    {
      const object &ob = *ctx->objs[o];
      for ( uint64_t v : { ob.n, static_cast< uint64_t >( ob.V ), static_cast< uint64_t >( ob.store_slabs ),
                           static_cast< uint64_t >( ob.dense_ok ),
                           reinterpret_cast< uint64_t >( ob.verts ),
                           reinterpret_cast< uint64_t >( ob.gid ), reinterpret_cast< uint64_t >( ob.scal.p ),
                           reinterpret_cast< uint64_t >( ob.keys.p ), reinterpret_cast< uint64_t >( ob.bucket_box.p ),
                           reinterpret_cast< uint64_t >( ob.node_box.p ) } )
        key.push_back( v );
      srcs.push_back( &ob.sc()->error );
    }
    // the error-word sources of this batch's objects (every cached graph reads them from the same array)
    BVHG_CUDA( ctx, cudaMemcpyAsync( B.err_src.p, srcs.data(), srcs.size() * sizeof( void * ), cudaMemcpyHostToDevice,
                                     ctx->stream ) );
    BVHG_CUDA( ctx, cudaStreamSynchronize( ctx->stream ) );
    if ( !B.select( key ) )
    {
      const uint32_t V = batch_vertex_count( ctx, uniq );
      const bvhg_status st = B.groups > 0 && V ? capture_batch_fused( ctx, B, x, uniq, V, B.groups, B.lanes )
                                               : capture_batch( ctx, B, x, uniq, slot );
      if ( st != BVHG_OK ) return st;
      B.key = key;
      B.keep();
    } else {
      // a replay rebuilds the same objects: their host-side state is what the capture left
      for ( int32_t o : uniq )
      {
        object &ob = *ctx->objs[o];
        ob.built = true;
        ob.fresh = x.mode == BVHG_REBUILD;
        if ( x.mode == BVHG_REBUILD ) ob.clustered = false;
      }
    }
    BVHG_CUDA( ctx, cudaGraphLaunch( B.exec, ctx->stream ) );
    BVHG_CUDA( ctx, cudaMemcpyAsync( B.host_ps, B.ps.p, x.nscenes * sizeof( pair_scalars ), cudaMemcpyDeviceToHost,
                                     ctx->stream ) );
    BVHG_CUDA( ctx, cudaMemcpyAsync( B.host_err, B.err_words.p, uniq.size() * sizeof( int ), cudaMemcpyDeviceToHost,
                                     ctx->stream ) );
    BVHG_CUDA( ctx, cudaStreamSynchronize( ctx->stream ) );
    for ( size_t i = 0; i < uniq.size(); ++i )
    {
      const bvhg_status st = object_error( ctx, B.host_err[i] );
      if ( st != BVHG_OK ) return st;
    }
    bool grown = false;
    uint64_t cand_total = 0;
    for ( uint32_t sc = 0; sc < x.nscenes; ++sc )
    {
      const pair_scalars &h = B.host_ps[sc];
      if ( h.error == kErrOverflowStack && ctx->objs[x.a[sc]]->dense_ok && ctx->objs[x.b[sc]]->dense_ok )
      {
        // the batched dense walk reached its stack bound: this scene's objects take the single-node walk and the
        // batch runs again (a new layout: the graph is captured again)
        ctx->objs[x.a[sc]]->dense_ok = false;
        ctx->objs[x.b[sc]]->dense_ok = false;
        grown = true;
        continue;
      }
      if ( h.error ) return fail( ctx, BVHG_ERR_CUDA, "traversal stack overflow in batch scene " + std::to_string( sc ) );
      const uint64_t need = fp32 ? std::max( h.count, h.count2 ) : h.count;
      cand_total += h.count;
      counts[sc] = fp32 ? h.count2 : h.count;
      if ( need > B.cap[sc] )
      {
        B.cap[sc] = need + need / 4 + 64;
        grown = true;
      }
    }
    ctx->last_candidates = cand_total;
    if ( !grown )
    {
      // contact density per object over its scenes, for the next run's builds
      std::vector< uint64_t > cand_of( ctx->objs.size(), 0 ), elems_of( ctx->objs.size(), 0 );
      for ( uint32_t sc = 0; sc < x.nscenes; ++sc )
      {
        const uint64_t c = B.host_ps[sc].count;
        const uint64_t e = ctx->objs[x.a[sc]]->n + ( x.a[sc] == x.b[sc] ? 0 : ctx->objs[x.b[sc]]->n );
        for ( int32_t o : { x.a[sc], x.b[sc] } )
        {
          cand_of[o] += c;
          elems_of[o] += e;
        }
      }
      for ( int32_t o : uniq ) ctx->objs[o]->store_slabs = cand_of[o] > 0 && cand_of[o] * 50 >= elems_of[o];
      return BVHG_OK;
    }
  }
  return fail( ctx, BVHG_ERR_CUDA, "batch pair capacities did not converge" );
}
}  // namespace

extern "C" {

void bvhg_config_default(bvhg_config *cfg)
{
  if ( !cfg ) return;
  std::memset( cfg, 0, sizeof( *cfg ) );
  cfg->k = 18;
  cfg->precision = BVHG_PLAIN_FP64;
  cfg->sort_digit_bits = 8;
  cfg->device = 0;
  cfg->epsilon = 0.0;
  cfg->stream = nullptr;
  cfg->spin_limit = 0;
  cfg->flags = 0;
}

bvhg_status bvhg_create(bvhg_ctx **out, const bvhg_config *cfg)
{
  if ( !out ) return BVHG_ERR_ARG;
  *out = nullptr;
  bvhg_config c;
  bvhg_config_default( &c );
  if ( cfg ) c = *cfg;
  if ( c.k != 6 && c.k != 18 && c.k != 26 ) return BVHG_ERR_ARG;
  if ( c.precision != BVHG_PLAIN_FP64 && c.precision != BVHG_FILTER_FP32 ) return BVHG_ERR_ARG;
  if ( c.sort_digit_bits != 1 && c.sort_digit_bits != 2 && c.sort_digit_bits != 4 && c.sort_digit_bits != 8 )
    return BVHG_ERR_ARG;
  if ( !( c.epsilon >= 0.0 ) || c.epsilon > 1e300 ) return BVHG_ERR_ARG;
  if ( cudaSetDevice( c.device ) != cudaSuccess ) return BVHG_ERR_CUDA;
  auto ctx = std::make_unique< bvhg_ctx >();
  ctx->cfg = c;
  ctx->spin_limit = c.spin_limit ? c.spin_limit : kDefaultSpinLimit;
  if ( c.stream )
  {
    ctx->stream = static_cast< cudaStream_t >( c.stream );
  } else {
    if ( cudaStreamCreateWithFlags( &ctx->stream, cudaStreamNonBlocking ) != cudaSuccess ) return BVHG_ERR_CUDA;
    ctx->own_stream = true;
  }
  if ( cudaMallocHost( reinterpret_cast< void ** >( &ctx->host_ps ), sizeof( pair_scalars ) ) != cudaSuccess ||
       cudaMallocHost( reinterpret_cast< void ** >( &ctx->host_err ), 2 * sizeof( int ) ) != cudaSuccess ||
       cudaMallocHost( reinterpret_cast< void ** >( &ctx->init_template ), sizeof( obj_scalars ) ) != cudaSuccess )
    return BVHG_ERR_CUDA;
  std::memset( ctx->init_template, 0, sizeof( obj_scalars ) );
  for ( int c = 0; c < 3; ++c )
  {
    ctx->init_template->bounds_enc[c] = ~0ull;  // min accumulators start at the largest encoding
    ctx->init_template->bounds_enc[3 + c] = 0ull;
  }
  *out = ctx.release();
  return BVHG_OK;
}

bvhg_status bvhg_destroy(bvhg_ctx *ctx)
{
  if ( !ctx ) return BVHG_ERR_ARG;
  cudaSetDevice( ctx->cfg.device );
  for ( auto &o : ctx->objs )
    if ( o ) join_object( ctx, *o );
  cudaStreamSynchronize( ctx->stream );
  collect_timing( ctx );
  for ( auto e : ctx->event_pool ) cudaEventDestroy( e );
  if ( ctx->host_ps ) cudaFreeHost( ctx->host_ps );
  if ( ctx->host_err ) cudaFreeHost( ctx->host_err );
  if ( ctx->init_template ) cudaFreeHost( ctx->init_template );
  ctx->objs.clear();
  if ( ctx->fork_evt ) cudaEventDestroy( ctx->fork_evt );
  if ( ctx->own_stream ) cudaStreamDestroy( ctx->stream );
  delete ctx;
  return BVHG_OK;
}

bvhg_status bvhg_object_create(bvhg_ctx *ctx, int32_t *obj)
{
  if ( !ctx || !obj ) return fail( ctx, BVHG_ERR_ARG, "null argument" );
  cudaSetDevice( ctx->cfg.device );
  auto o = std::make_unique< object >();
  BVHG_CUDA( ctx, o->scal.reserve( sizeof( obj_scalars ) ) );
  BVHG_CUDA( ctx, cudaMemsetAsync( o->scal.p, 0, sizeof( obj_scalars ), ctx->stream ) );
  ctx->objs.push_back( std::move( o ) );
  *obj = static_cast< int32_t >( ctx->objs.size() - 1 );
  return BVHG_OK;
}

bvhg_status bvhg_object_destroy(bvhg_ctx *ctx, int32_t obj)
{
  if ( !valid_obj( ctx, obj ) ) return fail( ctx, BVHG_ERR_ARG, "invalid object" );
  cudaSetDevice( ctx->cfg.device );
  cudaStreamSynchronize( ctx->stream );
  ctx->objs[obj].reset();
  return BVHG_OK;
}

bvhg_status bvhg_set_elements(bvhg_ctx *ctx, int32_t obj, const double *xyz, uint32_t V, const uint64_t *gid,
                              uint64_t n, int32_t mem)
{
  if ( !valid_obj( ctx, obj ) ) return fail( ctx, BVHG_ERR_ARG, "invalid object" );
  if ( V == 0 || V > 32 ) return fail( ctx, BVHG_ERR_ARG, "verts_per_elem must be in [1, 32]" );
  if ( n > kMaxElements ) return fail( ctx, BVHG_ERR_ARG, "too many elements (limit 2^30 - 1)" );
  if ( n > 0 && !xyz ) return fail( ctx, BVHG_ERR_ARG, "null vertex pointer" );
  if ( mem != BVHG_MEM_HOST && mem != BVHG_MEM_DEVICE ) return fail( ctx, BVHG_ERR_ARG, "bad memory kind" );
  cudaSetDevice( ctx->cfg.device );
  object &o = *ctx->objs[obj];
  join_object( ctx, o );  // the last build may still read the owned vertex buffer
  if ( n != o.n || V != o.V )
  {
    o.topo = false;
    o.dense_ok = true;
  }
  o.n = n;
  o.V = V;
  o.built = false;
  o.fresh = false;
  o.has_data = true;
  o.clustered = false;
  if ( n == 0 )
  {
    o.verts = nullptr;
    o.gid = nullptr;
    return BVHG_OK;
  }
  if ( mem == BVHG_MEM_DEVICE )
  {
    o.verts = xyz;
    o.gid = gid;
  } else {
    const size_t vb = n * V * 3 * sizeof( double );
    BVHG_CUDA( ctx, o.verts_own.reserve( vb ) );
    BVHG_CUDA( ctx, cudaMemcpyAsync( o.verts_own.p, xyz, vb, cudaMemcpyHostToDevice, ctx->stream ) );
    o.verts = o.verts_own.as< double >();
    if ( gid )
    {
      BVHG_CUDA( ctx, o.gid_own.reserve( n * 8 ) );
      BVHG_CUDA( ctx, cudaMemcpyAsync( o.gid_own.p, gid, n * 8, cudaMemcpyHostToDevice, ctx->stream ) );
      o.gid = o.gid_own.as< uint64_t >();
    } else {
      o.gid = nullptr;
    }
  }
  return BVHG_OK;
}

bvhg_status bvhg_build(bvhg_ctx *ctx, int32_t obj, int32_t mode)
{
  if ( !valid_obj( ctx, obj ) ) return fail( ctx, BVHG_ERR_ARG, "invalid object" );
  if ( mode != BVHG_REBUILD && mode != BVHG_REFIT ) return fail( ctx, BVHG_ERR_ARG, "bad build mode" );
  object &o = *ctx->objs[obj];
  if ( !o.has_data ) return fail( ctx, BVHG_ERR_STATE, "build before set_elements" );
  cudaSetDevice( ctx->cfg.device );
  return do_build( ctx, o, mode );
}

bvhg_status bvhg_broadphase(bvhg_ctx *ctx, int32_t obj_a, int32_t obj_b, uint64_t *pairs, uint64_t capacity,
                            uint64_t *count, int32_t mem)
{
  if ( !valid_obj( ctx, obj_a ) || !valid_obj( ctx, obj_b ) ) return fail( ctx, BVHG_ERR_ARG, "invalid object" );
  if ( !count ) return fail( ctx, BVHG_ERR_ARG, "null count" );
  if ( capacity > 0 && !pairs ) return fail( ctx, BVHG_ERR_ARG, "null pair buffer" );
  object &a = *ctx->objs[obj_a];
  object &b = *ctx->objs[obj_b];
  if ( !a.built || !b.built ) return fail( ctx, BVHG_ERR_STATE, "broadphase before build" );
  cudaSetDevice( ctx->cfg.device );
  join_object( ctx, a );
  join_object( ctx, b );
  *count = 0;
  if ( a.n == 0 || b.n == 0 )
  {
    ctx->last_candidates = 0;
    return BVHG_OK;
  }
  const uint2 *lp = nullptr;
  uint64_t np = 0;
  bvhg_status st = find_pairs( ctx, a, b, false, &lp, &np );
  if ( st != BVHG_OK ) return st;
  note_density( a, b, false, ctx->last_candidates );
  return emit_pairs( ctx, a, b, false, lp, np, pairs, capacity, count, mem );
}

namespace {
// True when p is device memory of any GPU (managed memory counts as host here: the host may access it).
bool is_device_pointer(const void *p)
{
  cudaPointerAttributes at{};
  if ( cudaPointerGetAttributes( &at, p ) != cudaSuccess )
  {
    cudaGetLastError();  // not a pointer CUDA knows: host memory (the error is not sticky; clear it)
    return false;
  }
  return at.type == cudaMemoryTypeDevice;
}
}  // namespace

bvhg_status bvhg_batch_broadphase(bvhg_ctx *ctx, uint32_t nscenes, const int32_t *obj_a, const int32_t *obj_b,
                                  int32_t mode, uint64_t *pairs, uint64_t capacity, uint64_t *counts,
                                  uint64_t *offsets, int32_t mem)
{
  if ( !ctx ) return BVHG_ERR_ARG;
  if ( nscenes > 0 && ( !obj_a || !obj_b || !counts ) ) return fail( ctx, BVHG_ERR_ARG, "null scene arrays" );
  if ( mode != BVHG_REBUILD && mode != BVHG_REFIT ) return fail( ctx, BVHG_ERR_ARG, "bad build mode" );
  if ( mem != BVHG_MEM_HOST && mem != BVHG_MEM_DEVICE ) return fail( ctx, BVHG_ERR_ARG, "bad memory kind" );
  if ( capacity > 0 && !pairs ) return fail( ctx, BVHG_ERR_ARG, "null pair buffer" );
  if ( nscenes == 0 ) return BVHG_OK;
  cudaSetDevice( ctx->cfg.device );
  // the scene arrays, counts and offsets are host memory: a device pointer is refused, not dereferenced
  for ( const void *h : { static_cast< const void * >( obj_a ), static_cast< const void * >( obj_b ),
                          static_cast< const void * >( counts ), static_cast< const void * >( offsets ) } )
    if ( h && is_device_pointer( h ) ) return fail( ctx, BVHG_ERR_ARG, "scene arrays, counts and offsets must be host memory" );
  const batch_args x{ nscenes, obj_a, obj_b, mode };
  bvhg_status st = run_batch( ctx, x, counts );
  if ( st != BVHG_OK ) return st;
  // compact the scenes' pairs into the caller's buffer in scene order
  uint64_t total = 0;
  for ( uint32_t sc = 0; sc < nscenes; ++sc )
  {
    if ( offsets ) offsets[sc] = total;
    total += counts[sc];
  }
  if ( total > capacity ) return fail( ctx, BVHG_ERR_OVERFLOW, "pair buffer too small: " + std::to_string( total ) + " pairs" );
  batch_state &B = *ctx->batch;
  uint64_t at = 0;
  for ( uint32_t sc = 0; sc < nscenes; ++sc )
  {
    if ( counts[sc] )
      BVHG_CUDA( ctx, cudaMemcpyAsync( pairs + 2 * at, B.out.as< uint64_t >() + 2 * B.off[sc], counts[sc] * 16,
                                       mem == BVHG_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                                       ctx->stream ) );
    at += counts[sc];
  }
  BVHG_CUDA( ctx, cudaStreamSynchronize( ctx->stream ) );
  return BVHG_OK;
}

bvhg_status bvhg_batch_autotune(bvhg_ctx *ctx, uint32_t nscenes, const int32_t *obj_a, const int32_t *obj_b,
                                int32_t mode, uint32_t *groups, uint32_t *lanes, double *ms)
{
  if ( !ctx ) return BVHG_ERR_ARG;
  if ( nscenes == 0 || !obj_a || !obj_b ) return fail( ctx, BVHG_ERR_ARG, "empty batch" );
  if ( mode != BVHG_REBUILD && mode != BVHG_REFIT ) return fail( ctx, BVHG_ERR_ARG, "bad build mode" );
  cudaSetDevice( ctx->cfg.device );
  if ( !ctx->batch ) ctx->batch = std::make_unique< batch_state >();
  const batch_args x{ nscenes, obj_a, obj_b, mode };
  std::vector< uint64_t > counts( nscenes );
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  BVHG_CUDA( ctx, cudaEventCreate( &e0 ) );
  BVHG_CUDA( ctx, cudaEventCreate( &e1 ) );
  int best_groups = ctx->batch->groups, best_lanes = ctx->batch->lanes;
  float best_ms = 0.f;
  bvhg_status st = BVHG_OK;
  // fused form: groups of objects (the batch's tile), one stream per group up to 16; laned form: per-object launches
  const std::pair< int, int > configs[] = { { 1, 1 }, { 4, 4 }, { 16, 16 }, { 64, 16 }, { 256, 16 },
                                            { 0, 16 }, { 0, 64 } };
  for ( const auto &cfg : configs )
  {
    ctx->batch->groups = cfg.first;
    ctx->batch->lanes = cfg.second;
    st = run_batch( ctx, x, counts.data() );  // captures this configuration's graph and settles the capacities
    if ( st != BVHG_OK ) break;
    float t = 0.f;
    cudaEventRecord( e0, ctx->stream );
    for ( int r = 0; r < 3; ++r ) cudaGraphLaunch( ctx->batch->exec, ctx->stream );
    cudaEventRecord( e1, ctx->stream );
    if ( cudaEventSynchronize( e1 ) != cudaSuccess || cudaEventElapsedTime( &t, e0, e1 ) != cudaSuccess )
    {
      st = fail( ctx, BVHG_ERR_CUDA, "autotune timing" );
      break;
    }
    t /= 3.f;
    if ( best_ms == 0.f || t < best_ms )
    {
      best_ms = t;
      best_groups = cfg.first;
      best_lanes = cfg.second;
    }
  }
  cudaEventDestroy( e0 );
  cudaEventDestroy( e1 );
  ctx->batch->groups = best_groups;
  ctx->batch->lanes = best_lanes;
  ctx->batch->drop_graph();
  if ( lanes ) *lanes = static_cast< uint32_t >( best_lanes );
  if ( groups ) *groups = static_cast< uint32_t >( best_groups );
  if ( ms ) *ms = best_ms;
  return st;
}

bvhg_status bvhg_self_collision(bvhg_ctx *ctx, int32_t obj, uint64_t *pairs, uint64_t capacity, uint64_t *count,
                                int32_t mem)
{
  if ( !valid_obj( ctx, obj ) ) return fail( ctx, BVHG_ERR_ARG, "invalid object" );
  if ( !count ) return fail( ctx, BVHG_ERR_ARG, "null count" );
  if ( capacity > 0 && !pairs ) return fail( ctx, BVHG_ERR_ARG, "null pair buffer" );
  object &o = *ctx->objs[obj];
  if ( !o.built ) return fail( ctx, BVHG_ERR_STATE, "self_collision before build" );
  cudaSetDevice( ctx->cfg.device );
  join_object( ctx, o );
  *count = 0;
  if ( o.n < 2 )
  {
    ctx->last_candidates = 0;
    return BVHG_OK;
  }
  const uint2 *lp = nullptr;
  uint64_t np = 0;
  bvhg_status st = find_pairs( ctx, o, o, true, &lp, &np );
  if ( st != BVHG_OK ) return st;
  note_density( o, o, true, ctx->last_candidates );
  return emit_pairs( ctx, o, o, true, lp, np, pairs, capacity, count, mem );
}

bvhg_status bvhg_sort_and_sweep(bvhg_ctx *ctx, int32_t obj_a, int32_t obj_b, int32_t axis, uint64_t *pairs,
                                uint64_t capacity, uint64_t *count, int32_t *axis_used, int32_t mem)
{
  if ( !valid_obj( ctx, obj_a ) || !valid_obj( ctx, obj_b ) ) return fail( ctx, BVHG_ERR_ARG, "invalid object" );
  if ( obj_a == obj_b ) return fail( ctx, BVHG_ERR_ARG, "sort-and-sweep needs two objects (bvhg_self_collision for one)" );
  if ( !count ) return fail( ctx, BVHG_ERR_ARG, "null count" );
  if ( capacity > 0 && !pairs ) return fail( ctx, BVHG_ERR_ARG, "null pair buffer" );
  if ( axis < -1 || axis > 2 ) return fail( ctx, BVHG_ERR_ARG, "axis must be -1, 0, 1 or 2" );
  if ( mem != BVHG_MEM_HOST && mem != BVHG_MEM_DEVICE ) return fail( ctx, BVHG_ERR_ARG, "bad memory kind" );
  object &a = *ctx->objs[obj_a];
  object &b = *ctx->objs[obj_b];
  if ( !a.built || !b.built ) return fail( ctx, BVHG_ERR_STATE, "sort-and-sweep before build" );
  // the global range and the axis come from the objects' bounds and centroids, which only a rebuild computes
  if ( !a.fresh || !b.fresh ) return fail( ctx, BVHG_ERR_STATE, "sort-and-sweep needs a rebuild (not a refit) since set_elements" );
  cudaSetDevice( ctx->cfg.device );
  join_object( ctx, a );
  join_object( ctx, b );
  *count = 0;
  if ( axis_used ) *axis_used = axis < 0 ? 0 : axis;
  if ( a.n == 0 || b.n == 0 ) return BVHG_OK;
  const int K = ctx->cfg.k;
  const uint64_t nb = b.n;
  const uint64_t nb4 = ( nb + 3 ) & ~3ull;  // second halves of the ping-pong buffers start 16-byte aligned
  const uint64_t tiles = ( nb + kSortTile - 1 ) / kSortTile;
  const uint64_t status_words = 4 * ( tiles + 1 ) * 256;
  cudaStream_t s = ctx->stream;
  BVHG_CUDA( ctx, ctx->sw_keys.reserve( 2 * nb4 * 8 ) );
  BVHG_CUDA( ctx, ctx->sw_vals.reserve( 2 * nb4 * 4 ) );
  BVHG_CUDA( ctx, ctx->sw_rows.reserve( nb * K * 8 ) );
  BVHG_CUDA( ctx, ctx->sw_srows.reserve( nb * K * 8 ) );
  BVHG_CUDA( ctx, ctx->sw_sbmax.reserve( nb * 8 ) );
  BVHG_CUDA( ctx, ctx->sw_hist.reserve( 4 * 256 * 4 ) );
  BVHG_CUDA( ctx, ctx->sw_status.reserve( status_words * 4 ) );
  BVHG_CUDA( ctx, ctx->sw_sc.reserve( sizeof( obj_scalars ) ) );
  BVHG_CUDA( ctx, ctx->sw_params.reserve( sweep_params_bytes() ) );
  BVHG_CUDA( ctx, ctx->sw_partial.reserve( sweep_partial_bytes() ) );
  BVHG_CUDA( ctx, ctx->pscal.reserve( sizeof( pair_scalars ) ) );
  if ( ctx->pair_cap == 0 )
  {
    ctx->pair_cap = 1u << 20;
    BVHG_CUDA( ctx, ctx->pairs.reserve( ctx->pair_cap * sizeof( uint2 ) ) );
  }
  uint64_t *k0 = ctx->sw_keys.as< uint64_t >(), *k1 = k0 + nb4;
  uint32_t *v0 = ctx->sw_vals.as< uint32_t >(), *v1 = v0 + nb4;
  obj_scalars *ssc = ctx->sw_sc.as< obj_scalars >();
  pair_scalars *ps = ctx->pscal.as< pair_scalars >();
  sweep_launch x{};
  x.K = K;
  x.averts = a.verts;
  x.bverts = b.verts;
  x.aV = a.V;
  x.bV = b.V;
  x.na = a.n;
  x.nb = nb;
  x.eps = ctx->cfg.epsilon;
  x.acx = a.cx.as< double >();
  x.acy = a.cy.as< double >();
  x.acz = a.cz.as< double >();
  x.bcx = b.cx.as< double >();
  x.bcy = b.cy.as< double >();
  x.bcz = b.cz.as< double >();
  x.asc = a.sc();
  x.bsc = b.sc();
  x.partial = ctx->sw_partial.as< double >();
  x.params = ctx->sw_params.p;
  x.rows = ctx->sw_rows.as< double >();
  x.keys = k0;
  x.hist = ctx->sw_hist.as< uint32_t >();
  x.skeys = k0;  // four passes: k0 -> k1 -> k0 -> k1 -> k0
  x.svals = v0;
  x.srows = ctx->sw_srows.as< double >();
  x.sbmax = ctx->sw_sbmax.as< double >();
  x.aperm = a.sorted_vals();
  x.sc = ssc;
  x.ps = ps;
  x.s = s;
  for ( int attempt = 0; attempt < 3; ++attempt )
  {
    x.pairs = ctx->pairs.as< uint2 >();
    x.cap = ctx->pair_cap;
    BVHG_CUDA( ctx, cudaMemsetAsync( ssc, 0, sizeof( obj_scalars ), s ) );
    BVHG_CUDA( ctx, cudaMemsetAsync( x.hist, 0, 4 * 256 * 4, s ) );
    BVHG_CUDA( ctx, cudaMemsetAsync( ctx->sw_status.p, 0, status_words * 4, s ) );
    BVHG_CUDA( ctx, cudaMemsetAsync( ps, 0, sizeof( pair_scalars ), s ) );
    BVHG_CUDA( ctx, launch_sweep_setup( x, axis ) );
    BVHG_CUDA( ctx, launch_sweep_keys( x ) );
    for ( int pass = 0; pass < 4; ++pass )
    {
      const bool even = ( pass & 1 ) == 0;
      BVHG_CUDA( ctx, launch_onesweep( 8, even ? k0 : k1, pass == 0 ? nullptr : ( even ? v0 : v1 ), even ? k1 : k0,
                                       even ? v1 : v0, nb, pass, x.hist, ctx->sw_status.as< uint32_t >(), ssc,
                                       ctx->spin_limit, 0, s ) );
    }
    BVHG_CUDA( ctx, launch_sweep( x ) );
    BVHG_CUDA( ctx, cudaMemcpyAsync( ctx->host_ps, ps, sizeof( pair_scalars ), cudaMemcpyDeviceToHost, s ) );
    BVHG_CUDA( ctx, cudaMemcpyAsync( ctx->host_err, &ssc->error, sizeof( int ), cudaMemcpyDeviceToHost, s ) );
    BVHG_CUDA( ctx, cudaMemcpyAsync( ctx->host_err + 1, x.params, sizeof( int ), cudaMemcpyDeviceToHost, s ) );
    BVHG_CUDA( ctx, cudaStreamSynchronize( s ) );
    const bvhg_status st = object_error( ctx, ctx->host_err[0] );
    if ( st != BVHG_OK ) return st;
    if ( axis_used ) *axis_used = ctx->host_err[1];
    const uint64_t np = ctx->host_ps->count;
    if ( np > ctx->pair_cap )
    {
      ctx->pair_cap = np + np / 8;
      BVHG_CUDA( ctx, ctx->pairs.reserve( ctx->pair_cap * sizeof( uint2 ) ) );
      continue;
    }
    return emit_pairs( ctx, a, b, false, ctx->pairs.as< uint2 >(), np, pairs, capacity, count, mem );
  }
  return fail( ctx, BVHG_ERR_CUDA, "pair buffer did not converge" );
}

bvhg_status bvhg_cluster(bvhg_ctx *ctx, int32_t obj, uint32_t patches, uint64_t *bounds, uint32_t *order,
                         int32_t mem)
{
  if ( !valid_obj( ctx, obj ) ) return fail( ctx, BVHG_ERR_ARG, "invalid object" );
  if ( patches == 0 || patches > ( 1u << 24 ) ) return fail( ctx, BVHG_ERR_ARG, "patches must be in [1, 2^24]" );
  if ( mem != BVHG_MEM_HOST && mem != BVHG_MEM_DEVICE ) return fail( ctx, BVHG_ERR_ARG, "bad memory kind" );
  object &o = *ctx->objs[obj];
  if ( !o.built || ( o.n > 0 && !o.topo ) ) return fail( ctx, BVHG_ERR_STATE, "cluster before a rebuild" );
  cudaSetDevice( ctx->cfg.device );
  join_object( ctx, o );
  const uint64_t n = o.n;
  const uint64_t nb = cluster_block_count( n ) + 1;
  BVHG_CUDA( ctx, o.cl_order.reserve( n * 4 ) );
  BVHG_CUDA( ctx, o.cl_rank.reserve( n * 4 ) );
  BVHG_CUDA( ctx, o.cl_tmp.reserve( n * 4 ) );
  BVHG_CUDA( ctx, o.cl_runs.reserve( long_run_capacity( n ) * 4 ) );
  BVHG_CUDA( ctx, o.cl_bhist.reserve( nb * 33 * 4 ) );
  BVHG_CUDA( ctx, o.cl_bbase.reserve( nb * 2 * 4 ) );
  BVHG_CUDA( ctx, o.cl_splits.reserve( static_cast< size_t >( patches ) * 4 ) );
  BVHG_CUDA( ctx, o.cl_bounds.reserve( ( static_cast< size_t >( patches ) + 1 ) * 8 ) );
  BVHG_CUDA( ctx, o.cl_scal.reserve( sizeof( cluster_scalars ) ) );
  if ( n > 0 )
  {
    // the keys' order must be the build's valid one
    const bvhg_status st = check_scalar_errors( ctx, o );
    if ( st != BVHG_OK ) return st;
  }
  cluster_launch x;
  x.keys = o.n ? o.sorted_keys() : nullptr;
  x.perm = o.n ? o.sorted_vals() : nullptr;
  x.n = n;
  x.patches = patches;
  x.order = o.cl_order.as< uint32_t >();
  x.rank = o.cl_rank.as< uint32_t >();
  x.tmp = o.cl_tmp.as< uint32_t >();
  x.runs = o.cl_runs.as< uint32_t >();
  x.bhist = o.cl_bhist.as< uint32_t >();
  x.bbase = o.cl_bbase.as< uint32_t >();
  x.splits = o.cl_splits.as< uint32_t >();
  x.bounds = o.cl_bounds.as< uint64_t >();
  x.cs = o.cl_scal.as< cluster_scalars >();
  x.s = ctx->stream;
  BVHG_CUDA( ctx, launch_cluster( x ) );
  ctx->launches += 8;
  const cudaMemcpyKind kind = mem == BVHG_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  if ( bounds )
    BVHG_CUDA( ctx, cudaMemcpyAsync( bounds, x.bounds, ( static_cast< size_t >( patches ) + 1 ) * 8, kind, ctx->stream ) );
  if ( order && n ) BVHG_CUDA( ctx, cudaMemcpyAsync( order, x.order, n * 4, kind, ctx->stream ) );
  BVHG_CUDA( ctx, cudaStreamSynchronize( ctx->stream ) );
  o.clustered = true;
  o.cl_patches = patches;
  return BVHG_OK;
}

bvhg_status bvhg_patch_kdops(bvhg_ctx *ctx, int32_t obj, double *boxes, int32_t mem)
{
  if ( !valid_obj( ctx, obj ) ) return fail( ctx, BVHG_ERR_ARG, "invalid object" );
  if ( !boxes ) return fail( ctx, BVHG_ERR_ARG, "null box buffer" );
  if ( mem != BVHG_MEM_HOST && mem != BVHG_MEM_DEVICE ) return fail( ctx, BVHG_ERR_ARG, "bad memory kind" );
  object &o = *ctx->objs[obj];
  if ( !o.clustered ) return fail( ctx, BVHG_ERR_STATE, "patch k-DOPs before bvhg_cluster" );
  cudaSetDevice( ctx->cfg.device );
  join_object( ctx, o );
  const uint32_t P = o.cl_patches;
  const int K = ctx->cfg.k;
  const size_t bytes = static_cast< size_t >( P ) * K * 8;
  BVHG_CUDA( ctx, o.cl_enc.reserve( bytes ) );
  BVHG_CUDA( ctx, o.cl_boxes.reserve( bytes ) );
  BVHG_CUDA( ctx, launch_patch_kdops( K, o.verts, o.V, o.n, ctx->cfg.epsilon, o.cl_order.as< uint32_t >(),
                                      o.cl_bounds.as< uint64_t >(), P, o.cl_enc.as< unsigned long long >(),
                                      o.cl_boxes.as< double >(), ctx->stream ) );
  ctx->launches += o.n ? 3 : 2;
  BVHG_CUDA( ctx, cudaMemcpyAsync( boxes, o.cl_boxes.p, bytes,
                                   mem == BVHG_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, ctx->stream ) );
  BVHG_CUDA( ctx, cudaStreamSynchronize( ctx->stream ) );
  return BVHG_OK;
}

bvhg_status bvhg_patch_pairs(bvhg_ctx *ctx, int32_t obj_a, int32_t obj_b, uint32_t *groups, uint64_t group_capacity,
                             uint64_t *group_count, uint32_t *pairs, uint64_t pair_capacity, uint64_t *pair_count,
                             int32_t mem)
{
  if ( !valid_obj( ctx, obj_a ) || !valid_obj( ctx, obj_b ) ) return fail( ctx, BVHG_ERR_ARG, "invalid object" );
  if ( obj_a == obj_b ) return fail( ctx, BVHG_ERR_ARG, "patch pairs need two distinct objects" );
  if ( !group_count || !pair_count ) return fail( ctx, BVHG_ERR_ARG, "null count" );
  if ( ( group_capacity > 0 && !groups ) || ( pair_capacity > 0 && !pairs ) )
    return fail( ctx, BVHG_ERR_ARG, "null output buffer" );
  if ( mem != BVHG_MEM_HOST && mem != BVHG_MEM_DEVICE ) return fail( ctx, BVHG_ERR_ARG, "bad memory kind" );
  object &a = *ctx->objs[obj_a];
  object &b = *ctx->objs[obj_b];
  if ( !a.built || !b.built ) return fail( ctx, BVHG_ERR_STATE, "patch pairs before build" );
  if ( !a.clustered || !b.clustered ) return fail( ctx, BVHG_ERR_STATE, "patch pairs before bvhg_cluster" );
  cudaSetDevice( ctx->cfg.device );
  join_object( ctx, a );
  join_object( ctx, b );
  *group_count = 0;
  *pair_count = 0;
  if ( a.n == 0 || b.n == 0 )
  {
    ctx->last_candidates = 0;
    return BVHG_OK;
  }
  const uint2 *lp = nullptr;
  uint64_t np = 0;
  bvhg_status st = find_pairs( ctx, a, b, false, &lp, &np );
  if ( st != BVHG_OK ) return st;
  note_density( a, b, false, ctx->last_candidates );
  if ( np >= ( 1ull << 32 ) ) return fail( ctx, BVHG_ERR_ARG, "more than 2^32 - 1 pairs" );
  const uint64_t bins = static_cast< uint64_t >( a.cl_patches ) * b.cl_patches;
  const uint64_t rows = std::min< uint64_t >( bins, np );
  cudaStream_t s = ctx->stream;
  BVHG_CUDA( ctx, ctx->grp_count.reserve( bins * 4 ) );
  BVHG_CUDA( ctx, ctx->grp_off.reserve( bins * 4 ) );
  BVHG_CUDA( ctx, ctx->grp_rows.reserve( ( rows + 1 ) * 16 ) );
  BVHG_CUDA( ctx, ctx->grp_pairs.reserve( ( np + 1 ) * 8 ) );
  BVHG_CUDA( ctx, ctx->grp_scal.reserve( sizeof( cluster_scalars ) ) );
  group_launch g;
  g.bounds_a = a.cl_bounds.as< uint64_t >();
  g.bounds_b = b.cl_bounds.as< uint64_t >();
  g.rank_a = a.cl_rank.as< uint32_t >();
  g.rank_b = b.cl_rank.as< uint32_t >();
  g.patches_a = a.cl_patches;
  g.patches_b = b.cl_patches;
  cluster_scalars *cs = ctx->grp_scal.as< cluster_scalars >();
  BVHG_CUDA( ctx, launch_group_pairs( lp, np, g, ctx->grp_count.as< uint32_t >(), ctx->grp_off.as< uint32_t >(),
                                      ctx->grp_rows.as< uint32_t >(), rows, ctx->grp_pairs.as< uint32_t >(), cs, s ) );
  ctx->launches += 3;
  cluster_scalars h{};
  BVHG_CUDA( ctx, cudaMemcpyAsync( &h, cs, sizeof( h ), cudaMemcpyDeviceToHost, s ) );
  BVHG_CUDA( ctx, cudaStreamSynchronize( s ) );
  *group_count = h.groups;
  *pair_count = np;
  const cudaMemcpyKind kind = mem == BVHG_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  if ( h.groups > group_capacity || np > pair_capacity )
    return fail( ctx, BVHG_ERR_OVERFLOW, "patch pair buffers too small: " + std::to_string( h.groups ) + " groups, " +
                                           std::to_string( np ) + " pairs" );
  if ( h.groups ) BVHG_CUDA( ctx, cudaMemcpyAsync( groups, ctx->grp_rows.p, h.groups * 16, kind, s ) );
  if ( np ) BVHG_CUDA( ctx, cudaMemcpyAsync( pairs, ctx->grp_pairs.p, np * 8, kind, s ) );
  BVHG_CUDA( ctx, cudaStreamSynchronize( s ) );
  return BVHG_OK;
}

bvhg_status bvhg_get_morton(bvhg_ctx *ctx, int32_t obj, uint64_t *sorted_keys, uint32_t *perm, double *min3,
                            double *inv3)
{
  if ( !valid_obj( ctx, obj ) ) return fail( ctx, BVHG_ERR_ARG, "invalid object" );
  object &o = *ctx->objs[obj];
  if ( !o.built ) return fail( ctx, BVHG_ERR_STATE, "probe before build" );
  cudaSetDevice( ctx->cfg.device );
  join_object( ctx, o );
  BVHG_CUDA( ctx, cudaStreamSynchronize( ctx->stream ) );
  if ( o.n == 0 ) return BVHG_OK;
  bvhg_status st = check_scalar_errors( ctx, o );
  if ( st != BVHG_OK ) return st;
  obj_scalars h;
  BVHG_CUDA( ctx, cudaMemcpy( &h, o.sc(), sizeof( h ), cudaMemcpyDeviceToHost ) );
  if ( sorted_keys ) BVHG_CUDA( ctx, cudaMemcpy( sorted_keys, o.sorted_keys(), o.n * 8, cudaMemcpyDeviceToHost ) );
  if ( perm ) BVHG_CUDA( ctx, cudaMemcpy( perm, o.sorted_vals(), o.n * 4, cudaMemcpyDeviceToHost ) );
  if ( min3 ) std::memcpy( min3, h.min3, sizeof( h.min3 ) );
  if ( inv3 ) std::memcpy( inv3, h.inv3, sizeof( h.inv3 ) );
  return BVHG_OK;
}

static bvhg_status probe_kdops(bvhg_ctx *ctx, int32_t obj, void *out, bool fp32)
{
  if ( !valid_obj( ctx, obj ) || !out ) return fail( ctx, BVHG_ERR_ARG, "invalid argument" );
  object &o = *ctx->objs[obj];
  if ( !o.has_data ) return fail( ctx, BVHG_ERR_STATE, "probe before set_elements" );
  cudaSetDevice( ctx->cfg.device );
  join_object( ctx, o );
  if ( o.n == 0 ) return BVHG_OK;
  const int D = ctx->cfg.k / 2;
  const size_t bytes = o.n * D * 2 * ( fp32 ? 4 : 8 );
  dev_buf tmp;
  BVHG_CUDA( ctx, tmp.reserve( bytes ) );
  BVHG_CUDA( ctx, launch_probe_kdops( ctx->cfg.k, fp32, o.verts, o.V, o.n, ctx->cfg.epsilon, tmp.p, ctx->stream ) );
  ctx->launches += 1;
  BVHG_CUDA( ctx, cudaStreamSynchronize( ctx->stream ) );
  BVHG_CUDA( ctx, cudaMemcpy( out, tmp.p, bytes, cudaMemcpyDeviceToHost ) );
  return BVHG_OK;
}

bvhg_status bvhg_get_kdops(bvhg_ctx *ctx, int32_t obj, double *slabs)
{
  if ( ctx && ctx->cfg.precision != BVHG_PLAIN_FP64 ) return fail( ctx, BVHG_ERR_STATE, "FP64 slabs: FP64 form only" );
  return probe_kdops( ctx, obj, slabs, false );
}

bvhg_status bvhg_get_kdops_f32(bvhg_ctx *ctx, int32_t obj, float *slabs)
{
  if ( ctx && ctx->cfg.precision != BVHG_FILTER_FP32 ) return fail( ctx, BVHG_ERR_STATE, "FP32 slabs: FP32 form only" );
  return probe_kdops( ctx, obj, slabs, true );
}

bvhg_status bvhg_get_centroids(bvhg_ctx *ctx, int32_t obj, double *centroids)
{
  if ( !valid_obj( ctx, obj ) || !centroids ) return fail( ctx, BVHG_ERR_ARG, "invalid argument" );
  object &o = *ctx->objs[obj];
  if ( !o.built ) return fail( ctx, BVHG_ERR_STATE, "probe before build" );
  cudaSetDevice( ctx->cfg.device );
  join_object( ctx, o );
  BVHG_CUDA( ctx, cudaStreamSynchronize( ctx->stream ) );
  if ( o.n == 0 ) return BVHG_OK;
  std::vector< double > x( o.n ), y( o.n ), z( o.n );
  BVHG_CUDA( ctx, cudaMemcpy( x.data(), o.cx.p, o.n * 8, cudaMemcpyDeviceToHost ) );
  BVHG_CUDA( ctx, cudaMemcpy( y.data(), o.cy.p, o.n * 8, cudaMemcpyDeviceToHost ) );
  BVHG_CUDA( ctx, cudaMemcpy( z.data(), o.cz.p, o.n * 8, cudaMemcpyDeviceToHost ) );
  for ( uint64_t i = 0; i < o.n; ++i )
  {
    centroids[3 * i] = x[i];
    centroids[3 * i + 1] = y[i];
    centroids[3 * i + 2] = z[i];
  }
  return BVHG_OK;
}

bvhg_status bvhg_validate_tree(bvhg_ctx *ctx, int32_t obj, uint32_t *depth_out)
{
  if ( !valid_obj( ctx, obj ) ) return fail( ctx, BVHG_ERR_ARG, "invalid object" );
  object &o = *ctx->objs[obj];
  if ( !o.built ) return fail( ctx, BVHG_ERR_STATE, "validate before build" );
  cudaSetDevice( ctx->cfg.device );
  join_object( ctx, o );
  BVHG_CUDA( ctx, cudaStreamSynchronize( ctx->stream ) );
  if ( depth_out ) *depth_out = 0;
  const uint64_t n = o.n;
  if ( n == 0 ) return BVHG_OK;
  const int D = ctx->cfg.k / 2;
  const bool fp32 = ctx->cfg.precision == BVHG_FILTER_FP32;
  const size_t sb = fp32 ? 4 : 8;
  const uint64_t m = ( n + kLeafSize - 1 ) / kLeafSize;
  const uint64_t nw = ( n + 31 ) / 32;
  auto fetch = [&](const void *src, size_t count, std::vector< double > &dst) -> cudaError_t {
    dst.resize( count );
    if ( !count ) return cudaSuccess;
    if ( fp32 )
    {
      std::vector< float > f( count );
      cudaError_t e = cudaMemcpy( f.data(), src, count * 4, cudaMemcpyDeviceToHost );
      for ( size_t k = 0; k < count; ++k ) dst[k] = f[k];
      return e;
    }
    return cudaMemcpy( dst.data(), src, count * 8, cudaMemcpyDeviceToHost );
  };
  // element slabs recomputed from the vertices, original order
  dev_buf tmp;
  BVHG_CUDA( ctx, tmp.reserve( n * D * 2 * sb ) );
  BVHG_CUDA( ctx, launch_probe_kdops( ctx->cfg.k, fp32, o.verts, o.V, n, ctx->cfg.epsilon, tmp.p, ctx->stream ) );
  BVHG_CUDA( ctx, cudaStreamSynchronize( ctx->stream ) );
  std::vector< double > lb, nb, wb, bb, rootb;
  BVHG_CUDA( ctx, fetch( tmp.p, n * D * 2, lb ) );
  BVHG_CUDA( ctx, fetch( o.node_box.p, ( m - 1 ) * D * 4, nb ) );
  BVHG_CUDA( ctx, fetch( o.warp_box.p, nw * D * 2, wb ) );
  BVHG_CUDA( ctx, fetch( o.bucket_box.p, m * D * 2, bb ) );
  obj_scalars h;
  BVHG_CUDA( ctx, cudaMemcpy( &h, o.sc(), sizeof( h ), cudaMemcpyDeviceToHost ) );
  BVHG_CUDA( ctx, fetch( o.sc()->root_box, D * 2, rootb ) );
  std::vector< uint32_t > perm( n );
  BVHG_CUDA( ctx, cudaMemcpy( perm.data(), o.sorted_vals(), n * 4, cudaMemcpyDeviceToHost ) );
  // the elements' slabs in rank order (the build does not store them)
  std::vector< double > eb( n * D * 2 );
  for ( uint64_t r = 0; r < n; ++r )
  {
    if ( perm[r] >= n ) return fail( ctx, BVHG_ERR_STATE, "permutation entry out of range" );
    for ( int k = 0; k < 2 * D; ++k ) eb[r * D * 2 + k] = lb[static_cast< size_t >( perm[r] ) * D * 2 + k];
  }
  // union of ranks [lo, hi) into out (2 D values)
  auto unite = [&](uint64_t lo, uint64_t hi, std::vector< double > &out) {
    out.assign( 2 * D, 0.0 );
    for ( int a = 0; a < D; ++a )
    {
      double mn = eb[lo * D * 2 + 2 * a], mx = eb[lo * D * 2 + 2 * a + 1];
      for ( uint64_t r = lo + 1; r < hi; ++r )
      {
        mn = std::min( mn, eb[r * D * 2 + 2 * a] );
        mx = std::max( mx, eb[r * D * 2 + 2 * a + 1] );
      }
      out[2 * a] = mn;
      out[2 * a + 1] = mx;
    }
  };
  std::vector< double > u;
  for ( uint64_t w = 0; w < nw; ++w )
  {
    unite( 32 * w, std::min< uint64_t >( n, 32 * w + 32 ), u );
    for ( int k = 0; k < 2 * D; ++k )
      if ( wb[w * D * 2 + k] != u[k] ) return fail( ctx, BVHG_ERR_STATE, "query group box is not the union of its ranks" );
  }
  std::vector< std::vector< double > > bucket( m );
  for ( uint64_t b = 0; b < m; ++b )
  {
    unite( kLeafSize * b, std::min< uint64_t >( n, kLeafSize * b + kLeafSize ), bucket[b] );
    for ( int k = 0; k < 2 * D; ++k )
      if ( bb[b * D * 2 + k] != bucket[b][k] ) return fail( ctx, BVHG_ERR_STATE, "bucket box is not the union of its ranks" );
  }
  if ( m == 1 )
  {
    if ( h.root != ~0 ) return fail( ctx, BVHG_ERR_STATE, "bad root of a one-bucket tree" );
    for ( int k = 0; k < 2 * D; ++k )
      if ( rootb[k] != bucket[0][k] ) return fail( ctx, BVHG_ERR_STATE, "one-bucket root box differs" );
    if ( depth_out ) *depth_out = 1;
    return BVHG_OK;
  }
  std::vector< int2 > child( m - 1 );
  BVHG_CUDA( ctx, cudaMemcpy( child.data(), o.child.p, ( m - 1 ) * 8, cudaMemcpyDeviceToHost ) );
  if ( h.root < 0 || static_cast< uint64_t >( h.root ) >= m - 1 ) return fail( ctx, BVHG_ERR_STATE, "bad root" );
  for ( int a = 0; a < D; ++a )
  {
    const double *slot = &nb[static_cast< size_t >( h.root ) * D * 4];
    if ( rootb[2 * a] != std::min( slot[a * 4], slot[a * 4 + 2] ) ||
         rootb[2 * a + 1] != std::max( slot[a * 4 + 1], slot[a * 4 + 3] ) )
      return fail( ctx, BVHG_ERR_STATE, "root box is not the union of the root's children" );
  }
  std::vector< uint8_t > seen_leaf( m, 0 ), seen_node( m - 1, 0 );
  // (node, depth): every child's slot is the exact union of what it covers; buckets reached once
  std::vector< std::pair< int, uint32_t > > st{ { h.root, 1u } };
  uint32_t maxd = 0;
  uint64_t leaves = 0, nodes = 0;
  while ( !st.empty() )
  {
    auto [k, d] = st.back();
    st.pop_back();
    if ( seen_node[k] ) return fail( ctx, BVHG_ERR_STATE, "node reached twice" );
    seen_node[k] = 1;
    ++nodes;
    const int c[2] = { child[k].x, child[k].y };
    const double *slot = &nb[static_cast< size_t >( k ) * D * 4];
    for ( int side = 0; side < 2; ++side )
    {
      if ( c[side] < 0 )
      {
        const uint64_t bb = static_cast< uint64_t >( ~c[side] );
        if ( bb >= m || seen_leaf[bb] ) return fail( ctx, BVHG_ERR_STATE, "bucket missing or reached twice" );
        seen_leaf[bb] = 1;
        ++leaves;
        maxd = d + 1 > maxd ? d + 1 : maxd;
        for ( int a = 0; a < D; ++a )
          if ( slot[a * 4 + side * 2] != bucket[bb][2 * a] || slot[a * 4 + side * 2 + 1] != bucket[bb][2 * a + 1] )
            return fail( ctx, BVHG_ERR_STATE, "bucket slot differs from the union of its elements" );
      } else {
        if ( static_cast< uint64_t >( c[side] ) >= m - 1 ) return fail( ctx, BVHG_ERR_STATE, "bad child index" );
        const double *cs = &nb[static_cast< size_t >( c[side] ) * D * 4];
        for ( int a = 0; a < D; ++a )
          if ( slot[a * 4 + side * 2] != std::min( cs[a * 4], cs[a * 4 + 2] ) ||
               slot[a * 4 + side * 2 + 1] != std::max( cs[a * 4 + 1], cs[a * 4 + 3] ) )
            return fail( ctx, BVHG_ERR_STATE, "node slot is not the union of the child's children" );
        st.push_back( { c[side], d + 1 } );
      }
    }
  }
  if ( leaves != m || nodes != m - 1 ) return fail( ctx, BVHG_ERR_STATE, "tree does not cover every bucket once" );
  if ( depth_out ) *depth_out = maxd;
  return BVHG_OK;
}

bvhg_status bvhg_last_candidates(bvhg_ctx *ctx, uint64_t *candidates)
{
  if ( !ctx || !candidates ) return BVHG_ERR_ARG;
  *candidates = ctx->last_candidates;
  return BVHG_OK;
}

bvhg_status bvhg_get_stage_times(bvhg_ctx *ctx, double *ms, uint64_t *launches)
{
  if ( !ctx ) return BVHG_ERR_ARG;
  cudaSetDevice( ctx->cfg.device );
  collect_timing( ctx );
  for ( int s = 0; s < BVHG_NUM_STAGES; ++s )
  {
    if ( ms ) ms[s] = ctx->stage_ms[s];
    if ( launches ) launches[s] = ctx->stage_launches[s];
    ctx->stage_ms[s] = 0.0;
    ctx->stage_launches[s] = 0;
  }
  return BVHG_OK;
}

bvhg_status bvhg_launch_count(bvhg_ctx *ctx, uint64_t *launches)
{
  if ( !ctx || !launches ) return BVHG_ERR_ARG;
  *launches = ctx->launches;
  return BVHG_OK;
}

bvhg_status bvhg_set_spin_limit(bvhg_ctx *ctx, uint32_t limit)
{
  if ( !ctx ) return BVHG_ERR_ARG;
  ctx->spin_limit = limit ? limit : ( ctx->cfg.spin_limit ? ctx->cfg.spin_limit : kDefaultSpinLimit );
  return BVHG_OK;
}

bvhg_status bvhg_test_stall_sort(bvhg_ctx *ctx, int32_t enable)
{
  if ( !ctx ) return BVHG_ERR_ARG;
  ctx->stall_sort = enable ? 1 : 0;
  return BVHG_OK;
}

bvhg_status bvhg_test_batch_form(bvhg_ctx *ctx, uint32_t groups, uint32_t lanes)
{
  if ( !ctx || lanes == 0 || lanes > 64 || groups > 4096 ) return BVHG_ERR_ARG;
  if ( !ctx->batch ) ctx->batch = std::make_unique< batch_state >();
  ctx->batch->groups = static_cast< int >( groups );
  ctx->batch->lanes = static_cast< int >( lanes );
  return BVHG_OK;
}

bvhg_status bvhg_test_dense_stack(bvhg_ctx *ctx, int32_t limit)
{
  if ( !ctx || limit < 0 ) return BVHG_ERR_ARG;
  ctx->dense_stack = limit;
  return BVHG_OK;
}

bvhg_status bvhg_debug_normal(int32_t k, int32_t axis, int32_t comp, double *value, float *lo, float *hi)
{
  if ( ( k != 6 && k != 18 && k != 26 ) || axis < 0 || axis >= k / 2 || comp < 0 || comp > 2 ) return BVHG_ERR_ARG;
  double v = 0.0;
  float l = 0.f, h = 0.f;
  if ( k == 6 )
  {
    v = normal_comp< 6 >( axis, comp );
    l = normal_lo< 6 >( axis, comp );
    h = normal_hi< 6 >( axis, comp );
  } else if ( k == 18 ) {
    v = normal_comp< 18 >( axis, comp );
    l = normal_lo< 18 >( axis, comp );
    h = normal_hi< 18 >( axis, comp );
  } else {
    v = normal_comp< 26 >( axis, comp );
    l = normal_lo< 26 >( axis, comp );
    h = normal_hi< 26 >( axis, comp );
  }
  if ( value ) *value = v;
  if ( lo ) *lo = l;
  if ( hi ) *hi = h;
  return BVHG_OK;
}

bvhg_status bvhg_synchronize(bvhg_ctx *ctx)
{
  if ( !ctx ) return BVHG_ERR_ARG;
  cudaSetDevice( ctx->cfg.device );
  for ( auto &o : ctx->objs )
    if ( o ) join_object( ctx, *o );
  BVHG_CUDA( ctx, cudaStreamSynchronize( ctx->stream ) );
  for ( auto &o : ctx->objs )
    if ( o && o->built && o->n > 0 )
    {
      bvhg_status st = check_scalar_errors( ctx, *o );
      if ( st != BVHG_OK ) return st;
    }
  return BVHG_OK;
}

const char *bvhg_last_error(const bvhg_ctx *ctx)
{
  if ( !ctx ) return "null context";
  return ctx->err.c_str();
}

const char *bvhg_status_string(bvhg_status status)
{
  switch ( status )
  {
    case BVHG_OK: return "ok";
    case BVHG_ERR_ARG: return "invalid argument";
    case BVHG_ERR_CUDA: return "CUDA error";
    case BVHG_ERR_OVERFLOW: return "pair buffer overflow";
    case BVHG_ERR_TIMEOUT: return "device wait timed out";
    case BVHG_ERR_STATE: return "invalid state";
    case BVHG_ERR_NOMEM: return "out of device memory";
  }
  return "unknown status";
}

}  // extern "C"
