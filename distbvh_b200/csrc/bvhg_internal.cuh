// bvhg_internal.cuh — device data layout shared by the kernels and the C ABI implementation.
//
// Per object of n elements with V vertices each and D = K/2 slabs (T = double in the FP64 form, float in the
// FP32 form), all in HBM. The tree's leaves are buckets of kLeafSize consecutive Morton ranks (m = ceil(n /
// kLeafSize) buckets, m - 1 internal nodes); the pair set does not depend on the tree shape.
//   verts      n * V * 3 doubles, element-major (input, owned copy or borrowed device pointer)
//   cx, cy, cz n doubles each: centroids, structure of arrays (coalesced write in K1, read in K2)
//   keys/vals  n u64 Morton keys and n u32 element indices, ping-ponged by the radix passes; after the sort
//              keys[r], vals[r] hold the key and original index of rank r (vals = the permutation)
//   warp_box   ceil(n / 32) * D * 2 T: union of the slabs of ranks [32 w, 32 w + 31] (the query side's cull)
//   bucket_box m * D * 2 T: union of the slabs of leaf bucket b (ranks [8 b, 8 b + 7]), input of the tree build
//   elem_cache n * D * 2 T: element slabs in rank order, written by the slab kernel for objects in dense contact
//              only (sparse traversals compute the few they test from the vertices)
//   node_box   (m - 1) * D * 2 * 2 T: both children's slabs of internal node k, [k][a][child][min,max], so one
//              32-byte (FP64) or 16-byte (FP32) sector per axis tests both children
//   child      (m - 1) int2: child index, >= 0 internal node, < 0 bucket with ~child = bucket index
//   range      (m - 1) int2: [first bucket, last bucket] covered by the node (self-collision pruning)
//   parent     m + (m - 1) int32: parent * 2 + side of every bucket and internal node (refit)
//   exch       m - 1 int32: the agglomerative build's exchange slot per internal node (-1 = empty)
//   bdel       m - 1 u8: dissimilarity of every bucket boundary (written by the block-local build for the climb)
//   queue      m int4: subtrees the block-local build phases leave to the global phase
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "batch.cuh"

namespace bvhg {

// Device-side scalars of one object (one allocation, read back for probes).
struct obj_scalars
{
  unsigned long long bounds_enc[6];  // order-preserving encodings: min x,y,z then max x,y,z of cardinal slabs
  double min3[3];                    // Morton bounds min (contact_entity.hpp:136-148)
  double inv3[3];                    // 1 / (max - min)
  int root;                          // root internal node, or ~elem when n == 1
  int error;                         // bvhg_status raised by a kernel (first one wins)
  unsigned int climb_count;          // subtrees queued for the global phase of the tree build
  unsigned int long_runs;            // runs of equal high key halves listed by the fix-up for the run sort
  alignas( 16 ) unsigned char root_box[26 * 8];  // the root's slabs, D (min, max) pairs of the slab type
  unsigned int sort_tile_counter[64];// tile dispenser per radix pass
};

// Candidate/pair accumulators of one broadphase.
struct pair_scalars
{
  unsigned long long count;   // pairs found (may exceed capacity)
  unsigned long long count2;  // pairs surviving the FP64 recheck
  int error;
  unsigned packet_next;       // the traversal's dispenser of packet chunks
};

constexpr int kLeafSize = 8;  // elements per tree leaf (consecutive Morton ranks)

constexpr int kErrArg = 1;
constexpr int kErrTimeout = 4;
constexpr int kErrOverflowStack = 7;

__host__ __device__ inline unsigned long long ord_encode(double x)
{
  unsigned long long b;
#ifdef __CUDA_ARCH__
  b = static_cast< unsigned long long >( __double_as_longlong( x ) );
#else
  __builtin_memcpy( &b, &x, 8 );
#endif
  return ( b & 0x8000000000000000ull ) ? ~b : ( b | 0x8000000000000000ull );
}

__host__ __device__ inline double ord_decode(unsigned long long e)
{
  const unsigned long long b = ( e & 0x8000000000000000ull ) ? ( e & 0x7fffffffffffffffull ) : ~e;
  double x;
#ifdef __CUDA_ARCH__
  x = __longlong_as_double( static_cast< long long >( b ) );
#else
  __builtin_memcpy( &x, &b, 8 );
#endif
  return x;
}

// Radix sort geometry: 63 significant key bits (morton64 never sets bit 63, hash.hpp:100-103).
constexpr int kKeyBits = 63;
constexpr int kSortThreads = 512;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;
inline int sort_passes(int bits) { return ( kKeyBits + bits - 1 ) / bits; }

// ---- kernel arguments: every pipeline kernel is a body over one of these structs, launched per object or, for
// a batch, for many objects at once (batch.cuh) ----

struct init_args  // reset state of a rebuild
{
  obj_scalars *sc;
  uint32_t *hist;
  uint64_t hist_words;
  uint32_t *status;
  uint64_t status_words;
  int *exch;
  uint64_t exch_words;
};

struct cb_args  // K1: centroids and Morton bounds
{
  const double *verts;
  uint32_t V;
  uint64_t n;
  double eps;
  double *cx, *cy, *cz;
  obj_scalars *sc;
  uint32_t spin_limit;
};

struct kh_args  // K2: Morton keys and digit histograms
{
  const double *cx, *cy, *cz;
  uint64_t n;
  obj_scalars *sc;
  uint64_t *keys;
  uint32_t *hist;
};

struct sort_pass_args  // one radix pass of one object
{
  const uint64_t *keys_in;
  const uint32_t *vals_in;  // NULL: the element index
  uint64_t *keys_out;
  uint32_t *vals_out;
  uint64_t n;
  int pass;
  const uint32_t *hist;     // this pass's digit histogram
  uint32_t *status;         // this pass's look-back words
  obj_scalars *sc;
  uint32_t spin_limit;
  int stall;
  int use_tma;
};

struct fixup_args  // the low-half fix-up and the sort of the long runs it lists
{
  const uint64_t *keys_in;
  const uint32_t *vals_in;
  uint64_t *keys_out;
  uint32_t *vals_out;
  uint64_t n;
  uint32_t *runs;  // long_run_capacity(n) first elements of long runs
  obj_scalars *sc;
};

struct slabs_args  // element slabs, leaf-bucket and query-group boxes
{
  const double *verts;
  uint32_t V;
  uint64_t n;
  double eps;
  float eps_hi;
  const uint32_t *vals;
  void *bucket_box;
  void *warp_box;
  void *elem_rows;  // NULL: not stored
  obj_scalars *sc;
};

struct tree_args  // the block-local build, the climb and the refit of one object's tree
{
  uint64_t n;
  const uint64_t *keys;
  uint8_t *bdel;
  const void *bucket_box;
  void *node_box;
  int2 *child;
  int2 *range;
  int *parent;
  int *exch;
  int4 *queue;
  obj_scalars *sc;
};

// ---- launch wrappers (one per kernel family), implemented in the k_*.cu files ----
// All return cudaGetLastError() of the launch.

cudaError_t launch_centroid_bounds(int K, const double *verts, uint32_t V, uint64_t n, double eps, double *cx,
                                   double *cy, double *cz, obj_scalars *sc, uint32_t spin_limit, cudaStream_t s);

cudaError_t launch_keys_hist(int bits, const double *cx, const double *cy, const double *cz, uint64_t n,
                             obj_scalars *sc, uint64_t *keys, uint32_t *hist, cudaStream_t s);

// Batched forms (items: the per-object argument structs, blocks per item from the *_blocks functions).
uint32_t obj_init_blocks(const init_args &a);
cudaError_t launch_obj_init_batch(const batch_launch &b, cudaStream_t s);
// tma: every item's vertices 16-byte aligned and V in {3, 4, 8} (then the bulk-copy form), else the plain form.
cudaError_t centroid_bounds_blocks(int K, uint32_t V, uint64_t n, bool tma, uint32_t *blocks);
cudaError_t launch_centroid_bounds_batch(int K, uint32_t V, bool tma, const batch_launch &b, cudaStream_t s);
uint32_t keys_hist_blocks(uint64_t n);
cudaError_t launch_keys_hist_batch(int bits, const batch_launch &b, cudaStream_t s);

// Stable sort of each run of equal high key halves by the low half (in -> out), after the passes over bits 32..62:
// the fix-up ranks runs of up to 32 elements in place and lists longer ones (runs[], count in sc->long_runs), which
// a second small launch sorts with the input arrays as scratch (nothing else reads them afterwards).
cudaError_t launch_sort_fixup(const uint64_t *keys_in, const uint32_t *vals_in, uint64_t *keys_out,
                              uint32_t *vals_out, uint64_t n, uint32_t *runs, obj_scalars *sc, cudaStream_t s);
inline uint64_t long_run_capacity(uint64_t n) { return n / 33 + 1; }

// ---- patches (k_cluster.cu) ----
struct cluster_scalars
{
  unsigned int runs;    // equal-hash runs listed for k_cluster_runs
  unsigned int t;       // threshold split depth
  unsigned int need;    // positions of depth t taken
  unsigned int groups;  // non-empty patch pairs of the last grouping
};

// Arguments of the Morton clustering of one object (src/bvh/split/cluster.hpp:89-179) from its build's sorted keys.
struct cluster_launch
{
  const uint64_t *keys;  // n sorted Morton keys (the build's)
  const uint32_t *perm;  // n element indices in key order (the build's)
  uint64_t n;
  uint32_t patches;      // od_factor >= 1
  uint32_t *order;       // n: element indices in patch order (stable by the 32-bit hash)
  uint32_t *rank;        // n: position of every element in the patch order
  uint32_t *tmp;         // n: scratch of the long-run sort
  uint32_t *runs;        // n / 33 + 1: long equal-hash runs
  uint32_t *bhist;       // cluster_block_count(n) * 33: per-block depth histograms
  uint32_t *bbase;       // cluster_block_count(n) * 2
  uint32_t *splits;      // max(patches - 1, 1)
  uint64_t *bounds;      // patches + 1: patch p = positions [bounds[p], bounds[p + 1])
  cluster_scalars *cs;
  cudaStream_t s;
};
size_t cluster_block_count(uint64_t n);
cudaError_t launch_cluster(const cluster_launch &x);

// Patch boxes of a clustered object: out[(p * K/2 + a) * 2 + {0 min, 1 max}] = the union of the FP64 slabs of patch
// p's elements (+inf / -inf for an empty patch); enc: patches * K words of scratch.
cudaError_t launch_patch_kdops(int K, const double *verts, uint32_t V, uint64_t n, double eps, const uint32_t *order,
                               const uint64_t *bounds, uint32_t patches, unsigned long long *enc, double *out,
                               cudaStream_t s);

// Two clustered objects: element pairs (local indices) grouped by patch pair.
struct group_launch
{
  const uint64_t *bounds_a, *bounds_b;
  const uint32_t *rank_a, *rank_b;
  uint32_t patches_a, patches_b;
};
// pairs: np (a, b) local index pairs. bin_count, bin_off: patches_a * patches_b words each. groups: rows (patch a,
// patch b, first pair, pair count) of the non-empty patch pairs in (a, b) order, at most group_cap (their number in
// cs->groups). out: np (index in patch a, index in patch b) pairs grouped by patch pair.
cudaError_t launch_group_pairs(const uint2 *pairs, uint64_t np, const group_launch &g, uint32_t *bin_count,
                               uint32_t *bin_off, uint32_t *groups, uint64_t group_cap, uint32_t *out,
                               cluster_scalars *cs, cudaStream_t s);

// Passes of the sort that build() runs: those whose digit lies in the high key half (the fix-up sorts the rest).
inline int sort_first_pass(int bits) { return 32 / bits; }

// Reset state of a rebuild in one launch (scalars, histograms, look-back words, climb exchange slots).
cudaError_t launch_obj_init(obj_scalars *sc, uint32_t *hist, uint64_t hist_words, uint32_t *status,
                            uint64_t status_words, int *exch, uint64_t exch_words, cudaStream_t s);

// Sort-and-sweep between two objects (k_sweep.cu): the arguments of its three phases.
struct sweep_launch
{
  int K;
  const double *averts, *bverts;
  uint32_t aV, bV;
  uint64_t na, nb;
  double eps;
  const double *acx, *acy, *acz, *bcx, *bcy, *bcz;  // centroids (axis choice)
  const obj_scalars *asc, *bsc;                     // K1 bounds of both objects (global range)
  double *partial;                                  // sweep_partial_bytes()
  void *params;                                     // sweep_params_bytes()
  double *rows;                                     // nb * K doubles: B's element slabs, original order
  uint64_t *keys;                                   // nb: B's u32 keys, original order
  uint32_t *hist;                                   // 4 * 256: byte histograms of the keys
  const uint64_t *skeys;                            // sorted keys
  const uint32_t *svals;                            // B's element indices in key order
  double *srows;                                    // nb * K doubles: B's slab rows in key order
  double *sbmax;                                    // nb: B's scaled maxima on the axis in key order
  const uint32_t *aperm;                            // A's elements in Morton order (its build's permutation)
  const obj_scalars *sc;                            // scalars of the keys' sort (error word)
  uint2 *pairs;
  uint64_t cap;
  pair_scalars *ps;
  cudaStream_t s;
};
size_t sweep_params_bytes();
size_t sweep_partial_bytes();
int sweep_axis_read(const void *params_host_copy);
// The axis (axis < 0: the one of largest centroid variance) and its scale factor, from the objects' bounds.
cudaError_t launch_sweep_setup(const sweep_launch &x, int axis);
// B's slab rows, keys, byte histograms and the key window width.
cudaError_t launch_sweep_keys(const sweep_launch &x);
// A's sweeps over the sorted keys; pairs (index into A, index into B) counted in ps->count.
cudaError_t launch_sweep(const sweep_launch &x);

cudaError_t launch_onesweep(int bits, const uint64_t *keys_in, const uint32_t *vals_in, uint64_t *keys_out,
                            uint32_t *vals_out, uint64_t n, int pass, const uint32_t *hist, uint32_t *status,
                            obj_scalars *sc, uint32_t spin_limit, int stall, cudaStream_t s);
// Batched: the argument struct of one object's pass (hist and status offset to the pass), and its blocks.
sort_pass_args onesweep_args(int bits, const uint64_t *keys_in, const uint32_t *vals_in, uint64_t *keys_out,
                             uint32_t *vals_out, uint64_t n, int pass, const uint32_t *hist, uint32_t *status,
                             obj_scalars *sc, uint32_t spin_limit, int stall);
uint32_t onesweep_blocks(uint64_t n);
cudaError_t launch_onesweep_batch(int bits, const batch_launch &b, cudaStream_t s);
uint32_t sort_fixup_blocks(uint64_t n);
uint32_t sort_runs_blocks(uint64_t n);  // 0: no launch (no run can be long)
cudaError_t launch_sort_fixup_batch(const batch_launch &b, cudaStream_t s);
cudaError_t launch_sort_runs_batch(const batch_launch &b, cudaStream_t s);

// Element slabs + agglomerative LBVH build over leaf buckets with bottom-up refit (FP64 or FP32 slabs): the
// block-local phase, which queues unfinished subtrees for launch_climb.
// Element slabs in rank order (stored to elem_rows when given, for objects in dense contact), the union of each leaf
// bucket (bucket_box, m rows) and of each group of 32 ranks (warp_box); a one-bucket object's root. Marks a failed
// sort when perm is not a permutation.
cudaError_t launch_slabs(int K, bool fp32, const double *verts, uint32_t V, uint64_t n, double eps,
                         const uint32_t *vals, void *bucket_box, void *warp_box, void *elem_rows,
                         obj_scalars *sc, cudaStream_t s);

// Block-local LBVH build over the bucket boxes (nodes closed inside a block of 128 buckets; the rest queued for
// launch_climb). Nothing to do for one bucket.
// bdel (m - 1 bytes) receives the dissimilarity of every bucket boundary for the climb.
cudaError_t launch_build(int K, bool fp32, uint64_t n, const uint64_t *keys, uint8_t *bdel, const void *bucket_box,
                         void *node_box, int2 *child, int2 *range, int *parent, int4 *queue, obj_scalars *sc,
                         cudaStream_t s);

// Global climb of the build (subtrees the block-local phase queued); after launch_build, only when m > 1.
cudaError_t launch_climb(int K, bool fp32, uint64_t n, const uint8_t *bdel, void *node_box, int2 *child, int2 *range,
                         int *parent, int *exch, const int4 *queue, obj_scalars *sc, cudaStream_t s);

// Batched forms of the slab kernel (items: slabs_args; one V for all items), the block-local build, the climb and
// the refit (items: tree_args of objects with more than one bucket), with the blocks of one item.
uint32_t slabs_blocks(uint64_t n);
cudaError_t launch_slabs_batch(int K, bool fp32, uint32_t V, const batch_launch &b, cudaStream_t s);
uint32_t build_blocks(uint64_t n);
cudaError_t launch_build_batch(int K, bool fp32, const batch_launch &b, cudaStream_t s);
uint32_t climb_blocks(uint64_t n);
cudaError_t launch_climb_batch(int K, bool fp32, const batch_launch &b, cudaStream_t s);
uint32_t refit_blocks(uint64_t n);
cudaError_t launch_refit_batch(int K, bool fp32, const batch_launch &b, cudaStream_t s);

// Refit with the topology of the last build, after launch_slabs recomputed the bucket boxes: every internal node.
// Nodes inside one block's 128 buckets are refit in shared memory; the nodes whose ranges cross blocks by climbs with
// the global exchange (exch must hold -1).
cudaError_t launch_refit(int K, bool fp32, uint64_t n, const void *bucket_box, void *node_box, const int2 *child,
                         const int2 *range, const int *parent, int *exch, obj_scalars *sc, cudaStream_t s);

struct tree_view
{
  const void *node_box;
  const int2 *child;
  const int2 *range;
  const void *warp_box;
  const double *verts;  // element vertices, [element][vertex][xyz] (element slabs are recomputed from them)
  uint32_t V;
  const void *elem_cache;  // element slabs in rank order (valid when stored)
  bool stored;             // the slab kernel wrote every element's slabs to elem_cache
  const uint32_t *perm;
  uint64_t n;
  const obj_scalars *sc;
};

// The traversal of one scene (query object q against target tree t) as kernel arguments: the pointer members that
// hold slabs point to FP64 or FP32 values per the context's form.
struct trav_item
{
  const void *qwarp;
  const double *qverts;
  uint32_t qV;
  const void *qrows;
  const uint32_t *qperm;
  uint32_t nq;
  const int2 *child;
  const void *nbox;
  const int2 *range;
  const double *tverts;
  uint32_t tV;
  const void *tcache;
  const uint32_t *tperm;
  const obj_scalars *tsc;
  uint32_t nt;
  int self;
  double eps;
  float eps_hi;
  uint2 *pairs;
  uint64_t cap;
  pair_scalars *ps;
  int dense_stack;
  const obj_scalars *qsc;
};

// One scene's traversal for a batched launch: its item, its blocks and whether it takes the dense walk (the batch
// launches the dense and the other scenes separately).
void traverse_item(int K, bool fp32, tree_view q, tree_view t, bool self, bool dense, double eps, uint2 *pairs,
                   uint64_t cap, pair_scalars *ps, int dense_stack_limit, trav_item *item, uint32_t *blocks,
                   bool *dense_out);
// V: the vertex count of every query and target object of the items (0: mixed).
cudaError_t launch_traverse_batch(int K, bool fp32, bool dense, uint32_t V, const batch_launch &b, cudaStream_t s);

struct recheck_args
{
  const double *va;
  uint32_t Va;
  const double *vb;
  uint32_t Vb;
  double eps;
  const uint2 *cand;
  uint64_t cand_cap;
  uint2 *out;
  uint64_t cap;
  pair_scalars *ps;
};
uint32_t recheck_blocks(uint64_t ncand);
cudaError_t launch_recheck_batch(int K, uint32_t V, const batch_launch &b, cudaStream_t s);

struct gid_args
{
  const uint2 *pairs;
  const unsigned long long *count;
  uint64_t cap;
  const uint64_t *gid_a;
  const uint64_t *gid_b;
  int normalize;
  uint64_t *out;
};
uint32_t gid_pairs_dev_blocks(uint64_t cap);
cudaError_t launch_gid_pairs_dev_batch(const batch_launch &b, cudaStream_t s);

// Queries every leaf of q against tree t; writes (q element, t element) local index pairs. dense (both objects'
// element slabs stored): the walk that pops nodes in batches and tests leaves in batches; its deeper stack bound can
// be reached (ps->error = kErrOverflowStack), and the single-node walk (dense = false) then always completes.
// dense_stack_limit > 0 lowers that bound (test hook); 0 keeps it.
cudaError_t launch_traverse(int K, bool fp32, tree_view q, tree_view t, bool self, bool dense, double eps, uint2 *pairs,
                            uint64_t cap, pair_scalars *ps, cudaStream_t s, int dense_stack_limit = 0);

// FP64 recheck of FP32 candidates: keeps (a, b) iff the FP64 slabs of a and b overlap, compacted into out.
// The candidate count is min(ps->count, cand_cap), read on the device.
cudaError_t launch_recheck(int K, const double *verts_a, uint32_t Va, const double *verts_b, uint32_t Vb,
                           double eps, const uint2 *cand, uint64_t cand_cap, uint2 *out, uint64_t cap,
                           pair_scalars *ps, cudaStream_t s);

// Writes pairs as global ids: out[2p] = gid_a[a] (or a), out[2p + 1] = gid_b[b] (or b); normalize orders each
// pair by local index first (self-collision).
// Global-id mapping with the pair count read on the device (at most cap); for graph-captured batches.
cudaError_t launch_gid_pairs_dev(const uint2 *pairs, const unsigned long long *count, uint64_t cap,
                                 const uint64_t *gid_a, const uint64_t *gid_b, bool normalize, uint64_t *out,
                                 cudaStream_t s);

// dst[i] = *src[i] for i < n (src: device array of device pointers).
cudaError_t launch_gather_words(const int *const *src, int n, int *dst, cudaStream_t s);

cudaError_t launch_gid_pairs(const uint2 *pairs, uint64_t count, const uint64_t *gid_a, const uint64_t *gid_b,
                             bool normalize, uint64_t *out, cudaStream_t s);

// Original-order probes.
cudaError_t launch_probe_kdops(int K, bool fp32, const double *verts, uint32_t V, uint64_t n, double eps,
                               void *out, cudaStream_t s);

}  // namespace bvhg
