/*
 * bvhg.h — C ABI of the B200-native per-rank element broadphase (libbvhg.so).
 *
 * The reference (sandialabs/distBVH) has no C ABI: its boundary is the C++ template API of collision_world /
 * collision_object. Each entry point below replaces one step of that API for the element-level hot path:
 *
 *   bvhg_set_elements   <- collision_object::set_entity_data(Kokkos::View<const T*>, split_algorithm)
 *                          (src/bvh/collision_object.hpp:69-84) together with the element k-DOP the application
 *                          builds with kdop_base::from_vertices (src/bvh/kdop.hpp:238-264) and the element
 *                          centroid it reports through element_traits (src/bvh/traits.hpp:53-135).
 *   bvhg_build          <- collision_object::init_broadphase() (src/bvh/collision_object.cpp:148) plus the
 *                          Morton clustering inside set_entity_data_clustering (src/bvh/collision_object.hpp:89-131:
 *                          compute_bounds contact_entity.hpp:136-148, morton contact_entity.hpp:104-118,
 *                          radix_sorter util/sort.hpp:75-144) and the tree build (src/bvh/tree_build.hpp:103-185).
 *   bvhg_broadphase     <- collision_object::broadphase(collision_object&) (src/bvh/collision_object.cpp:248) at
 *                          element granularity, i.e. potential_collision_set (src/bvh/collision_query.hpp:370-379).
 *   bvhg_self_collision <- self_collision_set (src/bvh/collision_query.hpp:331-368).
 *   bvhg_sort_and_sweep <- sort_and_sweep_local with max_variant_axis (src/bvh/narrowphase/kokkos.hpp:125-248),
 *                          the two objects as the two patches.
 *   bvhg_get_morton     <- the Morton keys and permutation of morton_cluster (src/bvh/split/cluster.hpp:89-179) /
 *                          morton (src/bvh/contact_entity.hpp:175-191); a parity probe.
 *   bvhg_get_kdops      <- entity_snapshot::kdop() (src/bvh/snapshot.hpp:68-125); a parity probe.
 *
 * Pair-set contract: for objects A and B, (gid(a), gid(b)) is reported iff for every slab k < K/2
 * a.min_k < b.max_k and b.min_k < a.max_k (src/bvh/kdop.hpp:120-125, 538-549), with the slabs computed in FP64
 * exactly as kdop_base::from_vertices computes them, inflated by config.epsilon. Pairs are unordered as a set.
 *
 * Conventions.
 *   - All calls are ordered on the context's CUDA stream; a context is not thread-safe (one per host thread).
 *   - Device memory is owned by the library. Host input buffers are copied in stream order and must stay valid
 *     until the next call that returns a count or until bvhg_synchronize. Device input pointers are borrowed
 *     until the next bvhg_set_elements on that object or bvhg_object_destroy (the reference borrows its element
 *     view the same way, src/bvh/collision_object.cpp:128-129).
 *   - No exception crosses the ABI. Every call returns a bvhg_status; bvhg_last_error gives the message.
 *   - BVHG_ERR_OVERFLOW from bvhg_broadphase: *count holds the required capacity; pairs holds an arbitrary
 *     subset of `capacity` pairs. Retry with a larger buffer.
 *   - BVHG_ERR_TIMEOUT: a bounded device-side wait (radix-sort look-back) gave up; results are invalid and the
 *     context stays usable.
 */
#ifndef BVHG_H
#define BVHG_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define BVHG_API __attribute__((visibility("default")))
#else
#define BVHG_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum bvhg_status
{
  BVHG_OK = 0,
  BVHG_ERR_ARG = 1,       /* invalid argument (K, sizes, null pointers, non-finite vertex coordinates) */
  BVHG_ERR_CUDA = 2,      /* a CUDA runtime call failed */
  BVHG_ERR_OVERFLOW = 3,  /* pair buffer too small; *count = required */
  BVHG_ERR_TIMEOUT = 4,   /* a bounded device spin hit its limit */
  BVHG_ERR_STATE = 5,     /* call out of order (e.g. broadphase before build) */
  BVHG_ERR_NOMEM = 6      /* device allocation failed */
} bvhg_status;

typedef enum bvhg_precision
{
  BVHG_PLAIN_FP64 = 0,  /* FP64 slabs end to end */
  BVHG_FILTER_FP32 = 1  /* FP32 outward-rounded slabs for the tree, FP64 recheck of every candidate pair */
} bvhg_precision;

typedef enum bvhg_mem
{
  BVHG_MEM_HOST = 0,
  BVHG_MEM_DEVICE = 1
} bvhg_mem;

typedef enum bvhg_build_mode
{
  BVHG_REBUILD = 0,  /* bounds, Morton keys, radix sort, LBVH build and refit */
  BVHG_REFIT = 1     /* keep the tree topology of the last rebuild, recompute every node's slabs */
} bvhg_build_mode;

#define BVHG_FLAG_STAGE_TIMING 0x1u  /* record CUDA events around each stage (bvhg_get_stage_times) */

typedef struct bvhg_config
{
  int32_t k;               /* 6, 18 or 26 */
  int32_t precision;       /* bvhg_precision */
  int32_t sort_digit_bits; /* radix digit width: 1 (one bit per pass, as util/sort.hpp), 2, 4 or 8 */
  int32_t device;          /* CUDA device ordinal */
  double epsilon;          /* every slab is inflated by epsilon: (proj - eps, proj + eps), kdop.hpp:252-259 */
  void *stream;            /* cudaStream_t to run on; NULL = a stream the context creates and owns */
  uint32_t spin_limit;     /* iteration limit of every device-side wait; 0 = default */
  uint32_t flags;          /* BVHG_FLAG_* */
} bvhg_config;

typedef struct bvhg_ctx bvhg_ctx;

/* Stage indices of bvhg_get_stage_times. */
enum
{
  BVHG_STAGE_BOUNDS = 0,     /* centroids + Morton bounds */
  BVHG_STAGE_KEYS = 1,       /* Morton keys + digit histograms */
  BVHG_STAGE_SORT = 2,       /* radix passes over the high key half */
  BVHG_STAGE_BUILD = 3,      /* block-local LBVH build and node boxes over the buckets (or the refit climb) */
  BVHG_STAGE_TRAVERSE = 4,   /* tree traversal (candidate pairs) */
  BVHG_STAGE_RECHECK = 5,    /* FP64 recheck of FP32 candidates */
  BVHG_STAGE_OUTPUT = 6,     /* gid mapping + output copy */
  BVHG_STAGE_CLIMB = 7,      /* global climb of the LBVH build (subtrees left open by the block-local phase) */
  BVHG_STAGE_SLABS = 8,      /* element slabs in Morton rank order, leaf-bucket and query-group boxes */
  BVHG_STAGE_FIXUP = 9,      /* stable order of each run of equal high key halves by the low half */
  BVHG_NUM_STAGES = 10
};

BVHG_API void bvhg_config_default(bvhg_config *cfg);

BVHG_API bvhg_status bvhg_create(bvhg_ctx **ctx, const bvhg_config *cfg);
BVHG_API bvhg_status bvhg_destroy(bvhg_ctx *ctx);

/* collision_world::create_collision_object (src/bvh/collision_world.cpp:76-84). */
BVHG_API bvhg_status bvhg_object_create(bvhg_ctx *ctx, int32_t *obj);
BVHG_API bvhg_status bvhg_object_destroy(bvhg_ctx *ctx, int32_t obj);

/* Element data: n elements of verts_per_elem vertices (3 triangle, 4 tetrahedron, 8 hexahedron, any 1..32),
 * xyz[(i * verts_per_elem + v) * 3 + c]. gid may be NULL (gid = local index). mem = bvhg_mem of xyz and gid. */
BVHG_API bvhg_status bvhg_set_elements(bvhg_ctx *ctx, int32_t obj, const double *xyz, uint32_t verts_per_elem,
                              const uint64_t *gid, uint64_t n, int32_t mem);

BVHG_API bvhg_status bvhg_build(bvhg_ctx *ctx, int32_t obj, int32_t mode);

/* Inter-object pairs: pairs[2p] = gid in obj_a, pairs[2p + 1] = gid in obj_b. mem = bvhg_mem of pairs.
 * Blocks until the count is known. */
BVHG_API bvhg_status bvhg_broadphase(bvhg_ctx *ctx, int32_t obj_a, int32_t obj_b, uint64_t *pairs, uint64_t capacity,
                            uint64_t *count, int32_t mem);

/* Intra-object pairs with pairs[2p] < pairs[2p + 1] in local index order, reported as gids. */
BVHG_API bvhg_status bvhg_self_collision(bvhg_ctx *ctx, int32_t obj, uint64_t *pairs, uint64_t capacity, uint64_t *count,
                                int32_t mem);

/* Sort-and-sweep between two built objects (sort_and_sweep_local, src/bvh/narrowphase/kokkos.hpp:164-248): B's
 * slab minima on one cardinal axis become u32 keys over the union of both objects' extents there, a stable sort
 * orders them, and every element of A sweeps B in key order, emitting the elements that overlap it strictly on
 * every slab. axis = 0, 1 or 2, or -1 for the axis of largest centroid variance over both objects
 * (max_variant_axis, kokkos.hpp:125-160); *axis_used (may be NULL) receives the axis swept. The pair set is the
 * exact S(A, B), the same as bvhg_broadphase's, for any axis (pairs as there: gid in obj_a, gid in obj_b); its
 * cost grows with the elements of B whose extents on the axis meet each element of A, so it suits patch-sized
 * objects. FP64 slabs in both precision forms. obj_a != obj_b. Both objects must have been rebuilt (BVHG_REBUILD)
 * since their last bvhg_set_elements: the range and the axis come from a rebuild's bounds and centroids, which a
 * refit does not recompute (BVHG_ERR_STATE otherwise). Blocks until the count is known. */
BVHG_API bvhg_status bvhg_sort_and_sweep(bvhg_ctx *ctx, int32_t obj_a, int32_t obj_b, int32_t axis, uint64_t *pairs,
                                         uint64_t capacity, uint64_t *count, int32_t *axis_used, int32_t mem);

/* Batching form (no single counterpart in the reference: it runs many broadphase(other) calls of
 * src/bvh/collision_object.cpp:248 at once). Scene s pairs objects obj_a[s] and obj_b[s] (obj_a[s] == obj_b[s]: that
 * object's self-collision); objects already hold their elements (bvhg_set_elements) and may appear in several
 * scenes. Every object in the batch is built once (mode: BVHG_REBUILD, or BVHG_REFIT after a rebuild) and every
 * scene traversed, as one CUDA graph with no host round trip between scenes. When every object has the same vertex
 * count the graph is the fused form: the objects are split into groups, and each group runs each pipeline stage of
 * all its objects as one launch, then the traversal of its scenes as one launch, groups on concurrent streams;
 * otherwise per-object launches spread over concurrent streams. The graph is captured on the first call for a batch
 * layout (objects, element counts, vertex pointers, per-scene capacities) and replayed while the layout stays the
 * same, so a time-stepped loop that updates coordinates in place replays it. counts[s] (host, required) receives
 * scene s's exact pair count; the pairs go to `pairs` (mem) scene after scene, (gid_a, gid_b) like bvhg_broadphase,
 * scene s starting at pair offsets[s] (offsets may be NULL). BVHG_ERR_OVERFLOW when the total exceeds capacity
 * (counts are then still valid). Objects built by a batch are built as by bvhg_build. */
BVHG_API bvhg_status bvhg_batch_broadphase(bvhg_ctx *ctx, uint32_t nscenes, const int32_t *obj_a,
                                          const int32_t *obj_b, int32_t mode, uint64_t *pairs, uint64_t capacity,
                                          uint64_t *counts, uint64_t *offsets, int32_t mem);
/* Autotuner of the batching form: times the batch's graph in the fused form with 1, 4, 16, 64 and 256 groups of
 * objects (the batch's tile: groups whose working sets stay in L2 between stages) and in the per-object form with 16
 * and 64 streams, and keeps the fastest for later bvhg_batch_broadphase calls on this context. groups (0 = the
 * per-object form), lanes (streams) and ms (may be NULL) receive the choice and its time per batch. */
BVHG_API bvhg_status bvhg_batch_autotune(bvhg_ctx *ctx, uint32_t nscenes, const int32_t *obj_a, const int32_t *obj_b,
                                        int32_t mode, uint32_t *groups, uint32_t *lanes, double *ms);

/* Patches: the reference's Morton clustering of an object (morton_cluster, src/bvh/split/cluster.hpp:89-179, as
 * set_entity_data_clustering uses it, src/bvh/collision_object.hpp:89-131), on the device from the last rebuild's
 * keys. The elements are ordered stably by their 32-bit Morton hash (the 63-bit key >> 33; equal hashes in element
 * order), and the order is cut at the `patches` - 1 neighbouring positions whose hashes split highest in the Morton
 * tree (smallest 31 - floor(log2(h_i ^ h_i+1)); equal hashes last; ties by position); patch p holds positions
 * [bounds[p], bounds[p + 1]) (src/bvh/collision_object.cpp:134-141). bounds (patches + 1 values, may be NULL) and
 * order (n element indices in patch order, may be NULL) are in `mem`. The object keeps the patches for
 * bvhg_patch_pairs until its next bvhg_set_elements or rebuild. Blocks until done. */
BVHG_API bvhg_status bvhg_cluster(bvhg_ctx *ctx, int32_t obj, uint32_t patches, uint64_t *bounds, uint32_t *order,
                                  int32_t mem);
/* Patch boxes of a clustered object (the k-DOP of the reference's patch snapshot, make_snapshot,
 * src/bvh/snapshot.hpp:139-149, which the reference gathers to build its patch tree, src/bvh/collision_object/
 * top_down.cpp:103-127): boxes[(p * K/2 + a) * 2 + {0 min, 1 max}] is the union of the FP64 slabs
 * (kdop_base::from_vertices with the context's epsilon) of patch p's elements, from their present vertices; an
 * empty patch gets (+inf, -inf). `mem` is the memory kind of boxes. Blocks until done. */
BVHG_API bvhg_status bvhg_patch_kdops(bvhg_ctx *ctx, int32_t obj, double *boxes, int32_t mem);
/* The exact element pairs of two clustered objects (the set of bvhg_broadphase) grouped by patch pair on the device,
 * for a narrowphase functor per patch pair (collision_world::set_narrowphase_functor, src/bvh/collision_world.hpp:
 * 58-94, run per patch pair in src/bvh/collision_object/impl.cpp:269-350). groups: 4 words per non-empty patch pair
 * (patch in obj_a, patch in obj_b, first pair, pair count), in (patch a, patch b) order; pairs: 2 words per element
 * pair (position in the patch of obj_a, position in the patch of obj_b; positions within a patch follow the
 * patch order of bvhg_cluster), grouped in that order, unordered within a group. BVHG_ERR_OVERFLOW when either
 * capacity is too small (*group_count and *pair_count are then the required sizes). Blocks until done. */
BVHG_API bvhg_status bvhg_patch_pairs(bvhg_ctx *ctx, int32_t obj_a, int32_t obj_b, uint32_t *groups,
                                      uint64_t group_capacity, uint64_t *group_count, uint32_t *pairs,
                                      uint64_t pair_capacity, uint64_t *pair_count, int32_t mem);

/* Parity probes (host buffers). sorted_keys[r] and perm[r] (original index of rank r) may be NULL; min3/inv3 are
 * the Morton bounds (3 doubles each, may be NULL). Keys, permutation, bounds and centroids are those of the last
 * rebuild: a refit keeps the order and does not recompute them. The slab probes compute from the present
 * vertices. */
BVHG_API bvhg_status bvhg_get_morton(bvhg_ctx *ctx, int32_t obj, uint64_t *sorted_keys, uint32_t *perm, double *min3,
                            double *inv3);
/* Per-element slabs in original element order, slabs[(i * K/2 + a) * 2 + {0 min, 1 max}]. FP64 form only. */
BVHG_API bvhg_status bvhg_get_kdops(bvhg_ctx *ctx, int32_t obj, double *slabs);
/* Per-element FP32 outward-rounded slabs, original order. FP32 form only. */
BVHG_API bvhg_status bvhg_get_kdops_f32(bvhg_ctx *ctx, int32_t obj, float *slabs);
/* Per-element centroids (3 doubles), original order. */
BVHG_API bvhg_status bvhg_get_centroids(bvhg_ctx *ctx, int32_t obj, double *centroids);
/* Tree check: walks the tree on the host; returns BVHG_OK iff every leaf is reached once, parent slabs contain
 * child slabs and the node count is 2n - 1. depth (may be NULL) receives the maximum leaf depth. */
BVHG_API bvhg_status bvhg_validate_tree(bvhg_ctx *ctx, int32_t obj, uint32_t *depth);

/* Candidate count of the last FP32-form broadphase before the FP64 recheck (false-positive accounting). */
BVHG_API bvhg_status bvhg_last_candidates(bvhg_ctx *ctx, uint64_t *candidates);

/* Stage times (ms) accumulated since the last call, when BVHG_FLAG_STAGE_TIMING is set. ms[BVHG_NUM_STAGES],
 * launches[BVHG_NUM_STAGES] (either may be NULL). Resets the accumulators. */
BVHG_API bvhg_status bvhg_get_stage_times(bvhg_ctx *ctx, double *ms, uint64_t *launches);
/* Number of kernels this context launched since creation. */
BVHG_API bvhg_status bvhg_launch_count(bvhg_ctx *ctx, uint64_t *launches);

/* Test hook: overrides the device spin limit (0 restores the configured one). */
BVHG_API bvhg_status bvhg_set_spin_limit(bvhg_ctx *ctx, uint32_t limit);
/* Test hook: when enabled, every radix-sort look-back after the first tile polls a status word that no block
 * publishes, so the bounded wait runs out and the build reports BVHG_ERR_TIMEOUT (the context stays usable). */
BVHG_API bvhg_status bvhg_test_stall_sort(bvhg_ctx *ctx, int32_t enable);
/* Test hook: sets the batching form's configuration instead of the autotuner (groups 0: per-object launches on
 * `lanes` streams; else the fused form with that many groups of objects on `lanes` streams, lanes 1..64). */
BVHG_API bvhg_status bvhg_test_batch_form(bvhg_ctx *ctx, uint32_t groups, uint32_t lanes);
/* Test hook: lowers the stack bound of the dense-contact walk to `limit` entries (0 restores it), so that it is
 * reached and the library's fallback to the single-node walk runs (the pair set stays exact). */
BVHG_API bvhg_status bvhg_test_dense_stack(bvhg_ctx *ctx, int32_t limit);

/* Stable sort of n device-resident 64-bit keys (Morton keys or any others): keys_out[r] is the r-th smallest key,
 * perm_out[r] its index in keys_in (ties keep input order). No counterpart in the reference: it is the library's
 * radix sort for callers that cannot allocate device memory (a host whose pool allocator owns all device memory, a
 * step loop with a fixed device-memory budget, a library boundary that forbids the callee from owning device
 * memory). It allocates nothing: its scratch is a fixed static device array (about 14 MB on every GPU that loads
 * the library, held until the process exits), so n is limited to 1,048,576 (BVHG_ERR_ARG beyond). The first call
 * on a device resolves the array's address; make it before any stream capture, and do not call again on a device
 * after cudaDeviceReset of it. Calls share the array: calls that overlap on the GPU race. Runs on `stream` (NULL =
 * the default stream) and returns when the sort is complete. keys_in, keys_out and perm_out must not overlap. */
BVHG_API bvhg_status bvhg_radix_sort_noalloc(const uint64_t *keys_in, uint64_t *keys_out, uint32_t *perm_out,
                                             uint64_t n, void *stream);

/* Test hook (no GPU needed): component comp of normal axis of the k-DOP as the kernels use it, and its FP32
 * enclosure [lo, hi]. Any of the outputs may be NULL. */
BVHG_API bvhg_status bvhg_debug_normal(int32_t k, int32_t axis, int32_t comp, double *value, float *lo, float *hi);

BVHG_API bvhg_status bvhg_synchronize(bvhg_ctx *ctx);
BVHG_API const char *bvhg_last_error(const bvhg_ctx *ctx);
BVHG_API const char *bvhg_status_string(bvhg_status status);

#ifdef __cplusplus
}
#endif

#endif /* BVHG_H */
