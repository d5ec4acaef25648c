/*
 * apo2 -- C ABI of the B200-native Apollonius-diagram builder.
 *
 * The library builds the additively weighted Voronoi (Apollonius) diagram of weighted
 * sites (x, y, z, r) on one GPU: LBVH over the sites, kNN search, warp-per-cell cell
 * update with the security-radius certificate, the vertex / edge / bisector validation
 * passes, and the output extraction. Results are those of the reference apo library
 * (PlathC/apo, FP64 `apo` target) on the same input.
 *
 * Conventions
 *   - Every entry point returns an apo2_status; no C++ exception crosses this boundary.
 *   - Pointers are plain host or device addresses; `location` says which.
 *   - All device work of a handle runs on the stream given to apo2_build (0 = the legacy
 *     default stream). A handle must not be used from two threads at once.
 *   - Output site ids are indices into the caller's input array.
 *
 * Reference interfaces replaced (paths relative to the PlathC/apo tree):
 *   apo/include/apo/gpu/algorithm.hpp:35-59   Algorithm, VertexDiagram, FullDiagram,
 *                                              Topology, computeApolloniusDiagram,
 *                                              computeFullApolloniusDiagram
 *   apo/include/apo/gpu/algorithm.cuh:12-46   AlgorithmGPU<K>::build/toHost/toHostFull/
 *                                              toTopology, Sample
 *   apo/src/gpu/lbvh.cu:274-323               LBVH::build (node arrays)
 */
#ifndef APO2_H
#define APO2_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum apo2_status
{
    APO2_OK                = 0,
    APO2_ERR_INVALID_ARG   = 1, /* null pointer, n < 2, unknown dtype / location */
    APO2_ERR_CAPACITY      = 2, /* a per-cell store overflowed (152 vertices / 264 edges / 64 new
                                   edges / 512 bisectors / traversal stack); results are flagged */
    APO2_ERR_ITER_LIMIT    = 3, /* validation still had uncertified cells after the last round */
    APO2_ERR_CUDA          = 4, /* a CUDA call failed; apo2_last_error_string has the text */
    APO2_ERR_NOT_BUILT     = 5, /* result requested before apo2_build */
    APO2_ERR_OUT_OF_MEMORY = 6,
    APO2_ERR_TOO_LARGE     = 7  /* a size above a stated maximum */
} apo2_status;

typedef enum apo2_dtype
{
    APO2_F32 = 0, /* float  x, y, z, r */
    APO2_F64 = 1  /* double x, y, z, r (the reference's FP64 Real) */
} apo2_dtype;

typedef enum apo2_location
{
    APO2_HOST   = 0,
    APO2_DEVICE = 1
} apo2_location;

typedef struct apo2_handle apo2_handle;

/* Build options. Zero-initialise, then set what differs; `struct_size` must be
 * sizeof(apo2_options). */
typedef struct apo2_options
{
    uint32_t struct_size;
    uint32_t k;                    /* kNN neighbours per cell; 0 = 16 (reference default) */
    uint32_t max_iterations;       /* validation rounds; 0 = 10 (algorithm.inl:1554) */
    uint32_t device;               /* CUDA device ordinal */
    uint32_t stage_timing;         /* 1 = record per-stage CUDA-event times (apo2_stats) */
    uint32_t edge_search;          /* 0 = edge-parallel search with exact per-cell fallback (default),
                                      1 = warp-per-cell edge validation only; both give the same result */
    uint32_t knn_steps;            /* kNN + cell-construction steps, the reference's knnValidationStep
                                      (algorithm.inl:1535-1549): 0 = 1 (its default), APO2_NO_KNN_STEPS
                                      = none (every cell starts from the initial cell), at most 64 */
    uint32_t stop_after;           /* parity checks only: 0 = the whole build; 1 = stop after the kNN
                                      cell construction; 2 + 2r / 3 + 2r = stop after the vertex / edge
                                      validation of round r (0-based). Output extraction still works */
    uint32_t shard_index;          /* one diagram over several GPUs: this handle builds the cells of
                                      shard shard_index of shard_count (shard_count 0 = 1: the whole
                                      diagram), a contiguous range of the Morton-sorted sites. Every
                                      shard needs all the sites; its output is its cells' share of the
                                      diagram's, and the shards' outputs in shard order are the whole
                                      diagram's output, in order */
    uint32_t shard_count;
    uint32_t wait_limit;           /* polls per look-back wait of the LBVH's radix sort before the tile
                                      counts its digits itself (exact either way; 0 = 2^22). Tests set
                                      it small to exercise that path; apo2_stats.error_flags bit 32
                                      reports that a wait ran out */
    uint32_t precision;            /* APO2_PRECISION_FP64 (0, the plain form) or APO2_PRECISION_FP32_FILTER:
                                      conflict predicates against sites are first evaluated in single
                                      precision from a float copy of the sites under a static error
                                      bound, and only those inside the bound in the reference's FP64
                                      arithmetic; every decision, and so the diagram, is the same */
    uint32_t reserved[ 4 ];
} apo2_options;

#define APO2_PRECISION_FP64        0u
#define APO2_PRECISION_FP32_FILTER 1u

#define APO2_NO_KNN_STEPS 0xffffffffu

/* Per-build statistics, the counterpart of AlgorithmGPU::Sample (algorithm.cuh:18-27). */
typedef struct apo2_stats
{
    uint32_t n;
    uint32_t buried;               /* cells of sites inside another site */
    uint32_t certified_after_knn;  /* cells certified by the kNN security radius */
    uint32_t validation_rounds;    /* vertex+edge validation rounds that had work */
    uint32_t error_flags;          /* capacity flags (1 vertex, 2 edge, 4 new edge, 8 bisector, 16 stack),
                                      32 a sort look-back wait ran out (recounted: the order is exact),
                                      64 a walk or restart loop reached its bound */
    uint32_t kernel_launches;      /* kernels launched by the last build (+ extraction) */
    uint64_t vertex_records;       /* sum of per-cell vertex counts */
    uint64_t edge_records;         /* sum of per-cell edge counts */
    uint64_t output_vertices;      /* vertices owned by their smallest site (toHost) */
    uint64_t output_closed_edges;  /* closed trisectors owned by their smallest site */
    double   ms_bounds;            /* bbox, Morton codes */
    double   ms_sort;              /* onesweep radix sort */
    double   ms_tree;              /* leaves, hierarchy, refit */
    double   ms_knn;
    double   ms_cells;
    double   ms_vertex_validation;
    double   ms_edge_validation;
    double   ms_bisector_validation;
    double   ms_output;
    uint64_t device_bytes;         /* device memory held by the handle */
    uint32_t uncertified;          /* cells still in validation after the last round (APO2_ERR_ITER_LIMIT) */
    uint32_t reserved32;
    uint64_t knn_insertions;       /* neighbours inserted by the kNN cell construction (all steps) */
    uint64_t proposal_cells;       /* learned form: cells whose certificate was checked at a proposed rank */
    uint64_t proposal_fallbacks;   /* ... of which failed there and went on through their list */
    uint64_t proposal_skipped;     /* neighbours not inserted because the cell certified earlier */
    uint64_t filter_tests;         /* FP32-filtered form: conflict predicates of the cell kernels */
    uint64_t filter_escalations;   /* ... that fell inside the bound and were evaluated in FP64 */
    uint64_t proposal_second_step; /* learned form: cells that took the second kNN step */
} apo2_stats;

/* Library version string. */
const char * apo2_version( void );

/* Text of the last error raised on this thread. */
const char * apo2_last_error_string( void );

/* Creates a handle over `n` sites. The sites are copied (or converted) to device memory
 * immediately; the caller keeps ownership of `sites`.
 * Replaces: AlgorithmGPU<K>::AlgorithmGPU(ConstSpan<Real>, uint32_t)
 *           (apo/include/apo/gpu/algorithm.inl:1404-1408, src/gpu/algorithm.cpp:5-25). */
apo2_status apo2_create( const void * sites, uint32_t n, apo2_dtype dtype, apo2_location location,
                         const apo2_options * options, apo2_handle ** out );

/* Replaces the sites of an existing handle (same n), reusing its device memory. */
apo2_status apo2_set_sites( apo2_handle * h, const void * sites, apo2_dtype dtype, apo2_location location,
                            void * stream );

/* Builds the diagram on `stream` (a cudaStream_t; 0 = default). Asynchronous with respect to
 * the host unless `synchronize` is non-zero, in which case the build's status is returned:
 * APO2_ERR_CAPACITY when a per-cell store overflowed, APO2_ERR_ITER_LIMIT when cells were still
 * uncertified after max_iterations validation rounds (or a bounded walk stopped early). The
 * diagram is complete in both cases, as the reference leaves it (the reference prints or ignores
 * these conditions); apo2_get_stats gives the flags and the uncertified count.
 * Replaces: AlgorithmGPU<K>::build() (apo/include/apo/gpu/algorithm.inl:1410-1594). */
apo2_status apo2_build( apo2_handle * h, void * stream, int synchronize );

/* Builds and then extracts the output vertices / closed edges into device buffers owned by
 * the handle (no host synchronisation); apo2_output_device returns their addresses. */
apo2_status apo2_build_and_extract( apo2_handle * h, void * stream );

/* Counts of the output (synchronises the handle's stream). */
apo2_status apo2_output_counts( apo2_handle * h, uint64_t * vertices, uint64_t * closed_edges );

/* Device addresses of the extracted output (valid until the next build or destroy):
 * positions double4 [count], ids uint32[4*count] (original site indices i,j,k,l). */
apo2_status apo2_output_device( apo2_handle * h, const double ** vertex_positions, const uint32_t ** vertex_ids,
                                const double ** closed_positions, const uint32_t ** closed_ids );

/* Copies the vertices owned by their smallest site (cell i < j,k,l) into caller buffers:
 * positions (x,y,z,w) double[4*capacity], ids uint32[4*capacity] (i,j,k,l original ids).
 * Replaces: AlgorithmGPU<K>::toHost (apo/include/apo/gpu/algorithm.inl:1596-1646). */
apo2_status apo2_get_vertices( apo2_handle * h, double * positions, uint32_t * ids, uint64_t capacity,
                               apo2_location location, uint64_t * written );

/* Closed (vertex-free elliptic) trisectors: the trisector vertex of smaller radius and the
 * ids (i, j, k, 0). Replaces the closed-edge half of AlgorithmGPU<K>::toHostFull
 * (apo/include/apo/gpu/algorithm.inl:1648-1730). */
apo2_status apo2_get_closed_edges( apo2_handle * h, double * positions, uint32_t * ids, uint64_t capacity,
                                   apo2_location location, uint64_t * written );

/* Topology as the reference's toTopology (apo/include/apo/gpu/algorithm.inl:1732-1821):
 * per cell (sorted order) the unique bisectors (i<j), trisectors (i<j,k) and quadrisectors
 * (i<j,k,l), mapped to original ids. Pass NULL arrays to query the counts first. */
apo2_status apo2_get_topology( apo2_handle * h, uint32_t * quadrisectors, uint64_t quad_capacity,
                               uint32_t * trisectors, uint64_t tri_capacity, uint32_t * bisectors,
                               uint64_t bi_capacity, uint64_t * quad_count, uint64_t * tri_count,
                               uint64_t * bi_count );

/* The topology as the JSON text the reference's topology harness writes
 * (app/topology/topology.cpp:11-57, same layout and order: "bisectors", "trisectors",
 * "quadrisectors" lists of id tuples). *length receives the text's size without the NUL; with
 * json == NULL only the size is computed, otherwise capacity must hold length + 1 bytes. */
apo2_status apo2_topology_json( apo2_handle * h, char * json, uint64_t capacity, uint64_t * length );

/* Interval certificate of output points, as the reference's precision check
 * (app/precision/precision.cpp:14-163): every weighted distance |c - p| - r is an outward-rounded
 * interval, and a point is bad when a site other than its own is certainly closer than the
 * largest of its own sites' distances. arity 4 checks vertices (ids i, j, k, l), 3 closed
 * edges (ids i, j, k). positions/ids: double[4*count] / uint32[4*count] (original site ids) on
 * the host or the device; both NULL certifies the handle's last extracted output (count is
 * then taken from it). flags (optional, host, count bytes) receives 1 for each bad point. The
 * search walks the handle's BVH instead of all sites. */
apo2_status apo2_certify( apo2_handle * h, const double * positions, const uint32_t * ids, uint64_t count, uint32_t arity,
                          apo2_location location, uint8_t * flags, uint64_t * bad );

/* Learned k-proposal (a per-cell kNN rank chosen by a network; the reference only measures the labels,
 * app/benchmarks/benchmark_contributing_nearest.cu:10-129). A 16 -> 64 -> 64 -> 1 network with
 * ReLU, bf16 weights and fp32 accumulation predicts log2 of the kNN rank at which a site's cell
 * passes the security-radius certificate, from 16 features of the site (radius, Morton-local
 * density, radii and distances of its nearest neighbours; see apo2_proposal_features). With a
 * model attached (apo2_set_proposal), the kNN kernel runs the network for every site and each cell
 * gets the proposed rank ceil(2^(prediction + margin)) in [1, max_rank]:
 *   - a rank r <= K: the kNN cell construction checks the certificate after r neighbours; a cell
 *     that passes stops there (its later neighbours cannot change a certified cell), one that
 *     does not (a fallback) goes on through its list as the plain form does;
 *   - a rank r > K (max_rank > K, with one kNN step configured): the cell goes through its K
 *     neighbours, then -- if still uncertified -- through a second kNN step, the next K sites
 *     beyond the last (the reference's expanding search, knnValidationStep = 2,
 *     algorithm.inl:1535-1549), with its certificate checked after r - K of them.
 * Either way the certificate alone decides, and every cell ends as the reference's build with one
 * kNN step (r <= K) or two (r > K) leaves it. */
#define APO2_PROPOSAL_INPUTS 16
#define APO2_PROPOSAL_HIDDEN 64
#define APO2_PROPOSAL_PARAMS 5313 /* fp32 training vector: W1 (64 x 16), b1, W2 (64 x 64), b2, w3, b3 */

typedef struct apo2_proposal
{
    uint32_t struct_size;                                         /* sizeof(apo2_proposal) */
    uint32_t version;                                             /* 1 */
    uint32_t max_rank;                                            /* largest proposed rank: K (early checks
                                                                     only) up to 2K (a second kNN step for
                                                                     cells proposed beyond K) */
    float    mean[ APO2_PROPOSAL_INPUTS ];                        /* inputs are (x - mean) * inv_scale */
    float    inv_scale[ APO2_PROPOSAL_INPUTS ];
    float    margin;                                              /* added to the prediction before 2^() */
    float    b3;
    float    b1[ APO2_PROPOSAL_HIDDEN ];
    float    b2[ APO2_PROPOSAL_HIDDEN ];
    uint16_t w1[ APO2_PROPOSAL_HIDDEN * APO2_PROPOSAL_INPUTS ];   /* bf16 bits, row-major (out x in) */
    uint16_t w2[ APO2_PROPOSAL_HIDDEN * APO2_PROPOSAL_HIDDEN ];
    uint16_t w3[ APO2_PROPOSAL_HIDDEN ];
} apo2_proposal;

/* Switches the precision form of a handle's next builds (apo2_options.precision). */
apo2_status apo2_set_precision( apo2_handle * h, uint32_t precision );

/* Features of every site of a built handle, in sorted (Morton) order as apo2_debug_array:
 * host float[16 * n]. */
apo2_status apo2_proposal_features( apo2_handle * h, float * features );

/* Predictions (log2 rank) of a model for n feature rows (host arrays). */
apo2_status apo2_proposal_predict( const apo2_proposal * model, const float * features, uint64_t n, float * out );

/* Mean squared error of one batch and its gradient with respect to the fp32 parameter vector
 * `master` (APO2_PROPOSAL_PARAMS floats; the forward pass uses it rounded to bf16), computed by
 * the training kernels; model supplies mean / inv_scale. For gradient checks. */
apo2_status apo2_proposal_gradients( const apo2_proposal * model, const float * master, const float * features,
                                     const float * targets, uint32_t n, float * loss, float * grads );

/* Trains the network on the GPU (Adam, mean squared error on `targets`, batches of `batch`
 * samples in a seeded random order each epoch). master: the fp32 parameter vector, initial on
 * entry, trained on return; model: mean / inv_scale on entry, the bf16 weights and biases of the
 * trained vector on return (margin untouched). epoch_loss (optional) receives each epoch's mean
 * loss. All host arrays. */
apo2_status apo2_proposal_train( const float * features, const float * targets, uint64_t n, uint32_t epochs, uint32_t batch,
                                 float learning_rate, uint64_t seed, float * master, apo2_proposal * model, float * epoch_loss );

/* Attaches a model to a handle (copied to the device): its next builds use the learned form.
 * NULL detaches it (the plain form). */
apo2_status apo2_set_proposal( apo2_handle * h, const apo2_proposal * model );

/* Error of output vertices against an FP64 oracle, per result: each vertex (x, y, z, w) with its
 * four original site ids is refined by Newton steps on |p - c_a| - r_a - w = 0 (a = the four
 * sites) in IEEE double precision, and its error is max over x, y, z, w of
 * |given - refined| / max(1, |refined|). The reference computes vertices in double precision but
 * with a single-precision square root inside every length (gpu/math.cuh:307-309); the required
 * bound for every result is 1e-5. positions/ids: double[4*count] / uint32[4*count] on the host
 * or the device, or both NULL for the handle's last extracted vertices (count is then taken
 * from it). errors (optional, host float[count]) receives each vertex's error; *max_error the
 * largest; *above (optional) how many exceed `threshold`; *singular (optional) how many
 * vertices have a singular system (their error is reported as 0). No counterpart in the
 * reference, whose precision harness (app/precision/precision.cpp) checks emptiness only. */
apo2_status apo2_vertex_error( apo2_handle * h, const double * positions, const uint32_t * ids, uint64_t count,
                               apo2_location location, double threshold, float * errors, double * max_error,
                               uint64_t * above, uint64_t * singular );

/* Labels of the kNN cell construction, as the reference's measurement harness records them
 * (app/benchmarks/benchmark_contributing_nearest.cu:10-129): `steps` kNN steps of the handle's K
 * neighbours each; for cell i (sorted order, as apo2_debug_array) and rank r < steps * K,
 * contributed[i * steps * K + r] = 1 when that neighbour changed the cell and certified[...] = 1
 * when the security-radius certificate held after it; a cell stops at the rank where it
 * certifies. Both arrays are host buffers of n * steps * K bytes. The run replaces the handle's
 * stores (build again before reading a diagram). Ranks past a cell's end stay 0. */
apo2_status apo2_contribution_profile( apo2_handle * h, uint32_t steps, uint8_t * contributed, uint8_t * certified );

/* Cavity detection over the diagram, as the reference's cavity application does it
 * (app/cavity/main.cpp:8-88) with CUDA kernels over a sphere BVH where the reference uses OptiX.
 *
 * Directions of the occlusion rays: the first `count` points (1..1024) of the Halton sequence
 * on the sphere in bases 2 and 3 (Wong, Luk and Heng, "Sampling with Hammersley and Halton
 * points", 1997) as app/cavity/utils.cu:201-242 generates them, scaled to unit length;
 * xyz: host float[3 * count]. */
apo2_status apo2_cavity_directions( uint32_t count, float * xyz );

/* Hit ratio of every output vertex, in apo2_get_vertices order (app/cavity/utils.cu:17-65,
 * app/cavity/shaders/find_occlusion.cu:26-69): the share of `samples` rays from the vertex centre
 * (in float), one along each direction of apo2_cavity_directions(samples), that meet a sphere of
 * `spheres` (float x, y, z, r; host or device) with 0.01 <= t <= 1e16; a ray that starts inside
 * a sphere meets it where it leaves it. Sphere i stands for the site of original id i (the
 * reference traces the sites as loaded, before the joggle the diagram was built from). Each
 * ray / sphere decision is the single-precision test of cavity.cu, so the ratios are exactly
 * those of testing every ray against every sphere. The ratios stay on the device for
 * apo2_cavity_vertices; hit_ratios (optional, host, capacity floats) receives a copy and
 * *count their number. ms (optional, 2 floats) receives the device times of the sphere tree
 * build and of the ray casting. */
apo2_status apo2_cavity_hit_ratios( apo2_handle * h, const float * spheres_xyzr, uint32_t sphere_count,
                                    apo2_location location, uint32_t samples, float * hit_ratios, uint64_t capacity,
                                    uint64_t * count, float * ms );

/* Cavity vertices (app/cavity/utils.cu:67-83, 244-264, 527-559): the output vertices whose hit ratio is
 * above hit_ratio_threshold and whose radius is above radius_threshold (the reference's
 * application starts at 0.5 and 5), in output order, as float (x, y, z, w). Needs
 * apo2_cavity_hit_ratios after the last build (APO2_ERR_NOT_BUILT otherwise). xyzw: host
 * float[4 * capacity], or NULL to count only; *count receives the number found. */
apo2_status apo2_cavity_vertices( apo2_handle * h, float hit_ratio_threshold, float radius_threshold, float * xyzw,
                                  uint64_t capacity, uint64_t * count );

/* Per-cell store of one site (given by original id): its vertices as (j, k, l, type) and
 * edges as (j, k, vertex count or 0xffffffff for a closed trisector), ids original. */
apo2_status apo2_get_cell( apo2_handle * h, uint32_t site, uint32_t * vertices, uint32_t vertex_capacity,
                           uint32_t * vertex_count, uint32_t * edges, uint32_t edge_capacity,
                           uint32_t * edge_count );

/* Raw internal arrays for parity checks, host copies. `name` is one of: "indices"
 * (sorted -> original id, u32[n]), "parent", "left", "right" (i32[2n-1]), "aabb"
 * (f32[8(2n-1)], min xyz 0 max xyz 0), "sizes" (u32[2n-1]), "morton" (u64[n], sorted),
 * "sites_sorted" (f64[4(n+6)]), "status" (u8[n]), "knn" (u32[n*k]), "known_radii"
 * (f32[n]), "proposed_k" (u8[n], the learned form's proposed ranks), "vertex_nb", "edge_nb" (u32[n]), "vertices", "edges" (u32 records of 4 words,
 * cells in sorted order, sorted-space ids). With dst == NULL only *count is set (elements). */
apo2_status apo2_debug_array( apo2_handle * h, const char * name, void * dst, uint64_t capacity_bytes,
                              uint64_t * count );

apo2_status apo2_get_stats( apo2_handle * h, apo2_stats * stats );

/* Kernel launches of the last build as JSON text: {"launches": L, "timed": bool, "kernels":
 * {"name": [count, total_ms, longest_launch_ms], ...}} (times only with stage_timing). With json == NULL only
 * *length is set. */
apo2_status apo2_kernel_profile( apo2_handle * h, char * json, uint64_t capacity, uint64_t * length );

apo2_status apo2_destroy( apo2_handle * h );

/* One-call forms of the reference's free functions (apo/include/apo/gpu/algorithm.hpp:58-59):
 * build the diagram of host sites and copy the vertices (and closed edges) out. The output
 * arrays are allocated with malloc and released with apo2_free. */
apo2_status apo2_compute_diagram( const void * sites, uint32_t n, apo2_dtype dtype, double ** positions,
                                  uint32_t ** ids, uint64_t * count );
apo2_status apo2_compute_full_diagram( const void * sites, uint32_t n, apo2_dtype dtype, double ** positions,
                                       uint32_t ** ids, uint64_t * count, double ** closed_positions,
                                       uint32_t ** closed_ids, uint64_t * closed_count );
void apo2_free( void * p );

/* LBVH only (apo/src/gpu/lbvh.cu:274-323): Morton codes of device float4 sites inside the
 * scene box, stable onesweep radix sort, Karras hierarchy and refit. All pointers are device
 * pointers of the sizes given in apo2_debug_array's list; `scratch` is a device buffer of at
 * least apo2_lbvh_scratch_bytes(n) bytes. */
uint64_t    apo2_lbvh_scratch_bytes( uint32_t n );
apo2_status apo2_lbvh_build( const float * sites_xyzr, uint32_t n, const float scene_min[ 3 ],
                             const float scene_max[ 3 ], uint32_t * indices, uint64_t * sorted_codes,
                             int32_t * parent, int32_t * left, int32_t * right, float * aabb, uint32_t * sizes,
                             void * scratch, void * stream );

/* Stable radix sort of (u64 key, u32 value) pairs by key on the device (the LBVH's sort):
 * keys/values are sorted in place; `scratch` must hold apo2_radix_sort_scratch_bytes(n). Its
 * first 4 bytes receive the sort's status word on the stream: 0, or 32 when a look-back wait
 * ran out and the tile counted its digits itself (the order is exact either way). The same
 * holds for apo2_lbvh_build's scratch. */
uint64_t    apo2_radix_sort_scratch_bytes( uint32_t n );
apo2_status apo2_radix_sort_pairs( uint64_t * keys, uint32_t * values, uint32_t n, void * scratch, void * stream );

/* The same sort for callers that cannot allocate device memory where they sort (memory owned by
 * another allocator, a latency-critical path where cudaMalloc would synchronise). No counterpart
 * in the reference. Its scratch is a fixed __device__ array of the library (about 12.3 MiB per GPU,
 * held until exit); at most 2^20 pairs, APO2_ERR_TOO_LARGE above. All calls on a device share
 * that array, so calls that overlap on the GPU race; calls in sequence are independent. The first
 * call on a device looks the array up with that device current. A look-back wait that runs out is
 * recounted exactly (see apo2_radix_sort_pairs); this entry point does not report it. */
apo2_status apo2_radix_sort_pairs_static( uint64_t * keys, uint32_t * values, uint32_t n, void * stream );

/* Batched form: many independent diagrams of uneven size in one call (the reference builds one
 * diagram per AlgorithmGPU object; a caller with thousands of small site sets loops over it,
 * app/benchmarks/benchmark.cu:9-22). `streams` workers, each with its own stream, host thread and
 * device memory for `max_sites` sites, take the diagrams largest first, so small builds overlap
 * on the GPU. All allocation happens in apo2_batch_create. */
typedef struct apo2_batch apo2_batch;
apo2_status apo2_batch_create( uint32_t max_sites, uint32_t streams, const apo2_options * options, apo2_batch ** out );

/* Builds `count` diagrams. Diagram d is sites_xyzr[4*site_offsets[d] .. 4*site_offsets[d+1]) (host,
 * float x, y, z, r; at least 2 and at most max_sites sites). On return vertex_offsets[0..count]
 * holds the prefix sums of the per-diagram output vertex counts; when positions and ids are not
 * NULL they receive malloc'd arrays (release with apo2_free) of all diagrams' vertices in diagram
 * order, as apo2_get_vertices gives them (ids index the diagram's own sites). build_ms (optional,
 * count floats) receives each diagram's device time from its upload to the end of its extraction. */
apo2_status apo2_batch_build( apo2_batch * b, const float * sites_xyzr, const uint64_t * site_offsets, uint32_t count,
                              uint64_t * vertex_offsets, double ** positions, uint32_t ** ids, float * build_ms );
/* Attaches a learned k-proposal to every worker of a batch (NULL: the plain form). */
apo2_status apo2_batch_set_proposal( apo2_batch * b, const apo2_proposal * model );
apo2_status apo2_batch_destroy( apo2_batch * b );

/* Measured peak throughput of the FMA pipes of the current device, in TFLOP/s (2 FLOPs per fused
 * multiply-add, many independent chains per thread, best of five launches): the denominators of
 * the build's compute roofline, whose arithmetic is scalar FP64 and FP32. No counterpart in the
 * reference. */
apo2_status apo2_fma_peak( double * fp64_tflops, double * fp32_tflops );

/* Seeded protein-like site set (host): `chains` self-avoiding random-walk chains of
 * `atoms_per_chain` atoms (bond 1.53 A, bond angle 109.5 +/- 10 deg, uniform torsion, van der
 * Waals radii mix) in a cube of `density` atoms per A^3, written as float (x, y, z, r).
 * Stand-in for the reference's PDB inputs (app/common/samples.cpp:10-61), which need chemfiles. */
apo2_status apo2_generate_chains( uint32_t chains, uint32_t atoms_per_chain, double density, uint64_t seed, float * out_xyzr );

#ifdef __cplusplus
}
#endif

#endif /* APO2_H */
