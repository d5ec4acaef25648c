/*
 * CPU oracle for the Apollonius-diagram construction path -- TEST INFRASTRUCTURE ONLY.
 *
 * A single-GPU-free restatement, in C++ on the host, of the reference algorithm
 * (PlathC/apo): the LBVH build (apo/src/gpu/lbvh.cu), the kNN search
 * (apo/include/apo/gpu/lbvh.inl, algorithm.inl:32-99), the warp-per-cell cell update
 * (apo/include/apo/gpu/topology_update.inl), the security-radius certificate, the three
 * validation passes and the output extraction (apo/include/apo/gpu/algorithm.inl).
 * Warp-collective steps (ballots, shuffles, scans, the new-edge sort) are simulated lane
 * by lane so that every per-cell store ends in the same order as on the GPU.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm may
 * load this library, and only as the checker or the timed CPU baseline. The product
 * path never calls it.
 *
 * Floating-point: double arithmetic is evaluated in the reference's source order without
 * fused multiply-adds; single-precision traversal math uses IEEE sqrtf where the
 * reference's --use_fast_math build uses the approximate hardware square root. Values can
 * therefore differ in the last bits from a GPU run; decisions (topology) agree unless a
 * predicate lands within a few ulps of its 1e-8 threshold.
 */
#ifndef APO_ORACLE_H
#define APO_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_run oracle_run;

/* Stages run by oracle_build, cumulative. */
enum
{
    ORACLE_STAGE_LBVH       = 1, /* bbox, Morton codes, stable sort, Karras tree, refit */
    ORACLE_STAGE_KNN        = 2, /* + kNN lists and buried flags */
    ORACLE_STAGE_CELLS      = 3, /* + kNN cell construction and certificate */
    ORACLE_STAGE_VALIDATION = 4, /* + vertex / edge / bisector validation passes */
    ORACLE_STAGE_OUTPUT     = 5  /* + vertices, closed edges and topology */
};

/* Builds the diagram of `n` float32 (x, y, z, r) sites up to `last_stage`, with `threads`
 * OpenMP threads (0 = all). Returns NULL on invalid input. */
oracle_run * oracle_build( const float * sites_xyzr, uint32_t n, int last_stage, int threads );

/* Same input given as float64 (x, y, z, r), as the reference's FP64 public API takes it. */
oracle_run * oracle_build_f64( const double * sites_xyzr, uint32_t n, int last_stage, int threads );

/* General form: float32 (is_f64 = 0) or float64 input, `k` neighbours per kNN step (1..16,
 * the AlgorithmGPU<K> argument) and `knn_steps` kNN + cell steps (the knnValidationStep
 * argument, algorithm.inl:1535-1549; 0 = none). */
oracle_run * oracle_build_ex( const void * sites_xyzr, int is_f64, uint32_t n, uint32_t k, uint32_t knn_steps,
                              int last_stage, int threads );

/* The contributing-nearest study (app/benchmarks/benchmark_contributing_nearest.cu:10-302) on
 * float32 sites: `steps` kNN steps of 16 neighbours, each followed by the labelling kNN cell
 * construction. Arrays "contribution" and "reached": steps * 16 bytes per site, sorted order. */
oracle_run * oracle_contribution_profile( const float * sites_xyzr, uint32_t n, uint32_t steps, int threads );

/* Looks up one result array by name; returns its element count (0 if absent) and its
 * address in *data. Names: indices parent left right aabb sizes morton sites_sorted
 * status knn known_radii vertex_nb edge_nb vertices edges out_vertices out_vertices_id
 * out_closed out_closed_id topo_quad topo_tri topo_bi (contribution reached of a profile). */
uint64_t oracle_get( const oracle_run * run, const char * name, const void ** data );

/* Bit set of capacity overflows met while building (1: vertex store, 2: edge store,
 * 4: new-edge list, 8: bisector list, 16: traversal stack). */
uint32_t oracle_flags( const oracle_run * run );

void oracle_free( oracle_run * run );

/* PCG-hash based joggle of the reference (apo/src/core/utils.cpp:15-25), in place. */
void oracle_joggle( double * sites_xyzr, uint64_t n, double range );

#ifdef __cplusplus
}
#endif

#endif /* APO_ORACLE_H */
