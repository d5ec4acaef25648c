// Cavity detection over the diagram's vertices (cavity.cu).
#pragma once

#include "internal.cuh"

namespace apo2
{
    // Padding of the trace tree's boxes in the ray / box test: an absolute part and a part
    // per unit of the largest coordinate magnitude (origin or sphere). The single-precision
    // ray / sphere test can accept a ray passing up to about 6 ulp of that magnitude outside
    // a sphere; the padding is far above that, so no box that holds a hit is skipped.
    constexpr float kCavityPadBase  = 1e-3f;
    constexpr float kCavityPadScale = 4e-6f;

    // Largest number of ray directions per vertex (their table sits in shared memory).
    constexpr uint32_t kCavityMaxSamples = 1024;

    // Ray directions (host): xyz (optional) float[3 count]; dirs4 (optional) float[8 count],
    // the directions as float4 and then their reciprocals.
    void cavity_directions( uint32_t count, float * xyz, float * dirs4 );

    // BVH over the trace spheres (float x, y, z, r), built like the diagram's tree.
    struct TraceTree
    {
        uint64_t *  codes    = nullptr;
        uint32_t *  indices  = nullptr; // Morton order -> sphere index
        int32_t *   parent   = nullptr;
        int32_t *   left     = nullptr;
        int32_t *   right    = nullptr;
        float4 *    boxes    = nullptr;
        uint32_t *  arrivals = nullptr;
        WideNode *  nodes    = nullptr;
        float4 *    sorted   = nullptr; // spheres in Morton order
        int *       acc      = nullptr; // bounds reduction
        float *     box      = nullptr; // lo xyz, 1 / extent xyz, pad, -
        SortScratch sort;
        uint32_t    n = 0;
    };
    size_t trace_tree_bytes( uint32_t n );
    void   trace_tree_carve( TraceTree & t, void * base, uint32_t n, uint32_t * error_word );
    void   launch_trace_tree( TraceTree & t, const float4 * spheres, cudaStream_t s );

    // Hit ratio of each of `count` vertices (positions double x, y, z, w; ids of their four
    // sites, indices into `spheres`). dirs: `samples` unit directions then their reciprocals
    // (float4 each, w unused).
    void launch_occlusion( const TraceTree & t, const float4 * spheres, const double4 * vpos, const uint4 * vids, uint64_t count,
                           const float4 * dirs, uint32_t samples, float * ratios, uint32_t * error, cudaStream_t s );

    // Vertices with ratio > ratio_min and radius > radius_min, in order, into out[0, capacity)
    // as float4; *total receives their number. offsets: count words; sums:
    // output_scan_scratch_words(count) words.
    void launch_cavity_filter( const double4 * vpos, const float * ratios, uint64_t count, float ratio_min, float radius_min,
                               uint32_t * offsets, uint32_t * sums, uint64_t * total, float4 * out, uint64_t capacity,
                               cudaStream_t s );
} // namespace apo2
