// Cell-construction kernels: shared constants, the device context and launch helpers.
#pragma once

#include "internal.cuh"

namespace apo2
{
    constexpr uint32_t kCellBlock = 128; // 4 warps, one cell per warp at a time
    constexpr uint32_t kKnnBlock  = 256; // one site per thread
    constexpr uint32_t kMaxK      = 16;  // kNN heap slots per thread (the reference's K)
    constexpr uint32_t kStack     = 64;  // traversal stack entries (the tree height bound)

    // Shared-memory slots per warp: the reference capacities plus room for the records an
    // update appends before it compacts; writes past the slots are dropped and flagged.
    constexpr uint32_t kVertexSlots   = 192;
    constexpr uint32_t kEdgeSlots     = 296;
    constexpr size_t   kWarpCellBytes = ( sizeof( double4 ) + sizeof( uint4 ) ) * kVertexSlots + sizeof( uint4 ) * kEdgeSlots;
    constexpr size_t   kBisectorBytes = sizeof( uint32_t ) * 2 * kMaxBisectors;
    static_assert( kWarpCellBytes % 32 == 0, "warp cell must keep double4 alignment" );

    inline size_t cell_smem_bytes( bool bisector )
    {
        return ( kWarpCellBytes + ( bisector ? kBisectorBytes : 0 ) ) * ( kCellBlock / 32 );
    }

    struct CellContext
    {
        uint32_t         n = 0, k = 16;
        const double4 *  sites   = nullptr; // n + 6, Morton order then the artificial sites
        const float4 *   sites_f = nullptr; // n
        const WideNode * nodes   = nullptr;
        const uint32_t * indices = nullptr; // sorted -> original
        uint8_t *        status  = nullptr;
        uint32_t *       knn     = nullptr; // n * k
        float *          known_radii = nullptr;
        uint32_t *       vertex_nb   = nullptr;
        uint32_t *       edge_nb     = nullptr;
        uint4 *          vertices    = nullptr; // n * 152 records (j, k, l, type | status << 8)
        uint4 *          edges       = nullptr; // n * 264 records (j, k, vertex count, status)
        uint32_t *       error       = nullptr;
    };

    void configure_cell_kernels();
    void launch_knn( const CellContext & c, cudaStream_t s );
    void launch_cells( const CellContext & c, cudaStream_t s );
    void launch_tasks( const CellContext & c, uint32_t * tasks, uint32_t * count, cudaStream_t s );
    void launch_vertex_validation( const CellContext & c, const uint32_t * tasks, const uint32_t * count, cudaStream_t s );
    void launch_edge_validation( const CellContext & c, const uint32_t * tasks, const uint32_t * count, cudaStream_t s );
    void launch_bisector_validation( const CellContext & c, cudaStream_t s );

    // Output extraction: per-cell owned counts, exclusive scans (totals[0] vertices,
    // totals[1] closed edges), then the writes bounded by the capacities.
    struct OutputBuffers
    {
        uint32_t * vcount = nullptr; // n, then offsets
        uint32_t * ccount = nullptr;
        uint32_t * tile_sums = nullptr; // scan scratch
        uint64_t * totals    = nullptr; // [2]
        double4 *  vpos      = nullptr;
        uint4 *    vids      = nullptr;
        double4 *  cpos      = nullptr;
        uint4 *    cids      = nullptr;
        uint64_t   vcap = 0, ccap = 0;
    };
    size_t output_scan_scratch_words( uint32_t n );
    void   launch_output( const CellContext & c, const OutputBuffers & o, cudaStream_t s );
} // namespace apo2
