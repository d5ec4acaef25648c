// Cell-construction kernels: shared constants, the device context and launch helpers.
#pragma once

#include "internal.cuh"
#include "proposal.cuh"

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
        uint32_t         lo = 0, hi = 0; // cells built: sorted ids [lo, hi) (a shard of the diagram)
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
        const Scene *    scene       = nullptr; // bounds and radius range of the sites
        uint32_t *       walk_scratch = nullptr; // kWalkScratchWords per warp of the exact edge pass
        uint32_t *       work_counter = nullptr; // next cell of the dynamically scheduled passes
        // learned k-proposal (null: the plain form): the network, the Morton codes its features
        // read, and the proposed rank of every site (written by the first kNN step)
        const ProposalNet * proposal   = nullptr;
        const uint64_t *    codes      = nullptr;
        uint8_t *           proposed_k = nullptr;
        uint32_t            proposal_max = 0; // largest proposed rank (k .. 2k)
        uint32_t            scheduled    = 0; // 1: cells proposed beyond k get a second kNN step
        // build counters: kNN insertions, cells checked at a proposed rank, fallbacks, skipped
        // neighbours, conflict predicates decided by the FP32 filter, those it left to FP64
        unsigned long long * counters = nullptr;
        // FP32-filtered form: conflict predicates against sites first in single precision
        uint32_t fp32 = 0;
    };
    constexpr uint32_t kCountInsertions = 0, kCountChecked = 1, kCountFallbacks = 2, kCountSkipped = 3, kCountFiltered = 4,
                       kCountEscalated = 5, kCountSecondStep = 6, kCounters = 7;

    // Learned form with a second kNN step: is cell i one of those proposed beyond k?
    __device__ __forceinline__ bool second_step_cell( const CellContext & c, uint32_t i )
    {
        return c.scheduled && c.proposed_k[ i ] > c.k;
    }

    // Lane-local tallies of the FP32 filter, added to the build's counters when a kernel ends.
    struct FilterTally
    {
        uint32_t tests = 0, escalated = 0;
    };

    // The reference's conflict test of site `id` against the sphere x (gpu/math.cuh:374-388),
    // decided by the FP32 filter where it can in the filtered form.
    __device__ __forceinline__ bool site_conflict( const CellContext & c, uint32_t id, double4 x, FilterTally & t )
    {
        if ( c.fp32 )
        {
            t.tests++;
            // the float copy holds the n input sites; the six bounding sites are rounded here
            const float4 s = id < c.n ? c.sites_f[ id ] : to_float( c.sites[ id ] );
            const int    f = conflict_filter( s, x );
            if ( f != 2 )
                return f == 1;
            t.escalated++;
        }
        return intersects( c.sites[ id ], x );
    }
    // The same for a site given by value (its float copy is exact for float input and bounded otherwise).
    __device__ __forceinline__ bool sphere_conflict( const CellContext & c, double4 site, double4 x, FilterTally & t )
    {
        if ( c.fp32 )
        {
            t.tests++;
            const int f = conflict_filter( to_float( site ), x );
            if ( f != 2 )
                return f == 1;
            t.escalated++;
        }
        return intersects( site, x );
    }

    // Row of cell i in the per-cell stores (vertices, edges), which hold only the cells
    // [lo, hi) a handle builds: a shard of the diagram needs stores for its own cells alone.
    __host__ __device__ __forceinline__ size_t store_row( const CellContext & c, uint32_t i ) { return size_t( i - c.lo ); }

    // Exact edge validation: a lane walks its edge's search alone for kLaneWalk steps; a
    // search still running then is finished by the whole warp, in the same order, from a
    // frontier of at most kCoopCap nodes kept in global scratch (plus each lane's saved stack),
    // kCoopWidth x 32 frontier nodes per step.
#ifndef APO2_EXACT_LANE_WALK
#define APO2_EXACT_LANE_WALK 256
#endif
    constexpr uint32_t kLaneWalk         = APO2_EXACT_LANE_WALK;
#ifndef APO2_COOP_WIDTH
#define APO2_COOP_WIDTH 4
#endif
    constexpr uint32_t kCoopWidth        = APO2_COOP_WIDTH; // frontier nodes per lane per step
    constexpr uint32_t kCoopCap          = 8192;
    constexpr uint32_t kWalkScratchWords = kCoopCap + 32 * ( kStack + 1 );

    // Position of a stored vertex: root `type` of quadrisector(si, sj, sk, sl) with the
    // sorted ids (topology_update.inl:104-111).
    __device__ __forceinline__ double4 solve_vertex( const CellContext & c, double4 si, uint4 r )
    {
        double4 x[ 2 ] = { make_double4( 0, 0, 0, 0 ), make_double4( 0, 0, 0, 0 ) };
        quadrisector( si, c.sites[ r.x ], c.sites[ r.y ], c.sites[ r.z ], x[ 0 ], x[ 1 ] );
        return ( r.w & 0xffu ) ? x[ 1 ] : x[ 0 ];
    }

    // ---------------------------------------------------------------------------------
    // Reach of an edge search. A site j contributes to edge (k, l) of cell i only through a
    // root x that passes the emptiness test against the cell's neighbours, i.e. a point of
    // the edge's arc inside the current cell, whose empty-sphere radius w(x) is at most the
    // largest radius over the arc: its vertices and, on an elliptic trisector, an apex that
    // may lie on the arc (the cell certificate of the reference rests on the same bound,
    // algorithm.inl:186-190, topology_update.inl:595-653). Then
    //     |c_j - c_i| <= |c_j - x| + |x - c_i| = 2 w(x) + r_i + r_j,
    // so the search may skip every BVH node and leaf outside that ball: the leaves it
    // visits are a subsequence of the reference's, in the same order, and every site that
    // could contribute is among them, so the first contributor found is the same.
    // ---------------------------------------------------------------------------------
    __device__ __forceinline__ bool vertex_on_edge( uint4 r, uint32_t k, uint32_t l )
    {
        return ( r.x == k || r.y == k || r.z == k ) && ( r.x == l || r.y == l || r.z == l );
    }

    // An apex (trisector root in the plane of the centres) counts unless a neighbour other
    // than k, l clearly intersects its sphere (IEEE double distance, relative margin 1e-4).
    __device__ __forceinline__ bool clearly_outside( double4 site, double4 apex )
    {
        const double dx = site.x - apex.x, dy = site.y - apex.y, dz = site.z - apex.z;
        const double d  = __dsqrt_rn( __dadd_rn( __dadd_rn( __dmul_rn( dx, dx ), __dmul_rn( dy, dy ) ), __dmul_rn( dz, dz ) ) );
        const double pen = ( site.w + apex.w ) - d;
        return pen > 1e-4 * ( site.w + fabs( apex.w ) ) + 1e-6;
    }

    // Radius of the ball around c_i that holds every possible contributor, with margins.
    __device__ __forceinline__ float reach_radius( double wmax, double ri, double rmax )
    {
        const double r = 2.0 * wmax * 1.01 + ri + rmax + 1e-3 * ( 1.0 + wmax );
        return float( r ) * 1.0001f + 1e-3f;
    }
    void configure_cell_kernels();
    // bytes of CellContext::walk_scratch: one region per warp the cell kernels launch
    size_t walk_scratch_bytes();
    // k_cells modes: first kNN step, a later kNN step, initial cells only (no kNN step)
    constexpr uint32_t kCellsFirst    = 0;
    constexpr uint32_t kCellsNext     = 1;
    constexpr uint32_t kCellsInitOnly = 2;
    void launch_knn( const CellContext & c, uint32_t step, cudaStream_t s );
    // kNN cells with per-rank labels (contribution, certificate), rows of `row` bytes per cell
    void launch_cells_profile( const CellContext & c, uint32_t step, uint32_t row, uint8_t * contributed, uint8_t * certified,
                               cudaStream_t s );
    void launch_cells( const CellContext & c, uint32_t mode, cudaStream_t s );
    void launch_tasks( const CellContext & c, uint32_t * tasks, uint32_t * count, cudaStream_t s );
    void launch_vertex_validation( const CellContext & c, const uint32_t * tasks, const uint32_t * count, cudaStream_t s );
    constexpr uint32_t kMaybeWords = ( kMaxEdges + 31 ) / 32; // 9 words of edge bits per task
    constexpr uint32_t kNbrCap     = 272;                     // neighbour slots per task cell (>= the 265 a full cell can have)

    // What the edge-parallel search proved, handed to the exact pass of the same cells.
    struct SearchProof
    {
        const uint32_t * slots      = nullptr; // task index of each listed cell
        const uint32_t * maybe_bits = nullptr; // per task, bit e: edge e may have a contributor
        const uint32_t * nbr        = nullptr; // per task, the sorted neighbour ids searched against
        const uint32_t * nbr_count  = nullptr;
    };
    void launch_edge_validation( const CellContext & c, const uint32_t * tasks, const uint32_t * count, cudaStream_t s,
                                 SearchProof proof = SearchProof {} );
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

    // Exclusive scan of n u32 values in place; the total goes to *total. `sums` holds
    // output_scan_scratch_words(n) words.
    void scan_exclusive( uint32_t * data, uint32_t n, uint32_t * sums, uint64_t * total, cudaStream_t s );

    // Edge-parallel edge validation with an exact per-cell fallback (speculate.cu).
    struct SpecBuffers
    {
        uint32_t * nbr          = nullptr; // per task: sorted unique neighbour ids (64 slots)
        uint32_t * nbr_count    = nullptr;
        uint32_t * item_count   = nullptr; // per task: edges to search; scanned into item_offset
        uint32_t * item_offset  = nullptr;
        uint32_t * cell_flag    = nullptr; // 1: a contributor was found, 2: neighbour list too long
        uint32_t * exact_tasks  = nullptr; // cells re-run by the exact warp algorithm
        uint32_t * exact_slot   = nullptr; // their task index (row of maybe_bits)
        uint32_t * exact_count  = nullptr;
        uint32_t * maybe_bits   = nullptr; // per task, bit e: edge e may have a contributor
        uint64_t * item_total   = nullptr;
        uint64_t * item_counter = nullptr;
        uint32_t * scan_sums    = nullptr;
        uint2 *    heavy        = nullptr; // (task, edge) searches handed to whole warps
        uint32_t * heavy_count  = nullptr;
        uint32_t * heavy_next   = nullptr;
        uint32_t   heavy_cap    = 0;
        uint2 *    sub          = nullptr; // (search, BVH node) subtrees of long searches; the search is a
                                           // split set-up slot (high bit set) or a heavy item
        uint32_t * sub_count    = nullptr;
        uint32_t * sub_next     = nullptr;
        uint32_t   sub_cap      = 0;
        void *     splits       = nullptr; // set-up of each split search, computed once for its subtrees
        uint32_t * split_count  = nullptr;
        uint32_t   split_cap    = 0;
    };
    size_t spec_bytes( uint32_t n );
    // interval certificate of output points (certify.cu): flags (optional) and a count of the
    // points some other site is certainly closer to than their defining sites
    void launch_certify( const double4 * by_id, const double4 * sorted, const uint32_t * indices, const WideNode * nodes,
                         uint32_t n, const double4 * points, const uint4 * ids, uint32_t arity, uint64_t count, float rmax,
                         uint8_t * flags, unsigned long long * bad, uint32_t * error, cudaStream_t s );
    // relative error of output vertices against Newton-refined IEEE double solves (certify.cu):
    // per-vertex errors (optional), the largest (as the bits of a non-negative double), the
    // count above `threshold` and the count of singular systems
    void launch_vertex_error( const double4 * by_id, uint32_t n, const double4 * points, const uint4 * ids, uint64_t count,
                              double threshold, float * errors, unsigned long long * max_bits, unsigned long long * above,
                              unsigned long long * singular, cudaStream_t s );
    // grid sizes of the speculation kernels (once per process; call before concurrent builds)
    void configure_spec_kernels();
    void   spec_carve( SpecBuffers & b, void * base, uint32_t n );
    void   launch_edge_validation_speculative( const CellContext & c, const uint32_t * tasks, const uint32_t * task_count,
                                               const SpecBuffers & b, cudaStream_t s );
} // namespace apo2
