// Edge validation as an edge-parallel search with an exact fallback per cell.
//
// The reference validates the edges of a cell 32 at a time with one warp, and every
// candidate site met by any lane's BVH walk costs the whole warp a collective "is it a
// known neighbour" scan and a collective emptiness predicate over all edges
// (apo/include/apo/gpu/algorithm.inl:478-857). Almost no edge finds a contributor (a few
// per 100,000 edges on uniform clouds), and while none is found the cell does not change,
// so every edge's search sees the same cell and the searches are independent.
//
// Here each edge is one work item of a persistent kernel whose lanes fetch items one at a
// time: the walk, the neighbour test (binary search in the cell's sorted neighbour list)
// and the emptiness test (over that list) run lane-locally, with the reference's
// arithmetic and walk order. A cell none of whose edges found a contributor ends exactly
// as the reference leaves it (every edge validated, the cell validated); a cell where one
// did, or whose neighbour list is too long, is re-run from its stored state by the exact
// warp algorithm (k_edge_validation), so the result is the reference's in every case.
#include "cells.cuh"

namespace apo2
{
    constexpr uint32_t kNbrBlock      = 128; // 4 warps, one cell each
    constexpr uint32_t kSpecBlock     = 128;
    constexpr uint32_t kFlagFound     = 1;
    constexpr uint32_t kFlagOverflow  = 2;
#ifndef APO2_SPEC_LANE_BUDGET
#define APO2_SPEC_LANE_BUDGET 256
#endif
#ifndef APO2_SPEC_SPLIT_AT
#define APO2_SPEC_SPLIT_AT 192
#endif
#ifndef APO2_SPEC_MIN_BLOCKS
#define APO2_SPEC_MIN_BLOCKS 4
#endif
    constexpr uint32_t kLaneBudget    = APO2_SPEC_LANE_BUDGET; // walk steps one lane may take before the search goes to a warp
    constexpr uint32_t kHeavyBlock    = 128;
    constexpr uint32_t kHeavyStack    = 3072; // shared node stack per warp of the cooperative walk
    constexpr uint32_t kSplitAt       = APO2_SPEC_SPLIT_AT; // pending subtrees at which a long walk is handed out
    constexpr uint32_t kSplitSlot     = 0x80000000u; // marks a subtree whose search set-up is cached
#ifndef APO2_SPEC_REFILL_AT
#define APO2_SPEC_REFILL_AT 24
#endif
    // Idle lanes of a speculation warp fetch and set up new edges together, once at least
    // this many are idle (or none is walking): the set-up (bounding sphere, certificate test)
    // is long FP64 code, and run by one or two lanes at a time it held the warp for most
    // of its time.
    constexpr uint32_t kRefillAt = APO2_SPEC_REFILL_AT;

    __device__ __forceinline__ uint32_t lane_of() { return threadIdx.x & 31; }

    // Sorted unique ids of a task cell's edge sites (the set the reference's known-neighbour
    // and emptiness tests range over), and the cell's edge count for the item scan.
    __global__ void __launch_bounds__( kNbrBlock ) k_neighbor_lists( CellContext c, const uint32_t * __restrict__ tasks,
                                                                     const uint32_t * __restrict__ task_count,
                                                                     SpecBuffers b )
    {
        __shared__ uint32_t buf[ kNbrBlock / 32 ][ 1024 ];
        const uint32_t      warp  = threadIdx.x >> 5, lane = lane_of();
        const uint32_t      gwarp = blockIdx.x * ( kNbrBlock / 32 ) + warp;
        const uint32_t      nwarp = gridDim.x * ( kNbrBlock / 32 );
        const uint32_t      count = *task_count;
        uint32_t *          ids   = buf[ warp ];
        for ( uint32_t t = gwarp; t < c.n; t += nwarp )
        {
            if ( t >= count )
            {
                if ( lane == 0 )
                    b.item_count[ t ] = 0;
                continue;
            }
            const uint32_t i  = tasks[ t ];
            const uint32_t en = c.edge_nb[ i ];
            const uint8_t  st = c.status[ i ];
            if ( lane < kMaybeWords )
                b.maybe_bits[ size_t( t ) * kMaybeWords + lane ] = 0;
            if ( st == kFullyValidated || st == kBuried )
            {
                if ( lane == 0 )
                {
                    b.item_count[ t ] = 0;
                    b.cell_flag[ t ]  = 0;
                    b.nbr_count[ t ]  = 0;
                }
                continue;
            }
            const uint32_t total = 2 * en;
            uint32_t       size  = 64;
            while ( size < total )
                size <<= 1;
            for ( uint32_t x = lane; x < size; x += 32 )
            {
                uint32_t v = kNone;
                if ( x < total )
                {
                    const uint4 r = c.edges[ store_row( c, i ) * kMaxEdges + ( x >> 1 ) ];
                    v             = ( x & 1 ) ? r.y : r.x;
                }
                ids[ x ] = v;
            }
            __syncwarp();
            for ( uint32_t s2 = 2; s2 <= size; s2 <<= 1 )
                for ( uint32_t stride = s2 >> 1; stride > 0; stride >>= 1 )
                {
                    for ( uint32_t x = lane; x < size; x += 32 )
                    {
                        const uint32_t y = x ^ stride;
                        if ( y > x )
                        {
                            const uint32_t a = ids[ x ], bb = ids[ y ];
                            if ( ( a > bb ) == ( ( x & s2 ) == 0 ) )
                            {
                                ids[ x ] = bb;
                                ids[ y ] = a;
                            }
                        }
                    }
                    __syncwarp();
                }
            uint32_t kept = 0, carried = kNone;
            for ( uint32_t base = 0; base < size; base += 32 )
            {
                const uint32_t x    = base + lane;
                const uint32_t v    = ids[ x ];
                uint32_t       prev = __shfl_up_sync( 0xffffffffu, v, 1 );
                if ( lane == 0 )
                    prev = carried;
                const bool     keep = v != kNone && ( x == 0 || v != prev );
                const uint32_t bal  = __ballot_sync( 0xffffffffu, keep );
                carried             = __shfl_sync( 0xffffffffu, v, 31 );
                const uint32_t dst  = kept + __popc( bal & ( ( 1u << lane ) - 1u ) );
                if ( keep && dst < kNbrCap )
                    b.nbr[ size_t( t ) * kNbrCap + dst ] = v;
                kept += __popc( bal );
            }
            __syncwarp();
            if ( kept > kNbrCap && lane < kMaybeWords )
                b.maybe_bits[ size_t( t ) * kMaybeWords + lane ] = 0xffffffffu; // nothing decided: full exact pass
            if ( lane == 0 )
            {
                b.nbr_count[ t ]  = min( kept, kNbrCap );
                b.cell_flag[ t ]  = kept > kNbrCap ? kFlagOverflow : 0u;
                b.item_count[ t ] = kept > kNbrCap ? 0u : en;
            }
        }
    }

    __device__ __forceinline__ bool in_sorted( const uint32_t * __restrict__ list, uint32_t count, uint32_t v )
    {
        uint32_t lo = 0, hi = count;
        while ( lo < hi )
        {
            const uint32_t mid = ( lo + hi ) >> 1;
            const uint32_t x   = list[ mid ];
            if ( x == v )
                return true;
            if ( x < v )
                lo = mid + 1;
            else
                hi = mid;
        }
        return false;
    }

    // Per-lane state of one edge search.
    struct EdgeSearch
    {
        uint32_t t, e, i, k, l;
        double4  si, sk, sl;
        float4   bsph;
        float4   reach; // ball around c_i holding every possible contributor
        bool     closed;
        float3   n1, n2, pp1, pp2;
        bool     hyperbola;
        const uint32_t * nbr;
        uint32_t nbr_count;
        // the third sites of the edge's vertices: the neighbours bounding its arc, which a
        // candidate root outside the arc almost always lies inside (tested first)
        uint32_t hint[ 2 ];
    };

    // Bounding volume of edge (k, l) of cell i and the security-radius test
    // (algorithm.inl:555-614). Returns false when the edge needs no search.
    __device__ __forceinline__ bool setup_edge( const CellContext & c, EdgeSearch & s, float known )
    {
        uint32_t type = 0;
        double4  ev0 = make_double4( 0, 0, 0, 0 ), ev1 = make_double4( 0, 0, 0, 0 );
        type          = trisector( s.si, s.sk, s.sl, ev0, ev1 );
        s.hyperbola   = type == 1;
        const bool   ellipse = type == 2;
        const float4 v1 = to_float( ev0 ), v2 = to_float( ev1 );
        s.n1 = s.n2 = s.pp1 = s.pp2 = make_float3( 0, 0, 0 );
        if ( ellipse )
        {
            const float3 center = ( f3( v1 ) + f3( v2 ) ) * .5f;
            const float  radius = flength( center - f3( v1 ) ) + v1.w;
            s.bsph              = make_float4( center.x, center.y, center.z, radius );
        }
        else
        {
            double3 nn1, nn2;
            tangent_planes( s.si, s.sk, s.sl, nn1, nn2 );
            s.n1             = to_float( nn1 );
            s.n2             = to_float( nn2 );
            const double3 p1 = d3( s.si ) + nn1 * s.si.w;
            const double3 p2 = d3( s.sk ) + nn1 * s.sk.w;
            const double3 p3 = d3( s.sl ) + nn1 * s.sl.w;
            const double3 p4 = d3( s.si ) + nn2 * s.si.w;
            const double3 p5 = d3( s.sk ) + nn2 * s.sk.w;
            s.bsph           = to_float( sphere_from_points( p1, p2, p3, p5 ) );
            s.pp1            = to_float( p1 );
            s.pp2            = to_float( p4 );
        }
        const float4 fsi    = to_float( s.si );
        const bool   inside = lt_eps( flength( f3( fsi ) - f3( s.bsph ) ), known - s.bsph.w );
        if ( inside )
            return false;

        // reach of the search: largest radius over the edge's arc
        double         wmax = 0.0;
        const uint32_t vn   = c.vertex_nb[ s.i ];
        s.hint[ 0 ] = s.hint[ 1 ] = kNone;
        for ( uint32_t v = 0; v < vn; v++ )
        {
            const uint4 r = c.vertices[ store_row( c, s.i ) * kMaxVertices + v ];
            if ( vertex_on_edge( r, s.k, s.l ) )
            {
                wmax             = fmax( wmax, solve_vertex( c, s.si, r ).w );
                const uint32_t m = ( r.x != s.k && r.x != s.l ) ? r.x : ( ( r.y != s.k && r.y != s.l ) ? r.y : r.z );
                if ( s.hint[ 0 ] == kNone )
                    s.hint[ 0 ] = m;
                else if ( s.hint[ 1 ] == kNone && m != s.hint[ 0 ] )
                    s.hint[ 1 ] = m;
            }
        }
        if ( ellipse || s.closed )
        {
            const double4 apex[ 2 ] = { ev0, ev1 };
            for ( uint32_t a = 0; a < 2; a++ )
            {
                bool out = false;
                for ( uint32_t q = 0; q < s.nbr_count && !out; q++ )
                {
                    const uint32_t u = s.nbr[ q ];
                    if ( u != s.k && u != s.l )
                        out = clearly_outside( c.sites[ u ], apex[ a ] );
                }
                if ( !out )
                    wmax = fmax( wmax, apex[ a ].w );
            }
        }
        s.reach = make_float4( fsi.x, fsi.y, fsi.z, reach_radius( wmax, s.si.w, c.scene->rmax ) );
        return true;
    }

    // The reference's test for entering a child box (algorithm.inl:642-667: the box meets
    // the bounding sphere and, for a hyperbolic edge, the closest point of the box lies
    // below both tangent planes), and the reach test (skipping keeps the visit order).
    __device__ __forceinline__ bool enter_child( const EdgeSearch & s, const Box & b, float d )
    {
        bool enter = d < 0.f;
        if ( s.hyperbola && enter )
        {
            const float3 p = b.closest( s.bsph );
            enter          = fdot( s.n1, p - s.pp1 ) < 0.f && fdot( s.n2, p - s.pp2 ) < 0.f;
        }
        return enter && b.distance( s.reach ) < 0.f;
    }

    // Does site j give the edge two vertices, one of them empty of every other neighbour?
    // (algorithm.inl:683-774, with the known-neighbour and emptiness tests lane-local.)
    __device__ __forceinline__ bool contributes( const CellContext & c, const EdgeSearch & s, uint32_t j )
    {
        if ( j == s.i || j == s.k || j == s.l || c.status[ j ] == kBuried )
            return false;
        const double4 sj = c.sites[ j ];
        const float4  fj = to_float( sj );
        if ( !intersects( fj, s.bsph ) )
            return false;
        if ( flength( f3( fj ) - f3( s.reach ) ) > s.reach.w )
            return false;
        if ( s.hyperbola
             && !( double( fdot( s.n1, f3( fj ) - s.pp1 ) ) < -sj.w && double( fdot( s.n2, f3( fj ) - s.pp2 ) ) < -sj.w ) )
            return false;
        if ( in_sorted( s.nbr, s.nbr_count, j ) )
            return false;
        double4        x[ 2 ] = { make_double4( 0, 0, 0, 0 ), make_double4( 0, 0, 0, 0 ) };
        const uint32_t mask   = quadrisector( s.si, sj, s.sk, s.sl, x[ 0 ], x[ 1 ] );
        if ( mask != 3 )
            return false;
        // the FP32 filter decides here too; its counts are kept for the cell kernels only
        FilterTally untallied;
        // A root is empty when no neighbour other than k, l conflicts with it: the neighbours
        // bounding the edge's arc go first (a root outside the arc is nearly always inside one of
        // them), then the whole sorted list. The conjunction is the same.
        bool hint_ok[ 2 ] = { false, false };
        for ( uint32_t h = 0; h < 2; h++ )
            hint_ok[ h ] = s.hint[ h ] != kNone && in_sorted( s.nbr, s.nbr_count, s.hint[ h ] );
        for ( uint32_t r = 0; r < 2; r++ )
        {
            bool ok = true;
            for ( uint32_t h = 0; h < 2 && ok; h++ )
                if ( hint_ok[ h ] )
                    ok = !site_conflict( c, s.hint[ h ], x[ r ], untallied );
            for ( uint32_t q = 0; q < s.nbr_count && ok; q++ )
            {
                const uint32_t u = s.nbr[ q ];
                if ( u != s.k && u != s.l )
                    ok = !site_conflict( c, u, x[ r ], untallied );
            }
            if ( ok )
                return true;
        }
        return false;
    }

    __global__ void __launch_bounds__( kSpecBlock, APO2_SPEC_MIN_BLOCKS ) k_edge_speculate( CellContext c, const uint32_t * __restrict__ tasks,
                                                                      const uint32_t * __restrict__ task_count,
                                                                      SpecBuffers b, uint32_t * error )
    {
        const uint32_t count = *task_count;
        if ( count == 0 )
            return;
        const uint64_t total = *b.item_total;
        const uint32_t n     = c.n;
        uint32_t       err   = 0;

        EdgeSearch s;
        bool       active    = false;
        bool       exhausted = false; // the queue is empty for this lane
        uint32_t   stack[ kStack ];
        int        sp    = 0;
        uint32_t   node  = 0;
        uint32_t   steps = 0;
        while ( true )
        {
            // warp-uniform choice between a refill round and a walk step
            const uint32_t idle = __ballot_sync( 0xffffffffu, !active && !exhausted );
            const uint32_t busy = __ballot_sync( 0xffffffffu, active );
            if ( idle == 0 && busy == 0 )
                break;
            if ( idle != 0 && ( busy == 0 || uint32_t( __popc( idle ) ) >= kRefillAt ) )
            {
                if ( !active && !exhausted )
                {
                    // warp-aggregated fetch of the next item by the idle lanes
                    const uint32_t leader = __ffs( idle ) - 1;
                    uint64_t       base   = 0;
                    if ( lane_of() == leader )
                        base = atomicAdd( reinterpret_cast<unsigned long long *>( b.item_counter ), __popc( idle ) );
                    base                = __shfl_sync( idle, base, leader );
                    const uint64_t item = base + __popc( idle & ( ( 1u << lane_of() ) - 1u ) );
                    if ( item >= total )
                        exhausted = true;
                    else
                    {
                        // task holding this item: last t with offset[t] <= item
                        uint32_t lo = 0, hi = count;
                        while ( hi - lo > 1 )
                        {
                            const uint32_t mid = ( lo + hi ) >> 1;
                            if ( b.item_offset[ mid ] <= item )
                                lo = mid;
                            else
                                hi = mid;
                        }
                        s.t              = lo;
                        const uint32_t e = uint32_t( item - b.item_offset[ s.t ] );
                        s.e              = e;
                        if ( b.cell_flag[ s.t ] & kFlagOverflow )
                        {
                            // no neighbour list for this cell: the exact path searches this edge
                            atomicOr( &b.maybe_bits[ size_t( s.t ) * kMaybeWords + ( e >> 5 ) ], 1u << ( e & 31 ) );
                        }
                        else
                        {
                            s.i           = tasks[ s.t ];
                            const uint4 r = c.edges[ store_row( c, s.i ) * kMaxEdges + e ];
                            s.k           = r.x;
                            s.l           = r.y;
                            s.closed      = r.z == kNone;
                            s.si          = c.sites[ s.i ];
                            s.nbr         = b.nbr + size_t( s.t ) * kNbrCap;
                            s.nbr_count   = b.nbr_count[ s.t ];
                            // an edge validated before is not searched (algorithm.inl:522-526, 552)
                            if ( ( r.w & 0xffu ) != 1u )
                            {
                                s.sk = c.sites[ s.k ];
                                s.sl = c.sites[ s.l ];
                                if ( setup_edge( c, s, c.known_radii[ s.i ] ) )
                                {
                                    active = true;
                                    sp     = 0;
                                    node   = 0;
                                    steps  = 0;
                                }
                            }
                        }
                    }
                }
                continue;
            }
            if ( !active )
                continue;

            // one step of the walk: descend to a leaf (or prune), test it, pop
            if ( ++steps > kLaneBudget )
            {
                // a long search: restart it on a whole warp (k_edge_heavy)
                const uint32_t slot = atomicAdd( b.heavy_count, 1u );
                if ( slot < b.heavy_cap )
                    b.heavy[ slot ] = make_uint2( s.t, s.e );
                else
                {
                    // exact path instead, with a full search of this edge
                    atomicOr( &b.maybe_bits[ size_t( s.t ) * kMaybeWords + ( s.e >> 5 ) ], 1u << ( s.e & 31 ) );
                    atomicOr( &b.cell_flag[ s.t ], kFlagFound );
                }
                active = false;
                continue;
            }
            while ( node < n - 1 )
            {
                Box      lb, rb;
                uint32_t lc, rc;
                load_node( c.nodes, node, lb, rb, lc, rc );
                const float    dL = lb.distance( s.bsph ), dR = rb.distance( s.bsph );
                const bool     leftClosest = dL < dR;
                const uint32_t farChild = leftClosest ? rc : lc, closeChild = leftClosest ? lc : rc;
                const bool     exploreL = enter_child( s, lb, dL ), exploreR = enter_child( s, rb, dR );
                const bool     exploreFar = leftClosest ? exploreR : exploreL, exploreClose = leftClosest ? exploreL : exploreR;
                if ( !exploreFar && !exploreClose )
                    break;
                node = exploreClose ? closeChild : farChild;
                if ( exploreClose && exploreFar )
                {
                    if ( sp < int( kStack ) )
                        stack[ sp++ ] = farChild;
                    else
                        err |= kErrStack;
                }
            }
            if ( node >= n - 1 && node < 2 * n - 1 && contributes( c, s, node - ( n - 1 ) ) )
            {
                atomicOr( &b.maybe_bits[ size_t( s.t ) * kMaybeWords + ( s.e >> 5 ) ], 1u << ( s.e & 31 ) );
                atomicOr( &b.cell_flag[ s.t ], kFlagFound );
                active = false;
                continue;
            }
            if ( sp == 0 )
                active = false;
            else
                node = stack[ --sp ];
        }
        if ( err )
            atomicOr( error, err );
    }

    // Searches that outgrew one lane: the warp walks the tree together, 32 nodes per step
    // from a shared stack. Only whether a contributor exists matters here, which does not
    // depend on the visit order, so a long walk can also be cut into subtrees that other
    // warps finish (k_edge_heavy spills its stack once it holds kSplitAt nodes; k_edge_heavy_sub
    // walks each spilled subtree).
    enum WalkEnd : uint32_t
    {
        kWalkDone,
        kWalkFound,
        kWalkOverflow,
        kWalkSplit
    };

    __device__ uint32_t cooperative_walk( const CellContext & c, const EdgeSearch & s, uint32_t * st, uint32_t & size,
                                          uint32_t split_at )
    {
        const uint32_t lane = lane_of();
        const uint32_t n    = c.n;
        while ( size > 0 )
        {
            if ( size >= split_at )
                return kWalkSplit;
            const uint32_t take = min( size, 32u );
            uint32_t       node = kNone;
            if ( lane < take )
                node = st[ size - take + lane ];
            size -= take;
            __syncwarp();
            bool     hit = false, eL = false, eR = false;
            uint32_t lc = 0, rc = 0;
            if ( node != kNone )
            {
                if ( node >= n - 1 )
                    hit = node < 2 * n - 1 && contributes( c, s, node - ( n - 1 ) );
                else
                {
                    Box lb, rb;
                    load_node( c.nodes, node, lb, rb, lc, rc );
                    eL = enter_child( s, lb, lb.distance( s.bsph ) );
                    eR = enter_child( s, rb, rb.distance( s.bsph ) );
                }
            }
            if ( __any_sync( 0xffffffffu, hit ) )
                return kWalkFound;
            const uint32_t pushes = uint32_t( eL ) + uint32_t( eR );
            uint32_t       x      = pushes;
#pragma unroll
            for ( int o = 1; o < 32; o <<= 1 )
            {
                const uint32_t y = __shfl_up_sync( 0xffffffffu, x, o );
                if ( lane >= uint32_t( o ) )
                    x += y;
            }
            const uint32_t total = __shfl_sync( 0xffffffffu, x, 31 );
            uint32_t       off   = x - pushes;
            if ( size + total > kHeavyStack )
                return kWalkOverflow;
            if ( eL )
                st[ size + off++ ] = lc;
            if ( eR )
                st[ size + off ] = rc;
            size += total;
            __syncwarp();
        }
        return kWalkDone;
    }

    __device__ __forceinline__ void search_of_heavy( const CellContext & c, const uint32_t * tasks, const SpecBuffers & b,
                                                     uint2 h, EdgeSearch & s )
    {
        s.t           = h.x;
        s.e           = h.y;
        s.i           = tasks[ s.t ];
        const uint4 r = c.edges[ store_row( c, s.i ) * kMaxEdges + s.e ];
        s.k           = r.x;
        s.l           = r.y;
        s.closed      = r.z == kNone;
        s.si          = c.sites[ s.i ];
        s.sk          = c.sites[ s.k ];
        s.sl          = c.sites[ s.l ];
        s.nbr         = b.nbr + size_t( s.t ) * kNbrCap;
        s.nbr_count   = b.nbr_count[ s.t ];
        setup_edge( c, s, c.known_radii[ s.i ] ); // the lane path already found it needs a search
    }

    __device__ __forceinline__ void send_to_exact( const SpecBuffers & b, uint32_t t, uint32_t e )
    {
        // the exact path decides, searching this edge again
        atomicOr( &b.maybe_bits[ size_t( t ) * kMaybeWords + ( e >> 5 ) ], 1u << ( e & 31 ) );
        atomicOr( &b.cell_flag[ t ], kFlagFound );
    }

    __global__ void __launch_bounds__( kHeavyBlock, 4 ) k_edge_heavy( CellContext c, const uint32_t * __restrict__ tasks,
                                                                      SpecBuffers b, uint32_t * error )
    {
        __shared__ uint32_t stacks[ kHeavyBlock / 32 ][ kHeavyStack ];
        const uint32_t      warp  = threadIdx.x >> 5, lane = lane_of();
        uint32_t *          st    = stacks[ warp ];
        const uint32_t      count = min( *b.heavy_count, b.heavy_cap );
        while ( true )
        {
            uint32_t item = 0;
            if ( lane == 0 )
                item = atomicAdd( b.heavy_next, 1u );
            item = __shfl_sync( 0xffffffffu, item, 0 );
            if ( item >= count )
                break;
            const uint2 h = b.heavy[ item ];
            // Edges of a cell that already goes to the exact path are still searched: every
            // edge proven empty here is one the exact pass skips.
            if ( b.cell_flag[ h.x ] & kFlagOverflow )
            {
                if ( lane == 0 )
                    atomicOr( &b.maybe_bits[ size_t( h.x ) * kMaybeWords + ( h.y >> 5 ) ], 1u << ( h.y & 31 ) );
                continue;
            }
            EdgeSearch s;
            search_of_heavy( c, tasks, b, h, s );
            uint32_t size = 1;
            if ( lane == 0 )
                st[ 0 ] = 0;
            __syncwarp();
            const uint32_t end = cooperative_walk( c, s, st, size, kSplitAt );
            if ( end == kWalkSplit )
            {
                // hand the pending subtrees to other warps, with the search's set-up computed once
                // for all of them (a full slot table leaves them to recompute it)
                uint32_t base = 0, slot = 0;
                if ( lane == 0 )
                {
                    base = atomicAdd( b.sub_count, size );
                    slot = atomicAdd( b.split_count, 1u );
                    if ( slot < b.split_cap )
                        static_cast<EdgeSearch *>( b.splits )[ slot ] = s;
                }
                base = __shfl_sync( 0xffffffffu, base, 0 );
                slot = __shfl_sync( 0xffffffffu, slot, 0 );
                const uint32_t search = slot < b.split_cap ? ( slot | kSplitSlot ) : item;
                if ( base + size <= b.sub_cap )
                {
                    for ( uint32_t q = lane; q < size; q += 32 )
                        b.sub[ base + q ] = make_uint2( search, st[ q ] );
                }
                else if ( lane == 0 )
                    send_to_exact( b, s.t, s.e );
            }
            else if ( ( end == kWalkFound || end == kWalkOverflow ) && lane == 0 )
                send_to_exact( b, s.t, s.e );
            __syncwarp();
        }
    }

    __global__ void __launch_bounds__( kHeavyBlock, 4 ) k_edge_heavy_sub( CellContext c, const uint32_t * __restrict__ tasks,
                                                                          SpecBuffers b, uint32_t * error )
    {
        __shared__ uint32_t stacks[ kHeavyBlock / 32 ][ kHeavyStack ];
        const uint32_t      warp  = threadIdx.x >> 5, lane = lane_of();
        uint32_t *          st    = stacks[ warp ];
        const uint32_t      count = min( *b.sub_count, b.sub_cap );
        while ( true )
        {
            uint32_t q = 0;
            if ( lane == 0 )
                q = atomicAdd( b.sub_next, 1u );
            q = __shfl_sync( 0xffffffffu, q, 0 );
            if ( q >= count )
                break;
            const uint2 sub    = b.sub[ q ];
            const bool  cached = ( sub.x & kSplitSlot ) != 0;
            EdgeSearch  s;
            uint2       h;
            if ( cached )
            {
                s = static_cast<const EdgeSearch *>( b.splits )[ sub.x & ~kSplitSlot ];
                h = make_uint2( s.t, s.e );
            }
            else
                h = b.heavy[ sub.x ];
            // another part of this edge's search already found a contributor
            if ( ( b.cell_flag[ h.x ] & kFlagOverflow )
                 || ( ( b.maybe_bits[ size_t( h.x ) * kMaybeWords + ( h.y >> 5 ) ] >> ( h.y & 31 ) ) & 1u ) )
            {
                if ( lane == 0 )
                    atomicOr( &b.maybe_bits[ size_t( h.x ) * kMaybeWords + ( h.y >> 5 ) ], 1u << ( h.y & 31 ) );
                continue;
            }
            if ( !cached )
                search_of_heavy( c, tasks, b, h, s );
            uint32_t size = 1;
            if ( lane == 0 )
                st[ 0 ] = sub.y;
            __syncwarp();
            const uint32_t end = cooperative_walk( c, s, st, size, kHeavyStack + 1 );
            if ( ( end == kWalkFound || end == kWalkOverflow ) && lane == 0 )
                send_to_exact( b, s.t, s.e );
            __syncwarp();
        }
    }

    // Cells with no contributor are final: every edge validated, the cell validated
    // (what the reference's pass leaves when no update happens). The others are listed for
    // the exact pass.
    __global__ void k_edge_commit( CellContext c, const uint32_t * __restrict__ tasks, const uint32_t * __restrict__ task_count,
                                   SpecBuffers b )
    {
        const uint32_t gwarp = ( blockIdx.x * blockDim.x + threadIdx.x ) >> 5;
        const uint32_t nwarp = ( gridDim.x * blockDim.x ) >> 5;
        const uint32_t lane  = lane_of();
        const uint32_t count = *task_count;
        for ( uint32_t t = gwarp; t < count; t += nwarp )
        {
            const uint32_t i  = tasks[ t ];
            const uint8_t  st = c.status[ i ];
            if ( st == kFullyValidated || st == kBuried )
                continue;
            if ( b.cell_flag[ t ] )
            {
                if ( lane == 0 )
                {
                    const uint32_t q  = atomicAdd( b.exact_count, 1u );
                    b.exact_tasks[ q ] = i;
                    b.exact_slot[ q ]  = t;
                }
                continue;
            }
            const uint32_t en = c.edge_nb[ i ];
            for ( uint32_t e = lane; e < en; e += 32 )
            {
                uint32_t * w = &c.edges[ store_row( c, i ) * kMaxEdges + e ].w;
                *w           = ( *w & 0xffffff00u ) | 1u;
            }
            if ( lane == 0 )
                c.status[ i ] = kFullyValidated;
        }
    }

    // long lane searches per round: log-normal radii reach 1.5 per site
    static size_t heavy_capacity( uint32_t n ) { return 6 * size_t( n ) + 65536; }
    static size_t sub_capacity( uint32_t n ) { return 4 * size_t( n ) + 65536; }
    // searches split into subtrees per round (each hands out up to kSplitAt subtrees)
    static size_t split_capacity( uint32_t n ) { return size_t( n ) / 8 + 4096; }

    size_t spec_bytes( uint32_t n )
    {
        auto a = []( size_t x ) { return ( x + 255 ) & ~size_t( 255 ); };
        return a( 4 * size_t( n ) * kNbrCap ) + a( 4 * size_t( n ) ) * 4 + a( 4 * size_t( n ) ) + a( 16 ) * 3
               + a( 4 * output_scan_scratch_words( n ) ) + a( sizeof( uint2 ) * heavy_capacity( n ) ) + a( 16 ) * 2
               + a( 4 * size_t( n ) * kMaybeWords ) + a( sizeof( uint2 ) * sub_capacity( n ) ) + a( 16 ) * 2
               + a( sizeof( EdgeSearch ) * split_capacity( n ) ) + a( 16 );
    }

    void spec_carve( SpecBuffers & b, void * base, uint32_t n )
    {
        auto   a = []( size_t x ) { return ( x + 255 ) & ~size_t( 255 ); };
        char * p = static_cast<char *>( base );
        b.nbr    = reinterpret_cast<uint32_t *>( p );
        p += a( 4 * size_t( n ) * kNbrCap );
        b.nbr_count = reinterpret_cast<uint32_t *>( p );
        p += a( 4 * size_t( n ) );
        b.item_count = reinterpret_cast<uint32_t *>( p ); // becomes the offsets after the scan
        b.item_offset = b.item_count;
        p += a( 4 * size_t( n ) );
        b.cell_flag = reinterpret_cast<uint32_t *>( p );
        p += a( 4 * size_t( n ) );
        b.exact_tasks = reinterpret_cast<uint32_t *>( p );
        p += a( 4 * size_t( n ) );
        b.exact_slot = reinterpret_cast<uint32_t *>( p );
        p += a( 4 * size_t( n ) );
        b.item_total = reinterpret_cast<uint64_t *>( p );
        p += a( 16 );
        b.item_counter = reinterpret_cast<uint64_t *>( p );
        p += a( 16 );
        b.exact_count = reinterpret_cast<uint32_t *>( p );
        p += a( 16 );
        b.scan_sums = reinterpret_cast<uint32_t *>( p );
        p += a( 4 * output_scan_scratch_words( n ) );
        b.heavy = reinterpret_cast<uint2 *>( p );
        p += a( sizeof( uint2 ) * heavy_capacity( n ) );
        b.heavy_count = reinterpret_cast<uint32_t *>( p );
        p += a( 16 );
        b.heavy_next = reinterpret_cast<uint32_t *>( p );
        p += a( 16 );
        b.maybe_bits = reinterpret_cast<uint32_t *>( p );
        p += a( 4 * size_t( n ) * kMaybeWords );
        b.sub = reinterpret_cast<uint2 *>( p );
        p += a( sizeof( uint2 ) * sub_capacity( n ) );
        b.sub_count = reinterpret_cast<uint32_t *>( p );
        p += a( 16 );
        b.sub_next  = reinterpret_cast<uint32_t *>( p );
        p += a( 16 );
        b.splits = p;
        p += a( sizeof( EdgeSearch ) * split_capacity( n ) );
        b.split_count = reinterpret_cast<uint32_t *>( p );
        b.split_cap   = uint32_t( split_capacity( n ) );
        b.sub_cap   = uint32_t( sub_capacity( n ) );
        b.heavy_cap = uint32_t( heavy_capacity( n ) );
    }

    // Persistent grid sizes per device (148 SMs x resident blocks of each kernel on B200).
    constexpr int        kSpecDevices = 64;
    static int           g_spec_grid[ kSpecDevices ], g_heavy_grid[ kSpecDevices ];
    static PerDeviceOnce g_spec_config;

    static int spec_device()
    {
        int dev = 0;
        cudaGetDevice( &dev );
        return ( dev >= 0 && dev < kSpecDevices ) ? dev : -1;
    }

    void configure_spec_kernels()
    {
        g_spec_config.run( [] {
            const int dev = spec_device();
            if ( dev < 0 )
                return;
            int sms = 148, per_sm = 0;
            cudaDeviceGetAttribute( &sms, cudaDevAttrMultiProcessorCount, dev );
            cudaOccupancyMaxActiveBlocksPerMultiprocessor( &per_sm, k_edge_speculate, kSpecBlock, 0 );
            g_spec_grid[ dev ] = sms * std::max( 1, per_sm );
            cudaOccupancyMaxActiveBlocksPerMultiprocessor( &per_sm, k_edge_heavy, kHeavyBlock, 0 );
            g_heavy_grid[ dev ] = sms * std::max( 1, per_sm );
        } );
    }

    void launch_edge_validation_speculative( const CellContext & c, const uint32_t * tasks, const uint32_t * task_count,
                                             const SpecBuffers & b, cudaStream_t s )
    {
        configure_spec_kernels();
        const int dev        = spec_device();
        const int spec_grid  = dev >= 0 ? g_spec_grid[ dev ] : 148 * 4; // an ordinal outside the table
        const int heavy_grid = dev >= 0 ? g_heavy_grid[ dev ] : 148 * 4;
        const uint32_t nbr_blocks = std::max( 1u, std::min<uint32_t>( ( c.n + 3 ) / 4, 148 * 32 ) );
        APO2_LAUNCH( "k_neighbor_lists", s, k_neighbor_lists<<<nbr_blocks, kNbrBlock, 0, s>>>( c, tasks, task_count, b ) );
        scan_exclusive( b.item_count, c.n, b.scan_sums, b.item_total, s );
        cudaMemsetAsync( b.item_counter, 0, sizeof( uint64_t ), s );
        cudaMemsetAsync( b.exact_count, 0, sizeof( uint32_t ), s );
        cudaMemsetAsync( b.heavy_count, 0, sizeof( uint32_t ), s );
        cudaMemsetAsync( b.heavy_next, 0, sizeof( uint32_t ), s );
        cudaMemsetAsync( b.sub_count, 0, sizeof( uint32_t ), s );
        cudaMemsetAsync( b.sub_next, 0, sizeof( uint32_t ), s );
        cudaMemsetAsync( b.split_count, 0, sizeof( uint32_t ), s );
        APO2_LAUNCH( "k_edge_speculate", s, k_edge_speculate<<<spec_grid, kSpecBlock, 0, s>>>( c, tasks, task_count, b, c.error ) );
        APO2_LAUNCH( "k_edge_heavy", s, k_edge_heavy<<<heavy_grid, kHeavyBlock, 0, s>>>( c, tasks, b, c.error ) );
        APO2_LAUNCH( "k_edge_heavy_sub", s, k_edge_heavy_sub<<<heavy_grid, kHeavyBlock, 0, s>>>( c, tasks, b, c.error ) );
        APO2_LAUNCH( "k_edge_commit", s, k_edge_commit<<<std::max( 1u, std::min<uint32_t>( ( c.n + 7 ) / 8, 148 * 16 ) ), 256, 0, s>>>( c, tasks, task_count, b ) );
        SearchProof proof;
        proof.slots      = b.exact_slot;
        proof.maybe_bits = b.maybe_bits;
        proof.nbr        = b.nbr;
        proof.nbr_count  = b.nbr_count;
        launch_edge_validation( c, b.exact_tasks, b.exact_count, s, proof );
    }
} // namespace apo2
