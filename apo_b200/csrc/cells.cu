// Cell construction: kNN search, warp-per-cell cell update with the security-radius
// certificate, the vertex / edge / bisector validation passes and the output extraction.
//
// The decisions follow the reference step for step (apo/include/apo/gpu/topology_update.inl
// and algorithm.inl, cited per function), so every per-cell store ends with the same
// records in the same order. What differs is how the work maps onto a B200 SM:
//   - each warp keeps its cell in shared memory together with the FP64 position of every
//     vertex, solved once when the vertex is created instead of at every later use (the
//     reference re-solves each vertex's quadrisector in every cell update, every radius
//     evaluation and every validation step);
//   - the initial bounding cell is synthesised in shared memory, not written to and read
//     back from the per-cell store;
//   - BVH walks read 64-byte wide nodes;
//   - the validation rounds read their task count from device memory, so the whole build
//     runs without a host round trip and can be captured in one CUDA graph;
//   - each validation predicate leaves its edge loop as soon as one lane found a conflict.
#include "cells.cuh"

namespace apo2
{
    constexpr uint32_t kFull        = 0xffffffffu;
    constexpr uint32_t kMaxRestarts = 4096; // bound of the restart loops of the edge / bisector passes

    __device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31; }
    __device__ __forceinline__ uint32_t highest( uint32_t m ) { return 31u - __clz( m ); }

    __device__ __forceinline__ double4 shfl4( double4 v, int src )
    {
        return make_double4( __shfl_sync( kFull, v.x, src ), __shfl_sync( kFull, v.y, src ), __shfl_sync( kFull, v.z, src ),
                             __shfl_sync( kFull, v.w, src ) );
    }
    __device__ __forceinline__ float4 shfl4( float4 v, int src )
    {
        return make_float4( __shfl_sync( kFull, v.x, src ), __shfl_sync( kFull, v.y, src ), __shfl_sync( kFull, v.z, src ),
                            __shfl_sync( kFull, v.w, src ) );
    }

    __device__ __forceinline__ uint32_t warp_exclusive_scan( uint32_t v, uint32_t & total )
    {
        const uint32_t lane = lane_id();
        uint32_t       x    = v;
#pragma unroll
        for ( int o = 1; o < 32; o <<= 1 )
        {
            const uint32_t y = __shfl_up_sync( kFull, x, o );
            if ( lane >= uint32_t( o ) )
                x += y;
        }
        total = __shfl_sync( kFull, x, 31 );
        return x - v;
    }

    __device__ __forceinline__ double4 site( const CellContext & c, uint32_t id ) { return c.sites[ id ]; }

    // -----------------------------------------------------------------------------------
    // The cell of one warp, in shared memory
    // -----------------------------------------------------------------------------------
    struct WarpCell
    {
        uint4 * v;       // (j, k, l, type | status << 8), capacity kVertexSlots
        double4 * pos;   // solved position of v[*]
        uint4 * e;       // (j, k, vertex count, status | validated << 8), capacity kEdgeSlots
        uint32_t vn, en; // warp-uniform sizes
        mutable FilterTally tally; // this lane's FP32-filter counts
    };

    __device__ __forceinline__ uint32_t vstatus( uint4 r ) { return ( r.w >> 8 ) & 0xffu; }
    __device__ __forceinline__ uint32_t vtype( uint4 r ) { return r.w & 0xffu; }
    __device__ __forceinline__ uint32_t estatus( uint4 r ) { return r.w & 0xffu; }


    // Default validation predicate of the cell update (topology_update.inl:578-592): no site
    // of the cell's edges other than skip1 / skip2 intersects `sphere`. Warp-collective;
    // returns the warp-wide result. The reference tests every edge; the loop stops once a
    // conflict is known, which does not change the result.
    __device__ __forceinline__ bool edges_clear( const CellContext & c, const WarpCell & w, double4 sphere, uint32_t skip1,
                                                 uint32_t skip2 )
    {
        bool ok = true;
        for ( uint32_t base = 0; base < w.en; base += 32 )
        {
            const uint32_t e = base + lane_id();
            if ( e < w.en )
            {
                const uint4 r = w.e[ e ];
                if ( r.x != skip1 && r.x != skip2 )
                    ok = ok && !site_conflict( c, r.x, sphere, w.tally );
                if ( r.y != skip1 && r.y != skip2 )
                    ok = ok && !site_conflict( c, r.y, sphere, w.tally );
            }
            if ( !__all_sync( kFull, ok ) )
                return false;
        }
        return true;
    }

#ifndef APO2_LANE_CLEAR_EDGES
#define APO2_LANE_CLEAR_EDGES 8
#endif
    // cells with at most this many edges check new roots lane by lane in update_cell
    constexpr uint32_t kLaneClearEdges = APO2_LANE_CLEAR_EDGES;

    // Lane-local forms of is_known / edges_clear (same predicates, one lane scanning all edges).
    __device__ __forceinline__ bool known_by_lane( const WarpCell & w, uint32_t id )
    {
        for ( uint32_t e = 0; e < w.en; e++ )
        {
            const uint4 r = w.e[ e ];
            if ( r.x == id || r.y == id )
                return true;
        }
        return false;
    }
    __device__ __forceinline__ bool clear_by_lane( const CellContext & c, const WarpCell & w, double4 sphere, uint32_t skip1,
                                                   uint32_t skip2 )
    {
        for ( uint32_t e = 0; e < w.en; e++ )
        {
            const uint4 r = w.e[ e ];
            if ( r.x != skip1 && r.x != skip2 && site_conflict( c, r.x, sphere, w.tally ) )
                return false;
            if ( r.y != skip1 && r.y != skip2 && site_conflict( c, r.y, sphere, w.tally ) )
                return false;
        }
        return true;
    }

    // Is `id` already a neighbour of the cell (one of its edges' sites)? Warp-collective.
    __device__ __forceinline__ bool is_known( const WarpCell & w, uint32_t id )
    {
        for ( uint32_t base = 0; base < w.en; base += 32 )
        {
            const uint32_t e   = base + lane_id();
            bool           hit = false;
            if ( e < w.en )
            {
                const uint4 r = w.e[ e ];
                hit           = r.x == id || r.y == id;
            }
            if ( __any_sync( kFull, hit ) )
                return true;
        }
        return false;
    }

    // New-edge candidates, two per lane, packed as (site << 2) | (two roots << 1) | closed so
    // that an unsigned sort orders them by site (topology_update.inl:56-74).
    constexpr uint32_t kNoEdge = ( 0x0fffffffu << 2 ) | 3u;
    __device__ __forceinline__ uint32_t pack_edge( uint32_t k, bool two, bool closed )
    {
        return ( ( k & 0x3fffffffu ) << 2 ) | ( two ? 2u : 0u ) | ( closed ? 1u : 0u );
    }

    struct NewEdges
    {
        uint32_t slot[ 2 ];
        uint32_t count; // warp-uniform
        __device__ __forceinline__ void push( uint32_t k, bool two, bool closed, uint32_t & err )
        {
            if ( count < kMaxNewEdges )
            {
                if ( lane_id() == count / 2 )
                    slot[ count & 1 ] = pack_edge( k, two, closed );
            }
            else
                err |= kErrNewEdgeCap;
            count++;
        }
        __device__ __forceinline__ bool contains( uint32_t k ) const
        {
            const bool hit = ( slot[ 0 ] >> 2 ) == k || ( slot[ 1 ] >> 2 ) == k;
            return __any_sync( kFull, hit );
        }
    };

    // Ascending bitonic sort of the 64 packed candidates (element 2*lane + s in slot[s]).
    __device__ __forceinline__ void sort64( uint32_t ( &a )[ 2 ] )
    {
        const uint32_t lane = lane_id();
#pragma unroll
        for ( uint32_t size = 2; size <= 64; size <<= 1 )
        {
#pragma unroll
            for ( uint32_t stride = size >> 1; stride > 0; stride >>= 1 )
            {
                if ( stride == 1 )
                {
                    const bool up = ( ( 2 * lane ) & size ) == 0;
                    if ( ( a[ 0 ] > a[ 1 ] ) == up )
                    {
                        const uint32_t t = a[ 0 ];
                        a[ 0 ]           = a[ 1 ];
                        a[ 1 ]           = t;
                    }
                }
                else
                {
#pragma unroll
                    for ( uint32_t s = 0; s < 2; s++ )
                    {
                        const uint32_t f     = 2 * lane + s;
                        const uint32_t other = __shfl_xor_sync( kFull, a[ s ], stride >> 1 );
                        const bool     lower = ( f & stride ) == 0;
                        const bool     up    = ( f & size ) == 0;
                        a[ s ]               = ( lower == up ) ? min( a[ s ], other ) : max( a[ s ], other );
                    }
                }
            }
        }
    }

    // Flags a store that went past the reference's capacity; records written beyond the
    // shared slots are dropped.
    __device__ __forceinline__ void check_capacity( const WarpCell & w, uint32_t & err )
    {
        if ( w.vn > kMaxVertices )
            err |= kErrVertexCap;
        if ( w.en > kMaxEdges )
            err |= kErrEdgeCap;
    }

    // -----------------------------------------------------------------------------------
    // Cell update: clip the cell of site i by site j (topology_update.inl:49-555)
    // -----------------------------------------------------------------------------------
    __device__ bool update_cell( const CellContext & c, WarpCell & w, uint32_t i, double4 si, uint32_t j, double4 sj,
                                 uint32_t & err )
    {
        const uint32_t lane = lane_id();
        if ( w.vn == 0 && w.en == 0 )
            return false;

        // inclusion (:70-84)
        {
            const double ri = si.w, rj = sj.w;
            const double bigger = fmax( ri, rj ), smaller = fmin( ri, rj );
            if ( lt_eps( dlength( d3( si ) - d3( sj ) ), bigger - smaller ) )
            {
                if ( lt_eps( rj, ri ) )
                    return false;
                w.vn = 0;
                w.en = 0;
                return false;
            }
        }

        NewEdges ne;
        ne.slot[ 0 ] = kNoEdge;
        ne.slot[ 1 ] = kNoEdge;
        ne.count     = 0;

        const uint32_t baseV = w.vn, baseE = w.en;

        // 1. Vertices inside sj are marked; each one removes a vertex from its three edges
        //    (:96-154). The 8-bit edge index of the reference is kept.
        for ( uint32_t vs = 0; vs <= baseV / 32; vs++ )
        {
            const uint32_t id      = lane + 32 * vs;
            bool           invalid = false;
            if ( id < baseV )
            {
                invalid = sphere_conflict( c, sj, w.pos[ id ], w.tally );
                if ( invalid )
                    w.v[ id ].w |= 0xff00u;
            }
            uint32_t m = __ballot_sync( kFull, invalid );
            while ( m )
            {
                const uint32_t t = highest( m );
                m &= ~( 1u << t );
                const uint4 vx = w.v[ 32 * vs + t ];
                for ( uint32_t es = 0; es <= baseE / 32; es++ )
                {
                    const uint8_t eid = uint8_t( lane + 32 * es );
                    if ( eid < w.en )
                    {
                        const uint4 r = w.e[ eid ];
                        if ( ( r.x == vx.x && r.y == vx.y ) || ( r.x == vx.x && r.y == vx.z ) || ( r.x == vx.y && r.y == vx.z ) )
                            w.e[ eid ].z = r.z - 1u;
                    }
                }
                __syncwarp();
            }
        }
        __syncwarp();

        // 2. New vertices on every edge (:156-323).
        uint32_t closed_bits = 0;
        for ( uint32_t es = 0; es <= baseE / 32; es++ )
        {
            const uint32_t e   = lane + 32 * es;
            const uint4    r   = e < kEdgeSlots ? w.e[ e ] : make_uint4( 0, 0, 0, 0 );
            bool           has = e < baseE;
            const uint32_t k = r.x, l = r.y;
            uint32_t       mask = 0;
            double4        q0 = make_double4( 0, 0, 0, 0 ), q1 = make_double4( 0, 0, 0, 0 );
            double4        sk = make_double4( 0, 0, 0, 0 ), sl = make_double4( 0, 0, 0, 0 );
            if ( has )
            {
                sk   = site( c, k );
                sl   = site( c, l );
                mask = quadrisector( si, sj, sk, sl, q0, q1 );
                has  = mask != 0;
            }
            // a closed edge is emptied when its trisector point falls inside sj (:184-191)
            if ( e < baseE && mask == 0 && r.z == kNone )
            {
                trisector( si, sk, sl, q0, q0 );
                if ( intersects( q0, sj ) )
                    w.e[ e ].z = 0;
            }

            // The emptiness predicate of every root (topology_update.inl:577-590): on a small
            // cell each lane checks its own roots against every edge site; on a large one the
            // whole warp checks one root at a time, 32 edges per step.
            uint32_t valid = mask;
            if ( baseE <= kLaneClearEdges )
            {
                if ( has )
                {
                    if ( ( mask & 1u ) && !clear_by_lane( c, w, q0, k, l ) )
                        valid &= ~1u;
                    if ( ( mask & 2u ) && !clear_by_lane( c, w, q1, k, l ) )
                        valid &= ~2u;
                }
            }
            else
            {
                uint32_t hm = __ballot_sync( kFull, has );
                while ( hm )
                {
                    const uint32_t t = highest( hm );
                    hm &= ~( 1u << t );
                    uint32_t       tm = __shfl_sync( kFull, mask, t );
                    const uint32_t tk = __shfl_sync( kFull, k, t ), tl = __shfl_sync( kFull, l, t );
                    while ( tm )
                    {
                        const uint32_t nv = __ffs( tm ) - 1;
                        tm &= ~( 1u << nv );
                        const double4 cand = shfl4( nv ? q1 : q0, t );
                        const bool    ok   = edges_clear( c, w, cand, tk, tl );
                        if ( lane == t && !ok )
                            valid &= ~( 1u << nv );
                    }
                }
            }

            const uint32_t count = __popc( valid );
            has                  = has && count > 0;
            if ( has )
            {
                uint32_t vnb = w.e[ e ].z;
                if ( vnb == kNone )
                    vnb = 0;
                w.e[ e ].z = vnb + count;
            }
            uint32_t total;
            uint32_t off = warp_exclusive_scan( count, total );

            // new vertex records with sorted ids, and their positions (:256-275)
            uint32_t jj = j, kk = k, ll = l, t;
            if ( jj > ll )
            {
                t  = jj;
                jj = ll;
                ll = t;
            }
            if ( jj > kk )
            {
                t  = jj;
                jj = kk;
                kk = t;
            }
            if ( kk > ll )
            {
                t  = kk;
                kk = ll;
                ll = t;
            }
            uint32_t vm = valid;
            while ( vm )
            {
                const uint32_t nv = __ffs( vm ) - 1;
                vm &= ~( 1u << nv );
                const uint32_t dst = w.vn + off;
                if ( dst < kVertexSlots )
                {
                    w.v[ dst ] = make_uint4( jj, kk, ll, nv );
                    // same call as a later re-solve when the new site is the smallest id
                    w.pos[ dst ] = ( jj == j ) ? ( nv ? q1 : q0 ) : solve_vertex( c, si, make_uint4( jj, kk, ll, nv ) );
                }
                else
                    err |= kErrVertexCap;
                off++;
            }

            // two new-edge candidates per new vertex, lanes from the highest (:277-316)
            uint32_t lm = __ballot_sync( kFull, valid != 0 );
            while ( lm )
            {
                const uint32_t tl2 = highest( lm );
                lm &= ~( 1u << tl2 );
                uint32_t       tv = __shfl_sync( kFull, valid, tl2 );
                const uint32_t tc = __shfl_sync( kFull, count, tl2 );
                const uint32_t tk = __shfl_sync( kFull, k, tl2 ), tl = __shfl_sync( kFull, l, tl2 );
                while ( tv )
                {
                    tv &= tv - 1;
                    ne.push( tk, tc == 2, false, err );
                    ne.push( tl, tc == 2, false, err );
                }
            }
            w.vn += total;
            closed_bits = ( closed_bits | ( ( e < baseE && mask == 0 ) ? ( 1u << es ) : 0u ) ) & 0xffu;
            __syncwarp();
        }
        check_capacity( w, err );

        // 3. Closed elliptic trisectors with the sites of edges that got no vertex (:325-433).
        if ( __any_sync( kFull, closed_bits != 0 ) )
        {
            for ( uint32_t es = 0; es <= baseE / 32; es++ )
            {
                const bool can = ( closed_bits >> es ) & 1u;
                if ( !__any_sync( kFull, can ) )
                    continue;
                const uint32_t e = lane + 32 * es;
                const uint4    r = e < kEdgeSlots ? w.e[ e ] : make_uint4( 0, 0, 0, 0 );
                double4        sites2[ 2 ] = { make_double4( 0, 0, 0, 0 ), make_double4( 0, 0, 0, 0 ) };
                if ( e < baseE )
                {
                    sites2[ 0 ] = site( c, r.x );
                    sites2[ 1 ] = site( c, r.y );
                }
                for ( uint32_t s = 0; s < 2; s++ )
                {
                    const uint32_t id  = s ? r.y : r.x;
                    bool           cur = can;
                    uint32_t       cm  = __ballot_sync( kFull, cur );
                    while ( cm )
                    {
                        const uint32_t t = highest( cm );
                        cm &= ~( 1u << t );
                        const uint32_t tid = __shfl_sync( kFull, id, t );
                        const bool     shared = ne.contains( tid );
                        if ( lane == t && shared )
                            cur = false;
                    }
                    double4  x0 = make_double4( 0, 0, 0, 0 ), x1 = make_double4( 0, 0, 0, 0 );
                    uint32_t cnt = 0;
                    if ( cur )
                        cnt = trisector( si, sj, sites2[ s ], x0, x1 );
                    cur = cur && cnt == 2;
                    cm  = __ballot_sync( kFull, cur );
                    while ( cm )
                    {
                        const uint32_t t = highest( cm );
                        cm &= ~( 1u << t );
                        const uint32_t tid = __shfl_sync( kFull, id, t );
                        const double4  tv  = shfl4( x0, t );
                        if ( edges_clear( c, w, tv, tid, i ) )
                            ne.push( tid, false, true, err );
                    }
                }
            }
        }

        // 4. Unique new edges by site, with the number of new vertices on each (:435-515).
        sort64( ne.slot );
        const uint32_t next0 = ne.slot[ 1 ];
        const uint32_t next1 = __shfl_down_sync( kFull, ne.slot[ 0 ], 1 );
        const bool     last0 = ( ( next0 >> 2 ) != ( ne.slot[ 0 ] >> 2 ) ) && ( ne.slot[ 0 ] & 3u ) != 3u;
        const bool     last1 = ( lane == 31 || ( next1 >> 2 ) != ( ne.slot[ 1 ] >> 2 ) ) && ( ne.slot[ 1 ] & 3u ) != 3u;
        // index of the previous group end (exclusive max-scan over elements)
        int lane_last = last1 ? int( 2 * lane + 1 ) : ( last0 ? int( 2 * lane ) : -1 );
        int prev      = lane_last;
#pragma unroll
        for ( int o = 1; o < 32; o <<= 1 )
        {
            const int y = __shfl_up_sync( kFull, prev, o );
            if ( int( lane ) >= o )
                prev = max( prev, y );
        }
        int before = __shfl_up_sync( kFull, prev, 1 );
        if ( lane == 0 )
            before = -1;
        uint32_t written;
        uint32_t woff = warp_exclusive_scan( uint32_t( last0 ) + uint32_t( last1 ), written );
        for ( uint32_t s = 0; s < 2; s++ )
        {
            const bool     isLast = s ? last1 : last0;
            const int      f      = int( 2 * lane + s );
            const uint32_t v      = ne.slot[ s ];
            if ( isLast )
            {
                const uint32_t other = v >> 2;
                const uint32_t dst   = w.en + woff;
                if ( dst < kEdgeSlots )
                    w.e[ dst ] = make_uint4( min( j, other ), max( j, other ), ( v & 1u ) ? kNone : uint32_t( f - before ), 0u );
                else
                    err |= kErrEdgeCap;
                woff++;
                before = f;
            }
        }
        w.en += written;
        check_capacity( w, err );
        w.vn = min( w.vn, kVertexSlots );
        w.en = min( w.en, kEdgeSlots );
        __syncwarp();

        // 5. Stable compaction of the marked vertices and the emptied edges (:520-542).
        if ( w.vn > 0 )
        {
            uint32_t kept = 0;
            for ( uint32_t base = 0; base < w.vn; base += 32 )
            {
                const uint32_t id   = base + lane;
                uint4          r    = make_uint4( 0, 0, 0, 0 );
                double4        p    = make_double4( 0, 0, 0, 0 );
                bool           keep = false;
                if ( id < w.vn )
                {
                    r    = w.v[ id ];
                    p    = w.pos[ id ];
                    keep = !( vstatus( r ) == 0xffu && id < baseV );
                }
                const uint32_t bal = __ballot_sync( kFull, keep );
                const uint32_t dst = kept + __popc( bal & ( ( 1u << lane ) - 1u ) );
                __syncwarp();
                if ( keep )
                {
                    w.v[ dst ]   = r;
                    w.pos[ dst ] = p;
                }
                kept += __popc( bal );
                __syncwarp();
            }
            w.vn = kept;
        }
        {
            uint32_t kept = 0;
            for ( uint32_t base = 0; base < w.en; base += 32 )
            {
                const uint32_t id   = base + lane;
                uint4          r    = make_uint4( 0, 0, 0, 0 );
                bool           keep = false;
                if ( id < w.en )
                {
                    r    = w.e[ id ];
                    keep = !( r.z == 0 && id < baseE );
                }
                const uint32_t bal = __ballot_sync( kFull, keep );
                const uint32_t dst = kept + __popc( bal & ( ( 1u << lane ) - 1u ) );
                __syncwarp();
                if ( keep )
                    w.e[ dst ] = r;
                kept += __popc( bal );
                __syncwarp();
            }
            w.en = kept;
        }
        return written != 0;
    }

    // Largest vertex or closed-trisector radius of the cell (topology_update.inl:595-653).
    __device__ double cell_radius( const CellContext & c, const WarpCell & w, double4 si )
    {
        double m = 0.0;
        for ( uint32_t base = 0; base < w.vn; base += 32 )
        {
            const uint32_t v = base + lane_id();
            if ( v < w.vn )
                m = fmax( m, w.pos[ v ].w );
        }
        for ( uint32_t base = 0; base < w.en; base += 32 )
        {
            const uint32_t e = base + lane_id();
            if ( e < w.en )
            {
                const uint4 r = w.e[ e ];
                double4     x0 = make_double4( 0, 0, 0, 0 ), x1 = make_double4( 0, 0, 0, 0 );
                if ( trisector( si, site( c, r.x ), site( c, r.y ), x0, x1 ) == 2 )
                    m = fmax( m, fmax( x0.w, x1.w ) );
            }
        }
#pragma unroll
        for ( int o = 16; o > 0; o >>= 1 )
            m = fmax( m, __shfl_xor_sync( kFull, m, o ) );
        return m;
    }

    // -----------------------------------------------------------------------------------
    // Shared-memory carving and the per-cell store
    // -----------------------------------------------------------------------------------
    __device__ __forceinline__ WarpCell carve( unsigned char * smem, uint32_t warp, uint32_t extra )
    {
        unsigned char * base = smem + size_t( warp ) * ( kWarpCellBytes + extra );
        WarpCell        w;
        w.pos = reinterpret_cast<double4 *>( base );
        w.v   = reinterpret_cast<uint4 *>( base + sizeof( double4 ) * kVertexSlots );
        w.e   = reinterpret_cast<uint4 *>( base + ( sizeof( double4 ) + sizeof( uint4 ) ) * kVertexSlots );
        w.vn    = 0;
        w.en    = 0;
        w.tally = FilterTally {};
        return w;
    }

    __device__ __forceinline__ void load_cell( const CellContext & c, WarpCell & w, uint32_t i, double4 si, bool with_vertices,
                                               bool solve )
    {
        w.en = c.edge_nb[ i ];
        for ( uint32_t e = lane_id(); e < w.en; e += 32 )
            w.e[ e ] = c.edges[ store_row( c, i ) * kMaxEdges + e ];
        w.vn = 0;
        if ( with_vertices )
        {
            w.vn = c.vertex_nb[ i ];
            for ( uint32_t v = lane_id(); v < w.vn; v += 32 )
            {
                const uint4 r = c.vertices[ store_row( c, i ) * kMaxVertices + v ];
                w.v[ v ]      = r;
                if ( solve )
                    w.pos[ v ] = solve_vertex( c, si, r );
            }
        }
        __syncwarp();
    }

    __device__ __forceinline__ void store_cell( const CellContext & c, const WarpCell & w, uint32_t i, uint32_t vertex_base,
                                                uint32_t & err )
    {
        const uint32_t vn = min( vertex_base + w.vn, kMaxVertices );
        const uint32_t en = min( w.en, kMaxEdges );
        if ( vertex_base + w.vn > kMaxVertices )
            err |= kErrVertexCap;
        if ( w.en > kMaxEdges )
            err |= kErrEdgeCap;
        for ( uint32_t e = lane_id(); e < en; e += 32 )
            c.edges[ store_row( c, i ) * kMaxEdges + e ] = w.e[ e ];
        for ( uint32_t v = lane_id(); v + vertex_base < vn; v += 32 )
            c.vertices[ store_row( c, i ) * kMaxVertices + vertex_base + v ] = w.v[ v ];
        if ( lane_id() == 0 )
        {
            c.vertex_nb[ i ] = vn;
            c.edge_nb[ i ]   = en;
        }
    }

    __device__ __forceinline__ void report( const CellContext & c, uint32_t err )
    {
        err = __reduce_or_sync( kFull, err );
        if ( err && lane_id() == 0 )
            atomicOr( c.error, err );
    }
    // Error flags and the FP32 filter's counts of a warp at the end of a kernel.
    __device__ __forceinline__ void report( const CellContext & c, uint32_t err, const WarpCell & w )
    {
        report( c, err );
        if ( c.fp32 && c.counters )
        {
            const uint32_t tests = __reduce_add_sync( kFull, w.tally.tests );
            const uint32_t esc   = __reduce_add_sync( kFull, w.tally.escalated );
            if ( lane_id() == 0 )
            {
                atomicAdd( c.counters + kCountFiltered, static_cast<unsigned long long>( tests ) );
                atomicAdd( c.counters + kCountEscalated, static_cast<unsigned long long>( esc ) );
            }
        }
    }

    // -----------------------------------------------------------------------------------
    // kNN search: thread per site, max-heap of K in shared memory (lbvh.inl:8-105,
    // heap.hpp:11-43, algorithm.inl:32-99)
    // -----------------------------------------------------------------------------------
    __device__ __forceinline__ void heap_down( uint32_t * keys, float * dist, uint32_t stride, uint32_t k )
    {
        uint32_t j = 0;
        while ( true )
        {
            const uint32_t l = 2 * j + 1, r = 2 * j + 2;
            uint32_t       largest = j;
            if ( l < k && dist[ l * stride ] > dist[ largest * stride ] )
                largest = l;
            if ( r < k && dist[ r * stride ] > dist[ largest * stride ] )
                largest = r;
            if ( largest == j )
                return;
            const float    td = dist[ j * stride ];
            const uint32_t tk = keys[ j * stride ];
            dist[ j * stride ]       = dist[ largest * stride ];
            keys[ j * stride ]       = keys[ largest * stride ];
            dist[ largest * stride ] = td;
            keys[ largest * stride ] = tk;
            j                        = largest;
        }
    }

    // kNN step `step` (algorithm.inl:32-99): step 0 takes the k nearest sites and flags buried
    // sites; a later step takes the next k, beyond the last neighbour of the previous step, or
    // none once the previous list ran short.
    // Propose: the learned form's first step, which also runs the k-proposal network (a separate
    // instantiation, so that the plain search keeps its small register footprint).
    template<bool Propose>
    __global__ void __launch_bounds__( kKnnBlock ) k_knn( CellContext c, uint32_t step )
    {
        __shared__ uint32_t    s_keys[ kMaxK * kKnnBlock ];
        __shared__ float       s_dist[ kMaxK * kKnnBlock ];
        extern __shared__ __align__( 16 ) unsigned char s_dyn[]; // the network (Propose only)
        ProposalNet *          s_net   = reinterpret_cast<ProposalNet *>( s_dyn );
        constexpr bool         propose = Propose;
        if ( propose )
        {
            // the network, staged once per block (broadcast reads during inference)
            for ( uint32_t t = threadIdx.x; t < sizeof( ProposalNet ) / 4; t += blockDim.x )
                reinterpret_cast<uint32_t *>( s_net )[ t ] = reinterpret_cast<const uint32_t *>( c.proposal )[ t ];
            __syncthreads();
        }
        const uint32_t id = blockIdx.x * blockDim.x + threadIdx.x;
        if ( id >= c.n )
            return;
        // learned form's second step: only the uncertified cells proposed beyond k search again
        if ( step != 0 && c.scheduled && ( !second_step_cell( c, id ) || c.status[ id ] != kInValidation ) )
            return;
        const uint32_t k      = c.k;
        const uint32_t n      = c.n;
        const float4   si     = c.sites_f[ id ];
        float          start  = -FLT_MAX;
        if ( step != 0 )
        {
            const uint32_t last = c.knn[ size_t( id ) * k + k - 1 ];
            if ( last >= n )
            {
                for ( uint32_t q = 0; q < k; q++ )
                    c.knn[ size_t( id ) * k + q ] = kNone;
                return;
            }
            start = sphere_distance( c.sites_f[ last ], si );
        }
        uint32_t *     keys   = s_keys + threadIdx.x;
        float *        dist   = s_dist + threadIdx.x;
        const uint32_t stride = kKnnBlock;
        for ( uint32_t q = 0; q < k; q++ )
        {
            keys[ q * stride ] = kNone;
            dist[ q * stride ] = FLT_MAX;
        }
        uint32_t       err  = 0;
        if ( step == 0 )
            c.known_radii[ id ] = -FLT_MAX;
        uint8_t buried      = kInValidation;
        uint2          stack[ kStack ];
        int            sp   = 0;
        uint32_t       node = 0;
        uint32_t       steps = 0;
        while ( true )
        {
            if ( ++steps > 4 * n + 64 )
            {
                err |= kErrWalk;
                break;
            }
            while ( node < n - 1 )
            {
                Box      lb, rb;
                uint32_t lc, rc;
                load_node( c.nodes, node, lb, rb, lc, rc );
                const float    dL = lb.distance( si ), dLMax = lb.farthest( si );
                const float    dR = rb.distance( si ), dRMax = rb.farthest( si );
                const bool     leftClosest = dL < dR;
                const float    minFar = leftClosest ? dR : dL, maxFar = leftClosest ? dRMax : dLMax;
                const uint32_t farChild = leftClosest ? rc : lc;
                const float    minClose = leftClosest ? dL : dR, maxClose = leftClosest ? dLMax : dRMax;
                const uint32_t closeChild = leftClosest ? lc : rc;
                const float    worst      = dist[ 0 ];
                const bool     exploreFar   = minFar < worst && maxFar > start;
                const bool     exploreClose = minClose < worst && maxClose > start;
                if ( !exploreFar && !exploreClose )
                    break;
                node = exploreClose ? closeChild : farChild;
                if ( exploreClose && exploreFar )
                {
                    if ( sp < int( kStack ) )
                        stack[ sp++ ] = make_uint2( farChild, __float_as_uint( minFar ) );
                    else
                        err |= kErrStack;
                }
            }
            if ( node >= n - 1 && node < 2 * n - 1 )
            {
                const uint32_t j = node - ( n - 1 );
                const float    d = sphere_distance( si, c.sites_f[ j ] );
                if ( id != j && d < dist[ 0 ] && d > start )
                {
                    dist[ 0 ] = d;
                    keys[ 0 ] = j;
                    heap_down( keys, dist, stride, k );
                }
            }
            bool more = false;
            while ( sp > 0 )
            {
                --sp;
                if ( __uint_as_float( stack[ sp ].y ) > dist[ 0 ] )
                    continue;
                node = stack[ sp ].x;
                more = true;
                break;
            }
            if ( !more )
                break;
        }
        // heapsort into ascending distance
        for ( uint32_t size = k; size > 0; )
        {
            const float    td = dist[ 0 ];
            const uint32_t tk = keys[ 0 ];
            dist[ 0 ]                      = dist[ ( size - 1 ) * stride ];
            keys[ 0 ]                      = keys[ ( size - 1 ) * stride ];
            dist[ ( size - 1 ) * stride ] = td;
            keys[ ( size - 1 ) * stride ] = tk;
            --size;
            heap_down( keys, dist, stride, size );
        }
        for ( uint32_t q = 0; q < k; q++ )
            c.knn[ size_t( id ) * k + q ] = keys[ q * stride ];
        if ( err )
            atomicOr( c.error, err );
        if ( step != 0 )
            return;
        if ( propose )
        {
            // fused inference of the k-proposal on the sorted list
            FeatureInputs in;
            in.sites_f = c.sites_f;
            in.codes   = c.codes;
            in.scene   = c.scene;
            in.n       = n;
            float f[ kPIn ];
            proposal_features( in, id, keys, stride, k, f );
            c.proposed_k[ id ] = uint8_t( proposal_rank( s_net[ 0 ], proposal_predict( s_net[ 0 ], f ), c.proposal_max ) );
        }

        // buried site: inside its nearest neighbour (algorithm.inl:85-98); `si` is the float copy
        const uint32_t nearest = keys[ 0 ];
        if ( nearest != kNone )
        {
            const double4 closest = c.sites[ nearest ];
            const double  ri = si.w, rj = closest.w;
            const double  bigger = fmax( ri, rj ), smaller = fmin( ri, rj );
            if ( lt_eps( dlength( make_double3( si.x, si.y, si.z ) - d3( closest ) ), bigger - smaller ) && !lt_eps( rj, ri ) )
                buried = kBuried;
        }
        c.status[ id ] = buried;
    }

    // -----------------------------------------------------------------------------------
    // Cells from the kNN lists (algorithm.inl:101-206)
    // -----------------------------------------------------------------------------------
    // The 12 edges of the initial cell, as pairs of artificial sites (algorithm.inl:1486-1499).
    __constant__ uint32_t c_initial_edges[ 12 ][ 2 ] = { { 0, 2 }, { 2, 4 }, { 1, 2 }, { 2, 5 }, { 1, 4 }, { 1, 5 },
                                                         { 0, 5 }, { 0, 4 }, { 1, 3 }, { 3, 5 }, { 0, 3 }, { 3, 4 } };

    __device__ __forceinline__ void initial_cell( const CellContext & c, WarpCell & w, double4 si )
    {
        // 8 vertices and 12 edges on the artificial sites (algorithm.inl:1466-1505)
        const uint32_t n    = c.n;
        const uint32_t lane = lane_id();
        if ( lane < 8 )
        {
            const uint4 r = make_uint4( n + ( lane >> 2 ), n + 2 + ( ( lane >> 1 ) & 1 ), n + 4 + ( lane & 1 ), 0u );
            w.v[ lane ]   = r;
            w.pos[ lane ] = solve_vertex( c, si, r );
        }
        if ( lane < 12 )
            w.e[ lane ] = make_uint4( n + c_initial_edges[ lane ][ 0 ], n + c_initial_edges[ lane ][ 1 ], 2u, 0u );
        w.vn = 8;
        w.en = 12;
        __syncwarp();
    }

    // Cell construction from the kNN lists (getCells, algorithm.inl:101-206). kCellsFirst
    // starts every cell from the initial cell of the six bounding sites (the reference's
    // initializeDataStructure, topology_update.inl:5-47, fused in); kCellsNext continues the
    // stored cells with the next kNN step; kCellsInitOnly writes the initial cells, statuses
    // and known radii alone (no kNN step at all).
    __global__ void __launch_bounds__( kCellBlock, 4 ) k_cells( CellContext c, uint32_t mode )
    {
        extern __shared__ __align__( 16 ) unsigned char smem[];
        const uint32_t warp  = threadIdx.x >> 5;
        const uint32_t gwarp = blockIdx.x * ( kCellBlock / 32 ) + warp;
        const uint32_t nwarp = gridDim.x * ( kCellBlock / 32 );
        WarpCell       w     = carve( smem, warp, 0 );
        uint32_t       err   = 0;
        // per-warp counters (lane 0 counts), added to the build's counters at the end
        __shared__ uint32_t s_counts[ kCellBlock / 32 ][ kCounters ];
        uint32_t *          counts = s_counts[ warp ];
        if ( lane_id() < kCounters )
            counts[ lane_id() ] = 0;
        __syncwarp();
        // cells are taken one at a time from a shared counter (uneven cells, see bisector pass)
        ( void ) gwarp;
        ( void ) nwarp;
        while ( true )
        {
            uint32_t i = 0;
            if ( lane_id() == 0 )
                i = c.lo + atomicAdd( c.work_counter, 1u );
            i = __shfl_sync( kFull, i, 0 );
            if ( i >= c.hi )
                break;
            if ( mode == kCellsInitOnly )
            {
                initial_cell( c, w, c.sites[ i ] );
                store_cell( c, w, i, 0, err );
                if ( lane_id() == 0 )
                {
                    c.status[ i ]      = kInValidation;
                    c.known_radii[ i ] = -FLT_MAX;
                }
                __syncwarp();
                continue;
            }
            const uint8_t status = c.status[ i ];
            if ( status == kFullyValidated || ( mode == kCellsNext && status == kBuried ) )
                continue;
            if ( mode == kCellsNext && c.scheduled && !second_step_cell( c, i ) )
                continue; // learned form: this cell was proposed within k, so it has one step only
            const double4 si = c.sites[ i ];
            if ( mode == kCellsNext )
            {
                load_cell( c, w, i, si, true, true );
                if ( c.scheduled && lane_id() == 0 )
                    counts[ kCountSecondStep ]++;
            }
            else
                initial_cell( c, w, si );
            if ( status == kBuried )
            {
                // a buried cell keeps the initial store (topology_update.inl:5-47)
                store_cell( c, w, i, 0, err );
                __syncwarp();
                continue;
            }
            // learned form: the certificate is first checked at the proposed rank; a cell that
            // passes there stops inserting (its later neighbours cannot change a certified cell)
            // but its known radius still covers its whole list, as the plain form's does
            uint32_t check_at = c.k;
            if ( c.proposed_k )
            {
                const uint32_t r = c.proposed_k[ i ];
                if ( mode == kCellsFirst )
                    check_at = min( r, c.k );
                else if ( c.scheduled )
                    check_at = r > c.k ? r - c.k : c.k; // rank r counts the first step's k neighbours
            }
            double         known    = -DBL_MAX;
            bool           done     = false;
            for ( uint32_t q = 0; q < c.k; q++ )
            {
                if ( q == check_at )
                {
                    const double radius = cell_radius( c, w, si );
                    done                = gt_eps( known, 2.0 * radius );
                    if ( lane_id() == 0 )
                        counts[ kCountChecked ]++;
                    if ( !done && lane_id() == 0 )
                        counts[ kCountFallbacks ]++;
                }
                const uint32_t j = c.knn[ size_t( i ) * c.k + q ];
                if ( j == kNone )
                    break;
                if ( c.status[ j ] == kBuried )
                    continue;
                const double4 sj = c.sites[ j ];
                if ( done )
                {
                    if ( lane_id() == 0 )
                        counts[ kCountSkipped ]++;
                }
                else
                {
                    update_cell( c, w, i, si, j, sj, err );
                    if ( lane_id() == 0 )
                        counts[ kCountInsertions ]++;
                }
                known = fmax( known, sphere_distance( si, sj ) );
            }
            if ( !done )
                done = gt_eps( known, 2.0 * cell_radius( c, w, si ) );
            if ( lane_id() == 0 )
            {
                if ( done )
                    c.status[ i ] = kFullyValidated;
                c.known_radii[ i ] = float( known );
            }
            store_cell( c, w, i, 0, err );
            __syncwarp();
        }
        report( c, err, w );
        __syncwarp();
        if ( c.counters && lane_id() == 0 )
            for ( uint32_t t = 0; t < kCounters; t++ )
                if ( counts[ t ] )
                    atomicAdd( c.counters + t, static_cast<unsigned long long>( counts[ t ] ) );
    }

    // Per-neighbour labels of the kNN cell construction (the reference's measurement harness
    // app/benchmarks/benchmark_contributing_nearest.cu:10-129): for each cell and each kNN rank,
    // whether that neighbour changed the cell and whether the security-radius certificate held
    // after it. A cell stops at the rank where it certifies (and is then FullyValidated). Row i
    // of `contributed` / `certified` holds steps x k bytes; this step writes its k.
    __global__ void __launch_bounds__( kCellBlock, 4 ) k_cells_profile( CellContext c, uint32_t step, uint32_t row,
                                                                       uint8_t * __restrict__ contributed,
                                                                       uint8_t * __restrict__ certified )
    {
        extern __shared__ __align__( 16 ) unsigned char smem[];
        const uint32_t warp = threadIdx.x >> 5;
        WarpCell       w    = carve( smem, warp, 0 );
        uint32_t       err  = 0;
        while ( true )
        {
            uint32_t i = 0;
            if ( lane_id() == 0 )
                i = c.lo + atomicAdd( c.work_counter, 1u );
            i = __shfl_sync( kFull, i, 0 );
            if ( i >= c.hi )
                break;
            const uint8_t status = c.status[ i ];
            if ( status == kFullyValidated || ( step > 0 && status == kBuried ) )
                continue;
            const double4 si = c.sites[ i ];
            if ( step > 0 )
                load_cell( c, w, i, si, true, true );
            else
                initial_cell( c, w, si );
            if ( status == kBuried )
            {
                store_cell( c, w, i, 0, err );
                __syncwarp();
                continue;
            }
            double known = -DBL_MAX;
            for ( uint32_t q = 0; q < c.k; q++ )
            {
                const uint32_t j = c.knn[ size_t( i ) * c.k + q ];
                if ( j == kNone )
                    break;
                if ( c.status[ j ] == kBuried )
                    continue;
                const double4 sj      = c.sites[ j ];
                const bool    changed = update_cell( c, w, i, si, j, sj, err );
                known                 = fmax( known, sphere_distance( si, sj ) );
                const double radius   = cell_radius( c, w, si );
                const bool   over     = gt_eps( known, 2.0 * radius );
                if ( lane_id() == 0 )
                {
                    const size_t at = size_t( row ) * i + size_t( step ) * c.k + q;
                    contributed[ at ] = changed ? 1 : 0;
                    certified[ at ]   = over ? 1 : 0;
                    if ( over )
                        c.status[ i ] = kFullyValidated;
                }
                if ( over )
                    break;
            }
            if ( lane_id() == 0 )
                c.known_radii[ i ] = float( known );
            store_cell( c, w, i, 0, err );
            __syncwarp();
        }
        report( c, err, w );
    }

    // -----------------------------------------------------------------------------------
    // Vertex validation (algorithm.inl:208-476)
    // -----------------------------------------------------------------------------------
    __global__ void __launch_bounds__( kCellBlock, 4 ) k_vertex_validation( CellContext c, const uint32_t * __restrict__ tasks,
                                                                        const uint32_t * __restrict__ task_count )
    {
        extern __shared__ __align__( 16 ) unsigned char smem[];
        const uint32_t warp  = threadIdx.x >> 5;
        const uint32_t gwarp = blockIdx.x * ( kCellBlock / 32 ) + warp;
        const uint32_t nwarp = gridDim.x * ( kCellBlock / 32 );
        const uint32_t lane  = lane_id();
        WarpCell       w     = carve( smem, warp, 0 );
        uint32_t       err   = 0;
        const uint32_t count = *task_count;
        const uint32_t n     = c.n;
        const float    rmax  = float( c.scene->rmax );
        // tasks are taken one at a time from a shared counter (uneven cells, see bisector pass)
        ( void ) gwarp;
        ( void ) nwarp;
        while ( true )
        {
            uint32_t t = 0;
            if ( lane == 0 )
                t = atomicAdd( c.work_counter, 1u );
            t = __shfl_sync( kFull, t, 0 );
            if ( t >= count )
                break;
            const uint32_t i      = tasks[ t ];
            const uint8_t  status = c.status[ i ];
            if ( status == kFullyValidated || status == kBuried )
                continue;
            const double4 si = c.sites[ i ];
            load_cell( c, w, i, si, true, true );
            const float known = c.known_radii[ i ];

            uint32_t vs = 0, restarts = 0;
            while ( vs < w.vn / 32 + 1 && restarts < 100 )
            {
                const uint32_t vid = vs * 32 + lane;
                vs++;
                bool    need = vid < w.vn;
                uint4   vx   = make_uint4( 0, 0, 0, 0 );
                double4 cur  = make_double4( 0, 0, 0, 0 );
                if ( need )
                {
                    vx   = w.v[ vid ];
                    need = vstatus( vx ) == 0;
                }
                if ( need )
                {
                    cur = w.pos[ vid ];
                    if ( 2.0 * cur.w < double( known ) )
                    {
                        need = false;
                        w.v[ vid ].w = ( vx.w & 0xffff00ffu ) | 0x100u;
                    }
                }
                const float4 fc = to_float( cur );

                // Nearest admissible site to the vertex sphere, in up to two passes. The vertex
                // only changes when that site conflicts with it (FP64 sphere distance below
                // 1e-8); a site whose single-precision distance d is above `bound` cannot
                // conflict (the float distance is within ~1e-6 relative of the double one).
                // Pass 0 searches from best = bound instead of +inf. A box's distance is at most
                // max(d, -w) for every site it holds, so every ancestor of a site with
                // d < bound is entered while best stays at bound: if pass 0 finds no site, none
                // conflicts and the reference's nearest (whatever it is) leaves the vertex valid.
                // If it finds one with d > -w, no site holds the vertex centre, box distances
                // bound every leaf below them, and both searches are exact nearest searches in
                // the same walk order: same site. Only when the nearest holds the vertex centre
                // (d <= -w) can the reference's answer depend on its visiting history; pass 1
                // then repeats its search from +inf for those lanes.
                const float scale = 1e-5f * ( fabsf( fc.x ) + fabsf( fc.y ) + fabsf( fc.z ) + fabsf( fc.w ) + rmax );
                const float bound = 1e-2f + scale + fmaxf( 0.f, -fc.w );
                const float deep  = -fc.w + 1e-3f + scale;
                uint32_t    neighbor  = kNone;
                bool        searching = need;
                for ( uint32_t pass = 0; pass < 2; pass++ )
                {
                    uint2    stack[ kStack ];
                    int      sp         = 0;
                    uint32_t node       = 0;
                    float    best       = pass == 0 ? bound : FLT_MAX;
                    bool     walking    = searching;
                    uint32_t walk_steps = 0;
                    if ( searching )
                        neighbor = kNone;
                    while ( true )
                    {
                        if ( walking && ++walk_steps > 4 * n + 64 )
                        {
                            err |= kErrWalk;
                            walking = false;
                        }
                        while ( walking && node < n - 1 )
                        {
                            Box      lb, rb;
                            uint32_t lc, rc;
                            load_node( c.nodes, node, lb, rb, lc, rc );
                            const float    dL = lb.distance( fc ), dR = rb.distance( fc );
                            const bool     leftClosest = dL < dR;
                            const float    minFar = leftClosest ? dR : dL, minClose = leftClosest ? dL : dR;
                            const uint32_t farChild = leftClosest ? rc : lc, closeChild = leftClosest ? lc : rc;
                            const bool     exploreFar = minFar < best, exploreClose = minClose < best;
                            if ( !exploreFar && !exploreClose )
                                break;
                            node = exploreClose ? closeChild : farChild;
                            if ( exploreClose && exploreFar )
                            {
                                if ( sp < int( kStack ) )
                                    stack[ sp++ ] = make_uint2( farChild, __float_as_uint( minFar ) );
                                else
                                    err |= kErrStack;
                            }
                        }
                        const uint32_t j   = node - ( n - 1 );
                        bool           can = walking && node >= n - 1 && node < 2 * n - 1 && j != i && j != vx.x && j != vx.y
                                     && j != vx.z && c.status[ j ] != kBuried;
                        // Only a leaf closer than the best so far can become the answer, so the
                        // distance is tested first and the warp-collective neighbour scan runs
                        // for those leaves alone (the same conjunction, fewer scans).
                        float d = FLT_MAX;
                        if ( can )
                        {
                            d   = sphere_distance( c.sites_f[ j ], fc );
                            can = d < best;
                        }
                        uint32_t cm = __ballot_sync( kFull, can );
                        while ( cm )
                        {
                            const uint32_t t2 = highest( cm );
                            cm &= ~( 1u << t2 );
                            const uint32_t tj     = __shfl_sync( kFull, j, t2 );
                            const bool     known2 = is_known( w, tj );
                            if ( lane == t2 )
                                can = !known2;
                        }
                        if ( can )
                        {
                            best     = d;
                            neighbor = j;
                        }
                        while ( walking )
                        {
                            if ( sp == 0 )
                            {
                                walking = false;
                                break;
                            }
                            --sp;
                            if ( __uint_as_float( stack[ sp ].y ) > best )
                                continue;
                            node = stack[ sp ].x;
                            break;
                        }
                        if ( !__any_sync( kFull, walking ) )
                            break;
                    }
                    searching = searching && neighbor != kNone && best <= deep;
                    if ( !__any_sync( kFull, searching ) )
                        break;
                }

                const bool isValid = neighbor == kNone || !intersects( cur, c.sites[ neighbor ] );
                if ( need )
                    w.v[ vid ].w = ( w.v[ vid ].w & 0xffff00ffu ) | 0x100u;
                __syncwarp();
                const uint32_t changed = __ballot_sync( kFull, !isValid );
                uint32_t       pending = changed;
                while ( pending )
                {
                    const uint32_t t2 = highest( pending );
                    pending &= ~( 1u << t2 );
                    const uint32_t tj = __shfl_sync( kFull, neighbor, t2 );
                    if ( is_known( w, tj ) )
                        continue;
                    update_cell( c, w, i, si, tj, c.sites[ tj ], err );
                }
                if ( changed )
                {
                    vs = 0;
                    restarts++;
                }
            }
            store_cell( c, w, i, 0, err );
            __syncwarp();
        }
        report( c, err, w );
    }

    // -----------------------------------------------------------------------------------
    // Edge validation (algorithm.inl:478-857)
    // -----------------------------------------------------------------------------------
    // `proof` (optional): what the edge-parallel search proved for these cells. It searched
    // every edge against the neighbour set U0 of the stored cell. A site contributes to an
    // edge only if it is not a neighbour and one of its roots is empty of every neighbour, so
    // while the cell's neighbours still include all of U0 (updates only added some), an edge
    // with no contributor then has none now: its search would find nothing and is skipped.
    // Once a neighbour of U0 has left the cell, every edge is searched again.
    // One edge's contributor search in the exact edge pass: the bounding volume of the
    // trisector and the ball its contributors must reach (see k_edge_validation).
    struct EdgeWalk
    {
        float4   bsph, reach;
        float3   n1, n2, pp1, pp2;
        bool     hyperbola;
        uint32_t k, l;
        double4  sk, sl;
    };

    __device__ __forceinline__ float3 shfl3( float3 v, uint32_t src )
    {
        return make_float3( __shfl_sync( kFull, v.x, src ), __shfl_sync( kFull, v.y, src ), __shfl_sync( kFull, v.z, src ) );
    }
    __device__ __forceinline__ float4 shfl4f( float4 v, uint32_t src )
    {
        return make_float4( __shfl_sync( kFull, v.x, src ), __shfl_sync( kFull, v.y, src ), __shfl_sync( kFull, v.z, src ),
                            __shfl_sync( kFull, v.w, src ) );
    }

    // The rest of a long edge search, walked by the whole warp in the lane walk's order.
    // The walk has no running bound: which children of a node are entered, and in which order
    // (closer first), depends on the node alone, so its leaves come in one fixed order and the
    // answer is the first contributing leaf of that order. The frontier (nodes not yet expanded,
    // in that order) is a stack in `frontier`, its earliest node on top. Each step expands the
    // 32 earliest nodes at once: an internal node is replaced by its entered children, a leaf
    // is tested. When the earliest contributing leaf of a step sits at position q, the answer
    // is it or a leaf under one of the q nodes before it: everything after it is dropped and
    // the walk continues over those. `saved` holds the suspended lane's position (its current
    // node, then its stack from the top), `count` entries, earliest first.
    // One frontier node of the ordered walk: an internal node gives its entered children in walk
    // order (kids, first, second), a leaf whether it contributes.
    __device__ __forceinline__ void ordered_step( const CellContext & c, const WarpCell & w, uint32_t i, double4 si,
                                                  const EdgeWalk & p, uint32_t node, uint32_t & kids, uint32_t & first,
                                                  uint32_t & second, bool & contrib, uint32_t & j )
    {
        const uint32_t n = c.n;
        kids             = 0;
        contrib          = false;
        j                = kNone;
        if ( node < n - 1 )
        {
            Box      lb, rb;
            uint32_t lc, rc;
            load_node( c.nodes, node, lb, rb, lc, rc );
            const float3   closeL = lb.closest( p.bsph ), closeR = rb.closest( p.bsph );
            const float    dL = lb.distance( p.bsph ), dR = rb.distance( p.bsph );
            const bool     leftClosest = dL < dR;
            const float    minFar = leftClosest ? dR : dL, minClose = leftClosest ? dL : dR;
            const float3   farPoint = leftClosest ? closeR : closeL, closePoint = leftClosest ? closeL : closeR;
            const uint32_t farChild = leftClosest ? rc : lc, closeChild = leftClosest ? lc : rc;
            bool           exploreFar = minFar < 0.f;
            if ( p.hyperbola && exploreFar )
                exploreFar = fdot( p.n1, farPoint - p.pp1 ) < 0.f && fdot( p.n2, farPoint - p.pp2 ) < 0.f;
            bool exploreClose = minClose < 0.f;
            if ( p.hyperbola && exploreClose )
                exploreClose = fdot( p.n1, closePoint - p.pp1 ) < 0.f && fdot( p.n2, closePoint - p.pp2 ) < 0.f;
            exploreFar   = exploreFar && ( leftClosest ? rb : lb ).distance( p.reach ) < 0.f;
            exploreClose = exploreClose && ( leftClosest ? lb : rb ).distance( p.reach ) < 0.f;
            if ( exploreClose )
            {
                first = closeChild;
                kids  = 1;
                if ( exploreFar )
                {
                    second = farChild;
                    kids   = 2;
                }
            }
            else if ( exploreFar )
            {
                first = farChild;
                kids  = 1;
            }
        }
        else if ( node < 2 * n - 1 )
        {
            j        = node - ( n - 1 );
            bool can = j != i && j != p.k && j != p.l && c.status[ j ] != kBuried;
            double4 sj = make_double4( 0, 0, 0, 0 );
            if ( can )
            {
                sj              = c.sites[ j ];
                const float4 fj = to_float( sj );
                can             = intersects( fj, p.bsph ) && flength( f3( fj ) - f3( p.reach ) ) <= p.reach.w;
                if ( p.hyperbola )
                    can = can && double( fdot( p.n1, f3( fj ) - p.pp1 ) ) < -sj.w
                          && double( fdot( p.n2, f3( fj ) - p.pp2 ) ) < -sj.w;
            }
            if ( can )
                can = !known_by_lane( w, j );
            if ( can )
            {
                double4 x0 = make_double4( 0, 0, 0, 0 ), x1 = make_double4( 0, 0, 0, 0 );
                const uint32_t mask = quadrisector( si, sj, p.sk, p.sl, x0, x1 );
                contrib = mask == 3 && ( clear_by_lane( c, w, x0, p.k, p.l ) || clear_by_lane( c, w, x1, p.k, p.l ) );
            }
        }
    }

    // The rest of a long edge search, walked by the whole warp in the lane walk's order.
    // The walk has no running bound: which children of a node are entered, and in which order
    // (closer first), depends on the node alone, so its leaves come in one fixed order and the
    // answer is the first contributing leaf of that order. The frontier (nodes not yet expanded,
    // in that order) is a stack in `frontier`, its earliest node on top. Each step expands the
    // kCoopWidth x 32 earliest nodes at once (position r * 32 + lane for a lane's r-th node, so
    // each lane's loads overlap): an internal node is replaced by its entered children, a leaf
    // is tested. When the earliest contributing leaf of a step sits at position q, the answer
    // is it or a leaf under one of the q nodes before it: everything after it is dropped and
    // the walk continues over those. `saved` holds the suspended lane's position (its current
    // node, then its stack from the top), `count` entries, earliest first.
    __device__ uint32_t ordered_edge_walk( const CellContext & c, const WarpCell & w, uint32_t i, double4 si, const EdgeWalk & p,
                                           uint32_t * frontier, const uint32_t * saved, uint32_t count, uint32_t & err )
    {
        const uint32_t lane = lane_id();
        const uint32_t n    = c.n;
        for ( uint32_t q = lane; q < count; q += 32 )
            frontier[ count - 1 - q ] = saved[ q ];
        __syncwarp();
        uint32_t top = count, found = kNone, steps = 0;
        while ( top > 0 )
        {
            if ( ++steps > 4 * n + 64 )
            {
                err |= kErrWalk;
                break;
            }
            const uint32_t m = min( 32u * kCoopWidth, top );
            uint32_t       node[ kCoopWidth ];
#pragma unroll
            for ( uint32_t r = 0; r < kCoopWidth; r++ )
            {
                const uint32_t q = r * 32 + lane;
                node[ r ]        = q < m ? frontier[ top - 1 - q ] : kNone;
            }
            __syncwarp();
            uint32_t kids[ kCoopWidth ], first[ kCoopWidth ], second[ kCoopWidth ], jj[ kCoopWidth ];
            bool     contrib[ kCoopWidth ];
#pragma unroll
            for ( uint32_t r = 0; r < kCoopWidth; r++ )
            {
                first[ r ] = second[ r ] = 0;
                ordered_step( c, w, i, si, p, node[ r ], kids[ r ], first[ r ], second[ r ], contrib[ r ], jj[ r ] );
            }
            // earliest contributing position of this step
            uint32_t keep = m, base = top - m;
#pragma unroll
            for ( uint32_t r = 0; r < kCoopWidth; r++ )
            {
                const uint32_t hits = __ballot_sync( kFull, contrib[ r ] );
                if ( hits && keep == m )
                {
                    const uint32_t q = __ffs( hits ) - 1;
                    found            = __shfl_sync( kFull, jj[ r ], q );
                    keep             = r * 32 + q;
                    base             = 0;
                }
            }
            // children of the positions before `keep`, in position order, the earliest on top
            uint32_t off[ kCoopWidth ], mine[ kCoopWidth ], total = 0;
#pragma unroll
            for ( uint32_t r = 0; r < kCoopWidth; r++ )
            {
                mine[ r ]        = r * 32 + lane < keep ? kids[ r ] : 0u;
                uint32_t round   = 0;
                off[ r ]         = total + warp_exclusive_scan( mine[ r ], round );
                total           += round;
            }
            if ( base + total > kCoopCap )
            {
                err |= kErrStack;
                break;
            }
#pragma unroll
            for ( uint32_t r = 0; r < kCoopWidth; r++ )
            {
                if ( mine[ r ] >= 1 )
                    frontier[ base + total - 1 - off[ r ] ] = first[ r ];
                if ( mine[ r ] == 2 )
                    frontier[ base + total - 2 - off[ r ] ] = second[ r ];
            }
            __syncwarp();
            top = base + total;
        }
        return found;
    }

    __global__ void __launch_bounds__( kCellBlock, 4 ) k_edge_validation( CellContext c, const uint32_t * __restrict__ tasks,
                                                                      const uint32_t * __restrict__ task_count,
                                                                      SearchProof proof )
    {
        extern __shared__ __align__( 16 ) unsigned char smem[];
        const uint32_t warp  = threadIdx.x >> 5;
        const uint32_t gwarp = blockIdx.x * ( kCellBlock / 32 ) + warp;
        const uint32_t nwarp = gridDim.x * ( kCellBlock / 32 );
        const uint32_t lane  = lane_id();
        WarpCell       w     = carve( smem, warp, 0 );
        uint32_t       err   = 0;
        const uint32_t count = *task_count;
        const uint32_t n     = c.n;
        uint32_t *     frontier = c.walk_scratch + size_t( gwarp ) * kWalkScratchWords;
        uint32_t *     saved    = frontier + kCoopCap + lane * ( kStack + 1 );
        // tasks are taken one at a time from a shared counter; `gwarp` only names the scratch
        ( void ) nwarp;
        while ( true )
        {
            uint32_t t = 0;
            if ( lane == 0 )
                t = atomicAdd( c.work_counter, 1u );
            t = __shfl_sync( kFull, t, 0 );
            if ( t >= count )
                break;
            const uint32_t i      = tasks[ t ];
            const uint8_t  status = c.status[ i ];
            if ( status == kFullyValidated || status == kBuried )
                continue;
            const float   known = c.known_radii[ i ];
            const double4 si    = c.sites[ i ];
            const float4  fsi   = to_float( si );
            load_cell( c, w, i, si, false, false );
            for ( uint32_t e = lane; e < w.en; e += 32 )
                if ( estatus( w.e[ e ] ) != 1 )
                    w.e[ e ].w = ( w.e[ e ].w & 0xffffff00u ) | 2u;
            __syncwarp();
            bool           changedCell = false;
            bool           pristine    = true; // no update has touched the loaded cell yet
            const uint32_t steps       = w.en / 32 + 1;
            uint32_t       restarts    = 0;
            bool             monotone = proof.maybe_bits != nullptr; // neighbours still include U0
            const uint32_t   slot     = monotone ? proof.slots[ t ] : 0u;
            const uint32_t * maybe    = monotone ? proof.maybe_bits + size_t( slot ) * kMaybeWords : nullptr;
            const uint32_t   stored_en = w.en;
            for ( uint32_t es = 0; es < steps; es++ )
            {
                const uint32_t eid  = es * 32 + lane;
                uint32_t       k = kNone, l = kNone;
                bool           need = eid < w.en;
                if ( need )
                {
                    const uint4 r = w.e[ eid ];
                    k             = r.x;
                    l             = r.y;
                    need          = estatus( r ) == 2;
                }
                uint32_t type = 0, cnt = 0;
                double4  ev0 = make_double4( 0, 0, 0, 0 ), ev1 = make_double4( 0, 0, 0, 0 );
                if ( eid < w.en )
                    cnt = w.e[ eid ].z;
                double4  sk = make_double4( 0, 0, 0, 0 ), sl = make_double4( 0, 0, 0, 0 );
                if ( need )
                {
                    sk   = c.sites[ k ];
                    sl   = c.sites[ l ];
                    type = trisector( si, sk, sl, ev0, ev1 );
                }
                const bool   hyperbola = type == 1, ellipse = type == 2;
                const float4 v1 = to_float( ev0 ), v2 = to_float( ev1 );
                float3       n1 = make_float3( 0, 0, 0 ), n2 = make_float3( 0, 0, 0 );
                float3       pp1 = make_float3( 0, 0, 0 ), pp2 = make_float3( 0, 0, 0 );
                float4       bsph = make_float4( 0, 0, 0, 0 );
                if ( need && ellipse )
                {
                    const float3 center = ( f3( v1 ) + f3( v2 ) ) * .5f;
                    const float  radius = flength( center - f3( v1 ) ) + v1.w;
                    bsph                = make_float4( center.x, center.y, center.z, radius );
                }
                else if ( need )
                {
                    double3 nn1, nn2;
                    tangent_planes( si, sk, sl, nn1, nn2 );
                    n1               = to_float( nn1 );
                    n2               = to_float( nn2 );
                    const double3 p1 = d3( si ) + nn1 * si.w;
                    const double3 p2 = d3( sk ) + nn1 * sk.w;
                    const double3 p3 = d3( sl ) + nn1 * sl.w;
                    const double3 p4 = d3( si ) + nn2 * si.w;
                    const double3 p5 = d3( sk ) + nn2 * sk.w;
                    bsph             = to_float( sphere_from_points( p1, p2, p3, p5 ) );
                    pp1              = to_float( p1 );
                    pp2              = to_float( p4 );
                }
                const bool inside = lt_eps( flength( f3( fsi ) - f3( bsph ) ), known - bsph.w );
                if ( eid < w.en && inside )
                {
                    w.e[ eid ].w = ( w.e[ eid ].w & 0xffffff00u ) | 1u;
                    need         = false;
                }
                // reach of the search (see reach_radius): the stored vertices and the ones
                // added by this pass that lie on the edge, and its possible apexes
                float4 reach = make_float4( fsi.x, fsi.y, fsi.z, 0.f );
                // the third sites of the stored vertices on this edge: the neighbours bounding its
                // arc, tested first against a candidate root while the cell is the stored one
                // (whose vertex sites are all edge sites, so they belong to the same conjunction)
                uint32_t hint0 = kNone, hint1 = kNone;
                if ( need )
                {
                    double         wmax = 0.0;
                    const uint32_t svn  = c.vertex_nb[ i ];
                    for ( uint32_t v = 0; v < svn; v++ )
                    {
                        const uint4 r = c.vertices[ store_row( c, i ) * kMaxVertices + v ];
                        if ( vertex_on_edge( r, k, l ) )
                        {
                            wmax             = fmax( wmax, solve_vertex( c, si, r ).w );
                            const uint32_t m = ( r.x != k && r.x != l ) ? r.x : ( ( r.y != k && r.y != l ) ? r.y : r.z );
                            if ( hint0 == kNone )
                                hint0 = m;
                            else if ( hint1 == kNone && m != hint0 )
                                hint1 = m;
                        }
                    }
                    for ( uint32_t v = 0; v < w.vn; v++ )
                        if ( vertex_on_edge( w.v[ v ], k, l ) )
                            wmax = fmax( wmax, w.pos[ v ].w );
                    if ( ellipse || cnt == kNone )
                    {
                        const double4 apex[ 2 ] = { ev0, ev1 };
                        for ( uint32_t a = 0; a < 2; a++ )
                        {
                            bool out = false;
                            for ( uint32_t e2 = 0; e2 < w.en && !out; e2++ )
                            {
                                const uint4 r2 = w.e[ e2 ];
                                if ( r2.x != k && r2.x != l )
                                    out = clearly_outside( c.sites[ r2.x ], apex[ a ] );
                                if ( !out && r2.y != k && r2.y != l )
                                    out = clearly_outside( c.sites[ r2.y ], apex[ a ] );
                            }
                            if ( !out )
                                wmax = fmax( wmax, apex[ a ].w );
                        }
                    }
                    reach.w = reach_radius( wmax, si.w, c.scene->rmax );
                }

                // proven free of contributors on this very cell state
                bool skip = false;
                if ( monotone && need )
                {
                    // the edge's index in the stored cell, where the proof's bits refer
                    for ( uint32_t e0 = 0; e0 < stored_en; e0++ )
                    {
                        const uint4 r0 = c.edges[ store_row( c, i ) * kMaxEdges + e0 ];
                        if ( r0.x == k && r0.y == l )
                        {
                            skip = !( ( maybe[ e0 >> 5 ] >> ( e0 & 31 ) ) & 1u );
                            break;
                        }
                    }
                }

                // first site inside the bounding volume that gives the edge two valid vertices
                uint32_t stack[ kStack ];
                int      sp      = 0;
                uint32_t node    = 0;
                uint32_t found   = kNone;
                bool     walking = need && !skip;
                uint32_t walk_steps = 0;
                bool     suspended  = false;
                uint32_t saved_count = 0;
                while ( true )
                {
                    if ( walking && ++walk_steps > 4 * n + 64 )
                    {
                        err |= kErrWalk;
                        walking = false;
                    }
                    if ( walking && walk_steps > kLaneWalk )
                    {
                        // a long search: its position (current node, then the stack from the
                        // top) goes to scratch and the warp finishes it below
                        saved[ 0 ] = node;
                        for ( int q = 0; q < sp; q++ )
                            saved[ 1 + q ] = stack[ sp - 1 - q ];
                        saved_count = uint32_t( sp ) + 1;
                        suspended   = true;
                        walking     = false;
                    }
                    while ( walking && node < n - 1 )
                    {
                        Box      lb, rb;
                        uint32_t lc, rc;
                        load_node( c.nodes, node, lb, rb, lc, rc );
                        const float3   closeL = lb.closest( bsph ), closeR = rb.closest( bsph );
                        const float    dL = lb.distance( bsph ), dR = rb.distance( bsph );
                        const bool     leftClosest = dL < dR;
                        const float    minFar = leftClosest ? dR : dL, minClose = leftClosest ? dL : dR;
                        const float3   farPoint = leftClosest ? closeR : closeL, closePoint = leftClosest ? closeL : closeR;
                        const uint32_t farChild = leftClosest ? rc : lc, closeChild = leftClosest ? lc : rc;
                        bool           exploreFar = minFar < 0.f;
                        if ( hyperbola && exploreFar )
                            exploreFar = fdot( n1, farPoint - pp1 ) < 0.f && fdot( n2, farPoint - pp2 ) < 0.f;
                        bool exploreClose = minClose < 0.f;
                        if ( hyperbola && exploreClose )
                            exploreClose = fdot( n1, closePoint - pp1 ) < 0.f && fdot( n2, closePoint - pp2 ) < 0.f;
                        exploreFar   = exploreFar && ( leftClosest ? rb : lb ).distance( reach ) < 0.f;
                        exploreClose = exploreClose && ( leftClosest ? lb : rb ).distance( reach ) < 0.f;
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
                    const uint32_t j   = node - ( n - 1 );
                    bool           can = walking && node >= n - 1 && node < 2 * n - 1 && j != i && j != k && j != l
                                 && c.status[ j ] != kBuried;
                    double4 sj = make_double4( 0, 0, 0, 0 );
                    if ( can )
                    {
                        sj              = c.sites[ j ];
                        const float4 fj = to_float( sj );
                        can             = intersects( fj, bsph ) && flength( f3( fj ) - f3( reach ) ) <= reach.w;
                        if ( hyperbola )
                            can = can && double( fdot( n1, f3( fj ) - pp1 ) ) < -sj.w
                                  && double( fdot( n2, f3( fj ) - pp2 ) ) < -sj.w;
                    }
                    uint32_t cm = __ballot_sync( kFull, can );
                    while ( cm )
                    {
                        const uint32_t t2 = highest( cm );
                        cm &= ~( 1u << t2 );
                        const uint32_t tj     = __shfl_sync( kFull, j, t2 );
                        const bool     known2 = is_known( w, tj );
                        if ( lane == t2 )
                            can = !known2;
                    }
                    uint32_t mask = 0;
                    double4  x0 = make_double4( 0, 0, 0, 0 ), x1 = make_double4( 0, 0, 0, 0 );
                    if ( can )
                    {
                        mask = quadrisector( si, sj, sk, sl, x0, x1 );
                        if ( mask != 3 )
                            mask = 0;
                    }
                    uint32_t valid = mask;
                    uint32_t mm    = __ballot_sync( kFull, mask != 0 );
                    while ( mm )
                    {
                        const uint32_t t2 = highest( mm );
                        mm &= ~( 1u << t2 );
                        uint32_t       tm = __shfl_sync( kFull, mask, t2 );
                        const uint32_t tk = __shfl_sync( kFull, k, t2 ), tl = __shfl_sync( kFull, l, t2 );
                        while ( tm )
                        {
                            const uint32_t nv = __ffs( tm ) - 1;
                            tm &= ~( 1u << nv );
                            const double4  cand = shfl4( nv ? x1 : x0, t2 );
                            const uint32_t h0 = __shfl_sync( kFull, hint0, t2 ), h1 = __shfl_sync( kFull, hint1, t2 );
                            const bool     hinted = pristine && ( ( h0 != kNone && site_conflict( c, h0, cand, w.tally ) )
                                                              || ( h1 != kNone && site_conflict( c, h1, cand, w.tally ) ) );
                            const bool     ok   = !hinted && edges_clear( c, w, cand, tk, tl );
                            if ( lane == t2 && !ok )
                                valid &= ~( 1u << nv );
                        }
                    }
                    if ( valid )
                    {
                        found   = j;
                        walking = false;
                    }
                    if ( walking )
                    {
                        if ( sp == 0 )
                            walking = false;
                        else
                            node = stack[ --sp ];
                    }
                    if ( !__any_sync( kFull, walking ) )
                        break;
                }
                __syncwarp();
                uint32_t pending = __ballot_sync( kFull, suspended );
                while ( pending )
                {
                    const uint32_t src = __ffs( pending ) - 1;
                    pending &= pending - 1;
                    EdgeWalk p;
                    p.bsph      = shfl4f( bsph, src );
                    p.reach     = shfl4f( reach, src );
                    p.n1        = shfl3( n1, src );
                    p.n2        = shfl3( n2, src );
                    p.pp1       = shfl3( pp1, src );
                    p.pp2       = shfl3( pp2, src );
                    p.hyperbola = __shfl_sync( kFull, int( hyperbola ), src ) != 0;
                    p.k         = __shfl_sync( kFull, k, src );
                    p.l         = __shfl_sync( kFull, l, src );
                    p.sk        = shfl4( sk, src );
                    p.sl        = shfl4( sl, src );
                    const uint32_t cnt = __shfl_sync( kFull, saved_count, src );
                    const uint32_t got = ordered_edge_walk( c, w, i, si, p, frontier,
                                                            frontier + kCoopCap + src * ( kStack + 1 ), cnt, err );
                    if ( lane == src )
                        found = got;
                }
                if ( need && found == kNone )
                    w.e[ eid ].w = ( w.e[ eid ].w & 0xffffff00u ) | 1u;
                __syncwarp();

                uint32_t fm = __ballot_sync( kFull, found != kNone );
                while ( fm )
                {
                    const uint32_t t2 = highest( fm );
                    fm &= ~( 1u << t2 );
                    const uint32_t tj = __shfl_sync( kFull, found, t2 );
                    if ( is_known( w, tj ) )
                        continue;
                    const bool changed = update_cell( c, w, i, si, tj, c.sites[ tj ], err );
                    pristine           = false;
                    if ( monotone )
                    {
                        const uint32_t   cnt0 = proof.nbr_count[ slot ];
                        const uint32_t * u0   = proof.nbr + size_t( slot ) * kNbrCap;
                        for ( uint32_t q = 0; q < cnt0 && monotone; q++ )
                            monotone = is_known( w, u0[ q ] );
                    }
                    changedCell        = changedCell || changed;
                    if ( changed )
                    {
                        es = 0; // the reference restarts here; the loop's increment follows
                        if ( ++restarts > kMaxRestarts )
                        {
                            err |= kErrWalk;
                            es = steps;
                            break;
                        }
                    }
                }
            }
            const uint32_t base = c.vertex_nb[ i ];
            if ( lane == 0 )
                c.status[ i ] = changedCell ? 0 : 1;
            store_cell( c, w, i, base, err );
            __syncwarp();
        }
        report( c, err, w );
    }

    // -----------------------------------------------------------------------------------
    // Bisector validation (algorithm.inl:859-1233)
    // -----------------------------------------------------------------------------------
    // Cells are taken one at a time from a shared counter: their costs are uneven (a few hold
    // long searches), and a fixed share per warp left most warps idle at the end.
    __global__ void __launch_bounds__( kCellBlock, 3 ) k_bisector_validation( CellContext c, uint32_t * __restrict__ next )
    {
        extern __shared__ __align__( 16 ) unsigned char smem[];
        const uint32_t warp  = threadIdx.x >> 5;
        const uint32_t lane  = lane_id();
        WarpCell       w     = carve( smem, warp, kBisectorBytes );
        uint32_t *     bis   = reinterpret_cast<uint32_t *>( reinterpret_cast<unsigned char *>( w.e ) + sizeof( uint4 ) * kEdgeSlots );
        uint32_t       err   = 0;
        const uint32_t n     = c.n;
        while ( true )
        {
            uint32_t i = 0;
            if ( lane == 0 )
                i = c.lo + atomicAdd( next, 1u );
            i = __shfl_sync( kFull, i, 0 );
            if ( i >= c.hi )
                break;
            if ( c.status[ i ] == kBuried )
                continue;
            const float   known = c.known_radii[ i ];
            const double4 si    = c.sites[ i ];
            load_cell( c, w, i, si, false, false );

            // unique neighbour ids above i, ascending: bitonic sort of the edge sites
            uint32_t bisectorNb = 0;
            {
                const uint32_t total = 2 * w.en;
                uint32_t       size  = 64;
                while ( size < total )
                    size <<= 1;
                if ( size > 2 * kMaxBisectors )
                {
                    err |= kErrBisector;
                    size = 2 * kMaxBisectors;
                }
                for ( uint32_t x = lane; x < size; x += 32 )
                {
                    uint32_t v = kNone;
                    if ( x < total )
                    {
                        const uint4 r = w.e[ x >> 1 ];
                        v             = ( x & 1 ) ? r.y : r.x;
                        if ( v >= n )
                            v = kNone;
                    }
                    bis[ x ] = v;
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
                                const uint32_t a = bis[ x ], b = bis[ y ];
                                const bool     up = ( x & s2 ) == 0;
                                if ( ( a > b ) == up )
                                {
                                    bis[ x ] = b;
                                    bis[ y ] = a;
                                }
                            }
                        }
                        __syncwarp();
                    }
                // keep the first of each run, above i
                uint32_t kept = 0, carried = kNone;
                for ( uint32_t base = 0; base < size; base += 32 )
                {
                    const uint32_t x    = base + lane;
                    const uint32_t v    = bis[ x ];
                    uint32_t       prev = __shfl_up_sync( kFull, v, 1 );
                    if ( lane == 0 )
                        prev = carried;
                    const bool     keep = v != kNone && ( x == 0 || v != prev ) && v > i;
                    const uint32_t bal  = __ballot_sync( kFull, keep );
                    carried             = __shfl_sync( kFull, v, 31 );
                    __syncwarp();
                    if ( keep )
                        bis[ kept + __popc( bal & ( ( 1u << lane ) - 1u ) ) ] = v;
                    kept += __popc( bal );
                    __syncwarp();
                }
                bisectorNb = kept;
                if ( bisectorNb >= kMaxBisectors )
                    err |= kErrBisector;
            }

            const float3 fci = make_float3( float( si.x ), float( si.y ), float( si.z ) );
            const float  fri = float( si.w );
            bool         changedCell = false;
            const uint32_t steps     = bisectorNb / 32 + 1;
            uint32_t       restarts  = 0;
            for ( uint32_t bs = 0; bs < steps; bs++ )
            {
                const uint32_t bid      = bs * 32 + lane;
                uint32_t       bisector = kNone;
                bool           need     = bid < bisectorNb;
                if ( need )
                {
                    bisector = bis[ bid ];
                    need     = bisector != kNone;
                }
                double4 sk  = make_double4( 0, 0, 0, 0 );
                float3  fck = make_float3( 0, 0, 0 );
                float   frk = 0.f;
                if ( need )
                {
                    sk                   = c.sites[ bisector ];
                    fck                  = make_float3( float( sk.x ), float( sk.y ), float( sk.z ) );
                    frk                  = float( sk.w );
                    const float distance = flength( fci - fck ) + fri + frk;
                    if ( lt_eps( distance, known ) )
                    {
                        bis[ bid ] = kNone;
                        need       = false;
                    }
                }
                float  cylinder = 0.f;
                float4 bsph     = make_float4( 0, 0, 0, 0 );
                if ( need )
                {
                    const float3 center = ( fci + fck ) * .5f;
                    const float  radius = flength( center - fci ) + fmaxf( fri, frk );
                    bsph                = make_float4( center.x, center.y, center.z, radius );
                    cylinder            = fmaxf( fri, frk );
                }

                uint32_t stack[ kStack ];
                int      sp      = 0;
                uint32_t node    = 0;
                uint32_t found   = kNone;
                bool     walking = need;
                uint32_t walk_steps = 0;
                while ( true )
                {
                    if ( walking && ++walk_steps > 4 * n + 64 )
                    {
                        err |= kErrWalk;
                        walking = false;
                    }
                    while ( walking && node < n - 1 )
                    {
                        Box      lb, rb;
                        uint32_t lc, rc;
                        load_node( c.nodes, node, lb, rb, lc, rc );
                        const float    dL = lb.distance( bsph ), dR = rb.distance( bsph );
                        const bool     leftClosest = dL < dR;
                        const float    minFar = leftClosest ? dR : dL, minClose = leftClosest ? dL : dR;
                        const uint32_t farChild = leftClosest ? rc : lc, closeChild = leftClosest ? lc : rc;
                        const bool     exploreFar = minFar < 0.f, exploreClose = minClose < 0.f;
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
                    const uint32_t j   = node - ( n - 1 );
                    bool           can = walking && node >= n - 1 && node < 2 * n - 1 && j != i && j != bisector;
                    double4        sj  = make_double4( 0, 0, 0, 0 );
                    if ( can )
                    {
                        sj              = c.sites[ j ];
                        const float4 fj = to_float( sj );
                        const float3 cj = f3( fj );
                        can             = bsph.w >= fj.w && ( flength( f3( bsph ) - cj ) <= ( bsph.w - fj.w ) );
                        if ( can )
                        {
                            const float3 itoj = cj - fci;
                            const float  v    = fdot( itoj, fnormalize( fck - fci ) );
                            const float  d    = sqrtf( fdot( itoj, itoj ) - v * v );
                            can               = ( d + fj.w ) < cylinder;
                        }
                    }
                    uint32_t cm = __ballot_sync( kFull, can );
                    while ( cm )
                    {
                        const uint32_t t2 = highest( cm );
                        cm &= ~( 1u << t2 );
                        const uint32_t tj     = __shfl_sync( kFull, j, t2 );
                        const bool     known2 = is_known( w, tj );
                        if ( lane == t2 )
                            can = !known2;
                    }
                    double4 vtx = make_double4( 0, 0, 0, 0 );
                    if ( can )
                    {
                        double4 x0 = make_double4( 0, 0, 0, 0 ), x1 = make_double4( 0, 0, 0, 0 );
                        const uint32_t cnt = trisector( si, sj, sk, x0, x1 );
                        vtx                = x1;
                        can                = cnt == 2;
                    }
                    cm = __ballot_sync( kFull, can );
                    while ( cm )
                    {
                        const uint32_t t2 = highest( cm );
                        cm &= ~( 1u << t2 );
                        const uint32_t tk = __shfl_sync( kFull, bisector, t2 );
                        const double4  tv = shfl4( vtx, t2 );
                        const bool     ok = edges_clear( c, w, tv, tk, tk );
                        if ( lane == t2 )
                            can = can && ok;
                    }
                    if ( can )
                    {
                        found   = j;
                        walking = false;
                    }
                    if ( walking )
                    {
                        if ( sp == 0 )
                            walking = false;
                        else
                            node = stack[ --sp ];
                    }
                    if ( !__any_sync( kFull, walking ) )
                        break;
                }
                if ( need && found == kNone )
                    bis[ bid ] = kNone;
                __syncwarp();

                uint32_t fm = __ballot_sync( kFull, found != kNone );
                while ( fm )
                {
                    const uint32_t t2 = highest( fm );
                    fm &= ~( 1u << t2 );
                    const uint32_t tj = __shfl_sync( kFull, found, t2 );
                    if ( is_known( w, tj ) )
                        continue;
                    const bool changed = update_cell( c, w, i, si, tj, c.sites[ tj ], err );
                    changedCell        = changedCell || changed;
                    if ( changed )
                    {
                        bs = 0;
                        if ( ++restarts > kMaxRestarts )
                        {
                            err |= kErrWalk;
                            bs = steps;
                            break;
                        }
                    }
                }
            }
            const uint32_t base = c.vertex_nb[ i ];
            if ( lane == 0 )
                c.status[ i ] = changedCell ? 0 : 1;
            store_cell( c, w, i, base, err );
            __syncwarp();
        }
        report( c, err, w );
    }

    // -----------------------------------------------------------------------------------
    // Validation task lists on the device (replaces thrust::count / copy_if,
    // algorithm.inl:1551-1583)
    // -----------------------------------------------------------------------------------
    __global__ void k_tasks( const uint8_t * __restrict__ status, uint32_t lo, uint32_t hi, uint32_t * __restrict__ tasks,
                             uint32_t * __restrict__ count )
    {
        const uint32_t i    = lo + blockIdx.x * blockDim.x + threadIdx.x;
        const bool     open = i < hi && status[ i ] == kInValidation;
        const uint32_t bal  = __ballot_sync( kFull, open );
        uint32_t       base = 0;
        if ( lane_id() == 0 && bal )
            base = atomicAdd( count, __popc( bal ) );
        base = __shfl_sync( kFull, base, 0 );
        if ( open )
            tasks[ base + __popc( bal & ( ( 1u << lane_id() ) - 1u ) ) ] = i;
    }

    // -----------------------------------------------------------------------------------
    // Output: vertices owned by their smallest site (algorithm.inl:1235-1307) and closed
    // trisectors (:1309-1383); counts, an exclusive scan, then the writes.
    // -----------------------------------------------------------------------------------
    __device__ __forceinline__ bool owns_vertex( uint32_t id, uint4 r, uint32_t n )
    {
        return !( id > r.x || r.x >= n || r.y >= n || r.z >= n );
    }
    __device__ __forceinline__ bool owns_closed( uint32_t id, uint4 r, uint32_t n )
    {
        return !( r.z != kNone || id > r.x || r.x >= n || r.y >= n );
    }

    __global__ void k_count_owned( CellContext c, uint32_t * __restrict__ vcount, uint32_t * __restrict__ ccount )
    {
        const uint32_t gwarp = ( blockIdx.x * blockDim.x + threadIdx.x ) >> 5;
        const uint32_t nwarp = ( gridDim.x * blockDim.x ) >> 5;
        const uint32_t lane  = lane_id();
        for ( uint32_t i = gwarp; i < c.n; i += nwarp )
        {
            uint32_t vc = 0, cc = 0;
            if ( i >= c.lo && i < c.hi && c.status[ i ] != kBuried )
            {
                const uint32_t vn = c.vertex_nb[ i ], en = c.edge_nb[ i ];
                for ( uint32_t v = lane; v < vn; v += 32 )
                    vc += owns_vertex( i, c.vertices[ store_row( c, i ) * kMaxVertices + v ], c.n ) ? 1u : 0u;
                for ( uint32_t e = lane; e < en; e += 32 )
                    cc += owns_closed( i, c.edges[ store_row( c, i ) * kMaxEdges + e ], c.n ) ? 1u : 0u;
            }
            vc = __reduce_add_sync( kFull, vc );
            cc = __reduce_add_sync( kFull, cc );
            if ( lane == 0 )
            {
                vcount[ i ] = vc;
                ccount[ i ] = cc;
            }
        }
    }

    __global__ void k_write_owned( CellContext c, const uint32_t * __restrict__ voffset, const uint32_t * __restrict__ coffset,
                                   double4 * __restrict__ vpos, uint4 * __restrict__ vids, uint64_t vcap,
                                   double4 * __restrict__ cpos, uint4 * __restrict__ cids, uint64_t ccap )
    {
        const uint32_t gwarp = ( blockIdx.x * blockDim.x + threadIdx.x ) >> 5;
        const uint32_t nwarp = ( gridDim.x * blockDim.x ) >> 5;
        const uint32_t lane  = lane_id();
        for ( uint32_t i = gwarp; i < c.n; i += nwarp )
        {
            if ( i < c.lo || i >= c.hi || c.status[ i ] == kBuried )
                continue;
            const double4  si = c.sites[ i ];
            const uint32_t gi = c.indices[ i ];
            const uint32_t vn = c.vertex_nb[ i ], en = c.edge_nb[ i ];
            uint32_t       w  = voffset[ i ];
            for ( uint32_t base = 0; base < vn; base += 32 )
            {
                const uint32_t v   = base + lane;
                uint4          r   = make_uint4( 0, 0, 0, 0 );
                bool           own = false;
                if ( v < vn )
                {
                    r   = c.vertices[ store_row( c, i ) * kMaxVertices + v ];
                    own = owns_vertex( i, r, c.n );
                }
                const uint32_t bal = __ballot_sync( kFull, own );
                if ( own && w + __popc( bal & ( ( 1u << lane ) - 1u ) ) < vcap )
                {
                    const uint32_t dst = w + __popc( bal & ( ( 1u << lane ) - 1u ) );
                    vpos[ dst ]        = solve_vertex( c, si, r );
                    vids[ dst ]        = make_uint4( gi, c.indices[ r.x ], c.indices[ r.y ], c.indices[ r.z ] );
                }
                w += __popc( bal );
            }
            w = coffset[ i ];
            for ( uint32_t base = 0; base < en; base += 32 )
            {
                const uint32_t e   = base + lane;
                uint4          r   = make_uint4( 0, 0, 0, 0 );
                bool           own = false;
                if ( e < en )
                {
                    r   = c.edges[ store_row( c, i ) * kMaxEdges + e ];
                    own = owns_closed( i, r, c.n );
                }
                const uint32_t bal = __ballot_sync( kFull, own );
                if ( own && w + __popc( bal & ( ( 1u << lane ) - 1u ) ) < ccap )
                {
                    const uint32_t dst = w + __popc( bal & ( ( 1u << lane ) - 1u ) );
                    double4        x[ 2 ] = { make_double4( 0, 0, 0, 0 ), make_double4( 0, 0, 0, 0 ) };
                    trisector( si, c.sites[ r.x ], c.sites[ r.y ], x[ 0 ], x[ 1 ] );
                    if ( x[ 1 ].w < x[ 0 ].w )
                        x[ 0 ] = x[ 1 ];
                    cpos[ dst ] = x[ 0 ];
                    cids[ dst ] = make_uint4( gi, c.indices[ r.x ], c.indices[ r.y ], 0u );
                }
                w += __popc( bal );
            }
        }
    }

    // Exclusive scan of a u32 array in three steps: tile sums, a scan of the tile sums
    // (one block), and the tile scans with their offsets. Tiles are 2048 entries.
    constexpr uint32_t kScanBlock = 1024;
    constexpr uint32_t kScanTile  = 2 * kScanBlock;

    __device__ __forceinline__ uint32_t block_exclusive_scan( uint32_t v, uint32_t & total )
    {
        __shared__ uint32_t warp_sums[ 32 ];
        const uint32_t      lane = lane_id(), warp = threadIdx.x >> 5;
        uint32_t            wt;
        const uint32_t      ex = warp_exclusive_scan( v, wt );
        if ( lane == 0 )
            warp_sums[ warp ] = wt;
        __syncthreads();
        if ( warp == 0 )
        {
            const uint32_t s = lane < ( blockDim.x >> 5 ) ? warp_sums[ lane ] : 0u;
            uint32_t       t;
            const uint32_t e = warp_exclusive_scan( s, t );
            warp_sums[ lane ] = e;
            if ( lane == 31 )
                warp_sums[ 31 ] = e; // unchanged slot keeps its prefix
            if ( lane == 0 )
                total = t;
        }
        __syncthreads();
        const uint32_t r = warp_sums[ warp ] + ex;
        __syncthreads();
        return r;
    }

    __global__ void __launch_bounds__( kScanBlock ) k_tile_sums( const uint32_t * __restrict__ data, uint32_t n,
                                                                 uint32_t * __restrict__ sums )
    {
        const uint32_t base = blockIdx.x * kScanTile;
        uint32_t       v    = 0;
        for ( uint32_t x = threadIdx.x; x < kScanTile; x += kScanBlock )
            if ( base + x < n )
                v += data[ base + x ];
        v = __reduce_add_sync( kFull, v );
        __shared__ uint32_t part[ 32 ];
        if ( lane_id() == 0 )
            part[ threadIdx.x >> 5 ] = v;
        __syncthreads();
        if ( threadIdx.x < 32 )
        {
            uint32_t p = part[ threadIdx.x ];
            p          = __reduce_add_sync( kFull, p );
            if ( threadIdx.x == 0 )
                sums[ blockIdx.x ] = p;
        }
    }

    __global__ void __launch_bounds__( kScanBlock ) k_scan_tile_sums( uint32_t * sums, uint32_t tiles, uint64_t * total )
    {
        __shared__ uint32_t carry_s;
        if ( threadIdx.x == 0 )
            carry_s = 0;
        __syncthreads();
        for ( uint32_t base = 0; base < tiles; base += kScanBlock )
        {
            const uint32_t x = base + threadIdx.x;
            const uint32_t v = x < tiles ? sums[ x ] : 0u;
            __shared__ uint32_t chunk_total;
            uint32_t            t  = 0;
            const uint32_t      ex = block_exclusive_scan( v, t );
            if ( threadIdx.x == 0 )
                chunk_total = t;
            __syncthreads();
            if ( x < tiles )
                sums[ x ] = carry_s + ex;
            __syncthreads();
            if ( threadIdx.x == 0 )
                carry_s += chunk_total;
            __syncthreads();
        }
        if ( threadIdx.x == 0 )
            *total = carry_s;
    }

    __global__ void __launch_bounds__( kScanBlock ) k_scan_tiles( uint32_t * data, uint32_t n, const uint32_t * __restrict__ sums )
    {
        const uint32_t base = blockIdx.x * kScanTile;
        const uint32_t x0   = base + 2 * threadIdx.x;
        const uint32_t a    = x0 < n ? data[ x0 ] : 0u;
        const uint32_t b    = x0 + 1 < n ? data[ x0 + 1 ] : 0u;
        uint32_t       t;
        const uint32_t ex = block_exclusive_scan( a + b, t ) + sums[ blockIdx.x ];
        if ( x0 < n )
            data[ x0 ] = ex;
        if ( x0 + 1 < n )
            data[ x0 + 1 ] = ex + a;
    }

    size_t output_scan_scratch_words( uint32_t n ) { return ( n + kScanTile - 1 ) / kScanTile + 1; }

    void scan_exclusive( uint32_t * data, uint32_t n, uint32_t * sums, uint64_t * total, cudaStream_t s )
    {
        const uint32_t tiles = std::max( 1u, ( n + kScanTile - 1 ) / kScanTile );
        APO2_LAUNCH( "k_tile_sums", s, k_tile_sums<<<tiles, kScanBlock, 0, s>>>( data, n, sums ) );
        APO2_LAUNCH( "k_scan_tile_sums", s, k_scan_tile_sums<<<1, kScanBlock, 0, s>>>( sums, tiles, total ) );
        APO2_LAUNCH( "k_scan_tiles", s, k_scan_tiles<<<tiles, kScanBlock, 0, s>>>( data, n, sums ) );
    }

    // -----------------------------------------------------------------------------------
    // Launch helpers
    // -----------------------------------------------------------------------------------
    // Kernel attributes (dynamic shared memory above 48 KB) are per device, and so is the
    // persistent grid size derived from the device's SM count: both are set up once per
    // device, on the device current at the launch.
    constexpr int       kGridDevices = 64;
    static int          g_cell_grid[ kGridDevices ] = {};
    static PerDeviceOnce g_cell_config;

    static int current_device()
    {
        int dev = 0;
        cudaGetDevice( &dev );
        return dev;
    }

    static int & cell_grid_slot()
    {
        static int fallback = 0;
        const int  dev      = current_device();
        return ( dev >= 0 && dev < kGridDevices ) ? g_cell_grid[ dev ] : fallback;
    }

    void configure_cell_kernels()
    {
        g_cell_config.run( [] {
            const int dev = current_device();
            int       sms = 148;
            cudaDeviceGetAttribute( &sms, cudaDevAttrMultiProcessorCount, dev );
            cudaFuncSetAttribute( k_cells, cudaFuncAttributeMaxDynamicSharedMemorySize, int( cell_smem_bytes( false ) ) );
            cudaFuncSetAttribute( k_cells_profile, cudaFuncAttributeMaxDynamicSharedMemorySize, int( cell_smem_bytes( false ) ) );
            cudaFuncSetAttribute( k_vertex_validation, cudaFuncAttributeMaxDynamicSharedMemorySize, int( cell_smem_bytes( false ) ) );
            cudaFuncSetAttribute( k_edge_validation, cudaFuncAttributeMaxDynamicSharedMemorySize, int( cell_smem_bytes( false ) ) );
            cudaFuncSetAttribute( k_bisector_validation, cudaFuncAttributeMaxDynamicSharedMemorySize, int( cell_smem_bytes( true ) ) );
            int per_sm = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor( &per_sm, k_cells, kCellBlock, cell_smem_bytes( false ) );
            cell_grid_slot() = sms * std::max( 1, per_sm );
        } );
        if ( cell_grid_slot() == 0 ) // an ordinal outside the table: size it for 148 SMs x 4 blocks
            cell_grid_slot() = 148 * 4;
    }

    size_t walk_scratch_bytes()
    {
        configure_cell_kernels();
        return size_t( cell_grid_slot() ) * ( kCellBlock / 32 ) * kWalkScratchWords * sizeof( uint32_t );
    }

    static int cell_grid( uint32_t cells )
    {
        configure_cell_kernels();
        const int needed = int( ( uint64_t( cells ) + ( kCellBlock / 32 ) - 1 ) / ( kCellBlock / 32 ) );
        return std::max( 1, std::min( cell_grid_slot(), needed ) );
    }

    void launch_knn( const CellContext & c, uint32_t step, cudaStream_t s )
    {
        const uint32_t blocks = ( c.n + kKnnBlock - 1 ) / kKnnBlock;
        if ( c.proposal && step == 0 )
            APO2_LAUNCH( "k_knn_propose", s, k_knn<true><<<blocks, kKnnBlock, sizeof( ProposalNet ), s>>>( c, step ) );
        else
            APO2_LAUNCH( "k_knn", s, k_knn<false><<<blocks, kKnnBlock, 0, s>>>( c, step ) );
    }

    void launch_cells( const CellContext & c, uint32_t mode, cudaStream_t s )
    {
        cudaMemsetAsync( c.work_counter, 0, sizeof( uint32_t ), s );
        APO2_LAUNCH( "k_cells", s, k_cells<<<cell_grid( c.n ), kCellBlock, cell_smem_bytes( false ), s>>>( c, mode ) );
    }

    void launch_cells_profile( const CellContext & c, uint32_t step, uint32_t row, uint8_t * contributed, uint8_t * certified,
                               cudaStream_t s )
    {
        configure_cell_kernels();
        cudaMemsetAsync( c.work_counter, 0, sizeof( uint32_t ), s );
        APO2_LAUNCH( "k_cells_profile", s,
                     k_cells_profile<<<cell_grid( c.n ), kCellBlock, cell_smem_bytes( false ), s>>>( c, step, row, contributed, certified ) );
    }

    void launch_tasks( const CellContext & c, uint32_t * tasks, uint32_t * count, cudaStream_t s )
    {
        cudaMemsetAsync( count, 0, sizeof( uint32_t ), s );
        APO2_LAUNCH( "k_tasks", s, k_tasks<<<std::max( 1u, ( c.hi - c.lo + 255 ) / 256 ), 256, 0, s>>>( c.status, c.lo, c.hi, tasks, count ) );
    }

    void launch_vertex_validation( const CellContext & c, const uint32_t * tasks, const uint32_t * count, cudaStream_t s )
    {
        cudaMemsetAsync( c.work_counter, 0, sizeof( uint32_t ), s );
        APO2_LAUNCH( "k_vertex_validation", s, k_vertex_validation<<<cell_grid( c.n ), kCellBlock, cell_smem_bytes( false ), s>>>( c, tasks, count ) );
    }

    void launch_edge_validation( const CellContext & c, const uint32_t * tasks, const uint32_t * count, cudaStream_t s,
                                 SearchProof proof )
    {
        cudaMemsetAsync( c.work_counter, 0, sizeof( uint32_t ), s );
        APO2_LAUNCH( "k_edge_validation", s, k_edge_validation<<<cell_grid( c.n ), kCellBlock, cell_smem_bytes( false ), s>>>( c, tasks, count, proof ) );
    }

    void launch_bisector_validation( const CellContext & c, cudaStream_t s )
    {
        cudaMemsetAsync( c.work_counter, 0, sizeof( uint32_t ), s );
        APO2_LAUNCH( "k_bisector_validation", s, k_bisector_validation<<<cell_grid( c.n ), kCellBlock, cell_smem_bytes( true ), s>>>( c, c.work_counter ) );
    }

    void launch_output( const CellContext & c, const OutputBuffers & o, cudaStream_t s )
    {
        const uint32_t blocks = std::max( 1u, std::min<uint32_t>( ( c.n + 7 ) / 8, 148 * 16 ) );
        APO2_LAUNCH( "k_count_owned", s, k_count_owned<<<blocks, 256, 0, s>>>( c, o.vcount, o.ccount ) );
        const uint32_t tiles = std::max( 1u, ( c.n + kScanTile - 1 ) / kScanTile );
        scan_exclusive( o.vcount, c.n, o.tile_sums, o.totals + 0, s );
        scan_exclusive( o.ccount, c.n, o.tile_sums + tiles, o.totals + 1, s );
        APO2_LAUNCH( "k_write_owned", s, k_write_owned<<<blocks, 256, 0, s>>>( c, o.vcount, o.ccount, o.vpos, o.vids, o.vcap, o.cpos, o.cids, o.ccap ) );
    }
} // namespace apo2
