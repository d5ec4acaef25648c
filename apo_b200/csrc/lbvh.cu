// LBVH over weighted sites: scene bounds, 63-bit Morton codes, a stable onesweep LSD radix
// sort of (code, index) pairs, Karras hierarchy emission and bottom-up refit.
//
// Results are bit-identical to the reference's LBVH (apo/src/gpu/lbvh.cu:11-323) and to
// its host-side bounds and bounding sites (apo/src/gpu/algorithm.cpp:5-25,
// apo/include/apo/gpu/algorithm.inl:1437-1464): the Morton quantisation uses the same float
// operations (the host-side 1/extent is an IEEE division here too), the sort is stable like
// thrust::sort_by_key, and the tie-break of equal codes by index is the same.
//
// Layout for the B200: sites are gathered once into Morton order as double4 (one 32-byte
// sector per random gather in the cell kernels) plus a float4 copy for traversal, and the
// tree is packed into 64-byte "wide" nodes that carry both child boxes, so a traversal step
// is one 64-byte load instead of two index loads and two box loads.
#include "internal.cuh"

namespace apo2
{
    // ---------------------------------------------------------------------------------
    // Scene bounds, fused with the float64 copy of the input (algorithm.cpp:5-25)
    // ---------------------------------------------------------------------------------
    constexpr int kBoundsBlock = 256;

    template<class In>
    __device__ __forceinline__ double4 load_site( const In * p, uint32_t i );
    template<>
    __device__ __forceinline__ double4 load_site<float4>( const float4 * p, uint32_t i )
    {
        const float4 s = p[ i ];
        return make_double4( s.x, s.y, s.z, s.w );
    }
    template<>
    __device__ __forceinline__ double4 load_site<double4>( const double4 * p, uint32_t i )
    {
        return p[ i ];
    }

    struct BoundsPartial
    {
        double lo[ 3 ], hi[ 3 ], rmin, rmax;
    };

    __device__ __forceinline__ void bounds_merge( BoundsPartial & a, const BoundsPartial & b )
    {
        for ( int c = 0; c < 3; c++ )
        {
            a.lo[ c ] = fmin( a.lo[ c ], b.lo[ c ] );
            a.hi[ c ] = fmax( a.hi[ c ], b.hi[ c ] );
        }
        a.rmin = fmin( a.rmin, b.rmin );
        a.rmax = fmax( a.rmax, b.rmax );
    }

    // PCG hash in the ldexp form of the reference's joggle (apo/src/core/utils.cpp:8-13).
    __device__ __forceinline__ double pcg_ldexp( uint32_t v )
    {
        const uint32_t state = v * 747796405u + 2891336453u;
        const uint32_t word  = ( ( state >> ( ( state >> 28u ) + 4u ) ) ^ state ) * 277803737u;
        return ldexp( double( ( word >> 22u ) ^ word ), -32 );
    }

    // Turns the reduced bounds into the scene box of the Morton quantisation and the six
    // joggled bounding sites (algorithm.inl:1442-1464). The reference evaluates this on the
    // host, so the arithmetic here is written with explicit round-to-nearest operations: no
    // contraction into fused multiply-adds.
    __device__ void finalize_scene( const BoundsPartial & b, uint32_t n, Scene * scene, double4 * artificial )
    {
        for ( int c = 0; c < 3; c++ )
        {
            scene->lo[ c ]        = b.lo[ c ];
            scene->hi[ c ]        = b.hi[ c ];
            scene->box_lo[ c ]    = float( b.lo[ c ] );
            scene->box_hi[ c ]    = float( b.hi[ c ] );
            scene->scale[ c ]     = __fdiv_rn( 1.f, __fsub_rn( float( b.hi[ c ] ), float( b.lo[ c ] ) ) );
        }
        scene->rmin = b.rmin;
        scene->rmax = b.rmax;

        const double cx = __ddiv_rn( __dadd_rn( b.lo[ 0 ], b.hi[ 0 ] ), 2.0 );
        const double cy = __ddiv_rn( __dadd_rn( b.lo[ 1 ], b.hi[ 1 ] ), 2.0 );
        const double cz = __ddiv_rn( __dadd_rn( b.lo[ 2 ], b.hi[ 2 ] ), 2.0 );
        const double dx = __dsub_rn( cx, b.hi[ 0 ] ), dy = __dsub_rn( cy, b.hi[ 1 ] ), dz = __dsub_rn( cz, b.hi[ 2 ] );
        const double sq = __dadd_rn( __dadd_rn( __dmul_rn( dx, dx ), __dmul_rn( dy, dy ) ), __dmul_rn( dz, dz ) );
        // host-side length(): IEEE single-precision square root (see fsqrtd in geometry.cuh)
        const double aabbRadius = double( __fsqrt_rn( __double2float_rn( sq ) ) );
        const double radius     = __dmul_rn( aabbRadius, __dadd_rn( __dsqrt_rn( 3.0 ), 1e-1 ) );
        const double offsets[ 6 ][ 3 ] = { { radius, 0, 0 }, { -radius, 0, 0 }, { 0, radius, 0 },
                                           { 0, -radius, 0 }, { 0, 0, radius }, { 0, 0, -radius } };
        const double randA = __dmul_rn( 2.0, 1e-1 );
        const double randB = -1e-1;
        for ( uint32_t a = 0; a < 6; a++ )
        {
            double v[ 4 ] = { __dadd_rn( cx, offsets[ a ][ 0 ] ), __dadd_rn( cy, offsets[ a ][ 1 ] ),
                              __dadd_rn( cz, offsets[ a ][ 2 ] ), __dadd_rn( 0.0, b.rmin ) };
            for ( uint32_t c = 0; c < 4; c++ )
                v[ c ] = __dadd_rn( v[ c ], __dadd_rn( __dmul_rn( pcg_ldexp( a * 4 + c ), randA ), randB ) );
            artificial[ a ] = make_double4( v[ 0 ], v[ 1 ], v[ 2 ], v[ 3 ] );
        }
        scene->n = n;
    }

    // One pass over the input: float64 copy of every site and the bounds of c -/+ r and r,
    // reduced per block, then by the last block to finish (no host round trip).
    template<class In>
    __global__ void __launch_bounds__( kBoundsBlock ) k_bounds( const In * __restrict__ input, uint32_t n,
                                                                 double4 * __restrict__ copy, BoundsPartial * partials,
                                                                 uint32_t * done_counter, Scene * scene,
                                                                 double4 * artificial )
    {
        BoundsPartial local;
        for ( int c = 0; c < 3; c++ )
        {
            local.lo[ c ] = DBL_MAX;
            local.hi[ c ] = -DBL_MAX;
        }
        local.rmin = DBL_MAX;
        local.rmax = -DBL_MAX;
        for ( uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x )
        {
            const double4 s = load_site( input, i );
            copy[ i ]       = s;
            local.lo[ 0 ]   = fmin( local.lo[ 0 ], s.x - s.w );
            local.lo[ 1 ]   = fmin( local.lo[ 1 ], s.y - s.w );
            local.lo[ 2 ]   = fmin( local.lo[ 2 ], s.z - s.w );
            local.hi[ 0 ]   = fmax( local.hi[ 0 ], s.x + s.w );
            local.hi[ 1 ]   = fmax( local.hi[ 1 ], s.y + s.w );
            local.hi[ 2 ]   = fmax( local.hi[ 2 ], s.z + s.w );
            local.rmin      = fmin( local.rmin, s.w );
            local.rmax      = fmax( local.rmax, s.w );
        }
        // warp then block reduction
        for ( int off = 16; off > 0; off >>= 1 )
        {
            BoundsPartial o;
            for ( int c = 0; c < 3; c++ )
            {
                o.lo[ c ] = __shfl_xor_sync( 0xffffffffu, local.lo[ c ], off );
                o.hi[ c ] = __shfl_xor_sync( 0xffffffffu, local.hi[ c ], off );
            }
            o.rmin = __shfl_xor_sync( 0xffffffffu, local.rmin, off );
            o.rmax = __shfl_xor_sync( 0xffffffffu, local.rmax, off );
            bounds_merge( local, o );
        }
        __shared__ BoundsPartial warps[ kBoundsBlock / 32 ];
        __shared__ bool          last;
        if ( ( threadIdx.x & 31 ) == 0 )
            warps[ threadIdx.x >> 5 ] = local;
        __syncthreads();
        if ( threadIdx.x == 0 )
        {
            BoundsPartial b = warps[ 0 ];
            for ( int w = 1; w < kBoundsBlock / 32; w++ )
                bounds_merge( b, warps[ w ] );
            partials[ blockIdx.x ] = b;
            __threadfence();
            last = atomicAdd( done_counter, 1u ) == gridDim.x - 1;
        }
        __syncthreads();
        if ( last && threadIdx.x == 0 )
        {
            __threadfence();
            BoundsPartial b = partials[ 0 ];
            for ( uint32_t p = 1; p < gridDim.x; p++ )
            {
                BoundsPartial q;
                const volatile BoundsPartial * vp = partials + p;
                for ( int c = 0; c < 3; c++ )
                {
                    q.lo[ c ] = vp->lo[ c ];
                    q.hi[ c ] = vp->hi[ c ];
                }
                q.rmin = vp->rmin;
                q.rmax = vp->rmax;
                bounds_merge( b, q );
            }
            finalize_scene( b, n, scene, artificial );
            *done_counter = 0; // ready for the next build
        }
    }

    // ---------------------------------------------------------------------------------
    // Morton codes (lbvh.cu:11-67)
    // ---------------------------------------------------------------------------------
    __device__ __forceinline__ uint32_t spread10( uint32_t x )
    {
        x = ( x | ( x << 16 ) ) & 0x030000FFu;
        x = ( x | ( x << 8 ) ) & 0x0300F00Fu;
        x = ( x | ( x << 4 ) ) & 0x030C30C3u;
        x = ( x | ( x << 2 ) ) & 0x09249249u;
        return x;
    }

    __device__ __forceinline__ uint64_t morton63( uint32_t x, uint32_t y, uint32_t z )
    {
        const uint64_t lo = spread10( x & 1023u ) | ( spread10( y & 1023u ) << 1 ) | ( spread10( z & 1023u ) << 2 );
        const uint64_t hi = spread10( x >> 10u ) | ( spread10( y >> 10u ) << 1 ) | ( spread10( z >> 10u ) << 2 );
        return ( hi << 30 ) | lo;
    }

    // (c - min) * scale, then * (2^20 - 1) and truncation to unsigned, all in float with the
    // reference's rounding (no contraction: separate round-to-nearest operations).
    __device__ __forceinline__ uint32_t quantize( float c, float lo, float scale )
    {
        const float u = __fmul_rn( __fsub_rn( c, lo ), scale );
        return __float2uint_rz( __fmul_rn( u, 1048575.f ) );
    }

    __global__ void k_morton( const double4 * __restrict__ sites, const Scene * __restrict__ scene, uint32_t n,
                              uint64_t * __restrict__ codes, uint32_t * __restrict__ indices )
    {
        const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
        if ( i >= n )
            return;
        const double4 s  = sites[ i ];
        const float   cx = float( s.x ), cy = float( s.y ), cz = float( s.z );
        codes[ i ]       = morton63( quantize( cx, scene->box_lo[ 0 ], scene->scale[ 0 ] ),
                               quantize( cy, scene->box_lo[ 1 ], scene->scale[ 1 ] ),
                               quantize( cz, scene->box_lo[ 2 ], scene->scale[ 2 ] ) );
        indices[ i ] = i;
    }

    // Morton codes of float4 sites inside a caller-given scene box (LBVH-only entry point).
    __global__ void k_morton_f32( const float4 * __restrict__ sites, float3 lo, float3 scale, uint32_t n,
                                  uint64_t * __restrict__ codes, uint32_t * __restrict__ indices )
    {
        const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
        if ( i >= n )
            return;
        const float4 s = sites[ i ];
        codes[ i ]     = morton63( quantize( s.x, lo.x, scale.x ), quantize( s.y, lo.y, scale.y ), quantize( s.z, lo.z, scale.z ) );
        indices[ i ]   = i;
    }

    // Morton codes of float4 sites inside a box held on the device: box[0..2] = lo,
    // box[3..5] = 1 / extent per axis.
    __global__ void k_morton_box( const float4 * __restrict__ sites, const float * __restrict__ box, uint32_t n,
                                  uint64_t * __restrict__ codes, uint32_t * __restrict__ indices )
    {
        const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
        if ( i >= n )
            return;
        const float4 s = sites[ i ];
        codes[ i ]     = morton63( quantize( s.x, box[ 0 ], box[ 3 ] ), quantize( s.y, box[ 1 ], box[ 4 ] ),
                                   quantize( s.z, box[ 2 ], box[ 5 ] ) );
        indices[ i ]   = i;
    }

    // ---------------------------------------------------------------------------------
    // Leaves: Morton-order gather of the sites and the leaf boxes (lbvh.cu:88-114)
    // ---------------------------------------------------------------------------------
    __global__ void k_leaves( const double4 * __restrict__ input, const uint32_t * __restrict__ order, uint32_t n,
                              double4 * __restrict__ sorted, float4 * __restrict__ sorted_f, float4 * __restrict__ boxes,
                              int32_t * __restrict__ left, int32_t * __restrict__ right )
    {
        const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
        if ( b >= n )
            return;
        const double4  s    = input[ order[ b ] ];
        const uint32_t node = b + n - 1;
        sorted[ b ]         = s;
        sorted_f[ b ]       = to_float( s );
        boxes[ 2 * node + 0 ] = make_float4( float( s.x - s.w ), float( s.y - s.w ), float( s.z - s.w ), 0.f );
        boxes[ 2 * node + 1 ] = make_float4( float( s.x + s.w ), float( s.y + s.w ), float( s.z + s.w ), 0.f );
        if ( left )
        {
            left[ node ]  = int32_t( b );
            right[ node ] = int32_t( b ) + 1;
        }
    }

    __global__ void k_leaves_f32( const float4 * __restrict__ input, const uint32_t * __restrict__ order, uint32_t n,
                                  float4 * __restrict__ boxes, int32_t * __restrict__ left, int32_t * __restrict__ right )
    {
        const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
        if ( b >= n )
            return;
        const float4   s    = input[ order[ b ] ];
        const uint32_t node = b + n - 1;
        boxes[ 2 * node + 0 ] = make_float4( s.x - s.w, s.y - s.w, s.z - s.w, 0.f );
        boxes[ 2 * node + 1 ] = make_float4( s.x + s.w, s.y + s.w, s.z + s.w, 0.f );
        left[ node ]          = int32_t( b );
        right[ node ]         = int32_t( b ) + 1;
    }

    // ---------------------------------------------------------------------------------
    // Karras 2012 hierarchy (lbvh.cu:144-223)
    // ---------------------------------------------------------------------------------
    __device__ __forceinline__ int prefix_delta( const uint64_t * __restrict__ codes, int i, int j, uint32_t n )
    {
        if ( j < 0 || j >= int( n ) )
            return -1;
        const uint64_t a = codes[ i ], b = codes[ j ];
        if ( a != b )
            return __clzll( a ^ b );
        return __clzll( (long long)( i ^ j ) ) + 64;
    }

    __global__ void k_karras( const uint64_t * __restrict__ codes, uint32_t n, int32_t * __restrict__ parent,
                              int32_t * __restrict__ left, int32_t * __restrict__ right )
    {
        const int i = int( blockIdx.x * blockDim.x + threadIdx.x );
        if ( i >= int( n ) - 1 )
            return;
        const int dr = prefix_delta( codes, i, i + 1, n ), dl = prefix_delta( codes, i, i - 1, n );
        const int d  = ( dr - dl > 0 ) - ( dr - dl < 0 );

        const int deltaMin = prefix_delta( codes, i, i - d, n );
        int       lmax     = 2;
        while ( prefix_delta( codes, i, i + lmax * d, n ) > deltaMin )
            lmax <<= 1;
        int l = 0;
        for ( int t = lmax >> 1; t >= 1; t >>= 1 )
            if ( prefix_delta( codes, i, i + ( l + t ) * d, n ) > deltaMin )
                l += t;
        const int j = i + l * d;

        const int deltaNode = prefix_delta( codes, i, j, n );
        int       s = 0, k = 2, t;
        do
        {
            t = ( l + k - 1 ) / k;
            k <<= 1;
            if ( prefix_delta( codes, i, i + ( s + t ) * d, n ) > deltaNode )
                s += t;
        } while ( t > 1 );
        const int gamma = i + s * d + min( d, 0 );

        int lc = gamma, rc = gamma + 1;
        if ( min( i, j ) == gamma )
            lc += int( n ) - 1;
        if ( max( i, j ) == gamma + 1 )
            rc += int( n ) - 1;
        left[ i ]    = lc;
        right[ i ]   = rc;
        parent[ lc ] = i;
        parent[ rc ] = i;
        if ( i == 0 )
            parent[ 0 ] = -1;
    }

    // ---------------------------------------------------------------------------------
    // Bottom-up refit (lbvh.cu:225-272): the second thread to reach a node merges its
    // children. Every step is a bounded climb (at most the tree height).
    // ---------------------------------------------------------------------------------
    __global__ void k_refit( uint32_t n, uint32_t * __restrict__ arrivals, const int32_t * __restrict__ parent,
                             const int32_t * __restrict__ left, const int32_t * __restrict__ right, float4 * boxes,
                             uint32_t * sizes )
    {
        const uint32_t leaf = blockIdx.x * blockDim.x + threadIdx.x + ( n - 1 );
        if ( leaf >= 2 * n - 1 )
            return;
        if ( sizes )
            sizes[ leaf ] = 1;
        int      node  = parent[ leaf ];
        uint32_t climb = 0;
        while ( node >= 0 && atomicAdd( &arrivals[ node ], 1u ) > 0 && ++climb <= 2 * n )
        {
            __threadfence();
            const int    l  = left[ node ], r = right[ node ];
            const float4 a0 = __ldcg( &boxes[ 2 * l ] ), a1 = __ldcg( &boxes[ 2 * l + 1 ] );
            const float4 b0 = __ldcg( &boxes[ 2 * r ] ), b1 = __ldcg( &boxes[ 2 * r + 1 ] );
            float3       lo = make_float3( FLT_MAX, FLT_MAX, FLT_MAX ), hi = make_float3( -FLT_MAX, -FLT_MAX, -FLT_MAX );
            lo              = fmin3( f3( a0 ), lo );
            hi              = fmax3( f3( a0 ), hi );
            lo              = fmin3( f3( a1 ), lo );
            hi              = fmax3( f3( a1 ), hi );
            lo              = fmin3( f3( b0 ), lo );
            hi              = fmax3( f3( b0 ), hi );
            lo              = fmin3( f3( b1 ), lo );
            hi              = fmax3( f3( b1 ), hi );
            __stcg( &boxes[ 2 * node ], make_float4( lo.x, lo.y, lo.z, 0.f ) );
            __stcg( &boxes[ 2 * node + 1 ], make_float4( hi.x, hi.y, hi.z, 0.f ) );
            if ( sizes )
                __stcg( &sizes[ node ], __ldcg( &sizes[ l ] ) + __ldcg( &sizes[ r ] ) );
            node = parent[ node ];
            __threadfence();
        }
    }

    // Wide nodes: internal node i carries both child boxes and both child ids.
    __global__ void k_pack( uint32_t n, const int32_t * __restrict__ left, const int32_t * __restrict__ right,
                            const float4 * __restrict__ boxes, WideNode * __restrict__ nodes )
    {
        const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
        if ( i + 1 >= n )
            return;
        const int    l  = left[ i ], r = right[ i ];
        const float4 a0 = boxes[ 2 * l ], a1 = boxes[ 2 * l + 1 ], b0 = boxes[ 2 * r ], b1 = boxes[ 2 * r + 1 ];
        WideNode     w;
        w.a        = make_float4( a0.x, a0.y, a0.z, a1.x );
        w.b        = make_float4( a1.y, a1.z, b0.x, b0.y );
        w.c        = make_float4( b0.z, b1.x, b1.y, b1.z );
        w.child    = make_int4( l, r, 0, 0 );
        nodes[ i ] = w;
    }

    // ---------------------------------------------------------------------------------
    // Host-side orchestration
    // ---------------------------------------------------------------------------------
    static inline uint32_t blocks_for( uint64_t n, uint32_t block ) { return uint32_t( ( n + block - 1 ) / block ); }

    void launch_bounds( const void * input, bool is_f64, uint32_t n, double4 * copy, BoundsPartial * partials,
                        uint32_t partial_count, uint32_t * counter, Scene * scene, double4 * artificial, cudaStream_t s )
    {
        const uint32_t grid = std::min<uint32_t>( partial_count, blocks_for( n, kBoundsBlock ) );
        if ( is_f64 )
            APO2_LAUNCH( "k_bounds", s, k_bounds<double4><<<grid, kBoundsBlock, 0, s>>>( static_cast<const double4 *>( input ), n, copy, partials,
                                                             counter, scene, artificial ) );
        else
            APO2_LAUNCH( "k_bounds", s, k_bounds<float4><<<grid, kBoundsBlock, 0, s>>>( static_cast<const float4 *>( input ), n, copy, partials,
                                                            counter, scene, artificial ) );
    }

    size_t bounds_partial_bytes( uint32_t count ) { return sizeof( BoundsPartial ) * count; }

    void launch_tree( const Tree & t, uint32_t n, const double4 * input, const Scene * scene, SortScratch & sort,
                      cudaStream_t s, uint32_t spin_limit )
    {
        APO2_LAUNCH( "k_morton", s, k_morton<<<blocks_for( n, 256 ), 256, 0, s>>>( input, scene, n, t.codes, t.indices ) );
        radix_sort_pairs( t.codes, t.indices, n, sort, s, spin_limit );
        APO2_LAUNCH( "k_leaves", s, k_leaves<<<blocks_for( n, 256 ), 256, 0, s>>>( input, t.indices, n, t.sites, t.sites_f, t.boxes, t.left, t.right ) );
        if ( n > 1 )
        {
            APO2_LAUNCH( "k_karras", s, k_karras<<<blocks_for( n - 1, 256 ), 256, 0, s>>>( t.codes, n, t.parent, t.left, t.right ) );
            cudaMemsetAsync( t.arrivals, 0, sizeof( uint32_t ) * ( n - 1 ), s );
            APO2_LAUNCH( "k_refit", s, k_refit<<<blocks_for( n, 256 ), 256, 0, s>>>( n, t.arrivals, t.parent, t.left, t.right, t.boxes, t.sizes ) );
            APO2_LAUNCH( "k_pack", s, k_pack<<<blocks_for( n - 1, 256 ), 256, 0, s>>>( n, t.left, t.right, t.boxes, t.nodes ) );
        }
    }

    void launch_morton_box( const float4 * sites, uint32_t n, const float * box, uint64_t * codes, uint32_t * indices,
                            cudaStream_t s )
    {
        APO2_LAUNCH( "k_morton_box", s, k_morton_box<<<blocks_for( n, 256 ), 256, 0, s>>>( sites, box, n, codes, indices ) );
    }

    void launch_hierarchy( const uint64_t * codes, uint32_t n, int32_t * parent, int32_t * left, int32_t * right, float4 * boxes,
                           uint32_t * arrivals, WideNode * nodes, cudaStream_t s )
    {
        if ( n < 2 )
            return;
        APO2_LAUNCH( "k_karras", s, k_karras<<<blocks_for( n - 1, 256 ), 256, 0, s>>>( codes, n, parent, left, right ) );
        cudaMemsetAsync( arrivals, 0, sizeof( uint32_t ) * ( n - 1 ), s );
        APO2_LAUNCH( "k_refit", s, k_refit<<<blocks_for( n, 256 ), 256, 0, s>>>( n, arrivals, parent, left, right, boxes, nullptr ) );
        APO2_LAUNCH( "k_pack", s, k_pack<<<blocks_for( n - 1, 256 ), 256, 0, s>>>( n, left, right, boxes, nodes ) );
    }

    void launch_lbvh_f32( const float4 * sites, uint32_t n, float3 lo, float3 scale, uint32_t * indices, uint64_t * codes,
                          int32_t * parent, int32_t * left, int32_t * right, float4 * boxes, uint32_t * sizes,
                          uint32_t * arrivals, SortScratch & sort, cudaStream_t s )
    {
        APO2_LAUNCH( "k_morton_f32", s, k_morton_f32<<<blocks_for( n, 256 ), 256, 0, s>>>( sites, lo, scale, n, codes, indices ) );
        radix_sort_pairs( codes, indices, n, sort, s );
        APO2_LAUNCH( "k_leaves_f32", s, k_leaves_f32<<<blocks_for( n, 256 ), 256, 0, s>>>( sites, indices, n, boxes, left, right ) );
        if ( n > 1 )
        {
            APO2_LAUNCH( "k_karras", s, k_karras<<<blocks_for( n - 1, 256 ), 256, 0, s>>>( codes, n, parent, left, right ) );
            cudaMemsetAsync( arrivals, 0, sizeof( uint32_t ) * ( n - 1 ), s );
            APO2_LAUNCH( "k_refit", s, k_refit<<<blocks_for( n, 256 ), 256, 0, s>>>( n, arrivals, parent, left, right, boxes, sizes ) );
        }
    }
} // namespace apo2
