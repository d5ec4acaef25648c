// Cavity detection over the diagram, the consumer of the reference's cavity application
// (app/cavity/main.cpp:8-88, app/cavity/utils.cu, app/cavity/shaders/find_occlusion.cu),
// as CUDA kernels over a BVH of this library where the reference uses OptiX:
//
//  - occlusion (utils.cu:17-65, find_occlusion.cu:26-69): from the centre of every output
//    vertex, one ray along each of `samples` fixed directions; the vertex's hit ratio is the
//    share of rays that meet a sphere of the trace set with 0.01 <= t <= 1e16. A ray that
//    starts inside a sphere meets it where it leaves it (the reference's sphere geometry is
//    two-sided: its build input, optix/sphere_module.cu:25-44, leaves OptiX's single-sided
//    option unset);
//  - filter (utils.cu:67-83, 244-264, 527-559): the vertices whose hit ratio and radius exceed two
//    thresholds, in output order, as float (x, y, z, w).
//
// Whether one ray meets one sphere is decided by ray_meets_sphere() alone, in single
// precision with every operation rounded on its own. The BVH only skips boxes that no such
// hit can lie in (each box is padded well beyond the test's rounding error), so every ray's
// answer is the OR of that test over all spheres, whatever the tree looks like.
#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>

#include "cells.cuh"
#include "cavity.cuh"

namespace apo2
{
    namespace
    {
        constexpr uint32_t kOcclusionBlock = 128;
        constexpr uint32_t kTraceStack     = 64;
        constexpr float    kRayMin         = 0.01f; // find_occlusion.cu:49
        constexpr float    kRayMax         = 1e16f; // find_occlusion.cu:50

        // Ray o + t d (d of unit length) against the sphere |x - c| = r. The squared distance
        // from c to the line comes from the component of c - o across d, which keeps the
        // precision that b^2 - (|c - o|^2 - r^2) loses to cancellation (E. Haines et al.,
        // "Precision Improvements for Ray/Sphere Intersection", Ray Tracing Gems, 2019).
        // The crossings are t = b -/+ sqrt(r^2 - h^2); the ray meets the sphere when the far
        // one is at least kRayMin and the near one at most kRayMax.
        __device__ __forceinline__ bool ray_meets_sphere( float3 o, float3 d, float4 s )
        {
            const float ox = __fsub_rn( s.x, o.x ), oy = __fsub_rn( s.y, o.y ), oz = __fsub_rn( s.z, o.z );
            const float b  = __fadd_rn( __fadd_rn( __fmul_rn( ox, d.x ), __fmul_rn( oy, d.y ) ), __fmul_rn( oz, d.z ) );
            const float hx = __fsub_rn( ox, __fmul_rn( b, d.x ) );
            const float hy = __fsub_rn( oy, __fmul_rn( b, d.y ) );
            const float hz = __fsub_rn( oz, __fmul_rn( b, d.z ) );
            const float h2 = __fadd_rn( __fadd_rn( __fmul_rn( hx, hx ), __fmul_rn( hy, hy ) ), __fmul_rn( hz, hz ) );
            const float disc = __fsub_rn( __fmul_rn( s.w, s.w ), h2 );
            if ( !( disc >= 0.f ) )
                return false;
            const float q = __fsqrt_rn( disc );
            return __fadd_rn( b, q ) >= kRayMin && __fsub_rn( b, q ) <= kRayMax;
        }

        // Slab test of the ray against a box grown by `pad` on every side; returns the entry
        // parameter in `enter` (used to visit the nearer child first).
        __device__ __forceinline__ bool ray_meets_box( float3 o, float3 inv, const Box & b, float pad, float & enter )
        {
            const float x0 = ( b.lo.x - pad - o.x ) * inv.x, x1 = ( b.hi.x + pad - o.x ) * inv.x;
            const float y0 = ( b.lo.y - pad - o.y ) * inv.y, y1 = ( b.hi.y + pad - o.y ) * inv.y;
            const float z0 = ( b.lo.z - pad - o.z ) * inv.z, z1 = ( b.hi.z + pad - o.z ) * inv.z;
            const float tn = fmaxf( fmaxf( fminf( x0, x1 ), fminf( y0, y1 ) ), fminf( z0, z1 ) );
            const float tf = fminf( fminf( fmaxf( x0, x1 ), fmaxf( y0, y1 ) ), fmaxf( z0, z1 ) );
            enter          = tn;
            return tn <= tf && tf >= 0.f;
        }

        // float -> int with the order of the floats (for atomic min / max)
        __device__ __forceinline__ int ordered( float f )
        {
            const int i = __float_as_int( f );
            return i >= 0 ? i : i ^ 0x7fffffff;
        }
        __device__ __forceinline__ float unordered( int i ) { return __int_as_float( i >= 0 ? i : i ^ 0x7fffffff ); }

        __global__ void k_trace_box_init( int * acc )
        {
            if ( threadIdx.x < 3 )
                acc[ threadIdx.x ] = INT_MAX;
            else if ( threadIdx.x < 7 )
                acc[ threadIdx.x ] = INT_MIN;
        }

        // acc: min x y z of the centres, max x y z, max radius
        __global__ void k_trace_box( const float4 * __restrict__ spheres, uint32_t n, int * acc )
        {
            float lo[ 3 ] = { FLT_MAX, FLT_MAX, FLT_MAX }, hi[ 4 ] = { -FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX };
            for ( uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x )
            {
                const float4 s = spheres[ i ];
                lo[ 0 ]        = fminf( lo[ 0 ], s.x );
                lo[ 1 ]        = fminf( lo[ 1 ], s.y );
                lo[ 2 ]        = fminf( lo[ 2 ], s.z );
                hi[ 0 ]        = fmaxf( hi[ 0 ], s.x );
                hi[ 1 ]        = fmaxf( hi[ 1 ], s.y );
                hi[ 2 ]        = fmaxf( hi[ 2 ], s.z );
                hi[ 3 ]        = fmaxf( hi[ 3 ], fabsf( s.w ) );
            }
            for ( int o = 16; o > 0; o >>= 1 )
            {
                for ( int a = 0; a < 3; a++ )
                    lo[ a ] = fminf( lo[ a ], __shfl_xor_sync( 0xffffffffu, lo[ a ], o ) );
                for ( int a = 0; a < 4; a++ )
                    hi[ a ] = fmaxf( hi[ a ], __shfl_xor_sync( 0xffffffffu, hi[ a ], o ) );
            }
            if ( ( threadIdx.x & 31 ) == 0 )
            {
                for ( int a = 0; a < 3; a++ )
                    atomicMin( &acc[ a ], ordered( lo[ a ] ) );
                for ( int a = 0; a < 4; a++ )
                    atomicMax( &acc[ 3 + a ], ordered( hi[ a ] ) );
            }
        }

        // box: lo xyz, 1 / extent xyz (0 for a flat axis), pad, unused
        __global__ void k_trace_box_finish( const int * acc, float * box )
        {
            if ( threadIdx.x != 0 )
                return;
            float m = 0.f;
            for ( int a = 0; a < 3; a++ )
            {
                const float lo = unordered( acc[ a ] ), hi = unordered( acc[ 3 + a ] );
                box[ a ]       = lo;
                box[ 3 + a ]   = hi > lo ? 1.f / ( hi - lo ) : 0.f;
                m              = fmaxf( m, fmaxf( fabsf( lo ), fabsf( hi ) ) );
            }
            m += fmaxf( unordered( acc[ 6 ] ), 0.f );
            box[ 6 ] = kCavityPadBase + kCavityPadScale * m;
            box[ 7 ] = 0.f;
        }

        __global__ void k_trace_leaves( const float4 * __restrict__ spheres, const uint32_t * __restrict__ order, uint32_t n,
                                        float4 * __restrict__ sorted, float4 * __restrict__ boxes, int32_t * __restrict__ left,
                                        int32_t * __restrict__ right )
        {
            const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
            if ( b >= n )
                return;
            const float4   s    = spheres[ order[ b ] ];
            const uint32_t node = b + n - 1;
            sorted[ b ]         = s;
            const float    r    = fabsf( s.w ); // the ray test squares the radius
            boxes[ 2 * node + 0 ] = make_float4( s.x - r, s.y - r, s.z - r, 0.f );
            boxes[ 2 * node + 1 ] = make_float4( s.x + r, s.y + r, s.z + r, 0.f );
            left[ node ]          = int32_t( b );
            right[ node ]         = int32_t( b ) + 1;
        }

        // One thread per vertex, all threads of a warp on the same direction at a time, so a
        // warp's rays (neighbouring vertices in owner-cell Morton order, one direction) walk
        // much the same part of the tree. The vertex's own four sites are tried first: a ray
        // towards one of them needs no walk.
        __global__ void __launch_bounds__( kOcclusionBlock )
            k_occlusion( const double4 * __restrict__ vpos, const uint4 * __restrict__ vids, uint64_t count,
                         const float4 * __restrict__ spheres, uint32_t sphere_count, const float4 * __restrict__ sorted,
                         const WideNode * __restrict__ nodes, const float * __restrict__ box, const float4 * __restrict__ dirs,
                         uint32_t samples, float * __restrict__ ratios, uint32_t * __restrict__ error )
        {
            extern __shared__ float4 dir_smem[];
            float4 * sd = dir_smem;           // unit directions
            float4 * si = dir_smem + samples; // their reciprocals
            for ( uint32_t k = threadIdx.x; k < 2 * samples; k += blockDim.x )
                dir_smem[ k ] = dirs[ k ];
            __syncthreads();
            const uint64_t v = blockIdx.x * uint64_t( blockDim.x ) + threadIdx.x;
            if ( v >= count )
                return;
            const double4 p   = vpos[ v ];
            const float3  o   = make_float3( float( p.x ), float( p.y ), float( p.z ) );
            const uint4   ids = vids[ v ];
            const uint32_t own_id[ 4 ] = { ids.x, ids.y, ids.z, ids.w };
            float4         own[ 4 ];
            bool           has[ 4 ];
            for ( int a = 0; a < 4; a++ )
            {
                has[ a ] = own_id[ a ] < sphere_count;
                own[ a ] = has[ a ] ? __ldg( &spheres[ own_id[ a ] ] ) : make_float4( 0.f, 0.f, 0.f, 0.f );
            }
            const float pad = __ldg( &box[ 6 ] ) + kCavityPadScale * fmaxf( fmaxf( fabsf( o.x ), fabsf( o.y ) ), fabsf( o.z ) );
            const uint32_t n = sphere_count;

            uint32_t hits = 0;
            uint32_t stack[ kTraceStack ];
            for ( uint32_t k = 0; k < samples; k++ )
            {
                const float4 dv = sd[ k ], iv = si[ k ];
                const float3 d = make_float3( dv.x, dv.y, dv.z ), inv = make_float3( iv.x, iv.y, iv.z );
                bool         hit = false;
                for ( int a = 0; a < 4 && !hit; a++ )
                    hit = has[ a ] && ray_meets_sphere( o, d, own[ a ] );
                if ( !hit && n > 0 )
                {
                    int      sp    = 0;
                    uint32_t node  = 0;
                    uint32_t steps = 0;
                    while ( true )
                    {
                        if ( ++steps > 2 * n + 64 )
                        {
                            atomicOr( error, kErrWalk );
                            break;
                        }
                        if ( node + 1 < n )
                        {
                            Box      lb, rb;
                            uint32_t lc, rc;
                            load_node( nodes, node, lb, rb, lc, rc );
                            float      el, er;
                            const bool ml = ray_meets_box( o, inv, lb, pad, el );
                            const bool mr = ray_meets_box( o, inv, rb, pad, er );
                            if ( ml && mr )
                            {
                                if ( sp == int( kTraceStack ) )
                                {
                                    atomicOr( error, kErrStack );
                                    break;
                                }
                                const bool left_first = el <= er;
                                stack[ sp++ ]         = left_first ? rc : lc;
                                node                  = left_first ? lc : rc;
                                continue;
                            }
                            if ( ml || mr )
                            {
                                node = ml ? lc : rc;
                                continue;
                            }
                        }
                        else if ( ray_meets_sphere( o, d, __ldg( &sorted[ node - ( n - 1 ) ] ) ) )
                        {
                            hit = true;
                            break;
                        }
                        if ( sp == 0 )
                            break;
                        node = stack[ --sp ];
                    }
                }
                hits += hit ? 1u : 0u;
            }
            ratios[ v ] = __fdiv_rn( float( hits ), float( samples ) );
        }

        __global__ void k_cavity_flags( const double4 * __restrict__ vpos, const float * __restrict__ ratios, uint64_t count,
                                        float ratio_min, float radius_min, uint32_t * __restrict__ keep )
        {
            const uint64_t v = blockIdx.x * uint64_t( blockDim.x ) + threadIdx.x;
            if ( v >= count )
                return;
            keep[ v ] = ( ratios[ v ] > ratio_min && float( vpos[ v ].w ) > radius_min ) ? 1u : 0u;
        }

        __global__ void k_cavity_write( const double4 * __restrict__ vpos, const float * __restrict__ ratios, uint64_t count,
                                        float ratio_min, float radius_min, const uint32_t * __restrict__ offsets,
                                        float4 * __restrict__ out, uint64_t capacity )
        {
            const uint64_t v = blockIdx.x * uint64_t( blockDim.x ) + threadIdx.x;
            if ( v >= count )
                return;
            const double4 p = vpos[ v ];
            if ( ratios[ v ] > ratio_min && float( p.w ) > radius_min && offsets[ v ] < capacity )
                out[ offsets[ v ] ] = make_float4( float( p.x ), float( p.y ), float( p.z ), float( p.w ) );
        }

        inline uint32_t blocks_of( uint64_t n, uint32_t b ) { return uint32_t( std::max<uint64_t>( ( n + b - 1 ) / b, 1 ) ); }
    } // namespace

    // Points k = 0 .. count-1 of the Halton sequence on the sphere in bases 2 and 3 (T.-T. Wong,
    // W.-S. Luk, P.-A. Heng, "Sampling with Hammersley and Halton points", J. Graphics Tools 2(2),
    // 1997), in the single precision of the reference's generator (app/cavity/utils.cu:201-242,
    // including its angle of 4 pi times the base-3 radical inverse and its pi of 3.1415926535),
    // then scaled to unit length. dirs4 receives the directions (w = 0) and then their
    // reciprocals, a zero component standing as 1e-20 with its sign.
    void cavity_directions( uint32_t count, float * xyz, float * dirs4 )
    {
        for ( uint32_t k = 0; k < count; k++ )
        {
            float t = 0.f;
            for ( uint32_t kk = k, bit = 0; kk; kk >>= 1, bit++ )
                if ( kk & 1u )
                    t += std::ldexp( 1.f, -int( bit ) - 1 );
            t               = 2.f * t - 1.f;
            const float st  = std::sqrt( 1.f - t * t );
            float       phi = 0.f;
            const float ip  = 1.f / 3.f;
            float       p   = ip;
            for ( uint32_t kk = k; kk; kk /= 3 )
            {
                const uint32_t digit = kk % 3;
                if ( digit )
                    phi += float( digit ) * p;
                p *= ip;
            }
            const float angle = float( double( phi * 4.f ) * 3.1415926535 );
            float       v[ 3 ] = { st * std::cos( angle ), st * std::sin( angle ), t };
            const float len    = std::sqrt( v[ 0 ] * v[ 0 ] + v[ 1 ] * v[ 1 ] + v[ 2 ] * v[ 2 ] );
            for ( int a = 0; a < 3; a++ )
                v[ a ] = v[ a ] / len;
            for ( int a = 0; a < 3; a++ )
            {
                if ( xyz )
                    xyz[ 3 * k + a ] = v[ a ];
                if ( dirs4 )
                {
                    dirs4[ 4 * k + a ] = v[ a ];
                    const float d      = v[ a ] == 0.f ? std::copysign( 1e-20f, v[ a ] ) : v[ a ];
                    dirs4[ 4 * ( count + k ) + a ] = 1.f / d;
                }
            }
            if ( dirs4 )
            {
                dirs4[ 4 * k + 3 ]           = 0.f;
                dirs4[ 4 * ( count + k ) + 3 ] = 0.f;
            }
        }
    }

    size_t trace_tree_bytes( uint32_t n )
    {
        const size_t m = std::max<uint32_t>( n, 2 );
        auto         a = []( size_t b ) { return ( b + 255 ) & ~size_t( 255 ); };
        return a( 8 * m ) + a( 4 * m ) + 3 * a( 4 * ( 2 * m - 1 ) ) + a( 32 * ( 2 * m - 1 ) ) + a( 4 * m ) + a( 64 * m )
               + a( 16 * m ) + a( 64 ) + a( 32 ) + sort_scratch_bytes( uint32_t( m ) ) + 256;
    }

    void trace_tree_carve( TraceTree & t, void * base, uint32_t n, uint32_t * error_word )
    {
        const size_t m = std::max<uint32_t>( n, 2 );
        auto         a = []( size_t b ) { return ( b + 255 ) & ~size_t( 255 ); };
        char *       p = static_cast<char *>( base );
        t.codes        = reinterpret_cast<uint64_t *>( p );
        p += a( 8 * m );
        t.indices = reinterpret_cast<uint32_t *>( p );
        p += a( 4 * m );
        t.parent = reinterpret_cast<int32_t *>( p );
        p += a( 4 * ( 2 * m - 1 ) );
        t.left = reinterpret_cast<int32_t *>( p );
        p += a( 4 * ( 2 * m - 1 ) );
        t.right = reinterpret_cast<int32_t *>( p );
        p += a( 4 * ( 2 * m - 1 ) );
        t.boxes = reinterpret_cast<float4 *>( p );
        p += a( 32 * ( 2 * m - 1 ) );
        t.arrivals = reinterpret_cast<uint32_t *>( p );
        p += a( 4 * m );
        t.nodes = reinterpret_cast<WideNode *>( p );
        p += a( 64 * m );
        t.sorted = reinterpret_cast<float4 *>( p );
        p += a( 16 * m );
        t.acc = reinterpret_cast<int *>( p );
        p += a( 64 );
        t.box = reinterpret_cast<float *>( p );
        p += a( 32 );
        sort_scratch_carve( t.sort, p, uint32_t( m ), error_word );
        t.n = n;
    }

    void launch_trace_tree( TraceTree & t, const float4 * spheres, cudaStream_t s )
    {
        const uint32_t n = t.n;
        APO2_LAUNCH( "k_trace_box_init", s, k_trace_box_init<<<1, 32, 0, s>>>( t.acc ) );
        if ( n == 0 )
        {
            APO2_LAUNCH( "k_trace_box_finish", s, k_trace_box_finish<<<1, 32, 0, s>>>( t.acc, t.box ) );
            return;
        }
        APO2_LAUNCH( "k_trace_box", s, k_trace_box<<<std::min<uint32_t>( blocks_of( n, 256 ), 148 * 4 ), 256, 0, s>>>( spheres, n, t.acc ) );
        APO2_LAUNCH( "k_trace_box_finish", s, k_trace_box_finish<<<1, 32, 0, s>>>( t.acc, t.box ) );
        launch_morton_box( spheres, n, t.box, t.codes, t.indices, s );
        radix_sort_pairs( t.codes, t.indices, n, t.sort, s );
        APO2_LAUNCH( "k_trace_leaves", s,
                     k_trace_leaves<<<blocks_of( n, 256 ), 256, 0, s>>>( spheres, t.indices, n, t.sorted, t.boxes, t.left, t.right ) );
        launch_hierarchy( t.codes, n, t.parent, t.left, t.right, t.boxes, t.arrivals, t.nodes, s );
    }

    void launch_occlusion( const TraceTree & t, const float4 * spheres, const double4 * vpos, const uint4 * vids, uint64_t count,
                           const float4 * dirs, uint32_t samples, float * ratios, uint32_t * error, cudaStream_t s )
    {
        if ( count == 0 )
            return;
        const size_t smem = sizeof( float4 ) * 2 * samples;
        APO2_LAUNCH( "k_occlusion", s,
                     k_occlusion<<<blocks_of( count, kOcclusionBlock ), kOcclusionBlock, smem, s>>>(
                         vpos, vids, count, spheres, t.n, t.sorted, t.nodes, t.box, dirs, samples, ratios, error ) );
    }

    void launch_cavity_filter( const double4 * vpos, const float * ratios, uint64_t count, float ratio_min, float radius_min,
                               uint32_t * offsets, uint32_t * sums, uint64_t * total, float4 * out, uint64_t capacity,
                               cudaStream_t s )
    {
        if ( count == 0 )
        {
            cudaMemsetAsync( total, 0, sizeof( uint64_t ), s );
            return;
        }
        APO2_LAUNCH( "k_cavity_flags", s,
                     k_cavity_flags<<<blocks_of( count, 256 ), 256, 0, s>>>( vpos, ratios, count, ratio_min, radius_min, offsets ) );
        scan_exclusive( offsets, uint32_t( count ), sums, total, s );
        if ( out )
            APO2_LAUNCH( "k_cavity_write", s,
                         k_cavity_write<<<blocks_of( count, 256 ), 256, 0, s>>>( vpos, ratios, count, ratio_min, radius_min, offsets,
                                                                                out, capacity ) );
    }
} // namespace apo2
