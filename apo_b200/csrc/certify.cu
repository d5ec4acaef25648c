// Interval certificate of output vertices and closed edges on the GPU: the reference's
// precision check (app/precision/precision.cpp:14-163), which runs on the CPU over all
// Q x N (vertex, site) pairs, restated over the LBVH.
//
// For an output point p with defining sites S (four for a vertex, three for a closed edge)
// the check computes each weighted distance d_s(p) = |c_s - p| - r_s as an interval
// (every operation rounded outward), takes R = max over S, and calls p bad when another
// site t is certainly closer: upper(d_t) < lower(R). Here the search for such a t walks the
// BVH and skips every box whose float distance to p, less a rounding allowance, is at
// least lower(R): no site in such a box can be closer than that.
#include <algorithm>
#include <cfloat>

#include "cells.cuh"

namespace apo2
{
    namespace
    {
        struct Interval
        {
            double lo, hi;
        };

        // Interval product [a, b] x [a, b] as a general product (both operands the same
        // interval, but not treated as a square, as an interval library multiplies them).
        __device__ __forceinline__ Interval self_product( double a, double b )
        {
            const double p0l = __dmul_rd( a, a ), p0h = __dmul_ru( a, a );
            const double p1l = __dmul_rd( a, b ), p1h = __dmul_ru( a, b );
            const double p2l = __dmul_rd( b, b ), p2h = __dmul_ru( b, b );
            return { fmin( p0l, fmin( p1l, p2l ) ), fmax( p0h, fmax( p1h, p2h ) ) };
        }

        // precision.cpp:14-24
        __device__ __forceinline__ Interval weighted_distance( double4 s, double px, double py, double pz )
        {
            const double c[ 3 ] = { s.x, s.y, s.z }, q[ 3 ] = { px, py, pz };
            double       lo = 0.0, hi = 0.0;
            for ( int a = 0; a < 3; a++ )
            {
                const Interval d2 = self_product( __dsub_rd( c[ a ], q[ a ] ), __dsub_ru( c[ a ], q[ a ] ) );
                lo                = __dadd_rd( lo, d2.lo );
                hi                = __dadd_ru( hi, d2.hi );
            }
            const double rlo = lo > 0.0 ? __dsqrt_rd( lo ) : 0.0;
            const double rhi = __dsqrt_ru( fmax( hi, 0.0 ) );
            return { __dsub_rd( rlo, s.w ), __dsub_ru( rhi, s.w ) };
        }

        __device__ __forceinline__ float box_distance( const Box & b, float3 p )
        {
            const float dx = fmaxf( fmaxf( b.lo.x - p.x, 0.f ), p.x - b.hi.x );
            const float dy = fmaxf( fmaxf( b.lo.y - p.y, 0.f ), p.y - b.hi.y );
            const float dz = fmaxf( fmaxf( b.lo.z - p.z, 0.f ), p.z - b.hi.z );
            return sqrtf( dx * dx + dy * dy + dz * dz );
        }

        __global__ void k_certify( const double4 * __restrict__ by_id, const double4 * __restrict__ sorted,
                                   const uint32_t * __restrict__ indices, const WideNode * __restrict__ nodes, uint32_t n,
                                   const double4 * __restrict__ points, const uint4 * __restrict__ ids, uint32_t arity,
                                   uint64_t count, float rmax, uint8_t * __restrict__ flags,
                                   unsigned long long * __restrict__ bad, uint32_t * __restrict__ error )
        {
            for ( uint64_t v = blockIdx.x * uint64_t( blockDim.x ) + threadIdx.x; v < count; v += uint64_t( gridDim.x ) * blockDim.x )
            {
                const double4 p  = points[ v ];
                const uint4   id = ids[ v ];
                const uint32_t own[ 4 ] = { id.x, id.y, id.z, arity == 4 ? id.w : id.z };
                // R = max of the defining sites' weighted distances (precision.cpp:37-71)
                Interval r = { -DBL_MAX, -DBL_MAX };
                bool     ok = true;
                for ( uint32_t a = 0; a < arity; a++ )
                {
                    if ( own[ a ] >= n )
                    {
                        ok = false;
                        break;
                    }
                    const Interval d = weighted_distance( by_id[ own[ a ] ], p.x, p.y, p.z );
                    r.lo             = fmax( r.lo, d.lo );
                    r.hi             = fmax( r.hi, d.hi );
                }
                bool closer = !ok;
                // float lower bound of the distance from p to a box, with an allowance for the
                // float rounding of p and of the box corners
                const float3 fp    = make_float3( float( p.x ), float( p.y ), float( p.z ) );
                const float  slack = 1e-5f * ( fabsf( fp.x ) + fabsf( fp.y ) + fabsf( fp.z ) + 1.f );
                const double limit = r.lo;
                uint32_t     stack[ kStack ];
                int          sp    = 0;
                uint32_t     node  = 0;
                uint32_t     steps = 0;
                while ( !closer )
                {
                    if ( ++steps > 4 * n + 64 )
                    {
                        atomicOr( error, kErrWalk );
                        break;
                    }
                    if ( node < n - 1 )
                    {
                        Box      lb, rb;
                        uint32_t lc, rc;
                        load_node( nodes, node, lb, rb, lc, rc );
                        // a site holding p can be as close as -rmax, whatever the box distance
                        const float bl = box_distance( lb, fp ), br = box_distance( rb, fp );
                        const bool  el = double( ( bl > 0.f ? bl : -rmax ) - slack ) < limit;
                        const bool  er = double( ( br > 0.f ? br : -rmax ) - slack ) < limit;
                        if ( el && er )
                        {
                            if ( sp < int( kStack ) )
                                stack[ sp++ ] = rc;
                            else
                            {
                                atomicOr( error, kErrStack );
                                break;
                            }
                            node = lc;
                            continue;
                        }
                        if ( el || er )
                        {
                            node = el ? lc : rc;
                            continue;
                        }
                    }
                    else if ( node < 2 * n - 1 )
                    {
                        const uint32_t j  = node - ( n - 1 );
                        const uint32_t sj = indices[ j ];
                        bool           mine = false;
                        for ( uint32_t a = 0; a < arity; a++ )
                            mine = mine || sj == own[ a ];
                        if ( !mine )
                        {
                            const Interval d = weighted_distance( sorted[ j ], p.x, p.y, p.z );
                            closer           = d.hi < r.lo; // certainly closer (precision.cpp:72-88)
                        }
                    }
                    if ( sp == 0 )
                        break;
                    node = stack[ --sp ];
                }
                if ( flags )
                    flags[ v ] = closer ? 1 : 0;
                if ( closer )
                    atomicAdd( bad, 1ull );
            }
        }
    } // namespace

    namespace
    {
        // Relative error of output vertices against an FP64 re-solve (the per-result error the
        // build reports). The reference solves a vertex in double precision but takes every
        // length with a single-precision square root (its `length`, gpu/math.cuh:307-309); the
        // check here refines the stored vertex (x, y, z, w) with Newton steps on the four
        // equations |p - c_a| - r_a - w = 0 of its sites, in IEEE double (correctly rounded
        // square roots, 4x4 solves with partial pivoting), and reports
        //     max over x, y, z, w of |stored - refined| / max(1, |refined|)
        // (the measure of the parity tests). A vertex whose system is singular keeps its
        // stored value as the refined one (error 0) and is counted in `singular`.
        __device__ bool solve4( double a[ 4 ][ 5 ] )
        {
            for ( int c = 0; c < 4; c++ )
            {
                int    piv  = c;
                double best = fabs( a[ c ][ c ] );
                for ( int r = c + 1; r < 4; r++ )
                    if ( fabs( a[ r ][ c ] ) > best )
                    {
                        best = fabs( a[ r ][ c ] );
                        piv  = r;
                    }
                if ( !( best > 1e-300 ) )
                    return false;
                if ( piv != c )
                    for ( int k = 0; k < 5; k++ )
                    {
                        const double t = a[ c ][ k ];
                        a[ c ][ k ]    = a[ piv ][ k ];
                        a[ piv ][ k ]  = t;
                    }
                for ( int r = c + 1; r < 4; r++ )
                {
                    const double f = a[ r ][ c ] / a[ c ][ c ];
                    for ( int k = c; k < 5; k++ )
                        a[ r ][ k ] = __fma_rn( -f, a[ c ][ k ], a[ r ][ k ] );
                }
            }
            for ( int r = 3; r >= 0; r-- )
            {
                double v = a[ r ][ 4 ];
                for ( int k = r + 1; k < 4; k++ )
                    v = __fma_rn( -a[ r ][ k ], a[ k ][ 4 ], v );
                a[ r ][ 4 ] = v / a[ r ][ r ];
            }
            return true;
        }

        __global__ void k_vertex_error( const double4 * __restrict__ by_id, uint32_t n, const double4 * __restrict__ points,
                                        const uint4 * __restrict__ ids, uint64_t count, double threshold,
                                        float * __restrict__ errors, unsigned long long * __restrict__ max_bits,
                                        unsigned long long * __restrict__ above, unsigned long long * __restrict__ singular )
        {
            for ( uint64_t v = blockIdx.x * uint64_t( blockDim.x ) + threadIdx.x; v < count; v += uint64_t( gridDim.x ) * blockDim.x )
            {
                const double4  p0 = points[ v ];
                const uint4    id = ids[ v ];
                const uint32_t own[ 4 ] = { id.x, id.y, id.z, id.w };
                double4        s[ 4 ];
                bool           ok = true;
                for ( int a = 0; a < 4; a++ )
                {
                    ok = ok && own[ a ] < n;
                    s[ a ] = ok ? by_id[ own[ a ] ] : make_double4( 0, 0, 0, 0 );
                }
                double x[ 4 ] = { p0.x, p0.y, p0.z, p0.w };
                for ( int it = 0; it < 4 && ok; it++ )
                {
                    double m[ 4 ][ 5 ];
                    for ( int a = 0; a < 4; a++ )
                    {
                        const double dx = x[ 0 ] - s[ a ].x, dy = x[ 1 ] - s[ a ].y, dz = x[ 2 ] - s[ a ].z;
                        const double d  = __dsqrt_rn( __fma_rn( dx, dx, __fma_rn( dy, dy, dz * dz ) ) );
                        if ( !( d > 0.0 ) )
                        {
                            ok = false;
                            break;
                        }
                        m[ a ][ 0 ] = dx / d;
                        m[ a ][ 1 ] = dy / d;
                        m[ a ][ 2 ] = dz / d;
                        m[ a ][ 3 ] = -1.0;
                        m[ a ][ 4 ] = -( d - s[ a ].w - x[ 3 ] );
                    }
                    if ( !ok || !solve4( m ) )
                    {
                        ok = false;
                        break;
                    }
                    for ( int k = 0; k < 4; k++ )
                        x[ k ] += m[ k ][ 4 ];
                }
                double err = 0.0;
                if ( ok )
                {
                    const double got[ 4 ] = { p0.x, p0.y, p0.z, p0.w };
                    for ( int k = 0; k < 4; k++ )
                        err = fmax( err, fabs( got[ k ] - x[ k ] ) / fmax( 1.0, fabs( x[ k ] ) ) );
                    if ( !( err == err ) ) // NaN: treat as singular
                    {
                        err = 0.0;
                        ok  = false;
                    }
                }
                if ( !ok )
                    atomicAdd( singular, 1ull );
                if ( errors )
                    errors[ v ] = float( err );
                if ( err > threshold )
                    atomicAdd( above, 1ull );
                atomicMax( max_bits, static_cast<unsigned long long>( __double_as_longlong( err ) ) );
            }
        }
    } // namespace

    void launch_vertex_error( const double4 * by_id, uint32_t n, const double4 * points, const uint4 * ids, uint64_t count,
                              double threshold, float * errors, unsigned long long * max_bits, unsigned long long * above,
                              unsigned long long * singular, cudaStream_t s )
    {
        const uint64_t blocks = std::min<uint64_t>( ( count + 255 ) / 256, 148 * 32 );
        APO2_LAUNCH( "k_vertex_error", s,
                     k_vertex_error<<<unsigned( std::max<uint64_t>( blocks, 1 ) ), 256, 0, s>>>( by_id, n, points, ids, count, threshold,
                                                                                                errors, max_bits, above, singular ) );
    }

    void launch_certify( const double4 * by_id, const double4 * sorted, const uint32_t * indices, const WideNode * nodes,
                         uint32_t n, const double4 * points, const uint4 * ids, uint32_t arity, uint64_t count, float rmax,
                         uint8_t * flags, unsigned long long * bad, uint32_t * error, cudaStream_t s )
    {
        const uint64_t blocks = std::min<uint64_t>( ( count + 255 ) / 256, 148 * 32 );
        APO2_LAUNCH( "k_certify", s,
                     k_certify<<<unsigned( std::max<uint64_t>( blocks, 1 ) ), 256, 0, s>>>( by_id, sorted, indices, nodes, n, points,
                                                                                           ids, arity, count, rmax, flags, bad, error ) );
    }
} // namespace apo2
