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
