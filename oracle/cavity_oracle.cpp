// CPU oracle of the cavity detection (TEST INFRASTRUCTURE ONLY: loaded by tests/ and by
// bench.py's CPU legs as the checker or the timed CPU baseline, never by the product).
//
// Restates the reference's cavity application (app/cavity/main.cpp:8-88):
//   - ray directions: the Halton sequence on the sphere in bases 2 and 3 (Wong, Luk and Heng,
//     "Sampling with Hammersley and Halton points", 1997) as app/cavity/utils.cu:201-242
//     generates it in single precision, scaled to unit length;
//   - occlusion (app/cavity/utils.cu:17-65, app/cavity/shaders/find_occlusion.cu:26-69): the
//     share of rays from a vertex centre that meet a sphere with 0.01 <= t <= 1e16, a ray from
//     inside a sphere meeting it where it leaves it. The reference traces with OptiX's sphere
//     intersector, whose arithmetic is not published; this oracle and the CUDA kernels both
//     decide each ray / sphere pair with the same single-precision test (component of c - o
//     across the ray, every operation rounded on its own; compiled with -ffp-contract=off), so
//     GPU and oracle agree bit for bit while the reference's OptiX run is not reproducible here;
//   - filter (app/cavity/utils.cu:67-83, 244-264, 527-559): hit ratio and radius above two thresholds.
//
// Two forms of the occlusion: every ray against every sphere (the definition), and a CPU
// sphere tree (median splits, boxes padded beyond the test's rounding, any-hit walk) that
// returns the same ratios faster, for larger checks and the CPU baseline.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

#include <omp.h>

namespace
{
    struct F3
    {
        float x, y, z;
    };
    struct F4
    {
        float x, y, z, w;
    };

    // find_occlusion.cu:46-58 (tmin 0.01, tmax 1e16), two-sided sphere
    bool meets( F3 o, F3 d, F4 s )
    {
        const float ox = s.x - o.x, oy = s.y - o.y, oz = s.z - o.z;
        const float b  = ( ox * d.x + oy * d.y ) + oz * d.z;
        const float hx = ox - b * d.x;
        const float hy = oy - b * d.y;
        const float hz = oz - b * d.z;
        const float h2 = ( hx * hx + hy * hy ) + hz * hz;
        const float disc = s.w * s.w - h2;
        if ( !( disc >= 0.f ) )
            return false;
        const float q = std::sqrt( disc );
        return b + q >= 0.01f && b - q <= 1e16f;
    }

    void directions( uint32_t count, std::vector<F3> & out )
    {
        out.resize( count );
        for ( uint32_t k = 0; k < count; k++ )
        {
            // base-2 radical inverse, as the reference accumulates it (p = 1/2, 1/4, ...)
            float t = 0.f;
            float p = 0.5f;
            for ( uint32_t kk = k; kk; kk >>= 1, p *= 0.5f )
                if ( kk & 1u )
                    t += p;
            t = 2.f * t - 1.f;
            const float st = std::sqrt( 1.f - t * t );
            // base-3 radical inverse
            float       phi = 0.f;
            const float ip  = 1.f / 3.f;
            p               = ip;
            for ( uint32_t kk = k; kk; kk /= 3, p *= ip )
            {
                const int a = int( kk % 3 );
                if ( a )
                    phi += float( a ) * p;
            }
            const float angle = float( double( phi * 4.f ) * 3.1415926535 );
            F3          v     = { st * std::cos( angle ), st * std::sin( angle ), t };
            const float len   = std::sqrt( v.x * v.x + v.y * v.y + v.z * v.z );
            out[ k ]          = { v.x / len, v.y / len, v.z / len };
        }
    }

    // CPU sphere tree: nodes over index ranges of a permutation, leaves of <= 4 spheres.
    struct Node
    {
        float    lo[ 3 ], hi[ 3 ];
        uint32_t left, right; // children, or (first, count) for a leaf
        bool     leaf;
    };

    struct Tree
    {
        std::vector<Node>     nodes;
        std::vector<uint32_t> order;
        const F4 *            s = nullptr;

        uint32_t build( uint32_t first, uint32_t count )
        {
            Node n {};
            for ( int a = 0; a < 3; a++ )
            {
                n.lo[ a ] = INFINITY;
                n.hi[ a ] = -INFINITY;
            }
            float clo[ 3 ] = { INFINITY, INFINITY, INFINITY }, chi[ 3 ] = { -INFINITY, -INFINITY, -INFINITY };
            for ( uint32_t i = first; i < first + count; i++ )
            {
                const F4    q      = s[ order[ i ] ];
                const float r      = std::fabs( q.w );
                const float c[ 3 ] = { q.x, q.y, q.z };
                for ( int a = 0; a < 3; a++ )
                {
                    n.lo[ a ] = std::min( n.lo[ a ], c[ a ] - r );
                    n.hi[ a ] = std::max( n.hi[ a ], c[ a ] + r );
                    clo[ a ]  = std::min( clo[ a ], c[ a ] );
                    chi[ a ]  = std::max( chi[ a ], c[ a ] );
                }
            }
            const uint32_t id = uint32_t( nodes.size() );
            nodes.push_back( n );
            if ( count <= 4 )
            {
                nodes[ id ].leaf  = true;
                nodes[ id ].left  = first;
                nodes[ id ].right = count;
                return id;
            }
            int axis = 0;
            for ( int a = 1; a < 3; a++ )
                if ( chi[ a ] - clo[ a ] > chi[ axis ] - clo[ axis ] )
                    axis = a;
            const uint32_t half = count / 2;
            std::nth_element( order.begin() + first, order.begin() + first + half, order.begin() + first + count,
                              [ & ]( uint32_t x, uint32_t y )
                              {
                                  const float cx = axis == 0 ? s[ x ].x : axis == 1 ? s[ x ].y : s[ x ].z;
                                  const float cy = axis == 0 ? s[ y ].x : axis == 1 ? s[ y ].y : s[ y ].z;
                                  return cx < cy;
                              } );
            const uint32_t l  = build( first, half );
            const uint32_t r  = build( first + half, count - half );
            nodes[ id ].leaf  = false;
            nodes[ id ].left  = l;
            nodes[ id ].right = r;
            return id;
        }
    };

    // padded slab test in double (conservative: the pad is far above the float test's error)
    bool meets_box( const double o[ 3 ], const double inv[ 3 ], const Node & n, double pad )
    {
        double tn = -INFINITY, tf = INFINITY;
        for ( int a = 0; a < 3; a++ )
        {
            const double t0 = ( double( n.lo[ a ] ) - pad - o[ a ] ) * inv[ a ];
            const double t1 = ( double( n.hi[ a ] ) + pad - o[ a ] ) * inv[ a ];
            tn              = std::max( tn, std::min( t0, t1 ) );
            tf              = std::min( tf, std::max( t0, t1 ) );
        }
        return tn <= tf && tf >= 0.0;
    }
} // namespace

extern "C" {

void oracle_cavity_directions( uint32_t count, float * xyz )
{
    std::vector<F3> d;
    directions( count, d );
    std::memcpy( xyz, d.data(), sizeof( F3 ) * count );
}

// vertices: float (x, y, z, w) [nv]; spheres: float (x, y, z, r) [ns]; ratios: float[nv].
// use_tree = 0: every ray against every sphere; 1: the CPU sphere tree.
void oracle_cavity_hit_ratios( const float * vertices, uint64_t nv, const float * spheres, uint32_t ns, uint32_t samples,
                               int use_tree, int threads, float * ratios )
{
    std::vector<F3> dirs;
    directions( samples, dirs );
    const F4 * v = reinterpret_cast<const F4 *>( vertices );
    const F4 * s = reinterpret_cast<const F4 *>( spheres );
    Tree       tree;
    double     scale = 0.0;
    if ( use_tree && ns )
    {
        tree.s = s;
        tree.order.resize( ns );
        std::iota( tree.order.begin(), tree.order.end(), 0u );
        tree.nodes.reserve( 2 * size_t( ns ) );
        tree.build( 0, ns );
        for ( uint32_t i = 0; i < ns; i++ )
            scale = std::max( { scale, double( std::fabs( s[ i ].x ) ), double( std::fabs( s[ i ].y ) ), double( std::fabs( s[ i ].z ) ),
                                double( std::fabs( s[ i ].w ) ) } );
    }
    if ( threads > 0 )
        omp_set_num_threads( threads );
#pragma omp parallel for schedule( dynamic, 64 )
    for ( int64_t i = 0; i < int64_t( nv ); i++ )
    {
        const F3 o    = { v[ i ].x, v[ i ].y, v[ i ].z };
        uint32_t hits = 0;
        const double od[ 3 ] = { o.x, o.y, o.z };
        const double pad = 1e-3 + 8e-6 * ( scale + std::max( { std::fabs( od[ 0 ] ), std::fabs( od[ 1 ] ), std::fabs( od[ 2 ] ) } ) );
        for ( uint32_t k = 0; k < samples; k++ )
        {
            const F3 d   = dirs[ k ];
            bool     hit = false;
            if ( !use_tree )
            {
                for ( uint32_t j = 0; j < ns && !hit; j++ )
                    hit = meets( o, d, s[ j ] );
            }
            else if ( ns )
            {
                const double inv[ 3 ] = { d.x != 0.f ? 1.0 / d.x : 1e300, d.y != 0.f ? 1.0 / d.y : 1e300,
                                          d.z != 0.f ? 1.0 / d.z : 1e300 };
                uint32_t     stack[ 128 ];
                int          sp = 0;
                stack[ sp++ ]   = 0;
                while ( sp && !hit )
                {
                    const Node & n = tree.nodes[ stack[ --sp ] ];
                    if ( !meets_box( od, inv, n, pad ) )
                        continue;
                    if ( n.leaf )
                    {
                        for ( uint32_t j = n.left; j < n.left + n.right && !hit; j++ )
                            hit = meets( o, d, s[ tree.order[ j ] ] );
                    }
                    else
                    {
                        stack[ sp++ ] = n.right;
                        stack[ sp++ ] = n.left;
                    }
                }
            }
            hits += hit ? 1u : 0u;
        }
        ratios[ i ] = float( hits ) / float( samples );
    }
}

// Cavity vertices: indices of the vertices with ratio > ratio_min and w > radius_min, in
// order; returns their number (app/cavity/utils.cu:527-559).
uint64_t oracle_cavity_filter( const float * vertices, const float * ratios, uint64_t nv, float ratio_min, float radius_min,
                               uint64_t * keep )
{
    uint64_t c = 0;
    for ( uint64_t i = 0; i < nv; i++ )
        if ( ratios[ i ] > ratio_min && vertices[ 4 * i + 3 ] > radius_min )
            keep[ c++ ] = i;
    return c;
}
}
