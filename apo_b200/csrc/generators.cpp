// Seeded protein-like site sets: self-avoiding random-walk chains with covalent geometry.
//
// Stand-in for the PDB structures the reference measures on (chemfiles is not available
// to read them): chains of atoms with bond length 1.53 A, bond angle 109.5 +/- 10 degrees
// (uniform) and uniform torsion, started at uniform positions with a uniform initial
// direction inside a cube sized for the requested atom density, radii drawn from the
// van der Waals mix {1.20: 40%, 1.70: 32%, 1.55: 14%, 1.52: 13%, 1.80: 1%}. An atom is
// rejected when it overlaps a non-bonded atom by more than 0.5 A (checked on a uniform hash
// grid; "non-bonded" leaves out the 1-2 and 1-3 neighbours of the chain, whose distance is
// fixed by the bond geometry); after 64 rejections in a row the chain is restarted.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/apo2.h"

namespace
{
    // splitmix64: seeds the per-generator stream
    uint64_t splitmix( uint64_t & x )
    {
        uint64_t z = ( x += 0x9E3779B97F4A7C15ull );
        z          = ( z ^ ( z >> 30 ) ) * 0xBF58476D1CE4E5B9ull;
        z          = ( z ^ ( z >> 27 ) ) * 0x94D049BB133111EBull;
        return z ^ ( z >> 31 );
    }

    // xoshiro256** uniform generator
    struct Rng
    {
        uint64_t s[ 4 ];
        explicit Rng( uint64_t seed )
        {
            for ( auto & v : s )
                v = splitmix( seed );
        }
        static uint64_t rotl( uint64_t x, int k ) { return ( x << k ) | ( x >> ( 64 - k ) ); }
        uint64_t next()
        {
            const uint64_t r = rotl( s[ 1 ] * 5, 7 ) * 9;
            const uint64_t t = s[ 1 ] << 17;
            s[ 2 ] ^= s[ 0 ];
            s[ 3 ] ^= s[ 1 ];
            s[ 1 ] ^= s[ 2 ];
            s[ 0 ] ^= s[ 3 ];
            s[ 2 ] ^= t;
            s[ 3 ] = rotl( s[ 3 ], 45 );
            return r;
        }
        double uniform() { return double( next() >> 11 ) * 0x1.0p-53; }
    };

    struct V3
    {
        double x, y, z;
    };
    V3     operator+( V3 a, V3 b ) { return { a.x + b.x, a.y + b.y, a.z + b.z }; }
    V3     operator-( V3 a, V3 b ) { return { a.x - b.x, a.y - b.y, a.z - b.z }; }
    V3     operator*( V3 a, double s ) { return { a.x * s, a.y * s, a.z * s }; }
    double dot( V3 a, V3 b ) { return a.x * b.x + a.y * b.y + a.z * b.z; }
    V3     cross( V3 a, V3 b ) { return { a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x }; }
    V3     unit( V3 a ) { return a * ( 1.0 / std::sqrt( dot( a, a ) ) ); }

    V3 random_direction( Rng & rng )
    {
        const double z = 2.0 * rng.uniform() - 1.0;
        const double p = 2.0 * M_PI * rng.uniform();
        const double s = std::sqrt( std::max( 0.0, 1.0 - z * z ) );
        return { s * std::cos( p ), s * std::sin( p ), z };
    }

    double random_radius( Rng & rng )
    {
        const double u = rng.uniform();
        if ( u < 0.40 )
            return 1.20;
        if ( u < 0.72 )
            return 1.70;
        if ( u < 0.86 )
            return 1.55;
        if ( u < 0.99 )
            return 1.52;
        return 1.80;
    }

    struct Grid
    {
        double               lo, cell;
        int                  dim;
        std::vector<int32_t> head;
        std::vector<int32_t> next;
        int                  clampi( double v ) const
        {
            int c = int( std::floor( ( v - lo ) / cell ) );
            return c < 0 ? 0 : ( c >= dim ? dim - 1 : c );
        }
        size_t key( int x, int y, int z ) const { return ( size_t( x ) * dim + y ) * dim + z; }
    };
} // namespace

extern "C" apo2_status apo2_generate_chains( uint32_t chains, uint32_t atoms_per_chain, double density, uint64_t seed,
                                             float * out_xyzr )
{
    if ( !out_xyzr || chains == 0 || atoms_per_chain < 2 || !( density > 0.0 ) )
        return APO2_ERR_INVALID_ARG;
    const uint64_t total = uint64_t( chains ) * atoms_per_chain;
    if ( total > ( 1ull << 28 ) )
        return APO2_ERR_TOO_LARGE;
    const double side = std::cbrt( double( total ) / density );
    const double bond = 1.53, maxR = 1.80, overlap = 0.5;

    Grid g;
    g.cell = 2.0 * maxR;
    g.lo   = -60.0;
    g.dim  = int( std::ceil( ( side + 120.0 ) / g.cell ) );
    g.head.assign( size_t( g.dim ) * g.dim * g.dim, -1 );
    g.next.assign( total, -1 );
    std::vector<V3>     pos( total );
    std::vector<double> rad( total );
    Rng                 rng( seed );

    auto clashes = [ & ]( V3 p, double r, int64_t bonded, int64_t angle ) {
        const int cx = g.clampi( p.x ), cy = g.clampi( p.y ), cz = g.clampi( p.z );
        for ( int dx = -1; dx <= 1; dx++ )
            for ( int dy = -1; dy <= 1; dy++ )
                for ( int dz = -1; dz <= 1; dz++ )
                {
                    const int x = cx + dx, y = cy + dy, z = cz + dz;
                    if ( x < 0 || y < 0 || z < 0 || x >= g.dim || y >= g.dim || z >= g.dim )
                        continue;
                    for ( int32_t a = g.head[ g.key( x, y, z ) ]; a >= 0; a = g.next[ a ] )
                    {
                        if ( a == bonded || a == angle )
                            continue;
                        const V3 d = pos[ a ] - p;
                        const double lim = r + rad[ a ] - overlap;
                        if ( lim > 0 && dot( d, d ) < lim * lim )
                            return true;
                    }
                }
        return false;
    };
    auto insert = [ & ]( int64_t a ) {
        const size_t k = g.key( g.clampi( pos[ a ].x ), g.clampi( pos[ a ].y ), g.clampi( pos[ a ].z ) );
        g.next[ a ]    = g.head[ k ];
        g.head[ k ]    = int32_t( a );
    };
    auto remove = [ & ]( int64_t a ) {
        const size_t k = g.key( g.clampi( pos[ a ].x ), g.clampi( pos[ a ].y ), g.clampi( pos[ a ].z ) );
        int32_t *    p = &g.head[ k ];
        while ( *p >= 0 && *p != a )
            p = &g.next[ *p ];
        if ( *p == a )
            *p = g.next[ a ];
    };

    const double theta0 = 109.5 * M_PI / 180.0, dtheta = 10.0 * M_PI / 180.0;
    for ( uint32_t c = 0; c < chains; c++ )
    {
        const int64_t start    = int64_t( c ) * atoms_per_chain;
        int           restarts = 0;
        bool          done     = false;
        while ( !done )
        {
            for ( int64_t a = start; a < start + atoms_per_chain; a++ )
                if ( rad[ a ] > 0 )
                {
                    remove( a );
                    rad[ a ] = 0;
                }
            // first atom, uniform in the cube and clear of earlier chains
            int tries = 0;
            do
            {
                pos[ start ] = { rng.uniform() * side, rng.uniform() * side, rng.uniform() * side };
                rad[ start ] = random_radius( rng );
            } while ( clashes( pos[ start ], rad[ start ], -1, -1 ) && ++tries < 1000 );
            insert( start );
            V3 dir  = random_direction( rng ); // direction of the previous bond
            V3 perp = unit( cross( dir, std::fabs( dir.x ) < 0.9 ? V3 { 1, 0, 0 } : V3 { 0, 1, 0 } ) );
            done    = true;
            for ( int64_t a = start + 1; a < start + atoms_per_chain && done; a++ )
            {
                bool placed = false;
                for ( int t = 0; t < 64 && !placed; t++ )
                {
                    const double theta = theta0 + ( 2.0 * rng.uniform() - 1.0 ) * dtheta;
                    const double phi   = 2.0 * M_PI * rng.uniform();
                    // next bond at angle theta to the previous bond's reverse, torsion phi
                    const V3     b2 = cross( dir, perp );
                    const double ca = std::cos( M_PI - theta ), sa = std::sin( M_PI - theta );
                    const V3     nd = unit( dir * ca + ( perp * std::cos( phi ) + b2 * std::sin( phi ) ) * sa );
                    const V3     p  = pos[ a - 1 ] + nd * bond;
                    const double r  = random_radius( rng );
                    if ( !clashes( p, r, a - 1, a >= start + 2 ? a - 2 : -1 ) )
                    {
                        pos[ a ] = p;
                        rad[ a ] = r;
                        insert( a );
                        perp   = unit( cross( nd, dir ) );
                        dir    = nd;
                        placed = true;
                    }
                }
                if ( !placed )
                {
                    if ( ++restarts > 1000 )
                        return APO2_ERR_ITER_LIMIT;
                    done = false;
                }
            }
        }
    }
    for ( uint64_t a = 0; a < total; a++ )
    {
        out_xyzr[ 4 * a + 0 ] = float( pos[ a ].x );
        out_xyzr[ 4 * a + 1 ] = float( pos[ a ].y );
        out_xyzr[ 4 * a + 2 ] = float( pos[ a ].z );
        out_xyzr[ 4 * a + 3 ] = float( rad[ a ] );
    }
    return APO2_OK;
}
