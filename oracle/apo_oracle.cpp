// CPU oracle for the Apollonius-diagram construction path -- TEST INFRASTRUCTURE ONLY.
// See apo_oracle.h for what it restates and who may call it. Every function cites the
// reference file and lines it follows (paths relative to the PlathC/apo tree).
//
// Build: oracle/Makefile (g++ -O2 -fopenmp -ffp-contract=off).
#include "apo_oracle.h"

#include <algorithm>
#include <array>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace
{
    // ------------------------------------------------------------------------------------
    // Small vector types (single and double precision) and the reference's eps predicates
    // ------------------------------------------------------------------------------------
    struct F3 { float x, y, z; };
    struct F4 { float x, y, z, w; };
    struct D2 { double x, y; };
    struct D3 { double x, y, z; };
    struct D4 { double x, y, z, w; };

    constexpr uint32_t kNone = 0xffffffffu;

    // core/math.inl:217-244 -- absolute-eps comparisons used by every geometric decision.
    template<class T> inline bool lessThan( T a, T b, T eps = T( 1e-8 ) ) { return ( a - b ) < eps; }
    template<class T> inline bool greaterThan( T a, T b, T eps = T( 1e-8 ) ) { return ( a - b ) > -eps; }
    template<class T> inline bool isCloseToZero( T v, T eps = T( 1e-8 ) ) { return std::fabs( v ) < eps; }
    template<class T> inline T signOf( T a ) { return lessThan( a, T( 0 ) ) ? T( -1 ) : T( 1 ); }
    // core/math.inl:204-211 (numpy isclose with atol 1e-5, rtol 1e-8)
    inline bool isClose( double a, double ref ) { return std::fabs( a - ref ) <= ( 1e-5 + 1e-8 * std::fabs( ref ) ); }
    // Device min/max on double and float follow fmin/fmax (a NaN operand is ignored).
    inline double dmax( double a, double b ) { return std::fmax( a, b ); }
    inline double dmin( double a, double b ) { return std::fmin( a, b ); }
    inline float fmaxf_( float a, float b ) { return std::fmax( a, b ); }
    inline float fminf_( float a, float b ) { return std::fmin( a, b ); }

    inline D3 xyz( const D4 & s ) { return { s.x, s.y, s.z }; }
    inline F3 xyz( const F4 & s ) { return { s.x, s.y, s.z }; }
    inline D3 sub( const D3 & a, const D3 & b ) { return { a.x - b.x, a.y - b.y, a.z - b.z }; }
    inline D3 add( const D3 & a, const D3 & b ) { return { a.x + b.x, a.y + b.y, a.z + b.z }; }
    inline D4 sub( const D4 & a, const D4 & b ) { return { a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w }; }
    inline D3 scale( const D3 & a, double b ) { return { b * a.x, b * a.y, b * a.z }; }
    inline double dot( const D3 & a, const D3 & b ) { return a.x * b.x + a.y * b.y + a.z * b.z; }
    inline double dot( const D2 & a, const D2 & b ) { return a.x * b.x + a.y * b.y; }
    inline D3 cross( const D3 & a, const D3 & b )
    {
        return { a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x };
    }
    // gpu/math.cuh:307-309 resolve their unqualified `sqrt` to apo::sqrt (core/math.inl:89-104),
    // whose double branch is behind a misspelled macro, so under nvcc every double length is
    // a single-precision square root of the float-rounded dot product. Restated as such.
    inline double fsqrtd( double v ) { return double( std::sqrt( float( v ) ) ); }
    inline double length( const D3 & v ) { return fsqrtd( dot( v, v ) ); }
    // gpu/math.cuh:276-280. The GPU uses the CUDA rsqrt(double); here 1/sqrt.
    inline D3 normalize( const D3 & v )
    {
        const double inv = 1.0 / std::sqrt( dot( v, v ) );
        return { v.x * inv, v.y * inv, v.z * inv };
    }

    inline F3 sub( const F3 & a, const F3 & b ) { return { a.x - b.x, a.y - b.y, a.z - b.z }; }
    inline F3 add( const F3 & a, const F3 & b ) { return { a.x + b.x, a.y + b.y, a.z + b.z }; }
    inline F3 scale( const F3 & a, float b ) { return { a.x * b, a.y * b, a.z * b }; }
    inline float dot( const F3 & a, const F3 & b ) { return a.x * b.x + a.y * b.y + a.z * b.z; }
    inline float length( const F3 & v ) { return std::sqrt( dot( v, v ) ); }
    inline F3 normalize( const F3 & v )
    {
        const float inv = 1.0f / std::sqrt( dot( v, v ) );
        return scale( v, inv );
    }

    inline F4 toFloat( const D4 & v )
    {
        return { float( v.x ), float( v.y ), float( v.z ), float( v.w ) };
    }
    inline F3 toFloat( const D3 & v ) { return { float( v.x ), float( v.y ), float( v.z ) }; }

    // gpu/math.cuh:368-388
    inline float sphereDistance( const F4 & a, const F4 & b )
    {
        return length( sub( xyz( a ), xyz( b ) ) ) - ( a.w + b.w );
    }
    inline double sphereDistance( const D4 & a, const D4 & b )
    {
        const D3 d { a.x - b.x, a.y - b.y, a.z - b.z };
        return length( d ) - ( a.w + b.w );
    }
    inline bool intersect( const F4 & a, const F4 & b ) { return lessThan( sphereDistance( a, b ), 0.f ); }
    inline bool intersect( const D4 & a, const D4 & b ) { return lessThan( sphereDistance( a, b ), 0. ); }

    // gpu/math.cuh:339-366, gpu/math.inl:79-101 -- axis-aligned box queries in float.
    struct Box
    {
        F3 lo, hi;
        F3 closestPoint( const F4 & s ) const
        {
            return { fminf_( fmaxf_( s.x, lo.x ), hi.x ), fminf_( fmaxf_( s.y, lo.y ), hi.y ),
                     fminf_( fmaxf_( s.z, lo.z ), hi.z ) };
        }
        float distance( const F4 & s ) const { return length( sub( xyz( s ), closestPoint( s ) ) ) - s.w; }
        float farthestDistance( const F4 & s ) const
        {
            const F3 centroid = scale( add( lo, hi ), .5f );
            const F3 c        = sub( xyz( s ), centroid );
            const F3 radius   = scale( F3 { std::fabs( lo.x - hi.x ), std::fabs( lo.y - hi.y ), std::fabs( lo.z - hi.z ) }, .5f );
            const F3 far { radius.x * signOf( -c.x ), radius.y * signOf( -c.y ), radius.z * signOf( -c.z ) };
            return length( sub( c, far ) ) - s.w;
        }
    };

    // ------------------------------------------------------------------------------------
    // Geometric kernels (gpu/math.cuh:390-780), double precision, reference operation order
    // ------------------------------------------------------------------------------------

    // gpu/math.cuh:398-411: inverse of the 3x3 matrix given by its columns (cofactor rule).
    inline void inverse3( const D3 & c1, const D3 & c2, const D3 & c3, D3 & i1, D3 & i2, D3 & i3 )
    {
        const double invD = 1.0 / dot( c1, cross( c2, c3 ) );
        const D3     r1   = cross( c2, c3 );
        const D3     r2   = cross( c3, c1 );
        const D3     r3   = cross( c1, c2 );
        i1                = { invD * r1.x, invD * r2.x, invD * r3.x };
        i2                = { invD * r1.y, invD * r2.y, invD * r3.y };
        i3                = { invD * r1.z, invD * r2.z, invD * r3.z };
    }

    // gpu/math.cuh:419-426: matrix (given by columns) times vector.
    inline D3 mul3( const D3 & c1, const D3 & c2, const D3 & c3, const D3 & b )
    {
        return { dot( D3 { c1.x, c2.x, c3.x }, b ), dot( D3 { c1.y, c2.y, c3.y }, b ), dot( D3 { c1.z, c2.z, c3.z }, b ) };
    }

    // gpu/math.cuh:636-701: vertices of the trisector of (s1, s2, s3) on the plane through
    // the three centres. x1 and x2 may alias (the reference calls it that way).
    uint8_t trisectorVertex( const D4 & s1, const D4 & s2, const D4 & s3, D4 & x1, D4 & x2 )
    {
        const D3     p1 = xyz( s1 ), p2 = xyz( s2 ), p3 = xyz( s3 );
        const double r1 = s1.w, r2 = s2.w, r3 = s3.w;
        const D4     nh1 = sub( s1, s2 ), nh2 = sub( s1, s3 );

        const D3     nIjk = normalize( cross( sub( p2, p1 ), sub( p3, p1 ) ) );
        const double w    = -dot( nIjk, p1 );
        const D3     mC { .5 * ( -dot( p1, p1 ) + dot( p2, p2 ) + r1 * r1 - r2 * r2 ),
                      .5 * ( -dot( p1, p1 ) + dot( p3, p3 ) + r1 * r1 - r3 * r3 ),
                      w };
        D3 i1, i2, i3;
        inverse3( { nh1.x, nh2.x, nIjk.x }, { nh1.y, nh2.y, nIjk.y }, { nh1.z, nh2.z, nIjk.z }, i1, i2, i3 );
        const D3 t  = mul3( i1, i2, i3, D3 { nh1.w, nh2.w, 0.0 } );
        const D3 mN { -t.x, -t.y, -t.z };
        const D3 mB = mul3( i1, i2, i3, mC );

        const double e1 = -mN.x * r1 - mB.x - p1.x;
        const double e2 = -mN.y * r1 - mB.y - p1.y;
        const double e3 = -mN.z * r1 - mB.z - p1.z;
        const double a  = mN.x * mN.x + mN.y * mN.y + mN.z * mN.z - 1.0;
        const double b  = 2.0 * ( mN.x * e1 + mN.y * e2 + mN.z * e3 );
        const double c  = e1 * e1 + e2 * e2 + e3 * e3;

        const double delta = b * b - 4.0 * a * c;
        uint8_t      count = 0;
        const double q     = -.5 * ( b - signOf( b ) * std::sqrt( delta ) );

        const double xd1 = ( c / q ) - r1;
        const D3     v1  = sub( scale( mN, xd1 ), mB );
        if ( greaterThan( xd1 + r1, 0.0 ) )
        {
            x1 = { v1.x, v1.y, v1.z, xd1 };
            count++;
        }
        const double xd2 = ( q / a ) - r1;
        const D3     v2  = sub( scale( mN, xd2 ), mB );
        if ( greaterThan( xd2 + r1, 0.0 ) )
        {
            x2 = { v2.x, v2.y, v2.z, xd2 };
            if ( count == 0 )
                x1 = x2;
            count++;
        }
        return count;
    }

    // gpu/math.cuh:703-780: the (up to two) Apollonius vertices tangent to four spheres.
    // Bit k of the result says that root k has a non-negative radius.
    uint8_t quadrisector( const D4 & s1, const D4 & s2, const D4 & s3, const D4 & s4, D4 & x1, D4 & x2 )
    {
        const D3     p1 = xyz( s1 ), p2 = xyz( s2 ), p3 = xyz( s3 ), p4 = xyz( s4 );
        const double r1 = s1.w, r2 = s2.w, r3 = s3.w, r4 = s4.w;
        const D4     nh1 = sub( s1, s2 ), nh2 = sub( s1, s3 ), nh3 = sub( s1, s4 );

        const D3 mC { .5 * ( -dot( p1, p1 ) + dot( p2, p2 ) + r1 * r1 - r2 * r2 ),
                      .5 * ( -dot( p1, p1 ) + dot( p3, p3 ) + r1 * r1 - r3 * r3 ),
                      .5 * ( -dot( p1, p1 ) + dot( p4, p4 ) + r1 * r1 - r4 * r4 ) };
        D3 i1, i2, i3;
        inverse3( { nh1.x, nh2.x, nh3.x }, { nh1.y, nh2.y, nh3.y }, { nh1.z, nh2.z, nh3.z }, i1, i2, i3 );
        const D3 t = mul3( i1, i2, i3, D3 { nh1.w, nh2.w, nh3.w } );
        const D3 mN { 0.0 - t.x, 0.0 - t.y, 0.0 - t.z };
        const D3 mB = mul3( i1, i2, i3, mC );

        const double e1 = -mN.x * r1 - mB.x - p1.x;
        const double e2 = -mN.y * r1 - mB.y - p1.y;
        const double e3 = -mN.z * r1 - mB.z - p1.z;
        const double a  = mN.x * mN.x + mN.y * mN.y + mN.z * mN.z - 1.0;
        const double b  = 2.0 * ( mN.x * e1 + mN.y * e2 + mN.z * e3 );
        const double c  = e1 * e1 + e2 * e2 + e3 * e3;

        const double delta = b * b - 4.0 * a * c;
        if ( lessThan( delta, 0.0 ) )
            return 0;

        const double q   = -.5 * ( b - signOf( b ) * std::sqrt( delta ) );
        const double xd1 = ( c / q ) - r1;
        const D3     v1  = sub( scale( mN, xd1 ), mB );
        x1               = { v1.x, v1.y, v1.z, xd1 };
        uint8_t mask     = uint8_t( greaterThan( xd1 + r1, 0.0 ) );
        if ( greaterThan( xd1 + r1, 0.0 ) )
            x1.w = length( sub( p1, v1 ) ) - s1.w;

        if ( !isCloseToZero( delta ) )
        {
            const double xd2 = ( q / a ) - r1;
            const D3     v2  = sub( scale( mN, xd2 ), mB );
            x2               = { v2.x, v2.y, v2.z, xd2 };
            if ( greaterThan( xd2 + r1, 0.0 ) )
                x2.w = length( sub( p1, v2 ) ) - s1.w;
            mask |= uint8_t( uint8_t( greaterThan( xd2 + r1, 0.0 ) ) << 1 );
        }
        return mask;
    }

    // gpu/math.cuh:428-503: symmetric 2x2 eigen-decomposition (LAPACK dlaev2 scheme).
    void eigendecomposition( const D2 & m1, const D2 & m2, D2 & e, D2 & v )
    {
        const double a = m1.x, b = m2.x, c = m2.y;
        const double sm = a + c, df = a - c, adf = std::fabs( df ), tb = b + b, ab = std::fabs( tb );
        double       acmx = a, acmn = c;
        if ( std::fabs( a ) <= std::fabs( c ) )
            std::swap( acmx, acmn );
        double aa = ab, bb = adf;
        if ( adf < ab )
            std::swap( aa, bb );
        const double temp = aa / bb;
        const double rt   = bb * fsqrtd( 1.0 + temp * temp );
        const double sgn1 = std::copysign( 1.0, sm );
        const double rt1  = .5 * ( sm + sgn1 * rt );
        const double rt2  = ( acmx / rt1 ) * acmn - ( b / rt1 ) * b;

        const double sgn2 = std::copysign( 1.0, df );
        const double cs   = df + sgn2 * rt;
        const double acs  = std::fabs( cs );
        aa                = tb;
        bb                = cs;
        if ( lessThan( acs, ab ) )
            std::swap( aa, bb );
        const double t   = -aa / bb;
        double       sn1 = 1.0 / fsqrtd( 1.0 + t * t );
        double       cs1 = t * sn1;
        if ( lessThan( acs, ab ) )
            std::swap( sn1, cs1 );
        if ( lessThan( acs, ab ) && isCloseToZero( ab ) )
        {
            cs1 = 1.0;
            sn1 = 0.0;
        }
        if ( isClose( sgn1, sgn2 ) )
        {
            const double tn = cs1;
            cs1             = -sn1;
            sn1             = tn;
        }
        e = { rt2, rt1 };
        v = { -sn1, cs1 };
    }

    // gpu/math.cuh:519-531
    double determinant( const D4 & c1, const D4 & c2, const D4 & c3, const D4 & c4 )
    {
        const double d1 = dot( D3 { c2.y, c2.z, c2.w }, cross( D3 { c3.y, c3.z, c3.w }, D3 { c4.y, c4.z, c4.w } ) );
        const double d2 = dot( D3 { c2.x, c2.z, c2.w }, cross( D3 { c3.x, c3.z, c3.w }, D3 { c4.x, c4.z, c4.w } ) );
        const double d3 = dot( D3 { c2.x, c2.y, c2.w }, cross( D3 { c3.x, c3.y, c3.w }, D3 { c4.x, c4.y, c4.w } ) );
        const double d4 = dot( D3 { c2.x, c2.y, c2.z }, cross( D3 { c3.x, c3.y, c3.z }, D3 { c4.x, c4.y, c4.z } ) );
        return c1.x * d1 - c1.y * d2 + c1.z * d3 - c1.w * d4;
    }

    // gpu/math.cuh:533-575: sphere through four points.
    D4 sphereFromPoints( const D3 & p1, const D3 & p2, const D3 & p3, const D3 & p4 )
    {
        const double t1 = -dot( p1, p1 ), t2 = -dot( p2, p2 ), t3 = -dot( p3, p3 ), t4 = -dot( p4, p4 );
        const D4     X { p1.x, p2.x, p3.x, p4.x }, Y { p1.y, p2.y, p3.y, p4.y }, Z { p1.z, p2.z, p3.z, p4.z };
        const D4     O { 1, 1, 1, 1 }, T { t1, t2, t3, t4 };
        const double t = determinant( X, Y, Z, O );
        const double d = determinant( T, Y, Z, O ) / t;
        const double e = determinant( X, T, Z, O ) / t;
        const double f = determinant( X, Y, T, O ) / t;
        const double g = determinant( X, Y, Z, T ) / t;
        return { -d * .5, -e * .5, -f * .5, .5 * std::sqrt( d * d + e * e + f * f - 4. * g ) };
    }

    // gpu/math.cuh:390-396 (2x2 inverse) and :413-417 (2x2 product), used by getTangentPlanes.
    void inverse2( const D2 & a1, const D2 & a2, D2 & c1, D2 & c2 )
    {
        const double inv = 1.0 / std::fma( a1.x, a2.y, -a2.x * a1.y );
        c1               = { inv * a2.y, -inv * a1.y };
        c2               = { -inv * a2.x, inv * a1.x };
    }
    void mul2( const D2 & a1, const D2 & a2, const D2 & b1, const D2 & b2, D2 & c1, D2 & c2 )
    {
        c1 = { a1.x * b1.x + a2.x * b1.y, a1.y * b1.x + a2.y * b1.y };
        c2 = { a1.x * b2.x + a2.x * b2.y, a1.y * b2.x + a2.y * b2.y };
    }

    // gpu/math.cuh:577-634: normals of the two planes tangent to three spheres.
    void getTangentPlanes( const D4 & s1, const D4 & s2, const D4 & s3, D3 & n1, D3 & n2 )
    {
        const D3 p1 = xyz( s1 ), p2 = xyz( s2 ), p3 = xyz( s3 );
        const D4 nh1 = sub( s1, s2 ), nh2 = sub( s1, s3 );
        const D2 aC1 { nh1.x, nh2.x }, aC2 { nh1.y, nh2.y }, bC1 { nh1.z, nh2.z }, bC2 { nh1.w, nh2.w };
        D2       iA1, iA2;
        inverse2( aC1, aC2, iA1, iA2 );
        D2 cC1, cC2;
        mul2( iA1, iA2, bC1, bC2, cC1, cC2 );
        const D2 eC1 { 1.0 + cC1.x * cC1.x + cC1.y * cC1.y, 0.0 + cC1.x * cC2.x + cC1.y * cC2.y };
        const D2 eC2 { 0.0 + cC1.x * cC2.x + cC1.y * cC2.y, -1.0 + cC2.x * cC2.x + cC2.y * cC2.y };
        D2       ev, evec;
        eigendecomposition( eC1, eC2, ev, evec );
        const double alpha0 = std::sqrt( std::fabs( ev.x ) );
        const double alpha1 = std::sqrt( std::fabs( ev.y ) );

        D2 z { 1, alpha0 / alpha1 };
        D2 y34 { dot( D2 { evec.x, -evec.y }, z ), dot( D2 { evec.y, evec.x }, z ) };
        double x1 = -dot( D2 { cC1.x, cC2.x }, y34 );
        double x2 = -dot( D2 { cC1.y, cC2.y }, y34 );
        n1        = normalize( D3 { x1, x2, y34.x } );

        z   = { 1, -alpha0 / alpha1 };
        y34 = { dot( D2 { evec.x, -evec.y }, z ), dot( D2 { evec.y, evec.x }, z ) };
        x1  = -dot( D2 { cC1.x, cC2.x }, y34 );
        x2  = -dot( D2 { cC1.y, cC2.y }, y34 );
        n2  = normalize( D3 { x1, x2, y34.x } );

        const D3 p = add( p1, scale( n1, s1.w ) );
        if ( greaterThan( std::fabs( dot( n1, sub( p, p1 ) ) - s1.w ), 1e-4 )
             || greaterThan( std::fabs( dot( n1, sub( p, p2 ) ) - s2.w ), 1e-4 )
             || greaterThan( std::fabs( dot( n1, sub( p, p3 ) ) - s3.w ), 1e-4 ) )
        {
            n1 = scale( n1, -1.0 );
            n2 = scale( n2, -1.0 );
        }
    }

    // ------------------------------------------------------------------------------------
    // Per-cell stores (gpu/topology_update.cuh:20-97, algorithm.inl:25-30)
    // ------------------------------------------------------------------------------------
    constexpr uint32_t kMaxVertices  = 152;
    constexpr uint32_t kMaxEdges     = 264;
    constexpr uint32_t kMaxNewEdges  = 64;
    constexpr uint32_t kMaxBisectors = 512;
    constexpr uint32_t kK            = 16;
    constexpr uint8_t  kInValidation = 0, kFullyValidated = 1, kBuried = 0xff;

    struct Vertex
    {
        uint32_t j, k, l;
        uint8_t  type, status;
    };
    struct Edge
    {
        uint32_t j, k, vertexNb;
        uint8_t  status, validatedNb;
    };
    struct Cell
    {
        std::vector<Vertex> v;
        std::vector<Edge>   e;
        uint32_t            vn = 0, en = 0;
        void reserve()
        {
            v.resize( 1024 );
            e.resize( 1024 );
        }
    };

    struct NewEdge
    {
        uint32_t k; // 30-bit field in the reference
        bool     two, closed;
        bool     valid() const { return !( two && closed ); }
    };

    enum Flags : uint32_t
    {
        kFlagVertexCap = 1,
        kFlagEdgeCap   = 2,
        kFlagNewEdge   = 4,
        kFlagBisector  = 8,
        kFlagStack     = 16,
    };

    // Work counters (for profiling the restated algorithm; no effect on results).
    enum Counter
    {
        cEdgeTasks, cEdgeSearched, cEdgeSecurity, cEdgeLeaves, cEdgeCandidates, cEdgeSolves, cEdgeFound, cEdgeCellsChanged,
        cVertexSearched, cVertexLeaves, cVertexInvalid, cVertexCellsChanged, cBisSearched, cBisLeaves, cBisCandidates,
        cBisFound, cBisCellsChanged, cEdgeCellsFound, cEdgeCandInBall, cEdgeFoundOutsideBall, cEdgeSolvesInBall, cCounterCount
    };

    struct Context
    {
        std::vector<uint64_t> counters = std::vector<uint64_t>( cCounterCount, 0 );
        void count( Counter c, uint64_t v = 1 )
        {
#pragma omp atomic
            counters[ c ] += v;
        }
        uint32_t             n        = 0;
        uint32_t             k        = kK; // neighbours per kNN step (the AlgorithmGPU<K> argument)
        uint32_t             knnSteps = 1;  // knnValidationStep (algorithm.inl:1535)
        std::vector<D4>      sites; // n + 6, Morton order then the 6 artificial sites
        std::vector<uint8_t> status;
        // LBVH (lbvh.cuh:9-62)
        std::vector<uint32_t> indices;
        std::vector<uint64_t> morton;
        std::vector<int32_t>  parent, left, right;
        std::vector<float>    aabb; // 8 floats per node: min xyz 0, max xyz 0
        std::vector<uint32_t> sizes;
        // kNN and cells
        std::vector<uint32_t> knn;
        std::vector<float>    knownRadii;
        std::vector<Cell>     cells;
        std::vector<uint32_t> flags; // per cell
        // outputs
        std::vector<double>   outVertices, outClosed;
        std::vector<uint32_t> outVerticesId, outClosedId, topoQuad, topoTri, topoBi;
        // flattened stores for inspection
        std::vector<uint32_t> vertexNb, edgeNb, flatVertices, flatEdges;
        // per searched edge of the edge passes: cell, k, l, leaves reached, candidates, round
        std::vector<uint32_t> edgeSearchLog;
        double                rmax = 0.0;
        int                   round = 0;
        uint32_t              flagsAll = 0;
        // contributing-nearest study (app/benchmarks/benchmark_contributing_nearest.cu): per
        // cell, knnSteps * k rank labels of the kNN cell construction
        bool                  profile = false;
        std::vector<uint8_t>  contribution, reached;

        Box box( uint32_t node ) const
        {
            const float * p = &aabb[ std::size_t( node ) * 8 ];
            return { { p[ 0 ], p[ 1 ], p[ 2 ] }, { p[ 4 ], p[ 5 ], p[ 6 ] } };
        }
    };

    // ------------------------------------------------------------------------------------
    // Artificial bounding sites and the LBVH (algorithm.cpp:5-25, algorithm.inl:1437-1464,
    // lbvh.cu:11-323)
    // ------------------------------------------------------------------------------------

    // utils.cpp:8-13 (ldexp variant of the PCG hash)
    double pcgLdexp( uint32_t v )
    {
        const uint32_t state = v * 747796405u + 2891336453u;
        const uint32_t word  = ( ( state >> ( ( state >> 28u ) + 4u ) ) ^ state ) * 277803737u;
        return std::ldexp( double( ( word >> 22u ) ^ word ), -32 );
    }

    void joggle( double * s, uint64_t count, double range )
    {
        const double randA = 2.0 * range;
        const double randB = -range;
        for ( uint64_t i = 0; i < count; i++ )
            for ( uint32_t c = 0; c < 4; c++ )
                s[ i * 4 + c ] += pcgLdexp( uint32_t( i * 4 + c ) ) * randA + randB;
    }

    // lbvh.cu:11-48
    uint32_t spread10( uint32_t x )
    {
        x = ( x | ( x << 16 ) ) & 0x030000FF;
        x = ( x | ( x << 8 ) ) & 0x0300F00F;
        x = ( x | ( x << 4 ) ) & 0x030C30C3;
        x = ( x | ( x << 2 ) ) & 0x09249249;
        return x;
    }
    uint64_t morton64( uint32_t x, uint32_t y, uint32_t z )
    {
        const uint64_t lo = spread10( x & 1023u ) | ( spread10( y & 1023u ) << 1 ) | ( spread10( z & 1023u ) << 2 );
        const uint64_t hi = spread10( x >> 10u ) | ( spread10( y >> 10u ) << 1 ) | ( spread10( z >> 10u ) << 2 );
        return ( hi << 30 ) | lo;
    }
    uint32_t quantize( float v )
    {
        // float -> unsigned conversion of the device (round toward zero, saturating)
        const float s = v * float( ( 1u << 20 ) - 1 );
        if ( !( s > 0.f ) )
            return 0;
        if ( s >= 4294967296.f )
            return 0xffffffffu;
        return uint32_t( s );
    }

    // lbvh.cu:144-155
    int delta( const std::vector<uint64_t> & codes, int i, int j, uint32_t n )
    {
        if ( j < 0 || j >= int( n ) )
            return -1;
        const uint64_t a = codes[ i ], b = codes[ j ];
        if ( a != b )
            return __builtin_clzll( a ^ b );
        const uint64_t x = uint64_t( int64_t( i ^ j ) );
        return ( x ? __builtin_clzll( x ) : 64 ) + 64;
    }

    void buildLbvh( Context & ctx, const std::vector<D4> & input, const double bboxMin[ 3 ], const double bboxMax[ 3 ] )
    {
        const uint32_t n = ctx.n;
        const float    sceneMin[ 3 ] = { float( bboxMin[ 0 ] ), float( bboxMin[ 1 ] ), float( bboxMin[ 2 ] ) };
        const float    sceneMax[ 3 ] = { float( bboxMax[ 0 ] ), float( bboxMax[ 1 ] ), float( bboxMax[ 2 ] ) };
        // lbvh.cu:287-288 (host float arithmetic)
        float scale[ 3 ];
        for ( int c = 0; c < 3; c++ )
            scale[ c ] = 1.f / ( sceneMax[ c ] - sceneMin[ c ] );

        // getMortonCodes (lbvh.cu:50-67)
        std::vector<uint64_t> codes( n );
        std::vector<uint32_t> idx( n );
        for ( uint32_t i = 0; i < n; i++ )
        {
            const F4 s = toFloat( input[ i ] );
            const float cx = ( s.x - sceneMin[ 0 ] ) * scale[ 0 ];
            const float cy = ( s.y - sceneMin[ 1 ] ) * scale[ 1 ];
            const float cz = ( s.z - sceneMin[ 2 ] ) * scale[ 2 ];
            codes[ i ]     = morton64( quantize( cx ), quantize( cy ), quantize( cz ) );
            idx[ i ]       = i;
        }
        // thrust::sort_by_key (lbvh.cu:294-295): stable radix sort by key.
        std::stable_sort( idx.begin(), idx.end(), [ & ]( uint32_t a, uint32_t b ) { return codes[ a ] < codes[ b ]; } );
        ctx.indices = idx;
        ctx.morton.resize( n );
        for ( uint32_t i = 0; i < n; i++ )
            ctx.morton[ i ] = codes[ idx[ i ] ];

        const uint32_t nodes = 2 * n - 1;
        ctx.parent.assign( nodes, 0 );
        ctx.left.assign( nodes, 0 );
        ctx.right.assign( nodes, 0 );
        ctx.aabb.assign( std::size_t( nodes ) * 8, 0.f );
        ctx.sizes.assign( nodes, 0 );

        // setLeaves (lbvh.cu:88-114): leaves are nodes n-1 .. 2n-2.
        ctx.sites.assign( n + 6, D4 {} );
        for ( uint32_t b = 0; b < n; b++ )
        {
            const uint32_t node = b + n - 1;
            ctx.left[ node ]    = int32_t( b );
            ctx.right[ node ]   = int32_t( b ) + 1;
            const D4 s          = input[ idx[ b ] ];
            float *  box        = &ctx.aabb[ std::size_t( node ) * 8 ];
            box[ 0 ]            = float( s.x - s.w );
            box[ 1 ]            = float( s.y - s.w );
            box[ 2 ]            = float( s.z - s.w );
            box[ 4 ]            = float( s.x + s.w );
            box[ 5 ]            = float( s.y + s.w );
            box[ 6 ]            = float( s.z + s.w );
            ctx.sites[ b ]      = s;
        }

        // construct (lbvh.cu:163-223), Karras 2012.
        const auto & mc = ctx.morton;
        for ( int i = 0; i + 1 < int( n ); i++ )
        {
            const int dr = delta( mc, i, i + 1, n ), dl = delta( mc, i, i - 1, n );
            const int d  = ( dr - dl > 0 ) - ( dr - dl < 0 );
            const int deltaMin = delta( mc, i, i - d, n );
            int       lmax     = 2;
            while ( delta( mc, i, i + lmax * d, n ) > deltaMin )
                lmax <<= 1;
            int l = 0;
            for ( int t = lmax >> 1; t >= 1; t >>= 1 )
                if ( delta( mc, i, i + ( l + t ) * d, n ) > deltaMin )
                    l += t;
            const int j         = i + l * d;
            const int deltaNode = delta( mc, i, j, n );
            int       s = 0, k = 2, t;
            do
            {
                t = ( l + k - 1 ) / k;
                k <<= 1;
                if ( delta( mc, i, i + ( s + t ) * d, n ) > deltaNode )
                    s += t;
            } while ( t > 1 );
            const int gamma = i + s * d + std::min( d, 0 );
            int       lc = gamma, rc = gamma + 1;
            if ( std::min( i, j ) == gamma )
                lc += int( n ) - 1;
            if ( std::max( i, j ) == gamma + 1 )
                rc += int( n ) - 1;
            ctx.left[ i ]    = lc;
            ctx.right[ i ]   = rc;
            ctx.parent[ lc ] = i;
            ctx.parent[ rc ] = i;
        }
        ctx.parent[ 0 ] = -1;

        // refit (lbvh.cu:225-272): union of child boxes and subtree sizes, bottom-up.
        for ( uint32_t b = 0; b < n; b++ )
            ctx.sizes[ b + n - 1 ] = 1;
        if ( n > 1 )
        {
            std::vector<int32_t> order;
            order.reserve( n - 1 );
            std::vector<int32_t> stack { 0 };
            while ( !stack.empty() )
            {
                const int32_t node = stack.back();
                stack.pop_back();
                order.push_back( node );
                if ( ctx.left[ node ] < int32_t( n ) - 1 )
                    stack.push_back( ctx.left[ node ] );
                if ( ctx.right[ node ] < int32_t( n ) - 1 )
                    stack.push_back( ctx.right[ node ] );
            }
            for ( auto it = order.rbegin(); it != order.rend(); ++it )
            {
                const int32_t node = *it;
                const float * a    = &ctx.aabb[ std::size_t( ctx.left[ node ] ) * 8 ];
                const float * b    = &ctx.aabb[ std::size_t( ctx.right[ node ] ) * 8 ];
                float *       o    = &ctx.aabb[ std::size_t( node ) * 8 ];
                for ( int c = 0; c < 3; c++ )
                {
                    float lo = FLT_MAX, hi = -FLT_MAX;
                    lo       = fminf_( a[ c ], lo );
                    hi       = fmaxf_( a[ c ], hi );
                    lo       = fminf_( a[ 4 + c ], lo );
                    hi       = fmaxf_( a[ 4 + c ], hi );
                    lo       = fminf_( b[ c ], lo );
                    hi       = fmaxf_( b[ c ], hi );
                    lo       = fminf_( b[ 4 + c ], lo );
                    hi       = fmaxf_( b[ 4 + c ], hi );
                    o[ c ]     = lo;
                    o[ 4 + c ] = hi;
                }
                o[ 3 ]            = 0.f;
                o[ 7 ]            = 0.f;
                ctx.sizes[ node ] = ctx.sizes[ ctx.left[ node ] ] + ctx.sizes[ ctx.right[ node ] ];
            }
        }
    }

    // ------------------------------------------------------------------------------------
    // kNN search (lbvh.inl:8-105, heap.hpp:11-43, algorithm.inl:32-99)
    // ------------------------------------------------------------------------------------
    void heapify( uint32_t * keys, float * values, uint32_t node, uint32_t size )
    {
        uint32_t j = node;
        while ( true )
        {
            const uint32_t left = 2 * j + 1, right = 2 * j + 2;
            uint32_t       largest = j;
            if ( left < size && values[ left ] > values[ largest ] )
                largest = left;
            if ( right < size && values[ right ] > values[ largest ] )
                largest = right;
            if ( largest == j )
                return;
            std::swap( values[ j ], values[ largest ] );
            std::swap( keys[ j ], keys[ largest ] );
            j = largest;
        }
    }
    void heapsort( uint32_t * keys, float * values, int size )
    {
        while ( size )
        {
            std::swap( values[ 0 ], values[ size - 1 ] );
            std::swap( keys[ 0 ], keys[ size - 1 ] );
            heapify( keys, values, 0, uint32_t( --size ) );
        }
    }

    // getKnns<K> (algorithm.inl:32-99): step 0 takes the K nearest and flags buried sites;
    // a later step the next K beyond the previous step's last neighbour, or none once the
    // previous list ran short.
    void knnSite( Context & ctx, uint32_t id, uint32_t step )
    {
        const uint32_t n  = ctx.n;
        const uint32_t kk = ctx.k;
        const F4       si = toFloat( ctx.sites[ id ] );
        float          startingDistance = -FLT_MAX;
        if ( step != 0 )
        {
            const uint32_t last = ctx.knn[ std::size_t( id ) * kk + kk - 1 ];
            if ( last >= n )
            {
                for ( uint32_t k = 0; k < kk; k++ )
                    ctx.knn[ std::size_t( id ) * kk + k ] = kNone;
                return;
            }
            startingDistance = sphereDistance( toFloat( ctx.sites[ last ] ), si );
        }
        uint32_t keys[ kK ];
        float    dist[ kK ];
        for ( uint32_t k = 0; k < kk; k++ )
        {
            keys[ k ] = kNone;
            dist[ k ] = FLT_MAX;
        }

        struct Entry { uint32_t node; float d; };
        Entry    stack[ 64 ];
        int      sp   = 0;
        uint32_t node = 0;
        while ( true )
        {
            while ( true )
            {
                if ( node >= n - 1 )
                    break;
                const uint32_t l = uint32_t( ctx.left[ node ] ), r = uint32_t( ctx.right[ node ] );
                const Box      lb = ctx.box( l ), rb = ctx.box( r );
                const float    dL = lb.distance( si ), dLMax = lb.farthestDistance( si );
                const float    dR = rb.distance( si ), dRMax = rb.farthestDistance( si );
                const bool     leftClosest = dL < dR;
                const float    minFar = leftClosest ? dR : dL, maxFar = leftClosest ? dRMax : dLMax;
                const uint32_t farChild = leftClosest ? r : l;
                const float    minClose = leftClosest ? dL : dR, maxClose = leftClosest ? dLMax : dRMax;
                const uint32_t closeChild = leftClosest ? l : r;
                const bool     exploreFar   = minFar < dist[ 0 ] && maxFar > startingDistance;
                const bool     exploreClose = minClose < dist[ 0 ] && maxClose > startingDistance;
                if ( !exploreFar && !exploreClose )
                    break;
                node = exploreClose ? closeChild : farChild;
                if ( exploreClose && exploreFar )
                {
                    if ( sp >= 64 )
                        ctx.flagsAll |= kFlagStack;
                    else
                        stack[ sp++ ] = { farChild, minFar };
                }
            }
            if ( node >= n - 1 && node < 2 * n - 1 )
            {
                const uint32_t j = node - ( n - 1 );
                const float    d = sphereDistance( si, toFloat( ctx.sites[ j ] ) );
                if ( id != j && d < dist[ 0 ] && d > startingDistance )
                {
                    dist[ 0 ] = d;
                    keys[ 0 ] = j;
                    heapify( keys, dist, 0, kk );
                }
            }
            bool more = false;
            while ( sp > 0 )
            {
                --sp;
                if ( stack[ sp ].d > dist[ 0 ] )
                    continue;
                node = stack[ sp ].node;
                more = true;
                break;
            }
            if ( !more )
                break;
        }
        heapsort( keys, dist, int( kk ) );
        for ( uint32_t k = 0; k < kk; k++ )
            ctx.knn[ std::size_t( id ) * kk + k ] = keys[ k ];
        if ( step != 0 )
            return;

        // buried test (algorithm.inl:85-98); `si` is the float copy of the site.
        if ( keys[ 0 ] == kNone )
            return;
        const D4     closest = ctx.sites[ keys[ 0 ] ];
        const double ri = si.w, rj = closest.w;
        const double bigger = dmax( ri, rj ), smaller = dmin( ri, rj );
        const D3     d { double( si.x ) - closest.x, double( si.y ) - closest.y, double( si.z ) - closest.z };
        if ( lessThan( length( d ), bigger - smaller ) )
        {
            if ( lessThan( rj, ri ) )
                return;
            ctx.status[ id ] = kBuried;
        }
    }

    // ------------------------------------------------------------------------------------
    // Cell update (topology_update.inl:49-593), one warp of 32 lanes simulated in order
    // ------------------------------------------------------------------------------------
    inline uint32_t highestLane( uint32_t mask ) { return 31u - uint32_t( __builtin_clz( mask ) ); }

    struct CellWork
    {
        const Context & ctx;
        uint32_t        i;
        D4              si;
        Cell &          c;
        uint32_t &      flags;

        D4 vertexPosition( const Vertex & v ) const
        {
            D4 x[ 2 ] = {};
            quadrisector( si, ctx.sites[ v.j ], ctx.sites[ v.k ], ctx.sites[ v.l ], x[ 0 ], x[ 1 ] );
            return x[ v.type & 1 ];
        }

        // topology_update.inl:578-592: a sphere is valid if no site of the cell's edges
        // (other than skip1 / skip2) intersects it.
        bool predicate( const D4 & sphere, uint32_t skip1, uint32_t skip2 ) const
        {
            if ( c.en > 255 )
                flags |= kFlagEdgeCap; // the reference's 8-bit loop counter never ends here
            bool valid = true;
            for ( uint32_t e = 0; e < c.en; e++ )
            {
                const Edge & edge = c.e[ e ];
                if ( edge.j != skip1 && edge.j != skip2 )
                    valid &= !intersect( ctx.sites[ edge.j ], sphere );
                if ( edge.k != skip1 && edge.k != skip2 )
                    valid &= !intersect( ctx.sites[ edge.k ], sphere );
            }
            return valid;
        }

        bool known( uint32_t j ) const
        {
            for ( uint32_t e = 0; e < c.en; e++ )
                if ( c.e[ e ].j == j || c.e[ e ].k == j )
                    return true;
            return false;
        }

        void checkCapacity()
        {
            if ( c.vn >= kMaxVertices )
                flags |= kFlagVertexCap;
            if ( c.en >= kMaxEdges )
                flags |= kFlagEdgeCap;
            if ( c.vn > 900 || c.en > 900 )
            {
                // keep the simulation in bounds; the reference corrupts memory long before
                c.vn = std::min( c.vn, 900u );
                c.en = std::min( c.en, 900u );
            }
        }

        bool update( uint32_t j, const D4 & sj )
        {
            if ( c.vn == 0 && c.en == 0 )
                return false;

            const double ri = si.w, rj = sj.w;
            const double bigger = dmax( ri, rj ), smaller = dmin( ri, rj );
            if ( lessThan( length( sub( xyz( si ), xyz( sj ) ) ), bigger - smaller ) )
            {
                if ( lessThan( rj, ri ) )
                    return false;
                c.vn = 0;
                c.en = 0;
                return false;
            }

            NewEdge ne[ kMaxNewEdges ];
            for ( auto & x : ne )
                x = { 0x0fffffffu, true, true };
            uint32_t neCount = 0;
            auto     push    = [ & ]( uint32_t k, bool two, bool closed ) {
                if ( neCount < kMaxNewEdges )
                    ne[ neCount ] = { k & 0x3fffffffu, two, closed };
                else
                    flags |= kFlagNewEdge;
                neCount++;
            };

            const uint32_t baseV = c.vn, baseVSteps = baseV / 32 + 1;
            const uint32_t baseE = c.en, baseESteps = baseE / 32 + 1;

            // Vertices inside sj are invalidated; their edges lose one vertex (:96-154).
            for ( uint32_t vs = 0; vs < baseVSteps; vs++ )
            {
                uint32_t invalid = 0;
                for ( uint32_t lane = 0; lane < 32; lane++ )
                {
                    const uint32_t id = lane + 32 * vs;
                    if ( id < baseV && intersect( vertexPosition( c.v[ id ] ), sj ) )
                    {
                        c.v[ id ].status = 0xff;
                        invalid |= 1u << lane;
                    }
                }
                while ( invalid )
                {
                    const uint32_t lane = highestLane( invalid );
                    invalid &= ~( 1u << lane );
                    const Vertex vtx = c.v[ 32 * vs + lane ];
                    for ( uint32_t es = 0; es < baseESteps; es++ )
                        for ( uint32_t l2 = 0; l2 < 32; l2++ )
                        {
                            const uint8_t id = uint8_t( l2 + 32 * es );
                            if ( id < c.en )
                            {
                                Edge &     edge = c.e[ id ];
                                const bool m1   = edge.j == vtx.j && edge.k == vtx.k;
                                const bool m2   = edge.j == vtx.j && edge.k == vtx.l;
                                const bool m3   = edge.j == vtx.k && edge.k == vtx.l;
                                if ( m1 || m2 || m3 )
                                    edge.vertexNb--;
                            }
                        }
                }
            }

            // New vertices on every edge (:156-323).
            uint8_t closedEll[ 32 ] = {};
            for ( uint32_t es = 0; es < baseESteps; es++ )
            {
                uint32_t k[ 32 ], l[ 32 ], e[ 32 ];
                uint8_t  mask[ 32 ], valid[ 32 ];
                bool     has[ 32 ];
                D4       q[ 32 ][ 2 ];
                for ( uint32_t lane = 0; lane < 32; lane++ )
                {
                    e[ lane ]         = lane + 32 * es;
                    const Edge edge   = c.e[ e[ lane ] ];
                    has[ lane ]       = e[ lane ] < baseE;
                    k[ lane ]         = edge.j;
                    l[ lane ]         = edge.k;
                    mask[ lane ]      = 0;
                    q[ lane ][ 0 ]    = D4 {};
                    q[ lane ][ 1 ]    = D4 {};
                    D4 sk {}, sl {};
                    if ( has[ lane ] )
                    {
                        sk           = ctx.sites[ k[ lane ] ];
                        sl           = ctx.sites[ l[ lane ] ];
                        mask[ lane ] = quadrisector( si, sj, sk, sl, q[ lane ][ 0 ], q[ lane ][ 1 ] );
                        has[ lane ]  = has[ lane ] && mask[ lane ] != 0;
                    }
                    if ( e[ lane ] < baseE && mask[ lane ] == 0 && edge.vertexNb == kNone )
                    {
                        trisectorVertex( si, sk, sl, q[ lane ][ 0 ], q[ lane ][ 0 ] );
                        if ( intersect( q[ lane ][ 0 ], sj ) )
                            c.e[ e[ lane ] ].vertexNb = 0;
                    }
                    valid[ lane ] = mask[ lane ];
                }
                for ( uint32_t lane = 0; lane < 32; lane++ )
                {
                    if ( !has[ lane ] )
                        continue;
                    uint8_t m = mask[ lane ];
                    while ( m )
                    {
                        const uint32_t nv = uint32_t( __builtin_ctz( m ) );
                        m &= uint8_t( ~( 1u << nv ) );
                        if ( !predicate( q[ lane ][ nv ], k[ lane ], l[ lane ] ) )
                            valid[ lane ] &= uint8_t( ~( 1u << nv ) );
                    }
                }
                uint32_t newCount[ 32 ], offset[ 32 ], total = 0;
                for ( uint32_t lane = 0; lane < 32; lane++ )
                {
                    newCount[ lane ] = uint32_t( __builtin_popcount( valid[ lane ] ) );
                    has[ lane ]      = has[ lane ] && newCount[ lane ] > 0;
                    if ( has[ lane ] )
                    {
                        Edge & edge = c.e[ e[ lane ] ];
                        if ( edge.vertexNb == kNone )
                            edge.vertexNb = 0;
                        edge.vertexNb += newCount[ lane ];
                    }
                    offset[ lane ] = total;
                    total += newCount[ lane ];
                }
                for ( uint32_t lane = 0; lane < 32; lane++ )
                {
                    uint32_t jj = j, kk = k[ lane ], ll = l[ lane ];
                    if ( jj > ll )
                        std::swap( jj, ll );
                    if ( jj > kk )
                        std::swap( jj, kk );
                    if ( kk > ll )
                        std::swap( kk, ll );
                    uint32_t m = valid[ lane ], w = c.vn + offset[ lane ];
                    while ( m )
                    {
                        const uint32_t nv = uint32_t( __builtin_ctz( m ) );
                        m &= ~( 1u << nv );
                        if ( w < c.v.size() )
                            c.v[ w ] = { jj, kk, ll, uint8_t( nv ), 0 };
                        w++;
                    }
                }
                uint32_t withVertices = 0;
                for ( uint32_t lane = 0; lane < 32; lane++ )
                    if ( valid[ lane ] )
                        withVertices |= 1u << lane;
                while ( withVertices )
                {
                    const uint32_t lane = highestLane( withVertices );
                    withVertices &= ~( 1u << lane );
                    uint32_t m = valid[ lane ];
                    while ( m )
                    {
                        const uint32_t nv = uint32_t( __builtin_ctz( m ) );
                        m &= ~( 1u << nv );
                        push( k[ lane ], newCount[ lane ] == 2, false );
                        push( l[ lane ], newCount[ lane ] == 2, false );
                    }
                }
                c.vn += total;
                for ( uint32_t lane = 0; lane < 32; lane++ )
                    closedEll[ lane ] = uint8_t( closedEll[ lane ] | ( uint32_t( e[ lane ] < baseE && mask[ lane ] == 0 ) << es ) );
                checkCapacity();
            }

            // Closed elliptic trisectors (:325-433).
            bool anyClosed = false;
            for ( uint32_t lane = 0; lane < 32; lane++ )
                anyClosed = anyClosed || closedEll[ lane ] != 0;
            if ( anyClosed )
            {
                for ( uint32_t es = 0; es < baseESteps; es++ )
                {
                    bool can[ 32 ], anyCan = false;
                    for ( uint32_t lane = 0; lane < 32; lane++ )
                    {
                        can[ lane ] = ( closedEll[ lane ] >> es ) & 1;
                        anyCan      = anyCan || can[ lane ];
                    }
                    if ( !anyCan )
                        continue;
                    uint32_t ids[ 32 ][ 2 ];
                    D4       sites[ 32 ][ 2 ];
                    for ( uint32_t lane = 0; lane < 32; lane++ )
                    {
                        const uint32_t e    = lane + 32 * es;
                        const Edge     edge = c.e[ e ];
                        ids[ lane ][ 0 ]    = edge.j;
                        ids[ lane ][ 1 ]    = edge.k;
                        sites[ lane ][ 0 ]  = D4 {};
                        sites[ lane ][ 1 ]  = D4 {};
                        if ( e < baseE )
                        {
                            sites[ lane ][ 0 ] = ctx.sites[ edge.j ];
                            sites[ lane ][ 1 ] = ctx.sites[ edge.k ];
                        }
                    }
                    for ( uint32_t s = 0; s < 2; s++ )
                    {
                        bool cur[ 32 ];
                        for ( uint32_t lane = 0; lane < 32; lane++ )
                        {
                            cur[ lane ] = can[ lane ];
                            if ( !cur[ lane ] )
                                continue;
                            bool share = false;
                            for ( uint32_t f = 0; f < kMaxNewEdges && !share; f++ )
                                share = ne[ f ].k == ids[ lane ][ s ];
                            cur[ lane ] = !share;
                        }
                        D4 vt[ 32 ][ 2 ];
                        for ( uint32_t lane = 0; lane < 32; lane++ )
                        {
                            vt[ lane ][ 0 ] = D4 {};
                            vt[ lane ][ 1 ] = D4 {};
                            uint8_t count   = 0;
                            if ( cur[ lane ] )
                                count = trisectorVertex( si, sj, sites[ lane ][ s ], vt[ lane ][ 0 ], vt[ lane ][ 1 ] );
                            cur[ lane ] = cur[ lane ] && count == 2;
                        }
                        for ( int lane = 31; lane >= 0; lane-- )
                        {
                            if ( !cur[ lane ] )
                                continue;
                            if ( !predicate( vt[ lane ][ 0 ], ids[ lane ][ s ], i ) )
                                continue;
                            push( ids[ lane ][ s ], false, true );
                        }
                    }
                }
            }

            // Unique new edges, ordered by site id (:435-515). Entries with the same id only
            // differ in `two`, which the written edge does not use, so any ordering by id
            // gives the same edges as the reference's warp merge sort.
            std::stable_sort( ne, ne + kMaxNewEdges, []( const NewEdge & a, const NewEdge & b ) { return a.k < b.k; } );
            uint32_t written = 0;
            int      prevLast = -1;
            for ( uint32_t f = 0; f < kMaxNewEdges; f++ )
            {
                const bool last = ( f == kMaxNewEdges - 1 || ne[ f + 1 ].k != ne[ f ].k ) && ne[ f ].valid();
                if ( !last )
                    continue;
                const uint32_t other = ne[ f ].k;
                const uint32_t w     = c.en + written;
                if ( w < c.e.size() )
                    c.e[ w ] = { std::min( j, other ), std::max( j, other ),
                                 ne[ f ].closed ? kNone : uint32_t( int( f ) - prevLast ), 0, 0 };
                written++;
                prevLast = int( f );
            }
            c.en += written;
            checkCapacity();

            // Stable compaction of invalidated vertices and emptied edges (:520-542).
            if ( c.vn > 0 )
            {
                uint32_t w = 0;
                for ( uint32_t id = 0; id < c.vn; id++ )
                    if ( !( c.v[ id ].status == 0xff && id < baseV ) )
                        c.v[ w++ ] = c.v[ id ];
                c.vn = w;
            }
            {
                uint32_t w = 0;
                for ( uint32_t id = 0; id < c.en; id++ )
                    if ( !( c.e[ id ].vertexNb == 0 && id < baseE ) )
                        c.e[ w++ ] = c.e[ id ];
                c.en = w;
            }
            return written != 0;
        }

        // topology_update.inl:595-653
        double radius() const
        {
            double maxRadius = 0.0;
            for ( uint32_t v = 0; v < c.vn; v++ )
                maxRadius = dmax( maxRadius, vertexPosition( c.v[ v ] ).w );
            for ( uint32_t e = 0; e < c.en; e++ )
            {
                D4 x[ 2 ] = {};
                if ( trisectorVertex( si, ctx.sites[ c.e[ e ].j ], ctx.sites[ c.e[ e ].k ], x[ 0 ], x[ 1 ] ) == 2 )
                    maxRadius = dmax( maxRadius, dmax( x[ 0 ].w, x[ 1 ].w ) );
            }
            return maxRadius;
        }
    };

    // ------------------------------------------------------------------------------------
    // Stages (algorithm.inl:101-1233)
    // ------------------------------------------------------------------------------------

    // Initial cell: 8 vertices and 12 edges on the artificial sites (algorithm.inl:1466-1505,
    // topology_update.inl:5-47).
    void initialCell( Context & ctx, Cell & c )
    {
        const uint32_t n = ctx.n;
        static const uint32_t vt[ 8 ][ 3 ] = { { 0, 2, 4 }, { 0, 2, 5 }, { 0, 3, 4 }, { 0, 3, 5 },
                                               { 1, 2, 4 }, { 1, 2, 5 }, { 1, 3, 4 }, { 1, 3, 5 } };
        static const uint32_t et[ 12 ][ 2 ] = { { 0, 2 }, { 2, 4 }, { 1, 2 }, { 2, 5 }, { 1, 4 }, { 1, 5 },
                                                { 0, 5 }, { 0, 4 }, { 1, 3 }, { 3, 5 }, { 0, 3 }, { 3, 4 } };
        c.reserve();
        for ( uint32_t v = 0; v < 8; v++ )
            c.v[ v ] = { n + vt[ v ][ 0 ], n + vt[ v ][ 1 ], n + vt[ v ][ 2 ], 0, 0 };
        for ( uint32_t e = 0; e < 12; e++ )
            c.e[ e ] = { n + et[ e ][ 0 ], n + et[ e ][ 1 ], 2, 0, 0 };
        c.vn = 8;
        c.en = 12;
    }

    // getCells (algorithm.inl:101-206)
    void cellFromKnn( Context & ctx, uint32_t i )
    {
        if ( ctx.status[ i ] == kFullyValidated || ctx.status[ i ] == kBuried )
            return;
        CellWork w { ctx, i, ctx.sites[ i ], ctx.cells[ i ], ctx.flags[ i ] };
        double   knownRadius = -DBL_MAX;
        for ( uint32_t nId = 0; nId < ctx.k; nId++ )
        {
            const uint32_t j = ctx.knn[ std::size_t( i ) * ctx.k + nId ];
            if ( j == kNone )
                break;
            if ( ctx.status[ j ] == kBuried )
                continue;
            const D4 sj = ctx.sites[ j ];
            w.update( j, sj );
            knownRadius = dmax( knownRadius, sphereDistance( w.si, sj ) );
        }
        const double maxRadius = w.radius();
        if ( greaterThan( knownRadius, 2.0 * maxRadius ) )
            ctx.status[ i ] = kFullyValidated;
        ctx.knownRadii[ i ] = float( knownRadius );
    }

    // getCellsContribution (app/benchmarks/benchmark_contributing_nearest.cu:10-129): the kNN
    // cell construction of one step, labelling every rank with whether its neighbour changed the
    // cell and whether the security-radius certificate held after it; the known radius starts
    // over at every step, and a certified cell stops there.
    void cellContribution( Context & ctx, uint32_t i, uint32_t step )
    {
        if ( ctx.status[ i ] == kFullyValidated || ctx.status[ i ] == kBuried )
            return;
        CellWork          w { ctx, i, ctx.sites[ i ], ctx.cells[ i ], ctx.flags[ i ] };
        double            knownRadius = -DBL_MAX;
        const std::size_t row         = std::size_t( i ) * ctx.knnSteps * ctx.k + std::size_t( ctx.k ) * step;
        for ( uint32_t nId = 0; nId < ctx.k; nId++ )
        {
            const uint32_t j = ctx.knn[ std::size_t( i ) * ctx.k + nId ];
            if ( j == kNone )
                break;
            if ( ctx.status[ j ] == kBuried )
                continue;
            const D4   sj          = ctx.sites[ j ];
            const bool contributed = w.update( j, sj );
            knownRadius            = dmax( knownRadius, sphereDistance( w.si, sj ) );
            if ( contributed )
                ctx.contribution[ row + nId ] = 1;
            const bool over = greaterThan( knownRadius, 2.0 * w.radius() );
            if ( over )
            {
                ctx.reached[ row + nId ] = 1;
                ctx.status[ i ]          = kFullyValidated;
                break;
            }
        }
        ctx.knownRadii[ i ] = float( knownRadius );
    }

    // globalVertexValidation (algorithm.inl:208-476)
    void vertexValidation( Context & ctx, uint32_t i )
    {
        if ( ctx.status[ i ] == kFullyValidated || ctx.status[ i ] == kBuried )
            return;
        const uint32_t n = ctx.n;
        Cell &         c = ctx.cells[ i ];
        CellWork       w { ctx, i, ctx.sites[ i ], c, ctx.flags[ i ] };
        const float    knownRadius = ctx.knownRadii[ i ];

        uint32_t vs = 0, restarts = 0;
        while ( vs < c.vn / 32 + 1 && restarts < 100 )
        {
            const uint32_t step = vs++;
            uint32_t       neighbor[ 32 ];
            D4             current[ 32 ];
            bool           needSearch[ 32 ];
            for ( uint32_t lane = 0; lane < 32; lane++ )
            {
                const uint32_t vid = step * 32 + lane;
                neighbor[ lane ]   = kNone;
                needSearch[ lane ] = vid < c.vn;
                current[ lane ]    = D4 {};
                if ( needSearch[ lane ] )
                    needSearch[ lane ] = c.v[ vid ].status == 0;
                if ( needSearch[ lane ] )
                {
                    current[ lane ] = w.vertexPosition( c.v[ vid ] );
                    if ( 2.0 * current[ lane ].w < double( knownRadius ) )
                    {
                        needSearch[ lane ] = false;
                        c.v[ vid ].status  = 1;
                    }
                }
                if ( !needSearch[ lane ] )
                    continue;

                // nearest admissible site to the vertex sphere (per-lane BVH walk)
                ctx.count( cVertexSearched );
                const Vertex vtx = c.v[ vid ];
                const F4     fc  = toFloat( current[ lane ] );
                struct Entry { uint32_t node; float d; };
                Entry    stack[ 64 ];
                int      sp = 0;
                uint32_t node = 0;
                float    best = FLT_MAX;
                while ( true )
                {
                    while ( true )
                    {
                        if ( node >= n - 1 )
                            break;
                        const uint32_t l = uint32_t( ctx.left[ node ] ), r = uint32_t( ctx.right[ node ] );
                        const float    dL = ctx.box( l ).distance( fc ), dR = ctx.box( r ).distance( fc );
                        const bool     leftClosest = dL < dR;
                        const float    minFar = leftClosest ? dR : dL, minClose = leftClosest ? dL : dR;
                        const uint32_t farChild = leftClosest ? r : l, closeChild = leftClosest ? l : r;
                        const bool     exploreFar = minFar < best, exploreClose = minClose < best;
                        if ( !exploreFar && !exploreClose )
                            break;
                        node = exploreClose ? closeChild : farChild;
                        if ( exploreClose && exploreFar )
                        {
                            if ( sp >= 64 )
                                ctx.flags[ i ] |= kFlagStack;
                            else
                                stack[ sp++ ] = { farChild, minFar };
                        }
                    }
                    if ( node >= n - 1 && node < 2 * n - 1 )
                    {
                        ctx.count( cVertexLeaves );
                        const uint32_t j = node - ( n - 1 );
                        if ( j != i && j != vtx.j && j != vtx.k && j != vtx.l && ctx.status[ j ] != kBuried
                             && !w.known( j ) )
                        {
                            const float d = sphereDistance( toFloat( ctx.sites[ j ] ), fc );
                            if ( d < best )
                            {
                                best             = d;
                                neighbor[ lane ] = j;
                            }
                        }
                    }
                    bool more = false;
                    while ( sp > 0 )
                    {
                        --sp;
                        if ( stack[ sp ].d > best )
                            continue;
                        node = stack[ sp ].node;
                        more = true;
                        break;
                    }
                    if ( !more )
                        break;
                }
            }
            uint32_t changed = 0;
            for ( uint32_t lane = 0; lane < 32; lane++ )
            {
                const bool isValid = neighbor[ lane ] == kNone || !intersect( current[ lane ], ctx.sites[ neighbor[ lane ] ] );
                if ( needSearch[ lane ] )
                    c.v[ step * 32 + lane ].status = 1;
                if ( !isValid )
                    changed |= 1u << lane;
            }
            uint32_t pending = changed;
            while ( pending )
            {
                const uint32_t lane = highestLane( pending );
                pending &= ~( 1u << lane );
                const uint32_t j = neighbor[ lane ];
                if ( w.known( j ) )
                    continue;
                w.update( j, ctx.sites[ j ] );
            }
            if ( changed )
            {
                ctx.count( cVertexInvalid, uint64_t( __builtin_popcount( changed ) ) );
                if ( restarts == 0 )
                    ctx.count( cVertexCellsChanged );
                vs = 0;
                restarts++;
            }
        }
    }

    // Shared end of the edge and bisector passes: new vertices are appended after the
    // vertices stored before the pass (algorithm.inl:840-855, 1216-1231).
    void appendPassVertices( Cell & c, const std::vector<Vertex> & base, uint32_t baseN, Cell & pass )
    {
        std::vector<Vertex> merged( std::max<std::size_t>( 1024, baseN + pass.vn ) );
        for ( uint32_t v = 0; v < baseN; v++ )
            merged[ v ] = base[ v ];
        for ( uint32_t v = 0; v < pass.vn; v++ )
            merged[ baseN + v ] = pass.v[ v ];
        c.v  = std::move( merged );
        c.vn = baseN + pass.vn;
        c.e  = std::move( pass.e );
        c.en = pass.en;
    }

    // globalEdgeValidation (algorithm.inl:478-857)
    void edgeValidation( Context & ctx, uint32_t i )
    {
        if ( ctx.status[ i ] == kFullyValidated || ctx.status[ i ] == kBuried )
            return;
        const uint32_t n = ctx.n;
        Cell &         stored = ctx.cells[ i ];
        const float    knownRadius = ctx.knownRadii[ i ];

        Cell pass;
        pass.reserve();
        pass.en = stored.en;
        for ( uint32_t e = 0; e < stored.en; e++ )
        {
            pass.e[ e ] = stored.e[ e ];
            if ( pass.e[ e ].status != 1 )
                pass.e[ e ].status = 2;
        }
        pass.vn = 0;
        CellWork w { ctx, i, ctx.sites[ i ], pass, ctx.flags[ i ] };
        const D4 si  = w.si;
        const F4 fsi = toFloat( si );
        bool     didChange = false, anyFound = false;

        const uint32_t stepNb = pass.en / 32 + 1;
        for ( uint32_t es = 0; es < stepNb; es++ )
        {
            uint32_t found[ 32 ], eid[ 32 ];
            bool     needSearch[ 32 ];
            for ( uint32_t lane = 0; lane < 32; lane++ )
            {
                eid[ lane ]        = es * 32 + lane;
                found[ lane ]      = kNone;
                needSearch[ lane ] = eid[ lane ] < pass.en;
                uint32_t k = kNone, l = kNone;
                if ( needSearch[ lane ] )
                {
                    k                  = pass.e[ eid[ lane ] ].j;
                    l                  = pass.e[ eid[ lane ] ].k;
                    needSearch[ lane ] = pass.e[ eid[ lane ] ].status == 2;
                }
                uint32_t edgeType = 0;
                D4       ev[ 2 ] = {};
                D4       sk {}, sl {};
                if ( needSearch[ lane ] )
                {
                    sk       = ctx.sites[ k ];
                    sl       = ctx.sites[ l ];
                    edgeType = trisectorVertex( si, sk, sl, ev[ 0 ], ev[ 1 ] );
                }
                const bool isHyperbola = edgeType == 1, isEllipsis = edgeType == 2;
                const F4   v1 = toFloat( ev[ 0 ] ), v2 = toFloat( ev[ 1 ] );
                const F3   c1 = xyz( v1 ), c2 = xyz( v2 );
                F3         n1 { 0, 0, 0 }, n2 { 0, 0, 0 }, pp1 { 0, 0, 0 }, pp2 { 0, 0, 0 };
                F4         bsph { 0, 0, 0, 0 };
                if ( needSearch[ lane ] && isEllipsis )
                {
                    const F3    center = scale( add( c1, c2 ), .5f );
                    const float radius = length( sub( center, c1 ) ) + v1.w;
                    bsph               = { center.x, center.y, center.z, radius };
                }
                else if ( needSearch[ lane ] )
                {
                    D3 nn1, nn2;
                    getTangentPlanes( si, sk, sl, nn1, nn2 );
                    n1          = toFloat( nn1 );
                    n2          = toFloat( nn2 );
                    const D3 p1 = add( xyz( si ), scale( nn1, si.w ) );
                    const D3 p2 = add( xyz( sk ), scale( nn1, sk.w ) );
                    const D3 p3 = add( xyz( sl ), scale( nn1, sl.w ) );
                    const D3 p4 = add( xyz( si ), scale( nn2, si.w ) );
                    const D3 p5 = add( xyz( sk ), scale( nn2, sk.w ) );
                    bsph        = toFloat( sphereFromPoints( p1, p2, p3, p5 ) );
                    pp1         = toFloat( p1 );
                    pp2         = toFloat( p4 );
                }
                const bool inSecurity = lessThan( length( sub( xyz( fsi ), xyz( bsph ) ) ), knownRadius - bsph.w );
                if ( eid[ lane ] < pass.en && inSecurity )
                {
                    pass.e[ eid[ lane ] ].status = 1;
                    needSearch[ lane ]           = false;
                }
                if ( eid[ lane ] < pass.en )
                    ctx.count( cEdgeTasks );
                if ( eid[ lane ] < pass.en && inSecurity )
                    ctx.count( cEdgeSecurity );
                if ( !needSearch[ lane ] )
                    continue;
                ctx.count( cEdgeSearched );

                // (profiling only) radius bound of the edge arc: its vertices and, for an
                // elliptic trisector, its apexes
                double wEdge = 0.0;
                for ( uint32_t v = 0; v < stored.vn; v++ )
                {
                    const Vertex & vx = stored.v[ v ];
                    const bool hasK = vx.j == k || vx.k == k || vx.l == k;
                    const bool hasL = vx.j == l || vx.k == l || vx.l == l;
                    if ( hasK && hasL )
                        wEdge = dmax( wEdge, w.vertexPosition( vx ).w );
                }
                if ( edgeType == 2 || pass.e[ eid[ lane ] ].vertexNb == kNone )
                {
                    // an apex counts when it may lie on the cell's arc: no neighbour other
                    // than k, l clearly intersects its sphere
                    for ( int a = 0; a < 2; a++ )
                    {
                        bool clearlyOut = false;
                        for ( uint32_t e2 = 0; e2 < pass.en && !clearlyOut; e2++ )
                            for ( uint32_t u : { pass.e[ e2 ].j, pass.e[ e2 ].k } )
                            {
                                if ( u == k || u == l )
                                    continue;
                                const D4     su  = ctx.sites[ u ];
                                const double d   = std::sqrt( dot( sub( xyz( su ), xyz( ev[ a ] ) ), sub( xyz( su ), xyz( ev[ a ] ) ) ) );
                                const double pen = ( su.w + ev[ a ].w ) - d;
                                if ( pen > 1e-4 * ( su.w + std::fabs( ev[ a ].w ) ) + 1e-6 )
                                    clearlyOut = true;
                            }
                        if ( !clearlyOut )
                            wEdge = dmax( wEdge, ev[ a ].w );
                    }
                }
                const double ballR = 2.0 * wEdge * 1.01 + si.w + ctx.rmax + 1e-3;
                uint32_t logLeaves = 0, logCandidates = 0, logInBall = 0;
                uint32_t stack[ 64 ];
                int      sp = 0;
                uint32_t node = 0;
                bool     cont = true;
                while ( cont )
                {
                    while ( true )
                    {
                        if ( node >= n - 1 )
                            break;
                        const uint32_t lc = uint32_t( ctx.left[ node ] ), rc = uint32_t( ctx.right[ node ] );
                        const Box      lb = ctx.box( lc ), rb = ctx.box( rc );
                        const F3       closestL = lb.closestPoint( bsph ), closestR = rb.closestPoint( bsph );
                        const float    dL = lb.distance( bsph ), dR = rb.distance( bsph );
                        const bool     leftClosest = dL < dR;
                        const float    minFar = leftClosest ? dR : dL, minClose = leftClosest ? dL : dR;
                        const F3       farPoint = leftClosest ? closestR : closestL;
                        const F3       closePoint = leftClosest ? closestL : closestR;
                        const uint32_t farChild = leftClosest ? rc : lc, closeChild = leftClosest ? lc : rc;
                        bool           exploreFar = minFar < 0.f;
                        if ( isHyperbola && exploreFar )
                            exploreFar = dot( n1, sub( farPoint, pp1 ) ) < 0.f && dot( n2, sub( farPoint, pp2 ) ) < 0.f;
                        bool exploreClose = minClose < 0.f;
                        if ( isHyperbola && exploreClose )
                            exploreClose = dot( n1, sub( closePoint, pp1 ) ) < 0.f && dot( n2, sub( closePoint, pp2 ) ) < 0.f;
                        if ( !exploreFar && !exploreClose )
                            break;
                        node = exploreClose ? closeChild : farChild;
                        if ( exploreClose && exploreFar )
                        {
                            if ( sp >= 64 )
                                ctx.flags[ i ] |= kFlagStack;
                            else
                                stack[ sp++ ] = farChild;
                        }
                    }
                    if ( node >= n - 1 && node < 2 * n - 1 )
                    {
                        ctx.count( cEdgeLeaves );
                        logLeaves++;
                        const uint32_t j   = node - ( n - 1 );
                        bool           can = j != i && j != k && j != l && ctx.status[ j ] != kBuried;
                        D4             sj {};
                        if ( can )
                        {
                            sj          = ctx.sites[ j ];
                            const F4 fj = toFloat( sj );
                            can         = intersect( fj, bsph );
                            if ( isHyperbola )
                                can = can && double( dot( n1, sub( xyz( fj ), pp1 ) ) ) < -sj.w
                                      && double( dot( n2, sub( xyz( fj ), pp2 ) ) ) < -sj.w;
                        }
                        bool inBall = false;
                        if ( can )
                        {
                            ctx.count( cEdgeCandidates );
                            logCandidates++;
                            inBall = length( sub( xyz( sj ), xyz( si ) ) ) <= ballR;
                            if ( inBall )
                            {
                                ctx.count( cEdgeCandInBall );
                                logInBall++;
                            }
                        }
                        can = can && !w.known( j );
                        uint8_t mask = 0;
                        D4      x[ 2 ] = {};
                        if ( can )
                        {
                            ctx.count( cEdgeSolves );
                            mask = quadrisector( si, sj, sk, sl, x[ 0 ], x[ 1 ] );
                            if ( mask != 3 )
                                mask = 0;
                        }
                        uint8_t valid = mask, m = mask;
                        while ( m )
                        {
                            const uint32_t nv = uint32_t( __builtin_ctz( m ) );
                            m &= uint8_t( ~( 1u << nv ) );
                            if ( !w.predicate( x[ nv ], k, l ) )
                                valid &= uint8_t( ~( 1u << nv ) );
                        }
                        if ( can && inBall )
                            ctx.count( cEdgeSolvesInBall );
                        if ( valid )
                        {
                            if ( !inBall )
                                ctx.count( cEdgeFoundOutsideBall );
                            found[ lane ] = j;
                            cont          = false;
                        }
                    }
                    if ( cont )
                    {
                        if ( sp == 0 )
                            cont = false;
                        else
                            node = stack[ --sp ];
                    }
                }
#pragma omp critical( edge_log )
                {
                    uint32_t b[ 4 ];
                    std::memcpy( b, &bsph, 16 );
                    ctx.edgeSearchLog.insert( ctx.edgeSearchLog.end(),
                                              { i, k, l, logLeaves, logCandidates, uint32_t( ctx.round ), edgeType, b[ 0 ], b[ 1 ], b[ 2 ], b[ 3 ], logInBall, uint32_t( std::min( ballR, 4e9 ) ) } );
                }
                if ( found[ lane ] == kNone )
                    pass.e[ eid[ lane ] ].status = 1;
                else
                {
                    ctx.count( cEdgeFound );
                    anyFound = true;
                }
            }
            for ( int lane = 31; lane >= 0; lane-- )
            {
                if ( found[ lane ] == kNone )
                    continue;
                const uint32_t j = found[ lane ];
                if ( w.known( j ) )
                    continue;
                const bool changed = w.update( j, ctx.sites[ j ] );
                didChange          = didChange || changed;
                if ( changed )
                    es = 0;
            }
        }
        if ( didChange )
            ctx.count( cEdgeCellsChanged );
        if ( anyFound )
            ctx.count( cEdgeCellsFound );
        appendPassVertices( stored, stored.v, stored.vn, pass );
        ctx.status[ i ] = didChange ? 0 : 1;
    }

    // globalBisectorValidation (algorithm.inl:859-1233)
    void bisectorValidation( Context & ctx, uint32_t i )
    {
        if ( ctx.status[ i ] == kBuried )
            return;
        const uint32_t n = ctx.n;
        Cell &         stored = ctx.cells[ i ];
        const float    knownRadius = ctx.knownRadii[ i ];

        Cell pass;
        pass.reserve();
        pass.en = stored.en;
        for ( uint32_t e = 0; e < stored.en; e++ )
            pass.e[ e ] = stored.e[ e ];
        pass.vn = 0;

        // unique neighbour ids greater than i, ascending (:903-968)
        std::vector<uint32_t> bis;
        {
            std::vector<uint32_t> perLane( 32, 0 );
            for ( uint32_t e = 0; e < pass.en; e++ )
            {
                const uint32_t lane = e % 32;
                if ( pass.e[ e ].j < n )
                {
                    bis.push_back( pass.e[ e ].j );
                    perLane[ lane ]++;
                }
                if ( pass.e[ e ].k < n )
                {
                    bis.push_back( pass.e[ e ].k );
                    perLane[ lane ]++;
                }
            }
            for ( uint32_t lane = 0; lane < 32; lane++ )
                if ( perLane[ lane ] >= kMaxBisectors / 32 )
                    ctx.flags[ i ] |= kFlagBisector;
            std::sort( bis.begin(), bis.end() );
            bis.erase( std::unique( bis.begin(), bis.end() ), bis.end() );
            bis.erase( std::remove_if( bis.begin(), bis.end(), [ & ]( uint32_t b ) { return b <= i; } ), bis.end() );
            if ( bis.size() >= kMaxBisectors )
                ctx.flags[ i ] |= kFlagBisector;
        }

        CellWork w { ctx, i, ctx.sites[ i ], pass, ctx.flags[ i ] };
        const D4    si  = w.si;
        const F3    fci { float( si.x ), float( si.y ), float( si.z ) };
        const float fri = float( si.w );
        bool        didChange = false;

        const uint32_t bisectorNb = uint32_t( bis.size() );
        const uint32_t stepNb     = bisectorNb / 32 + 1;
        for ( uint32_t bs = 0; bs < stepNb; bs++ )
        {
            uint32_t found[ 32 ];
            for ( uint32_t lane = 0; lane < 32; lane++ )
            {
                found[ lane ]      = kNone;
                const uint32_t bid = bs * 32 + lane;
                uint32_t       bisector = kNone;
                bool           needSearch = bid < bisectorNb;
                if ( needSearch )
                {
                    bisector   = bis[ bid ];
                    needSearch = bisector != kNone;
                }
                D4    sk {};
                F3    fck { 0, 0, 0 };
                float frk = 0.f;
                if ( needSearch )
                {
                    sk                   = ctx.sites[ bisector ];
                    fck                  = { float( sk.x ), float( sk.y ), float( sk.z ) };
                    frk                  = float( sk.w );
                    const float distance = length( sub( fci, fck ) ) + fri + frk;
                    if ( lessThan( distance, knownRadius ) )
                    {
                        bis[ bid ]  = kNone;
                        needSearch  = false;
                    }
                }
                if ( !needSearch )
                    continue;
                ctx.count( cBisSearched );
                const F3    center = scale( add( fci, fck ), .5f );
                const float radius = length( sub( center, fci ) ) + fmaxf_( fri, frk );
                const F4    bsph { center.x, center.y, center.z, radius };
                const float cylinderRadius = fmaxf_( fri, frk );

                uint32_t stack[ 64 ];
                int      sp = 0;
                uint32_t node = 0;
                bool     cont = true;
                while ( cont )
                {
                    while ( true )
                    {
                        if ( node >= n - 1 )
                            break;
                        const uint32_t lc = uint32_t( ctx.left[ node ] ), rc = uint32_t( ctx.right[ node ] );
                        const float    dL = ctx.box( lc ).distance( bsph ), dR = ctx.box( rc ).distance( bsph );
                        const bool     leftClosest = dL < dR;
                        const float    minFar = leftClosest ? dR : dL, minClose = leftClosest ? dL : dR;
                        const uint32_t farChild = leftClosest ? rc : lc, closeChild = leftClosest ? lc : rc;
                        const bool     exploreFar = minFar < 0.f, exploreClose = minClose < 0.f;
                        if ( !exploreFar && !exploreClose )
                            break;
                        node = exploreClose ? closeChild : farChild;
                        if ( exploreClose && exploreFar )
                        {
                            if ( sp >= 64 )
                                ctx.flags[ i ] |= kFlagStack;
                            else
                                stack[ sp++ ] = farChild;
                        }
                    }
                    if ( node >= n - 1 && node < 2 * n - 1 )
                    {
                        ctx.count( cBisLeaves );
                        const uint32_t j   = node - ( n - 1 );
                        bool           can = j != i && j != bisector;
                        D4             sj {};
                        if ( can )
                        {
                            sj          = ctx.sites[ j ];
                            const F4 fj = toFloat( sj );
                            const F3 cj = xyz( fj );
                            can = bsph.w >= fj.w && length( sub( xyz( bsph ), cj ) ) <= ( bsph.w - fj.w );
                            if ( can )
                            {
                                const F3    itoj = sub( cj, fci );
                                const float v    = dot( itoj, normalize( sub( fck, fci ) ) );
                                const float d    = std::sqrt( dot( itoj, itoj ) - v * v );
                                can              = ( d + fj.w ) < cylinderRadius;
                            }
                        }
                        if ( can )
                            ctx.count( cBisCandidates );
                        can = can && !w.known( j );
                        D4 vtx {};
                        if ( can )
                        {
                            D4 x[ 2 ] = {};
                            const uint8_t count = trisectorVertex( si, sj, sk, x[ 0 ], x[ 1 ] );
                            vtx                 = x[ 1 ];
                            can                 = count == 2;
                        }
                        if ( can )
                            can = w.predicate( vtx, bisector, bisector );
                        if ( can )
                        {
                            found[ lane ] = j;
                            cont          = false;
                        }
                    }
                    if ( cont )
                    {
                        if ( sp == 0 )
                            cont = false;
                        else
                            node = stack[ --sp ];
                    }
                }
                if ( found[ lane ] == kNone )
                    bis[ bid ] = kNone;
                else
                    ctx.count( cBisFound );
            }
            for ( int lane = 31; lane >= 0; lane-- )
            {
                if ( found[ lane ] == kNone )
                    continue;
                const uint32_t j = found[ lane ];
                if ( w.known( j ) )
                    continue;
                const bool changed = w.update( j, ctx.sites[ j ] );
                didChange          = didChange || changed;
                if ( changed )
                    bs = 0;
            }
        }
        if ( didChange )
            ctx.count( cBisCellsChanged );
        appendPassVertices( stored, stored.v, stored.vn, pass );
        ctx.status[ i ] = didChange ? 0 : 1;
    }

    template<class F>
    void parallelFor( uint32_t count, int threads, F && f )
    {
#ifdef _OPENMP
#pragma omp parallel for schedule( dynamic, 64 ) num_threads( threads )
        for ( int64_t i = 0; i < int64_t( count ); i++ )
            f( uint32_t( i ) );
#else
        (void)threads;
        for ( uint32_t i = 0; i < count; i++ )
            f( i );
#endif
    }

    // ------------------------------------------------------------------------------------
    // Driver (algorithm.inl:1410-1594) and outputs (algorithm.inl:1235-1383, 1596-1821)
    // ------------------------------------------------------------------------------------
    void run( Context & ctx, const std::vector<D4> & input, int lastStage, int threads )
    {
        const uint32_t n = ctx.n;
        // bbox and radius range on the host (algorithm.cpp:5-25)
        double mn[ 3 ] = { DBL_MAX, DBL_MAX, DBL_MAX }, mx[ 3 ] = { -DBL_MAX, -DBL_MAX, -DBL_MAX };
        double minRadius = DBL_MAX;
        for ( uint32_t v = 0; v < n; v++ )
        {
            const D4 s = input[ v ];
            mn[ 0 ]    = std::min( mn[ 0 ], s.x - s.w );
            mn[ 1 ]    = std::min( mn[ 1 ], s.y - s.w );
            mn[ 2 ]    = std::min( mn[ 2 ], s.z - s.w );
            mx[ 0 ]    = std::max( mx[ 0 ], s.x + s.w );
            mx[ 1 ]    = std::max( mx[ 1 ], s.y + s.w );
            mx[ 2 ]    = std::max( mx[ 2 ], s.z + s.w );
            minRadius  = std::min( minRadius, s.w );
            ctx.rmax   = std::max( ctx.rmax, s.w );
        }
        buildLbvh( ctx, input, mn, mx );

        // six joggled bounding sites after the real ones (algorithm.inl:1442-1464)
        {
            const D3     center { ( mn[ 0 ] + mx[ 0 ] ) / 2.0, ( mn[ 1 ] + mx[ 1 ] ) / 2.0, ( mn[ 2 ] + mx[ 2 ] ) / 2.0 };
            const double aabbRadius = length( sub( center, D3 { mx[ 0 ], mx[ 1 ], mx[ 2 ] } ) );
            const double radius     = aabbRadius * ( std::sqrt( 3.0 ) + 1e-1 );
            double       art[ 24 ]  = {
                center.x + radius, center.y + 0.0, center.z + 0.0, 0.0 + minRadius,
                center.x - radius, center.y + 0.0, center.z + 0.0, 0.0 + minRadius,
                center.x + 0.0, center.y + radius, center.z + 0.0, 0.0 + minRadius,
                center.x + 0.0, center.y - radius, center.z + 0.0, 0.0 + minRadius,
                center.x + 0.0, center.y + 0.0, center.z + radius, 0.0 + minRadius,
                center.x + 0.0, center.y + 0.0, center.z - radius, 0.0 + minRadius,
            };
            joggle( art, 6, 1e-1 );
            for ( uint32_t a = 0; a < 6; a++ )
                ctx.sites[ n + a ] = { art[ a * 4 + 0 ], art[ a * 4 + 1 ], art[ a * 4 + 2 ], art[ a * 4 + 3 ] };
        }
        ctx.status.assign( n, 0 );
        ctx.flags.assign( n, 0 );
        if ( lastStage < ORACLE_STAGE_KNN )
            return;

        ctx.knn.assign( std::size_t( n ) * ctx.k, kNone );
        if ( ctx.knnSteps > 0 )
            parallelFor( n, threads, [ & ]( uint32_t id ) { knnSite( ctx, id, 0 ); } );
        if ( lastStage < ORACLE_STAGE_CELLS )
            return;

        ctx.cells.resize( n );
        ctx.knownRadii.assign( n, -FLT_MAX );
        for ( uint32_t i = 0; i < n; i++ )
            initialCell( ctx, ctx.cells[ i ] );
        if ( ctx.profile )
        {
            ctx.contribution.assign( std::size_t( n ) * ctx.knnSteps * ctx.k, 0 );
            ctx.reached.assign( std::size_t( n ) * ctx.knnSteps * ctx.k, 0 );
        }
        for ( uint32_t step = 0; step < ctx.knnSteps; step++ )
        {
            if ( step > 0 )
                parallelFor( n, threads, [ & ]( uint32_t id ) { knnSite( ctx, id, step ); } );
            if ( ctx.profile )
                parallelFor( n, threads, [ & ]( uint32_t i ) { cellContribution( ctx, i, step ); } );
            else
                parallelFor( n, threads, [ & ]( uint32_t i ) { cellFromKnn( ctx, i ); } );
        }
        if ( ctx.profile )
            return;

        if ( lastStage >= ORACLE_STAGE_VALIDATION )
        {
            std::vector<uint32_t> tasks;
            for ( uint32_t i = 0; i < n; i++ )
                if ( ctx.status[ i ] == kInValidation )
                    tasks.push_back( i );
            for ( int iteration = 0; iteration < 10 && !tasks.empty(); iteration++ )
            {
                parallelFor( uint32_t( tasks.size() ), threads, [ & ]( uint32_t t ) { vertexValidation( ctx, tasks[ t ] ); } );
                ctx.round = iteration;
                parallelFor( uint32_t( tasks.size() ), threads, [ & ]( uint32_t t ) { edgeValidation( ctx, tasks[ t ] ); } );
                tasks.clear();
                for ( uint32_t i = 0; i < n; i++ )
                    if ( ctx.status[ i ] == kInValidation )
                        tasks.push_back( i );
            }
            parallelFor( n, threads, [ & ]( uint32_t i ) { bisectorValidation( ctx, i ); } );
        }

        // flattened per-cell stores
        ctx.vertexNb.resize( n );
        ctx.edgeNb.resize( n );
        for ( uint32_t i = 0; i < n; i++ )
        {
            const Cell & c = ctx.cells[ i ];
            ctx.vertexNb[ i ] = c.vn;
            ctx.edgeNb[ i ]   = c.en;
            for ( uint32_t v = 0; v < c.vn; v++ )
            {
                const Vertex & x = c.v[ v ];
                ctx.flatVertices.insert( ctx.flatVertices.end(), { x.j, x.k, x.l, uint32_t( x.type ) | ( uint32_t( x.status ) << 8 ) } );
            }
            for ( uint32_t e = 0; e < c.en; e++ )
            {
                const Edge & x = c.e[ e ];
                ctx.flatEdges.insert( ctx.flatEdges.end(), { x.j, x.k, x.vertexNb, uint32_t( x.status ) | ( uint32_t( x.validatedNb ) << 8 ) } );
            }
            ctx.flagsAll |= ctx.flags[ i ];
        }
        if ( lastStage < ORACLE_STAGE_OUTPUT )
            return;

        // saveVertices / saveClosedEdges (algorithm.inl:1235-1383)
        for ( uint32_t id = 0; id < n; id++ )
        {
            if ( ctx.status[ id ] == kBuried )
                continue;
            const Cell & c  = ctx.cells[ id ];
            const D4     si = ctx.sites[ id ];
            for ( uint32_t v = 0; v < c.vn; v++ )
            {
                const Vertex & x = c.v[ v ];
                if ( id > x.j || x.j >= n || x.k >= n || x.l >= n )
                    continue;
                D4 r[ 2 ] = {};
                quadrisector( si, ctx.sites[ x.j ], ctx.sites[ x.k ], ctx.sites[ x.l ], r[ 0 ], r[ 1 ] );
                const D4 p = r[ x.type & 1 ];
                ctx.outVertices.insert( ctx.outVertices.end(), { p.x, p.y, p.z, p.w } );
                ctx.outVerticesId.insert( ctx.outVerticesId.end(),
                                          { ctx.indices[ id ], ctx.indices[ x.j ], ctx.indices[ x.k ], ctx.indices[ x.l ] } );
            }
        }
        for ( uint32_t id = 0; id < n; id++ )
        {
            if ( ctx.status[ id ] == kBuried )
                continue;
            const Cell & c  = ctx.cells[ id ];
            const D4     si = ctx.sites[ id ];
            for ( uint32_t e = 0; e < c.en; e++ )
            {
                const Edge & x = c.e[ e ];
                if ( x.vertexNb != kNone || id > x.j || x.j >= n || x.k >= n )
                    continue;
                D4 r[ 2 ] = {};
                trisectorVertex( si, ctx.sites[ x.j ], ctx.sites[ x.k ], r[ 0 ], r[ 1 ] );
                if ( r[ 1 ].w < r[ 0 ].w )
                    r[ 0 ] = r[ 1 ];
                ctx.outClosed.insert( ctx.outClosed.end(), { r[ 0 ].x, r[ 0 ].y, r[ 0 ].z, r[ 0 ].w } );
                ctx.outClosedId.insert( ctx.outClosedId.end(), { ctx.indices[ id ], ctx.indices[ x.j ], ctx.indices[ x.k ], 0u } );
            }
        }

        // toTopology (algorithm.inl:1732-1821): per sorted cell, unique tuples in sorted
        // space with i smallest, then mapped to original ids.
        for ( uint32_t i = 0; i < n; i++ )
        {
            const Cell &                                   c = ctx.cells[ i ];
            std::vector<std::pair<uint32_t, uint32_t>>     bi;
            std::vector<std::array<uint32_t, 2>>           tri;
            std::vector<std::array<uint32_t, 3>>           quad;
            for ( uint32_t e = 0; e < c.en; e++ )
            {
                const Edge & x = c.e[ e ];
                if ( i < x.j && x.j < n )
                    bi.push_back( { i, x.j } );
                if ( i < x.k && x.k < n )
                    bi.push_back( { i, x.k } );
                if ( i < x.j && i < x.k && x.j < n && x.k < n )
                    tri.push_back( { x.j, x.k } );
            }
            for ( uint32_t v = 0; v < c.vn; v++ )
            {
                const Vertex & x = c.v[ v ];
                if ( i < x.j && i < x.k && i < x.l && x.j < n && x.k < n && x.l < n )
                    quad.push_back( { x.j, x.k, x.l } );
            }
            std::sort( bi.begin(), bi.end() );
            bi.erase( std::unique( bi.begin(), bi.end() ), bi.end() );
            std::sort( tri.begin(), tri.end() );
            tri.erase( std::unique( tri.begin(), tri.end() ), tri.end() );
            std::sort( quad.begin(), quad.end() );
            quad.erase( std::unique( quad.begin(), quad.end() ), quad.end() );
            const auto & ix = ctx.indices;
            for ( auto & b : bi )
                ctx.topoBi.insert( ctx.topoBi.end(), { ix[ b.first ], ix[ b.second ] } );
            for ( auto & t : tri )
                ctx.topoTri.insert( ctx.topoTri.end(), { ix[ i ], ix[ t[ 0 ] ], ix[ t[ 1 ] ] } );
            for ( auto & q : quad )
                ctx.topoQuad.insert( ctx.topoQuad.end(), { ix[ i ], ix[ q[ 0 ] ], ix[ q[ 1 ] ], ix[ q[ 2 ] ] } );
        }
    }
} // namespace

struct oracle_run
{
    Context ctx;
};

namespace
{
    oracle_run * buildFrom( std::vector<D4> && input, uint32_t n, int lastStage, int threads, uint32_t k = kK,
                            uint32_t knnSteps = 1, bool profile = false )
    {
        if ( n < 2 || k < 1 || k > kK )
            return nullptr;
#ifdef _OPENMP
        if ( threads <= 0 )
            threads = omp_get_max_threads();
#else
        threads = 1;
#endif
        oracle_run * r = new oracle_run {};
        r->ctx.n        = n;
        r->ctx.k        = k;
        r->ctx.knnSteps = knnSteps;
        r->ctx.profile  = profile;
        run( r->ctx, input, lastStage, threads );
        return r;
    }
} // namespace

extern "C" {

oracle_run * oracle_build( const float * sites, uint32_t n, int lastStage, int threads )
{
    std::vector<D4> input( n );
    for ( uint32_t i = 0; i < n; i++ )
        input[ i ] = { sites[ 4 * i ], sites[ 4 * i + 1 ], sites[ 4 * i + 2 ], sites[ 4 * i + 3 ] };
    return buildFrom( std::move( input ), n, lastStage, threads );
}

oracle_run * oracle_build_f64( const double * sites, uint32_t n, int lastStage, int threads )
{
    std::vector<D4> input( n );
    for ( uint32_t i = 0; i < n; i++ )
        input[ i ] = { sites[ 4 * i ], sites[ 4 * i + 1 ], sites[ 4 * i + 2 ], sites[ 4 * i + 3 ] };
    return buildFrom( std::move( input ), n, lastStage, threads );
}

oracle_run * oracle_build_ex( const void * sites, int is_f64, uint32_t n, uint32_t k, uint32_t knn_steps, int lastStage,
                              int threads )
{
    std::vector<D4> input( n );
    for ( uint32_t i = 0; i < n; i++ )
    {
        if ( is_f64 )
        {
            const double * p = static_cast<const double *>( sites ) + 4 * std::size_t( i );
            input[ i ]       = { p[ 0 ], p[ 1 ], p[ 2 ], p[ 3 ] };
        }
        else
        {
            const float * p = static_cast<const float *>( sites ) + 4 * std::size_t( i );
            input[ i ]      = { p[ 0 ], p[ 1 ], p[ 2 ], p[ 3 ] };
        }
    }
    return buildFrom( std::move( input ), n, lastStage, threads, k, knn_steps );
}

oracle_run * oracle_contribution_profile( const float * sites, uint32_t n, uint32_t steps, int threads )
{
    if ( steps < 1 )
        return nullptr;
    std::vector<D4> input( n );
    for ( uint32_t i = 0; i < n; i++ )
        input[ i ] = { sites[ 4 * i ], sites[ 4 * i + 1 ], sites[ 4 * i + 2 ], sites[ 4 * i + 3 ] };
    return buildFrom( std::move( input ), n, ORACLE_STAGE_CELLS, threads, kK, steps, true );
}

uint64_t oracle_get( const oracle_run * r, const char * name, const void ** data )
{
    const Context & c = r->ctx;
    const std::string key( name );
#define ORACLE_ARRAY( label, vec )           \
    if ( key == label )                      \
    {                                        \
        *data = ( vec ).data();              \
        return uint64_t( ( vec ).size() );   \
    }
    ORACLE_ARRAY( "indices", c.indices )
    ORACLE_ARRAY( "morton", c.morton )
    ORACLE_ARRAY( "parent", c.parent )
    ORACLE_ARRAY( "left", c.left )
    ORACLE_ARRAY( "right", c.right )
    ORACLE_ARRAY( "aabb", c.aabb )
    ORACLE_ARRAY( "sizes", c.sizes )
    ORACLE_ARRAY( "status", c.status )
    ORACLE_ARRAY( "knn", c.knn )
    ORACLE_ARRAY( "known_radii", c.knownRadii )
    ORACLE_ARRAY( "vertex_nb", c.vertexNb )
    ORACLE_ARRAY( "edge_nb", c.edgeNb )
    ORACLE_ARRAY( "vertices", c.flatVertices )
    ORACLE_ARRAY( "edges", c.flatEdges )
    ORACLE_ARRAY( "out_vertices", c.outVertices )
    ORACLE_ARRAY( "out_vertices_id", c.outVerticesId )
    ORACLE_ARRAY( "out_closed", c.outClosed )
    ORACLE_ARRAY( "out_closed_id", c.outClosedId )
    ORACLE_ARRAY( "topo_quad", c.topoQuad )
    ORACLE_ARRAY( "topo_tri", c.topoTri )
    ORACLE_ARRAY( "topo_bi", c.topoBi )
    ORACLE_ARRAY( "counters", c.counters )
    ORACLE_ARRAY( "edge_search_log", c.edgeSearchLog )
    ORACLE_ARRAY( "contribution", c.contribution )
    ORACLE_ARRAY( "reached", c.reached )
#undef ORACLE_ARRAY
    if ( key == "sites_sorted" )
    {
        *data = c.sites.data();
        return uint64_t( c.sites.size() ) * 4;
    }
    *data = nullptr;
    return 0;
}

uint32_t oracle_flags( const oracle_run * r ) { return r->ctx.flagsAll; }

void oracle_free( oracle_run * r ) { delete r; }

void oracle_joggle( double * sites, uint64_t n, double range ) { joggle( sites, n, range ); }

} // extern "C"
