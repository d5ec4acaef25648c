// Geometric predicates and solves of the Apollonius-diagram build, device side.
//
// Every decision of the build (which vertex is inside a neighbour, which root of a vertex
// quadratic exists, which BVH child a walk enters) is taken on values computed here, so
// the arithmetic follows the reference's formulas operation for operation, in the same
// order, and this file is compiled with the same floating-point mode as the reference
// library (--use_fast_math: approximate single-precision sqrt/rsqrt with flush-to-zero,
// FMA contraction on; double precision unaffected). That is what makes the per-site
// topology bit-identical to the reference's; see each function's citation (paths relative
// to the PlathC/apo tree).
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace apo2
{
    // ---------------------------------------------------------------------------------
    // eps comparisons (apo/include/apo/core/math.inl:217-244)
    // ---------------------------------------------------------------------------------
    __device__ __forceinline__ bool lt_eps( double a, double b ) { return ( a - b ) < 1e-8; }
    __device__ __forceinline__ bool gt_eps( double a, double b ) { return ( a - b ) > -1e-8; }
    __device__ __forceinline__ bool lt_eps( float a, float b ) { return ( a - b ) < 1e-8f; }
    __device__ __forceinline__ bool gt_eps( float a, float b ) { return ( a - b ) > -1e-8f; }
    __device__ __forceinline__ bool near_zero( double v ) { return fabs( v ) < 1e-8; }
    __device__ __forceinline__ double sign_eps( double a ) { return lt_eps( a, 0.0 ) ? -1.0 : 1.0; }
    __device__ __forceinline__ float sign_eps( float a ) { return lt_eps( a, 0.f ) ? -1.f : 1.f; }

    // ---------------------------------------------------------------------------------
    // single precision vectors (traversal side)
    // ---------------------------------------------------------------------------------
    __device__ __forceinline__ float3 f3( float4 v ) { return make_float3( v.x, v.y, v.z ); }
    __device__ __forceinline__ float3 operator-( float3 a, float3 b ) { return make_float3( a.x - b.x, a.y - b.y, a.z - b.z ); }
    __device__ __forceinline__ float3 operator+( float3 a, float3 b ) { return make_float3( a.x + b.x, a.y + b.y, a.z + b.z ); }
    __device__ __forceinline__ float3 operator*( float3 a, float b ) { return make_float3( a.x * b, a.y * b, a.z * b ); }
    __device__ __forceinline__ float fdot( float3 a, float3 b ) { return a.x * b.x + a.y * b.y + a.z * b.z; }
    __device__ __forceinline__ float flength( float3 v ) { return sqrtf( fdot( v, v ) ); }
    __device__ __forceinline__ float3 fnormalize( float3 v )
    {
        const float inv = rsqrtf( fdot( v, v ) );
        return v * inv;
    }
    __device__ __forceinline__ float3 fmin3( float3 a, float3 b ) { return make_float3( fminf( a.x, b.x ), fminf( a.y, b.y ), fminf( a.z, b.z ) ); }
    __device__ __forceinline__ float3 fmax3( float3 a, float3 b ) { return make_float3( fmaxf( a.x, b.x ), fmaxf( a.y, b.y ), fmaxf( a.z, b.z ) ); }

    // gpu/math.cuh:368-372
    __device__ __forceinline__ float sphere_distance( float4 a, float4 b )
    {
        const float d = flength( make_float3( a.x, a.y, a.z ) - make_float3( b.x, b.y, b.z ) );
        return d - ( a.w + b.w );
    }
    // gpu/math.cuh:380-383
    __device__ __forceinline__ bool intersects( float4 a, float4 b ) { return lt_eps( sphere_distance( a, b ), 0.f ); }

    // Axis-aligned box of a BVH child (gpu/math.cuh:339-366, gpu/math.inl:79-101).
    struct Box
    {
        float3 lo, hi;
        __device__ __forceinline__ float3 closest( float4 s ) const { return fmin3( fmax3( f3( s ), lo ), hi ); }
        __device__ __forceinline__ float distance( float4 s ) const { return flength( f3( s ) - closest( s ) ) - s.w; }
        __device__ __forceinline__ float farthest( float4 s ) const
        {
            const float3 c      = f3( s ) - ( lo + hi ) * .5f;
            const float3 radius = make_float3( fabsf( lo.x - hi.x ), fabsf( lo.y - hi.y ), fabsf( lo.z - hi.z ) ) * .5f;
            const float3 far    = make_float3( radius.x * sign_eps( -c.x ), radius.y * sign_eps( -c.y ), radius.z * sign_eps( -c.z ) );
            return flength( c - far ) - s.w;
        }
    };

    // ---------------------------------------------------------------------------------
    // double precision vectors (solve side)
    // ---------------------------------------------------------------------------------
    __device__ __forceinline__ double3 d3( double4 v ) { return make_double3( v.x, v.y, v.z ); }
    __device__ __forceinline__ double3 operator-( double3 a, double3 b ) { return make_double3( a.x - b.x, a.y - b.y, a.z - b.z ); }
    __device__ __forceinline__ double3 operator+( double3 a, double3 b ) { return make_double3( a.x + b.x, a.y + b.y, a.z + b.z ); }
    __device__ __forceinline__ double4 operator-( double4 a, double4 b )
    {
        return make_double4( a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w );
    }
    __device__ __forceinline__ double3 operator*( double3 a, double b ) { return make_double3( b * a.x, b * a.y, b * a.z ); }
    __device__ __forceinline__ double ddot( double3 a, double3 b ) { return a.x * b.x + a.y * b.y + a.z * b.z; }
    __device__ __forceinline__ double ddot( double2 a, double2 b ) { return a.x * b.x + a.y * b.y; }
    __device__ __forceinline__ double3 dcross( double3 a, double3 b )
    {
        return make_double3( a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x );
    }
    // The reference's double `length` (gpu/math.cuh:307-309) resolves its unqualified `sqrt`
    // to apo::sqrt (core/math.inl:89-104), whose double branch sits behind a misspelled macro
    // (AAPO_REAL_SIZE), so under nvcc it is `sqrtf` of the float-rounded value: with
    // --use_fast_math, the approximate single-precision square root. Kept as such, since
    // every conflict predicate compares such a length against an eps of 1e-8.
    __device__ __forceinline__ double fsqrtd( double v ) { return double( sqrtf( float( v ) ) ); }
    __device__ __forceinline__ double dlength( double3 v ) { return fsqrtd( ddot( v, v ) ); }
    __device__ __forceinline__ double3 dnormalize( double3 v )
    {
        const double inv = rsqrt( ddot( v, v ) );
        return v * inv;
    }
    __device__ __forceinline__ float4 to_float( double4 v ) { return make_float4( float( v.x ), float( v.y ), float( v.z ), float( v.w ) ); }
    __device__ __forceinline__ float3 to_float( double3 v ) { return make_float3( float( v.x ), float( v.y ), float( v.z ) ); }

    // gpu/math.cuh:374-388
    __device__ __forceinline__ double sphere_distance( double4 a, double4 b )
    {
        const double d = dlength( make_double3( a.x - b.x, a.y - b.y, a.z - b.z ) );
        return d - ( a.w + b.w );
    }
    __device__ __forceinline__ bool intersects( double4 a, double4 b ) { return lt_eps( sphere_distance( a, b ), 0. ); }

    // FP32 static filter of the conflict predicate intersects(site, x) above, as the reference
    // evaluates it: d = double(sqrtf(float(|c - x|^2))) - (r + w) < 1e-8, with the approximate
    // single-precision square root of --use_fast_math. The filter recomputes d from the float
    // copy of the site in single precision (products and sums rounded to nearest, u = 2^-24; the
    // root is the same approximate one) and bounds its distance from the reference's value:
    //   the rounding of x to float and of each difference        u (|x|_1 + 1.01 |d|_1)
    //   the dot product                                          3 u L
    //   this filter's approximate root (<= 8u relative)          8 u L
    //   the radii sum, the final difference                      u (r + 2.01 |w| + 1.01 |d32|)
    //   the reference: float(D) and its approximate root         16.5 u L
    //   a float copy of a double site                            u (|c|_1 + r)
    // with |d|_1 <= sqrt(3) L (the approximate roots are taken at four times their documented
    // accuracy); twice that sum, plus a tiny absolute term for flushed subnormals, is the bound
    // E. A value with d32 - E >= 1e-8 is certainly not a conflict of the reference, one with
    // d32 + E < 1e-8 certainly is; anything in between (2) is left to the exact test.
    __device__ __forceinline__ int conflict_filter( float4 s, double4 x )
    {
        const float xx = __double2float_rn( x.x ), xy = __double2float_rn( x.y ), xz = __double2float_rn( x.z );
        const float xw = __double2float_rn( x.w );
        const float dx = __fsub_rn( s.x, xx ), dy = __fsub_rn( s.y, xy ), dz = __fsub_rn( s.z, xz );
        const float dd = __fadd_rn( __fadd_rn( __fmul_rn( dx, dx ), __fmul_rn( dy, dy ) ), __fmul_rn( dz, dz ) );
        const float L  = sqrtf( dd );
        const float d  = __fsub_rn( L, __fadd_rn( s.w, xw ) );
        const float mag = fabsf( xx ) + fabsf( xy ) + fabsf( xz ) + fabsf( s.x ) + fabsf( s.y ) + fabsf( s.z );
        const float E   = 1.1920929e-7f * ( mag + 30.f * L + 2.f * fabsf( s.w ) + 2.02f * fabsf( xw ) + 1.01f * fabsf( d ) )
                        + 1e-18f;
        // d - E and d + E rounded outward, against the floats just above and just below the
        // double threshold 1e-8 (0x322bcc78 = 1.00000008e-8, 0x322bcc77 = 0.99999999e-8)
        if ( __fsub_rd( d, E ) >= __uint_as_float( 0x322bcc78u ) )
            return 0;
        if ( __fadd_ru( d, E ) < __uint_as_float( 0x322bcc77u ) )
            return 1;
        return 2;
    }

    // 3x3 inverse by cofactors from the columns (gpu/math.cuh:398-411).
    __device__ __forceinline__ void inverse3( double3 c1, double3 c2, double3 c3, double3 & i1, double3 & i2, double3 & i3 )
    {
        const double  invD = 1.0 / ddot( c1, dcross( c2, c3 ) );
        const double3 r1   = dcross( c2, c3 );
        const double3 r2   = dcross( c3, c1 );
        const double3 r3   = dcross( c1, c2 );
        i1                 = make_double3( invD * r1.x, invD * r2.x, invD * r3.x );
        i2                 = make_double3( invD * r1.y, invD * r2.y, invD * r3.y );
        i3                 = make_double3( invD * r1.z, invD * r2.z, invD * r3.z );
    }
    // matrix (by columns) times vector (gpu/math.cuh:419-426)
    __device__ __forceinline__ double3 mul3( double3 c1, double3 c2, double3 c3, double3 b )
    {
        return make_double3( ddot( make_double3( c1.x, c2.x, c3.x ), b ), ddot( make_double3( c1.y, c2.y, c3.y ), b ),
                             ddot( make_double3( c1.z, c2.z, c3.z ), b ) );
    }

    // Trisector vertices of (s1, s2, s3) on the plane through the centres
    // (gpu/math.cuh:636-701). Returns 0, 1 or 2; x1 and x2 may be the same object.
    __device__ __forceinline__ uint32_t trisector( const double4 s1, const double4 s2, const double4 s3, double4 & x1, double4 & x2 )
    {
        const double3 p1 = d3( s1 ), p2 = d3( s2 ), p3 = d3( s3 );
        const double  r1 = s1.w, r2 = s2.w, r3 = s3.w;
        const double4 nh1 = s1 - s2, nh2 = s1 - s3;

        const double3 nIjk = dnormalize( dcross( p2 - p1, p3 - p1 ) );
        const double  w    = -ddot( nIjk, p1 );
        const double3 mC   = make_double3( .5 * ( -ddot( p1, p1 ) + ddot( p2, p2 ) + r1 * r1 - r2 * r2 ),
                                         .5 * ( -ddot( p1, p1 ) + ddot( p3, p3 ) + r1 * r1 - r3 * r3 ), w );
        double3 i1, i2, i3;
        inverse3( make_double3( nh1.x, nh2.x, nIjk.x ), make_double3( nh1.y, nh2.y, nIjk.y ),
                  make_double3( nh1.z, nh2.z, nIjk.z ), i1, i2, i3 );
        const double3 t  = mul3( i1, i2, i3, make_double3( nh1.w, nh2.w, 0.0 ) );
        const double3 mN = make_double3( -t.x, -t.y, -t.z );
        const double3 mB = mul3( i1, i2, i3, mC );

        const double e1 = -mN.x * r1 - mB.x - p1.x;
        const double e2 = -mN.y * r1 - mB.y - p1.y;
        const double e3 = -mN.z * r1 - mB.z - p1.z;
        const double a  = mN.x * mN.x + mN.y * mN.y + mN.z * mN.z - 1.0;
        const double b  = 2.0 * ( mN.x * e1 + mN.y * e2 + mN.z * e3 );
        const double c  = e1 * e1 + e2 * e2 + e3 * e3;

        const double delta = b * b - 4.0 * a * c;
        uint32_t     count = 0;
        const double q     = -.5 * ( b - sign_eps( b ) * sqrt( delta ) );

        const double  xd1 = ( c / q ) - r1;
        const double3 v1  = mN * xd1 - mB;
        if ( gt_eps( xd1 + r1, 0.0 ) )
        {
            x1 = make_double4( v1.x, v1.y, v1.z, xd1 );
            count++;
        }
        const double  xd2 = ( q / a ) - r1;
        const double3 v2  = mN * xd2 - mB;
        if ( gt_eps( xd2 + r1, 0.0 ) )
        {
            x2 = make_double4( v2.x, v2.y, v2.z, xd2 );
            if ( count == 0 )
                x1 = x2;
            count++;
        }
        return count;
    }

    // The (up to two) spheres tangent to four sites (gpu/math.cuh:703-780). Bit k of the
    // result is set when root k has a non-negative radius; the radius of such a root is
    // re-measured from the first site.
    __device__ __forceinline__ uint32_t quadrisector( const double4 s1, const double4 s2, const double4 s3, const double4 s4,
                                                      double4 & x1, double4 & x2 )
    {
        const double3 p1 = d3( s1 ), p2 = d3( s2 ), p3 = d3( s3 ), p4 = d3( s4 );
        const double  r1 = s1.w, r2 = s2.w, r3 = s3.w, r4 = s4.w;
        const double4 nh1 = s1 - s2, nh2 = s1 - s3, nh3 = s1 - s4;

        const double3 mC = make_double3( .5 * ( -ddot( p1, p1 ) + ddot( p2, p2 ) + r1 * r1 - r2 * r2 ),
                                         .5 * ( -ddot( p1, p1 ) + ddot( p3, p3 ) + r1 * r1 - r3 * r3 ),
                                         .5 * ( -ddot( p1, p1 ) + ddot( p4, p4 ) + r1 * r1 - r4 * r4 ) );
        double3 i1, i2, i3;
        inverse3( make_double3( nh1.x, nh2.x, nh3.x ), make_double3( nh1.y, nh2.y, nh3.y ),
                  make_double3( nh1.z, nh2.z, nh3.z ), i1, i2, i3 );
        const double3 mN = make_double3( 0, 0, 0 ) - mul3( i1, i2, i3, make_double3( nh1.w, nh2.w, nh3.w ) );
        const double3 mB = mul3( i1, i2, i3, mC );

        const double e1 = -mN.x * r1 - mB.x - p1.x;
        const double e2 = -mN.y * r1 - mB.y - p1.y;
        const double e3 = -mN.z * r1 - mB.z - p1.z;
        const double a  = mN.x * mN.x + mN.y * mN.y + mN.z * mN.z - 1.0;
        const double b  = 2.0 * ( mN.x * e1 + mN.y * e2 + mN.z * e3 );
        const double c  = e1 * e1 + e2 * e2 + e3 * e3;

        const double delta = b * b - 4.0 * a * c;
        if ( lt_eps( delta, 0.0 ) )
            return 0;

        const double  q    = -.5 * ( b - sign_eps( b ) * sqrt( delta ) );
        const double  xd1  = ( c / q ) - r1;
        const double3 v1   = mN * xd1 - mB;
        x1                 = make_double4( v1.x, v1.y, v1.z, xd1 );
        uint32_t mask      = gt_eps( xd1 + r1, 0.0 ) ? 1u : 0u;
        if ( gt_eps( xd1 + r1, 0.0 ) )
            x1.w = dlength( p1 - v1 ) - s1.w;

        if ( !near_zero( delta ) )
        {
            const double  xd2 = ( q / a ) - r1;
            const double3 v2  = mN * xd2 - mB;
            x2                = make_double4( v2.x, v2.y, v2.z, xd2 );
            if ( gt_eps( xd2 + r1, 0.0 ) )
                x2.w = dlength( p1 - v2 ) - s1.w;
            mask |= ( gt_eps( xd2 + r1, 0.0 ) ? 1u : 0u ) << 1;
        }
        return mask;
    }

    // Symmetric 2x2 eigen-decomposition, LAPACK dlaev2 scheme (gpu/math.cuh:428-503).
    __device__ __forceinline__ void eigen2( double2 m1, double2 m2, double2 & e, double2 & v )
    {
        const double a = m1.x, b = m2.x, c = m2.y;
        const double sm = a + c, df = a - c, adf = fabs( df ), tb = b + b, ab = fabs( tb );
        double       acmx = a, acmn = c;
        if ( fabs( a ) <= fabs( c ) )
        {
            const double t = acmx;
            acmx           = acmn;
            acmn           = t;
        }
        double aa = ab, bb = adf;
        if ( adf < ab )
        {
            aa = adf;
            bb = ab;
        }
        const double temp = aa / bb;
        const double rt   = bb * fsqrtd( 1.0 + temp * temp );
        const double sgn1 = copysign( 1.0, sm );
        const double rt1  = .5 * ( sm + sgn1 * rt );
        const double rt2  = ( acmx / rt1 ) * acmn - ( b / rt1 ) * b;

        const double sgn2 = copysign( 1.0, df );
        const double cs   = df + sgn2 * rt;
        const double acs  = fabs( cs );
        aa                = tb;
        bb                = cs;
        const bool swapped = lt_eps( acs, ab );
        if ( swapped )
        {
            aa = cs;
            bb = tb;
        }
        const double t   = -aa / bb;
        double       sn1 = 1.0 / fsqrtd( 1.0 + t * t );
        double       cs1 = t * sn1;
        if ( swapped )
        {
            const double x = sn1;
            sn1            = cs1;
            cs1            = x;
        }
        if ( swapped && near_zero( ab ) )
        {
            cs1 = 1.0;
            sn1 = 0.0;
        }
        if ( fabs( sgn1 - sgn2 ) <= ( 1e-5 + 1e-8 * fabs( sgn2 ) ) )
        {
            const double tn = cs1;
            cs1             = -sn1;
            sn1             = tn;
        }
        e = make_double2( rt2, rt1 );
        v = make_double2( -sn1, cs1 );
    }

    // gpu/math.cuh:519-531
    __device__ __forceinline__ double det4( double4 c1, double4 c2, double4 c3, double4 c4 )
    {
        const double d1 = ddot( make_double3( c2.y, c2.z, c2.w ), dcross( make_double3( c3.y, c3.z, c3.w ), make_double3( c4.y, c4.z, c4.w ) ) );
        const double d2 = ddot( make_double3( c2.x, c2.z, c2.w ), dcross( make_double3( c3.x, c3.z, c3.w ), make_double3( c4.x, c4.z, c4.w ) ) );
        const double d3v = ddot( make_double3( c2.x, c2.y, c2.w ), dcross( make_double3( c3.x, c3.y, c3.w ), make_double3( c4.x, c4.y, c4.w ) ) );
        const double d4 = ddot( make_double3( c2.x, c2.y, c2.z ), dcross( make_double3( c3.x, c3.y, c3.z ), make_double3( c4.x, c4.y, c4.z ) ) );
        return c1.x * d1 - c1.y * d2 + c1.z * d3v - c1.w * d4;
    }

    // Sphere through four points (gpu/math.cuh:533-575).
    __device__ __forceinline__ double4 sphere_from_points( double3 p1, double3 p2, double3 p3, double3 p4 )
    {
        const double  t1 = -ddot( p1, p1 ), t2 = -ddot( p2, p2 ), t3 = -ddot( p3, p3 ), t4 = -ddot( p4, p4 );
        const double4 X = make_double4( p1.x, p2.x, p3.x, p4.x ), Y = make_double4( p1.y, p2.y, p3.y, p4.y );
        const double4 Z = make_double4( p1.z, p2.z, p3.z, p4.z ), O = make_double4( 1, 1, 1, 1 );
        const double4 T = make_double4( t1, t2, t3, t4 );
        const double  t = det4( X, Y, Z, O );
        const double  d = det4( T, Y, Z, O ) / t;
        const double  e = det4( X, T, Z, O ) / t;
        const double  f = det4( X, Y, T, O ) / t;
        const double  g = det4( X, Y, Z, T ) / t;
        return make_double4( -d * .5, -e * .5, -f * .5, .5 * sqrt( d * d + e * e + f * f - 4. * g ) );
    }

    // Normals of the two planes tangent to three spheres (gpu/math.cuh:577-634), with the
    // 2x2 helpers of gpu/math.cuh:390-417.
    __device__ __forceinline__ void tangent_planes( const double4 s1, const double4 s2, const double4 s3, double3 & n1, double3 & n2 )
    {
        const double3 p1 = d3( s1 ), p2 = d3( s2 ), p3 = d3( s3 );
        const double4 nh1 = s1 - s2, nh2 = s1 - s3;
        const double2 aC1 = make_double2( nh1.x, nh2.x ), aC2 = make_double2( nh1.y, nh2.y );
        const double2 bC1 = make_double2( nh1.z, nh2.z ), bC2 = make_double2( nh1.w, nh2.w );

        const double  inv = 1.0 / fma( aC1.x, aC2.y, -aC2.x * aC1.y );
        const double2 iA1 = make_double2( inv * aC2.y, -inv * aC1.y );
        const double2 iA2 = make_double2( -inv * aC2.x, inv * aC1.x );

        const double2 cC1 = make_double2( iA1.x * bC1.x + iA2.x * bC1.y, iA1.y * bC1.x + iA2.y * bC1.y );
        const double2 cC2 = make_double2( iA1.x * bC2.x + iA2.x * bC2.y, iA1.y * bC2.x + iA2.y * bC2.y );

        const double2 eC1 = make_double2( 1.0 + cC1.x * cC1.x + cC1.y * cC1.y, 0.0 + cC1.x * cC2.x + cC1.y * cC2.y );
        const double2 eC2 = make_double2( 0.0 + cC1.x * cC2.x + cC1.y * cC2.y, -1.0 + cC2.x * cC2.x + cC2.y * cC2.y );
        double2       ev, evec;
        eigen2( eC1, eC2, ev, evec );
        const double alpha0 = sqrt( fabs( ev.x ) );
        const double alpha1 = sqrt( fabs( ev.y ) );

        double2 z   = make_double2( 1, alpha0 / alpha1 );
        double2 y34 = make_double2( ddot( make_double2( evec.x, -evec.y ), z ), ddot( make_double2( evec.y, evec.x ), z ) );
        double  x1  = -ddot( make_double2( cC1.x, cC2.x ), y34 );
        double  x2  = -ddot( make_double2( cC1.y, cC2.y ), y34 );
        n1          = dnormalize( make_double3( x1, x2, y34.x ) );

        z   = make_double2( 1, -alpha0 / alpha1 );
        y34 = make_double2( ddot( make_double2( evec.x, -evec.y ), z ), ddot( make_double2( evec.y, evec.x ), z ) );
        x1  = -ddot( make_double2( cC1.x, cC2.x ), y34 );
        x2  = -ddot( make_double2( cC1.y, cC2.y ), y34 );
        n2  = dnormalize( make_double3( x1, x2, y34.x ) );

        const double3 p = p1 + n1 * s1.w;
        if ( gt_eps( fabs( ddot( n1, p - p1 ) - s1.w ), 1e-4 ) || gt_eps( fabs( ddot( n1, p - p2 ) - s2.w ), 1e-4 )
             || gt_eps( fabs( ddot( n1, p - p3 ) - s3.w ), 1e-4 ) )
        {
            n1.x *= -1.0;
            n1.y *= -1.0;
            n1.z *= -1.0;
            n2.x *= -1.0;
            n2.y *= -1.0;
            n2.z *= -1.0;
        }
    }
} // namespace apo2
