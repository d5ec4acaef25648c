// Learned k-proposal: a 16 -> 64 -> 64 -> 1 network (ReLU, bf16 weights, fp32 accumulation)
// that predicts, from a site's radius, its Morton-local density and its nearest neighbours,
// the kNN rank at which the site's cell will pass the security-radius certificate.
//
// The reference has no such network; its measurement harness records, per kNN rank, whether a
// neighbour contributed and whether the certificate held
// (app/benchmarks/benchmark_contributing_nearest.cu:10-129), which gives the training labels.
#pragma once

#include <cuda_bf16.h>

#include "../../include/apo2.h"
#include "internal.cuh"

namespace apo2
{
    constexpr uint32_t kPIn     = APO2_PROPOSAL_INPUTS; // 16
    constexpr uint32_t kPHid    = APO2_PROPOSAL_HIDDEN; // 64
    constexpr uint32_t kPParams = kPHid * kPIn + kPHid + kPHid * kPHid + kPHid + kPHid + 1; // 5,313

    // Offsets of the parameter vector (fp32 master copy): W1 (64 x 16), b1, W2 (64 x 64), b2, w3, b3.
    constexpr uint32_t kOffW1 = 0;
    constexpr uint32_t kOffB1 = kOffW1 + kPHid * kPIn;
    constexpr uint32_t kOffW2 = kOffB1 + kPHid;
    constexpr uint32_t kOffB2 = kOffW2 + kPHid * kPHid;
    constexpr uint32_t kOffW3 = kOffB2 + kPHid;
    constexpr uint32_t kOffB3 = kOffW3 + kPHid;

    // The network as inference reads it (device copy of apo2_proposal).
    struct ProposalNet
    {
        float          mean[ kPIn ], inv_scale[ kPIn ];
        float          margin, b3;
        float          b1[ kPHid ], b2[ kPHid ];
        __nv_bfloat16 w1[ kPHid * kPIn ];
        __nv_bfloat16 w2[ kPHid * kPHid ];
        __nv_bfloat16 w3[ kPHid ];
    };
    // ProposalNet is apo2_proposal without its three leading words
    constexpr size_t kProposalHeader = 3 * sizeof( uint32_t );
    static_assert( sizeof( ProposalNet ) == sizeof( apo2_proposal ) - kProposalHeader, "layout of apo2_proposal" );

    // Feature vector of site i (sorted order) from its sorted kNN list; see proposal.cu.
    struct FeatureInputs
    {
        const float4 *   sites_f = nullptr; // n, sorted
        const uint64_t * codes   = nullptr; // n, sorted Morton codes
        const Scene *    scene   = nullptr;
        uint32_t         n       = 0;
    };

    void launch_features( const FeatureInputs & in, const uint32_t * knn, uint32_t k, float * out, cudaStream_t s );

    // Predicted log2 rank; the proposed rank is ceil(2^(prediction + margin)) clamped to [1, max_rank].
    __device__ __forceinline__ uint32_t proposal_rank( const ProposalNet & net, float prediction, uint32_t max_rank )
    {
        const float r = ceilf( exp2f( fminf( prediction + net.margin, 30.f ) ) );
        return r < 1.f ? 1u : ( r >= float( max_rank ) ? max_rank : uint32_t( r ) );
    }
    // -----------------------------------------------------------------------------------
    // Features and inference
    // -----------------------------------------------------------------------------------
    __device__ __forceinline__ void proposal_features( const FeatureInputs & in, uint32_t i, const uint32_t * nbr, uint32_t stride,
                                       uint32_t count, float out[ kPIn ] )
    {
        const float4 si = in.sites_f[ i ];
        uint32_t     m  = 0;
        float        lam = 0.f;
        for ( uint32_t q = 0; q < min( count, 8u ); q++ )
        {
            const uint32_t j = nbr[ q * stride ];
            if ( j >= in.n )
                break;
            const float4 sj = in.sites_f[ j ];
            const float  dx = sj.x - si.x, dy = sj.y - si.y, dz = sj.z - si.z;
            lam += sqrtf( dx * dx + dy * dy + dz * dz );
            m++;
        }
        lam = m ? lam / float( m ) : fmaxf( si.w, 1e-3f );
        lam = fmaxf( lam, 1e-6f );
        const float ri = fmaxf( si.w, 1e-12f );
        out[ 0 ]       = log2f( ri / lam );

        // Morton-local density: sites per volume of the smallest aligned cube holding positions
        // i-16 .. i+16 of the Morton order
        const uint32_t a = i >= 16 ? i - 16 : 0, b = min( in.n - 1, i + 16 );
        const uint64_t x = in.codes[ a ] ^ in.codes[ b ];
        const int      level = x ? ( 63 - __clzll( x ) ) / 3 + 1 : 0;
        float          log_extent = 0.f;
        for ( int c = 0; c < 3; c++ )
            log_extent -= log2f( fmaxf( in.scene->scale[ c ], 1e-30f ) ); // extent = 1 / scale
        const float log_volume = 3.f * float( level ) + log_extent - 3.f * log2f( 1048575.f );
        out[ 1 ]               = log2f( float( b - a + 1 ) ) + 3.f * log2f( lam ) - log_volume;

        for ( uint32_t q = 0; q < 7; q++ )
        {
            float rr = 0.f, dd = 4.f;
            if ( q < m )
            {
                const uint32_t j  = nbr[ q * stride ];
                const float4   sj = in.sites_f[ j ];
                const float    dx = sj.x - si.x, dy = sj.y - si.y, dz = sj.z - si.z;
                rr                = log2f( fmaxf( sj.w, 1e-12f ) / ri );
                dd                = ( sqrtf( dx * dx + dy * dy + dz * dz ) - si.w - sj.w ) / lam;
            }
            out[ 2 + q ] = rr;
            out[ 9 + q ] = dd;
        }
    }

    __device__ __forceinline__ float proposal_predict( const ProposalNet & net, const float x[ kPIn ] )
    {
        float xn[ kPIn ];
#pragma unroll
        for ( uint32_t k = 0; k < kPIn; k++ )
            xn[ k ] = ( x[ k ] - net.mean[ k ] ) * net.inv_scale[ k ];
        float h1[ kPHid ];
#pragma unroll
        for ( uint32_t j = 0; j < kPHid; j++ )
        {
            float                  acc = net.b1[ j ];
            const __nv_bfloat162 * w   = reinterpret_cast<const __nv_bfloat162 *>( net.w1 + j * kPIn );
#pragma unroll
            for ( uint32_t k = 0; k < kPIn / 2; k++ )
            {
                const float2 wf = __bfloat1622float2( w[ k ] );
                acc             = fmaf( wf.x, xn[ 2 * k ], acc );
                acc             = fmaf( wf.y, xn[ 2 * k + 1 ], acc );
            }
            h1[ j ] = fmaxf( acc, 0.f );
        }
        float out = net.b3;
        for ( uint32_t j = 0; j < kPHid; j++ )
        {
            float                  acc = net.b2[ j ];
            const __nv_bfloat162 * w   = reinterpret_cast<const __nv_bfloat162 *>( net.w2 + j * kPHid );
#pragma unroll
            for ( uint32_t k = 0; k < kPHid / 2; k++ )
            {
                const float2 wf = __bfloat1622float2( w[ k ] );
                acc             = fmaf( wf.x, h1[ 2 * k ], acc );
                acc             = fmaf( wf.y, h1[ 2 * k + 1 ], acc );
            }
            out = fmaf( __bfloat162float( net.w3[ j ] ), fmaxf( acc, 0.f ), out );
        }
        return out;
    }

} // namespace apo2
