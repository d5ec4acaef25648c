// Peak non-tensor floating-point throughput of the current GPU, measured: the denominators of
// the build's compute roofline. The build's arithmetic is scalar FP64 (vertex solves and
// predicates) and FP32 (traversal, filters), issued by the FMA pipes, not the tensor cores, so
// a GEMM through a library (which may run on the tensor pipe) is the wrong peak for it.
//
// Each thread runs kChains independent fused multiply-add chains for kIters steps (enough
// independent work per warp to cover the pipe latency at full occupancy); the grid fills every
// SM several times over. FLOPs = 2 per FMA.
#include <algorithm>

#include <cuda_runtime.h>

#include "../../include/apo2.h"

namespace apo2
{
    namespace
    {
        constexpr int kChains  = 8;
        constexpr int kIters   = 4096;
        constexpr int kThreads = 256;

        template<class T>
        __global__ void __launch_bounds__( kThreads ) k_fma_peak( T * out, T seed )
        {
            T acc[ kChains ];
#pragma unroll
            for ( int c = 0; c < kChains; c++ )
                acc[ c ] = seed + T( threadIdx.x + c );
            const T a = T( 0.999999 ), b = T( 1e-7 );
#pragma unroll 4
            for ( int it = 0; it < kIters; it++ )
            {
#pragma unroll
                for ( int c = 0; c < kChains; c++ )
                    acc[ c ] = fma( acc[ c ], a, b );
            }
            T s = T( 0 );
#pragma unroll
            for ( int c = 0; c < kChains; c++ )
                s += acc[ c ];
            if ( s == T( -1 ) ) // never true; keeps the chains live
                out[ blockIdx.x ] = s;
        }

        template<class T>
        double measure( int blocks )
        {
            T * out = nullptr;
            if ( cudaMalloc( &out, sizeof( T ) * blocks ) != cudaSuccess )
                return 0.0;
            cudaEvent_t e0, e1;
            cudaEventCreate( &e0 );
            cudaEventCreate( &e1 );
            k_fma_peak<T><<<blocks, kThreads>>>( out, T( 1 ) ); // warm-up
            float best = 1e30f;
            for ( int r = 0; r < 5; r++ )
            {
                cudaEventRecord( e0 );
                k_fma_peak<T><<<blocks, kThreads>>>( out, T( r ) );
                cudaEventRecord( e1 );
                cudaEventSynchronize( e1 );
                float ms = 0.f;
                cudaEventElapsedTime( &ms, e0, e1 );
                best = std::min( best, ms );
            }
            cudaEventDestroy( e0 );
            cudaEventDestroy( e1 );
            cudaFree( out );
            const double flops = 2.0 * kChains * double( kIters ) * kThreads * double( blocks );
            return cudaGetLastError() == cudaSuccess ? flops / ( double( best ) * 1e-3 ) / 1e12 : 0.0;
        }
    } // namespace
} // namespace apo2

extern "C" apo2_status apo2_fma_peak( double * fp64_tflops, double * fp32_tflops )
{
    if ( !fp64_tflops || !fp32_tflops )
        return APO2_ERR_INVALID_ARG;
    int dev = 0, sms = 148;
    if ( cudaGetDevice( &dev ) != cudaSuccess )
        return APO2_ERR_CUDA;
    cudaDeviceGetAttribute( &sms, cudaDevAttrMultiProcessorCount, dev );
    const int blocks = sms * 8 * 4; // 8 resident blocks of 256 per SM, four waves
    *fp64_tflops     = apo2::measure<double>( blocks );
    *fp32_tflops     = apo2::measure<float>( blocks );
    return ( *fp64_tflops > 0.0 && *fp32_tflops > 0.0 ) ? APO2_OK : APO2_ERR_CUDA;
}
