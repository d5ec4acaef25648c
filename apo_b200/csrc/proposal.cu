// Learned k-proposal: features, inference, and the training kernels (forward, backward, Adam).
//
// Features of site i (sorted order), all dimensionless, from its kNN list sorted by sphere
// distance (lambda = mean centre distance of the first eight neighbours):
//   x0      log2(r_i / lambda)
//   x1      log2 of the Morton-local density times lambda^3: the 33 sites at sorted positions
//           i-16 .. i+16 all lie in the smallest aligned Morton cube holding the codes at both
//           ends (every code between two codes shares their common prefix)
//   x2..x8  log2(r_j / r_i) of neighbours 1..7
//   x9..x15 sphere distance |c_i - c_j| - r_i - r_j of neighbours 1..7, over lambda
// A list shorter than eight fills the missing entries with 0 and 4 (far).
//
// Training (apo2_proposal_train): mean squared error on log2 of the certified rank, Adam on an
// fp32 master copy of the parameters; the forward pass always uses the master rounded to bf16,
// exactly the weights inference reads. Per batch:
//   k_train_forward   thread per sample: activations, output error, the two hidden-layer deltas
//   k_train_grads     block per (parameter row, batch chunk): partial sums in a fixed order
//   k_train_reduce    sums the chunks in a fixed order (reproducible gradients), the loss
//   k_train_adam      the Adam step on the master copy
#include <algorithm>
#include <cstring>
#include <numeric>
#include <random>
#include <vector>

#include "proposal.cuh"

namespace apo2
{
    namespace
    {
        // Features of every site of a built handle (sorted order).
        __global__ void k_features( FeatureInputs in, const uint32_t * __restrict__ knn, uint32_t k, float * __restrict__ out )
        {
            const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
            if ( i >= in.n )
                return;
            float f[ kPIn ];
            proposal_features( in, i, knn + size_t( i ) * k, 1, k, f );
            for ( uint32_t q = 0; q < kPIn; q++ )
                out[ size_t( i ) * kPIn + q ] = f[ q ];
        }

        __global__ void k_predict( const ProposalNet * __restrict__ net, const float * __restrict__ x, uint64_t n,
                                   float * __restrict__ out )
        {
            __shared__ ProposalNet s;
            for ( uint32_t w = threadIdx.x; w < sizeof( ProposalNet ) / 4; w += blockDim.x )
                reinterpret_cast<uint32_t *>( &s )[ w ] = reinterpret_cast<const uint32_t *>( net )[ w ];
            __syncthreads();
            const uint64_t i = blockIdx.x * uint64_t( blockDim.x ) + threadIdx.x;
            if ( i >= n )
                return;
            float f[ kPIn ];
            for ( uint32_t q = 0; q < kPIn; q++ )
                f[ q ] = x[ i * kPIn + q ];
            out[ i ] = proposal_predict( s, f );
        }

        // -------------------------------------------------------------------------------
        // Training
        // -------------------------------------------------------------------------------
        constexpr uint32_t kTrainBlock = 128;
        constexpr uint32_t kChunk      = 512; // samples per partial sum of the weight gradients

        __device__ __forceinline__ float bf16_of( float v ) { return __bfloat162float( __float2bfloat16_rn( v ) ); }

        // Per-sample rows kept between the kernels of one batch.
        struct TrainRows
        {
            float * xn;  // batch x 16 (normalised inputs)
            float * h1;  // batch x 64
            float * h2;  // batch x 64
            float * d1;  // batch x 64 (delta of layer 1)
            float * d2;  // batch x 64 (delta of layer 2)
            float * g;   // batch (delta of the output)
            float * sq;  // batch (squared error)
        };

        __global__ void __launch_bounds__( kTrainBlock ) k_train_forward( const float * __restrict__ master, const float * __restrict__ mean,
                                                                          const float * __restrict__ inv_scale, const float * __restrict__ x,
                                                                          const float * __restrict__ y, const uint32_t * __restrict__ order,
                                                                          uint64_t first, uint32_t batch, float inv_batch, TrainRows rows )
        {
            __shared__ float w1[ kPHid * kPIn ], b1[ kPHid ], w2[ kPHid * kPHid ], b2[ kPHid ], w3[ kPHid ], b3;
            for ( uint32_t t = threadIdx.x; t < kPHid * kPHid; t += blockDim.x )
            {
                w2[ t ] = bf16_of( master[ kOffW2 + t ] );
                if ( t < kPHid * kPIn )
                    w1[ t ] = bf16_of( master[ kOffW1 + t ] );
                if ( t < kPHid )
                {
                    b1[ t ] = master[ kOffB1 + t ];
                    b2[ t ] = master[ kOffB2 + t ];
                    w3[ t ] = bf16_of( master[ kOffW3 + t ] );
                }
            }
            if ( threadIdx.x == 0 )
                b3 = master[ kOffB3 ];
            __syncthreads();
            const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
            if ( b >= batch )
                return;
            const uint64_t src = order ? order[ first + b ] : first + b;
            float          xn[ kPIn ];
            for ( uint32_t k = 0; k < kPIn; k++ )
            {
                xn[ k ]                      = ( x[ src * kPIn + k ] - mean[ k ] ) * inv_scale[ k ];
                rows.xn[ size_t( b ) * kPIn + k ] = xn[ k ];
            }
            float h1[ kPHid ];
            for ( uint32_t j = 0; j < kPHid; j++ )
            {
                float acc = b1[ j ];
                for ( uint32_t k = 0; k < kPIn; k++ )
                    acc = fmaf( w1[ j * kPIn + k ], xn[ k ], acc );
                h1[ j ]                            = fmaxf( acc, 0.f );
                rows.h1[ size_t( b ) * kPHid + j ] = h1[ j ];
            }
            float o = b3;
            for ( uint32_t j = 0; j < kPHid; j++ )
            {
                float acc = b2[ j ];
                for ( uint32_t k = 0; k < kPHid; k++ )
                    acc = fmaf( w2[ j * kPHid + k ], h1[ k ], acc );
                const float h = fmaxf( acc, 0.f );
                rows.h2[ size_t( b ) * kPHid + j ] = h;
                o                                  = fmaf( w3[ j ], h, o );
            }
            const float r = o - y[ src ];
            const float g = 2.f * r * inv_batch;
            rows.g[ b ]   = g;
            rows.sq[ b ]  = r * r;
            // delta of layer 2, then of layer 1 (W2^T delta2, masked by the ReLU of layer 1)
            float d1[ kPHid ];
            for ( uint32_t k = 0; k < kPHid; k++ )
                d1[ k ] = 0.f;
            for ( uint32_t j = 0; j < kPHid; j++ )
            {
                const float d2 = rows.h2[ size_t( b ) * kPHid + j ] > 0.f ? g * w3[ j ] : 0.f;
                rows.d2[ size_t( b ) * kPHid + j ] = d2;
                if ( d2 != 0.f )
                    for ( uint32_t k = 0; k < kPHid; k++ )
                        d1[ k ] = fmaf( w2[ j * kPHid + k ], d2, d1[ k ] );
            }
            for ( uint32_t k = 0; k < kPHid; k++ )
                rows.d1[ size_t( b ) * kPHid + k ] = h1[ k ] > 0.f ? d1[ k ] : 0.f;
        }

        // Partial weight gradients of one chunk of the batch. Block (row, chunk): row r < 64 is
        // row r of W1 and b1 (threads 0..15 the weights, thread 16 the bias); row 64 + r is row r
        // of W2 and b2 (threads 0..63, thread 64 the bias); row 128 is w3 and b3.
        __global__ void k_train_grads( TrainRows rows, uint32_t batch, float * __restrict__ partial )
        {
            const uint32_t row = blockIdx.x, chunk = blockIdx.y, t = threadIdx.x;
            const uint32_t b0 = chunk * kChunk, b1 = min( batch, b0 + kChunk );
            float *        out = partial + size_t( chunk ) * kPParams;
            float          acc = 0.f;
            if ( row < kPHid )
            {
                if ( t > kPIn )
                    return;
                for ( uint32_t b = b0; b < b1; b++ )
                {
                    const float d = rows.d1[ size_t( b ) * kPHid + row ];
                    acc           = fmaf( d, t < kPIn ? rows.xn[ size_t( b ) * kPIn + t ] : 1.f, acc );
                }
                out[ t < kPIn ? kOffW1 + row * kPIn + t : kOffB1 + row ] = acc;
            }
            else if ( row < 2 * kPHid )
            {
                const uint32_t r = row - kPHid;
                if ( t > kPHid )
                    return;
                for ( uint32_t b = b0; b < b1; b++ )
                {
                    const float d = rows.d2[ size_t( b ) * kPHid + r ];
                    acc           = fmaf( d, t < kPHid ? rows.h1[ size_t( b ) * kPHid + t ] : 1.f, acc );
                }
                out[ t < kPHid ? kOffW2 + r * kPHid + t : kOffB2 + r ] = acc;
            }
            else
            {
                if ( t > kPHid )
                    return;
                for ( uint32_t b = b0; b < b1; b++ )
                {
                    const float g = rows.g[ b ];
                    acc           = fmaf( g, t < kPHid ? rows.h2[ size_t( b ) * kPHid + t ] : 1.f, acc );
                }
                out[ t < kPHid ? kOffW3 + t : kOffB3 ] = acc;
            }
        }

        // Sums the chunks (fixed order) into grads; thread 0 of block 0 also sums the loss.
        __global__ void k_train_reduce( const float * __restrict__ partial, uint32_t chunks, float * __restrict__ grads,
                                        const float * __restrict__ sq, uint32_t batch, double * __restrict__ loss_sum )
        {
            const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
            if ( p < kPParams )
            {
                float s = 0.f;
                for ( uint32_t c = 0; c < chunks; c++ )
                    s += partial[ size_t( c ) * kPParams + p ];
                grads[ p ] = s;
            }
            if ( p == 0 && loss_sum )
            {
                double s = 0.0;
                for ( uint32_t b = 0; b < batch; b++ )
                    s += sq[ b ];
                *loss_sum += s;
            }
        }

        __global__ void k_train_adam( float * __restrict__ master, float * __restrict__ m, float * __restrict__ v,
                                      const float * __restrict__ grads, float lr, float c1, float c2 )
        {
            const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
            if ( p >= kPParams )
                return;
            const float g  = grads[ p ];
            const float mm = 0.9f * m[ p ] + 0.1f * g;
            const float vv = 0.999f * v[ p ] + 0.001f * g * g;
            m[ p ]         = mm;
            v[ p ]         = vv;
            master[ p ] -= lr * ( mm * c1 ) / ( sqrtf( vv * c2 ) + 1e-8f );
        }

        struct TrainScratch
        {
            void *    base = nullptr;
            TrainRows rows {};
            float *   master = nullptr, *m = nullptr, *v = nullptr, *grads = nullptr, *partial = nullptr;
            float *   mean = nullptr, *inv_scale = nullptr;
            double *  loss = nullptr;
            uint32_t  batch = 0, chunks = 0;

            bool allocate( uint32_t b )
            {
                batch  = b;
                chunks = ( b + kChunk - 1 ) / kChunk;
                const size_t floats = size_t( b ) * ( kPIn + 4 * kPHid + 2 ) + 4 * size_t( kPParams )
                                      + size_t( chunks ) * kPParams + 2 * kPIn;
                if ( cudaMalloc( &base, floats * sizeof( float ) + 64 ) != cudaSuccess )
                    return false;
                float * p = static_cast<float *>( base );
                loss      = reinterpret_cast<double *>( p );
                p += 16;
                rows.xn = p;
                p += size_t( b ) * kPIn;
                rows.h1 = p;
                p += size_t( b ) * kPHid;
                rows.h2 = p;
                p += size_t( b ) * kPHid;
                rows.d1 = p;
                p += size_t( b ) * kPHid;
                rows.d2 = p;
                p += size_t( b ) * kPHid;
                rows.g = p;
                p += b;
                rows.sq = p;
                p += b;
                master = p;
                p += kPParams;
                m = p;
                p += kPParams;
                v = p;
                p += kPParams;
                grads = p;
                p += kPParams;
                partial = p;
                p += size_t( chunks ) * kPParams;
                mean = p;
                p += kPIn;
                inv_scale = p;
                return true;
            }
            ~TrainScratch()
            {
                if ( base )
                    cudaFree( base );
            }
        };

        // One forward/backward over samples [first, first + count) of (x, y) (through `order`
        // when given); gradients land in s.grads, the squared errors are added to *s.loss.
        void batch_gradients( TrainScratch & s, const float * x, const float * y, const uint32_t * order, uint64_t first,
                              uint32_t count, float inv_batch, cudaStream_t st )
        {
            APO2_LAUNCH( "k_train_forward", st,
                         k_train_forward<<<( count + kTrainBlock - 1 ) / kTrainBlock, kTrainBlock, 0, st>>>(
                             s.master, s.mean, s.inv_scale, x, y, order, first, count, inv_batch, s.rows ) );
            const uint32_t chunks = ( count + kChunk - 1 ) / kChunk;
            APO2_LAUNCH( "k_train_grads", st, k_train_grads<<<dim3( 2 * kPHid + 1, chunks ), kPHid + 1, 0, st>>>( s.rows, count, s.partial ) );
            APO2_LAUNCH( "k_train_reduce", st,
                         k_train_reduce<<<( kPParams + 255 ) / 256, 256, 0, st>>>( s.partial, chunks, s.grads, s.rows.sq, count, s.loss ) );
        }

        uint16_t bf16_bits( float v )
        {
            uint32_t u;
            std::memcpy( &u, &v, 4 );
            if ( ( u & 0x7fffffffu ) > 0x7f800000u )
                return uint16_t( ( u >> 16 ) | 0x40u ); // NaN stays NaN
            u += 0x7fffu + ( ( u >> 16 ) & 1u );
            return uint16_t( u >> 16 );
        }
    } // namespace

    // Model <-> parameter vector.
    void proposal_from_master( const float * master, apo2_proposal & m )
    {
        for ( uint32_t t = 0; t < kPHid * kPIn; t++ )
            m.w1[ t ] = bf16_bits( master[ kOffW1 + t ] );
        for ( uint32_t t = 0; t < kPHid * kPHid; t++ )
            m.w2[ t ] = bf16_bits( master[ kOffW2 + t ] );
        for ( uint32_t t = 0; t < kPHid; t++ )
        {
            m.w3[ t ] = bf16_bits( master[ kOffW3 + t ] );
            m.b1[ t ] = master[ kOffB1 + t ];
            m.b2[ t ] = master[ kOffB2 + t ];
        }
        m.b3 = master[ kOffB3 ];
    }

    void launch_features( const FeatureInputs & in, const uint32_t * knn, uint32_t k, float * out, cudaStream_t s )
    {
        APO2_LAUNCH( "k_features", s, k_features<<<( in.n + 255 ) / 256, 256, 0, s>>>( in, knn, k, out ) );
    }
} // namespace apo2

using namespace apo2;

extern "C" apo2_status apo2_proposal_predict( const apo2_proposal * model, const float * features, uint64_t n, float * out )
{
    if ( !model || !features || !out || model->struct_size != sizeof( apo2_proposal ) )
        return APO2_ERR_INVALID_ARG;
    if ( n == 0 )
        return APO2_OK;
    void * base = nullptr;
    const size_t bytes = sizeof( ProposalNet ) + 256 + sizeof( float ) * n * ( kPIn + 1 );
    if ( cudaMalloc( &base, bytes ) != cudaSuccess )
        return APO2_ERR_OUT_OF_MEMORY;
    char *        p   = static_cast<char *>( base );
    ProposalNet * net = reinterpret_cast<ProposalNet *>( p );
    float *       x   = reinterpret_cast<float *>( p + ( ( sizeof( ProposalNet ) + 255 ) & ~size_t( 255 ) ) );
    float *       o   = x + n * kPIn;
    cudaError_t   e   = cudaMemcpy( net, reinterpret_cast<const char *>( model ) + kProposalHeader, sizeof( ProposalNet ),
                                    cudaMemcpyHostToDevice );
    if ( e == cudaSuccess )
        e = cudaMemcpy( x, features, sizeof( float ) * n * kPIn, cudaMemcpyHostToDevice );
    if ( e == cudaSuccess )
    {
        APO2_LAUNCH( "k_predict", 0, k_predict<<<unsigned( ( n + 127 ) / 128 ), 128>>>( net, x, n, o ) );
        e = cudaGetLastError();
    }
    if ( e == cudaSuccess )
        e = cudaMemcpy( out, o, sizeof( float ) * n, cudaMemcpyDeviceToHost );
    cudaFree( base );
    return e == cudaSuccess ? APO2_OK : APO2_ERR_CUDA;
}

extern "C" apo2_status apo2_proposal_gradients( const apo2_proposal * model, const float * master, const float * features,
                                                const float * targets, uint32_t n, float * loss, float * grads )
{
    if ( !model || !master || !features || !targets || !grads || n == 0 || model->struct_size != sizeof( apo2_proposal ) )
        return APO2_ERR_INVALID_ARG;
    TrainScratch s;
    if ( !s.allocate( n ) )
        return APO2_ERR_OUT_OF_MEMORY;
    float * x = nullptr;
    if ( cudaMalloc( &x, sizeof( float ) * size_t( n ) * ( kPIn + 1 ) ) != cudaSuccess )
        return APO2_ERR_OUT_OF_MEMORY;
    float *     y = x + size_t( n ) * kPIn;
    cudaError_t e = cudaMemcpy( x, features, sizeof( float ) * size_t( n ) * kPIn, cudaMemcpyHostToDevice );
    if ( e == cudaSuccess )
        e = cudaMemcpy( y, targets, sizeof( float ) * n, cudaMemcpyHostToDevice );
    if ( e == cudaSuccess )
        e = cudaMemcpy( s.master, master, sizeof( float ) * kPParams, cudaMemcpyHostToDevice );
    if ( e == cudaSuccess )
        e = cudaMemcpy( s.mean, model->mean, sizeof( float ) * kPIn, cudaMemcpyHostToDevice );
    if ( e == cudaSuccess )
        e = cudaMemcpy( s.inv_scale, model->inv_scale, sizeof( float ) * kPIn, cudaMemcpyHostToDevice );
    if ( e == cudaSuccess )
        e = cudaMemset( s.loss, 0, sizeof( double ) );
    if ( e == cudaSuccess )
    {
        batch_gradients( s, x, y, nullptr, 0, n, 1.f / float( n ), 0 );
        e = cudaGetLastError();
    }
    double l = 0.0;
    if ( e == cudaSuccess )
        e = cudaMemcpy( grads, s.grads, sizeof( float ) * kPParams, cudaMemcpyDeviceToHost );
    if ( e == cudaSuccess )
        e = cudaMemcpy( &l, s.loss, sizeof( double ), cudaMemcpyDeviceToHost );
    cudaFree( x );
    if ( loss )
        *loss = float( l / n );
    return e == cudaSuccess ? APO2_OK : APO2_ERR_CUDA;
}

extern "C" apo2_status apo2_proposal_train( const float * features, const float * targets, uint64_t n, uint32_t epochs,
                                            uint32_t batch, float learning_rate, uint64_t seed, float * master,
                                            apo2_proposal * model, float * epoch_loss )
{
    if ( !features || !targets || !master || !model || n == 0 || batch == 0 || epochs == 0
         || model->struct_size != sizeof( apo2_proposal ) || n > ( 1ull << 31 ) )
        return APO2_ERR_INVALID_ARG;
    batch = uint32_t( std::min<uint64_t>( batch, n ) );
    TrainScratch s;
    if ( !s.allocate( batch ) )
        return APO2_ERR_OUT_OF_MEMORY;
    float * x = nullptr;
    if ( cudaMalloc( &x, sizeof( float ) * n * ( kPIn + 1 ) + sizeof( uint32_t ) * n ) != cudaSuccess )
        return APO2_ERR_OUT_OF_MEMORY;
    float *     y     = x + n * kPIn;
    uint32_t *  order = reinterpret_cast<uint32_t *>( y + n );
    cudaError_t e     = cudaMemcpy( x, features, sizeof( float ) * n * kPIn, cudaMemcpyHostToDevice );
    if ( e == cudaSuccess )
        e = cudaMemcpy( y, targets, sizeof( float ) * n, cudaMemcpyHostToDevice );
    if ( e == cudaSuccess )
        e = cudaMemcpy( s.master, master, sizeof( float ) * kPParams, cudaMemcpyHostToDevice );
    if ( e == cudaSuccess )
        e = cudaMemcpy( s.mean, model->mean, sizeof( float ) * kPIn, cudaMemcpyHostToDevice );
    if ( e == cudaSuccess )
        e = cudaMemcpy( s.inv_scale, model->inv_scale, sizeof( float ) * kPIn, cudaMemcpyHostToDevice );
    if ( e == cudaSuccess )
        e = cudaMemset( s.m, 0, sizeof( float ) * 2 * kPParams ); // m and v are adjacent
    std::vector<uint32_t> perm( n );
    std::iota( perm.begin(), perm.end(), 0u );
    std::mt19937_64 rng( seed );
    uint64_t        step = 0;
    for ( uint32_t ep = 0; ep < epochs && e == cudaSuccess; ep++ )
    {
        std::shuffle( perm.begin(), perm.end(), rng ); // the sample order of this epoch
        e = cudaMemcpy( order, perm.data(), sizeof( uint32_t ) * n, cudaMemcpyHostToDevice );
        if ( e == cudaSuccess )
            e = cudaMemset( s.loss, 0, sizeof( double ) );
        for ( uint64_t first = 0; first + batch <= n && e == cudaSuccess; first += batch )
        {
            batch_gradients( s, x, y, order, first, batch, 1.f / float( batch ), 0 );
            step++;
            const float c1 = 1.f / ( 1.f - powf( 0.9f, float( step ) ) );
            const float c2 = 1.f / ( 1.f - powf( 0.999f, float( step ) ) );
            APO2_LAUNCH( "k_train_adam", 0, k_train_adam<<<( kPParams + 255 ) / 256, 256>>>( s.master, s.m, s.v, s.grads, learning_rate, c1, c2 ) );
            e = cudaGetLastError();
        }
        double l = 0.0;
        if ( e == cudaSuccess )
            e = cudaMemcpy( &l, s.loss, sizeof( double ), cudaMemcpyDeviceToHost );
        if ( epoch_loss )
            epoch_loss[ ep ] = float( l / double( ( n / batch ) * batch ) );
    }
    if ( e == cudaSuccess )
        e = cudaMemcpy( master, s.master, sizeof( float ) * kPParams, cudaMemcpyDeviceToHost );
    cudaFree( x );
    if ( e != cudaSuccess )
        return APO2_ERR_CUDA;
    proposal_from_master( master, *model );
    return APO2_OK;
}
