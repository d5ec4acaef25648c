// Stable onesweep LSD radix sort of (u64 key, u32 value) pairs (Adinets & Merrill, 2022):
// one histogram pass over all digits, then one kernel per 8-bit digit that ranks a tile of
// 4096 keys in shared memory, obtains the tile's global digit offsets by decoupled
// look-back over the preceding tiles, and scatters the tile in digit-major order so that
// global writes are contiguous runs.
//
// It replaces thrust::sort_by_key in the LBVH build (apo/src/gpu/lbvh.cu:294-295). Like
// that sort it is stable, which fixes the Morton order of equal codes (the input index
// order) and therefore the tie-break of the hierarchy.
//
// The look-back spins on flags published by blocks that started earlier (tile ids are
// handed out by an atomic counter in start order, so every awaited tile is resident and
// finishes its count without waiting). Every spin still has an iteration limit: a digit
// whose wait runs out stops waiting, and the block then counts that digit's keys in all
// earlier tiles itself from the pass's input (which the previous launch wrote completely),
// so the result stays exact; the kernel records kErrSortSpin in the error word to say that
// a wait ran out.
#include "internal.cuh"

namespace apo2
{
    constexpr uint32_t kRadixBits   = 8;
    constexpr uint32_t kRadix       = 1u << kRadixBits;
    constexpr uint32_t kPasses      = 8;
    constexpr uint32_t kSortThreads = 256;
    constexpr uint32_t kSortWarps   = kSortThreads / 32;
    constexpr uint32_t kItems       = 16;
    constexpr uint32_t kTile        = kSortThreads * kItems; // 4096
    constexpr uint32_t kFlagAggregate = 1u << 30;
    constexpr uint32_t kFlagPrefix    = 2u << 30;
    constexpr uint32_t kValueMask     = ( 1u << 30 ) - 1;
    constexpr uint32_t kSpinLimit     = 1u << 22; // default polls per look-back wait

    static inline size_t align256( size_t b ) { return ( b + 255 ) & ~size_t( 255 ); }

    static inline uint32_t tiles_for( uint32_t n ) { return ( n + kTile - 1 ) / kTile; }

    size_t sort_scratch_bytes( uint32_t n )
    {
        const uint32_t tiles = std::max( 1u, tiles_for( n ) );
        return align256( sizeof( uint64_t ) * size_t( n ) ) + align256( sizeof( uint32_t ) * size_t( n ) )
               + align256( sizeof( uint32_t ) * kPasses * kRadix ) + align256( sizeof( uint32_t ) * size_t( tiles ) * kRadix )
               + align256( sizeof( uint32_t ) * kPasses );
    }

    void sort_scratch_carve( SortScratch & s, void * base, uint32_t n, uint32_t * error_word )
    {
        char * p       = static_cast<char *>( base );
        s.tiles        = std::max( 1u, tiles_for( n ) );
        s.keys_alt     = reinterpret_cast<uint64_t *>( p );
        p += align256( sizeof( uint64_t ) * size_t( n ) );
        s.values_alt = reinterpret_cast<uint32_t *>( p );
        p += align256( sizeof( uint32_t ) * size_t( n ) );
        s.histograms = reinterpret_cast<uint32_t *>( p );
        p += align256( sizeof( uint32_t ) * kPasses * kRadix );
        s.lookback = reinterpret_cast<uint32_t *>( p );
        p += align256( sizeof( uint32_t ) * size_t( s.tiles ) * kRadix );
        s.tile_counter = reinterpret_cast<uint32_t *>( p );
        s.error        = error_word;
    }

    // Digit counts of all eight passes in one read of the keys.
    __global__ void __launch_bounds__( kSortThreads ) k_digit_histograms( const uint64_t * __restrict__ keys, uint32_t n,
                                                                          uint32_t * __restrict__ histograms )
    {
        __shared__ uint32_t local[ kPasses * kRadix ];
        for ( uint32_t i = threadIdx.x; i < kPasses * kRadix; i += blockDim.x )
            local[ i ] = 0;
        __syncthreads();
        for ( uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x )
        {
            const uint64_t k = keys[ i ];
#pragma unroll
            for ( uint32_t p = 0; p < kPasses; p++ )
                atomicAdd( &local[ p * kRadix + uint32_t( ( k >> ( p * kRadixBits ) ) & ( kRadix - 1 ) ) ], 1u );
        }
        __syncthreads();
        for ( uint32_t i = threadIdx.x; i < kPasses * kRadix; i += blockDim.x )
            if ( local[ i ] )
                atomicAdd( &histograms[ i ], local[ i ] );
    }

    // Exclusive scan of each pass's 256 digit counts (one block per pass).
    __global__ void __launch_bounds__( kRadix ) k_scan_histograms( uint32_t * histograms )
    {
        __shared__ uint32_t warp_sums[ kRadix / 32 ];
        uint32_t *          h    = histograms + blockIdx.x * kRadix;
        const uint32_t      v    = h[ threadIdx.x ];
        const uint32_t      lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        uint32_t            x    = v;
#pragma unroll
        for ( int o = 1; o < 32; o <<= 1 )
        {
            const uint32_t y = __shfl_up_sync( 0xffffffffu, x, o );
            if ( lane >= uint32_t( o ) )
                x += y;
        }
        if ( lane == 31 )
            warp_sums[ warp ] = x;
        __syncthreads();
        uint32_t before = 0;
        for ( uint32_t w = 0; w < warp; w++ )
            before += warp_sums[ w ];
        h[ threadIdx.x ] = before + x - v;
    }

    struct OnesweepShared
    {
        uint64_t keys[ kTile ];
        uint32_t values[ kTile ];
        uint32_t warp_counts[ kSortWarps ][ kRadix ]; // counts, then exclusive offsets per warp
        uint32_t tile_prefix[ kRadix ];               // exclusive scan of the tile's digit counts
        uint32_t global_base[ kRadix ];               // global position of the tile's first key per digit
        uint32_t scan_tmp[ kSortWarps ];
        uint32_t tile;
        uint32_t gave_up; // some digit's look-back wait ran out
    };

    __global__ void __launch_bounds__( kSortThreads ) k_onesweep( const uint64_t * __restrict__ keys_in,
                                                                  const uint32_t * __restrict__ values_in,
                                                                  uint64_t * __restrict__ keys_out,
                                                                  uint32_t * __restrict__ values_out, uint32_t n,
                                                                  uint32_t shift, const uint32_t * __restrict__ digit_offsets,
                                                                  uint32_t * lookback, uint32_t * tile_counter,
                                                                  uint32_t * error, uint32_t spin_limit )
    {
        extern __shared__ __align__( 16 ) unsigned char smem_raw[];
        OnesweepShared & sh   = *reinterpret_cast<OnesweepShared *>( smem_raw );
        const uint32_t   lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

        if ( threadIdx.x == 0 )
        {
            sh.tile    = atomicAdd( tile_counter, 1u );
            sh.gave_up = 0;
        }
        for ( uint32_t d = threadIdx.x; d < kSortWarps * kRadix; d += kSortThreads )
            ( &sh.warp_counts[ 0 ][ 0 ] )[ d ] = 0;
        __syncthreads();
        const uint32_t tile = sh.tile;
        const uint32_t base = tile * kTile;

        // warp-striped load: item k of lane l of warp w is key base + w*32*kItems + k*32 + l
        uint64_t key[ kItems ];
        uint32_t val[ kItems ];
        uint32_t rank[ kItems ];
#pragma unroll
        for ( uint32_t k = 0; k < kItems; k++ )
        {
            const uint32_t i = base + warp * 32 * kItems + k * 32 + lane;
            key[ k ]         = i < n ? keys_in[ i ] : ~0ull;
            val[ k ]         = i < n ? values_in[ i ] : 0u;
        }
        const uint32_t lanemask_lt = ( 1u << lane ) - 1u;
#pragma unroll
        for ( uint32_t k = 0; k < kItems; k++ )
        {
            const uint32_t i      = base + warp * 32 * kItems + k * 32 + lane;
            const bool     valid  = i < n;
            const uint32_t digit  = uint32_t( ( key[ k ] >> shift ) & ( kRadix - 1 ) );
            const uint32_t active = __ballot_sync( 0xffffffffu, valid );
            uint32_t       peers  = __match_any_sync( 0xffffffffu, valid ? digit : kRadix + lane );
            peers &= active;
            uint32_t before = 0;
            if ( valid )
            {
                const uint32_t leader = __ffs( peers ) - 1;
                before                = ( lane == leader ) ? sh.warp_counts[ warp ][ digit ] : 0u;
                before                = __shfl_sync( peers, before, leader );
                rank[ k ]             = before + __popc( peers & lanemask_lt );
            }
            __syncwarp();
            if ( valid && lane == __ffs( peers ) - 1 )
                sh.warp_counts[ warp ][ digit ] = before + __popc( peers );
            __syncwarp();
        }
        __syncthreads();

        // per digit: warp offsets, tile count, then decoupled look-back
        {
            const uint32_t d     = threadIdx.x; // kSortThreads == kRadix
            uint32_t       count = 0;
#pragma unroll
            for ( uint32_t w = 0; w < kSortWarps; w++ )
            {
                const uint32_t c          = sh.warp_counts[ w ][ d ];
                sh.warp_counts[ w ][ d ] = count;
                count += c;
            }
            uint32_t * slot = lookback + size_t( tile ) * kRadix + d;
            if ( tile == 0 )
                atomicExch( slot, kFlagPrefix | count );
            else
                atomicExch( slot, kFlagAggregate | count );

            uint32_t exclusive = 0;
            bool     waited_out = false;
            if ( tile > 0 )
            {
                int32_t  p      = int32_t( tile ) - 1;
                uint32_t spins  = 0;
                while ( p >= 0 )
                {
                    const uint32_t word = __ldcv( lookback + size_t( p ) * kRadix + d );
                    if ( ( word & ~kValueMask ) == 0 )
                    {
                        if ( ++spins > spin_limit )
                        {
                            waited_out = true;
                            break;
                        }
                        __nanosleep( 32 );
                        continue;
                    }
                    exclusive += word & kValueMask;
                    if ( word & kFlagPrefix )
                        break;
                    p--;
                }
                if ( waited_out )
                    sh.gave_up = 1; // this digit's prefix is counted below, then published
                else
                    atomicExch( slot, kFlagPrefix | ( ( exclusive + count ) & kValueMask ) );
            }
            __syncthreads();
            if ( sh.gave_up )
            {
                // Exact fallback: count the digits of every key in tiles [0, tile) from the
                // pass's input. tile_prefix serves as the counter array until the scan below.
                sh.tile_prefix[ d ] = 0;
                __syncthreads();
                const uint32_t end = min( n, tile * kTile );
                for ( uint32_t i = threadIdx.x; i < end; i += kSortThreads )
                    atomicAdd( &sh.tile_prefix[ uint32_t( ( keys_in[ i ] >> shift ) & ( kRadix - 1 ) ) ], 1u );
                __syncthreads();
                if ( waited_out )
                {
                    exclusive = sh.tile_prefix[ d ];
                    atomicExch( slot, kFlagPrefix | ( ( exclusive + count ) & kValueMask ) );
                }
                if ( threadIdx.x == 0 )
                    atomicOr( error, uint32_t( kErrSortSpin ) );
                __syncthreads();
            }
            sh.global_base[ d ] = digit_offsets[ d ] + exclusive;

            // tile-local exclusive scan of the digit counts (digit-major order in shared memory)
            uint32_t x = count;
#pragma unroll
            for ( int o = 1; o < 32; o <<= 1 )
            {
                const uint32_t y = __shfl_up_sync( 0xffffffffu, x, o );
                if ( lane >= uint32_t( o ) )
                    x += y;
            }
            if ( lane == 31 )
                sh.scan_tmp[ warp ] = x;
            __syncthreads();
            uint32_t before = 0;
            for ( uint32_t w = 0; w < warp; w++ )
                before += sh.scan_tmp[ w ];
            sh.tile_prefix[ d ] = before + x - count;
        }
        __syncthreads();

        // shared-memory scatter in digit-major order
#pragma unroll
        for ( uint32_t k = 0; k < kItems; k++ )
        {
            const uint32_t i = base + warp * 32 * kItems + k * 32 + lane;
            if ( i < n )
            {
                const uint32_t digit = uint32_t( ( key[ k ] >> shift ) & ( kRadix - 1 ) );
                const uint32_t pos   = sh.tile_prefix[ digit ] + sh.warp_counts[ warp ][ digit ] + rank[ k ];
                sh.keys[ pos ]       = key[ k ];
                sh.values[ pos ]     = val[ k ];
            }
        }
        __syncthreads();

        // contiguous runs to global memory
        const uint32_t valid_in_tile = min( kTile, n - base );
        for ( uint32_t pos = threadIdx.x; pos < valid_in_tile; pos += kSortThreads )
        {
            const uint64_t k     = sh.keys[ pos ];
            const uint32_t digit = uint32_t( ( k >> shift ) & ( kRadix - 1 ) );
            const uint32_t dst   = sh.global_base[ digit ] + ( pos - sh.tile_prefix[ digit ] );
            keys_out[ dst ]      = k;
            values_out[ dst ]    = sh.values[ pos ];
        }
    }

    void radix_sort_pairs( uint64_t * keys, uint32_t * values, uint32_t n, SortScratch & s, cudaStream_t stream,
                           uint32_t spin_limit )
    {
        if ( n < 2 )
            return;
        // the tile's shared memory is above the 48 KB default: the attribute is set once per
        // device, on the device current when the sort is launched
        static PerDeviceOnce configured;
        configured.run( [] {
            cudaFuncSetAttribute( k_onesweep, cudaFuncAttributeMaxDynamicSharedMemorySize, int( sizeof( OnesweepShared ) ) );
        } );
        const uint32_t tiles = tiles_for( n );
        cudaMemsetAsync( s.histograms, 0, sizeof( uint32_t ) * kPasses * kRadix, stream );
        cudaMemsetAsync( s.tile_counter, 0, sizeof( uint32_t ) * kPasses, stream );
        const uint32_t hist_blocks = std::min<uint32_t>( 296, ( n + kSortThreads * 8 - 1 ) / ( kSortThreads * 8 ) );
        APO2_LAUNCH( "k_digit_histograms", stream, k_digit_histograms<<<std::max( 1u, hist_blocks ), kSortThreads, 0, stream>>>( keys, n, s.histograms ) );
        APO2_LAUNCH( "k_scan_histograms", stream, k_scan_histograms<<<kPasses, kRadix, 0, stream>>>( s.histograms ) );

        uint64_t * kin = keys;
        uint32_t * vin = values;
        uint64_t * kout = s.keys_alt;
        uint32_t * vout = s.values_alt;
        for ( uint32_t p = 0; p < kPasses; p++ )
        {
            cudaMemsetAsync( s.lookback, 0, sizeof( uint32_t ) * size_t( tiles ) * kRadix, stream );
            APO2_LAUNCH( "k_onesweep", stream, k_onesweep<<<tiles, kSortThreads, sizeof( OnesweepShared ), stream>>>(
                kin, vin, kout, vout, n, p * kRadixBits, s.histograms + p * kRadix, s.lookback, s.tile_counter + p, s.error,
                spin_limit ? spin_limit : kSpinLimit ) );
            std::swap( kin, kout );
            std::swap( vin, vout );
        }
        // eight passes: the result is back in (keys, values)
    }
} // namespace apo2
