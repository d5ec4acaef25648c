// apo2_radix_sort_pairs_static: the stable (u64 key, u32 value) radix sort of the LBVH build,
// working in scratch memory that the library reserves at load time instead of scratch the
// caller allocates.
//
// Some callers cannot allocate device memory at the point where they sort: processes whose
// device memory is owned by another allocator (a framework's caching allocator) that forbids
// foreign allocations, and latency-critical paths where cudaMalloc's implicit synchronisation
// would stall other streams. They pass only the keys and values; the scratch -- the ping-pong
// copies, the digit histograms, the look-back flags, the tile counters and an error word --
// lives in a file-scope __device__ array of fixed size, so every GPU that loads this library
// holds it (kStaticSortBytes, about 12.3 MiB) until the process exits.
//
// Limits and sharing:
//   - at most kStaticSortPairs = 2^20 pairs per call; larger sizes are rejected;
//   - all calls on a device share the one array and leave their state in it; each call
//     clears what must start at zero (histograms, look-back flags, tile counters, error
//     word) on its own stream, so calls that run one after the other are independent, but
//     calls that overlap on the GPU (other streams, other host threads) race and corrupt
//     each other's results;
//   - the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current;
//   - a look-back wait that runs out is recounted exactly inside the sort; the error word
//     that records it stays in the array and is not reported by this entry point.
#include <cstdint>
#include <mutex>

#include "../../include/apo2.h"
#include "internal.cuh"

namespace apo2
{
    constexpr uint32_t kStaticSortPairs = 1u << 20;
    // sort_scratch_bytes(2^20) is 12,853,760 bytes; 256 bytes in front hold the error word.
    constexpr size_t kStaticSortBytes = 256 + 12853760 + 4096;

    static __device__ __align__( 256 ) unsigned char g_static_sort_scratch[ kStaticSortBytes ];

    namespace
    {
        constexpr int kMaxDevices = 64;
        std::mutex    g_static_mutex;
        void *        g_static_address[ kMaxDevices ] = {};
    } // namespace
} // namespace apo2

extern "C" apo2_status apo2_radix_sort_pairs_static( uint64_t * keys, uint32_t * values, uint32_t n, void * stream )
{
    using namespace apo2;
    if ( !keys || !values )
        return APO2_ERR_INVALID_ARG;
    if ( n > kStaticSortPairs || sort_scratch_bytes( n ) + 256 > kStaticSortBytes )
        return APO2_ERR_TOO_LARGE; // more pairs than the preallocated scratch holds (2^20)

    int device = 0;
    if ( cudaGetDevice( &device ) != cudaSuccess || device < 0 || device >= kMaxDevices )
        return APO2_ERR_CUDA;
    void * base = nullptr;
    {
        std::lock_guard<std::mutex> lock( g_static_mutex );
        if ( !g_static_address[ device ] )
        {
            // once per device, with that device current
            void *            address = nullptr;
            const cudaError_t err     = cudaGetSymbolAddress( &address, g_static_sort_scratch );
            if ( err != cudaSuccess || !address )
                return APO2_ERR_CUDA;
            g_static_address[ device ] = address;
        }
        base = g_static_address[ device ];
    }

    cudaStream_t s     = static_cast<cudaStream_t>( stream );
    uint32_t *   error = static_cast<uint32_t *>( base );
    SortScratch  sort;
    sort_scratch_carve( sort, static_cast<char *>( base ) + 256, n, error );
    if ( cudaMemsetAsync( error, 0, sizeof( uint32_t ), s ) != cudaSuccess )
        return APO2_ERR_CUDA;
    radix_sort_pairs( keys, values, n, sort, s ); // clears histograms, tile counters and look-back flags
    return cudaGetLastError() == cudaSuccess ? APO2_OK : APO2_ERR_CUDA;
}
