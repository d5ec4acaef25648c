// Device data structures shared by the build's kernels.
#pragma once

#include <cfloat>
#include <cstdint>
#include <cstdio>

#include <algorithm>
#include <atomic>
#include <mutex>

#include <cuda_runtime.h>

#include "geometry.cuh"

// Launches kernel `name` on stream `s` through the launch observer.
#define APO2_LAUNCH( name, s, ... )             \
    do                                          \
    {                                           \
        ::apo2::observe( name, s, false );      \
        __VA_ARGS__;                            \
        ::apo2::observe( name, s, true );       \
    } while ( 0 )

namespace apo2
{
    // Launch observer: the C ABI installs it (per thread) to count the kernels of a build and,
    // when stage timing is on, to bracket each launch with CUDA events.
    using LaunchHook = void ( * )( const char * name, cudaStream_t s, bool after, void * ctx );
    struct LaunchObserver
    {
        LaunchHook hook = nullptr;
        void *     ctx  = nullptr;
    };
    inline LaunchObserver & launch_observer()
    {
        static thread_local LaunchObserver o;
        return o;
    }
    inline void observe( const char * name, cudaStream_t s, bool after )
    {
        const LaunchObserver & o = launch_observer();
        if ( o.hook )
            o.hook( name, s, after, o.ctx );
    }

    // Runs a set-up step (kernel attributes and the like) once per CUDA device, on the device
    // current at the call; safe from several host threads.
    class PerDeviceOnce
    {
      public:
        template<class F>
        void run( F && f )
        {
            int device = 0;
            if ( cudaGetDevice( &device ) != cudaSuccess || device < 0 || device >= kDevices )
            {
                f(); // unknown ordinal: do it every time
                return;
            }
            if ( done_[ device ].load( std::memory_order_acquire ) )
                return;
            std::lock_guard<std::mutex> lock( mutex_ );
            if ( !done_[ device ].load( std::memory_order_relaxed ) )
            {
                f();
                done_[ device ].store( true, std::memory_order_release );
            }
        }

      private:
        static constexpr int kDevices = 64;
        std::atomic<bool>    done_[ kDevices ] = {};
        std::mutex           mutex_;
    };

    constexpr uint32_t kNone = 0xffffffffu;

    // Per-cell capacities of the reference (apo/include/apo/gpu/algorithm.inl:25-30).
    constexpr uint32_t kMaxVertices  = 152;
    constexpr uint32_t kMaxEdges     = 264;
    constexpr uint32_t kMaxNewEdges  = 64;
    constexpr uint32_t kMaxBisectors = 512;
    constexpr uint32_t kArtificial   = 6;

    // Cell status (apo/include/apo/gpu/topology_update.cuh:76-81).
    constexpr uint8_t kInValidation   = 0;
    constexpr uint8_t kFullyValidated = 1;
    constexpr uint8_t kBuried         = 0xff;

    // Error flags reported through apo2_stats::error_flags.
    enum ErrorFlag : uint32_t
    {
        kErrVertexCap  = 1,
        kErrEdgeCap    = 2,
        kErrNewEdgeCap = 4,
        kErrBisector   = 8,
        kErrStack      = 16,
        kErrSortSpin   = 32,
        kErrWalk       = 64,  // a traversal or a validation restart loop hit its bound
    };

    // Scene box and radius range, written on the device by the bounds kernel.
    struct Scene
    {
        double   lo[ 3 ], hi[ 3 ];
        double   rmin, rmax;
        float    box_lo[ 3 ], box_hi[ 3 ], scale[ 3 ];
        uint32_t n;
    };

    // Internal BVH node with both child boxes inline (64 bytes, one aligned load):
    // a = (l.lo.x, l.lo.y, l.lo.z, l.hi.x), b = (l.hi.y, l.hi.z, r.lo.x, r.lo.y),
    // c = (r.lo.z, r.hi.x, r.hi.y, r.hi.z), child = (left, right, -, -).
    struct __align__( 16 ) WideNode
    {
        float4 a, b, c;
        int4   child;
    };

    __device__ __forceinline__ void load_node( const WideNode * __restrict__ nodes, uint32_t i, Box & l, Box & r, uint32_t & lc,
                                               uint32_t & rc )
    {
        const float4 a = __ldg( &nodes[ i ].a );
        const float4 b = __ldg( &nodes[ i ].b );
        const float4 c = __ldg( &nodes[ i ].c );
        const int4   d = __ldg( &nodes[ i ].child );
        l.lo           = make_float3( a.x, a.y, a.z );
        l.hi           = make_float3( a.w, b.x, b.y );
        r.lo           = make_float3( b.z, b.w, c.x );
        r.hi           = make_float3( c.y, c.z, c.w );
        lc             = uint32_t( d.x );
        rc             = uint32_t( d.y );
    }

    // Stable LSD radix sort scratch (onesweep).
    struct SortScratch
    {
        uint64_t * keys_alt   = nullptr;
        uint32_t * values_alt = nullptr;
        uint32_t * histograms = nullptr; // 8 x 256 global digit counts, then exclusive offsets
        uint32_t * lookback   = nullptr; // tiles x 256 status words (one pass)
        uint32_t * tile_counter = nullptr;
        uint32_t * error      = nullptr;
        uint32_t   tiles      = 0;
    };
    size_t sort_scratch_bytes( uint32_t n );
    void   sort_scratch_carve( SortScratch & s, void * base, uint32_t n, uint32_t * error_word );
    // spin_limit: polls per look-back wait before the exact recount takes over (0 = default)
    void   radix_sort_pairs( uint64_t * keys, uint32_t * values, uint32_t n, SortScratch & s, cudaStream_t stream,
                             uint32_t spin_limit = 0 );

    struct Tree
    {
        uint64_t * codes   = nullptr; // n, Morton order after the sort
        uint32_t * indices = nullptr; // n, sorted -> original
        double4 *  sites   = nullptr; // n + 6, Morton order then the artificial sites
        float4 *   sites_f = nullptr; // n, float copy for traversal
        int32_t *  parent  = nullptr; // 2n - 1
        int32_t *  left    = nullptr;
        int32_t *  right   = nullptr;
        float4 *   boxes   = nullptr; // 2 (2n - 1): min, max per node
        uint32_t * sizes   = nullptr; // 2n - 1
        uint32_t * arrivals = nullptr; // n - 1 refit counters
        WideNode * nodes   = nullptr; // n - 1 internal nodes
    };

    struct BoundsPartial;
    void   launch_bounds( const void * input, bool is_f64, uint32_t n, double4 * copy, BoundsPartial * partials,
                          uint32_t partial_count, uint32_t * counter, Scene * scene, double4 * artificial, cudaStream_t s );
    size_t bounds_partial_bytes( uint32_t count );
    void   launch_tree( const Tree & t, uint32_t n, const double4 * input, const Scene * scene, SortScratch & sort,
                        cudaStream_t s, uint32_t spin_limit = 0 );
    void   launch_lbvh_f32( const float4 * sites, uint32_t n, float3 lo, float3 scale, uint32_t * indices, uint64_t * codes,
                            int32_t * parent, int32_t * left, int32_t * right, float4 * boxes, uint32_t * sizes,
                            uint32_t * arrivals, SortScratch & sort, cudaStream_t s );
    // Pieces of the tree build for callers that build trees over other sphere sets: Morton
    // codes inside a box held on the device (lo xyz, 1 / extent xyz), and the Karras
    // hierarchy, refit and wide-node packing over n Morton-sorted leaves whose boxes are in
    // boxes[2 (n - 1 + i) + {0, 1}].
    void launch_morton_box( const float4 * sites, uint32_t n, const float * box, uint64_t * codes, uint32_t * indices,
                            cudaStream_t s );
    void launch_hierarchy( const uint64_t * codes, uint32_t n, int32_t * parent, int32_t * left, int32_t * right, float4 * boxes,
                           uint32_t * arrivals, WideNode * nodes, cudaStream_t s );
} // namespace apo2
