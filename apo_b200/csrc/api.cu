// C ABI of the builder (include/apo2.h): handle lifetime, device memory, the build
// sequence on one stream, output extraction and the host-side topology.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <set>
#include <string>
#include <tuple>
#include <vector>
#include <algorithm>
#include <atomic>
#include <thread>

#include "../../include/apo2.h"
#include "cells.cuh"
#include "cavity.cuh"

namespace
{
    using namespace apo2;

    thread_local std::string g_last_error;

    apo2_status fail( apo2_status code, const std::string & text )
    {
        g_last_error = text;
        return code;
    }

    apo2_status cuda_fail( cudaError_t err, const char * where )
    {
        return fail( err == cudaErrorMemoryAllocation ? APO2_ERR_OUT_OF_MEMORY : APO2_ERR_CUDA,
                     std::string( where ) + ": " + cudaGetErrorString( err ) );
    }

#define APO2_CUDA( call, where )                 \
    do                                           \
    {                                            \
        const cudaError_t e_ = ( call );         \
        if ( e_ != cudaSuccess )                 \
            return cuda_fail( e_, where );       \
    } while ( 0 )

    size_t align256( size_t b ) { return ( b + 255 ) & ~size_t( 255 ); }

    // One device allocation carved into the build's arrays.
    struct Arena
    {
        char * base = nullptr;
        size_t size = 0, used = 0;
        template<class T>
        T * take( size_t count )
        {
            T * p = reinterpret_cast<T *>( base + used );
            used += align256( sizeof( T ) * count );
            return p;
        }
    };

    constexpr int      kStages    = 10;
    constexpr uint32_t kMaxRounds = 64; // validation rounds at most (apo2_options.max_iterations)

    // Error-word flags that mean the per-cell stores could not hold a cell (the results of
    // those cells are incomplete), and those that mean a bounded loop stopped early.
    constexpr uint32_t kCapacityFlags = kErrVertexCap | kErrEdgeCap | kErrNewEdgeCap | kErrBisector | kErrStack;
} // namespace

struct apo2_handle
{
    uint32_t     n = 0;
    apo2_options options {};
    int          device = 0;

    Arena          arena;
    void *         input     = nullptr; // caller sites (device copy)
    bool           input_f64 = false;
    double4 *      input_d4  = nullptr; // float64 copy in input order
    BoundsPartial * partials = nullptr;
    uint32_t       partial_count = 0;
    uint32_t *     bounds_counter = nullptr;
    Scene *        scene          = nullptr;
    Tree           tree;
    SortScratch    sort;
    CellContext    cells;
    uint32_t *     tasks       = nullptr;
    uint32_t *     task_counts = nullptr; // one per validation round
    uint32_t *     error       = nullptr;

    SpecBuffers   spec;
    OutputBuffers out;
    void *        out_alloc = nullptr;
    bool          built     = false;
    bool          extracted = false;

    // cavity detection: hit ratios of the extraction numbered ratio_epoch
    void *   cavity_alloc  = nullptr;
    size_t   cavity_bytes  = 0;
    float *  ratios        = nullptr;
    uint64_t ratio_count   = 0;
    uint64_t extract_epoch = 0;
    uint64_t ratio_epoch   = ~0ull;

    // learned k-proposal: the network on the device and the proposed rank of every site
    void * proposal_alloc = nullptr;

    cudaEvent_t events[ kStages + 1 ] = {};
    bool        timing                = false;
    apo2_stats  stats {};

    // launch observer state: kernel count of the last build, and (timing on) per-launch events
    struct KernelRecord
    {
        const char * name;
        int          begin, end;
    };
    uint32_t                  launches = 0;
    std::vector<cudaEvent_t>  event_pool;
    size_t                    events_used = 0;
    std::vector<KernelRecord> records;
};

namespace
{
    apo2_status ensure_output_capacity( apo2_handle * h, uint64_t vcap, uint64_t ccap )
    {
        if ( h->out_alloc && vcap <= h->out.vcap && ccap <= h->out.ccap )
            return APO2_OK;
        if ( h->out_alloc )
            cudaFree( h->out_alloc );
        h->out_alloc        = nullptr;
        const size_t bytes  = align256( sizeof( double4 ) * vcap ) + align256( sizeof( uint4 ) * vcap )
                             + align256( sizeof( double4 ) * ccap ) + align256( sizeof( uint4 ) * ccap );
        APO2_CUDA( cudaMalloc( &h->out_alloc, bytes ), "output allocation" );
        char * p    = static_cast<char *>( h->out_alloc );
        h->out.vpos = reinterpret_cast<double4 *>( p );
        p += align256( sizeof( double4 ) * vcap );
        h->out.vids = reinterpret_cast<uint4 *>( p );
        p += align256( sizeof( uint4 ) * vcap );
        h->out.cpos = reinterpret_cast<double4 *>( p );
        p += align256( sizeof( double4 ) * ccap );
        h->out.cids = reinterpret_cast<uint4 *>( p );
        h->out.vcap = vcap;
        h->out.ccap = ccap;
        return APO2_OK;
    }

    apo2_status upload_sites( apo2_handle * h, const void * sites, apo2_dtype dtype, apo2_location location, cudaStream_t s )
    {
        const size_t bytes = size_t( h->n ) * ( dtype == APO2_F64 ? 32 : 16 );
        if ( ( dtype == APO2_F64 ) != h->input_f64 )
            return fail( APO2_ERR_INVALID_ARG, "dtype differs from the handle's" );
        APO2_CUDA( cudaMemcpyAsync( h->input, sites, bytes, location == APO2_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, s ),
                   "site upload" );
        h->built     = false;
        h->extracted = false;
        return APO2_OK;
    }

    int take_event( apo2_handle * h )
    {
        if ( h->events_used == h->event_pool.size() )
        {
            cudaEvent_t e;
            cudaEventCreate( &e );
            h->event_pool.push_back( e );
        }
        return int( h->events_used++ );
    }

    void on_launch( const char * name, cudaStream_t s, bool after, void * ctx )
    {
        apo2_handle * h = static_cast<apo2_handle *>( ctx );
        if ( !after )
        {
            h->launches++;
            if ( h->timing )
            {
                const int e = take_event( h );
                cudaEventRecord( h->event_pool[ e ], s );
                h->records.push_back( { name, e, -1 } );
            }
        }
        else if ( h->timing )
        {
            const int e = take_event( h );
            cudaEventRecord( h->event_pool[ e ], s );
            h->records.back().end = e;
        }
    }

    struct ObserveScope
    {
        LaunchObserver saved;
        explicit ObserveScope( apo2_handle * h )
        {
            saved                    = launch_observer();
            launch_observer().hook   = on_launch;
            launch_observer().ctx    = h;
        }
        ~ObserveScope() { launch_observer() = saved; }
    };

    void record( apo2_handle * h, int stage, cudaStream_t s )
    {
        if ( h->timing )
            cudaEventRecord( h->events[ stage ], s );
    }

    apo2_status enqueue_build( apo2_handle * h, cudaStream_t s )
    {
        const uint32_t n = h->n;
        // the error check below is about this build's launches: an error another call left
        // behind (not one that broke the context, which every call reports again) is dropped
        cudaGetLastError();
        ObserveScope   observe( h );
        h->launches    = 0;
        h->events_used = 0;
        h->records.clear();
        record( h, 0, s );
        cudaMemsetAsync( h->error, 0, sizeof( uint32_t ), s );
        cudaMemsetAsync( h->cells.counters, 0, sizeof( unsigned long long ) * kCounters, s );
        launch_bounds( h->input, h->input_f64, n, h->input_d4, h->partials, h->partial_count, h->bounds_counter, h->scene,
                       h->tree.sites + n, s );
        record( h, 1, s );
        launch_tree( h->tree, n, h->input_d4, h->scene, h->sort, s, h->options.wait_limit );
        record( h, 2, s ); // bounds+Morton+sort+tree recorded as one span plus the sort below
        // kNN steps (algorithm.inl:1535-1549); with several, the kNN span is the first
        // step's search and the cells span everything after it
        const uint32_t steps = h->options.knn_steps;
        if ( steps == 0 )
        {
            // no kNN list is ever searched; the reference leaves them all empty (0xff bytes)
            cudaMemsetAsync( h->cells.knn, 0xff, sizeof( uint32_t ) * size_t( n ) * h->cells.k, s );
            record( h, 3, s );
            launch_cells( h->cells, kCellsInitOnly, s );
        }
        for ( uint32_t step = 0; step < steps; step++ )
        {
            launch_knn( h->cells, step, s );
            if ( step == 0 )
                record( h, 3, s );
            launch_cells( h->cells, step == 0 ? kCellsFirst : kCellsNext, s );
        }
        if ( h->cells.scheduled )
        {
            // learned form: a second kNN step for the uncertified cells proposed beyond k
            launch_knn( h->cells, 1, s );
            launch_cells( h->cells, kCellsNext, s );
        }
        record( h, 4, s );
        // stop_after (parity checks): 1 after the cells, 2 + 2r / 3 + 2r after round r's passes
        const uint32_t stop   = h->options.stop_after;
        bool           halted = stop == 1;
        const uint32_t rounds = h->options.max_iterations;
        cudaMemsetAsync( h->task_counts, 0, sizeof( uint32_t ) * ( rounds + 1 ), s );
        for ( uint32_t r = 0; r < rounds && !halted; r++ )
        {
            launch_tasks( h->cells, h->tasks, h->task_counts + r, s );
            launch_vertex_validation( h->cells, h->tasks, h->task_counts + r, s );
            if ( stop == 2 + 2 * r )
                break;
            if ( h->options.edge_search == 1 )
                launch_edge_validation( h->cells, h->tasks, h->task_counts + r, s );
            else
                launch_edge_validation_speculative( h->cells, h->tasks, h->task_counts + r, h->spec, s );
            halted = stop == 3 + 2 * r;
        }
        // cells still in validation after the last round (the reference leaves them as they are)
        if ( stop == 0 )
            launch_tasks( h->cells, h->tasks, h->task_counts + rounds, s );
        record( h, 5, s );
        if ( stop == 0 )
            launch_bisector_validation( h->cells, s );
        record( h, 6, s );
        const cudaError_t err = cudaGetLastError();
        if ( err != cudaSuccess )
            return cuda_fail( err, "build launch" );
        h->built       = true;
        h->extracted   = false;
        h->ratio_epoch = ~0ull; // hit ratios belong to the previous build's vertices
        return APO2_OK;
    }

    apo2_status enqueue_extract( apo2_handle * h, cudaStream_t s )
    {
        ObserveScope observe( h );
        launch_output( h->cells, h->out, s );
        record( h, 7, s );
        h->extract_epoch++;
        const cudaError_t err = cudaGetLastError();
        if ( err != cudaSuccess )
            return cuda_fail( err, "output launch" );
        h->extracted = true;
        return APO2_OK;
    }

    // Error status of a finished build: per-cell store overflows first, then cells that were
    // still uncertified after the last validation round, or a bounded walk or restart loop
    // that stopped early. The diagram is complete either way, as the reference leaves it.
    apo2_status build_status( apo2_handle * h, uint32_t err, uint32_t uncertified )
    {
        h->stats.error_flags = err;
        h->stats.uncertified = uncertified;
        if ( err & kCapacityFlags )
            return fail( APO2_ERR_CAPACITY, "capacity flags " + std::to_string( err ) );
        if ( uncertified )
            return fail( APO2_ERR_ITER_LIMIT, std::to_string( uncertified ) + " cells still uncertified after " +
                                                  std::to_string( h->options.max_iterations ) + " validation rounds" );
        if ( err & kErrWalk )
            return fail( APO2_ERR_ITER_LIMIT, "a traversal or restart loop reached its bound" );
        return APO2_OK; // kErrSortSpin alone: a look-back wait ran out and its recount kept the order exact
    }

    apo2_status finish( apo2_handle * h, cudaStream_t s )
    {
        APO2_CUDA( cudaStreamSynchronize( s ), "build" );
        uint32_t err = 0, uncertified = 0;
        APO2_CUDA( cudaMemcpy( &err, h->error, sizeof( uint32_t ), cudaMemcpyDeviceToHost ), "error word" );
        if ( h->options.stop_after == 0 )
            APO2_CUDA( cudaMemcpy( &uncertified, h->task_counts + h->options.max_iterations, sizeof( uint32_t ),
                                   cudaMemcpyDeviceToHost ),
                       "uncertified count" );
        return build_status( h, err, uncertified );
    }

    // Makes sure the output arrays hold everything the last extraction counted (one
    // synchronisation; a re-extraction only when the capacity had to grow).
    apo2_status settle_output( apo2_handle * h, cudaStream_t s )
    {
        if ( !h->built )
            return fail( APO2_ERR_NOT_BUILT, "no build yet" );
        if ( !h->extracted )
        {
            apo2_status st = enqueue_extract( h, s );
            if ( st != APO2_OK )
                return st;
        }
        APO2_CUDA( cudaStreamSynchronize( s ), "extract" );
        uint64_t totals[ 2 ];
        APO2_CUDA( cudaMemcpy( totals, h->out.totals, sizeof( totals ), cudaMemcpyDeviceToHost ), "output totals" );
        if ( totals[ 0 ] > h->out.vcap || totals[ 1 ] > h->out.ccap )
        {
            apo2_status st = ensure_output_capacity( h, totals[ 0 ] + totals[ 0 ] / 8 + 1024, totals[ 1 ] + totals[ 1 ] / 8 + 1024 );
            if ( st != APO2_OK )
                return st;
            st = enqueue_extract( h, s );
            if ( st != APO2_OK )
                return st;
            APO2_CUDA( cudaStreamSynchronize( s ), "extract" );
        }
        h->stats.output_vertices     = totals[ 0 ];
        h->stats.output_closed_edges = totals[ 1 ];
        return APO2_OK;
    }

    template<class T>
    std::vector<T> download( const T * p, size_t count )
    {
        std::vector<T> v( count );
        if ( count )
            cudaMemcpy( v.data(), p, sizeof( T ) * count, cudaMemcpyDeviceToHost );
        return v;
    }
} // namespace

extern "C" {

const char * apo2_version( void ) { return "apo2 1.0 (sm_100a)"; }

const char * apo2_last_error_string( void ) { return g_last_error.c_str(); }

namespace
{
    // The cells a handle builds: shard shard_index of shard_count contiguous ranges of the
    // Morton-sorted sites.
    void shard_range( uint32_t n, const apo2_options & opt, uint32_t & lo, uint32_t & hi )
    {
        const uint32_t count = std::max( opt.shard_count, 1u );
        lo                   = uint32_t( uint64_t( n ) * opt.shard_index / count );
        hi                   = uint32_t( uint64_t( n ) * ( opt.shard_index + 1 ) / count );
    }

    // Device bytes of a handle for n sites (every array of the build, carved from one block;
    // the per-cell stores only for the shard's cells).
    size_t arena_bytes( uint32_t n, const apo2_options & opt, bool f64 )
    {
        uint32_t lo = 0, hi = 0;
        shard_range( n, opt, lo, hi );
        const size_t rows = std::max<size_t>( hi - lo, 1 );
        const size_t nodes     = 2 * size_t( n ) - 1;
        const size_t sortBytes = sort_scratch_bytes( n );
        const size_t scanWords = output_scan_scratch_words( n );
        size_t       total     = 0;
        total += align256( size_t( n ) * ( f64 ? 32 : 16 ) );
        total += align256( sizeof( double4 ) * n );
        total += align256( bounds_partial_bytes( 148 * 4 ) ) + align256( 4 ) + align256( sizeof( Scene ) );
        total += align256( 8 * size_t( n ) ) + align256( 4 * size_t( n ) ) + align256( sizeof( double4 ) * ( n + kArtificial ) )
                 + align256( sizeof( float4 ) * n ) + 3 * align256( 4 * nodes ) + align256( sizeof( float4 ) * 2 * nodes )
                 + align256( 4 * nodes ) + align256( 4 * size_t( n ) ) + align256( sizeof( WideNode ) * n );
        total += align256( sortBytes );
        total += align256( size_t( n ) ) + align256( 4 * size_t( n ) * opt.k ) + align256( 4 * size_t( n ) ) * 3
                 + align256( sizeof( uint4 ) * kMaxVertices * rows ) + align256( sizeof( uint4 ) * kMaxEdges * rows );
        total += align256( 4 * size_t( n ) ) + align256( 4 * ( kMaxRounds + 1 ) ) + align256( 4 );
        total += align256( 4 * size_t( n ) ) * 2 + align256( 4 * scanWords * 2 ) + align256( 16 );
        total += align256( spec_bytes( n ) );
        total += align256( walk_scratch_bytes() ) + align256( 4 );
        total += align256( sizeof( unsigned long long ) * kCounters );
        return total;
    }

    // Points every array of the handle into its arena for n sites (n at most the size the
    // arena was allocated for: every array grows with n). Returns false if it does not fit.
    bool carve( apo2_handle * h, uint32_t n )
    {
        const size_t nodes     = 2 * size_t( n ) - 1;
        const size_t sortBytes = sort_scratch_bytes( n );
        const size_t scanWords = output_scan_scratch_words( n );
        const apo2_options & opt = h->options;
        h->n             = n;
        h->partial_count = 148 * 4;
        Arena & a        = h->arena;
        a.used           = 0;
        h->input          = a.take<char>( size_t( n ) * ( h->input_f64 ? 32 : 16 ) );
        h->input_d4       = a.take<double4>( n );
        h->partials       = reinterpret_cast<BoundsPartial *>( a.take<char>( bounds_partial_bytes( h->partial_count ) ) );
        h->bounds_counter = a.take<uint32_t>( 1 );
        h->scene          = a.take<Scene>( 1 );
        Tree & t          = h->tree;
        t.codes           = a.take<uint64_t>( n );
        t.indices         = a.take<uint32_t>( n );
        t.sites           = a.take<double4>( n + kArtificial );
        t.sites_f         = a.take<float4>( n );
        t.parent          = a.take<int32_t>( nodes );
        t.left            = a.take<int32_t>( nodes );
        t.right           = a.take<int32_t>( nodes );
        t.boxes           = a.take<float4>( 2 * nodes );
        t.sizes           = a.take<uint32_t>( nodes );
        t.arrivals        = a.take<uint32_t>( n );
        t.nodes           = a.take<WideNode>( n );
        void * sortBase   = a.take<char>( sortBytes );
        CellContext & c   = h->cells;
        c.n               = n;
        c.k               = opt.k;
        shard_range( n, opt, c.lo, c.hi );
        const size_t rows = std::max<size_t>( c.hi - c.lo, 1 );
        c.sites           = t.sites;
        c.sites_f         = t.sites_f;
        c.nodes           = t.nodes;
        c.indices         = t.indices;
        c.status          = a.take<uint8_t>( n );
        c.knn             = a.take<uint32_t>( size_t( n ) * opt.k );
        c.known_radii     = a.take<float>( n );
        c.vertex_nb       = a.take<uint32_t>( n );
        c.edge_nb         = a.take<uint32_t>( n );
        c.vertices        = a.take<uint4>( rows * kMaxVertices ); // rows of cells [lo, hi)
        c.edges           = a.take<uint4>( rows * kMaxEdges );
        h->tasks          = a.take<uint32_t>( n );
        h->task_counts    = a.take<uint32_t>( kMaxRounds + 1 );
        h->error          = a.take<uint32_t>( 1 );
        c.error           = h->error;
        c.scene           = h->scene;
        h->out.vcount     = a.take<uint32_t>( n );
        h->out.ccount     = a.take<uint32_t>( n );
        h->out.tile_sums  = a.take<uint32_t>( scanWords * 2 );
        h->out.totals     = a.take<uint64_t>( 2 );
        spec_carve( h->spec, a.take<char>( spec_bytes( n ) ), n );
        c.walk_scratch    = a.take<uint32_t>( walk_scratch_bytes() / sizeof( uint32_t ) );
        c.work_counter    = a.take<uint32_t>( 1 );
        c.counters        = a.take<unsigned long long>( kCounters );
        c.fp32            = opt.precision == APO2_PRECISION_FP32_FILTER ? 1u : 0u;
        c.codes           = t.codes;
        sort_scratch_carve( h->sort, sortBase, n, h->error );
        return a.used <= a.size;
    }
} // namespace

namespace
{
    // Checks the caller's options and fills in the defaults.
    apo2_status normalize_options( const apo2_options * options, apo2_options & opt )
    {
        opt = apo2_options {};
        if ( options )
        {
            if ( options->struct_size != sizeof( apo2_options ) )
                return fail( APO2_ERR_INVALID_ARG, "apo2_options.struct_size mismatch" );
            opt = *options;
        }
        if ( opt.k == 0 )
            opt.k = 16;
        if ( opt.k > kMaxK )
            return fail( APO2_ERR_INVALID_ARG, "k is at most 16" );
        if ( opt.max_iterations == 0 )
            opt.max_iterations = 10;
        if ( opt.edge_search > 1 )
            return fail( APO2_ERR_INVALID_ARG, "edge_search is 0 or 1" );
        if ( opt.knn_steps == 0 )
            opt.knn_steps = 1;
        else if ( opt.knn_steps == APO2_NO_KNN_STEPS )
            opt.knn_steps = 0;
        else if ( opt.knn_steps > 64 )
            return fail( APO2_ERR_INVALID_ARG, "knn_steps is at most 64" );
        opt.max_iterations = std::min( opt.max_iterations, kMaxRounds );
        if ( opt.shard_count == 0 )
            opt.shard_count = 1;
        if ( opt.precision > APO2_PRECISION_FP32_FILTER )
            return fail( APO2_ERR_INVALID_ARG, "precision is APO2_PRECISION_FP64 or APO2_PRECISION_FP32_FILTER" );
        if ( opt.shard_index >= opt.shard_count )
            return fail( APO2_ERR_INVALID_ARG, "shard_index must be below shard_count" );
        return APO2_OK;
    }
} // namespace

apo2_status apo2_create( const void * sites, uint32_t n, apo2_dtype dtype, apo2_location location, const apo2_options * options,
                         apo2_handle ** out )
{
    if ( !out || !sites || n < 2 || ( dtype != APO2_F32 && dtype != APO2_F64 )
         || ( location != APO2_HOST && location != APO2_DEVICE ) )
        return fail( APO2_ERR_INVALID_ARG, "invalid argument to apo2_create" );
    if ( n > ( 1u << 28 ) )
        return fail( APO2_ERR_TOO_LARGE, "at most 2^28 sites" );
    apo2_options      opt {};
    const apo2_status ost = normalize_options( options, opt );
    if ( ost != APO2_OK )
        return ost;

    APO2_CUDA( cudaSetDevice( int( opt.device ) ), "cudaSetDevice" );
    apo2_handle * h = new ( std::nothrow ) apo2_handle {};
    if ( !h )
        return fail( APO2_ERR_OUT_OF_MEMORY, "host allocation" );
    h->n         = n;
    h->options   = opt;
    h->device    = int( opt.device );
    h->input_f64 = dtype == APO2_F64;
    configure_cell_kernels();

    configure_spec_kernels();
    const size_t total = arena_bytes( n, opt, h->input_f64 );
    h->arena.size      = total;
    cudaError_t err    = cudaMalloc( reinterpret_cast<void **>( &h->arena.base ), total );
    if ( err != cudaSuccess )
    {
        delete h;
        return cuda_fail( err, "device allocation" );
    }
    if ( !carve( h, n ) )
    {
        cudaFree( h->arena.base );
        delete h;
        return fail( APO2_ERR_CUDA, "arena accounting" );
    }
    cudaMemset( h->bounds_counter, 0, sizeof( uint32_t ) );
    cudaMemset( h->error, 0, sizeof( uint32_t ) );
    cudaMemset( h->out.totals, 0, 2 * sizeof( uint64_t ) );

    apo2_status st = ensure_output_capacity( h, 8 * uint64_t( n ) + 1024, uint64_t( n ) / 16 + 1024 );
    if ( st == APO2_OK )
    {
        h->timing = opt.stage_timing != 0;
        if ( h->timing )
            for ( auto & e : h->events )
                cudaEventCreate( &e );
        st = upload_sites( h, sites, dtype, location, 0 );
    }
    if ( st == APO2_OK )
    {
        err = cudaStreamSynchronize( 0 );
        if ( err != cudaSuccess )
            st = cuda_fail( err, "site upload" );
    }
    if ( st != APO2_OK )
    {
        apo2_destroy( h );
        return st;
    }
    h->stats.n            = n;
    h->stats.device_bytes = total + align256( sizeof( double4 ) * h->out.vcap ) * 2;
    *out                  = h;
    return APO2_OK;
}

apo2_status apo2_set_sites( apo2_handle * h, const void * sites, apo2_dtype dtype, apo2_location location, void * stream )
{
    if ( !h || !sites )
        return fail( APO2_ERR_INVALID_ARG, "null argument" );
    return upload_sites( h, sites, dtype, location, static_cast<cudaStream_t>( stream ) );
}

apo2_status apo2_build( apo2_handle * h, void * stream, int synchronize )
{
    if ( !h )
        return fail( APO2_ERR_INVALID_ARG, "null handle" );
    APO2_CUDA( cudaSetDevice( h->device ), "cudaSetDevice" );
    cudaStream_t s  = static_cast<cudaStream_t>( stream );
    apo2_status  st = enqueue_build( h, s );
    if ( st != APO2_OK || !synchronize )
        return st;
    return finish( h, s );
}

apo2_status apo2_build_and_extract( apo2_handle * h, void * stream )
{
    if ( !h )
        return fail( APO2_ERR_INVALID_ARG, "null handle" );
    APO2_CUDA( cudaSetDevice( h->device ), "cudaSetDevice" );
    cudaStream_t s  = static_cast<cudaStream_t>( stream );
    apo2_status  st = enqueue_build( h, s );
    if ( st != APO2_OK )
        return st;
    return enqueue_extract( h, s );
}

apo2_status apo2_output_counts( apo2_handle * h, uint64_t * vertices, uint64_t * closed )
{
    if ( !h )
        return fail( APO2_ERR_INVALID_ARG, "null handle" );
    apo2_status st = settle_output( h, 0 );
    if ( st != APO2_OK )
        return st;
    if ( vertices )
        *vertices = h->stats.output_vertices;
    if ( closed )
        *closed = h->stats.output_closed_edges;
    return APO2_OK;
}

apo2_status apo2_output_device( apo2_handle * h, const double ** vp, const uint32_t ** vi, const double ** cp, const uint32_t ** ci )
{
    if ( !h )
        return fail( APO2_ERR_INVALID_ARG, "null handle" );
    if ( !h->extracted )
        return fail( APO2_ERR_NOT_BUILT, "no extraction yet" );
    if ( vp )
        *vp = reinterpret_cast<const double *>( h->out.vpos );
    if ( vi )
        *vi = reinterpret_cast<const uint32_t *>( h->out.vids );
    if ( cp )
        *cp = reinterpret_cast<const double *>( h->out.cpos );
    if ( ci )
        *ci = reinterpret_cast<const uint32_t *>( h->out.cids );
    return APO2_OK;
}

static apo2_status copy_output( apo2_handle * h, bool closed, double * pos, uint32_t * ids, uint64_t capacity,
                                apo2_location location, uint64_t * written )
{
    if ( !h )
        return fail( APO2_ERR_INVALID_ARG, "null handle" );
    apo2_status st = settle_output( h, 0 );
    if ( st != APO2_OK )
        return st;
    const uint64_t count = closed ? h->stats.output_closed_edges : h->stats.output_vertices;
    if ( written )
        *written = count;
    if ( !pos && !ids )
        return APO2_OK;
    if ( capacity < count )
        return fail( APO2_ERR_INVALID_ARG, "output capacity too small" );
    const cudaMemcpyKind kind = location == APO2_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    if ( pos )
        APO2_CUDA( cudaMemcpy( pos, closed ? h->out.cpos : h->out.vpos, sizeof( double4 ) * count, kind ), "output copy" );
    if ( ids )
        APO2_CUDA( cudaMemcpy( ids, closed ? h->out.cids : h->out.vids, sizeof( uint4 ) * count, kind ), "output copy" );
    return APO2_OK;
}

apo2_status apo2_get_vertices( apo2_handle * h, double * positions, uint32_t * ids, uint64_t capacity, apo2_location location,
                               uint64_t * written )
{
    return copy_output( h, false, positions, ids, capacity, location, written );
}

apo2_status apo2_get_closed_edges( apo2_handle * h, double * positions, uint32_t * ids, uint64_t capacity,
                                   apo2_location location, uint64_t * written )
{
    return copy_output( h, true, positions, ids, capacity, location, written );
}

} // extern "C"

namespace
{
    // Unique bisectors, trisectors and quadrisectors, per sorted cell with the cell's id
    // smallest, mapped to original ids (algorithm.inl:1732-1821).
    apo2_status topology_arrays( apo2_handle * h, std::vector<uint32_t> & q, std::vector<uint32_t> & t, std::vector<uint32_t> & b )
    {
    APO2_CUDA( cudaDeviceSynchronize(), "topology" );
    const uint32_t n        = h->n;
    const auto     vnb      = download( h->cells.vertex_nb, n );
    const auto     enb      = download( h->cells.edge_nb, n );
    const CellContext & c   = h->cells;
    const auto     vertices = download( c.vertices, size_t( c.hi - c.lo ) * kMaxVertices );
    const auto     edges    = download( c.edges, size_t( c.hi - c.lo ) * kMaxEdges );
    const auto     ix       = download( h->tree.indices, n );
    std::vector<std::pair<uint32_t, uint32_t>> bis;
    std::vector<std::tuple<uint32_t, uint32_t>> tris;
    std::vector<std::tuple<uint32_t, uint32_t, uint32_t>> quads;
    for ( uint32_t i = h->cells.lo; i < h->cells.hi; i++ ) // this shard's cells
    {
        bis.clear();
        tris.clear();
        quads.clear();
        for ( uint32_t e = 0; e < std::min( enb[ i ], kMaxEdges ); e++ )
        {
            const uint4 r = edges[ store_row( c, i ) * kMaxEdges + e ];
            if ( i < r.x && r.x < n )
                bis.emplace_back( i, r.x );
            if ( i < r.y && r.y < n )
                bis.emplace_back( i, r.y );
            if ( i < r.x && i < r.y && r.x < n && r.y < n )
                tris.emplace_back( r.x, r.y );
        }
        for ( uint32_t v = 0; v < std::min( vnb[ i ], kMaxVertices ); v++ )
        {
            const uint4 r = vertices[ store_row( c, i ) * kMaxVertices + v ];
            if ( i < r.x && i < r.y && i < r.z && r.x < n && r.y < n && r.z < n )
                quads.emplace_back( r.x, r.y, r.z );
        }
        std::sort( bis.begin(), bis.end() );
        bis.erase( std::unique( bis.begin(), bis.end() ), bis.end() );
        std::sort( tris.begin(), tris.end() );
        tris.erase( std::unique( tris.begin(), tris.end() ), tris.end() );
        std::sort( quads.begin(), quads.end() );
        quads.erase( std::unique( quads.begin(), quads.end() ), quads.end() );
        for ( auto & x : bis )
            b.insert( b.end(), { ix[ x.first ], ix[ x.second ] } );
        for ( auto & x : tris )
            t.insert( t.end(), { ix[ i ], ix[ std::get<0>( x ) ], ix[ std::get<1>( x ) ] } );
        for ( auto & x : quads )
            q.insert( q.end(), { ix[ i ], ix[ std::get<0>( x ) ], ix[ std::get<1>( x ) ], ix[ std::get<2>( x ) ] } );
    }
    return APO2_OK;
    }
} // namespace

extern "C" {

apo2_status apo2_get_topology( apo2_handle * h, uint32_t * quad, uint64_t quad_cap, uint32_t * tri, uint64_t tri_cap,
                               uint32_t * bi, uint64_t bi_cap, uint64_t * quad_count, uint64_t * tri_count, uint64_t * bi_count )
{
    if ( !h )
        return fail( APO2_ERR_INVALID_ARG, "null handle" );
    if ( !h->built )
        return fail( APO2_ERR_NOT_BUILT, "no build yet" );
    std::vector<uint32_t> q, t, b;
    const apo2_status     st = topology_arrays( h, q, t, b );
    if ( st != APO2_OK )
        return st;
    if ( quad_count )
        *quad_count = q.size() / 4;
    if ( tri_count )
        *tri_count = t.size() / 3;
    if ( bi_count )
        *bi_count = b.size() / 2;
    if ( ( quad && quad_cap < q.size() / 4 ) || ( tri && tri_cap < t.size() / 3 ) || ( bi && bi_cap < b.size() / 2 ) )
        return fail( APO2_ERR_INVALID_ARG, "topology capacity too small" );
    if ( quad )
        std::memcpy( quad, q.data(), q.size() * 4 );
    if ( tri )
        std::memcpy( tri, t.data(), t.size() * 4 );
    if ( bi )
        std::memcpy( bi, b.data(), b.size() * 4 );
    return APO2_OK;
}

apo2_status apo2_topology_json( apo2_handle * h, char * json, uint64_t capacity, uint64_t * length )
{
    if ( !h || !length )
        return fail( APO2_ERR_INVALID_ARG, "null argument" );
    if ( !h->built )
        return fail( APO2_ERR_NOT_BUILT, "no build yet" );
    std::vector<uint32_t> q, t, b;
    const apo2_status     st = topology_arrays( h, q, t, b );
    if ( st != APO2_OK )
        return st;
    // the layout of the reference's topology writer (app/topology/topology.cpp:11-57)
    std::string out = "{\n\t\"bisectors\": [\n";
    char        line[ 96 ];
    const size_t nb = b.size() / 2, nt = t.size() / 3, nq = q.size() / 4;
    for ( size_t x = 0; x < nb; x++ )
    {
        std::snprintf( line, sizeof( line ), "\t\t[ %u, %u ]%s\n", b[ 2 * x ], b[ 2 * x + 1 ], x + 1 == nb ? "" : "," );
        out += line;
    }
    out += "\t],\n\t\"trisectors\": [\n";
    for ( size_t x = 0; x < nt; x++ )
    {
        std::snprintf( line, sizeof( line ), "\t\t[ %u, %u, %u ]%s\n", t[ 3 * x ], t[ 3 * x + 1 ], t[ 3 * x + 2 ], x + 1 == nt ? "" : "," );
        out += line;
    }
    out += "\t],\n\t\"quadrisectors\": [\n";
    for ( size_t x = 0; x < nq; x++ )
    {
        std::snprintf( line, sizeof( line ), "\t\t[ %u, %u, %u, %u ]%s\n", q[ 4 * x ], q[ 4 * x + 1 ], q[ 4 * x + 2 ], q[ 4 * x + 3 ],
                       x + 1 == nq ? "" : "," );
        out += line;
    }
    out += "\t]\n}\n";
    *length = out.size();
    if ( json )
    {
        if ( capacity < out.size() + 1 )
            return fail( APO2_ERR_INVALID_ARG, "json capacity too small" );
        std::memcpy( json, out.c_str(), out.size() + 1 );
    }
    return APO2_OK;
}

apo2_status apo2_certify( apo2_handle * h, const double * positions, const uint32_t * ids, uint64_t count, uint32_t arity,
                          apo2_location location, uint8_t * flags, uint64_t * bad )
{
    if ( !h || !bad || ( arity != 3 && arity != 4 ) || ( ( positions == nullptr ) != ( ids == nullptr ) )
         || ( location != APO2_HOST && location != APO2_DEVICE ) )
        return fail( APO2_ERR_INVALID_ARG, "invalid argument to apo2_certify" );
    if ( !h->built )
        return fail( APO2_ERR_NOT_BUILT, "no build yet" );
    APO2_CUDA( cudaSetDevice( h->device ), "cudaSetDevice" );
    const double4 * P = nullptr;
    const uint4 *   I = nullptr;
    void *          scratch = nullptr;
    if ( !positions )
    {
        // the handle's own extracted output
        apo2_status st = settle_output( h, 0 );
        if ( st != APO2_OK )
            return st;
        uint64_t totals[ 2 ];
        APO2_CUDA( cudaMemcpy( totals, h->out.totals, sizeof( totals ), cudaMemcpyDeviceToHost ), "output totals" );
        count = arity == 4 ? totals[ 0 ] : totals[ 1 ];
        P     = arity == 4 ? h->out.vpos : h->out.cpos;
        I     = arity == 4 ? h->out.vids : h->out.cids;
    }
    const size_t flag_bytes = align256( std::max<uint64_t>( count, 1 ) );
    const size_t in_bytes   = positions && location == APO2_HOST ? align256( sizeof( double4 ) * count ) + align256( sizeof( uint4 ) * count ) : 0;
    APO2_CUDA( cudaMalloc( &scratch, 256 + flag_bytes + in_bytes ), "certify scratch" );
    char *               base  = static_cast<char *>( scratch );
    unsigned long long * dbad  = reinterpret_cast<unsigned long long *>( base );
    uint8_t *            dflag = reinterpret_cast<uint8_t *>( base + 256 );
    if ( positions )
    {
        if ( location == APO2_HOST )
        {
            double4 * dp = reinterpret_cast<double4 *>( base + 256 + flag_bytes );
            uint4 *   di = reinterpret_cast<uint4 *>( base + 256 + flag_bytes + align256( sizeof( double4 ) * count ) );
            cudaMemcpy( dp, positions, sizeof( double4 ) * count, cudaMemcpyHostToDevice );
            cudaMemcpy( di, ids, sizeof( uint4 ) * count, cudaMemcpyHostToDevice );
            P = dp;
            I = di;
        }
        else
        {
            P = reinterpret_cast<const double4 *>( positions );
            I = reinterpret_cast<const uint4 *>( ids );
        }
    }
    cudaMemset( dbad, 0, sizeof( unsigned long long ) );
    cudaMemset( h->error, 0, sizeof( uint32_t ) );
    Scene scene;
    cudaMemcpy( &scene, h->scene, sizeof( Scene ), cudaMemcpyDeviceToHost );
    if ( count )
    {
        ObserveScope observe( h );
        launch_certify( h->input_d4, h->tree.sites, h->tree.indices, h->tree.nodes, h->n, P, I, arity, count, float( scene.rmax ),
                        dflag, dbad, h->error, 0 );
    }
    unsigned long long nbad = 0;
    uint32_t           err  = 0;
    cudaError_t        e    = cudaDeviceSynchronize();
    if ( e == cudaSuccess )
        e = cudaMemcpy( &nbad, dbad, sizeof( nbad ), cudaMemcpyDeviceToHost );
    if ( e == cudaSuccess )
        e = cudaMemcpy( &err, h->error, sizeof( err ), cudaMemcpyDeviceToHost );
    if ( e == cudaSuccess && flags && count )
        e = cudaMemcpy( flags, dflag, count, cudaMemcpyDeviceToHost );
    cudaFree( scratch );
    if ( e != cudaSuccess )
        return cuda_fail( e, "certify" );
    if ( err )
        return fail( APO2_ERR_CAPACITY, "certify walk flags " + std::to_string( err ) );
    *bad = nbad;
    return APO2_OK;
}

apo2_status apo2_vertex_error( apo2_handle * h, const double * positions, const uint32_t * ids, uint64_t count,
                               apo2_location location, double threshold, float * errors, double * max_error, uint64_t * above,
                               uint64_t * singular )
{
    if ( !h || !max_error || ( ( positions == nullptr ) != ( ids == nullptr ) )
         || ( location != APO2_HOST && location != APO2_DEVICE ) || !( threshold >= 0.0 ) )
        return fail( APO2_ERR_INVALID_ARG, "invalid argument to apo2_vertex_error" );
    if ( !h->built )
        return fail( APO2_ERR_NOT_BUILT, "no build yet" );
    APO2_CUDA( cudaSetDevice( h->device ), "cudaSetDevice" );
    const double4 * P = nullptr;
    const uint4 *   I = nullptr;
    if ( !positions )
    {
        apo2_status st = settle_output( h, 0 );
        if ( st != APO2_OK )
            return st;
        count = h->stats.output_vertices;
        P     = h->out.vpos;
        I     = h->out.vids;
    }
    const size_t err_bytes = errors ? align256( sizeof( float ) * std::max<uint64_t>( count, 1 ) ) : 0;
    const size_t in_bytes  = positions && location == APO2_HOST ? align256( sizeof( double4 ) * count ) + align256( sizeof( uint4 ) * count ) : 0;
    void *       scratch   = nullptr;
    APO2_CUDA( cudaMalloc( &scratch, 256 + err_bytes + in_bytes ), "vertex error scratch" );
    char *               base   = static_cast<char *>( scratch );
    unsigned long long * counts = reinterpret_cast<unsigned long long *>( base ); // max bits, above, singular
    float *              derr   = errors ? reinterpret_cast<float *>( base + 256 ) : nullptr;
    cudaError_t          e      = cudaSuccess;
    if ( positions )
    {
        if ( location == APO2_HOST )
        {
            double4 * dp = reinterpret_cast<double4 *>( base + 256 + err_bytes );
            uint4 *   di = reinterpret_cast<uint4 *>( base + 256 + err_bytes + align256( sizeof( double4 ) * count ) );
            e            = cudaMemcpy( dp, positions, sizeof( double4 ) * count, cudaMemcpyHostToDevice );
            if ( e == cudaSuccess )
                e = cudaMemcpy( di, ids, sizeof( uint4 ) * count, cudaMemcpyHostToDevice );
            P = dp;
            I = di;
        }
        else
        {
            P = reinterpret_cast<const double4 *>( positions );
            I = reinterpret_cast<const uint4 *>( ids );
        }
    }
    if ( e == cudaSuccess )
        e = cudaMemset( counts, 0, 3 * sizeof( unsigned long long ) );
    if ( e == cudaSuccess && count )
    {
        ObserveScope observe( h );
        launch_vertex_error( h->input_d4, h->n, P, I, count, threshold, derr, counts, counts + 1, counts + 2, 0 );
        e = cudaGetLastError();
    }
    unsigned long long host[ 3 ] = {};
    if ( e == cudaSuccess )
        e = cudaDeviceSynchronize();
    if ( e == cudaSuccess )
        e = cudaMemcpy( host, counts, sizeof( host ), cudaMemcpyDeviceToHost );
    if ( e == cudaSuccess && errors && count )
        e = cudaMemcpy( errors, derr, sizeof( float ) * count, cudaMemcpyDeviceToHost );
    cudaFree( scratch );
    if ( e != cudaSuccess )
        return cuda_fail( e, "vertex error" );
    double mx = 0.0;
    std::memcpy( &mx, &host[ 0 ], sizeof( mx ) );
    *max_error = mx;
    if ( above )
        *above = host[ 1 ];
    if ( singular )
        *singular = host[ 2 ];
    return APO2_OK;
}

apo2_status apo2_cavity_directions( uint32_t count, float * xyz )
{
    if ( !xyz || count == 0 || count > kCavityMaxSamples )
        return fail( APO2_ERR_INVALID_ARG, "invalid argument to apo2_cavity_directions" );
    cavity_directions( count, xyz, nullptr );
    return APO2_OK;
}

apo2_status apo2_cavity_hit_ratios( apo2_handle * h, const float * spheres, uint32_t sphere_count, apo2_location location,
                                    uint32_t samples, float * hit_ratios, uint64_t capacity, uint64_t * count, float * ms )
{
    if ( !h || !count || ( !spheres && sphere_count ) || samples == 0 || samples > kCavityMaxSamples
         || ( location != APO2_HOST && location != APO2_DEVICE ) )
        return fail( APO2_ERR_INVALID_ARG, "invalid argument to apo2_cavity_hit_ratios" );
    APO2_CUDA( cudaSetDevice( h->device ), "cudaSetDevice" );
    apo2_status st = settle_output( h, 0 );
    if ( st != APO2_OK )
        return st;
    const uint64_t q = h->stats.output_vertices;
    if ( hit_ratios && capacity < q )
    {
        *count = q;
        return fail( APO2_ERR_INVALID_ARG, "hit ratio capacity too small" );
    }
    if ( q > UINT32_MAX )
        return fail( APO2_ERR_TOO_LARGE, "more than 2^32 - 1 vertices" );
    // persistent: ratios, filter offsets and scan sums of q vertices
    const size_t keep = align256( sizeof( float ) * std::max<uint64_t>( q, 1 ) ) + align256( sizeof( uint32_t ) * std::max<uint64_t>( q, 1 ) )
                        + align256( sizeof( uint32_t ) * output_scan_scratch_words( uint32_t( q ) ) ) + 256;
    if ( keep > h->cavity_bytes )
    {
        if ( h->cavity_alloc )
            cudaFree( h->cavity_alloc );
        h->cavity_alloc = nullptr;
        h->cavity_bytes = 0;
        APO2_CUDA( cudaMalloc( &h->cavity_alloc, keep ), "cavity buffers" );
        h->cavity_bytes = keep;
    }
    h->ratios      = static_cast<float *>( h->cavity_alloc );
    h->ratio_epoch = ~0ull;
    // per call: the sphere tree, the spheres (host input) and the direction table
    const size_t tree_bytes  = trace_tree_bytes( sphere_count );
    const size_t copy_bytes  = location == APO2_HOST ? align256( sizeof( float4 ) * std::max<uint32_t>( sphere_count, 1 ) ) : 0;
    const size_t dir_bytes   = align256( sizeof( float4 ) * 2 * samples );
    void *       scratch     = nullptr;
    APO2_CUDA( cudaMalloc( &scratch, tree_bytes + copy_bytes + dir_bytes ), "cavity scratch" );
    char *         base  = static_cast<char *>( scratch );
    float4 *       dirs  = reinterpret_cast<float4 *>( base + tree_bytes + copy_bytes );
    const float4 * trace = reinterpret_cast<const float4 *>( spheres );
    std::vector<float> table( 8 * size_t( samples ) );
    cavity_directions( samples, nullptr, table.data() );
    cudaEvent_t ev[ 3 ] = {};
    for ( auto & e : ev )
        cudaEventCreate( &e );
    cudaError_t e = cudaSuccess;
    if ( location == APO2_HOST && sphere_count )
    {
        float4 * copy = reinterpret_cast<float4 *>( base + tree_bytes );
        e             = cudaMemcpyAsync( copy, spheres, sizeof( float4 ) * sphere_count, cudaMemcpyHostToDevice, 0 );
        trace         = copy;
    }
    if ( e == cudaSuccess )
        e = cudaMemcpyAsync( dirs, table.data(), sizeof( float ) * table.size(), cudaMemcpyHostToDevice, 0 );
    if ( e == cudaSuccess )
        e = cudaMemsetAsync( h->error, 0, sizeof( uint32_t ), 0 );
    if ( e == cudaSuccess )
    {
        ObserveScope observe( h );
        TraceTree    tree;
        trace_tree_carve( tree, base, sphere_count, h->error );
        cudaEventRecord( ev[ 0 ], 0 );
        launch_trace_tree( tree, trace, 0 );
        cudaEventRecord( ev[ 1 ], 0 );
        launch_occlusion( tree, trace, h->out.vpos, h->out.vids, q, dirs, samples, h->ratios, h->error, 0 );
        cudaEventRecord( ev[ 2 ], 0 );
        e = cudaGetLastError();
    }
    if ( e == cudaSuccess )
        e = cudaStreamSynchronize( 0 );
    uint32_t err = 0;
    if ( e == cudaSuccess )
        e = cudaMemcpy( &err, h->error, sizeof( err ), cudaMemcpyDeviceToHost );
    if ( e == cudaSuccess && hit_ratios && q )
        e = cudaMemcpy( hit_ratios, h->ratios, sizeof( float ) * q, cudaMemcpyDeviceToHost );
    if ( e == cudaSuccess && ms )
    {
        cudaEventElapsedTime( &ms[ 0 ], ev[ 0 ], ev[ 1 ] );
        cudaEventElapsedTime( &ms[ 1 ], ev[ 1 ], ev[ 2 ] );
    }
    for ( auto & x : ev )
        cudaEventDestroy( x );
    cudaFree( scratch );
    if ( e != cudaSuccess )
        return cuda_fail( e, "cavity hit ratios" );
    if ( err )
        return fail( APO2_ERR_CAPACITY, "ray walk flags " + std::to_string( err ) );
    h->ratio_count = q;
    h->ratio_epoch = h->extract_epoch;
    *count         = q;
    return APO2_OK;
}

apo2_status apo2_cavity_vertices( apo2_handle * h, float hit_ratio_threshold, float radius_threshold, float * xyzw,
                                  uint64_t capacity, uint64_t * count )
{
    if ( !h || !count )
        return fail( APO2_ERR_INVALID_ARG, "invalid argument to apo2_cavity_vertices" );
    if ( !h->built || h->ratio_epoch != h->extract_epoch )
        return fail( APO2_ERR_NOT_BUILT, "no hit ratios for the last build (apo2_cavity_hit_ratios)" );
    APO2_CUDA( cudaSetDevice( h->device ), "cudaSetDevice" );
    const uint64_t q       = h->ratio_count;
    char *         base    = static_cast<char *>( h->cavity_alloc );
    uint32_t *     offsets = reinterpret_cast<uint32_t *>( base + align256( sizeof( float ) * std::max<uint64_t>( q, 1 ) ) );
    uint32_t *     sums    = offsets + align256( sizeof( uint32_t ) * std::max<uint64_t>( q, 1 ) ) / sizeof( uint32_t );
    uint64_t *     total   = reinterpret_cast<uint64_t *>( base + h->cavity_bytes - 256 );
    float4 *       out     = nullptr;
    if ( xyzw && capacity )
        APO2_CUDA( cudaMalloc( &out, sizeof( float4 ) * capacity ), "cavity output" );
    {
        ObserveScope observe( h );
        launch_cavity_filter( h->out.vpos, h->ratios, q, hit_ratio_threshold, radius_threshold, offsets, sums, total, out,
                              capacity, 0 );
    }
    uint64_t    found = 0;
    cudaError_t e     = cudaGetLastError();
    if ( e == cudaSuccess )
        e = cudaMemcpy( &found, total, sizeof( found ), cudaMemcpyDeviceToHost );
    if ( e == cudaSuccess && out && found )
        e = cudaMemcpy( xyzw, out, sizeof( float4 ) * std::min( found, capacity ), cudaMemcpyDeviceToHost );
    if ( out )
        cudaFree( out );
    if ( e != cudaSuccess )
        return cuda_fail( e, "cavity vertices" );
    *count = found;
    if ( xyzw && found > capacity )
        return fail( APO2_ERR_INVALID_ARG, "cavity vertex capacity too small" );
    return APO2_OK;
}

apo2_status apo2_contribution_profile( apo2_handle * h, uint32_t steps, uint8_t * contributed, uint8_t * certified )
{
    if ( !h || !contributed || !certified || steps == 0 || steps > 64 )
        return fail( APO2_ERR_INVALID_ARG, "invalid argument to apo2_contribution_profile" );
    APO2_CUDA( cudaSetDevice( h->device ), "cudaSetDevice" );
    const uint32_t n   = h->n;
    const uint32_t row = steps * h->cells.k;
    const size_t   bytes = size_t( n ) * row;
    void *         buf   = nullptr;
    APO2_CUDA( cudaMalloc( &buf, 2 * bytes ), "profile buffers" );
    uint8_t * dc = static_cast<uint8_t *>( buf );
    uint8_t * dr = dc + bytes;
    cudaMemset( buf, 0, 2 * bytes );
    {
        ObserveScope observe( h );
        h->launches    = 0;
        h->events_used = 0;
        h->records.clear();
        cudaStream_t s = 0;
        cudaMemsetAsync( h->error, 0, sizeof( uint32_t ), s );
        launch_bounds( h->input, h->input_f64, n, h->input_d4, h->partials, h->partial_count, h->bounds_counter, h->scene,
                       h->tree.sites + n, s );
        launch_tree( h->tree, n, h->input_d4, h->scene, h->sort, s, h->options.wait_limit );
        // the labels are the plain construction's: no proposal takes part
        CellContext plain  = h->cells;
        plain.proposal     = nullptr;
        plain.proposed_k   = nullptr;
        plain.scheduled    = 0;
        for ( uint32_t step = 0; step < steps; step++ )
        {
            launch_knn( plain, step, s );
            launch_cells_profile( plain, step, row, dc, dr, s );
        }
    }
    uint32_t    err = 0;
    cudaError_t e   = cudaDeviceSynchronize();
    if ( e == cudaSuccess )
        e = cudaMemcpy( contributed, dc, bytes, cudaMemcpyDeviceToHost );
    if ( e == cudaSuccess )
        e = cudaMemcpy( certified, dr, bytes, cudaMemcpyDeviceToHost );
    if ( e == cudaSuccess )
        e = cudaMemcpy( &err, h->error, sizeof( err ), cudaMemcpyDeviceToHost );
    cudaFree( buf );
    h->built     = false; // the stores hold the profile run, not a build
    h->extracted = false;
    if ( e != cudaSuccess )
        return cuda_fail( e, "contribution profile" );
    if ( err )
        return fail( APO2_ERR_CAPACITY, "capacity flags " + std::to_string( err ) );
    return APO2_OK;
}

apo2_status apo2_get_cell( apo2_handle * h, uint32_t site, uint32_t * vertices, uint32_t vcap, uint32_t * vcount,
                           uint32_t * edges, uint32_t ecap, uint32_t * ecount )
{
    if ( !h || site >= h->n )
        return fail( APO2_ERR_INVALID_ARG, "invalid site" );
    if ( !h->built )
        return fail( APO2_ERR_NOT_BUILT, "no build yet" );
    APO2_CUDA( cudaDeviceSynchronize(), "cell" );
    const auto ix = download( h->tree.indices, h->n );
    uint32_t   sorted = 0;
    while ( sorted < h->n && ix[ sorted ] != site )
        sorted++;
    if ( sorted < h->cells.lo || sorted >= h->cells.hi )
        return fail( APO2_ERR_INVALID_ARG, "the site's cell belongs to another shard" );
    uint32_t vn = 0, en = 0;
    cudaMemcpy( &vn, h->cells.vertex_nb + sorted, 4, cudaMemcpyDeviceToHost );
    cudaMemcpy( &en, h->cells.edge_nb + sorted, 4, cudaMemcpyDeviceToHost );
    vn            = std::min( vn, kMaxVertices );
    en            = std::min( en, kMaxEdges );
    const auto vr = download( h->cells.vertices + store_row( h->cells, sorted ) * kMaxVertices, vn );
    const auto er = download( h->cells.edges + store_row( h->cells, sorted ) * kMaxEdges, en );
    auto       map = [ & ]( uint32_t id ) { return id < h->n ? ix[ id ] : id; };
    if ( vcount )
        *vcount = vn;
    if ( ecount )
        *ecount = en;
    if ( vertices )
        for ( uint32_t v = 0; v < std::min( vn, vcap ); v++ )
        {
            vertices[ 4 * v + 0 ] = map( vr[ v ].x );
            vertices[ 4 * v + 1 ] = map( vr[ v ].y );
            vertices[ 4 * v + 2 ] = map( vr[ v ].z );
            vertices[ 4 * v + 3 ] = vr[ v ].w & 0xffu;
        }
    if ( edges )
        for ( uint32_t e = 0; e < std::min( en, ecap ); e++ )
        {
            edges[ 3 * e + 0 ] = map( er[ e ].x );
            edges[ 3 * e + 1 ] = map( er[ e ].y );
            edges[ 3 * e + 2 ] = er[ e ].z;
        }
    return APO2_OK;
}

apo2_status apo2_debug_array( apo2_handle * h, const char * name, void * dst, uint64_t capacity_bytes, uint64_t * count )
{
    if ( !h || !name )
        return fail( APO2_ERR_INVALID_ARG, "null argument" );
    APO2_CUDA( cudaDeviceSynchronize(), "debug array" );
    const uint32_t    n     = h->n;
    const uint64_t    nodes = 2 * uint64_t( n ) - 1;
    const std::string key( name );
    const void *      src   = nullptr;
    uint64_t          elems = 0, esize = 4;
    std::vector<uint32_t> packed;
    if ( key == "indices" )
        src = h->tree.indices, elems = n;
    else if ( key == "parent" )
        src = h->tree.parent, elems = nodes;
    else if ( key == "left" )
        src = h->tree.left, elems = nodes;
    else if ( key == "right" )
        src = h->tree.right, elems = nodes;
    else if ( key == "aabb" )
        src = h->tree.boxes, elems = nodes * 8;
    else if ( key == "sizes" )
        src = h->tree.sizes, elems = nodes;
    else if ( key == "morton" )
        src = h->tree.codes, elems = n, esize = 8;
    else if ( key == "sites_sorted" )
        src = h->tree.sites, elems = 4 * ( uint64_t( n ) + kArtificial ), esize = 8;
    else if ( key == "status" )
        src = h->cells.status, elems = n, esize = 1;
    else if ( key == "knn" )
        src = h->cells.knn, elems = uint64_t( n ) * h->cells.k;
    else if ( key == "known_radii" )
        src = h->cells.known_radii, elems = n;
    else if ( key == "proposed_k" )
    {
        if ( !h->cells.proposed_k )
            return fail( APO2_ERR_INVALID_ARG, "no k-proposal attached" );
        src = h->cells.proposed_k, elems = n, esize = 1;
    }
    else if ( key == "vertex_nb" )
        src = h->cells.vertex_nb, elems = n;
    else if ( key == "edge_nb" )
        src = h->cells.edge_nb, elems = n;
    else if ( key == "vertices" || key == "edges" )
    {
        const bool  isV  = key == "vertices";
        const auto  nb   = download( isV ? h->cells.vertex_nb : h->cells.edge_nb, n );
        const uint32_t cap = isV ? kMaxVertices : kMaxEdges;
        const CellContext & c = h->cells;
        const auto  all  = download( isV ? c.vertices : c.edges, size_t( c.hi - c.lo ) * cap );
        for ( uint32_t i = c.lo; i < c.hi; i++ ) // the stores hold this shard's cells
            for ( uint32_t r = 0; r < std::min( nb[ i ], cap ); r++ )
            {
                const uint4 x = all[ store_row( c, i ) * cap + r ];
                packed.insert( packed.end(), { x.x, x.y, x.z, x.w } );
            }
        elems = packed.size();
    }
    else
        return fail( APO2_ERR_INVALID_ARG, "unknown array " + key );
    if ( count )
        *count = elems;
    if ( !dst )
        return APO2_OK;
    if ( capacity_bytes < elems * esize )
        return fail( APO2_ERR_INVALID_ARG, "capacity too small" );
    if ( !packed.empty() )
        std::memcpy( dst, packed.data(), elems * esize );
    else if ( elems )
        APO2_CUDA( cudaMemcpy( dst, src, elems * esize, cudaMemcpyDeviceToHost ), "debug copy" );
    return APO2_OK;
}

apo2_status apo2_get_stats( apo2_handle * h, apo2_stats * stats )
{
    if ( !h || !stats )
        return fail( APO2_ERR_INVALID_ARG, "null argument" );
    APO2_CUDA( cudaDeviceSynchronize(), "stats" );
    const uint32_t n = h->n;
    const auto     status = download( h->cells.status, n );
    const auto     vnb    = download( h->cells.vertex_nb, n );
    const auto     enb    = download( h->cells.edge_nb, n );
    uint32_t       err    = 0;
    cudaMemcpy( &err, h->error, 4, cudaMemcpyDeviceToHost );
    uint32_t counts[ kMaxRounds + 1 ] = {};
    cudaMemcpy( counts, h->task_counts, 4 * ( h->options.max_iterations + 1 ), cudaMemcpyDeviceToHost );
    apo2_stats s = h->stats;
    s.n          = n;
    s.buried = 0;
    s.vertex_records = 0;
    s.edge_records   = 0;
    for ( uint32_t i = h->cells.lo; i < h->cells.hi; i++ ) // this shard's cells
    {
        s.buried += status[ i ] == kBuried;
        s.vertex_records += vnb[ i ];
        s.edge_records += enb[ i ];
    }
    s.certified_after_knn = ( h->cells.hi - h->cells.lo ) - s.buried - counts[ 0 ];
    s.validation_rounds   = 0;
    for ( uint32_t r = 0; r < h->options.max_iterations; r++ )
        s.validation_rounds += counts[ r ] != 0;
    s.error_flags     = err;
    s.uncertified     = h->options.stop_after == 0 ? counts[ h->options.max_iterations ] : 0;
    unsigned long long cnt[ kCounters ] = {};
    cudaMemcpy( cnt, h->cells.counters, sizeof( cnt ), cudaMemcpyDeviceToHost );
    s.knn_insertions     = cnt[ kCountInsertions ];
    s.proposal_cells     = cnt[ kCountChecked ];
    s.proposal_fallbacks = cnt[ kCountFallbacks ];
    s.proposal_skipped   = cnt[ kCountSkipped ];
    s.filter_tests       = cnt[ kCountFiltered ];
    s.proposal_second_step = cnt[ kCountSecondStep ];
    s.filter_escalations = cnt[ kCountEscalated ];
    s.kernel_launches = h->launches;
    if ( h->timing && h->built )
    {
        // the output span's closing event is recorded by an extraction only; an elapsed time
        // asked of an unrecorded event would fail and leave a stale error behind
        float      ms[ kStages ] = {};
        const int  spans         = h->extracted ? 7 : 6;
        for ( int e = 0; e < spans; e++ )
            if ( cudaEventElapsedTime( &ms[ e ], h->events[ e ], h->events[ e + 1 ] ) != cudaSuccess )
            {
                ms[ e ] = 0.f;
                cudaGetLastError();
            }
        s.ms_bounds              = ms[ 0 ];
        s.ms_tree                = ms[ 1 ];
        s.ms_knn                 = ms[ 2 ];
        s.ms_cells               = ms[ 3 ];
        s.ms_vertex_validation   = ms[ 4 ]; // vertex and edge rounds together
        s.ms_bisector_validation = ms[ 5 ];
        s.ms_output              = h->extracted ? ms[ 6 ] : 0.0;
    }
    *stats = s;
    return APO2_OK;
}

apo2_status apo2_kernel_profile( apo2_handle * h, char * json, uint64_t capacity, uint64_t * length )
{
    if ( !h )
        return fail( APO2_ERR_INVALID_ARG, "null handle" );
    APO2_CUDA( cudaDeviceSynchronize(), "kernel profile" );
    struct PerKernel
    {
        uint32_t launches = 0;
        double   total_ms = 0.0, max_ms = 0.0;
    };
    std::map<std::string, PerKernel> per;
    for ( const auto & r : h->records )
    {
        float ms = 0.f;
        if ( r.end >= 0 && cudaEventElapsedTime( &ms, h->event_pool[ r.begin ], h->event_pool[ r.end ] ) != cudaSuccess )
        {
            ms = 0.f;
            cudaGetLastError();
        }
        auto & x = per[ r.name ];
        x.launches++;
        x.total_ms += ms;
        x.max_ms = std::max( x.max_ms, double( ms ) );
    }
    std::string out = "{\"launches\": " + std::to_string( h->launches ) + ", \"timed\": " + ( h->timing ? "true" : "false" )
                      + ", \"kernels\": {";
    bool first = true;
    for ( const auto & kv : per )
    {
        char buf[ 192 ];
        std::snprintf( buf, sizeof( buf ), "%s\"%s\": [%u, %.6f, %.6f]", first ? "" : ", ", kv.first.c_str(),
                       kv.second.launches, kv.second.total_ms, kv.second.max_ms );
        out += buf;
        first = false;
    }
    out += "}}";
    if ( length )
        *length = out.size();
    if ( json )
    {
        if ( capacity <= out.size() )
            return fail( APO2_ERR_INVALID_ARG, "profile buffer too small" );
        std::memcpy( json, out.c_str(), out.size() + 1 );
    }
    return APO2_OK;
}

apo2_status apo2_set_precision( apo2_handle * h, uint32_t precision )
{
    if ( !h || precision > APO2_PRECISION_FP32_FILTER )
        return fail( APO2_ERR_INVALID_ARG, "invalid argument to apo2_set_precision" );
    APO2_CUDA( cudaSetDevice( h->device ), "cudaSetDevice" );
    APO2_CUDA( cudaDeviceSynchronize(), "set precision" ); // no build may still run with the old one
    h->options.precision = precision;
    h->cells.fp32        = precision == APO2_PRECISION_FP32_FILTER ? 1u : 0u;
    return APO2_OK;
}

apo2_status apo2_set_proposal( apo2_handle * h, const apo2_proposal * model )
{
    if ( !h || ( model && ( model->struct_size != sizeof( apo2_proposal ) || model->version != 1 ) ) )
        return fail( APO2_ERR_INVALID_ARG, "invalid argument to apo2_set_proposal" );
    APO2_CUDA( cudaSetDevice( h->device ), "cudaSetDevice" );
    APO2_CUDA( cudaDeviceSynchronize(), "set proposal" ); // no build may still read the old model
    if ( !model )
    {
        h->cells.proposal     = nullptr;
        h->cells.proposed_k   = nullptr;
        h->cells.scheduled    = 0;
        h->cells.proposal_max = 0;
        return APO2_OK;
    }
    const uint32_t k = h->cells.k;
    if ( model->max_rank > std::min( 2 * k, 255u ) )
        return fail( APO2_ERR_INVALID_ARG, "apo2_proposal.max_rank is at most 2K" );
    if ( !h->proposal_alloc )
        APO2_CUDA( cudaMalloc( &h->proposal_alloc, align256( sizeof( ProposalNet ) ) + align256( h->n ) ), "proposal allocation" );
    char * p = static_cast<char *>( h->proposal_alloc );
    APO2_CUDA( cudaMemcpy( p, reinterpret_cast<const char *>( model ) + kProposalHeader, sizeof( ProposalNet ),
                           cudaMemcpyHostToDevice ),
               "proposal upload" );
    h->cells.proposal     = reinterpret_cast<const ProposalNet *>( p );
    h->cells.proposed_k   = reinterpret_cast<uint8_t *>( p + align256( sizeof( ProposalNet ) ) );
    h->cells.proposal_max = model->max_rank ? model->max_rank : k;
    // the second step applies to builds of one configured kNN step; with several, every cell
    // takes them all (the reference's schedule) and proposals only place the first check
    h->cells.scheduled = ( h->cells.proposal_max > k && h->options.knn_steps == 1 ) ? 1u : 0u;
    return APO2_OK;
}

apo2_status apo2_proposal_features( apo2_handle * h, float * features )
{
    if ( !h || !features )
        return fail( APO2_ERR_INVALID_ARG, "invalid argument to apo2_proposal_features" );
    if ( !h->built )
        return fail( APO2_ERR_NOT_BUILT, "no build yet" );
    if ( h->options.knn_steps != 1 )
        return fail( APO2_ERR_INVALID_ARG, "features need the first kNN step's lists (knn_steps = 1)" );
    APO2_CUDA( cudaSetDevice( h->device ), "cudaSetDevice" );
    float * d = nullptr;
    APO2_CUDA( cudaMalloc( &d, sizeof( float ) * kPIn * size_t( h->n ) ), "features allocation" );
    FeatureInputs in;
    in.sites_f = h->cells.sites_f;
    in.codes   = h->cells.codes;
    in.scene   = h->scene;
    in.n       = h->n;
    {
        ObserveScope observe( h );
        launch_features( in, h->cells.knn, h->cells.k, d, 0 );
    }
    cudaError_t e = cudaGetLastError();
    if ( e == cudaSuccess )
        e = cudaMemcpy( features, d, sizeof( float ) * kPIn * size_t( h->n ), cudaMemcpyDeviceToHost );
    cudaFree( d );
    if ( e != cudaSuccess )
        return cuda_fail( e, "features" );
    return APO2_OK;
}

apo2_status apo2_destroy( apo2_handle * h )
{
    if ( !h )
        return APO2_OK;
    cudaSetDevice( h->device );
    cudaDeviceSynchronize();
    if ( h->out_alloc )
        cudaFree( h->out_alloc );
    if ( h->cavity_alloc )
        cudaFree( h->cavity_alloc );
    if ( h->proposal_alloc )
        cudaFree( h->proposal_alloc );
    if ( h->arena.base )
        cudaFree( h->arena.base );
    if ( h->timing )
        for ( auto & e : h->events )
            if ( e )
                cudaEventDestroy( e );
    for ( auto e : h->event_pool )
        cudaEventDestroy( e );
    delete h;
    return APO2_OK;
}

static apo2_status compute( const void * sites, uint32_t n, apo2_dtype dtype, double ** positions, uint32_t ** ids,
                            uint64_t * count, double ** cpos, uint32_t ** cids, uint64_t * ccount )
{
    apo2_handle * h  = nullptr;
    apo2_status   st = apo2_create( sites, n, dtype, APO2_HOST, nullptr, &h );
    if ( st != APO2_OK )
        return st;
    st = apo2_build_and_extract( h, nullptr );
    if ( st == APO2_OK )
        st = finish( h, 0 );
    uint64_t vc = 0, cc = 0;
    if ( st == APO2_OK )
        st = apo2_output_counts( h, &vc, &cc );
    if ( st == APO2_OK )
    {
        *positions = static_cast<double *>( std::malloc( sizeof( double ) * 4 * std::max<uint64_t>( vc, 1 ) ) );
        *ids       = static_cast<uint32_t *>( std::malloc( sizeof( uint32_t ) * 4 * std::max<uint64_t>( vc, 1 ) ) );
        st         = apo2_get_vertices( h, *positions, *ids, vc, APO2_HOST, count );
    }
    if ( st == APO2_OK && cpos )
    {
        *cpos = static_cast<double *>( std::malloc( sizeof( double ) * 4 * std::max<uint64_t>( cc, 1 ) ) );
        *cids = static_cast<uint32_t *>( std::malloc( sizeof( uint32_t ) * 4 * std::max<uint64_t>( cc, 1 ) ) );
        st    = apo2_get_closed_edges( h, *cpos, *cids, cc, APO2_HOST, ccount );
    }
    apo2_destroy( h );
    return st;
}

apo2_status apo2_compute_diagram( const void * sites, uint32_t n, apo2_dtype dtype, double ** positions, uint32_t ** ids,
                                  uint64_t * count )
{
    if ( !positions || !ids || !count )
        return fail( APO2_ERR_INVALID_ARG, "null output" );
    return compute( sites, n, dtype, positions, ids, count, nullptr, nullptr, nullptr );
}

apo2_status apo2_compute_full_diagram( const void * sites, uint32_t n, apo2_dtype dtype, double ** positions, uint32_t ** ids,
                                       uint64_t * count, double ** cpos, uint32_t ** cids, uint64_t * ccount )
{
    if ( !positions || !ids || !count || !cpos || !cids || !ccount )
        return fail( APO2_ERR_INVALID_ARG, "null output" );
    return compute( sites, n, dtype, positions, ids, count, cpos, cids, ccount );
}

void apo2_free( void * p ) { std::free( p ); }

uint64_t apo2_lbvh_scratch_bytes( uint32_t n ) { return sort_scratch_bytes( n ) + align256( 4 * size_t( n ) ) + 256; }

apo2_status apo2_lbvh_build( const float * sites, uint32_t n, const float scene_min[ 3 ], const float scene_max[ 3 ],
                             uint32_t * indices, uint64_t * codes, int32_t * parent, int32_t * left, int32_t * right, float * aabb,
                             uint32_t * sizes, void * scratch, void * stream )
{
    if ( !sites || n < 2 || !scene_min || !scene_max || !indices || !codes || !parent || !left || !right || !aabb || !scratch )
        return fail( APO2_ERR_INVALID_ARG, "invalid argument to apo2_lbvh_build" );
    if ( n > ( 1u << 28 ) )
        return fail( APO2_ERR_TOO_LARGE, "at most 2^28 sites" );
    cudaStream_t s = static_cast<cudaStream_t>( stream );
    // host float arithmetic of the reference for the scale (lbvh.cu:287-288)
    const float3 lo    = make_float3( scene_min[ 0 ], scene_min[ 1 ], scene_min[ 2 ] );
    const float3 scale = make_float3( 1.f / ( scene_max[ 0 ] - scene_min[ 0 ] ), 1.f / ( scene_max[ 1 ] - scene_min[ 1 ] ),
                                      1.f / ( scene_max[ 2 ] - scene_min[ 2 ] ) );
    char *      p        = static_cast<char *>( scratch );
    uint32_t *  errw     = reinterpret_cast<uint32_t *>( p );
    uint32_t *  arrivals = reinterpret_cast<uint32_t *>( p + 256 );
    SortScratch sort;
    sort_scratch_carve( sort, p + 256 + align256( 4 * size_t( n ) ), n, errw );
    cudaMemsetAsync( errw, 0, 4, s );
    launch_lbvh_f32( reinterpret_cast<const float4 *>( sites ), n, lo, scale, indices, codes, parent, left, right,
                     reinterpret_cast<float4 *>( aabb ), sizes, arrivals, sort, s );
    const cudaError_t err = cudaGetLastError();
    if ( err != cudaSuccess )
        return cuda_fail( err, "lbvh launch" );
    return APO2_OK;
}

uint64_t apo2_radix_sort_scratch_bytes( uint32_t n ) { return sort_scratch_bytes( n ) + 256; }

apo2_status apo2_radix_sort_pairs( uint64_t * keys, uint32_t * values, uint32_t n, void * scratch, void * stream )
{
    if ( !keys || !values || !scratch )
        return fail( APO2_ERR_INVALID_ARG, "invalid argument to apo2_radix_sort_pairs" );
    if ( n > ( 1u << 30 ) - 1 )
        return fail( APO2_ERR_TOO_LARGE, "at most 2^30 - 1 pairs" );
    cudaStream_t s    = static_cast<cudaStream_t>( stream );
    uint32_t *   errw = static_cast<uint32_t *>( scratch );
    SortScratch  sort;
    sort_scratch_carve( sort, static_cast<char *>( scratch ) + 256, n, errw );
    cudaMemsetAsync( errw, 0, 4, s );
    radix_sort_pairs( keys, values, n, sort, s );
    const cudaError_t err = cudaGetLastError();
    if ( err != cudaSuccess )
        return cuda_fail( err, "sort launch" );
    return APO2_OK;
}

} // extern "C"

// -----------------------------------------------------------------------------------------
// Batched form: many independent diagrams of uneven size (thousands of small protein-like
// sets). Each of `streams` workers owns a handle sized for the largest diagram, a stream and a
// host thread; diagrams go to whichever worker is free, largest first, so small builds overlap
// on the GPU instead of queueing behind one another. A handle is re-pointed into its own
// arena for each diagram's size (carve), so nothing is allocated while the batch runs.
// -----------------------------------------------------------------------------------------
struct apo2_batch
{
    uint32_t     max_sites = 0;
    apo2_options options {};
    int          device = 0;
    struct Worker
    {
        apo2_handle * h  = nullptr;
        cudaStream_t  s  = nullptr;
        cudaEvent_t   e0 = nullptr, e1 = nullptr;
        uint64_t *    words = nullptr; // pinned: vertex total, closed total, error word
    };
    std::vector<Worker> workers;
};

namespace
{
    void destroy_batch( apo2_batch * b )
    {
        if ( !b )
            return;
        cudaSetDevice( b->device );
        for ( auto & w : b->workers )
        {
            if ( w.s )
                cudaStreamSynchronize( w.s );
            if ( w.h )
                apo2_destroy( w.h );
            if ( w.e0 )
                cudaEventDestroy( w.e0 );
            if ( w.e1 )
                cudaEventDestroy( w.e1 );
            if ( w.s )
                cudaStreamDestroy( w.s );
            if ( w.words )
                cudaFreeHost( w.words );
        }
        delete b;
    }

    // One diagram on one worker: upload, build, extract, counts (and the vertices when asked).
    apo2_status batch_one( apo2_batch::Worker & w, const float * sites, uint32_t n, bool want_vertices,
                           std::vector<double4> & pos, std::vector<uint4> & ids, uint64_t & count, float & ms )
    {
        apo2_handle * h = w.h;
        if ( !carve( h, n ) )
            return fail( APO2_ERR_CUDA, "arena accounting" );
        h->built     = false;
        h->extracted = false;
        APO2_CUDA( cudaMemsetAsync( h->bounds_counter, 0, sizeof( uint32_t ), w.s ), "batch reset" );
        APO2_CUDA( cudaEventRecord( w.e0, w.s ), "batch event" );
        APO2_CUDA( cudaMemcpyAsync( h->input, sites, sizeof( float4 ) * n, cudaMemcpyHostToDevice, w.s ), "batch upload" );
        apo2_status st = enqueue_build( h, w.s );
        if ( st == APO2_OK )
            st = enqueue_extract( h, w.s );
        if ( st != APO2_OK )
            return st;
        APO2_CUDA( cudaEventRecord( w.e1, w.s ), "batch event" );
        APO2_CUDA( cudaMemcpyAsync( w.words, h->out.totals, 2 * sizeof( uint64_t ), cudaMemcpyDeviceToHost, w.s ), "batch counts" );
        APO2_CUDA( cudaMemcpyAsync( w.words + 2, h->error, sizeof( uint32_t ), cudaMemcpyDeviceToHost, w.s ), "batch counts" );
        APO2_CUDA( cudaStreamSynchronize( w.s ), "batch build" );
        const uint32_t flags = uint32_t( w.words[ 2 ] & 0xffffffffu );
        if ( flags )
            return fail( APO2_ERR_CAPACITY, "capacity flags " + std::to_string( flags ) );
        count = w.words[ 0 ];
        if ( count > h->out.vcap )
            return fail( APO2_ERR_CAPACITY, "batch output capacity" );
        if ( want_vertices && count )
        {
            pos.resize( count );
            ids.resize( count );
            APO2_CUDA( cudaMemcpyAsync( pos.data(), h->out.vpos, sizeof( double4 ) * count, cudaMemcpyDeviceToHost, w.s ), "batch output" );
            APO2_CUDA( cudaMemcpyAsync( ids.data(), h->out.vids, sizeof( uint4 ) * count, cudaMemcpyDeviceToHost, w.s ), "batch output" );
            APO2_CUDA( cudaStreamSynchronize( w.s ), "batch output" );
        }
        APO2_CUDA( cudaEventElapsedTime( &ms, w.e0, w.e1 ), "batch timing" );
        return APO2_OK;
    }
} // namespace

extern "C" {

apo2_status apo2_batch_create( uint32_t max_sites, uint32_t streams, const apo2_options * options, apo2_batch ** out )
{
    if ( !out || max_sites < 2 || streams == 0 || streams > 64 )
        return fail( APO2_ERR_INVALID_ARG, "invalid argument to apo2_batch_create" );
    if ( max_sites > ( 1u << 28 ) )
        return fail( APO2_ERR_TOO_LARGE, "at most 2^28 sites" );
    apo2_options      opt {};
    const apo2_status ost = normalize_options( options, opt );
    if ( ost != APO2_OK )
        return ost;
    if ( opt.shard_count != 1 )
        return fail( APO2_ERR_INVALID_ARG, "a batch builds whole diagrams (shard_count 0 or 1)" );
    opt.stage_timing = 0;
    APO2_CUDA( cudaSetDevice( int( opt.device ) ), "cudaSetDevice" );
    configure_cell_kernels();
    configure_spec_kernels();
    apo2_batch * b = new ( std::nothrow ) apo2_batch {};
    if ( !b )
        return fail( APO2_ERR_OUT_OF_MEMORY, "host allocation" );
    b->max_sites = max_sites;
    b->options   = opt;
    b->device    = int( opt.device );
    b->workers.resize( streams );
    for ( auto & w : b->workers )
    {
        apo2_handle * h = new ( std::nothrow ) apo2_handle {};
        if ( !h )
        {
            destroy_batch( b );
            return fail( APO2_ERR_OUT_OF_MEMORY, "host allocation" );
        }
        w.h          = h;
        h->options   = opt;
        h->device    = b->device;
        h->input_f64 = false;
        h->arena.size = arena_bytes( max_sites, opt, false );
        cudaError_t err = cudaMalloc( reinterpret_cast<void **>( &h->arena.base ), h->arena.size );
        if ( err == cudaSuccess && !carve( h, max_sites ) )
            err = cudaErrorMemoryAllocation;
        if ( err == cudaSuccess )
            err = cudaStreamCreateWithFlags( &w.s, cudaStreamNonBlocking );
        if ( err == cudaSuccess )
            err = cudaEventCreate( &w.e0 );
        if ( err == cudaSuccess )
            err = cudaEventCreate( &w.e1 );
        if ( err == cudaSuccess )
            err = cudaMallocHost( reinterpret_cast<void **>( &w.words ), 4 * sizeof( uint64_t ) );
        if ( err != cudaSuccess )
        {
            destroy_batch( b );
            return cuda_fail( err, "batch allocation" );
        }
        const apo2_status st = ensure_output_capacity( h, 8 * uint64_t( max_sites ) + 1024, uint64_t( max_sites ) / 16 + 1024 );
        if ( st != APO2_OK )
        {
            destroy_batch( b );
            return st;
        }
    }
    *out = b;
    return APO2_OK;
}

apo2_status apo2_batch_build( apo2_batch * b, const float * sites_xyzr, const uint64_t * site_offsets, uint32_t count,
                              uint64_t * vertex_offsets, double ** positions, uint32_t ** ids, float * build_ms )
{
    if ( !b || !sites_xyzr || !site_offsets || !vertex_offsets || ( ( positions == nullptr ) != ( ids == nullptr ) ) )
        return fail( APO2_ERR_INVALID_ARG, "invalid argument to apo2_batch_build" );
    for ( uint32_t d = 0; d < count; d++ )
    {
        if ( site_offsets[ d + 1 ] < site_offsets[ d ] + 2 )
            return fail( APO2_ERR_INVALID_ARG, "every diagram needs at least 2 sites" );
        if ( site_offsets[ d + 1 ] - site_offsets[ d ] > b->max_sites )
            return fail( APO2_ERR_TOO_LARGE, "a diagram is larger than the batch's max_sites" );
    }
    const bool want = positions != nullptr;
    // largest diagrams first, so the last ones to finish are small
    std::vector<uint32_t> order( count );
    for ( uint32_t d = 0; d < count; d++ )
        order[ d ] = d;
    std::stable_sort( order.begin(), order.end(), [ & ]( uint32_t x, uint32_t y ) {
        return site_offsets[ x + 1 ] - site_offsets[ x ] > site_offsets[ y + 1 ] - site_offsets[ y ];
    } );
    std::vector<std::vector<double4>> pos( want ? count : 0 );
    std::vector<std::vector<uint4>>   idv( want ? count : 0 );
    std::vector<uint64_t>             counts( count, 0 );
    std::vector<float>                times( count, 0.f );
    std::atomic<uint32_t>             next { 0 };
    std::atomic<int>                  failed { 0 };
    std::mutex                        error_mutex;
    apo2_status                       first_status = APO2_OK;
    std::string                       first_error;
    std::vector<double4>              no_pos;
    std::vector<uint4>                no_ids;

    auto run = [ & ]( apo2_batch::Worker & w ) {
        cudaSetDevice( b->device );
        while ( !failed.load() )
        {
            const uint32_t k = next.fetch_add( 1 );
            if ( k >= count )
                break;
            const uint32_t d  = order[ k ];
            const uint32_t n  = uint32_t( site_offsets[ d + 1 ] - site_offsets[ d ] );
            std::vector<double4> & p = want ? pos[ d ] : no_pos;
            std::vector<uint4> &   q = want ? idv[ d ] : no_ids;
            const apo2_status st = batch_one( w, sites_xyzr + 4 * site_offsets[ d ], n, want, p, q, counts[ d ], times[ d ] );
            if ( st != APO2_OK )
            {
                std::lock_guard<std::mutex> lock( error_mutex );
                if ( !failed.exchange( 1 ) )
                {
                    first_status = st;
                    first_error  = "diagram " + std::to_string( d ) + ": " + g_last_error;
                }
            }
        }
    };
    std::vector<std::thread> threads;
    for ( size_t t = 1; t < b->workers.size(); t++ )
        threads.emplace_back( run, std::ref( b->workers[ t ] ) );
    run( b->workers[ 0 ] );
    for ( auto & t : threads )
        t.join();
    if ( failed.load() )
        return fail( first_status, first_error );

    vertex_offsets[ 0 ] = 0;
    for ( uint32_t d = 0; d < count; d++ )
        vertex_offsets[ d + 1 ] = vertex_offsets[ d ] + counts[ d ];
    if ( build_ms )
        for ( uint32_t d = 0; d < count; d++ )
            build_ms[ d ] = times[ d ];
    if ( want )
    {
        const uint64_t total = vertex_offsets[ count ];
        double *       P     = static_cast<double *>( std::malloc( sizeof( double4 ) * std::max<uint64_t>( total, 1 ) ) );
        uint32_t *     I     = static_cast<uint32_t *>( std::malloc( sizeof( uint4 ) * std::max<uint64_t>( total, 1 ) ) );
        if ( !P || !I )
        {
            std::free( P );
            std::free( I );
            return fail( APO2_ERR_OUT_OF_MEMORY, "batch output (host)" );
        }
        for ( uint32_t d = 0; d < count; d++ )
        {
            if ( !counts[ d ] )
                continue;
            std::memcpy( P + 4 * vertex_offsets[ d ], pos[ d ].data(), sizeof( double4 ) * counts[ d ] );
            std::memcpy( I + 4 * vertex_offsets[ d ], idv[ d ].data(), sizeof( uint4 ) * counts[ d ] );
        }
        *positions = P;
        *ids       = I;
    }
    return APO2_OK;
}

apo2_status apo2_batch_set_proposal( apo2_batch * b, const apo2_proposal * model )
{
    if ( !b )
        return fail( APO2_ERR_INVALID_ARG, "null batch" );
    for ( auto & w : b->workers )
    {
        const apo2_status st = apo2_set_proposal( w.h, model );
        if ( st != APO2_OK )
            return st;
    }
    return APO2_OK;
}

apo2_status apo2_batch_destroy( apo2_batch * b )
{
    destroy_batch( b );
    return APO2_OK;
}

} // extern "C"
