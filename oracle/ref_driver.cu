// Driver for the reference library built from its own sources (oracle/ref_build.sh).
//
// It runs the reference's public path -- `AlgorithmGPU<K>{sites, knnValidationStep}.build()`
// (K = 16 and one kNN step unless --k / --knn-steps say otherwise) followed by
// `toHostFull()` and `toTopology()` (apo/include/apo/gpu/algorithm.inl:1410-1821) -- on a
// site file and writes every array the parity tests pin: the LBVH node arrays and the
// Morton permutation (apo/src/gpu/lbvh.cu:274-323), the kNN lists of the first search
// round (apo/include/apo/gpu/algorithm.inl:32-99), the per-cell vertex and edge stores,
// the cell status bytes, the full diagram and the topology. With --time it also times the
// reference's own benchmark region (constructor + build(),
// app/benchmarks/benchmark.cu:9-22) with CUDA events.
//
// This is test infrastructure: it only produces golden data and the reference GPU
// timing beside the product's numbers; nothing in the product links it.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "apo/gpu/algorithm.cuh"

namespace
{
    template<class T>
    void writeArray( const std::string & dir, const char * name, const T * data, std::size_t count )
    {
        const std::string path = dir + "/" + name;
        FILE *            f    = std::fopen( path.c_str(), "wb" );
        if ( !f )
        {
            std::fprintf( stderr, "cannot open %s\n", path.c_str() );
            std::exit( 3 );
        }
        if ( count )
            std::fwrite( data, sizeof( T ), count, f );
        std::fclose( f );
    }

    template<class T>
    std::vector<T> download( const T * device, std::size_t count )
    {
        std::vector<T> host( count );
        if ( count )
            cudaMemcpy( host.data(), device, count * sizeof( T ), cudaMemcpyDeviceToHost );
        return host;
    }

    void check( const char * what )
    {
        const cudaError_t err = cudaDeviceSynchronize();
        if ( err != cudaSuccess )
        {
            std::fprintf( stderr, "%s: %s\n", what, cudaGetErrorString( err ) );
            std::exit( 4 );
        }
    }
} // namespace


// --stages: the reference's build sequence (algorithm.inl:1410-1594), stage by stage, calling
// its own kernels, with the per-cell stores dumped after the kNN cells ("s1"), after each
// round's vertex ("v<r>") and edge ("e<r>") validation, and after bisector validation ("b").
// Used to find the first stage at which another implementation departs from the reference.
namespace apo::gpu
{
    // `length` looked up from inside apo::gpu, as build() does
    inline Real stagedLength( Real3 v ) { return length( v ); }
} // namespace apo::gpu

template<uint32_t K>
struct StagedBuild : apo::gpu::AlgorithmGPU<K>
{
    using Base = apo::gpu::AlgorithmGPU<K>;
    using Base::Base;

    void dump( const std::string & dir, const std::string & tag, const float * knownRadii )
    {
        const uint32_t n        = this->m_siteNb;
        check( tag.c_str() );
        const auto vertexNb = download( this->dVerticesNb.template get<uint32_t>(), n );
        const auto edgeNb   = download( this->dEdgesNb.template get<uint32_t>(), n );
        const auto status   = download( this->dStatus.template get<uint8_t>(), n );
        const auto radii    = download( knownRadii, n );
        const auto vstore   = download( this->dVertices.template get<uint32_t>(), std::size_t( n ) * 152 * 4 );
        const auto estore   = download( this->dEdges.template get<uint32_t>(), std::size_t( n ) * 264 * 4 );
        std::vector<uint32_t> vertices, edges;
        for ( uint32_t i = 0; i < n; i++ )
        {
            const uint32_t vn = std::min( vertexNb[ i ], 152u ), en = std::min( edgeNb[ i ], 264u );
            vertices.insert( vertices.end(), vstore.begin() + std::size_t( i ) * 608, vstore.begin() + std::size_t( i ) * 608 + vn * 4 );
            edges.insert( edges.end(), estore.begin() + std::size_t( i ) * 1056, estore.begin() + std::size_t( i ) * 1056 + en * 4 );
        }
        writeArray( dir, ( tag + "_vertex_nb.u32" ).c_str(), vertexNb.data(), vertexNb.size() );
        writeArray( dir, ( tag + "_edge_nb.u32" ).c_str(), edgeNb.data(), edgeNb.size() );
        writeArray( dir, ( tag + "_status.u8" ).c_str(), status.data(), status.size() );
        writeArray( dir, ( tag + "_known_radii.f32" ).c_str(), radii.data(), radii.size() );
        writeArray( dir, ( tag + "_vertices.u32" ).c_str(), vertices.data(), vertices.size() );
        writeArray( dir, ( tag + "_edges.u32" ).c_str(), edges.data(), edges.size() );
    }

    void stagedBuild( const std::string & dir )
    {
        using namespace apo::gpu;
        using apo::Real;
        const uint32_t n = this->m_siteNb;

        ContextCellOriented context {};
        context.siteNb    = n;
        this->dSites      = DeviceBuffer { ( n + 6 ) * sizeof( Real4 ), false };
        context.sites     = this->dSites.template get<Real4>();
        context.minRadius = this->m_minRadius;
        context.maxRadius = this->m_maxRadius;
        this->dStatus     = { n * sizeof( uint8_t ), true };
        context.status    = this->dStatus.template get<uint8_t>();
        this->dVertices   = DeviceBuffer { sizeof( Vertex ) * 152 * std::size_t( n ), false };
        this->dVerticesNb = DeviceBuffer { sizeof( uint32_t ) * n, true };
        context.vertexNb  = this->dVerticesNb.template get<uint32_t>();
        context.vertices  = this->dVertices.template get<Vertex>();
        this->dEdges      = DeviceBuffer { sizeof( Edge ) * 264 * std::size_t( n ), false };
        this->dEdgesNb    = DeviceBuffer { sizeof( uint32_t ) * n, true };
        context.edges     = this->dEdges.template get<Edge>();
        context.edgeNb    = this->dEdgesNb.template get<uint32_t>();

        // sites, then the six joggled bounding sites around the box centre
        mmemcpy<MemcpyType::HostToDevice>( this->dSites.template get<Real>(), this->m_sites.ptr, this->m_sites.size );
        {
            const Real cx = ( this->m_minX + this->m_maxX ) / Real( 2 ), cy = ( this->m_minY + this->m_maxY ) / Real( 2 ),
                       cz = ( this->m_minZ + this->m_maxZ ) / Real( 2 );
            const Real3 centre { cx, cy, cz };
            const Real  aabbRadius = apo::gpu::stagedLength( centre - Real3 { this->m_maxX, this->m_maxY, this->m_maxZ } );
            const Real  radius     = aabbRadius * ( std::sqrt( Real( 3. ) ) + Real( 1e-1 ) );
            const Real  r0         = context.minRadius;
            std::vector<Real4> art = {
                Real4 { cx + radius, cy + Real( 0 ), cz + Real( 0 ), Real( 0 ) + r0 },
                Real4 { cx - radius, cy + Real( 0 ), cz + Real( 0 ), Real( 0 ) + r0 },
                Real4 { cx + Real( 0 ), cy + radius, cz + Real( 0 ), Real( 0 ) + r0 },
                Real4 { cx + Real( 0 ), cy - radius, cz + Real( 0 ), Real( 0 ) + r0 },
                Real4 { cx + Real( 0 ), cy + Real( 0 ), cz + radius, Real( 0 ) + r0 },
                Real4 { cx + Real( 0 ), cy + Real( 0 ), cz - radius, Real( 0 ) + r0 },
            };
            apo::joggle( { reinterpret_cast<Real *>( art.data() ), 6 * 4 }, 1e-1 );
            mmemcpy<MemcpyType::HostToDevice>( this->dSites.template get<Real4>() + n, art.data(), 6 );
        }
        // initial cell: 8 vertices and 12 edges on the bounding sites
        std::vector<uint32_t> init;
        const uint32_t vt[ 8 ][ 3 ] = { { 0, 2, 4 }, { 0, 2, 5 }, { 0, 3, 4 }, { 0, 3, 5 }, { 1, 2, 4 }, { 1, 2, 5 }, { 1, 3, 4 }, { 1, 3, 5 } };
        const uint32_t et[ 12 ][ 2 ] = { { 0, 2 }, { 2, 4 }, { 1, 2 }, { 2, 5 }, { 1, 4 }, { 1, 5 }, { 0, 5 }, { 0, 4 }, { 1, 3 }, { 3, 5 }, { 0, 3 }, { 3, 4 } };
        for ( auto & v : vt )
            init.insert( init.end(), { n + v[ 0 ], n + v[ 1 ], n + v[ 2 ], 0u } );
        for ( auto & e : et )
            init.insert( init.end(), { n + e[ 0 ], n + e[ 1 ] } );
        DeviceBuffer initData = DeviceBuffer::Typed<uint32_t>( init.size() );
        mmemcpy<MemcpyType::HostToDevice>( initData.template get<uint32_t>(), init.data(), init.size() );

        Aabbf aabb = { make_float3( this->m_minX, this->m_minY, this->m_minZ ), make_float3( this->m_maxX, this->m_maxY, this->m_maxZ ) };
        this->bvh  = LBVH {};
        this->bvh.build( n, aabb, context.sites );

        auto [ gridDim, blockDim ] = KernelConfig::From( n, impl::KnnBlockSize );
        initializeDataStructure<impl::TotalMaxVertexNb, impl::TotalMaxEdgeNb><<<gridDim, blockDim>>>(
            context, initData.template get<uint32_t>(), initData.template get<uint32_t>() + 32 );
        check( "initializeDataStructure" );

        DeviceBuffer knns = DeviceBuffer( n * K * ( sizeof( uint32_t ) + sizeof( Real ) ), false );
        cudaMemset( knns.template get<uint32_t>(), 0xff, sizeof( uint32_t ) * n * K );
        std::vector<float> lowest( n, std::numeric_limits<float>::lowest() );
        DeviceBuffer       knownRadii = DeviceBuffer::Typed<float>( n, false );
        mmemcpy<MemcpyType::HostToDevice>( knownRadii.template get<float>(), lowest.data(), n );
        for ( uint32_t step = 0; step < this->knnValidationStep; step++ )
        {
            impl::getKnns<K><<<gridDim, blockDim>>>( step, context, this->bvh.getDeviceView(), knns.template get<uint32_t>() );
            auto [ cg, cb ] = KernelConfig::From( n * WarpSize, impl::BlockSize );
            impl::getCells<<<cg, cb>>>( context, K, knns.template get<uint32_t>(), knownRadii.template get<float>() );
        }
        dump( dir, "s1", knownRadii.template get<float>() );

        uint32_t taskNb = thrust::count( thrust::device, context.status, context.status + n, CellStatus::InValidation );
        for ( uint32_t round = 0; round < 10 && taskNb != 0; round++ )
        {
            DeviceBuffer tasks = DeviceBuffer::Typed<uint32_t>( taskNb );
            thrust::copy_if( thrust::device, thrust::make_counting_iterator<uint32_t>( 0 ),
                             thrust::make_counting_iterator<uint32_t>( n ), context.status, tasks.template get<uint32_t>(),
                             thrust::placeholders::_1 == 0 );
            auto [ cg, cb ] = KernelConfig::From( taskNb * WarpSize, impl::BlockSize );
            impl::globalVertexValidation<<<cg, cb>>>( context, this->bvh.getDeviceView(), taskNb, tasks.template get<uint32_t>(),
                                                      knownRadii.template get<float>() );
            dump( dir, "v" + std::to_string( round ), knownRadii.template get<float>() );
            impl::globalEdgeValidation<<<cg, cb>>>( context, this->bvh.getDeviceView(), taskNb, tasks.template get<uint32_t>(),
                                                    knownRadii.template get<float>() );
            dump( dir, "e" + std::to_string( round ), knownRadii.template get<float>() );
            taskNb = thrust::count( thrust::device, context.status, context.status + n, uint8_t( 0 ) );
        }
        auto [ cg, cb ] = KernelConfig::From( n * WarpSize, impl::BlockSize );
        impl::globalBisectorValidation<<<cg, cb>>>( context, this->bvh.getDeviceView(), knownRadii.template get<float>() );
        dump( dir, "b", knownRadii.template get<float>() );
    }
};

template<uint32_t K>
void runReference( std::vector<apo::Real> & sites, const uint32_t n, const std::string & outDir, const int repeat,
                   const bool dump, const uint32_t knnSteps, std::string & json, const int warmup = 3,
                   const bool withTopology = true )
{

    if ( repeat > 0 )
    {
        cudaEvent_t start, stop;
        cudaEventCreate( &start );
        cudaEventCreate( &stop );
        std::vector<float> times;
        double stage[ 7 ] = { 0, 0, 0, 0, 0, 0, 0 };
        for ( int r = -warmup; r < repeat; r++ )
        {
            cudaDeviceSynchronize();
            cudaEventRecord( start );
            {
                apo::gpu::AlgorithmGPU<K> algorithm { apo::ConstSpan<apo::Real> { sites.data(), sites.size() }, knnSteps };
                algorithm.build();
                if ( r >= 0 )
                {
                    stage[ 0 ] += algorithm.sample.initialization;
                    stage[ 1 ] += algorithm.sample.bvhConstruction;
                    stage[ 2 ] += algorithm.sample.knnSearch;
                    stage[ 3 ] += algorithm.sample.knnConstruction;
                    stage[ 4 ] += algorithm.sample.vertexValidation;
                    stage[ 5 ] += algorithm.sample.edgeValidation;
                    stage[ 6 ] += algorithm.sample.bisectorValidation;
                }
            }
            cudaEventRecord( stop );
            cudaEventSynchronize( stop );
            float ms = 0.f;
            cudaEventElapsedTime( &ms, start, stop );
            if ( r >= 0 )
                times.push_back( ms );
        }
        check( "timed builds" );
        std::sort( times.begin(), times.end() );
        char buffer[ 512 ];
        std::snprintf( buffer,
                       sizeof( buffer ),
                       ", \"build_ms_median\": %.6f, \"build_ms_min\": %.6f, \"repeat\": %d, \"stage_ms\": {"
                       "\"initialization\": %.6f, \"bvh\": %.6f, \"knn_search\": %.6f, \"knn_cells\": %.6f, "
                       "\"vertex_validation\": %.6f, \"edge_validation\": %.6f, \"bisector_validation\": %.6f}",
                       times[ times.size() / 2 ],
                       times.front(),
                       repeat,
                       stage[ 0 ] / repeat,
                       stage[ 1 ] / repeat,
                       stage[ 2 ] / repeat,
                       stage[ 3 ] / repeat,
                       stage[ 4 ] / repeat,
                       stage[ 5 ] / repeat,
                       stage[ 6 ] / repeat );
        json += buffer;
    }

    if ( dump )
    {
        apo::gpu::AlgorithmGPU<K> algorithm { apo::ConstSpan<apo::Real> { sites.data(), sites.size() }, knnSteps };
        algorithm.build();
        check( "build" );

        const uint32_t nodeCount = 2 * n - 1;
        const auto     view      = algorithm.bvh.getDeviceView();
        {
            const auto indices = download( view.indices, n );
            writeArray( outDir, "indices.u32", indices.data(), indices.size() );
            const auto parent = download( view.nodesParent, nodeCount );
            writeArray( outDir, "parent.i32", parent.data(), parent.size() );
            const auto left = download( view.nodesLeft, nodeCount );
            writeArray( outDir, "left.i32", left.data(), left.size() );
            const auto right = download( view.nodesRight, nodeCount );
            writeArray( outDir, "right.i32", right.data(), right.size() );
            const auto aabb = download( view.nodesAabb, 2 * std::size_t( nodeCount ) );
            writeArray( outDir, "aabb.f32", reinterpret_cast<const float *>( aabb.data() ), aabb.size() * 4 );
            const auto sizes = download( view.sizes, nodeCount );
            writeArray( outDir, "sizes.u32", sizes.data(), sizes.size() );
        }

        const auto sorted = download( algorithm.dSites.template get<apo::Real>(), ( n + 6 ) * 4 );
        writeArray( outDir, "sites_sorted.f64", sorted.data(), sorted.size() );

        const auto status = download( algorithm.dStatus.template get<uint8_t>(), n );
        writeArray( outDir, "status.u8", status.data(), status.size() );

        const auto vertexNb = download( algorithm.dVerticesNb.template get<uint32_t>(), n );
        const auto edgeNb   = download( algorithm.dEdgesNb.template get<uint32_t>(), n );
        writeArray( outDir, "vertex_nb.u32", vertexNb.data(), vertexNb.size() );
        writeArray( outDir, "edge_nb.u32", edgeNb.data(), edgeNb.size() );
        {
            const auto vertexStore = download( algorithm.dVertices.template get<uint32_t>(), std::size_t( n ) * 152 * 4 );
            const auto edgeStore   = download( algorithm.dEdges.template get<uint32_t>(), std::size_t( n ) * 264 * 4 );
            std::vector<uint32_t> vertices, edges;
            for ( uint32_t i = 0; i < n; i++ )
            {
                const uint32_t vn = std::min( vertexNb[ i ], 152u );
                const uint32_t en = std::min( edgeNb[ i ], 264u );
                vertices.insert( vertices.end(),
                                 vertexStore.begin() + std::size_t( i ) * 152 * 4,
                                 vertexStore.begin() + std::size_t( i ) * 152 * 4 + vn * 4 );
                edges.insert( edges.end(),
                              edgeStore.begin() + std::size_t( i ) * 264 * 4,
                              edgeStore.begin() + std::size_t( i ) * 264 * 4 + en * 4 );
            }
            writeArray( outDir, "vertices.u32", vertices.data(), vertices.size() );
            writeArray( outDir, "edges.u32", edges.data(), edges.size() );
        }

        // kNN lists of the first round: relaunch the reference's own kNN kernel on the final
        // context (it only re-marks buried cells, which are already marked).
        {
            apo::gpu::ContextCellOriented context {};
            context.siteNb   = n;
            context.sites    = algorithm.dSites.template get<apo::gpu::Real4>();
            context.status   = algorithm.dStatus.template get<uint8_t>();
            uint32_t * knns  = nullptr;
            cudaMalloc( &knns, sizeof( uint32_t ) * n * K );
            cudaMemset( knns, 0xff, sizeof( uint32_t ) * n * K );
            auto [ gridDim, blockDim ] = apo::gpu::KernelConfig::From( n, apo::gpu::impl::KnnBlockSize );
            apo::gpu::impl::getKnns<K><<<gridDim, blockDim>>>( 0, context, view, knns );
            check( "getKnns" );
            const auto knnHost = download( knns, std::size_t( n ) * K );
            writeArray( outDir, "knn.u32", knnHost.data(), knnHost.size() );
            cudaFree( knns );
        }

        const apo::gpu::FullDiagram full = algorithm.toHostFull( true );
        check( "toHostFull" );
        writeArray( outDir, "vertices_pos.f64", full.vertices.data(), full.vertices.size() );
        writeArray( outDir, "vertices_id.u32", full.verticesId.data(), full.verticesId.size() );
        writeArray( outDir, "closed_pos.f64", full.closedEdgesMin.data(), full.closedEdgesMin.size() );
        writeArray( outDir, "closed_id.u32", full.closedEdgesId.data(), full.closedEdgesId.size() );

        // The reference's toTopology grows its output vectors with a reserve per cell, which
        // copies them once per cell (quadratic): beyond ~10^5 sites it runs for hours, so large
        // cases skip it (--no-topology; the topology is a function of the stores dumped above).
        if ( withTopology )
        {
            const apo::gpu::Topology topology = algorithm.toTopology();
            writeArray( outDir, "topo_quad.u32", topology.quadrisectors.data(), topology.quadrisectors.size() );
            writeArray( outDir, "topo_tri.u32", topology.trisectors.data(), topology.trisectors.size() );
            writeArray( outDir, "topo_bi.u32", topology.bisectors.data(), topology.bisectors.size() );
        }

        json += ", \"vertices\": " + std::to_string( full.vertices.size() / 4 );
        json += ", \"closed_edges\": " + std::to_string( full.closedEdgesMin.size() / 4 );
    }

}

int main( int argc, char ** argv )
{
    if ( argc < 3 )
    {
        std::fprintf( stderr, "usage: %s sites.f32 outdir [--time R] [--warmup W] [--no-dump] [--no-topology] [--k 1|4|8|16] [--knn-steps S] [--stages]\n", argv[ 0 ] );
        return 1;
    }
    const std::string input  = argv[ 1 ];
    const std::string outDir = argv[ 2 ];
    int               repeat = 0;
    int               warmup = 3; // untimed builds before the timed ones
    bool              withTopology = true;
    bool              dump   = true;
    uint32_t          k        = 16; // AlgorithmGPU<K>
    uint32_t          knnSteps = 1;  // knnValidationStep
    bool              staged   = false;
    for ( int a = 3; a < argc; a++ )
    {
        if ( !std::strcmp( argv[ a ], "--time" ) && a + 1 < argc )
            repeat = std::atoi( argv[ ++a ] );
        else if ( !std::strcmp( argv[ a ], "--warmup" ) && a + 1 < argc )
            warmup = std::max( 0, std::atoi( argv[ ++a ] ) );
        else if ( !std::strcmp( argv[ a ], "--no-topology" ) )
            withTopology = false;
        else if ( !std::strcmp( argv[ a ], "--no-dump" ) )
            dump = false;
        else if ( !std::strcmp( argv[ a ], "--k" ) && a + 1 < argc )
            k = uint32_t( std::atoi( argv[ ++a ] ) );
        else if ( !std::strcmp( argv[ a ], "--knn-steps" ) && a + 1 < argc )
            knnSteps = uint32_t( std::atoi( argv[ ++a ] ) );
        else if ( !std::strcmp( argv[ a ], "--stages" ) )
            staged = true;
    }

    // Sites are stored as float32 (x, y, z, r); the reference's FP64 build reads `double`.
    FILE * f = std::fopen( input.c_str(), "rb" );
    if ( !f )
    {
        std::fprintf( stderr, "cannot open %s\n", input.c_str() );
        return 2;
    }
    std::fseek( f, 0, SEEK_END );
    const long bytes = std::ftell( f );
    std::fseek( f, 0, SEEK_SET );
    std::vector<float> raw( static_cast<std::size_t>( bytes ) / sizeof( float ) );
    if ( std::fread( raw.data(), sizeof( float ), raw.size(), f ) != raw.size() )
        return 2;
    std::fclose( f );
    std::vector<apo::Real> sites( raw.begin(), raw.end() );
    const uint32_t         n = static_cast<uint32_t>( sites.size() / 4 );

    std::string json = "{\"n\": " + std::to_string( n );
    json += ", \"k\": " + std::to_string( k ) + ", \"knn_steps\": " + std::to_string( knnSteps );
    if ( staged )
    {
        if ( k != 16 )
            return 1;
        StagedBuild<16> algorithm { apo::ConstSpan<apo::Real> { sites.data(), sites.size() }, knnSteps };
        algorithm.stagedBuild( outDir );
        std::puts( "staged dumps written" );
        return 0;
    }
    switch ( k )
    {
    case 1: runReference<1>( sites, n, outDir, repeat, dump, knnSteps, json, warmup, withTopology ); break;
    case 4: runReference<4>( sites, n, outDir, repeat, dump, knnSteps, json, warmup, withTopology ); break;
    case 8: runReference<8>( sites, n, outDir, repeat, dump, knnSteps, json, warmup, withTopology ); break;
    case 16: runReference<16>( sites, n, outDir, repeat, dump, knnSteps, json, warmup, withTopology ); break;
    default: std::fprintf( stderr, "k must be 1, 4, 8 or 16\n" ); return 1;
    }

    json += "}\n";
    writeArray( outDir, "meta.json", json.data(), json.size() );
    std::fputs( json.c_str(), stdout );
    return 0;
}
