// C++ mirror of the reference's public GPU interface (apo/include/apo/gpu/algorithm.hpp:9-59
// and apo/include/apo/gpu/algorithm.cuh:12-46), header-only, on top of the C ABI of
// libapo2.so (include/apo2.h). Code written against the reference's
//     apo::gpu::computeApolloniusDiagram(sites)
//     apo::gpu::AlgorithmGPU<16> algo{sites}; algo.build(); algo.toHostFull(true); algo.toTopology();
// compiles unchanged against this header and links with -lapo2.
//
// `Real` is double, the reference's default target; define APO_REAL_SIZE=4 before including
// for the `apo-fp32` spelling (float storage; the build itself is the FP64-semantics one).
// Errors of the C ABI are thrown as apo::gpu::Error (the reference prints and continues).
#ifndef APO2_COMPAT_ALGORITHM_HPP
#define APO2_COMPAT_ALGORITHM_HPP

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../apo2.h"

#ifndef APO_REAL_SIZE
#define APO_REAL_SIZE 8
#endif

namespace apo
{
#if APO_REAL_SIZE == 8
    using Real = double;
#else
    using Real = float;
#endif

    // apo/include/apo/core/type.hpp:26-41
    template<class Type>
    struct ConstSpan
    {
        const Type * ptr  = nullptr;
        std::size_t  size = 0;

        ConstSpan() = default;
        ConstSpan( const Type * p, std::size_t s ) : ptr( p ), size( s ) {}
        ConstSpan( const std::vector<Type> & data ) : ptr( data.data() ), size( data.size() ) {}
        const Type & operator[]( std::size_t i ) const { return ptr[ i ]; }
    };

    namespace gpu
    {
        struct Error : std::runtime_error
        {
            apo2_status status;
            Error( apo2_status s, const std::string & what ) : std::runtime_error( what ), status( s ) {}
        };

        inline void check( apo2_status s )
        {
            if ( s != APO2_OK )
                throw Error( s, apo2_last_error_string() );
        }

        // Host structures (algorithm.hpp:10-33)
        struct VertexDiagram
        {
            std::vector<Real>     vertices;   // Real4 {x, y, z, w}
            std::vector<uint32_t> verticesId; // {i, j, k, l}
            std::vector<uint32_t> invalidationId;
        };

        struct FullDiagram
        {
            std::vector<Real>     vertices;
            std::vector<uint32_t> verticesId;
            std::vector<uint32_t> invalidationId;
            std::vector<uint32_t> closedEdgesId;  // {i, j, k, 0}
            std::vector<Real>     closedEdgesMin; // Real4 {x, y, z, w}
        };

        struct Topology
        {
            std::vector<uint32_t> quadrisectors; // uint4
            std::vector<uint32_t> trisectors;    // uint3
            std::vector<uint32_t> bisectors;     // uint2
        };

        // algorithm.hpp:35-56
        class Algorithm
        {
          public:
            explicit Algorithm( ConstSpan<Real> sites ) : m_sites( sites ), m_siteNb( uint32_t( sites.size / 4 ) ) {}
            virtual ~Algorithm() = default;

            virtual void          build()                     = 0;
            virtual VertexDiagram toHost( bool validate )     = 0;
            virtual FullDiagram   toHostFull( bool validate ) = 0;
            virtual Topology      toTopology()                = 0;

            ConstSpan<Real> m_sites;
            uint32_t        m_siteNb = 0;
        };

        // algorithm.cuh:12-46 (the device buffers are internal to the library here)
        template<uint32_t K = 16>
        class AlgorithmGPU : public Algorithm
        {
          public:
            struct Sample
            {
                double initialization, bvhConstruction, knnSearch, knnConstruction, vertexValidation, edgeValidation,
                    bisectorValidation;
            };

            explicit AlgorithmGPU( ConstSpan<Real> sites, uint32_t knnValidationStep = 1 ) :
                Algorithm( sites ), knnValidationStep( knnValidationStep )
            {
                apo2_options options {};
                options.struct_size  = sizeof( apo2_options );
                options.k            = K;
                options.stage_timing = 1;
                options.knn_steps    = knnValidationStep == 0 ? APO2_NO_KNN_STEPS : knnValidationStep;
                check( apo2_create( sites.ptr, m_siteNb, sizeof( Real ) == 8 ? APO2_F64 : APO2_F32, APO2_HOST, &options,
                                    &m_handle ) );
            }
            ~AlgorithmGPU() override { apo2_destroy( m_handle ); }
            AlgorithmGPU( const AlgorithmGPU & )             = delete;
            AlgorithmGPU & operator=( const AlgorithmGPU & ) = delete;

            void build() override
            {
                check( apo2_build_and_extract( m_handle, nullptr ) );
                apo2_stats s {};
                check( apo2_get_stats( m_handle, &s ) );
                sample = Sample { 0.0, s.ms_bounds + s.ms_tree, s.ms_knn, s.ms_cells, s.ms_vertex_validation,
                                  s.ms_edge_validation, s.ms_bisector_validation };
            }

            VertexDiagram toHost( bool ) override
            {
                VertexDiagram d;
                readVertices( d.vertices, d.verticesId );
                return d;
            }

            FullDiagram toHostFull( bool ) override
            {
                FullDiagram d;
                readVertices( d.vertices, d.verticesId );
                uint64_t count = 0;
                check( apo2_get_closed_edges( m_handle, nullptr, nullptr, 0, APO2_HOST, &count ) );
                std::vector<double> pos( 4 * count );
                d.closedEdgesId.resize( 4 * count );
                check( apo2_get_closed_edges( m_handle, pos.data(), d.closedEdgesId.data(), count, APO2_HOST, &count ) );
                d.closedEdgesMin.assign( pos.begin(), pos.end() );
                return d;
            }

            Topology toTopology() override
            {
                Topology t;
                uint64_t q = 0, tr = 0, b = 0;
                check( apo2_get_topology( m_handle, nullptr, 0, nullptr, 0, nullptr, 0, &q, &tr, &b ) );
                t.quadrisectors.resize( 4 * q );
                t.trisectors.resize( 3 * tr );
                t.bisectors.resize( 2 * b );
                check( apo2_get_topology( m_handle, t.quadrisectors.data(), q, t.trisectors.data(), tr, t.bisectors.data(), b, &q,
                                          &tr, &b ) );
                return t;
            }

            uint32_t       knnValidationStep;
            Sample         sample {};
            apo2_handle *  handle() const { return m_handle; }

          private:
            void readVertices( std::vector<Real> & positions, std::vector<uint32_t> & ids )
            {
                uint64_t count = 0;
                check( apo2_get_vertices( m_handle, nullptr, nullptr, 0, APO2_HOST, &count ) );
                std::vector<double> pos( 4 * count );
                ids.resize( 4 * count );
                check( apo2_get_vertices( m_handle, pos.data(), ids.data(), count, APO2_HOST, &count ) );
                positions.assign( pos.begin(), pos.end() );
            }

            apo2_handle * m_handle = nullptr;
        };

        // algorithm.hpp:58-59, src/gpu/algorithm.cu:6-26
        inline VertexDiagram computeApolloniusDiagram( ConstSpan<Real> sites )
        {
            AlgorithmGPU<> algorithm { sites };
            algorithm.build();
            return algorithm.toHost( true );
        }

        inline FullDiagram computeFullApolloniusDiagram( ConstSpan<Real> sites )
        {
            AlgorithmGPU<> algorithm { sites };
            algorithm.build();
            return algorithm.toHostFull( true );
        }
    } // namespace gpu
} // namespace apo

#endif // APO2_COMPAT_ALGORITHM_HPP
