// C++ mirror of the reference cavity application's interface (app/cavity/utils.hpp:8-33),
// header-only, on top of the C ABI of libapo2.so (include/apo2.h). The reference keeps the
// vertices and the hit ratios in device buffers between its calls; here they stay inside the
// diagram handle, so the calls take a `CavityDetection` object where the reference passes
// DeviceBuffers:
//
//     reference                                              this header
//     getVertices( sites, dVertices ) -> vertexNb            CavityDetection cavity{ sites }; cavity.vertexNb()
//     getHitRatios( vertexNb, dVertices, traceSites )        cavity.getHitRatios( traceSites )
//     getVertices( vertexNb, dVertices, hitRatios, t, r )    cavity.getVertices( t, r )
//     getDirections( count )                                 apo::gpu::getDirections( count )
//
// Errors of the C ABI are thrown as apo::gpu::Error.
#ifndef APO2_COMPAT_CAVITY_HPP
#define APO2_COMPAT_CAVITY_HPP

#include <cstdint>
#include <vector>

#include "algorithm.hpp"

namespace apo::gpu
{
    // utils.hpp:24-29
    struct FilterConfiguration
    {
        uint32_t vertexNb;
        float    hitRatioThreshold;
        float    radiusThreshold;
    };

    // utils.cu:201-242: the first `count` Halton directions on the sphere, unit length,
    // as float (x, y, z) triples.
    inline std::vector<float> getDirections( uint32_t count )
    {
        std::vector<float> xyz( 3 * size_t( count ) );
        check( apo2_cavity_directions( count, xyz.data() ) );
        return xyz;
    }

    // The application's pipeline (app/cavity/main.cpp:8-88) over one diagram.
    class CavityDetection
    {
      public:
        // utils.cu:153-199: the diagram of `sites` and its vertices
        explicit CavityDetection( ConstSpan<Real> sites ) : m_algorithm( sites )
        {
            m_algorithm.build();
            uint64_t vertices = 0, closed = 0;
            check( apo2_output_counts( m_algorithm.handle(), &vertices, &closed ) );
            m_vertexNb = uint32_t( vertices );
        }

        uint32_t vertexNb() const { return m_vertexNb; }

        // utils.cu:17-65: the share of `sampleNb` rays from each vertex that meet a trace sphere
        // (float x, y, z, r; the application passes the sites as loaded, before its joggle)
        std::vector<float> getHitRatios( ConstSpan<float> traceSites, uint32_t sampleNb = 64 )
        {
            std::vector<float> ratios( m_vertexNb );
            uint64_t           count = 0;
            check( apo2_cavity_hit_ratios( m_algorithm.handle(), traceSites.ptr, uint32_t( traceSites.size / 4 ), APO2_HOST,
                                           sampleNb, ratios.data(), ratios.size(), &count, nullptr ) );
            ratios.resize( count );
            return ratios;
        }

        // utils.cu:67-83, 527-559: vertices with hit ratio and radius above the thresholds, as
        // float (x, y, z, w), in output order (needs getHitRatios first)
        std::vector<float> getVertices( float hitRatioThreshold, float radiusThreshold )
        {
            uint64_t count = 0;
            check( apo2_cavity_vertices( m_algorithm.handle(), hitRatioThreshold, radiusThreshold, nullptr, 0, &count ) );
            std::vector<float> xyzw( 4 * count );
            check( apo2_cavity_vertices( m_algorithm.handle(), hitRatioThreshold, radiusThreshold, xyzw.data(), count, &count ) );
            xyzw.resize( 4 * count );
            return xyzw;
        }

        std::vector<float> filterVertices( FilterConfiguration configuration )
        {
            return getVertices( configuration.hitRatioThreshold, configuration.radiusThreshold );
        }

        AlgorithmGPU<16> & algorithm() { return m_algorithm; }

      private:
        AlgorithmGPU<16> m_algorithm;
        uint32_t         m_vertexNb = 0;
    };
} // namespace apo::gpu

#endif // APO2_COMPAT_CAVITY_HPP
