// Driver for the reference's contributing-nearest study (test infrastructure, built by
// oracle/ref_build.sh into oracle/_ref/apo_ref_contrib). The study's source
// (app/benchmarks/benchmark_contributing_nearest.cu) is compiled where it lies: its `main`,
// which reads the reference's sample files, is renamed out of the way, and this file calls
// its `apo::gpu::compute<16>` (lines 132-302: the library's LBVH and kNN, then
// `getCellsContribution`, lines 10-129, once per kNN step) on a given site file. Output: the
// two per-rank label arrays, sorted site order, (steps * 16) bytes per site:
//   <out>.contribution.u8      1 where the rank's neighbour changed the cell
//   <out>.reached.u8           1 where the security-radius certificate held after that rank
// Usage: apo_ref_contrib sites.f32 considered out
//   considered = the study's `iterationNb` (steps = considered / 16 + 1)
#define main apo_reference_contributing_nearest_main
#include APO_CONTRIB_SOURCE
#undef main

#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

// The study's sample loaders (app/common/samples.cpp) need chemfiles, which is absent; the
// renamed `main` is their only caller and is never run.
namespace apo
{
    std::vector<apo::Real> loadProtein( const apo::Path & ) { std::abort(); }
    std::vector<apo::Real> getUniform( uint32_t, apo::Real, apo::Real, apo::Real ) { std::abort(); }
    std::vector<apo::Real> parseFromDataset( const apo::Path & ) { std::abort(); }
} // namespace apo

int main( int argc, char ** argv )
{
    if ( argc != 4 )
    {
        std::fprintf( stderr, "usage: %s sites.f32 considered out\n", argv[ 0 ] );
        return 2;
    }
    std::FILE * f = std::fopen( argv[ 1 ], "rb" );
    if ( !f )
        return 2;
    std::vector<float> raw;
    float              buf[ 4096 ];
    std::size_t        got = 0;
    while ( ( got = std::fread( buf, sizeof( float ), 4096, f ) ) > 0 )
        raw.insert( raw.end(), buf, buf + got );
    std::fclose( f );
    std::vector<apo::Real> sites( raw.begin(), raw.end() );
    const uint32_t         considered = uint32_t( std::strtoul( argv[ 2 ], nullptr, 10 ) );

    const auto [ contribution, reached ] = apo::gpu::compute<16>( apo::ConstSpan<apo::Real> { sites.data(), sites.size() }, considered );

    const std::string out = argv[ 3 ];
    for ( const auto & [ suffix, data ] : { std::make_pair( std::string( ".contribution.u8" ), &contribution ),
                                            std::make_pair( std::string( ".reached.u8" ), &reached ) } )
    {
        std::FILE * o = std::fopen( ( out + suffix ).c_str(), "wb" );
        if ( !o )
            return 3;
        std::fwrite( data->data(), 1, data->size(), o );
        std::fclose( o );
    }
    std::printf( "%zu sites, %zu labels per site\n", sites.size() / 4, contribution.size() / ( sites.size() / 4 ) );
    return 0;
}
