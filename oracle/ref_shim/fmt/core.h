// Minimal stand-in for the `fmt` entry points the reference's GPU library names
// (`fmt::print` in its cudaCheck helper, `fmt::format` in its logger template) and
// `fmt::format_to`, which its contributing-nearest study's CSV writer names.
// The `fmt` submodule is not vendored with the reference; this stub only formats
// log text ("{}" placeholders, format specs ignored) and takes no part in any
// computation. Used solely by oracle/ref_build.sh.
#pragma once
#include <cstdio>
#include <sstream>
#include <string>
#include <string_view>

namespace fmt
{
    namespace detail
    {
        inline void append( std::ostringstream & out, std::string_view & rest ) { out << rest; rest = {}; }

        template<class T, class... Rest>
        void append( std::ostringstream & out, std::string_view & rest, const T & value, const Rest &... others )
        {
            const std::size_t open = rest.find( '{' );
            if ( open == std::string_view::npos )
            {
                out << rest;
                rest = {};
                return;
            }
            const std::size_t close = rest.find( '}', open );
            out << rest.substr( 0, open ) << value;
            rest = rest.substr( close == std::string_view::npos ? rest.size() : close + 1 );
            append( out, rest, others... );
        }
    } // namespace detail

    template<class... T>
    std::string format( std::string_view pattern, const T &... args )
    {
        std::ostringstream out;
        std::string_view   rest = pattern;
        detail::append( out, rest, args... );
        return out.str();
    }

    template<class OutputIt, class... T>
    OutputIt format_to( OutputIt out, std::string_view pattern, const T &... args )
    {
        const std::string text = format( pattern, args... );
        for ( const char ch : text )
            *out++ = ch;
        return out;
    }

    template<class... T>
    void print( std::string_view pattern, const T &... args )
    {
        const std::string text = format( pattern, args... );
        std::fwrite( text.data(), 1, text.size(), stdout );
    }
} // namespace fmt
