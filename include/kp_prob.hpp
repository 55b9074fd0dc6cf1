// kratos_polrad_b200 — the user problem entry, over the C ABI.
//
// Mirrors the reference's user interface (src/user/probgen.h:11-15,
// probgen.cpp:8-22) and its main (src/main.cpp:7-13): a problem file defines
// kp::prob::run, and KP_PROB_MAIN() supplies the main that calls it with the
// command line, refusing to start without an input file.
//
//   #include "kp_module.hpp"
//   #include "kp_prob.hpp"
//
//   void kp::prob::run( int argc, char * argv[] )
//   {
//       const std::string ini = kp::prob::cmd( argc, argv );   // merged inputs
//       kp::mesh_t mesh( ini );                                // [mesh], [refine_region*]
//       kp::particle::radiation::base_t rad;
//       rad.read( ini );                                       // [particle], [device]
//       ...
//   }
//   KP_PROB_MAIN(  )
//
// Host C++17.  Failures throw std::runtime_error (kp::api).
#ifndef KP_PROB_HPP
#define KP_PROB_HPP

#include "kp_transport.hpp"

#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

#include <unistd.h>

namespace kp::prob
{

// The user's problem (prob::run): defined by the problem file.
void run( int argc, char * argv[  ] );

// prob::cmd: the input files given on the command line (argv[1..]), read in
// order with later values overriding earlier ones, as one INI file; returns
// its path.  One file is used as it is; several are merged into `merged`,
// or into a new file in $TMPDIR (default /tmp) when `merged` is empty.
inline std::string cmd( int argc, char * argv[  ], std::string merged = "" )
{
    if( argc <= 1 )
        throw std::runtime_error( "No input file." );
    if( argc == 2 )
        return argv[ 1 ];
    if( merged.empty(  ) )
    {
        const char * tmp = std::getenv( "TMPDIR" );
        std::string pattern = std::string( tmp && * tmp ? tmp : "/tmp" ) + "/kp_input_XXXXXX";
        std::vector< char > name( pattern.begin(  ), pattern.end(  ) );
        name.push_back( '\0' );
        const int fd = mkstemp( name.data(  ) );
        if( fd < 0 )
            throw std::runtime_error( "kratos_polrad_b200: cannot create the merged input file" );
        close( fd );
        merged = name.data(  );
    }
    std::vector< const char * > paths( argv + 1, argv + argc );
    api( kp_ini_merge( ( int ) paths.size(  ), paths.data(  ), merged.c_str(  ) ) );
    return merged;
}

}   // namespace kp::prob

// main() of a problem file (src/main.cpp:7-13): needs at least one input file.
#define KP_PROB_MAIN(  )                                                    \
    int main( int argc, char * argv[  ] )                                  \
    {                                                                      \
        if( argc <= 1 )                                                    \
            throw std::runtime_error( "No input file." );                  \
        kp::prob::run( argc, argv );                                       \
        return 0;                                                          \
    }

#endif
