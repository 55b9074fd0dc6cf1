// The particle radiation module's configuration keys, read with the
// reference's names and defaults (kp_particle_read).
#include "../../../include/kp_transport.h"
#include "../kp_common.cuh"
#include "ini.h"

#include <fstream>
#include <string>

extern "C" int kp_ini_merge( int n, const char * const * paths, const char * out_path )
{
    return kp::guarded( "kp_ini_merge", [ & ]
    {
        kp::require( n >= 1 && paths && out_path, "need at least one input file and an output path" );
        kp::ini_t ini;
        for( int k = 0; k < n; ++ k )
        {
            kp::require( paths[ k ] != nullptr, "null input file" );
            kp::require( ini.read_file( paths[ k ] ),
                         ( std::string( "cannot read the input file " ) + paths[ k ] ).c_str(  ),
                         KP_ERR_CONFIG );
        }
        std::ofstream f( out_path );
        kp::require( f.good(  ), "cannot write the merged input file", KP_ERR_CONFIG );
        f << ini.text(  );
        f.close(  );
        kp::require( ! f.fail(  ), "cannot write the merged input file", KP_ERR_CONFIG );
    } );
}

extern "C" int kp_particle_read( const char * ini_path, kp_particle_cfg_t * out )
{
    return kp::guarded( "kp_particle_read", [ & ]
    {
        kp::require( ini_path && out, "null argument" );
        kp::ini_t ini;
        kp::require( ini.read_file( ini_path ), "cannot read the configuration file",
                     KP_ERR_CONFIG );
        kp_particle_cfg_t c {  };
        // modules/particle/evolve/generate_par.h:36-41
        c.step_max    = ini.get_or< int >( "particle", "step_max", 100 );
        c.n_par       = ini.get_or< double >( "particle", "n_par", 1.0 );
        c.f_par       = ini.get_or< double >( "particle", "f_par", 1.0 );
        // modules/particle/radiation/radiation.h:26
        c.n_hv        = ini.get_or< int >( "particle", "n_hv", 1 );
        // modules/particle/driver.cpp:18
        c.n_cycle_stp = ini.get_or< int >( "particle", "n_cycle_stp", 1 );
        // types/driver_base.h:30, evolve/integrator.h:35, types/block_map.h:39
        c.n_th        = ini.get_or< int >( "particle", "n_th", 64 );
        c.max_round   = ini.get_or< int >( "particle", "max_round", 16 );
        c.static_proxy = ini.get_or< int >( "particle", "static_proxy", 0 );
        // types/particle_pool.h:50 (the reference reads [particles] here)
        c.output      = ini.get_or< int >( "particles", "output", 1 );
        // src/device/device.cpp:67-69
        c.seed_rng    = ini.get_or< int >( "device", "seed_rng", 7 );
        c.idx_device  = ini.get_or< int >( "device", "idx_device", -1 );
        kp::require( c.n_par >= 0 && c.n_par < 9.2e18, "[particle] n_par out of range",
                     KP_ERR_CONFIG );
        kp::require( c.step_max >= 1, "[particle] step_max must be positive", KP_ERR_CONFIG );
        kp::require( c.n_hv >= 1, "[particle] n_hv must be positive", KP_ERR_CONFIG );
        kp::require( c.n_cycle_stp >= 1, "[particle] n_cycle_stp must be positive",
                     KP_ERR_CONFIG );
        * out = c;
    } );
}
