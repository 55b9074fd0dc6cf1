// A user problem file on the problem entry (include/kp_prob.hpp): its run
// merges the input files of the command line, reads the module's keys and
// builds the mesh from them, host-only, as a problem's set-up does before
// its first cycle.
#include "kp_prob.hpp"

#include <cstdio>

void kp::prob::run( int argc, char * argv[  ] )
{
    const std::string ini = kp::prob::cmd( argc, argv );
    kp_particle_cfg_t p {  };
    kp::api( kp_particle_read( ini.c_str(  ), & p ) );
    kp::mesh_t mesh( ini );
    const kp_mesh_info_t in = mesh.info(  );
    std::printf( "OK n_par=%g step_max=%d seed_rng=%d n_blocks=%d max_level=%d cells=%lld\n",
                 p.n_par, p.step_max, p.seed_rng, in.n_blocks, in.max_level, in.n_cells );
}

KP_PROB_MAIN(  )
