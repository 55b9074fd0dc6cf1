// A user problem on the radiation module (include/kp_module.hpp): its own
// packet generator (a __device__ functor, launched per packet as the
// reference's ker_gen launches the user's generate functor), enrolled,
// stepped through its cycles and saved.
//
//   module_check host <ini>            reads the keys, enrolls; no GPU
//   module_check gpu  <ini> <dir>      runs the cycles on the GPU: reads
//                                      <dir>/sigma.bin, writes each cycle's
//                                      generated packets to <dir>/tables.bin
//                                      and the module's container to
//                                      <dir>/run.bin
//   module_check pool <ini> <dir>      the same with a module that keeps its
//                                      unfinished packets (keep_pool, at most
//                                      100000 segments a packet), drained
//                                      after the cycles; writes <dir>/
//                                      tables_pool.bin and <dir>/run_pool.bin
#include "kp_generate.cuh"
#include "kp_module.hpp"

#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

namespace
{

// Packets from a ring of radius r about (0.5, 0.5) in the plane z = z0,
// isotropic, weights in [0.5, 1.5), every third one polarized; located on
// the device; every other one peels off at emission.
struct ring_gen_t
{
    double r, z0;
    __device__ static float uniform( unsigned long long k )
    {   // splitmix64 finaliser, top 24 bits
        k += 0x9E3779B97F4A7C15ull;
        k = ( k ^ ( k >> 30 ) ) * 0xBF58476D1CE4E5B9ull;
        k = ( k ^ ( k >> 27 ) ) * 0x94D049BB133111EBull;
        k ^= k >> 31;
        return ( float ) ( k >> 40 ) * 0x1p-24f;
    }
    __device__ void operator()( kp_packet_init_t & pk, long long pid ) const
    {
        const unsigned long long k = 8ull * ( unsigned long long ) pid;
        const double phi = 6.283185307179586 * uniform( k );
        pk.x[ 0 ] = 0.5 + r * cos( phi );
        pk.x[ 1 ] = 0.5 + r * sin( phi );
        pk.x[ 2 ] = z0;
        const float mu = 2.0f * uniform( k + 1 ) - 1.0f;
        const float ph = 6.2831853f * uniform( k + 2 );
        const float st = sqrtf( fmaxf( 0.0f, 1.0f - mu * mu ) );
        pk.d[ 0 ] = st * cosf( ph );
        pk.d[ 1 ] = st * sinf( ph );
        pk.d[ 2 ] = mu;
        pk.w = 0.5f + uniform( k + 3 );
        pk.stokes[ 0 ] = pid % 3 == 0 ? 0.3f : 0.0f;
        pk.stokes[ 1 ] = 0.0f;
        pk.stokes[ 2 ] = 0.0f;
        pk.ib = -1;
        pk.peel_I = pid % 2 == 0 ? 0.0795774715f : 0.0f;     // 1 / (4 pi)
        pk.pad = 0;
    }
};

// A module whose pool keeps the packets a cycle leaves unfinished.
struct pool_rad_t : kp::particle::radiation::base_t
{
    kp::particle::comm_mode_t comm_mode(  ) const override { return kp::particle::keep_pool; }
};

void configure( kp::particle::radiation::base_t & rad )
{
    auto & c = rad.transport_cfg(  );
    c.image_n = 32;
    c.inclination_deg = 60.0;
    c.image_center[ 0 ] = c.image_center[ 1 ] = c.image_center[ 2 ] = 0.5;
    c.image_half_width = 0.87;
    c.image_batch_n = 4;
    c.n_mu_bins = 8;
    c.mu_lo = -1.0f;
    c.mu_hi = 1.0f;
    c.w_min = 0.05f;
    c.fx_shift = 32;
    c.flux_fx_shift = 24;
    rad.enroll( kp::generate::on_device( ring_gen_t { 0.2, 0.45 }, rad.particle_cfg(  ).n_th ) );
}

}   // namespace

int main( int argc, char ** argv )
{
    if( argc < 3 )
    {
        std::fprintf( stderr, "usage: module_check host|gpu|pool <ini> [dir]\n" );
        return 2;
    }
    const std::string mode = argv[ 1 ], ini = argv[ 2 ];
    try
    {
        const bool pool = mode == "pool";
        pool_rad_t pool_rad;
        kp::particle::radiation::base_t plain_rad;
        kp::particle::radiation::base_t & rad = pool ? pool_rad : plain_rad;
        rad.read( ini );
        const auto & p = rad.particle_cfg(  );
        std::printf( "OK keys n_par=%g step_max=%d n_hv=%d n_cycle_stp=%d n_th=%d f_par=%g "
                     "seed_rng=%d output=%d max_round=%d\n", p.n_par, p.step_max, p.n_hv,
                     p.n_cycle_stp, p.n_th, p.f_par, p.seed_rng, p.output, p.max_round );
        configure( rad );
        if( rad.transport_cfg(  ).seed != ( uint32_t ) p.seed_rng
            || rad.transport_cfg(  ).max_steps != p.step_max )
            throw std::runtime_error( "keys not applied to the transport configuration" );
        std::printf( "OK enrolled\n" );
        if( mode == "host" )
            return 0;

        const std::string dir = argc > 3 ? argv[ 3 ] : ".";
        kp::device_t dev( 0 );
        kp::mesh_t mesh( ini );
        const long long n_cells = mesh.info(  ).n_cells;
        std::vector< float > sig( 2 * ( size_t ) n_cells );
        std::ifstream fs( dir + "/sigma.bin", std::ios::binary );
        fs.read( reinterpret_cast< char * >( sig.data(  ) ), sig.size(  ) * sizeof( float ) );
        if( ! fs )
            throw std::runtime_error( "cannot read sigma.bin" );
        mesh.set_sigma( sig.data(  ), ( long long ) sig.size(  ) );
        rad.init( mesh );
        if( pool )
            rad.pool_max_steps(  ) = 100000;
        const std::string sfx = pool ? "_pool" : "";
        std::ofstream ft( dir + "/tables" + sfx + ".bin", std::ios::binary );
        std::vector< kp_packet_init_t > table( ( size_t ) rad.packets_per_cycle(  ) );
        for( int c = 0; c < p.n_cycle_stp; ++ c )
        {
            rad.integrate( c );
            dev.cp( table.data(  ), rad.packet_table(  ), table.size(  ) );
            ft.write( reinterpret_cast< const char * >( table.data(  ) ),
                      table.size(  ) * sizeof( kp_packet_init_t ) );
            if( pool )
                std::printf( "OK pool after cycle %d: %lld packets\n", c, rad.pool_size(  ) );
        }
        rad.drain(  );
        dev.sync_all_streams(  );
        mesh.status(  );
        rad.save( dir + "/run" + sfx + ".bin" );
        std::printf( "OK module packets_done=%lld pool=%lld\n", rad.packets_done(  ),
                     rad.pool_size(  ) );
        return 0;
    }
    catch( const std::exception & e )
    {
        std::printf( "FAIL %s\n", e.what(  ) );
        return 1;
    }
}
