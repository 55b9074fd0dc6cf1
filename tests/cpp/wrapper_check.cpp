// Exercises the C++ layer (include/kp_transport.hpp) the way a reference
// build would call it.  `wrapper_check host <ini>` runs the host-only parts
// (mesh tables, point location, error translation); `wrapper_check gpu <ini>`
// adds a small forward solve on device 0 through device_t / mesh_t /
// transport, a host callback and event timing.  Prints "OK <what>" lines.
#include "kp_transport.hpp"

#include <atomic>
#include <cstdio>
#include <cstring>
#include <vector>

static int host_part( const char * ini )
{
    kp::mesh_t mesh( ini );
    const kp_mesh_info_t info = mesh.info(  );
    std::printf( "OK mesh blocks=%d cells=%lld\n", info.n_blocks, info.n_cells );
    std::vector< int > level;
    std::vector< std::array< int, 3 > > reg;
    mesh.blocks( level, reg );
    if( ( int ) level.size(  ) != info.n_blocks ) return 1;
    std::vector< std::array< double, 3 > > x = { { 0.5 * ( info.x_min[ 0 ] + info.x_max[ 0 ] ),
                                                   0.5 * ( info.x_min[ 1 ] + info.x_max[ 1 ] ),
                                                   0.5 * ( info.x_min[ 2 ] + info.x_max[ 2 ] ) },
                                                 { info.x_max[ 0 ] + 1.0, 0.0, 0.0 } };
    std::vector< int > ib;
    std::vector< std::array< int, 3 > > cell;
    mesh.locate( x, ib, cell );
    if( ib[ 0 ] < 0 || ib[ 1 ] != -1 ) return 2;
    std::printf( "OK locate ib=%d cell=%d,%d,%d\n", ib[ 0 ], cell[ 0 ][ 0 ], cell[ 0 ][ 1 ],
                 cell[ 0 ][ 2 ] );
    try
    {
        kp::mesh_t bad( "/nonexistent/problem.ini" );
        return 3;
    }
    catch( const std::runtime_error & e )
    {
        if( std::strlen( e.what(  ) ) < 24 ) return 4;
        std::printf( "OK throws \"%s\"\n", e.what(  ) );
    }
    std::printf( "OK abi %d\n", kp_abi_version(  ) );
    // peel-off queue limit: checked before any device work
    mesh.peel_queue_limit( 1 << 20 );
    try
    {
        mesh.peel_queue_limit( 100 );
        return 6;
    }
    catch( const std::runtime_error & e )
    {
        std::printf( "OK queue limit throws \"%s\"\n", e.what(  ) );
    }
    kp::transport::split_event( nullptr );
    // spherical mesh and runtime refinement through the C++ layer
    kp_mesh_desc_t d {};
    const double lo[ 3 ] = { 1.0, 0.4, 0.0 }, hi[ 3 ] = { 3.0, 2.7, 6.283185307179586 };
    for( int a = 0; a < 3; ++ a )
    {
        d.x_min[ a ] = lo[ a ]; d.x_max[ a ] = hi[ a ];
        d.n_cell_global[ a ] = 16; d.n_cell_block[ a ] = 8;
    }
    d.periodic[ 2 ] = 1;
    kp::mesh_t sph = kp::mesh_t::spherical( d, -1.0 );
    std::vector< int > flags( sph.info(  ).n_blocks, 0 );
    flags[ 0 ] = 1;
    kp::mesh_t fine = sph.adapt( flags );
    if( fine.info(  ).n_blocks != sph.info(  ).n_blocks + 7 ) return 5;
    std::printf( "OK spherical blocks=%d adapted=%d\n", sph.info(  ).n_blocks, fine.info(  ).n_blocks );
    return 0;
}

static int gpu_part( const char * ini )
{
    kp::device_t dev( 0 );
    kp::mesh_t mesh( ini );
    const long long n_cells = mesh.info(  ).n_cells;
    std::vector< float > sigma( 2 * n_cells );
    for( long long i = 0; i < n_cells; ++ i ) { sigma[ 2 * i ] = 2.0f; sigma[ 2 * i + 1 ] = 0.5f; }
    mesh.set_sigma( sigma.data(  ), ( long long ) sigma.size(  ) );

    const int nm = 10, nb = 4;
    kp_source_t src = { KP_SOURCE_POINT, KP_EMIT_ISOTROPIC, { 0.5, 0.5, 0.5 } };
    kp_transport_cfg_t cfg;
    std::memset( & cfg, 0, sizeof( cfg ) );
    cfg.n_packets = 20000; cfg.seed = 3; cfg.phase = KP_PHASE_RAYLEIGH;
    cfg.n_sources = 1; cfg.sources = & src;
    cfg.n_mu_bins = nm; cfg.mu_lo = -1.f; cfg.mu_hi = 1.f;
    cfg.tally_mode = KP_TALLY_FIXED; cfg.fx_shift = 30; cfg.n_batches = nb;
    cfg.w_min = 0.01f; cfg.max_scatter = 1000; cfg.max_steps = 1 << 20;

    long long * d_mu = dev.malloc_device< long long >( nb * nm * 4 );
    unsigned long long * d_cnt = dev.malloc_device< unsigned long long >( KP_NCOUNTERS );
    kp::stream_t s = dev.yield_stream(  );
    dev.mset( d_mu, 0, nb * nm * 4, s );
    dev.mset( d_cnt, 0, KP_NCOUNTERS, s );
    kp_tallies_t tal = { d_mu, nullptr, nullptr, d_cnt, nullptr };
    kp::event_t e0 = dev.event_create(  ), e1 = dev.event_create(  );
    dev.event_record( e0, s );
    kp::transport::forward( mesh, cfg, tal, s );
    dev.event_record( e1, s );
    std::atomic< int > called { 0 };
    dev.launch_host( s, [ & called ] {  called = 1; } );
    unsigned long long * h_cnt = dev.malloc_host< unsigned long long >( KP_NCOUNTERS );
    dev.cp_a( h_cnt, d_cnt, KP_NCOUNTERS, s );
    dev.sync_stream( s );
    if( mesh.status( s ) != 0 ) return 10;
    if( h_cnt[ KP_CNT_EMITTED ] != ( unsigned long long ) cfg.n_packets ) return 11;
    if( h_cnt[ KP_CNT_ESCAPED ] + h_cnt[ KP_CNT_ABSORBED ] + h_cnt[ KP_CNT_CAPPED ]
        + h_cnt[ KP_CNT_LOST ] != ( unsigned long long ) cfg.n_packets ) return 12;
    if( called != 1 ) return 13;
    std::printf( "OK forward emitted=%llu escaped=%llu steps=%llu ms=%.3f\n",
                 h_cnt[ KP_CNT_EMITTED ], h_cnt[ KP_CNT_ESCAPED ], h_cnt[ KP_CNT_STEPS ],
                 dev.elapsed_ms( e0, e1 ) );
    try
    {   // a bad configuration is refused with an exception, nothing launched
        kp_transport_cfg_t bad = cfg;
        bad.n_batches = 0;
        kp::transport::forward( mesh, bad, tal, s );
        return 14;
    }
    catch( const std::runtime_error & e ) { std::printf( "OK throws \"%s\"\n", e.what(  ) ); }
    dev.event_destroy( e0 );
    dev.event_destroy( e1 );
    dev.free_host( h_cnt );
    dev.free_device( d_mu );
    dev.free_device( d_cnt );
    return 0;
}

int main( int argc, char ** argv )
{
    if( argc < 3 ) return 64;
    try
    {
        const int rc = std::strcmp( argv[ 1 ], "gpu" ) == 0 ? gpu_part( argv[ 2 ] )
                                                          : host_part( argv[ 2 ] );
        if( rc ) std::printf( "FAIL %d\n", rc );
        return rc;
    }
    catch( const std::exception & e )
    {
        std::printf( "FAIL exception %s\n", e.what(  ) );
        return 99;
    }
}
