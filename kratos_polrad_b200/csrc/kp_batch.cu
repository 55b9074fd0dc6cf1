// Batched transport: many independent scenes in one persistent launch.
//
// The reference runs one mesh per process and one generate + integrate
// cycle at a time (modules/particle/driver.h:59-79).  Here the block tables
// of all scenes are concatenated into one multi-scene mesh (block ids and
// neighbour ids shifted by each scene's block offset, so the walk and its
// hand-offs never cross into another scene), and one persistent launch of the
// forward kernel serves every scene's packets: a packet index is mapped to its
// scene through a prefix table, emitted at the scene's source with the
// scene's RNG stream and local packet id, and tallied into the scene's own
// escape tallies.  A scene's packets are therefore identical to those of a
// single-scene solve with the same seed and stream id.  The launch (counter
// reset + kernel) can be captured once into a CUDA graph and replayed, and an
// autotuner picks the block size, the event batch and the grid fill.
#include "kp_transport.cuh"

#include <algorithm>
#include <vector>

using kp::guarded;
using kp::require;

struct kp_batch
{
    int        n_scenes = 0;
    int        device   = -1;
    long long  total    = 0;
    std::vector< kp_mesh_t * > meshes;
    std::vector< long long >   cell_off;       // first cell of each scene
    std::vector< long long >   prefix;         // packet index prefix [n + 1]
    long long                  n_cells = 0;    // of the concatenated mesh
    std::vector< kp::scene_dev_t > scenes;
    kp::mesh_view_t view {  };
    int        * d_nb = nullptr;
    kp::blk_meta_t * d_meta = nullptr;
    double     * d_geo = nullptr;
    float2     * d_sigma = nullptr;
    float      * d_ext = nullptr;              // sca + abs per cell, from d_sigma
    unsigned   * d_status = nullptr;
    unsigned long long * d_work = nullptr;
    long long  * d_prefix = nullptr;
    long long  * d_prefix_trial = nullptr;      // autotuner sample
    kp::scene_dev_t * d_scenes = nullptr;
    // launch shape (autotuned)
    int threads = 256, lane_batch = 6, grid_pct = 100;
    // CUDA graph of the last launch configuration
    cudaGraphExec_t gexec = nullptr;
    kp::fwd_params_t gparams {  };
    int g_tally_mode = -1;

    ~kp_batch(  )
    {
        if( gexec ) cudaGraphExecDestroy( gexec );
        cudaFree( d_nb ); cudaFree( d_meta ); cudaFree( d_geo ); cudaFree( d_sigma );
        cudaFree( d_ext );
        cudaFree( d_status ); cudaFree( d_work ); cudaFree( d_prefix );
        cudaFree( d_prefix_trial ); cudaFree( d_scenes );
    }
};

namespace
{

void copy_sigma( kp_batch_t * b, cudaStream_t s )
{
    for( int k = 0; k < b->n_scenes; ++ k )
    {
        kp_mesh_t * m = b->meshes[ k ];
        const auto & t = m->tree->tables(  );
        const size_t n = ( size_t ) t.n_blocks * t.cells_per_block;
        KP_CUDA( cudaMemcpyAsync( b->d_sigma + b->cell_off[ k ], m->d_sigma, n * sizeof( float2 ),
                                  cudaMemcpyDeviceToDevice, s ) );
    }
    kp::extinction( b->d_sigma, b->d_ext, b->n_cells, s );
}

// Launch parameters of a batched solve.
void make_batch_params( kp_batch_t * b, const kp_transport_cfg_t & c, void * mu,
                        unsigned long long * counters, kp::fwd_params_t & P, bool trial )
{
    require( c.image_n == 0, "batched solves tally escapes only (image_n must be 0)" );
    require( c.n_mu_bins > 0 && mu, "batched solves need escape tallies (n_mu_bins > 0, mu)" );
    require( c.packets == nullptr, "batched scenes emit from their point sources (packets must be null)" );
    kp_tallies_t t {  };
    t.mu = mu;
    t.counters = counters;
    kp_transport_cfg_t cc = c;
    cc.n_record = 0;
    cc.n_packets = trial ? b->prefix.back(  ) : b->total;
    kp::fill_common_params( cc, t, P );
    P.m = b->view;
    P.n_scenes = b->n_scenes;
    P.scene_prefix = trial ? b->d_prefix_trial : b->d_prefix;
    P.scenes = b->d_scenes;
    P.mu_scene_stride = ( long long ) c.n_batches * c.n_mu_bins * 4;
    P.n_src = 1;
    P.work = b->d_work;
    if( b->lane_batch > 0 && c.lane_batch == 0 ) P.ev_batch = b->lane_batch;
}

}   // namespace

extern "C" {

int kp_batch_create( int n_scenes, const kp_scene_t * sc, kp_batch_t ** out )
{
    return guarded( "kp_batch_create", [ & ]
    {
        require( n_scenes >= 1 && sc && out, "need at least one scene" );
        auto b = std::make_unique< kp_batch >(  );
        b->n_scenes = n_scenes;
        int nb_total = 0;
        std::vector< int > blk_off( n_scenes );
        for( int k = 0; k < n_scenes; ++ k )
        {
            require( sc[ k ].mesh && sc[ k ].mesh->tree, "scene without a mesh" );
            require( sc[ k ].n_packets >= 0, "negative packet count" );
            const auto & t = sc[ k ].mesh->tree->tables(  );
            const auto & t0 = sc[ 0 ].mesh->tree->tables(  );
            for( int a = 0; a < 3; ++ a )
                require( t.nc[ a ] == t0.nc[ a ], "scenes must share the cells per block",
                         KP_ERR_CONFIG );
            sc[ k ].mesh->upload(  );
            blk_off[ k ] = nb_total;
            nb_total += t.n_blocks;
            b->meshes.push_back( sc[ k ].mesh );
        }
        KP_CUDA( cudaGetDevice( & b->device ) );
        const auto & t0 = sc[ 0 ].mesh->tree->tables(  );
        const int cpb = t0.cells_per_block;
        // concatenated tables
        std::vector< int > nb( 24 * ( size_t ) nb_total );
        std::vector< kp::blk_meta_t > meta( nb_total );
        std::vector< double > geo( 16 * ( size_t ) nb_total, 0.0 );
        b->prefix.assign( n_scenes + 1, 0 );
        for( int k = 0; k < n_scenes; ++ k )
        {
            const auto & t = sc[ k ].mesh->tree->tables(  );
            for( int i = 0; i < t.n_blocks; ++ i )
            {
                const size_t g = blk_off[ k ] + i;
                for( int s = 0; s < 24; ++ s )
                {
                    const int id = t.nb_id[ 24 * ( size_t ) i + s ];
                    nb[ 24 * g + s ] = id < 0 ? -1 : id + blk_off[ k ];
                }
                auto & m = meta[ g ];
                std::memset( & m, 0, sizeof( m ) );
                for( int f = 0; f < 6; ++ f )
                {
                    m.d_lvl[ f ] = t.d_lvl[ 6 * ( size_t ) i + f ];
                    m.shift[ f ] = t.nb_shift[ 24 * ( size_t ) i + 4 * f ];
                }
                m.phybnd = t.phybnd[ i ];
                for( int a = 0; a < 3; ++ a )
                {
                    geo[ 16 * g + a ]     = t.xf0_d[ 3 * ( size_t ) i + a ];
                    geo[ 16 * g + 3 + a ] = t.dx0_d[ 3 * ( size_t ) i + a ];
                    geo[ 16 * g + 8 + a ] = 1.0 / t.dx0_d[ 3 * ( size_t ) i + a ];
                }
                geo[ 16 * g + 6 ] = t.vol0_d[ i ];
            }
            b->cell_off.push_back( ( long long ) blk_off[ k ] * cpb );
            b->prefix[ k + 1 ] = b->prefix[ k ] + sc[ k ].n_packets;
            kp::scene_dev_t d {  };
            kp::make_source( sc[ k ].mesh, sc[ k ].source, d.src );
            require( d.src.kind == KP_SOURCE_POINT, "batched scenes take point sources",
                     KP_ERR_CONFIG );
            d.src.ib += blk_off[ k ];
            d.stream = sc[ k ].stream_id;
            b->scenes.push_back( d );
        }
        b->total = b->prefix.back(  );
        const size_t n_cells = ( size_t ) nb_total * cpb;
        KP_CUDA( cudaMalloc( & b->d_nb, nb.size(  ) * sizeof( int ) ) );
        KP_CUDA( cudaMalloc( & b->d_meta, meta.size(  ) * sizeof( kp::blk_meta_t ) ) );
        KP_CUDA( cudaMalloc( & b->d_geo, geo.size(  ) * sizeof( double ) ) );
        KP_CUDA( cudaMalloc( & b->d_sigma, n_cells * sizeof( float2 ) ) );
        KP_CUDA( cudaMalloc( & b->d_ext, n_cells * sizeof( float ) ) );
        b->n_cells = ( long long ) n_cells;
        KP_CUDA( cudaMalloc( & b->d_status, 4 * sizeof( unsigned ) ) );
        KP_CUDA( cudaMalloc( & b->d_work, 4 * sizeof( unsigned long long ) ) );
        KP_CUDA( cudaMalloc( & b->d_prefix, b->prefix.size(  ) * sizeof( long long ) ) );
        KP_CUDA( cudaMalloc( & b->d_prefix_trial, b->prefix.size(  ) * sizeof( long long ) ) );
        KP_CUDA( cudaMalloc( & b->d_scenes, b->scenes.size(  ) * sizeof( kp::scene_dev_t ) ) );
        KP_CUDA( cudaMemcpy( b->d_nb, nb.data(  ), nb.size(  ) * sizeof( int ), cudaMemcpyHostToDevice ) );
        KP_CUDA( cudaMemcpy( b->d_meta, meta.data(  ), meta.size(  ) * sizeof( kp::blk_meta_t ),
                             cudaMemcpyHostToDevice ) );
        KP_CUDA( cudaMemcpy( b->d_geo, geo.data(  ), geo.size(  ) * sizeof( double ),
                             cudaMemcpyHostToDevice ) );
        KP_CUDA( cudaMemset( b->d_status, 0, 4 * sizeof( unsigned ) ) );
        KP_CUDA( cudaMemcpy( b->d_prefix, b->prefix.data(  ), b->prefix.size(  ) * sizeof( long long ),
                             cudaMemcpyHostToDevice ) );
        KP_CUDA( cudaMemcpy( b->d_scenes, b->scenes.data(  ),
                             b->scenes.size(  ) * sizeof( kp::scene_dev_t ), cudaMemcpyHostToDevice ) );
        copy_sigma( b.get(  ), nullptr );
        KP_CUDA( cudaDeviceSynchronize(  ) );
        auto & v = b->view;
        v.n_blocks = nb_total;
        for( int a = 0; a < 3; ++ a ) v.nc[ a ] = t0.nc[ a ];
        v.cpb = cpb;
        v.nb = b->d_nb;
        v.meta = b->d_meta;
        v.geo_d = b->d_geo;
        v.sigma = b->d_sigma;
        v.ext = b->d_ext;
        v.status = b->d_status;
        * out = b.release(  );
    } );
}

int kp_batch_destroy( kp_batch_t * b )
{
    return guarded( "kp_batch_destroy", [ & ] { delete b; } );
}

int kp_batch_refresh_sigma( kp_batch_t * b, void * stream )
{
    return guarded( "kp_batch_refresh_sigma", [ & ]
    {
        require( b != nullptr, "null batch" );
        copy_sigma( b, ( cudaStream_t ) stream );
    } );
}

int kp_batch_status( kp_batch_t * b, void * stream, unsigned * flags )
{
    return guarded( "kp_batch_status", [ & ]
    {
        require( b && flags, "null argument" );
        unsigned h[ 4 ];
        KP_CUDA( cudaMemcpyAsync( h, b->d_status, sizeof( h ), cudaMemcpyDeviceToHost,
                                  ( cudaStream_t ) stream ) );
        KP_CUDA( cudaStreamSynchronize( ( cudaStream_t ) stream ) );
        * flags = h[ 0 ];
        KP_CUDA( cudaMemsetAsync( b->d_status, 0, sizeof( h ), ( cudaStream_t ) stream ) );
    } );
}

int kp_batch_forward( kp_batch_t * b, const kp_transport_cfg_t * cfg, void * mu,
                      unsigned long long * counters, void * stream )
{
    return guarded( "kp_batch_forward", [ & ]
    {
        require( b && cfg, "null argument" );
        static thread_local kp::fwd_params_t P;
        make_batch_params( b, * cfg, mu, counters, P, false );
        kp::launch_forward( P, cfg->tally_mode, ( cudaStream_t ) stream, b->threads, b->grid_pct );
    } );
}

int kp_batch_graph_launch( kp_batch_t * b, const kp_transport_cfg_t * cfg, void * mu,
                           unsigned long long * counters, void * stream )
{
    return guarded( "kp_batch_graph_launch", [ & ]
    {
        require( b && cfg, "null argument" );
        auto s = ( cudaStream_t ) stream;
        require( s != nullptr, "graph launches need a non-default stream" );
        static thread_local kp::fwd_params_t P;
        make_batch_params( b, * cfg, mu, counters, P, false );
        if( ! b->gexec || std::memcmp( & P, & b->gparams, sizeof( P ) ) != 0
            || b->g_tally_mode != cfg->tally_mode )
        {   // (re)capture: counter reset + persistent kernel
            if( b->gexec ) { cudaGraphExecDestroy( b->gexec ); b->gexec = nullptr; }
            cudaGraph_t g = nullptr;
            KP_CUDA( cudaStreamBeginCapture( s, cudaStreamCaptureModeThreadLocal ) );
            try
            {
                kp::launch_forward( P, cfg->tally_mode, s, b->threads, b->grid_pct );
            }
            catch( ... )
            {
                cudaStreamEndCapture( s, & g );
                if( g ) cudaGraphDestroy( g );
                throw;
            }
            KP_CUDA( cudaStreamEndCapture( s, & g ) );
            const cudaError_t e = cudaGraphInstantiate( & b->gexec, g, 0 );
            cudaGraphDestroy( g );
            KP_CUDA( e );
            b->gparams = P;
            b->g_tally_mode = cfg->tally_mode;
        }
        KP_CUDA( cudaGraphLaunch( b->gexec, s ) );
    } );
}

// Times candidate launch shapes on a sample of every scene's packets (a
// fraction of each scene, at least 32 packets) and keeps the fastest.
int kp_batch_autotune( kp_batch_t * b, const kp_transport_cfg_t * cfg, double fraction,
                       void * mu_scratch, void * stream, kp_tune_result_t * res )
{
    return guarded( "kp_batch_autotune", [ & ]
    {
        require( b && cfg && mu_scratch, "null argument" );
        require( fraction > 0 && fraction <= 1, "fraction must be in (0, 1]" );
        auto s = ( cudaStream_t ) stream;
        std::vector< long long > tp( b->n_scenes + 1, 0 );
        for( int k = 0; k < b->n_scenes; ++ k )
        {
            const long long n = b->prefix[ k + 1 ] - b->prefix[ k ];
            tp[ k + 1 ] = tp[ k ] + std::min( n, std::max< long long >( 32, ( long long ) ( n * fraction ) ) );
        }
        KP_CUDA( cudaMemcpy( b->d_prefix_trial, tp.data(  ), tp.size(  ) * sizeof( long long ),
                             cudaMemcpyHostToDevice ) );
        // make_batch_params reads the sample's size from b->prefix.back(): swap in
        std::vector< long long > saved = b->prefix;
        b->prefix = tp;
        cudaEvent_t e0, e1;
        KP_CUDA( cudaEventCreate( & e0 ) );
        KP_CUDA( cudaEventCreate( & e1 ) );
        const int shapes[ ][ 3 ] = { { 256, 6, 100 }, { 256, 4, 100 }, { 256, 8, 100 },
                                     { 256, 12, 100 }, { 128, 6, 100 }, { 128, 8, 100 },
                                     { 256, 6, 75 }, { 128, 4, 100 } };
        constexpr int n_shapes = ( int ) ( sizeof( shapes ) / sizeof( shapes[ 0 ] ) );
        float t_min[ n_shapes ];
        for( int i = 0; i < n_shapes; ++ i ) t_min[ i ] = 1e30f;
        try
        {
            kp_transport_cfg_t c = * cfg;
            c.lane_batch = 0;
            // the first pass warms up; each shape keeps its best of three
            // timed passes (candidates differ by a few percent, a single
            // timing by about as much)
            for( int rep = 0; rep < 4; ++ rep )
                for( int i = 0; i < n_shapes; ++ i )
                {
                    b->threads = shapes[ i ][ 0 ];
                    b->lane_batch = shapes[ i ][ 1 ];
                    b->grid_pct = shapes[ i ][ 2 ];
                    kp::fwd_params_t P;
                    make_batch_params( b, c, mu_scratch, nullptr, P, true );
                    KP_CUDA( cudaEventRecord( e0, s ) );
                    kp::launch_forward( P, c.tally_mode, s, b->threads, b->grid_pct );
                    KP_CUDA( cudaEventRecord( e1, s ) );
                    KP_CUDA( cudaEventSynchronize( e1 ) );
                    float ms = 0;
                    KP_CUDA( cudaEventElapsedTime( & ms, e0, e1 ) );
                    if( rep > 0 && ms < t_min[ i ] ) t_min[ i ] = ms;
                }
        }
        catch( ... )
        {
            b->prefix = saved;
            cudaEventDestroy( e0 ); cudaEventDestroy( e1 );
            throw;
        }
        b->prefix = saved;
        cudaEventDestroy( e0 );
        cudaEventDestroy( e1 );
        int bi = 0;
        for( int i = 1; i < n_shapes; ++ i )
            if( t_min[ i ] < t_min[ bi ] ) bi = i;
        const float best = t_min[ bi ];
        b->threads = shapes[ bi ][ 0 ];
        b->lane_batch = shapes[ bi ][ 1 ];
        b->grid_pct = shapes[ bi ][ 2 ];
        if( b->gexec ) { cudaGraphExecDestroy( b->gexec ); b->gexec = nullptr; }
        if( res )
        {
            res->threads = b->threads;
            res->lane_batch = b->lane_batch;
            res->grid_pct = b->grid_pct;
            res->sample_ms = best;
            res->sample_packets = tp.back(  );
        }
    } );
}

}   // extern "C"
