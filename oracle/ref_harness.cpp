/* Reference harness: runs the reference's OWN traversal code on the host.
 *
 * Test infrastructure only (the oracle).  Built by oracle/Makefile from the
 * reference sources where they lie, together with this file, into
 * oracle/_ref/libkpref_p{1,2}.so (PRECISION=1: FP32 positions, PRECISION=2:
 * FP64 positions, src/types.h:12-27).  Nothing here is shipped.
 *
 * What is the reference's code (compiled unchanged from its tree):
 *   - INI reading                    io/args/input.cpp:72-167
 *   - mesh read / refine regions     mesh/meshgen/meshgen.cpp:13-42,111-142
 *   - 2:1 tree insert / neighbours   mesh/tree/tree.cpp:177-230
 *   - block geometry                 mesh/meshgen/meshgen.cpp:286-351
 *   - face-neighbour proxy table     modules/particle/types/proxy.h:22-62
 *   - the packet walk                modules/particle/radiation/photon.h:20-125
 *     (get_dl, proc_geo, proc_phys, proc_step, proc), geo_loc_t
 *     (types/particle_base.h:86-126), regulate (particle_base.h:37-56) and
 *     shift_blk (types/proxy.h:64-121).
 * What this harness restates (because the reference does it inside mesh_t,
 * which needs the whole framework):
 *   - meshgen::base_t::init's tree set-up (meshgen.cpp:44-55), the block
 *     loop of generate_tree (meshgen.cpp:144-163), dist_default's id order
 *     for one rank (meshgen.cpp:168-188) and the phybnd part of
 *     associate_mesh (meshgen.cpp:378-400);
 *   - block_map_t's device-facing members (types/block_map.h:21-31,
 *     84-114): periodic flags, box limits and operator[].
 */
#include "modules/particle/radiation/photon.h"
#include "modules/particle/radiation/rad_data.h"
#include "modules/particle/types/proxy.h"
#include "mesh/block/dual_data.h"
#include "mesh/meshgen/meshgen.h"
#include "mesh/meshgen/spherical.h"
// photon_sph.h names coord_t unqualified; nothing in the reference declares
// it in that namespace (the header is never instantiated there), so the
// harness supplies the name it means.
namespace particle::radiation::photon { using type::coord_t; }
#include "modules/particle/radiation/photon_sph.h"
#include "mesh/tree/tree.h"
#include "mesh/mesh.h"
#include "io/args/input.h"
#include "io/binary/binary_io_base.h"
#include "utilities/mapping/loop.h"

#include <atomic>
#include <cstdint>
#include <deque>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>
#include <thread>

using f_t = type::float_t;

////////////////////////////////////////////////////////////
// Stubs for mesh_t members that meshgen.o references but the harness never
// calls (mesh_t is the full framework; only its tree is needed here).

[[noreturn]] static void kp_ref_unreachable( const char * what )
{
    std::fprintf( stderr, "ref harness: %s is not available\n", what );
    std::abort(  );
}
namespace mesh
{
tree_t & mesh_t::tree(  ) const { kp_ref_unreachable( "mesh_t::tree" ); }
auto mesh_t::begin(  ) -> iter_t { kp_ref_unreachable( "mesh_t::begin" ); }
auto mesh_t::end  (  ) -> iter_t { kp_ref_unreachable( "mesh_t::end" ); }
block_t & mesh_t::iter_t::operator * (  )
{ kp_ref_unreachable( "mesh_t::iter_t" ); }
}

namespace
{
////////////////////////////////////////////////////////////
// Types

// A mesh generator (the Cartesian base_t, or the spherical sph_t with its
// cylindrical radial spacing) with the members the harness drives made
// accessible.
template< class G >
struct mgn_x : G
{
    using G::read;
    using mesh::meshgen::base_t::load_refinement;
    using G::set_uniformity;
    using G::set_coord_axes;
    using mesh::meshgen::base_t::set_geo_fulldim;
    const type::idx_t & nc_block(  ) const { return this->n_ceff_block; }
    const type::idx_t & lim     (  ) const { return this->i_logic_lim;  }
    int                 ndim    (  ) const { return this->n_dim;        }
    const std::vector< mesh::meshgen::refine_region_t > & regions(  ) const
    { return this->ref_regions; }
};

// Proxy carrying the radiation fields, as radiation::proxy_t does
// (radiation/radiation.h:12-14); photon.h:81 reads prx.rad.flx.
struct prx_t : particle::proxy_base_t
{
    particle::radiation::rad_t rad;
};

// Device-facing part of block_map_t (types/block_map.h:21-31, 111-114).
struct bmap_t
{
    bool            periodic[ 3 ];
    type::coord_t   l_box;
    type::coord_t   xlim[ 2 ];
    prx_t         * prx;
    prx_t & operator [  ] ( const int & i ) const { return prx[ i ]; }
};

struct harness_t
{
    std::unique_ptr< mesh::meshgen::base_t > mgn;
    type::idx_t                     nc;          // cells per block
    bool                            spherical = false;
    mesh::tree_t                    tree;
    std::deque< mesh::block_t >     blocks;     // id order
    std::vector< prx_t >            prx;
    bmap_t                          bmap;
    std::vector< f_t >              flux;       // reference float sums
    std::vector< long long >        flux_fx;    // int64 fixed point sums
    std::atomic< long long >        n_outside { 0 };  // deposits beyond the flux pool
    std::vector< f_t >              sigma;      // 2 comps per cell (mfp_i)
    int                             fx_shift = 32;
    int                             n_cell_blk = 0;
    bool                            serial = true;
};

// Runs f( p ) for p in [0, n) on n_threads host threads (contiguous chunks).
template< class F >
void parallel_for( long n, int n_threads, const F & f )
{
    if( n_threads <= 1 || n < 2 )
    {
        for( long p = 0; p < n; ++ p ) f( p );
        return;
    }
    std::vector< std::thread > pool;
    std::atomic< long > next( 0 );
    const long chunk = 256;
    for( int t = 0; t < n_threads; ++ t )
        pool.emplace_back( [ & ]
        {
            for( long b; ( b = next.fetch_add( chunk ) ) < n; )
                for( long p = b; p < std::min( n, b + chunk ); ++ p )
                    f( p );
        } );
    for( auto & th : pool ) th.join(  );
}

std::unique_ptr< harness_t > g_h;
alignas( 64 ) unsigned char g_mod_storage[ 64 ];

size_t carve_offset = 0;
}

////////////////////////////////////////////////////////////
// Deposit hook (see ref_compat.h): p points into g_h->flux.

static inline void deposit_impl( f_t * p, f_t v )
{
    auto & h = * g_h;
    const ptrdiff_t k = p - h.flux.data(  );
    if( k < 0 || k >= ( ptrdiff_t ) h.flux.size(  ) )
    {   // the spherical walk deposits with an out-of-range cell index after
        // some corner crossings; beyond the pool it would corrupt the heap
        h.n_outside.fetch_add( 1, std::memory_order_relaxed );
        return;
    }
    const long long q = std::llrint( std::ldexp( ( double ) v, h.fx_shift ) );
    if( h.serial )
        h.flux[ k ] += v;           // packet order, as one host thread
    else
    {   // CAS loop: float atomics as the device performs them
        std::atomic_ref< f_t > r( h.flux[ k ] );
        f_t cur = r.load( std::memory_order_relaxed );
        while( ! r.compare_exchange_weak( cur, cur + v,
                                          std::memory_order_relaxed ) ) {}
    }
    __atomic_fetch_add( & h.flux_fx[ k ], q, __ATOMIC_RELAXED );
}
void kp_ref_deposit( float  * p, float  v )
{
    if constexpr( std::is_same_v< f_t, float > ) deposit_impl( ( f_t * ) p, v );
}
void kp_ref_deposit( double * p, double v )
{
    if constexpr( std::is_same_v< f_t, double > ) deposit_impl( ( f_t * ) p, v );
}

////////////////////////////////////////////////////////////
// Mesh construction

template< class G >
static void build_mesh( const std::string & ini )
{
    g_h = std::make_unique< harness_t >(  );
    auto & h = * g_h;
    input args( ini, false );
    if( ! args.read(  ) )
        throw std::runtime_error( "cannot read " + ini );
    auto mg = std::make_unique< mgn_x< G > >(  );
    auto & mgn = * mg;

    // meshgen::base_t::init (meshgen.cpp:44-55)
    mgn.read( args );
    h.tree.n_dim    = mgn.ndim(  );
    h.tree.reg_max  = mgn.lim (  );
    h.tree.periodic = { false, false, false };
    std::vector< std::string > kinds;
    args( "boundary", "kinds", kinds );
    for( int side = 0; side < ( int ) kinds.size(  ); ++ side )
        h.tree.periodic[ side / 2 ] =
            kinds[ side ].find( "per" ) != std::string::npos;

    // generate_tree (meshgen.cpp:144-163) on the harness's own tree
    mgn.load_refinement( args );
    for( const auto & ref : mgn.regions(  ) )
        if( ref.level > 0 )
            for( const auto & i : utils::loop( ref.i[ 0 ], ref.i[ 1 ], true ) )
            {
                mesh::region_logic_t reg;
                reg       = i;
                reg.level = ref.level;
                h.tree.insert( reg );
            }
    h.tree.fill_base_level(  );

    // dist_default for a single rank (meshgen.cpp:168-188)
    int id = 0;
    for( auto & p : h.tree )
    {
        if( p.second.mask )
            continue;
        p.second.rank = 0;
        p.second.id_g = id;
        p.second.id_l = id;
        ++ id;
    }

    // create (meshgen.cpp:402-432) with associate_mesh's phybnd part
    for( auto & p : h.tree )
    {
        if( p.second.mask )
            continue;
        h.blocks.emplace_back(  );
        auto & b     = h.blocks.back(  );
        b.neighbors  = h.tree.neighbors( p.first );
        b.reg        = p.first;
        b.id_l       = p.second.id_l;
        b.id_g       = p.second.id_g;
        b.rank       = 0;
        const auto reg_lim = h.tree.region_max( b.reg.level );
        for( int a = 0; a < 3; ++ a )
            if( ! h.tree.periodic[ a ] )
            {
                b.geo.phybnd_flag[ a ][ 0 ] = ( b.reg[ a ] == 0 );
                b.geo.phybnd_flag[ a ][ 1 ] = ( reg_lim[ a ] - 1 == b.reg[ a ] );
            }
    }
    const mesh::f_new_t f_host = [ ]( const size_t & s ) -> void *
    { return std::malloc( s ); };
    for( auto & b : h.blocks )
    {
        mgn.set_uniformity( b );
        b.geo.setup( mgn.nc_block(  ), 1, f_host );
        mgn.set_coord_axes( b );
        mgn.set_geo_fulldim( b );
    }

    // Fields: one contiguous flux pool so that deposits map to cells.
    const auto & nc = mgn.nc_block(  );
    h.nc = nc;
    h.n_cell_blk = nc[ 0 ] * nc[ 1 ] * nc[ 2 ];
    const size_t nb = h.blocks.size(  );
    h.flux   .assign( nb * h.n_cell_blk, 0 );
    h.flux_fx.assign( nb * h.n_cell_blk, 0 );
    h.sigma  .assign( nb * h.n_cell_blk * 2, 0 );
    h.prx    .resize( nb );

    std::map< int, int > m_rank;
    auto & mod = * reinterpret_cast< particle::base_t * >( g_mod_storage );
    for( auto & b : h.blocks )
    {
        mesh::block::dual_t d( b );
        d.p_d = std::make_shared< mesh::block::base_data_t >(  );
        b.geo.cp_shlw( d.p_d->geo );
        auto & px = h.prx[ b.id_l ];
        // proxy.h:22-62; its `mod` argument is not used by the body.
        px.particle::proxy_base_t::setup( d, m_rank, mod );
        px.rad.flx.n_int = 1;
        carve_offset = ( size_t ) b.id_l * h.n_cell_blk;
        px.rad.flx.init( [ & ]( const size_t & ) -> void *
                         { return h.flux.data(  ) + carve_offset; },
                         nc, type::idx_t::null(  ), 1 );
        px.rad.mfp_i.init( [ & ]( const size_t & ) -> void *
                           { return h.sigma.data(  ) + carve_offset * 2; },
                           nc, type::idx_t::null(  ), 2 );
    }

    // block_map_t::update's box limits (block_map.h:84-103)
    const auto & xl = mgn.x_lim_global;
    for( int a = 0; a < 3; ++ a )
    {
        h.bmap.periodic[ a ] = h.tree.periodic[ a ];
        for( int l = 0; l < 2; ++ l )
            h.bmap.xlim[ l ][ a ] = xl[ l ][ a ];
        h.bmap.l_box[ a ] = xl[ 1 ][ a ] - xl[ 0 ][ a ];
    }
    h.bmap.prx = h.prx.data(  );
    h.mgn = std::move( mg );
}

////////////////////////////////////////////////////////////
// C ABI for the tests

extern "C" {

int kpref_float_size( void ) { return ( int ) sizeof( f_t ); }

int kpref_mesh_load( const char * ini_path )
{
    try { build_mesh< mesh::meshgen::base_t >( ini_path ); }
    catch( const std::exception & e )
    {
        std::fprintf( stderr, "kpref_mesh_load: %s\n", e.what(  ) );
        g_h.reset(  );
        return -1;
    }
    return ( int ) g_h->blocks.size(  );
}

int kpref_n_blocks( void ) { return g_h ? ( int ) g_h->blocks.size(  ) : 0; }

// Deposits since the last call whose cell lay beyond the flux pool (skipped).
long long kpref_deposits_outside( void )
{
    return g_h ? g_h->n_outside.exchange( 0 ) : 0;
}

int kpref_block_cells( int * n3 )
{
    const auto & nc = g_h->nc;
    for( int a = 0; a < 3; ++ a ) n3[ a ] = nc[ a ];
    return g_h->n_cell_blk;
}

/* Region keys (level, logical index) per block id. */
void kpref_blocks( int * level, int * reg3 )
{
    for( const auto & b : g_h->blocks )
    {
        level[ b.id_l ] = b.reg.level;
        for( int a = 0; a < 3; ++ a )
            reg3[ 3 * b.id_l + a ] = b.reg[ a ];
    }
}

/* Geometry per block id, as float_t widened to double. */
void kpref_geo( double * xf0, double * dx0, double * vol0, int * phybnd )
{
    for( const auto & px : g_h->prx )
    {
        const int i = ( int ) ( & px - g_h->prx.data(  ) );
        for( int a = 0; a < 3; ++ a )
        {
            xf0[ 3 * i + a ] = px.geo.xf0[ a ];
            dx0[ 3 * i + a ] = px.geo.dx0[ a ];
            for( int s = 0; s < 2; ++ s )
                phybnd[ 6 * i + 2 * a + s ] = px.geo.phybnd_flag[ a ][ s ];
        }
        vol0[ i ] = px.geo.vol0;
    }
}

/* Face-neighbour table per block id, layout [a][side][j0][j1]. */
void kpref_nb( int * nb_id, int * nb_shift, int * d_lvl )
{
    for( size_t i = 0; i < g_h->prx.size(  ); ++ i )
    {
        const auto & px = g_h->prx[ i ];
        for( int a = 0; a < 3; ++ a )
            for( int s = 0; s < 2; ++ s )
            {
                d_lvl[ 6 * i + 2 * a + s ] = px.d_lvl[ 2 * a + s ];
                for( int j0 = 0; j0 < 2; ++ j0 )
                    for( int j1 = 0; j1 < 2; ++ j1 )
                    {
                        const auto & n = px.neighbors[ a ][ s ][ j0 ][ j1 ];
                        const int k = ( ( a * 2 + s ) * 2 + j0 ) * 2 + j1;
                        nb_id   [ 24 * i + k ] = n.id;
                        nb_shift[ 48 * i + 2 * k + 0 ] = n.shift[ 0 ];
                        nb_shift[ 48 * i + 2 * k + 1 ] = n.shift[ 1 ];
                    }
            }
    }
}

void kpref_box( double * xlim, double * l_box, int * periodic )
{
    for( int a = 0; a < 3; ++ a )
    {
        xlim[ a ] = g_h->bmap.xlim[ 0 ][ a ];
        xlim[ 3 + a ] = g_h->bmap.xlim[ 1 ][ a ];
        l_box[ a ] = g_h->bmap.l_box[ a ];
        periodic[ a ] = g_h->bmap.periodic[ a ];
    }
}

/* Per-cell coefficients (sigma_sca, sigma_abs) in block-major, x-fastest
 * cell order; stored in the proxies' rad.mfp_i fields (two components). */
void kpref_set_sigma( const float * sig2 )
{
    for( size_t k = 0; k < g_h->sigma.size(  ); ++ k )
        g_h->sigma[ k ] = sig2[ k ];
}

/* Geometric walk: photon::cart_t<>::proc (photon.h:104-125) per packet.
 * Inputs are double arrays holding values representable in float_t. */
int kpref_trace( long n, const double * x, const double * dir,
                 const int * cell, const int * ib, const double * proper,
                 const int * steps, int fx_shift, int n_threads,
                 double * x_out, int * cell_out, int * ib_out,
                 int * step_out, int * todo_out,
                 double * flux_out, long long * flux_fx_out )
{
    if( ! g_h ) return -1;
    auto & h = * g_h;
    h.fx_shift = fx_shift;
    std::fill( h.flux.begin(  ), h.flux.end(  ), 0 );
    std::fill( h.flux_fx.begin(  ), h.flux_fx.end(  ), 0 );
    h.serial = ( n_threads <= 1 );
    parallel_for( n, n_threads, [ & ]( long p )
    {
        particle::radiation::photon::cart_t<  > par;
        par.dest.todo = particle::to_keep;
        par.id        = ( int ) p;
        for( int a = 0; a < 3; ++ a )
        {
            par.x  [ a ] = ( f_t ) x  [ 3 * p + a ];
            par.dir[ a ] = ( f_t ) dir[ 3 * p + a ];
            par.i  [ a ] = cell[ 3 * p + a ];
        }
        par.ib_l   = ib[ p ];
        par.proper = ( f_t ) proper[ p ];
        par.step   = steps[ p ];
        const int itg = 0;
        par.proc( h.bmap, itg );
        for( int a = 0; a < 3; ++ a )
        {
            x_out   [ 3 * p + a ] = par.x[ a ];
            cell_out[ 3 * p + a ] = par.i[ a ];
        }
        ib_out  [ p ] = par.ib_l;
        step_out[ p ] = par.step;
        todo_out[ p ] = par.dest.todo;
    } );
    if( flux_out )
        for( size_t k = 0; k < h.flux.size(  ); ++ k )
            flux_out[ k ] = h.flux[ k ];
    if( flux_fx_out )
        std::copy( h.flux_fx.begin(  ), h.flux_fx.end(  ), flux_fx_out );
    return 0;
}

// Spherical-polar mesh (meshgen::sph_t on cyl_t's radial spacing, [mesh]
// r_ratio; mesh/meshgen/spherical.h, cylindrical.h): axes (r, theta, phi).
int kpref_mesh_load_sph( const char * ini_path )
{
    try { build_mesh< mesh::meshgen::sph_t >( ini_path ); }
    catch( const std::exception & e )
    {
        std::fprintf( stderr, "kpref_mesh_load_sph: %s\n", e.what(  ) );
        g_h.reset(  );
        return -1;
    }
    g_h->spherical = true;
    return ( int ) g_h->blocks.size(  );
}

// Per block: the radial faces x_fc( 0, 0..nc0 ) and every cell's volume
// (geo_t::volume, x fastest), as float_t widened to double.
int kpref_geo_sph( double * r_faces, double * vol )
{
    if( ! g_h ) return -1;
    auto & h = * g_h;
    const auto & nc = h.nc;
    for( const auto & b : h.blocks )
    {
        const size_t id = b.id_l;
        for( int i = 0; i <= nc[ 0 ]; ++ i )
            r_faces[ id * ( nc[ 0 ] + 1 ) + i ] = b.geo.x_fc( 0, i );
        size_t k = id * h.n_cell_blk;
        for( int c2 = 0; c2 < nc[ 2 ]; ++ c2 )
            for( int c1 = 0; c1 < nc[ 1 ]; ++ c1 )
                for( int c0 = 0; c0 < nc[ 0 ]; ++ c0 )
                    vol[ k ++ ] = b.geo.volume( type::idx_t( c0, c1, c2 ) );
    }
    return 0;
}

// photon::sph_t::proc (modules/particle/radiation/photon_sph.h) for every
// packet: spherical x (r, theta, phi) and its Cartesian copy in, final state
// and flux out.
int kpref_trace_sph( long n, const double * x, const double * x_car, const double * dir,
                     const int * cell, const int * ib, const double * proper,
                     const int * steps, int fx_shift, int n_threads,
                     double * x_out, double * x_car_out, int * cell_out, int * ib_out,
                     int * step_out, int * todo_out,
                     double * flux_out, long long * flux_fx_out )
{
    if( ! g_h || ! g_h->spherical ) return -1;
    auto & h = * g_h;
    h.fx_shift = fx_shift;
    std::fill( h.flux.begin(  ), h.flux.end(  ), 0 );
    std::fill( h.flux_fx.begin(  ), h.flux_fx.end(  ), 0 );
    h.serial = ( n_threads <= 1 );
    parallel_for( n, n_threads, [ & ]( long p )
    {
        particle::radiation::photon::sph_t<  > par;
        par.dest.todo = particle::to_keep;
        par.id        = ( int ) p;
        for( int a = 0; a < 3; ++ a )
        {
            par.x    [ a ] = ( f_t ) x    [ 3 * p + a ];
            par.x_car[ a ] = ( f_t ) x_car[ 3 * p + a ];
            par.dir  [ a ] = ( f_t ) dir  [ 3 * p + a ];
            par.i    [ a ] = cell[ 3 * p + a ];
        }
        par.ib_l   = ib[ p ];
        par.proper = ( f_t ) proper[ p ];
        par.step   = steps[ p ];
        const int itg = 0;
        par.proc( h.bmap, itg );
        for( int a = 0; a < 3; ++ a )
        {
            x_out    [ 3 * p + a ] = par.x[ a ];
            x_car_out[ 3 * p + a ] = par.x_car[ a ];
            cell_out [ 3 * p + a ] = par.i[ a ];
        }
        ib_out  [ p ] = par.ib_l;
        step_out[ p ] = par.step;
        todo_out[ p ] = par.dest.todo;
    } );
    if( flux_out )
        for( size_t k = 0; k < h.flux.size(  ); ++ k )
            flux_out[ k ] = h.flux[ k ];
    if( flux_fx_out )
        std::copy( h.flux_fx.begin(  ), h.flux_fx.end(  ), flux_fx_out );
    return 0;
}

// The reference's binary container: binary_io::base_t::write for every entry
// (copied into its buffers), then save (io/binary/binary_io_base.cpp:89-131).
int kpref_bio_write( const char * path, int n, const char * const * tags,
                     const void * const * data, const unsigned long long * counts,
                     const int * unit_sizes )
{
    try
    {
        binary_io::base_t b;
        b.open( path, "w" );
        for( int i = 0; i < n; ++ i )
            b.write( data[ i ], ( size_t ) counts[ i ], ( size_t ) unit_sizes[ i ], tags[ i ],
                     true );
        b.save(  );
        b.close(  );
        return 0;
    }
    catch( const std::exception & )
    {
        return -1;
    }
}

// Loads a container with binary_io::base_t::load and reads one entry:
// returns its element count (base_t::read), or -1 if it cannot.
long long kpref_bio_read( const char * path, const char * tag, void * dst,
                          unsigned long long * size, int * unit_size )
{
    try
    {
        binary_io::base_t b;
        b.open( path, "r" );
        b.load(  );
        const auto & in = b.info( tag );
        if( size ) * size = in.size;
        if( unit_size ) * unit_size = in.u_size;
        long long n = 0;
        if( dst ) n = ( long long ) b.read( dst, tag );
        b.close(  );
        return n;
    }
    catch( const std::exception & )
    {
        return -1;
    }
}

}   // extern "C"
