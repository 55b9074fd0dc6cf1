// kratos_polrad_b200 — the particle radiation module, over the C ABI.
//
// Mirrors the reference's module layer for the transport path:
// particle::radiation::base_t::read/enroll (modules/particle/radiation/
// radiation.h:19-55) and particle::base_t::init/step/save/finalize with the
// per-cycle integrate (modules/particle/driver.h:15-101, driver.cpp:8-60):
//
//   base_t rad;
//   rad.read( "problem.ini" );            // [particle] n_par, step_max, n_hv,
//                                         // n_cycle_stp, [device] seed_rng ...
//   rad.transport_cfg(  ).image_n = 128;  // physics and tallies beyond the keys
//   rad.enroll( kp::generate::on_device( my_gen_t {  } ) );   // the user hook
//   rad.init( mesh );
//   rad.step(  );                         // n_cycle_stp cycles
//   rad.save( "out.bin" );                // rad_t::write's per-block tags
//
// A cycle is generate + integrate: the enrolled generator fills n_par packets
// (kp_packet_init_t, the pool entries the reference's generator functor
// writes; kp_generate.cuh launches a __device__ functor per packet as ker_gen
// does), then one kp_transport_forward walks them.  Without a generator the
// packets come from the sources(), so the default set compiles and runs.
// Packet ids continue across cycles (a cycle holds ids done .. done + n_par
// - 1), so every packet has its own RNG stream and the int64 tallies of a
// run are those of one solve over all its packets.  The tallies accumulate
// over the run: escape mu bins, the peel-off image, counters and the
// path-length flux (rad_t::flx; the walk deposits into field 0 of the n_hv
// fields, as photon.h:81 does).
//
// A packet that uses up its step_max segments in a cycle ends there, as in
// the reference (photon.h:122-123), unless the module's comm_mode() is
// keep_pool: then it waits in the module's pool and the next cycle resumes
// it before the cycle's new packets (kp_transport_forward_resume); drain()
// runs cycles without new packets until the pool is empty.
//
// Host C++17; the generator header needs nvcc.  Every failure throws
// std::runtime_error (kp::api), as the reference's cuda_api does.
#ifndef KP_MODULE_HPP
#define KP_MODULE_HPP

#include "kp_transport.hpp"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

namespace kp::particle
{
// Whether a cycle's unfinished packets stay in the pool (particle::
// comm_mode_t, modules/particle/types/driver_base.h:12).
enum comm_mode_t : int { refresh_pool, keep_pool };
}   // namespace kp::particle

namespace kp::particle::radiation
{

// Generator hook: fills `table` (device, n entries) for the packets with
// global ids pid0 .. pid0 + n - 1, on stream s.
using generator_t = std::function< void( kp_packet_init_t * table, long long n, long long pid0,
                                         void * s ) >;

class base_t
{
public:
    base_t(  )
    {
        std::memset( & par_, 0, sizeof( par_ ) );
        par_.n_par = 1.0; par_.f_par = 1.0; par_.step_max = 100; par_.n_hv = 1;
        par_.n_cycle_stp = 1; par_.n_th = 64; par_.max_round = 16; par_.output = 1;
        par_.seed_rng = 7; par_.idx_device = -1;
        std::memset( & cfg_, 0, sizeof( cfg_ ) );
        cfg_.seed = 7;
        cfg_.phase = KP_PHASE_RAYLEIGH;
        cfg_.pol_max = 1.0f;
        cfg_.mu_lo = -1.0f;
        cfg_.mu_hi = 1.0f;
        cfg_.inclination_deg = 90.0;
        cfg_.image_half_width = 1.0;
        cfg_.tau_peel_max = 40.0f;
        cfg_.tally_mode = KP_TALLY_FIXED;
        cfg_.fx_shift = 32;
        cfg_.flux_fx_shift = 24;
        cfg_.n_batches = 32;
        cfg_.image_batch_n = 1;
        cfg_.rr_survive = 0.1f;
        cfg_.max_scatter = 100000;
        cfg_.max_steps = par_.step_max;
    }
    virtual ~base_t(  ) { finalize(  ); }
    base_t( const base_t & ) = delete;
    base_t & operator=( const base_t & ) = delete;

    // radiation::base_t::read and the drivers' init(): the [particle],
    // [particles] and [device] keys (kp_particle_read).  seed_rng becomes the
    // RNG seed, step_max the segment cap of a packet.
    virtual void read( const std::string & ini_path )
    {
        api( kp_particle_read( ini_path.c_str(  ), & par_ ) );
        cfg_.seed = ( uint32_t ) par_.seed_rng;
        cfg_.max_steps = par_.step_max;
    }
    const kp_particle_cfg_t & particle_cfg(  ) const { return par_; }
    // Physics and tally settings that the INI keys do not cover (phase
    // matrix, image, mu bins, fixed-point scales, roulette ...).  n_packets,
    // packet_offset, sources and packets are set per cycle by integrate().
    kp_transport_cfg_t & transport_cfg(  ) { return cfg_; }
    // Sources of the default set (used when no generator is enrolled).
    std::vector< kp_source_t > & sources(  ) { return src_; }

    // radiation::base_t::enroll: the user's packet generator; an empty one
    // keeps the default set (the sources()).
    virtual void enroll( generator_t gen = nullptr ) { gen_ = std::move( gen ); }

    // particle::base_t::comm_mode (modules/particle/driver.cpp:67-69):
    // refresh_pool, the reference's default, ends a packet that uses up its
    // step_max segments in a cycle (photon.h:122-123).  A module that returns
    // keep_pool keeps such packets in its pool instead, as the reference's
    // pool keeps its to_keep particles (types/particle_pool.h:191-248): the
    // next cycle resumes them (kp_transport_forward_resume) before its new
    // packets, each cycle gives every packet step_max more segments, and a
    // packet ends for good after pool_max_steps() segments in all.
    virtual comm_mode_t comm_mode(  ) const { return refresh_pool; }
    long long & pool_max_steps(  ) { return pool_max_; }
    // Packets waiting in the pool for the next cycle (keep_pool).
    long long pool_size(  ) const { return n_pool_; }

    // particle::base_t::init: binds the mesh and allocates the packet table
    // (with a generator) and the tallies on the current device, zeroed.
    virtual void init( mesh_t & mesh, stream_t s = nullptr )
    {
        finalize(  );
        if( par_.idx_device >= 0 )
            api( kp_device_init( par_.idx_device ) );
        mesh_ = & mesh;
        mesh.upload(  );
        n_cells_ = mesh.info(  ).n_cells;
        n_par_ = ( long long ) par_.n_par;     // size_t n_par = float n_par
        const size_t tb = cfg_.tally_mode == KP_TALLY_FIXED ? 8 : 4;
        flux_ = alloc( tb * ( size_t ) n_cells_, s );
        counters_ = static_cast< unsigned long long * >(
            alloc( sizeof( unsigned long long ) * KP_NCOUNTERS, s ) );
        if( cfg_.n_mu_bins > 0 )
            mu_ = alloc( tb * ( size_t ) cfg_.n_batches * cfg_.n_mu_bins * 4, s );
        if( cfg_.image_n > 0 )
        {
            image_ = alloc( tb * ( size_t ) cfg_.image_n * cfg_.image_n * 4, s );
            image_batch_ = alloc( tb * ( size_t ) cfg_.n_batches * cfg_.image_batch_n
                                  * cfg_.image_batch_n * 4, s );
        }
        if( gen_ && n_par_ > 0 )
            table_ = static_cast< kp_packet_init_t * >(
                alloc( sizeof( kp_packet_init_t ) * ( size_t ) n_par_, s ) );
        if( cfg_.tally_mode == KP_TALLY_FLOAT )
        {   // the float atomics' rounding errors (kp_tallies_t::carry)
            size_t n = ( size_t ) n_cells_;
            if( cfg_.n_mu_bins > 0 )
                n += ( size_t ) cfg_.n_batches * cfg_.n_mu_bins * 4;
            if( cfg_.image_n > 0 )
                n += ( size_t ) cfg_.image_n * cfg_.image_n * 4
                     + ( size_t ) cfg_.n_batches * cfg_.image_batch_n * cfg_.image_batch_n * 4;
            carry_ = static_cast< float * >( alloc( sizeof( float ) * n, s ) );
        }
        done_ = 0;
    }

    // One cycle (particle::base_t::integrate, driver.h:59-79): generate
    // n_par packets, then walk them with their scattering, peel-off and
    // tallies (kp_transport_forward).
    virtual void integrate( int /*cycle*/, stream_t s = nullptr )
    {
        if( ! mesh_ )
            throw std::runtime_error( "kratos_polrad_b200: radiation module used before init" );
        kp_transport_cfg_t c = cfg_;
        c.n_packets = n_par_;
        c.packet_offset = cfg_.packet_offset + done_;
        c.n_sources = ( int ) src_.size(  );
        c.sources = src_.empty(  ) ? nullptr : src_.data(  );
        c.packets = nullptr;
        if( gen_ && n_par_ > 0 )
        {
            gen_( table_, n_par_, c.packet_offset, s );
            c.packets = table_;
        }
        const kp_tallies_t t = tallies(  );
        if( comm_mode(  ) == keep_pool )
            integrate_pool( c, t, s );
        else
            transport::forward( * mesh_, c, t, s );
        done_ += n_par_;
    }

    // keep_pool: cycles without new packets until the pool is empty, so that
    // every packet of the run has ended (at most pool_max_steps() / step_max
    // + 1 cycles).  Nothing to do in refresh_pool mode.
    virtual void drain( stream_t s = nullptr )
    {
        if( ! mesh_ || comm_mode(  ) != keep_pool )
            return;
        const long long max_cycles = pool_max_ / std::max( par_.step_max, 1 ) + 2;
        for( long long k = 0; n_pool_ > 0; ++ k )
        {
            if( k >= max_cycles )
                throw std::runtime_error( "kratos_polrad_b200: the packet pool does not drain" );
            kp_transport_cfg_t c = cfg_;
            c.n_packets = 0;
            c.packet_offset = cfg_.packet_offset + done_;
            c.n_sources = 0;
            c.sources = nullptr;
            c.packets = nullptr;
            integrate_pool( c, tallies(  ), s );
        }
    }

    // particle::base_t::step: n_cycle_stp cycles, then the stream is synced.
    virtual void step( stream_t s = nullptr )
    {
        for( int c = 0; c < par_.n_cycle_stp; ++ c )
            integrate( c, s );
        api( kp_stream_sync( s ) );
    }

    // particle::base_t::save: per block the reference's tags
    // block_<id>|i_logic, |level and the rad_t flux field
    // |rad_flx_flux_{n_int,n_step,n_cell,n_gh,field} (n_hv float components
    // per cell, the flux w * dl / volume in component 0; rad_data.cpp:45-49,
    // dat_3d.h:117-125), then the raw tallies under kp|<name> with their
    // shapes under kp|shape|<name> and kp|packets_done, as
    // kratos_polrad_b200.bio.save_solution writes them.
    virtual void save( const std::string & path ) const
    {
        if( ! mesh_ )
            throw std::runtime_error( "kratos_polrad_b200: radiation module used before init" );
        api( kp_stream_sync( nullptr ) );
        const kp_mesh_info_t in = mesh_->info(  );
        const int cpb = in.cells_per_block, nb = in.n_blocks, nh = par_.n_hv;
        const bool fx = cfg_.tally_mode == KP_TALLY_FIXED;
        std::vector< int > level;
        std::vector< std::array< int, 3 > > reg;
        mesh_->blocks( level, reg );
        std::vector< float > flux_f( n_cells_ );
        if( fx )
        {
            std::vector< long long > flux_i( n_cells_ );
            api( kp_memcpy( flux_i.data(  ), flux_, 8 * ( size_t ) n_cells_ ) );
            const int sh = cfg_.flux_fx_shift > 0 ? cfg_.flux_fx_shift : cfg_.fx_shift;
            for( long long k = 0; k < n_cells_; ++ k )
                flux_f[ k ] = ( float ) std::ldexp( ( double ) flux_i[ k ], -sh );
        }
        else
            api( kp_memcpy( flux_f.data(  ), flux_, 4 * ( size_t ) n_cells_ ) );
        std::vector< float > field( ( size_t ) n_cells_ * nh, 0.0f );
        for( long long k = 0; k < n_cells_; ++ k )
            field[ ( size_t ) k * nh ] = flux_f[ k ];
        const int one = 1, gh[ 3 ] = { 0, 0, 0 };
        std::vector< std::string > tags;
        std::vector< kp_bio_entry_t > ent;
        auto put = [ & ]( std::string tag, const void * data, size_t count, int unit )
        {
            tags.push_back( std::move( tag ) );
            ent.push_back( kp_bio_entry_t { nullptr, data, count, unit } );
        };
        for( int b = 0; b < nb; ++ b )
        {
            const std::string p = "block_" + std::to_string( b ) + "|";
            put( p + "i_logic", reg[ b ].data(  ), 3, 4 );
            put( p + "level", & level[ b ], 1, 4 );
            const std::string q = p + "rad_flx_flux_";
            put( q + "n_int", & nh, 1, 4 );
            put( q + "n_step", & one, 1, 4 );
            put( q + "n_cell", in.n_cell_block, 3, 4 );
            put( q + "n_gh", gh, 3, 4 );
            put( q + "field", field.data(  ) + ( size_t ) b * cpb * nh, ( size_t ) cpb * nh, 4 );
        }
        const int tb = fx ? 8 : 4;
        // stable storage for the host copies and their shapes
        std::vector< std::vector< unsigned char > > keep;
        std::vector< std::vector< long long > > shapes;
        keep.reserve( 8 );
        shapes.reserve( 8 );
        auto put_dev = [ & ]( const std::string & name, const void * d, std::vector< long long > shp )
        {
            if( ! d ) return;
            size_t n = 1;
            for( long long v : shp ) n *= ( size_t ) v;
            const int unit = name == "counters" ? 8 : tb;
            keep.emplace_back( n * unit );
            api( kp_memcpy( keep.back(  ).data(  ), d, n * unit ) );
            put( "kp|" + name, keep.back(  ).data(  ), n, unit );
            shapes.push_back( std::move( shp ) );
            put( "kp|shape|" + name, shapes.back(  ).data(  ), shapes.back(  ).size(  ), 8 );
        };
        put_dev( "flux", flux_, { n_cells_ } );
        put_dev( "mu", mu_, { cfg_.n_batches, cfg_.n_mu_bins, 4 } );
        put_dev( "image", image_, { cfg_.image_n, cfg_.image_n, 4 } );
        put_dev( "image_batch", image_batch_,
                 { cfg_.n_batches, cfg_.image_batch_n, cfg_.image_batch_n, 4 } );
        put_dev( "counters", counters_, { KP_NCOUNTERS } );
        const long long done = cfg_.packet_offset + done_;
        put( "kp|packets_done", & done, 1, 8 );
        for( size_t k = 0; k < ent.size(  ); ++ k )
            ent[ k ].tag = tags[ k ].c_str(  );
        api( kp_bio_write( path.c_str(  ), ( int ) ent.size(  ), ent.data(  ) ) );
    }

    // particle::base_t::finalize: frees the device buffers (also on
    // destruction and before a new init).
    virtual void finalize(  ) noexcept
    {
        for( void * p : { flux_, ( void * ) counters_, mu_, image_, image_batch_,
                          ( void * ) table_, ( void * ) carry_, ( void * ) pool_in_,
                          ( void * ) pool_out_, ( void * ) pool_count_ } )
            if( p ) kp_free( p );
        flux_ = nullptr; counters_ = nullptr; mu_ = image_ = image_batch_ = nullptr;
        table_ = nullptr; carry_ = nullptr;
        pool_in_ = pool_out_ = nullptr; pool_count_ = nullptr;
        cap_in_ = cap_out_ = n_pool_ = 0;
        mesh_ = nullptr;
    }

    // Device results of the run so far (element type int64 in fixed-point
    // mode, float otherwise; counters uint64[KP_NCOUNTERS]).
    void * flux(  ) const { return flux_; }
    void * mu(  ) const { return mu_; }
    void * image(  ) const { return image_; }
    void * image_batch(  ) const { return image_batch_; }
    unsigned long long * counters(  ) const { return counters_; }
    // The last cycle's generated packets (device, n_par entries; null
    // without a generator).
    const kp_packet_init_t * packet_table(  ) const { return table_; }
    long long packets_per_cycle(  ) const { return n_par_; }
    long long packets_done(  ) const { return done_; }
    long long n_cells(  ) const { return n_cells_; }

private:
    kp_tallies_t tallies(  ) const
    {
        kp_tallies_t t {  };
        t.mu = mu_;
        t.image = image_;
        t.image_batch = image_batch_;
        t.counters = counters_;
        t.flux = flux_;
        t.carry = carry_;
        t.flux_n = n_cells_;
        return t;
    }

    // One keep_pool cycle: resumes the pool, emits c's packets, and keeps the
    // packets that used up step_max for the next cycle.  Reads the pool's new
    // size back (a sync, as the reference's pool_t::regulate reads n_mv).
    void integrate_pool( kp_transport_cfg_t c, const kp_tallies_t & t, stream_t s )
    {
        const long long need = std::max< long long >( n_pool_ + c.n_packets, 1 );
        if( cap_out_ < need )
        {   // the out queue holds every packet of the cycle
            if( pool_out_ ) api( kp_free( pool_out_ ) );
            pool_out_ = nullptr;
            cap_out_ = 0;
            void * p = nullptr;
            api( kp_malloc( & p, sizeof( kp_packet_state_t ) * ( size_t ) need ) );
            pool_out_ = static_cast< kp_packet_state_t * >( p );
            cap_out_ = need;
        }
        if( ! pool_count_ )
            pool_count_ = static_cast< unsigned long long * >(
                alloc( sizeof( unsigned long long ), s ) );
        api( kp_memset_async( pool_count_, 0, sizeof( unsigned long long ), s ) );
        c.max_steps = pool_max_;
        kp_resume_t r {  };
        r.in = pool_in_;
        r.n_in = n_pool_;
        r.out = pool_out_;
        r.cap_out = cap_out_;
        r.out_count = pool_count_;
        r.step_budget = std::max( par_.step_max, 1 );
        transport::forward_resume( * mesh_, c, r, t, s );
        unsigned long long n = 0;
        api( kp_stream_sync( s ) );
        api( kp_memcpy( & n, pool_count_, sizeof( n ) ) );
        if( ( long long ) n > cap_out_ )
            throw std::runtime_error( "kratos_polrad_b200: packet pool overflow" );
        std::swap( pool_in_, pool_out_ );
        std::swap( cap_in_, cap_out_ );
        n_pool_ = ( long long ) n;
    }

    static void * alloc( size_t bytes, stream_t s )
    {
        void * p = nullptr;
        api( kp_malloc( & p, bytes ) );
        const int st = kp_memset_async( p, 0, bytes, s );
        if( st != KP_OK ) { kp_free( p ); api( st ); }
        return p;
    }

    kp_particle_cfg_t          par_;
    kp_transport_cfg_t         cfg_;
    std::vector< kp_source_t > src_;
    generator_t                gen_;
    mesh_t *                   mesh_ = nullptr;
    long long                  n_cells_ = 0, n_par_ = 0, done_ = 0;
    void *                     flux_ = nullptr;
    void *                     mu_ = nullptr;
    void *                     image_ = nullptr;
    void *                     image_batch_ = nullptr;
    unsigned long long *       counters_ = nullptr;
    kp_packet_init_t *         table_ = nullptr;
    float *                    carry_ = nullptr;
    // keep_pool: the packets carried to the next cycle (in), the queue this
    // cycle suspends into (out), their capacities and the device count
    kp_packet_state_t *        pool_in_ = nullptr;
    kp_packet_state_t *        pool_out_ = nullptr;
    unsigned long long *       pool_count_ = nullptr;
    long long                  cap_in_ = 0, cap_out_ = 0, n_pool_ = 0;
    long long                  pool_max_ = 1ll << 24;
};

}   // namespace kp::particle::radiation

#endif
