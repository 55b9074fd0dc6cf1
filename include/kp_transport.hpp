// kratos_polrad_b200 — header-only C++ layer over the C ABI (kp_transport.h).
//
// For a reference build that keeps its C++ conventions: every failed call
// throws std::runtime_error with the library's message, as the reference's
// cuda_api wrapper does (src/device/cuda/cuda.cpp:16-26), and handles free
// their device memory in their destructors, as the reference's owners do in
// finalize (modules/particle/types/particle_pool.h:55-65).
//
//   device_t   device::base_t's typed allocation, copy, stream, event and
//              host-callback members (src/device/device.h:37-186)
//   mesh_t     block tree + neighbour tables + per-cell coefficients
//              (meshgen::base_t, proxy_base_t::setup, rad_t::mfp_i)
//   transport  one solve: generate + integrate + the scattering hooks
//              (modules/particle/driver.h:59-79)
//   batch_t    many scenes in one persistent launch / CUDA graph
#ifndef KP_TRANSPORT_HPP
#define KP_TRANSPORT_HPP

#include "kp_transport.h"

#include <array>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace kp
{

// Throws std::runtime_error(kp_last_error()) on a non-zero status.
inline void api( int status )
{
    if( status != KP_OK )
        throw std::runtime_error( std::string( "kratos_polrad_b200: " ) + kp_last_error(  ) );
}

using stream_t = void *;
using event_t  = void *;

// Typed device layer with device::base_t's member names.  Streams come from
// a round-robin pool, as yield_stream hands them out (cuda.cpp:164-176).
class device_t
{
public:
    explicit device_t( int idx_device = 0, int max_streams = 16 )
        : max_streams_( max_streams ) { api( kp_device_init( idx_device ) ); }
    ~device_t(  ) { delete_all_streams(  ); }
    device_t( const device_t & ) = delete;
    device_t & operator=( const device_t & ) = delete;

    template< typename T > T * malloc_device( size_t n = 1 ) const
    {
        void * p = nullptr;
        api( kp_malloc( & p, n * sizeof( T ) ) );
        return static_cast< T * >( p );
    }
    template< typename T > T * malloc_host( size_t n = 1 ) const
    {
        void * p = nullptr;
        api( kp_malloc_host( & p, n * sizeof( T ) ) );
        return static_cast< T * >( p );
    }
    template< typename T > T * malloc( size_t n = 1, bool host = true ) const
    {
        return host ? malloc_host< T >( n ) : malloc_device< T >( n );
    }
    template< typename T > void free_device( T * & p ) const { api( kp_free( p ) ); p = nullptr; }
    template< typename T > void free_host( T * & p ) const { api( kp_free_host( p ) ); p = nullptr; }
    template< typename T > void free( T * & p, bool host = true ) const
    {
        host ? free_host( p ) : free_device( p );
    }
    template< typename T > void cp( T * tgt, const T * src, size_t n = 1 ) const
    {
        api( kp_memcpy( tgt, src, n * sizeof( T ) ) );
    }
    template< typename T > void cp_a( T * tgt, const T * src, size_t n = 1,
                                      stream_t s = nullptr ) const
    {
        api( kp_memcpy_async( tgt, src, n * sizeof( T ), s ) );
    }
    template< typename T > void mset( T * p, int value, size_t n = 1, stream_t s = nullptr ) const
    {
        api( kp_memset_async( p, value, n * sizeof( T ), s ) );
    }

    stream_t yield_stream(  )
    {
        if( ( int ) streams_.size(  ) < max_streams_ )
        {
            stream_t s = nullptr;
            api( kp_stream_create( & s ) );
            streams_.push_back( s );
            return s;
        }
        stream_t s = streams_[ next_ ];
        next_ = ( next_ + 1 ) % streams_.size(  );
        return s;
    }
    void sync_stream( stream_t s ) const { api( kp_stream_sync( s ) ); }
    void sync_all_streams(  ) const
    {
        for( stream_t s : streams_ ) sync_stream( s );
        sync_stream( nullptr );
    }
    void delete_all_streams(  ) noexcept
    {
        for( stream_t s : streams_ ) kp_stream_destroy( s );
        streams_.clear(  );
        next_ = 0;
    }

    event_t event_create(  ) const { event_t e = nullptr; api( kp_event_create( & e ) ); return e; }
    void event_destroy( event_t e ) const { api( kp_event_destroy( e ) ); }
    void event_record( event_t e, stream_t s ) const { api( kp_event_record( e, s ) ); }
    void event_wait( stream_t s, event_t e ) const { api( kp_event_wait( s, e ) ); }
    void event_sync( event_t e ) const { api( kp_event_sync( e ) ); }
    float elapsed_ms( event_t a, event_t b ) const
    {
        float ms = 0.f;
        api( kp_event_elapsed( & ms, a, b ) );
        return ms;
    }

    // Host function enqueued on a stream (f_launch_host / launch_host).  Each
    // callable owns its own heap slot, so concurrent threads may enqueue.
    void f_launch_host( stream_t s, void ( * fn )( void * ), void * arg ) const
    {
        api( kp_launch_host( s, fn, arg ) );
    }
    void launch_host( stream_t s, std::function< void(  ) > && fn ) const
    {
        auto * f = new std::function< void(  ) >( std::move( fn ) );
        const int st = kp_launch_host( s, & device_t::run_and_delete, f );
        if( st != KP_OK ) { delete f; api( st ); }
    }

private:
    static void run_and_delete( void * p )
    {
        std::unique_ptr< std::function< void(  ) > > f( static_cast< std::function< void(  ) > * >( p ) );
        ( * f )(  );
    }
    int max_streams_;
    std::vector< stream_t > streams_;
    size_t next_ = 0;
};

// Block-structured mesh with its neighbour tables and coefficients.
class mesh_t
{
public:
    explicit mesh_t( const std::string & ini_path ) { api( kp_mesh_create_ini( ini_path.c_str(  ), & m_ ) ); }
    explicit mesh_t( const kp_mesh_desc_t & d ) { api( kp_mesh_create( & d, & m_ ) ); }
    // Spherical-polar mesh (r, theta, phi) of meshgen::sph_t.
    static mesh_t spherical( const kp_mesh_desc_t & d, double r_ratio )
    {
        kp_mesh_t * m = nullptr;
        api( kp_mesh_create_sph( & d, r_ratio, & m ) );
        return mesh_t( m );
    }
    static mesh_t spherical( const std::string & ini_path )
    {
        kp_mesh_t * m = nullptr;
        api( kp_mesh_create_sph_ini( ini_path.c_str(  ), & m ) );
        return mesh_t( m );
    }
    ~mesh_t(  ) { if( m_ ) kp_mesh_destroy( m_ ); }
    mesh_t( const mesh_t & ) = delete;
    mesh_t & operator=( const mesh_t & ) = delete;
    mesh_t( mesh_t && o ) noexcept : m_( std::exchange( o.m_, nullptr ) ) {  }

    kp_mesh_t * get(  ) const { return m_; }
    kp_mesh_info_t info(  ) const { kp_mesh_info_t i {}; api( kp_mesh_info( m_, & i ) ); return i; }
    // (level, logical index) of every block id
    void blocks( std::vector< int > & level, std::vector< std::array< int, 3 > > & reg ) const
    {
        const int n = info(  ).n_blocks;
        level.resize( n );
        reg.resize( n );
        api( kp_mesh_blocks( m_, level.data(  ), reg.data(  )->data(  ) ) );
    }
    // block id and cell index of host points; ib = -1 outside the domain
    void locate( const std::vector< std::array< double, 3 > > & x, std::vector< int > & ib,
                 std::vector< std::array< int, 3 > > & cell ) const
    {
        ib.resize( x.size(  ) );
        cell.resize( x.size(  ) );
        api( kp_mesh_locate( m_, ( long long ) x.size(  ), x.data(  )->data(  ), ib.data(  ),
                             cell.data(  )->data(  ) ) );
    }
    void upload(  ) { api( kp_mesh_upload( m_ ) ); }
    // Runtime refinement: host flags per block (+1 refine, -1 coarsen a whole
    // family, 0 keep) -> a new mesh with the 2:1 balance restored.
    mesh_t adapt( const std::vector< int > & flags ) const
    {
        kp_mesh_t * out = nullptr;
        api( kp_mesh_adapt( m_, flags.data(  ), & out ) );
        return mesh_t( out );
    }
    // Device flags from the coefficients (optical depth across a cell).
    void flag_tau( float tau_refine, float tau_coarsen, int * d_flags, stream_t s = nullptr )
    {
        api( kp_mesh_flag_tau( m_, tau_refine, tau_coarsen, d_flags, s ) );
    }
    // Per-cell device field (n_comp floats per cell) of this mesh onto `to`.
    void remap_to( mesh_t & to, int n_comp, const float * src, float * dst, stream_t s = nullptr )
    {
        api( kp_mesh_remap( m_, to.m_, n_comp, src, dst, s ) );
    }
    // (sigma_sca, sigma_abs) per cell, block-id order, x fastest
    void set_sigma( const float * src, long long n_values, bool on_device = false,
                    stream_t s = nullptr )
    {
        api( kp_mesh_set_sigma( m_, src, n_values, on_device ? 1 : 0, s ) );
    }
    // Upper bound on the peel-off queue in rays (64 B each); larger solves
    // run in chunks of limit / 12 packets.
    void peel_queue_limit( long long max_rays ) { api( kp_mesh_peel_queue_limit( m_, max_rays ) ); }
    void peel_order( int order ) { api( kp_mesh_peel_order( m_, order ) ); }
    // Device error bits of the last kernels (0: none); throws if any is set
    // when `raise` is true, as the reference's debug flag aborts a run.
    unsigned status( stream_t s = nullptr, bool raise = true )
    {
        unsigned f = 0;
        api( kp_mesh_status( m_, s, & f ) );
        if( f && raise )
            throw std::runtime_error( "kratos_polrad_b200: device status " + std::to_string( f ) );
        return f;
    }

private:
    explicit mesh_t( kp_mesh_t * m ) : m_( m ) {  }
    kp_mesh_t * m_ = nullptr;
};

// One forward solve, its path-replay adjoint and the no-allocation variant.
struct transport
{
    static void forward( mesh_t & m, const kp_transport_cfg_t & c, const kp_tallies_t & t,
                         stream_t s = nullptr )
    {
        api( kp_transport_forward( m.get(  ), & c, & t, s ) );
    }
    // Profiling: later forward solves of this thread record `event` (a
    // cudaEvent_t) between the walk and the peel-off march (nullptr: off).
    static void split_event( void * event ) { api( kp_transport_split_event( event ) ); }
    static void forward_noalloc( mesh_t & m, const kp_transport_cfg_t & c,
                                 const kp_tallies_t & t, stream_t s = nullptr )
    {
        api( kp_transport_forward_noalloc( m.get(  ), & c, & t, s ) );
    }
    static void adjoint( mesh_t & m, const kp_transport_cfg_t & c, const float * adj_image,
                         int grad_fx_shift, void * grad_len, void * grad_int,
                         unsigned long long * counters = nullptr, stream_t s = nullptr )
    {
        api( kp_transport_adjoint( m.get(  ), & c, adj_image, grad_fx_shift, grad_len, grad_int,
                                   counters, s ) );
    }
    // Forward solve that keeps its peel-off rays for adjoint_tape; returns
    // the tape id (0: too many packets to tape, an untaped solve ran).
    static long long forward_tape( mesh_t & m, const kp_transport_cfg_t & c,
                                   const kp_tallies_t & t, stream_t s = nullptr )
    {
        long long id = 0;
        api( kp_transport_forward_tape( m.get(  ), & c, & t, s, & id ) );
        return id;
    }
    // adjoint() of the taped solve `tape_id`, from its tape.
    static void adjoint_tape( mesh_t & m, long long tape_id, const kp_transport_cfg_t & c,
                              const float * adj_image, int grad_fx_shift, void * grad_len,
                              void * grad_int, unsigned long long * counters = nullptr,
                              stream_t s = nullptr )
    {
        api( kp_transport_adjoint_tape( m.get(  ), tape_id, & c, adj_image, grad_fx_shift,
                                        grad_len, grad_int, counters, s ) );
    }
    static void trace( mesh_t & m, int precision, long long n, void * x, const void * dir,
                       int * cell, int * ib, const void * proper, int * step, int8_t * todo,
                       int flux_mode, int fx_shift, void * flux, stream_t s = nullptr )
    {
        api( kp_trace( m.get(  ), precision, n, x, dir, cell, ib, proper, step, todo, flux_mode,
                       fx_shift, flux, s ) );
    }
    static void trace_sph( mesh_t & m, int precision, long long n, void * x, void * x_car,
                           const void * dir, int * cell, int * ib, const void * proper,
                           int * step, int8_t * todo, int flux_mode, int fx_shift, void * flux,
                           stream_t s = nullptr )
    {
        api( kp_trace_sph( m.get(  ), precision, n, x, x_car, dir, cell, ib, proper, step, todo,
                           flux_mode, fx_shift, flux, s ) );
    }
    // A call with a step budget (see kp_resume_t): resumes r.in, emits c's
    // packets, suspends into r.out the packets that use up the budget.
    static void forward_resume( mesh_t & m, const kp_transport_cfg_t & c, const kp_resume_t & r,
                                const kp_tallies_t & t, stream_t s = nullptr )
    {
        api( kp_transport_forward_resume( m.get(  ), & c, & r, & t, s ) );
    }
    // One round of a decomposed solve on this rank (see kp_dd_round_t).
    static void forward_dd( mesh_t & m, const kp_transport_cfg_t & c, const kp_dd_round_t & r,
                            const kp_tallies_t & t, stream_t s = nullptr )
    {
        api( kp_transport_forward_dd( m.get(  ), & c, & r, & t, s ) );
    }
};

// Many scenes in one persistent launch (meshes must outlive the batch).
class batch_t
{
public:
    explicit batch_t( const std::vector< kp_scene_t > & scenes )
    {
        api( kp_batch_create( ( int ) scenes.size(  ), scenes.data(  ), & b_ ) );
    }
    ~batch_t(  ) { if( b_ ) kp_batch_destroy( b_ ); }
    batch_t( const batch_t & ) = delete;
    batch_t & operator=( const batch_t & ) = delete;

    void refresh_sigma( stream_t s = nullptr ) { api( kp_batch_refresh_sigma( b_, s ) ); }
    void forward( const kp_transport_cfg_t & c, void * mu, unsigned long long * counters = nullptr,
                  stream_t s = nullptr )
    {
        api( kp_batch_forward( b_, & c, mu, counters, s ) );
    }
    void graph_launch( const kp_transport_cfg_t & c, void * mu,
                       unsigned long long * counters = nullptr,
                       stream_t s = nullptr )
    {
        api( kp_batch_graph_launch( b_, & c, mu, counters, s ) );
    }
    kp_tune_result_t autotune( const kp_transport_cfg_t & c, double fraction, void * scratch_mu,
                               stream_t s = nullptr )
    {
        kp_tune_result_t r {};
        api( kp_batch_autotune( b_, & c, fraction, scratch_mu, s, & r ) );
        return r;
    }
    unsigned status( stream_t s = nullptr )
    {
        unsigned f = 0;
        api( kp_batch_status( b_, s, & f ) );
        return f;
    }

private:
    kp_batch_t * b_ = nullptr;
};

}   // namespace kp

#endif
