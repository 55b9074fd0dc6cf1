// Internal types shared by the C-ABI translation units.
#pragma once

#include "../../include/kp_transport.h"
#include "host/block_tree.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>

namespace kp
{

////////////////////////////////////////////////////////////
// Error handling: every entry point converts exceptions to a status and
// records the message for kp_last_error() (replaces cuda_api's throw,
// device/cuda/cuda.cpp:16-26, with a C-friendly status).

struct error_t : std::runtime_error
{
    int code;
    error_t( int c, const std::string & m ) : std::runtime_error( m ), code( c ) {}
};

void set_last_error( const std::string & msg );
void clear_last_error(  );

inline void cuda_check( cudaError_t e, const char * what )
{
    if( e != cudaSuccess )
        throw error_t( KP_ERR_CUDA, std::string( what ) + ": "
                                    + cudaGetErrorString( e ) );
}
#define KP_CUDA( call ) ::kp::cuda_check( ( call ), #call )

template< class F >
int guarded( const char * fn, F && f )
{
    try
    {
        clear_last_error(  );
        f(  );
        return KP_OK;
    }
    catch( const error_t & e )
    {
        set_last_error( std::string( fn ) + ": " + e.what(  ) );
        return e.code;
    }
    catch( const std::bad_alloc & )
    {
        set_last_error( std::string( fn ) + ": host allocation failed" );
        return KP_ERR_ALLOC;
    }
    catch( const std::exception & e )
    {
        set_last_error( std::string( fn ) + ": " + e.what(  ) );
        return KP_ERR_CONFIG;
    }
}

inline void require( bool ok, const char * msg, int code = KP_ERR_ARG )
{
    if( ! ok ) throw error_t( code, msg );
}

////////////////////////////////////////////////////////////
// Device error status word bits (set by kernels, read by kp_mesh_status).

enum status_bits : unsigned
{
    ST_BAD_BLOCK   = 1u << 0,   // packet block id out of range
    ST_BAD_CELL    = 1u << 1,   // cell index out of range at a deposit
    ST_QUEUE_FULL  = 1u << 2,   // a device queue overflowed
    ST_BAD_SOURCE  = 1u << 3,   // a source lies outside the mesh
};

////////////////////////////////////////////////////////////
// Device view of a mesh: passed by value to kernels.

struct alignas( 16 ) blk_meta_t
{
    int8_t  d_lvl[ 6 ];       // level delta per face (2a+side)
    uint8_t shift[ 6 ];       // shift bits of slot [a][side][0][0]
    uint8_t phybnd;           // bit (2a+side): physical boundary
    uint8_t pad[ 3 ];
};
static_assert( sizeof( blk_meta_t ) == 16, "meta record" );

struct mesh_view_t
{
    int n_blocks;
    int nc[ 3 ];
    int cpb;                              // cells per block
    const int        * __restrict__ nb;   // [n_blocks][24]
    const blk_meta_t * __restrict__ meta; // [n_blocks]
    const double     * __restrict__ geo_d;// [n_blocks][16]: xf0[3] dx0[3] vol0 -
                                          //   inv_dx[3] - ...
    const float      * __restrict__ geo_f;// [n_blocks][8]
    const float2     * __restrict__ sigma;// [n_blocks * cpb] (sca, abs)
    // [n_blocks * cpb] extinction sca + abs (one float add, the value each
    // walk and peel-off segment needs), derived from sigma before each solve
    const float      * __restrict__ ext;
    const int        * __restrict__ lookup;// finest-level block grid
    int lookup_n[ 3 ];
    int max_level;
    unsigned periodic;                    // bit a
    double xlim_d[ 2 ][ 3 ];
    double lbox_d[ 3 ];
    float  xlim_f[ 2 ][ 3 ];
    float  lbox_f[ 3 ];
    unsigned * status;
    // spherical meshes only (null otherwise): radial faces [n_blocks][nc0+3]
    // (faces -1..nc0+1) and cell volumes [n_blocks * cpb], per float_t
    const float  * rf_f;  const double * rf_d;
    const float  * vol_f; const double * vol_d;
};

}   // namespace kp

// The opaque mesh handle of the C ABI.
struct kp_mesh
{
    std::unique_ptr< kp::block_tree_t > tree;
    int          device   = -1;
    bool         uploaded = false;
    int        * d_nb     = nullptr;
    kp::blk_meta_t * d_meta = nullptr;
    double     * d_geo_d  = nullptr;
    float      * d_geo_f  = nullptr;
    float2     * d_sigma  = nullptr;
    float      * d_ext    = nullptr;     // sca + abs per cell (refresh_ext)
    int        * d_lookup = nullptr;
    unsigned   * d_status = nullptr;
    void       * d_pq    = nullptr;  long long pq_cap = 0;        // deferred peel-off rays
    long long    pq_limit = 1ll << 27;                             // ... at most this many
    // the order k_peel marches the queue in (KP_PEEL_ORDER_*) and the
    // buffers of the sort by starting cell: per-cell counts and offsets,
    // the scan's scratch, the permutation
    int          peel_order = KP_PEEL_ORDER_AUTO;
    unsigned   * d_sort_cnt = nullptr, * d_sort_off = nullptr;
    int        * d_sort_perm = nullptr;
    void       * d_sort_tmp = nullptr;
    size_t       sort_cells = 0, sort_perm = 0, sort_tmp_bytes = 0;
    void       * d_adj   = nullptr;  size_t adj_bytes = 0;      // deferred adjoint
    // the taped forward solve whose rays the queue and d_adj hold (0: none)
    long long    tape_id = 0, tape_serial = 0;
    long long    tape_n  = 0;                                      // its packets
    bool         tape_sorted = false;   // its march read d_sort_perm (the tape's order)
    kp_transport_cfg_t tape_cfg {  };
    kp_source_t  tape_src[ KP_MAX_SOURCES ] {  };
    float      * d_rf_f  = nullptr;  double * d_rf_d  = nullptr;   // spherical tables
    float      * d_vol_f = nullptr;  double * d_vol_d = nullptr;

    unsigned long long * d_work = nullptr;   // scratch: packet counters

    kp::mesh_view_t view(  ) const;
    unsigned long long * workspace(  ) { upload( false ); return d_work; }
    // Copies the tables to the current device; with_sigma also allocates the
    // (zeroed) coefficient array, which a decomposed rank does not hold.
    void upload( bool with_sigma = true );
    // Recomputes d_ext from d_sigma on stream s: every solve does this first,
    // since callers may write the coefficients through kp_mesh_sigma_ptr.
    void refresh_ext( cudaStream_t s );
    void release(  );
};

namespace kp
{
// ext[i] = sigma[i].x + sigma[i].y (IEEE float add) for n cells, on stream s.
void extinction( const float2 * sigma, float * ext, long long n, cudaStream_t s );
}
