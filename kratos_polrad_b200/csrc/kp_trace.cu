// Geometric walk with the path-length flux estimator, reference semantics.
//
// One thread per packet walks cell by cell until its step budget runs out or
// it leaves the domain, exactly as photon::cart_t::proc does
// (modules/particle/radiation/photon.h:104-125) when integrate::ker_itg runs
// it over the pool (evolve/integrator.h:80-106).  Every floating-point
// operation is an explicit round-to-nearest intrinsic in the reference's
// order, so that results equal the reference compiled for the host with
// contraction off, bit for bit, in FP32 (PRECISION=1) and FP64
// (PRECISION=2).  Packet state is structure-of-arrays (coalesced loads and
// stores) instead of the reference's 56-byte AoS pool records.
#include "kp_common.cuh"

#include <cfloat>

namespace kp
{
namespace
{

constexpr int8_t TO_KEEP = -2;      // particle::todo_t, types/particle_base.h:12
constexpr int8_t TO_RM   = -3;

// Round-to-nearest arithmetic without contraction, per float type.
__device__ __forceinline__ float  rn_add( float a, float b )   { return __fadd_rn( a, b ); }
__device__ __forceinline__ float  rn_sub( float a, float b )   { return __fsub_rn( a, b ); }
__device__ __forceinline__ float  rn_mul( float a, float b )   { return __fmul_rn( a, b ); }
__device__ __forceinline__ float  rn_div( float a, float b )   { return __fdiv_rn( a, b ); }
__device__ __forceinline__ double rn_add( double a, double b ) { return __dadd_rn( a, b ); }
__device__ __forceinline__ double rn_sub( double a, double b ) { return __dsub_rn( a, b ); }
__device__ __forceinline__ double rn_mul( double a, double b ) { return __dmul_rn( a, b ); }
__device__ __forceinline__ double rn_div( double a, double b ) { return __ddiv_rn( a, b ); }

template< class f_t > struct geo_ptr;
template<> struct geo_ptr< float >
{ static __device__ const float * get( const mesh_view_t & m ) { return m.geo_f; } };
template<> struct geo_ptr< double >
{ static __device__ const double * get( const mesh_view_t & m ) { return m.geo_d; } };

template< class f_t > __device__ __forceinline__ int geo_stride(  );
template<> __device__ __forceinline__ int geo_stride< float  >(  ) { return 8; }
template<> __device__ __forceinline__ int geo_stride< double >(  ) { return 16; }
template< class f_t > __device__ __forceinline__ f_t xlim( const mesh_view_t & m, int l, int a );
template<> __device__ __forceinline__ float  xlim< float  >( const mesh_view_t & m, int l, int a ) { return m.xlim_f[ l ][ a ]; }
template<> __device__ __forceinline__ double xlim< double >( const mesh_view_t & m, int l, int a ) { return m.xlim_d[ l ][ a ]; }
template< class f_t > __device__ __forceinline__ f_t lbox( const mesh_view_t & m, int a );
template<> __device__ __forceinline__ float  lbox< float  >( const mesh_view_t & m, int a ) { return m.lbox_f[ a ]; }
template<> __device__ __forceinline__ double lbox< double >( const mesh_view_t & m, int a ) { return m.lbox_d[ a ]; }

// Block geometry (geo_t with uniform spacing, geometry.h:199-256).
template< class f_t >
struct blk_geo_t
{
    f_t xf0[ 3 ], dx0[ 3 ], vol0;
    __device__ void load( const mesh_view_t & m, int b )
    {
        const f_t * g = geo_ptr< f_t >::get( m ) + geo_stride< f_t >(  ) * ( size_t ) b;
        #pragma unroll
        for( int a = 0; a < 3; ++ a ) { xf0[ a ] = g[ a ]; dx0[ a ] = g[ 3 + a ]; }
        vol0 = g[ 6 ];
    }
    // geo_t::x_fc for uniform blocks (geometry.h:206-221)
    __device__ __forceinline__ f_t x_fc( int a, int i ) const
    {
        return rn_add( xf0[ a ], rn_mul( ( f_t ) i, dx0[ a ] ) );
    }
};

// particle::geo_loc_t (types/particle_base.h:86-126), including fix()'s
// use of the unchanged cell index when it re-snaps.
template< class f_t >
struct geo_loc_t
{
    f_t x_l[ 3 ], x_r[ 3 ];
    __device__ __forceinline__ void load( const blk_geo_t< f_t > & g, const int i[ 3 ] )
    {
        #pragma unroll
        for( int a = 0; a < 3; ++ a )
        {
            x_l[ a ] = g.x_fc( a, i[ a ] );
            x_r[ a ] = g.x_fc( a, i[ a ] + 1 );
        }
    }
    __device__ __forceinline__ void shift( const blk_geo_t< f_t > & g, const int i[ 3 ],
                                           int ax, bool rhs )
    {
        #pragma unroll
        for( int a = 0; a < 3; ++ a )   // static indexing keeps x_l/x_r in registers
            if( a == ax )
            {
                if( rhs ) { x_l[ a ] = x_r[ a ]; x_r[ a ] = g.x_fc( a, i[ a ] + 1 ); }
                else      { x_r[ a ] = x_l[ a ]; x_l[ a ] = g.x_fc( a, i[ a ] ); }
            }
    }
    __device__ __forceinline__ void fix( const blk_geo_t< f_t > & g, const int i[ 3 ],
                                         const f_t x[ 3 ] )
    {
        #pragma unroll
        for( int a = 0; a < 3; ++ a )
            if( x[ a ] > x_r[ a ] )      shift( g, i, a, true );
            else if( x[ a ] < x_l[ a ] ) shift( g, i, a, false );
    }
};

template< class f_t, int FLUX >
__global__ void __launch_bounds__( 128 )
k_trace_ref( const mesh_view_t m, long long n, f_t * __restrict__ xs,
             const f_t * __restrict__ dirs, int * __restrict__ cells,
             int * __restrict__ ibs, const f_t * __restrict__ propers,
             int * __restrict__ steps, int8_t * __restrict__ todos,
             void * __restrict__ flux, double fx_scale )
{
    const long long stride = ( long long ) gridDim.x * blockDim.x;
    for( long long p = blockIdx.x * ( long long ) blockDim.x + threadIdx.x;
         p < n; p += stride )
    {
        // integrate::base_t::operator() only walks to_keep packets
        // (integrator.h:90-92).
        if( todos[ p ] != TO_KEEP )
            continue;
        f_t x[ 3 ], dir[ 3 ];
        int i[ 3 ];
        #pragma unroll
        for( int a = 0; a < 3; ++ a )
        {
            x  [ a ] = xs  [ 3 * p + a ];
            dir[ a ] = dirs[ 3 * p + a ];
            i  [ a ] = cells[ 3 * p + a ];
        }
        int ib   = ibs  [ p ];
        int step = steps[ p ];
        const f_t proper = propers[ p ];
        int8_t todo = -1;                       // dest.i_rank = -1 (photon.h:108)

        if( ib < 0 || ib >= m.n_blocks )
        {
            atomicOr( m.status, ST_BAD_BLOCK );
            continue;
        }

        blk_geo_t< f_t > g;
        geo_loc_t< f_t > gl;
        int ib_old = -1;
        for( ; step > 0; -- step )
        {
            if( ib != ib_old && ib >= 0 )
            {   // photon.h:113-118
                g.load( m, ib );
                gl.load( g, i );
                gl.fix( g, i, x );
                ib_old = ib;
            }
            // proc_step (photon.h:85-102) with prx = bmap[ib] bound here.
            const int ib_cur = ib;
            // get_dl (photon.h:20-44)
            f_t dl[ 3 ];
            #pragma unroll
            for( int a = 0; a < 3; ++ a )
            {
                if( dir[ a ] == 0 ) { dl[ a ] = -1; continue; }
                const f_t x_f = dir[ a ] > 0 ? gl.x_r[ a ] : gl.x_l[ a ];
                dl[ a ] = rn_div( rn_sub( x_f, x[ a ] ), dir[ a ] );
            }
            int a_proc = 0;
            f_t dl_min = ( f_t ) FLT_MAX;
            #pragma unroll
            for( int a = 0; a < 3; ++ a )
                if( dl[ a ] >= 0 && dl[ a ] <= dl_min ) { a_proc = a; dl_min = dl[ a ]; }
            f_t dl_p = dl[ 0 ];
            #pragma unroll
            for( int a = 1; a < 3; ++ a ) if( a == a_proc ) dl_p = dl[ a ];

            // proc_phys (photon.h:73-83): flux += proper * dl / volume
            {
                const f_t dsi = rn_div( dl_p, g.vol0 );
                const f_t v   = rn_mul( proper, dsi );
                const bool in = i[ 0 ] >= 0 && i[ 0 ] < m.nc[ 0 ] &&
                                i[ 1 ] >= 0 && i[ 1 ] < m.nc[ 1 ] &&
                                i[ 2 ] >= 0 && i[ 2 ] < m.nc[ 2 ];
                if( ! in )
                    atomicOr( m.status, ST_BAD_CELL );
                else
                {
                    const size_t c = ( size_t ) ib_cur * m.cpb + i[ 0 ] +
                                     m.nc[ 0 ] * ( i[ 1 ] + m.nc[ 1 ] * i[ 2 ] );
                    if( FLUX == KP_FLUX_FLOAT )
                        atomicAdd( ( f_t * ) flux + c, v );
                    else
                        atomicAdd( ( unsigned long long * ) flux + c,
                                   ( unsigned long long ) __double2ll_rn(
                                       ( double ) v * fx_scale ) );
                }
            }
            // proc_geo (photon.h:54-71)
            #pragma unroll
            for( int a = 0; a < 3; ++ a )
            {
                if( a == a_proc )
                {
                    const bool rhs = dir[ a ] > 0;
                    x[ a ] = rhs ? gl.x_r[ a ] : gl.x_l[ a ];
                    i[ a ] += rhs ? 1 : -1;
                    gl.shift( g, i, a, rhs );
                }
                else
                    x[ a ] = rn_add( x[ a ], rn_mul( dl_p, dir[ a ] ) );
            }
            // proxy_base_t::shift_blk (types/proxy.h:64-121) on block ib_cur
            todo = TO_KEEP;
            {
                const blk_meta_t md = m.meta[ ib_cur ];
                #pragma unroll
                for( int a = 0; a < 3; ++ a )
                {
                    if( i[ a ] >= 0 && i[ a ] < m.nc[ a ] )
                        continue;
                    const int side = i[ a ] > 0;
                    if( ( md.phybnd >> ( 2 * a + side ) ) & 1 )
                    {
                        todo = TO_RM;
                        break;
                    }
                    const int ap0 = a == 2 ? 0 : a + 1;
                    const int ap1 = a == 0 ? 2 : a - 1;   // (a + 2) % 3
                    const int dlv = md.d_lvl[ 2 * a + side ];
                    int j0 = 0, j1 = 0;
                    if( dlv > 0 )
                    {
                        j0 = i[ ap0 ] >= m.nc[ ap0 ] / 2;
                        j1 = i[ ap1 ] >= m.nc[ ap1 ] / 2;
                    }
                    const int nid = m.nb[ 24 * ( size_t ) ib_cur +
                                          ( ( a * 2 + side ) * 2 + j0 ) * 2 + j1 ];
                    ib = nid;
                    if( nid < 0 )
                    {
                        todo = TO_RM;
                        break;
                    }
                    i[ a ] = i[ a ] > 0 ? 0 : m.nc[ a ] - 1;
                    const int sh = md.shift[ 2 * a + side ];
                    if( dlv < 0 )
                    {
                        i[ ap0 ] = i[ ap0 ] / 2 + ( sh & 1 ) * m.nc[ ap0 ] / 2;
                        i[ ap1 ] = i[ ap1 ] / 2 + ( ( sh >> 1 ) & 1 ) * m.nc[ ap1 ] / 2;
                    }
                    else if( dlv > 0 )
                    {
                        const int h0 = m.nc[ ap0 ] / 2, h1 = m.nc[ ap1 ] / 2;
                        i[ ap0 ] = ( i[ ap0 ] < h0 ? i[ ap0 ] : i[ ap0 ] - h0 ) * 2;
                        i[ ap1 ] = ( i[ ap1 ] < h1 ? i[ ap1 ] : i[ ap1 ] - h1 ) * 2;
                    }
                    break;
                }
            }
            const bool proc_flag = todo != TO_RM;
            // par_base_t::regulate (particle_base.h:37-56), always evaluated
            bool wrapped = false;
            #pragma unroll
            for( int a = 0; a < 3; ++ a )
                if( ( m.periodic >> a ) & 1 )
                {
                    if( x[ a ] < xlim< f_t >( m, 0, a ) )
                    {
                        x[ a ] = rn_add( x[ a ], lbox< f_t >( m, a ) );
                        wrapped = true;
                    }
                    else if( x[ a ] >= xlim< f_t >( m, 1, a ) )
                    {
                        x[ a ] = rn_sub( x[ a ], lbox< f_t >( m, a ) );
                        wrapped = true;
                    }
                }
            if( proc_flag && wrapped )
            {
                if( ib < 0 || ib >= m.n_blocks )
                {
                    atomicOr( m.status, ST_BAD_BLOCK );
                    todo = TO_RM;
                    break;
                }
                g.load( m, ib );
                gl.load( g, i );
                gl.fix( g, i, x );
                ib_old = ib;   // geo_loc now describes block ib
            }
            if( ! proc_flag )
                break;
            if( ib < 0 || ib >= m.n_blocks )
            {
                atomicOr( m.status, ST_BAD_BLOCK );
                todo = TO_RM;
                break;
            }
        }
        if( step <= 0 )
            todo = TO_RM;

        #pragma unroll
        for( int a = 0; a < 3; ++ a )
        {
            xs   [ 3 * p + a ] = x[ a ];
            cells[ 3 * p + a ] = i[ a ];
        }
        ibs  [ p ] = ib;
        steps[ p ] = step;
        todos[ p ] = todo;
    }
}

template< class f_t, int FLUX >
void launch_trace( const mesh_view_t & m, long long n, void * x, const void * dir,
                   int * cell, int * ib, const void * proper, int * step,
                   int8_t * todo, void * flux, double fx_scale, cudaStream_t s )
{
    int dev = 0, n_sm = 148;
    cudaGetDevice( & dev );
    cudaDeviceGetAttribute( & n_sm, cudaDevAttrMultiProcessorCount, dev );
    const int threads = 128;
    long long blocks = ( n + threads - 1 ) / threads;
    blocks = std::min< long long >( blocks, ( long long ) n_sm * 16 );
    if( blocks < 1 ) return;
    k_trace_ref< f_t, FLUX ><<< ( unsigned ) blocks, threads, 0, s >>>(
        m, n, ( f_t * ) x, ( const f_t * ) dir, cell, ib, ( const f_t * ) proper,
        step, todo, flux, fx_scale );
    KP_CUDA( cudaGetLastError(  ) );
}

}   // namespace
}   // namespace kp

extern "C" int kp_trace( kp_mesh_t * mesh, int precision, long long n,
                         void * x, const void * dir, int * cell, int * ib,
                         const void * proper, int * step, int8_t * todo,
                         int flux_mode, int fx_shift, void * flux, void * stream )
{
    return kp::guarded( "kp_trace", [ & ]
    {
        kp::require( mesh != nullptr, "null mesh" );
        kp::require( precision == 4 || precision == 8, "precision must be 4 or 8" );
        kp::require( flux_mode == KP_FLUX_FLOAT || flux_mode == KP_FLUX_FIXED,
                     "unknown flux mode" );
        kp::require( fx_shift >= 0 && fx_shift <= 60, "fx_shift out of range" );
        kp::require( n >= 0, "n < 0" );
        if( n == 0 ) return;
        kp::require( x && dir && cell && ib && proper && step && todo && flux,
                     "null packet array" );
        mesh->upload(  );
        const auto v = mesh->view(  );
        const double sc = std::ldexp( 1.0, fx_shift );
        auto s = ( cudaStream_t ) stream;
        if( precision == 4 )
        {
            if( flux_mode == KP_FLUX_FLOAT )
                kp::launch_trace< float, KP_FLUX_FLOAT >( v, n, x, dir, cell, ib, proper, step, todo, flux, sc, s );
            else
                kp::launch_trace< float, KP_FLUX_FIXED >( v, n, x, dir, cell, ib, proper, step, todo, flux, sc, s );
        }
        else
        {
            if( flux_mode == KP_FLUX_FLOAT )
                kp::launch_trace< double, KP_FLUX_FLOAT >( v, n, x, dir, cell, ib, proper, step, todo, flux, sc, s );
            else
                kp::launch_trace< double, KP_FLUX_FIXED >( v, n, x, dir, cell, ib, proper, step, todo, flux, sc, s );
        }
    } );
}
