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

////////////////////////////////////////////////////////////
// Spherical-polar walk: photon::sph_t (modules/particle/radiation/
// photon_sph.h:11-265) over meshgen::sph_t blocks.  Positions are (r, theta,
// phi) with a Cartesian copy; every step solves for the next r-shell,
// theta-cone and phi-plane, moves in Cartesian coordinates with the
// reference's 1.001 overshoot and converts back.  Arithmetic follows the
// reference's operation order and types (float_t, and float where it calls
// cosf, sinf, sqrtf, acosf, atan2f, copysignf), with CUDA's functions for
// those calls: results equal the reference compiled for the host except
// where the two libraries round a transcendental differently.

template< class f_t > struct sph_tab;
template<> struct sph_tab< float >
{
    static __device__ const float * rf( const mesh_view_t & m )  { return m.rf_f; }
    static __device__ const float * vol( const mesh_view_t & m ) { return m.vol_f; }
};
template<> struct sph_tab< double >
{
    static __device__ const double * rf( const mesh_view_t & m )  { return m.rf_d; }
    static __device__ const double * vol( const mesh_view_t & m ) { return m.vol_d; }
};

// geo_t of a spherical block: radial faces from the table (faces -1..nc0+1)
// when not uniform, theta and phi uniform, volume per cell.
template< class f_t >
struct sph_geo_t
{
    f_t xf0[ 3 ], dx0[ 3 ];
    const f_t * rf;              // face -1 first; null when uniform
    const f_t * vol;
    int nc0;
    unsigned * status;
    __device__ void load( const mesh_view_t & m, int b )
    {
        const f_t * g = geo_ptr< f_t >::get( m ) + geo_stride< f_t >(  ) * ( size_t ) b;
        #pragma unroll
        for( int a = 0; a < 3; ++ a ) { xf0[ a ] = g[ a ]; dx0[ a ] = g[ 3 + a ]; }
        nc0 = m.nc[ 0 ];
        rf  = dx0[ 0 ] > 0 ? nullptr : sph_tab< f_t >::rf( m ) + ( size_t ) b * ( nc0 + 3 );
        vol = sph_tab< f_t >::vol( m ) + ( size_t ) b * m.cpb;
        status = m.status;
    }
    // geo_t::x_fc (geometry.h:70-83)
    __device__ __forceinline__ f_t x_fc( int a, int i ) const
    {
        if( a == 0 && rf != nullptr )
        {
            if( i < -1 || i > nc0 + 1 )
            {   // beyond the ghost faces: report, clamp
                atomicOr( status, ST_BAD_CELL );
                i = i < -1 ? -1 : nc0 + 1;
            }
            return rf[ i + 1 ];
        }
        return rn_add( xf0[ a ], rn_mul( ( f_t ) i, dx0[ a ] ) );
    }
};

template< class f_t >
struct sph_loc_t
{
    f_t x_l[ 3 ], x_r[ 3 ];
    __device__ __forceinline__ void load( const sph_geo_t< f_t > & g, const int i[ 3 ] )
    {
        #pragma unroll
        for( int a = 0; a < 3; ++ a ) { x_l[ a ] = g.x_fc( a, i[ a ] ); x_r[ a ] = g.x_fc( a, i[ a ] + 1 ); }
    }
    __device__ __forceinline__ void fix( const sph_geo_t< f_t > & g, const int i[ 3 ],
                                         const f_t x[ 3 ] )
    {
        #pragma unroll
        for( int a = 0; a < 3; ++ a )
            if( x[ a ] > x_r[ a ] )      { x_l[ a ] = x_r[ a ]; x_r[ a ] = g.x_fc( a, i[ a ] + 1 ); }
            else if( x[ a ] < x_l[ a ] ) { x_r[ a ] = x_l[ a ]; x_l[ a ] = g.x_fc( a, i[ a ] ); }
    }
};

template< class T > __device__ __forceinline__ int sgn( T a ) { return a > 0 ? 1 : ( a < 0 ? -1 : 0 ); }

// sph_t::root: both roots of a t^2 + b t + c = 0, the stable way
template< class f_t >
__device__ __forceinline__ bool sph_root( f_t & x_1, f_t & x_2, f_t a, f_t b, f_t c )
{
    const f_t det = rn_sub( rn_mul( b, b ), rn_mul( rn_mul( ( f_t ) 4, a ), c ) );
    if( det < 0 )
    {
        x_1 = det;
        return false;
    }
    const float sq = copysignf( __fsqrt_rn( ( float ) det ), ( float ) b );
    const f_t nom = rn_add( ( f_t ) sq, b );
    const f_t x0 = rn_div( nom, rn_mul( ( f_t ) -2, a ) );
    const f_t x1 = rn_div( rn_mul( ( f_t ) -2, c ), nom );
    x_1 = x0 < x1 ? x0 : x1;
    x_2 = x0 > x1 ? x0 : x1;
    return true;
}

template< class f_t, int FLUX >
__global__ void __launch_bounds__( 128 )
k_trace_sph( const mesh_view_t m, long long n, f_t * __restrict__ xs, f_t * __restrict__ xcs,
             const f_t * __restrict__ dirs, int * __restrict__ cells,
             int * __restrict__ ibs, const f_t * __restrict__ propers,
             int * __restrict__ steps, int8_t * __restrict__ todos,
             void * __restrict__ flux, double fx_scale )
{
    const long long stride = ( long long ) gridDim.x * blockDim.x;
    for( long long p = blockIdx.x * ( long long ) blockDim.x + threadIdx.x; p < n; p += stride )
    {
        if( todos[ p ] != TO_KEEP )
            continue;
        f_t x[ 3 ], xc[ 3 ], dir[ 3 ];
        int i[ 3 ];
        #pragma unroll
        for( int a = 0; a < 3; ++ a )
        {
            x  [ a ] = xs  [ 3 * p + a ];
            xc [ a ] = xcs [ 3 * p + a ];
            dir[ a ] = dirs[ 3 * p + a ];
            i  [ a ] = cells[ 3 * p + a ];
        }
        int ib   = ibs  [ p ];
        int step = steps[ p ];
        const f_t proper = propers[ p ];
        int8_t todo = -1;
        if( ib < 0 || ib >= m.n_blocks )
        {
            atomicOr( m.status, ST_BAD_BLOCK );
            continue;
        }
        sph_geo_t< f_t > g;
        sph_loc_t< f_t > gl;
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
            const int ib_cur = ib;
            // ---- get_dl (photon_sph.h:44-175) ----
            f_t th_hat[ 3 ];
            {
                const float cos_th = cosf( ( float ) x[ 1 ] );
                th_hat[ 0 ] = ( f_t ) __fmul_rn( cos_th, cosf( ( float ) x[ 2 ] ) );
                th_hat[ 1 ] = ( f_t ) __fmul_rn( cos_th, sinf( ( float ) x[ 2 ] ) );
                th_hat[ 2 ] = ( f_t ) ( -sinf( ( float ) x[ 1 ] ) );
            }
            f_t x_dot_d = 0, dt_dl = 0;
            #pragma unroll
            for( int a = 0; a < 3; ++ a )
            {
                x_dot_d = rn_add( x_dot_d, rn_mul( xc[ a ], dir[ a ] ) );
                dt_dl   = rn_add( dt_dl, rn_mul( th_hat[ a ], dir[ a ] ) );
            }
            const f_t x2 = rn_mul( x[ 0 ], x[ 0 ] );
            const f_t df_dl = rn_sub( rn_mul( xc[ 0 ], dir[ 1 ] ), rn_mul( xc[ 1 ], dir[ 0 ] ) );
            int idx_dir[ 3 ] = { sgn( x_dot_d ), sgn( dt_dl ), sgn( df_dl ) };
            f_t x_fwd[ 3 ], x_bck[ 3 ];
            #pragma unroll
            for( int a = 0; a < 3; ++ a )
            {
                x_fwd[ a ] = idx_dir[ a ] > 0 ? gl.x_r[ a ] : gl.x_l[ a ];
                x_bck[ a ] = idx_dir[ a ] < 0 ? gl.x_r[ a ] : gl.x_l[ a ];
            }
            f_t dl[ 3 ], x_1 = 0, x_2 = 0;
            // r-direction
            {
                const f_t a_r = 1, b_r = rn_mul( ( f_t ) 2, x_dot_d );
                f_t c_r = rn_sub( x2, rn_mul( x_fwd[ 0 ], x_fwd[ 0 ] ) );
                if( ! sph_root( x_1, x_2, a_r, b_r, c_r ) )
                {   // getting out through the same surface
                    c_r = rn_sub( x2, rn_mul( x_bck[ 0 ], x_bck[ 0 ] ) );
                    sph_root( x_1, x_2, a_r, b_r, c_r );
                    dl[ 0 ] = x_2;
                    idx_dir[ 0 ] *= -1;
                }
                else
                    dl[ 0 ] = x_1 > 0 ? x_1 : x_2;
            }
            // theta-direction
            {
                const f_t z = xc[ 2 ], dz = dir[ 2 ];
                float mu2 = cosf( ( float ) x_fwd[ 1 ] );
                mu2 = __fmul_rn( mu2, mu2 );
                f_t a_m = rn_sub( rn_mul( dz, dz ), ( f_t ) mu2 );
                f_t b_m = rn_mul( ( f_t ) 2, rn_sub( rn_mul( z, dz ), rn_mul( ( f_t ) mu2, x_dot_d ) ) );
                f_t c_m = rn_sub( rn_mul( z, z ), rn_mul( ( f_t ) mu2, x2 ) );
                if( a_m != 0 )
                {
                    if( ! sph_root( x_1, x_2, a_m, b_m, c_m ) )
                    {
                        mu2 = cosf( ( float ) x_bck[ 1 ] );
                        mu2 = __fmul_rn( mu2, mu2 );
                        a_m = rn_sub( rn_mul( dz, dz ), ( f_t ) mu2 );
                        b_m = rn_mul( ( f_t ) 2, rn_sub( rn_mul( z, dz ), rn_mul( ( f_t ) mu2, x_dot_d ) ) );
                        c_m = rn_sub( rn_mul( z, z ), rn_mul( ( f_t ) mu2, x2 ) );
                        if( a_m != 0 )
                        {
                            const bool real = sph_root( x_1, x_2, a_m, b_m, c_m );
                            dl[ 1 ] = real ? x_2 : ( f_t ) -1;
                        }
                        else
                            dl[ 1 ] = rn_div( -c_m, b_m );
                        idx_dir[ 1 ] *= -1;
                    }
                    else
                        dl[ 1 ] = x_1 > 0 ? x_1 : x_2;
                }
                else
                    dl[ 1 ] = rn_div( -c_m, b_m );
            }
            // phi-direction
            {
                float sin_ph = sinf( ( float ) x_fwd[ 2 ] ), cos_ph = cosf( ( float ) x_fwd[ 2 ] );
                f_t a_f = rn_sub( rn_mul( dir[ 0 ], ( f_t ) sin_ph ), rn_mul( dir[ 1 ], ( f_t ) cos_ph ) );
                f_t b_f = rn_sub( rn_mul( xc[ 1 ], ( f_t ) cos_ph ), rn_mul( xc[ 0 ], ( f_t ) sin_ph ) );
                dl[ 2 ] = a_f != 0 ? rn_div( b_f, a_f ) : ( f_t ) -1;
                if( dl[ 2 ] < 0 )
                {
                    sin_ph = sinf( ( float ) x_bck[ 2 ] ); cos_ph = cosf( ( float ) x_bck[ 2 ] );
                    a_f = rn_sub( rn_mul( dir[ 0 ], ( f_t ) sin_ph ), rn_mul( dir[ 1 ], ( f_t ) cos_ph ) );
                    b_f = rn_sub( rn_mul( xc[ 1 ], ( f_t ) cos_ph ), rn_mul( xc[ 0 ], ( f_t ) sin_ph ) );
                    dl[ 2 ] = a_f != 0 ? rn_div( b_f, a_f ) : ( f_t ) -1;
                    idx_dir[ 2 ] *= -1;
                }
            }
            int a_proc = 0;
            f_t dl_min = ( f_t ) FLT_MAX;
            #pragma unroll
            for( int a = 0; a < 3; ++ a )
                if( dl[ a ] > 0 && dl[ a ] < dl_min ) { a_proc = a; dl_min = dl[ a ]; }
            f_t dl_p = dl[ 0 ];
            int id_p = idx_dir[ 0 ];
            #pragma unroll
            for( int a = 1; a < 3; ++ a ) if( a == a_proc ) { dl_p = dl[ a ]; id_p = idx_dir[ a ]; }

            // ---- proc_phys (photon.h:73-83) ----
            {
                const bool in = i[ 0 ] >= 0 && i[ 0 ] < m.nc[ 0 ] && i[ 1 ] >= 0 &&
                                i[ 1 ] < m.nc[ 1 ] && i[ 2 ] >= 0 && i[ 2 ] < m.nc[ 2 ];
                if( ! in )
                    atomicOr( m.status, ST_BAD_CELL );
                else
                {
                    const int l = i[ 0 ] + m.nc[ 0 ] * ( i[ 1 ] + m.nc[ 1 ] * i[ 2 ] );
                    const f_t v = rn_mul( proper, rn_div( dl_p, g.vol[ l ] ) );
                    const size_t c = ( size_t ) ib_cur * m.cpb + l;
                    if( FLUX == KP_FLUX_FLOAT )
                        atomicAdd( ( f_t * ) flux + c, v );
                    else
                        atomicAdd( ( unsigned long long * ) flux + c,
                                   ( unsigned long long ) __double2ll_rn( ( double ) v * fx_scale ) );
                }
            }
            // ---- proc_geo (photon_sph.h:224-244) ----
            {
                const f_t over = ( f_t ) 1.001f;
                #pragma unroll
                for( int a = 0; a < 3; ++ a )
                    xc[ a ] = rn_add( xc[ a ], rn_mul( rn_mul( dl_p, dir[ a ] ), over ) );
                // to_sph (photon_sph.h:190-207)
                f_t r2 = 0;
                #pragma unroll
                for( int a = 0; a < 3; ++ a ) r2 = rn_add( r2, rn_mul( xc[ a ], xc[ a ] ) );
                x[ 0 ] = ( f_t ) __fsqrt_rn( ( float ) r2 );
                x[ 1 ] = rn_div( xc[ 2 ], x[ 0 ] );
                if( x[ 1 ] > 1 )
                    x[ 1 ] = 0;
                else if( x[ 1 ] < -1 )
                    x[ 1 ] = ( f_t ) 3.141592654f;
                else if( x[ 1 ] < ( f_t ) 1e-2f )            // every mu below 0.01, as written
                    x[ 1 ] = rn_sub( ( f_t ) 1.570796f, x[ 1 ] );
                else
                    x[ 1 ] = ( f_t ) acosf( ( float ) x[ 1 ] );
                x[ 2 ] = ( f_t ) atan2f( ( float ) xc[ 1 ], ( float ) xc[ 0 ] );
                // to_sph_guard (photon_sph.h:209-222), loops bounded
                const f_t pi = ( f_t ) 3.14159265358979323846;
                const f_t two_pi = rn_mul( pi, ( f_t ) 2 );
                for( int k = 0; k < 16 && x[ 2 ] < rn_sub( gl.x_l[ 2 ], pi ); ++ k )
                    x[ 2 ] = rn_add( x[ 2 ], two_pi );
                for( int k = 0; k < 16 && x[ 2 ] > rn_add( gl.x_r[ 2 ], pi ); ++ k )
                    x[ 2 ] = rn_sub( x[ 2 ], two_pi );
                if constexpr( sizeof( f_t ) == 4 )
                    x[ 1 ] = fmaxf( x[ 1 ], 1e-3f );
                #pragma unroll
                for( int a = 0; a < 3; ++ a )
                {
                    if( a == a_proc )
                        i[ a ] += id_p;
                    else if( x[ a ] >= gl.x_r[ a ] )
                        ++ i[ a ];
                    else if( x[ a ] <= gl.x_l[ a ] )
                        -- i[ a ];
                }
            }
            // ---- proxy_base_t::shift_blk (types/proxy.h:64-121) ----
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
                    const int ap1 = a == 0 ? 2 : a - 1;
                    const int dlv = md.d_lvl[ 2 * a + side ];
                    int j0 = 0, j1 = 0;
                    if( dlv > 0 )
                    {
                        j0 = i[ ap0 ] >= m.nc[ ap0 ] / 2;
                        j1 = i[ ap1 ] >= m.nc[ ap1 ] / 2;
                    }
                    const int nid = m.nb[ 24 * ( size_t ) ib_cur + ( ( a * 2 + side ) * 2 + j0 ) * 2 + j1 ];
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
            if( ! proc_flag )
                break;
            if( ib < 0 || ib >= m.n_blocks )
            {
                atomicOr( m.status, ST_BAD_BLOCK );
                todo = TO_RM;
                break;
            }
            // sph_t::proc_step (photon_sph.h:246-264): reload, fix if wrapped
            g.load( m, ib );
            gl.load( g, i );
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
            if( wrapped )
                gl.fix( g, i, x );
        }
        if( step <= 0 )
            todo = TO_RM;
        #pragma unroll
        for( int a = 0; a < 3; ++ a )
        {
            xs   [ 3 * p + a ] = x[ a ];
            xcs  [ 3 * p + a ] = xc[ a ];
            cells[ 3 * p + a ] = i[ a ];
        }
        ibs  [ p ] = ib;
        steps[ p ] = step;
        todos[ p ] = todo;
    }
}

template< class f_t, int FLUX >
void launch_trace_sph( const mesh_view_t & m, long long n, void * x, void * xc, const void * dir,
                       int * cell, int * ib, const void * proper, int * step, int8_t * todo,
                       void * flux, double fx_scale, cudaStream_t s )
{
    int dev = 0, n_sm = 148;
    cudaGetDevice( & dev );
    cudaDeviceGetAttribute( & n_sm, cudaDevAttrMultiProcessorCount, dev );
    long long blocks = std::min< long long >( ( n + 127 ) / 128, ( long long ) n_sm * 16 );
    if( blocks < 1 ) return;
    k_trace_sph< f_t, FLUX ><<< ( unsigned ) blocks, 128, 0, s >>>(
        m, n, ( f_t * ) x, ( f_t * ) xc, ( const f_t * ) dir, cell, ib, ( const f_t * ) proper,
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

extern "C" int kp_trace_sph( kp_mesh_t * mesh, int precision, long long n, void * x,
                             void * x_car, const void * dir, int * cell, int * ib,
                             const void * proper, int * step, int8_t * todo, int flux_mode,
                             int fx_shift, void * flux, void * stream )
{
    return kp::guarded( "kp_trace_sph", [ & ]
    {
        kp::require( mesh != nullptr, "null mesh" );
        kp::require( mesh->tree->tables(  ).coord == 1, "not a spherical mesh", KP_ERR_CONFIG );
        kp::require( precision == 4 || precision == 8, "precision must be 4 or 8" );
        kp::require( flux_mode == KP_FLUX_FLOAT || flux_mode == KP_FLUX_FIXED,
                     "unknown flux mode" );
        kp::require( fx_shift >= 0 && fx_shift <= 60, "fx_shift out of range" );
        kp::require( n >= 0, "n < 0" );
        if( n == 0 ) return;
        kp::require( x && x_car && dir && cell && ib && proper && step && todo && flux,
                     "null packet array" );
        mesh->upload( false );
        const auto v = mesh->view(  );
        const double sc = std::ldexp( 1.0, fx_shift );
        auto s = ( cudaStream_t ) stream;
        if( precision == 4 )
        {
            if( flux_mode == KP_FLUX_FLOAT )
                kp::launch_trace_sph< float, KP_FLUX_FLOAT >( v, n, x, x_car, dir, cell, ib, proper, step, todo, flux, sc, s );
            else
                kp::launch_trace_sph< float, KP_FLUX_FIXED >( v, n, x, x_car, dir, cell, ib, proper, step, todo, flux, sc, s );
        }
        else
        {
            if( flux_mode == KP_FLUX_FLOAT )
                kp::launch_trace_sph< double, KP_FLUX_FLOAT >( v, n, x, x_car, dir, cell, ib, proper, step, todo, flux, sc, s );
            else
                kp::launch_trace_sph< double, KP_FLUX_FIXED >( v, n, x, x_car, dir, cell, ib, proper, step, todo, flux, sc, s );
        }
    } );
}
