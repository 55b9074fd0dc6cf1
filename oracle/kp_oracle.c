/* Oracle: plain-C restatement of the transport path (test infrastructure;
 * see kp_oracle.h).  Compiled with -ffp-contract=off so that every float
 * operation rounds once, as the reference does on the host. */
#include "kp_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

enum { TO_KEEP = -2, TO_RM = -3 };   /* particle::todo_t, particle_base.h:12 */

/* One walk per float type: F is the float_t, S the suffix. */
#define KPO_DEFINE_WALK( F, S )                                                  \
static F x_fc_##S( const kpo_mesh_t * m, int b, int a, int i )                   \
{   /* geo_t::x_fc, uniform spacing (geometry.h:206-221) */                      \
    return ( F ) m->xf0[ 3 * b + a ] + ( F ) i * ( F ) m->dx0[ 3 * b + a ];      \
}                                                                                \
static void gl_load_##S( const kpo_mesh_t * m, int b, const int * i,             \
                         F * xl, F * xr )                                        \
{   /* geo_loc_t::load (particle_base.h:91-100) */                               \
    for( int a = 0; a < 3; ++ a )                                                \
    {                                                                            \
        xl[ a ] = x_fc_##S( m, b, a, i[ a ] );                                   \
        xr[ a ] = x_fc_##S( m, b, a, i[ a ] + 1 );                               \
    }                                                                            \
}                                                                                \
static void gl_shift_##S( const kpo_mesh_t * m, int b, const int * i,            \
                          F * xl, F * xr, int ax, int rhs )                      \
{   /* geo_loc_t::shift (particle_base.h:101-116) */                             \
    if( rhs ) { xl[ ax ] = xr[ ax ]; xr[ ax ] = x_fc_##S( m, b, ax, i[ ax ] + 1 ); } \
    else      { xr[ ax ] = xl[ ax ]; xl[ ax ] = x_fc_##S( m, b, ax, i[ ax ] ); }     \
}                                                                                \
static int gl_fix_##S( const kpo_mesh_t * m, int b, const int * i,               \
                       const F * x, F * xl, F * xr )                             \
{   /* geo_loc_t::fix (particle_base.h:117-126): the cell index is left as is;   \
       returns the number of axes it shifted (the cached cell is then not the   \
       indexed one) */                                                           \
    int n = 0;                                                                   \
    for( int a = 0; a < 3; ++ a )                                                \
        if( x[ a ] > xr[ a ] )      { gl_shift_##S( m, b, i, xl, xr, a, 1 ); ++ n; } \
        else if( x[ a ] < xl[ a ] ) { gl_shift_##S( m, b, i, xl, xr, a, 0 ); ++ n; } \
    return n;                                                                    \
}                                                                                \
static void walk_##S( const kpo_mesh_t * m, F * x, const F * dir, int * i,       \
                      int * ibp, F proper, int * stepp, int * todop,             \
                      double scale, double * flux_f, long long * flux_fx,        \
                      int * fixp )                                               \
{                                                                                \
    const int cpb = m->nc[ 0 ] * m->nc[ 1 ] * m->nc[ 2 ];                       \
    int ib = * ibp, step = * stepp, todo = -1;   /* photon.h:108 */              \
    int ib_old = -1;                                                             \
    F xl[ 3 ], xr[ 3 ];                                                          \
    for( ; step > 0; -- step )                   /* photon.h:111-121 */          \
    {                                                                            \
        if( ib != ib_old && ib >= 0 )                                            \
        {                                                                        \
            gl_load_##S( m, ib, i, xl, xr );                                     \
            * fixp += gl_fix_##S( m, ib, i, x, xl, xr );                         \
            ib_old = ib;                                                         \
        }                                                                        \
        const int b = ib;                        /* prx = bmap[ib_l] */          \
        F dl[ 3 ];                               /* get_dl, photon.h:20-44 */    \
        for( int a = 0; a < 3; ++ a )                                            \
        {                                                                        \
            if( dir[ a ] == 0 ) { dl[ a ] = -1; continue; }                      \
            const F xf = dir[ a ] > 0 ? xr[ a ] : xl[ a ];                       \
            dl[ a ] = ( xf - x[ a ] ) / dir[ a ];                                \
        }                                                                        \
        int ap = 0;                                                              \
        F dmin = ( F ) FLT_MAX;                                                  \
        for( int a = 0; a < 3; ++ a )                                            \
            if( dl[ a ] >= 0 && dl[ a ] <= dmin ) { ap = a; dmin = dl[ a ]; }    \
        {   /* proc_phys, photon.h:73-83 */                                      \
            const F dsi = dl[ ap ] / ( F ) m->vol0[ b ];                         \
            const F v   = proper * dsi;                                          \
            const long c = ( long ) b * cpb + i[ 0 ]                             \
                         + m->nc[ 0 ] * ( i[ 1 ] + m->nc[ 1 ] * i[ 2 ] );        \
            if( flux_f )  flux_f [ c ] = ( double ) ( ( F ) flux_f[ c ] + v );   \
            if( flux_fx ) flux_fx[ c ] += llrint( ( double ) v * scale );        \
        }                                                                        \
        for( int a = 0; a < 3; ++ a )            /* proc_geo, photon.h:54-71 */  \
            if( a == ap )                                                        \
            {                                                                    \
                const int rhs = dir[ a ] > 0;                                    \
                x[ a ] = rhs ? xr[ a ] : xl[ a ];                                \
                i[ a ] += rhs ? 1 : -1;                                          \
                gl_shift_##S( m, b, i, xl, xr, a, rhs );                         \
            }                                                                    \
            else                                                                 \
                x[ a ] += dl[ ap ] * dir[ a ];                                   \
        todo = TO_KEEP;                          /* shift_blk, proxy.h:64-121 */ \
        for( int a = 0; a < 3; ++ a )                                            \
        {                                                                        \
            if( i[ a ] >= 0 && i[ a ] < m->nc[ a ] ) continue;                   \
            const int side = i[ a ] > 0;                                         \
            if( m->phybnd[ 6 * b + 2 * a + side ] ) { todo = TO_RM; break; }     \
            const int a1 = ( a + 1 ) % 3, a2 = ( a + 2 ) % 3;                    \
            const int dlv = m->d_lvl[ 6 * b + 2 * a + side ];                    \
            int j0 = 0, j1 = 0;                                                  \
            if( dlv > 0 )                                                        \
            {                                                                    \
                j0 = i[ a1 ] >= m->nc[ a1 ] / 2;                                 \
                j1 = i[ a2 ] >= m->nc[ a2 ] / 2;                                 \
            }                                                                    \
            const int slot = ( ( a * 2 + side ) * 2 + j0 ) * 2 + j1;             \
            const int nid = m->nb_id[ 24 * b + slot ];                           \
            ib = nid;                                                            \
            if( nid < 0 ) { todo = TO_RM; break; }                               \
            i[ a ] = i[ a ] > 0 ? 0 : m->nc[ a ] - 1;                            \
            const int * sh = m->nb_shift + 48 * b + 2 * slot;                    \
            if( dlv < 0 )                                                        \
            {                                                                    \
                i[ a1 ] = i[ a1 ] / 2 + sh[ 0 ] * m->nc[ a1 ] / 2;               \
                i[ a2 ] = i[ a2 ] / 2 + sh[ 1 ] * m->nc[ a2 ] / 2;               \
            }                                                                    \
            else if( dlv > 0 )                                                   \
            {                                                                    \
                const int h1 = m->nc[ a1 ] / 2, h2 = m->nc[ a2 ] / 2;            \
                i[ a1 ] = ( i[ a1 ] < h1 ? i[ a1 ] : i[ a1 ] - h1 ) * 2;         \
                i[ a2 ] = ( i[ a2 ] < h2 ? i[ a2 ] : i[ a2 ] - h2 ) * 2;         \
            }                                                                    \
            break;                                                               \
        }                                                                        \
        const int ok = todo != TO_RM;                                            \
        int wrapped = 0;                         /* regulate, particle_base.h:37-56 */ \
        for( int a = 0; a < 3; ++ a )                                            \
            if( m->periodic[ a ] )                                               \
            {                                                                    \
                if( x[ a ] < ( F ) m->xlim[ 0 ][ a ] )                           \
                { x[ a ] += ( F ) m->lbox[ a ]; wrapped = 1; }                   \
                else if( x[ a ] >= ( F ) m->xlim[ 1 ][ a ] )                     \
                { x[ a ] -= ( F ) m->lbox[ a ]; wrapped = 1; }                   \
            }                                                                    \
        if( ok && wrapped )                      /* photon.h:96-100 */           \
        {                                                                        \
            gl_load_##S( m, ib, i, xl, xr );                                     \
            * fixp += gl_fix_##S( m, ib, i, x, xl, xr );                         \
        }                                                                        \
        if( ! ok ) break;                                                        \
    }                                                                            \
    if( step <= 0 ) todo = TO_RM;                /* photon.h:122-123 */          \
    * ibp = ib; * stepp = step; * todop = todo;                                  \
}

KPO_DEFINE_WALK( float,  f32 )
KPO_DEFINE_WALK( double, f64 )

int kpo_trace( const kpo_mesh_t * m, int precision, long n, double * x,
               const double * dir, int * cell, int * ib, const double * proper,
               int * step, int * todo, int fx_shift, double * flux_f,
               long long * flux_fx )
{
    return kpo_trace_ex( m, precision, n, x, dir, cell, ib, proper, step, todo, fx_shift,
                         flux_f, flux_fx, NULL );
}

int kpo_trace_ex( const kpo_mesh_t * m, int precision, long n, double * x,
                  const double * dir, int * cell, int * ib, const double * proper,
                  int * step, int * todo, int fx_shift, double * flux_f,
                  long long * flux_fx, int * fix_shifts )
{
    const double scale = ldexp( 1.0, fx_shift );
    for( long p = 0; p < n; ++ p )
    {
        int fx_dummy = 0;
        int * fixp = fix_shifts ? fix_shifts + p : & fx_dummy;
        if( todo[ p ] != TO_KEEP )          /* integrator.h:90-92 */
            continue;
        if( ib[ p ] < 0 || ib[ p ] >= m->n_blocks )
            return -1;
        if( precision == 4 )
        {
            float xf[ 3 ], df[ 3 ];
            for( int a = 0; a < 3; ++ a )
            { xf[ a ] = ( float ) x[ 3 * p + a ]; df[ a ] = ( float ) dir[ 3 * p + a ]; }
            walk_f32( m, xf, df, cell + 3 * p, ib + p, ( float ) proper[ p ], step + p,
                      todo + p, scale, flux_f, flux_fx, fixp );
            for( int a = 0; a < 3; ++ a ) x[ 3 * p + a ] = xf[ a ];
        }
        else
            walk_f64( m, x + 3 * p, dir + 3 * p, cell + 3 * p, ib + p, proper[ p ],
                      step + p, todo + p, scale, flux_f, flux_fx, fixp );
    }
    return 0;
}

/* ====================================================================== */
/* Polarized transport restatement                                         */

#include "oracle_math.h"

enum { ST_ESCAPED = 1, ST_ABSORBED = 2, ST_SCATTER_CAP = 3, ST_STEP_CAP = 4, ST_LOST = 5 };

typedef struct
{
    const kpo_mesh_t * m;
    const float      * sig;
    const int        * lookup;
    int                lk_n[ 3 ];
    double             lk_inv[ 3 ];
    double           * inv_dx;         /* [nb][3] */
    int                cpb;
    om_phase           ph;
    int                n_mu;
    float              mu_lo, mu_inv_w;
    int                img_n;
    om_v3              o, ev, eh;
    double             inv_o[ 3 ], o_d[ 3 ], ev_d[ 3 ], eh_d[ 3 ], img_c[ 3 ];
    double             img_inv_pix;
    float              tau_cut;
    double             fx_scale;
    int                n_batch, img_bn;
    float              w_min, rr_survive;
    int                max_scatter;
    long long          max_steps;
    long long         *mu, *image, *img_batch;
    long long         *flux;           /* path-length tally (null: off) */
    double             flux_scale;
} tctx;

typedef struct
{
    double    x[ 3 ], inv[ 3 ];
    om_v3     d, e1;
    om_stokes S;
    float     w, tau;
    int       b, c[ 3 ], n_scat;
    long long n_steps, pid;
    om_rng    rng;
} tpk;

static long tcell( const tctx * t, int b, const int * c )
{
    return ( long ) b * t->cpb + c[ 0 ] + t->m->nc[ 0 ] * ( c[ 1 ] + t->m->nc[ 1 ] * c[ 2 ] );
}

static void tset_inv( tpk * p )
{
    for( int a = 0; a < 3; ++ a )
    {
        const float da = om_comp( p->d, a );
        p->inv[ a ] = da != 0.0f ? 1.0 / ( double ) da : 0.0;
    }
}

static double texit( const tctx * t, int b, const int * c, const double * x, om_v3 d,
                     const double * inv, int * ax )
{
    double tm = 1e300;
    * ax = 0;
    for( int a = 0; a < 3; ++ a )
    {
        const float da = om_comp( d, a );
        if( da == 0.0f ) continue;
        const double face = fma( ( double ) ( c[ a ] + ( da > 0.0f ? 1 : 0 ) ),
                                 t->m->dx0[ 3 * b + a ], t->m->xf0[ 3 * b + a ] );
        double ta = ( face - x[ a ] ) * inv[ a ];
        ta = ta < 0.0 ? 0.0 : ta;
        if( ta < tm ) { tm = ta; * ax = a; }
    }
    return tm;
}

/* returns 1 if still inside, 0 if it left the domain (lost set if no
 * neighbour) */
static int tcross( const tctx * t, int * b, int * c, double * x, int ax, int pos, int * lost )
{
    const kpo_mesh_t * m = t->m;
    * lost = 0;
    const int cn = c[ ax ] + ( pos ? 1 : -1 );
    if( cn >= 0 && cn < m->nc[ ax ] )
    {
        c[ ax ] = cn;
        x[ ax ] = fma( ( double ) ( pos ? cn : cn + 1 ), m->dx0[ 3 * * b + ax ], m->xf0[ 3 * * b + ax ] );
        return 1;
    }
    const int side = pos ? 1 : 0;
    if( m->phybnd[ 6 * * b + 2 * ax + side ] )
    {   /* leaves the domain: the position ends on the boundary face */
        x[ ax ] = fma( ( double ) ( pos ? c[ ax ] + 1 : c[ ax ] ), m->dx0[ 3 * * b + ax ],
                       m->xf0[ 3 * * b + ax ] );
        return 0;
    }
    const int a1 = ( ax + 1 ) % 3, a2 = ( ax + 2 ) % 3;
    int j0 = 0, j1 = 0;
    if( m->d_lvl[ 6 * * b + 2 * ax + side ] > 0 )
    {
        j0 = c[ a1 ] >= m->nc[ a1 ] / 2;
        j1 = c[ a2 ] >= m->nc[ a2 ] / 2;
    }
    const int nid = m->nb_id[ 24 * * b + ( ( ax * 2 + side ) * 2 + j0 ) * 2 + j1 ];
    if( nid < 0 || nid >= m->n_blocks ) { * lost = 1; return 0; }
    * b = nid;
    for( int a = 0; a < 3; ++ a )
    {
        if( a == ax )
        {
            c[ a ] = pos ? 0 : m->nc[ a ] - 1;
            x[ a ] = pos ? m->xf0[ 3 * nid + a ]
                         : fma( ( double ) m->nc[ a ], m->dx0[ 3 * nid + a ], m->xf0[ 3 * nid + a ] );
        }
        else
        {
            const double f = floor( ( x[ a ] - m->xf0[ 3 * nid + a ] ) * t->inv_dx[ 3 * nid + a ] );
            c[ a ] = f < 0.0 ? 0 : ( f > ( double ) ( m->nc[ a ] - 1 ) ? m->nc[ a ] - 1 : ( int ) f );
        }
    }
    return 1;
}

/* Peel-off ray toward the observer: a fixed-direction cell march, block by
 * block, measured from the point x0 where the ray entered its current block
 * (or started).  tm[a] is the distance from x0 to the next face of the
 * current cell on axis a ((face - x0[a]) times the inverse direction; 1e300
 * on an axis the observer direction does not move along); a segment ends at
 * the nearest (the first axis wins ties) and its length is that distance
 * less the distance already travelled from x0 (tc; never negative).  A block
 * hand-off goes through the crossing point x0 + tc o, snapped to the new
 * block's face (which also wraps a periodic boundary), and makes it the new
 * x0.  The kernels march every peel-off ray this way (k_peel, and the rays of
 * k_forward and k_adjoint marched where they start). */
typedef struct
{
    int    b, c[ 3 ];
    double x0[ 3 ], tm[ 3 ], tc;
} tray;

static void tray_faces( const tctx * t, tray * r )
{
    const kpo_mesh_t * m = t->m;
    for( int a = 0; a < 3; ++ a )
    {
        const float oa = om_comp( t->o, a );
        if( oa == 0.0f ) { r->tm[ a ] = 1e300; continue; }
        const double face = fma( ( double ) ( r->c[ a ] + ( oa > 0.0f ? 1 : 0 ) ),
                                 m->dx0[ 3 * r->b + a ], m->xf0[ 3 * r->b + a ] );
        r->tm[ a ] = ( face - r->x0[ a ] ) * t->inv_o[ a ];
    }
}

static void tray_start( const tctx * t, tray * r, int b, const int * c0, const double * x0 )
{
    r->b = b;
    for( int a = 0; a < 3; ++ a ) { r->c[ a ] = c0[ a ]; r->x0[ a ] = x0[ a ]; }
    r->tc = 0.0;
    tray_faces( t, r );
}

/* Length of the ray's next segment; *ax receives the axis of its exit face. */
static double tray_segment( tray * r, int * ax )
{
    int a0 = 0;
    double tn = r->tm[ 0 ];
    if( r->tm[ 1 ] < tn ) { tn = r->tm[ 1 ]; a0 = 1; }
    if( r->tm[ 2 ] < tn ) { tn = r->tm[ 2 ]; a0 = 2; }
    double dt = tn - r->tc;
    dt = dt < 0.0 ? 0.0 : dt;
    if( tn > r->tc ) r->tc = tn;
    * ax = a0;
    return dt;
}

/* Into the next cell across face ax; 0 when the ray leaves the domain. */
static int tray_cross( const tctx * t, tray * r, int ax, unsigned long long * hops )
{
    const kpo_mesh_t * m = t->m;
    const int pos = om_comp( t->o, ax ) > 0.0f;
    const int cn = r->c[ ax ] + ( pos ? 1 : -1 );
    if( cn >= 0 && cn < m->nc[ ax ] )
    {
        r->c[ ax ] = cn;
        const double face = fma( ( double ) ( cn + pos ), m->dx0[ 3 * r->b + ax ],
                                 m->xf0[ 3 * r->b + ax ] );
        r->tm[ ax ] = ( face - r->x0[ ax ] ) * t->inv_o[ ax ];
        return 1;
    }
    double x[ 3 ];
    for( int a = 0; a < 3; ++ a ) x[ a ] = fma( r->tc, t->o_d[ a ], r->x0[ a ] );
    int lost;
    const int b_old = r->b;
    if( ! tcross( t, & r->b, r->c, x, ax, pos, & lost ) ) return 0;
    * hops += r->b != b_old;
    for( int a = 0; a < 3; ++ a ) r->x0[ a ] = x[ a ];
    r->tc = 0.0;
    tray_faces( t, r );
    return 1;
}

/* Optical depth from x0 to the domain boundary along the observer direction;
 * stops early (returns > tau_cut) once tau_cut is exceeded. */
static float tpeel_tau( const tctx * t, int b, const int * c0, const double * x0,
                        unsigned long long * steps, unsigned long long * hops )
{
    tray r;
    tray_start( t, & r, b, c0, x0 );
    float tau = 0.0f;
    for( int k = 0; k < ( 1 << 20 ); ++ k )
    {
        const long ci = tcell( t, r.b, r.c );
        const float ext = t->sig[ 2 * ci ] + t->sig[ 2 * ci + 1 ];
        int ax;
        const double dt = tray_segment( & r, & ax );
        tau = tau + ext * ( float ) dt;
        ++ * steps;
        if( tau > t->tau_cut ) return tau;
        if( ! tray_cross( t, & r, ax, hops ) ) return tau;
    }
    return tau;
}

static void tadd( long long * base, long i, float v, double sc )
{
    base[ i ] += llrint( ( double ) v * sc );
}

/* Path-length flux estimator of a walk segment of length dl in the packet's
 * cell: w dl / volume, as photon::cart_t::proc_phys deposits proper * dl /
 * volume (modules/particle/radiation/photon.h:73-83), the packet's weight
 * being its `proper`.  The kernel keeps w / volume per packet and multiplies
 * by dl, so this does the same. */
static void tflux( const tctx * t, const tpk * p, double dl )
{
    if( ! t->flux ) return;
    const double wv = ( double ) p->w / t->m->vol0[ p->b ];
    const double v = dl * wv;
    t->flux[ tcell( t, p->b, p->c ) ] += llrint( v * t->flux_scale );
}

/* Image pixel (iy * n + ix) under x, or -1 outside the image. */
static int timage_pixel( const tctx * t, const double * x )
{
    double r[ 3 ];
    for( int a = 0; a < 3; ++ a ) r[ a ] = x[ a ] - t->img_c[ a ];
    const double hp = ( r[ 0 ] * t->eh_d[ 0 ] + r[ 1 ] * t->eh_d[ 1 ] ) + r[ 2 ] * t->eh_d[ 2 ];
    const double vp = ( r[ 0 ] * t->ev_d[ 0 ] + r[ 1 ] * t->ev_d[ 1 ] ) + r[ 2 ] * t->ev_d[ 2 ];
    const double half = 0.5 * t->img_n;
    const double fx = floor( fma( hp, t->img_inv_pix, half ) );
    const double fy = floor( fma( vp, t->img_inv_pix, half ) );
    if( fx < 0.0 || fy < 0.0 || fx >= t->img_n || fy >= t->img_n ) return -1;
    return ( int ) fy * t->img_n + ( int ) fx;
}

/* Optional record of every image deposit: its pixel and (I, Q, U, V), in
 * deposit order, up to `cap` deposits (the count keeps growing past it).  Set
 * by kpo_set_pixel_sink; process-global, for sequential test use: the exact
 * sum of a pixel's float deposits bounds the rounding of both tally modes. */
static int *       s_pix_sink_pix = NULL;
static float *     s_pix_sink_val = NULL;
static long long   s_pix_sink_cap = 0;
static long long * s_pix_sink_n   = NULL;

void kpo_set_pixel_sink( int * pix, float * val, long long cap, long long * n )
{
    s_pix_sink_pix = pix; s_pix_sink_val = val; s_pix_sink_cap = cap; s_pix_sink_n = n;
}

static void tdeposit_pixel( const tctx * t, int pixel, long long pid,
                            float I, float Q, float U, float V )
{
    if( s_pix_sink_n )
    {
        const long long k = ( * s_pix_sink_n ) ++;
        if( k < s_pix_sink_cap )
        {
            s_pix_sink_pix[ k ] = pixel;
            s_pix_sink_val[ 4 * k + 0 ] = I; s_pix_sink_val[ 4 * k + 1 ] = Q;
            s_pix_sink_val[ 4 * k + 2 ] = U; s_pix_sink_val[ 4 * k + 3 ] = V;
        }
    }
    const int ix = pixel % t->img_n, iy = pixel / t->img_n;
    const long pix = ( long ) pixel * 4;
    tadd( t->image, pix + 0, I, t->fx_scale );
    tadd( t->image, pix + 1, Q, t->fx_scale );
    tadd( t->image, pix + 2, U, t->fx_scale );
    tadd( t->image, pix + 3, V, t->fx_scale );
    const int batch = ( int ) ( pid % t->n_batch );
    const long bp = ( ( ( long ) batch * t->img_bn + iy * t->img_bn / t->img_n ) * t->img_bn
                      + ix * t->img_bn / t->img_n ) * 4;
    tadd( t->img_batch, bp + 0, I, t->fx_scale );
    tadd( t->img_batch, bp + 1, Q, t->fx_scale );
    tadd( t->img_batch, bp + 2, U, t->fx_scale );
    tadd( t->img_batch, bp + 3, V, t->fx_scale );
}

static int ttally_escape( const tctx * t, const tpk * p )
{
    if( t->n_mu <= 0 ) return 0;
    const float fb = floorf( ( p->d.z - t->mu_lo ) * t->mu_inv_w );
    if( !( fb >= 0.0f && fb < ( float ) t->n_mu ) ) return 0;
    const int bin = ( int ) fb;
    const om_v3 e2 = om_cross( p->d, p->e1 );
    float c2, s2;
    om_double_angle( p->e1.z, e2.z, & c2, & s2 );
    float q = p->S.q, u = p->S.u;
    om_rotate( & q, & u, c2, s2 );
    const int batch = ( int ) ( p->pid % t->n_batch );
    const long i = ( ( long ) batch * t->n_mu + bin ) * 4;
    tadd( t->mu, i + 0, p->w, t->fx_scale );
    tadd( t->mu, i + 1, p->w * q, t->fx_scale );
    tadd( t->mu, i + 2, p->w * u, t->fx_scale );
    tadd( t->mu, i + 3, p->w * p->S.v, t->fx_scale );
    return 1;
}

static float tsample_tau( om_rng * g )
{
    const om_u4 r = om_next( g );
    return ( float ) ( -om_log( ( double ) om_u01( r.x ) ) );
}

static om_v3 temit_dir( om_rng * g, int emit )
{
    float mu = 0.0f, a = 1.0f, b = 0.0f, r2 = 1.0f;
    for( int trial = 0; trial < 64; ++ trial )
    {
        const om_u4 r = om_next( g );
        mu = emit == 1 ? om_u01( r.x ) : om_usym( r.x );
        a = om_usym( r.y );
        b = om_usym( r.z );
        r2 = a * a + b * b;
        if( r2 <= 1.0f && r2 > 0.0f ) break;
        a = 1.0f; b = 0.0f; r2 = 1.0f;
    }
    const float rr = sqrtf( r2 );
    return om_dir_from( mu, a / rr, b / rr );
}

/* Cell of block b holding x (floor, clamped to the block). */
static void tcell_of( const tctx * t, int b, const double * x, int * c )
{
    const kpo_mesh_t * m = t->m;
    for( int a = 0; a < 3; ++ a )
    {
        const double f = floor( ( x[ a ] - m->xf0[ 3 * b + a ] ) * t->inv_dx[ 3 * b + a ] );
        c[ a ] = f < 0.0 ? 0 : ( f > ( double ) ( m->nc[ a ] - 1 ) ? m->nc[ a ] - 1 : ( int ) f );
    }
}

/* Block and cell of x through the finest-level lookup grid; 0 if none. */
static int tlocate( const tctx * t, const double * x, int * b, int * c )
{
    const kpo_mesh_t * m = t->m;
    int li[ 3 ];
    for( int a = 0; a < 3; ++ a )
    {
        const double f = floor( ( x[ a ] - m->xlim[ 0 ][ a ] ) * t->lk_inv[ a ] );
        li[ a ] = f < 0.0 ? 0 : ( f >= t->lk_n[ a ] ? t->lk_n[ a ] - 1 : ( int ) f );
    }
    * b = t->lookup[ ( ( long ) li[ 2 ] * t->lk_n[ 1 ] + li[ 1 ] ) * t->lk_n[ 0 ] + li[ 0 ] ];
    if( * b < 0 || * b >= m->n_blocks ) return 0;
    tcell_of( t, * b, x, c );
    return 1;
}

/* Creates packet pid: from the caller's packet table (entry pid -
 * packet_offset) when the cfg has one, else from source pid % n_sources.
 * peel_I receives the emission's intensity per steradian toward the
 * observer per unit weight (1/(4 pi) for an isotropic point source, the
 * entry's own for a table; 0: no peel-off at emission). */
static int temit( const tctx * t, const kpo_cfg_t * c, long long pid, tpk * p, float * peel_I )
{
    const kpo_mesh_t * m = t->m;
    p->pid = pid;
    p->rng.k0 = c->seed; p->rng.k1 = c->stream_id;
    p->rng.pid_lo = ( uint32_t ) pid; p->rng.pid_hi = ( uint32_t ) ( pid >> 32 );
    p->rng.draw = 0;
    if( c->packets )
    {
        const kpo_packet_init_t * e = c->packets + ( pid - c->packet_offset );
        for( int a = 0; a < 3; ++ a ) p->x[ a ] = e->x[ a ];
        p->b = e->ib;
        if( p->b < 0 )
        {
            if( ! tlocate( t, p->x, & p->b, p->c ) ) return 0;
        }
        else
        {
            if( p->b >= m->n_blocks ) return 0;
            tcell_of( t, p->b, p->x, p->c );
        }
        p->d.x = e->d[ 0 ]; p->d.y = e->d[ 1 ]; p->d.z = e->d[ 2 ];
        p->e1 = om_frame_for( p->d );
        p->S.q = e->stokes[ 0 ]; p->S.u = e->stokes[ 1 ]; p->S.v = e->stokes[ 2 ];
        p->w = e->w;
        p->n_scat = 0;
        p->n_steps = 0;
        tset_inv( p );
        * peel_I = e->peel_I;
        return 1;
    }
    const kpo_source_t * s = c->sources + pid % c->n_sources;
    * peel_I = s->kind == 0 && s->emit == 0 ? OM_INV4PI : 0.0f;
    if( s->kind == 0 )
    {
        for( int a = 0; a < 3; ++ a ) { p->x[ a ] = s->pos[ a ]; p->c[ a ] = s->cell[ a ]; }
        p->b = s->ib;
    }
    else
    {
        const om_u4 r = om_next( & p->rng );
        p->x[ 0 ] = fma( ( double ) om_u01( r.x ), m->lbox[ 0 ], m->xlim[ 0 ][ 0 ] );
        p->x[ 1 ] = fma( ( double ) om_u01( r.y ), m->lbox[ 1 ], m->xlim[ 0 ][ 1 ] );
        p->x[ 2 ] = m->xlim[ 0 ][ 2 ];
        if( ! tlocate( t, p->x, & p->b, p->c ) ) return 0;
    }
    if( p->b < 0 || p->b >= m->n_blocks ) return 0;
    p->d = temit_dir( & p->rng, s->emit );
    p->e1 = om_frame_for( p->d );
    p->S.q = p->S.u = p->S.v = 0.0f;
    p->w = 1.0f;
    p->n_scat = 0;
    p->n_steps = 0;
    tset_inv( p );
    return 1;
}

static void trecord( const kpo_cfg_t * c, kpo_record_t * rec, const tpk * p, int status )
{
    const long long k = p->pid - c->packet_offset;
    if( ! rec || k < 0 || k >= c->n_record ) return;
    kpo_record_t * r = rec + k;
    for( int a = 0; a < 3; ++ a ) { r->x[ a ] = p->x[ a ]; r->cell[ a ] = p->c[ a ]; }
    r->d[ 0 ] = p->d.x; r->d[ 1 ] = p->d.y; r->d[ 2 ] = p->d.z;
    r->stokes[ 0 ] = p->S.q; r->stokes[ 1 ] = p->S.u; r->stokes[ 2 ] = p->S.v;
    r->w = p->w; r->ib = p->b; r->n_scatter = p->n_scat; r->status = status;
    r->rng_draws = p->rng.draw; r->n_steps = p->n_steps;
}

/* Fills the transport context from the mesh tables and configuration
 * (the host side of make_fwd_params in the device code). */
static int tsetup( tctx * tp, const kpo_mesh_t * m, const float * sigma2, const int * lookup,
                   const int * lookup_n, const kpo_cfg_t * c )
{
    tctx t;
    memset( & t, 0, sizeof( t ) );
    t.m = m; t.sig = sigma2; t.lookup = lookup;
    t.cpb = m->nc[ 0 ] * m->nc[ 1 ] * m->nc[ 2 ];
    t.inv_dx = ( double * ) malloc( sizeof( double ) * 3 * ( size_t ) m->n_blocks );
    if( ! t.inv_dx ) return -2;
    for( int b = 0; b < m->n_blocks; ++ b )
        for( int a = 0; a < 3; ++ a )
            t.inv_dx[ 3 * b + a ] = 1.0 / m->dx0[ 3 * b + a ];
    for( int a = 0; a < 3; ++ a )
    {
        t.lk_n[ a ] = lookup_n[ a ];
        t.lk_inv[ a ] = lookup_n[ a ] / m->lbox[ a ];
    }
    t.ph.kind = c->phase; t.ph.g = c->hg_g; t.ph.pmax = c->pol_max;
    t.n_mu = c->n_mu_bins;
    t.mu_lo = c->mu_lo;
    t.mu_inv_w = c->n_mu_bins > 0 ? ( float ) ( c->n_mu_bins / ( ( double ) c->mu_hi - c->mu_lo ) ) : 0.f;
    t.img_n = c->image_n;
    const double inc = c->inclination_deg * M_PI / 180.0, az = c->azimuth_deg * M_PI / 180.0;
    const float o[ 3 ]  = { ( float ) ( sin( inc ) * cos( az ) ), ( float ) ( sin( inc ) * sin( az ) ),
                            ( float ) cos( inc ) };
    const float ev[ 3 ] = { ( float ) ( -cos( inc ) * cos( az ) ), ( float ) ( -cos( inc ) * sin( az ) ),
                            ( float ) sin( inc ) };
    const float eh[ 3 ] = { ev[ 1 ] * o[ 2 ] - ev[ 2 ] * o[ 1 ], ev[ 2 ] * o[ 0 ] - ev[ 0 ] * o[ 2 ],
                            ev[ 0 ] * o[ 1 ] - ev[ 1 ] * o[ 0 ] };
    t.o.x = o[ 0 ]; t.o.y = o[ 1 ]; t.o.z = o[ 2 ];
    t.ev.x = ev[ 0 ]; t.ev.y = ev[ 1 ]; t.ev.z = ev[ 2 ];
    t.eh.x = eh[ 0 ]; t.eh.y = eh[ 1 ]; t.eh.z = eh[ 2 ];
    for( int a = 0; a < 3; ++ a )
    {
        t.o_d[ a ] = o[ a ]; t.ev_d[ a ] = ev[ a ]; t.eh_d[ a ] = eh[ a ];
        t.inv_o[ a ] = o[ a ] != 0.0f ? 1.0 / ( double ) o[ a ] : 0.0;
        t.img_c[ a ] = c->image_center[ a ];
    }
    t.img_inv_pix = c->image_n > 0 ? c->image_n / ( 2.0 * c->image_half_width ) : 0.0;
    t.tau_cut = c->tau_peel_max > 0 ? c->tau_peel_max : 40.0f;
    t.fx_scale = ldexp( 1.0, c->fx_shift );
    t.flux_scale = ldexp( 1.0, c->flux_fx_shift > 0 ? c->flux_fx_shift : c->fx_shift );
    t.n_batch = c->n_batches;
    t.img_bn = c->image_batch_n >= 1 ? c->image_batch_n : 1;
    t.w_min = c->w_min;
    t.rr_survive = c->rr_survive > 0 ? c->rr_survive : 0.1f;
    t.max_scatter = c->max_scatter;
    t.max_steps = c->max_steps;
    * tp = t;
    return 0;
}

int kpo_transport( const kpo_mesh_t * m, const float * sigma2, const int * lookup,
                   const int * lookup_n, const kpo_cfg_t * c, long long * mu,
                   long long * image, long long * img_batch,
                   unsigned long long * counters, kpo_record_t * rec, long long * flux )
{
    tctx t;
    if( tsetup( & t, m, sigma2, lookup, lookup_n, c ) ) return -2;
    t.mu = mu; t.image = image; t.img_batch = img_batch; t.flux = flux;
    unsigned long long cnt[ 10 ] = { 0, 0, 0, 0, 0, 0, 0, 0, 0, 0 };
    for( long long k = 0; k < c->n_packets; ++ k )
    {
        tpk p;
        float peel_I;
        if( ! temit( & t, c, c->packet_offset + k, & p, & peel_I ) ) { free( t.inv_dx ); return -1; }
        ++ cnt[ 7 ];
        if( t.img_n > 0 && peel_I > 0.0f )
        {   /* direct light: peel-off rays start only inside the image */
            const int pix = timage_pixel( & t, p.x );
            if( pix >= 0 )
            {
                const float tau = tpeel_tau( & t, p.b, p.c, p.x, & cnt[ 1 ], & cnt[ 8 ] );
                if( tau <= t.tau_cut )
                {
                    const float att = p.w * ( float ) om_exp_neg( -( double ) tau );
                    tdeposit_pixel( & t, pix, p.pid, att * peel_I, att * 0.0f,
                                    att * 0.0f, att * 0.0f );
                    ++ cnt[ 9 ];
                }
            }
        }
        p.tau = tsample_tau( & p.rng );
        for( ;; )
        {
            const long ci = tcell( & t, p.b, p.c );
            const float ss = sigma2[ 2 * ci ], sa = sigma2[ 2 * ci + 1 ];
            const float ext = ss + sa;
            int ax;
            const double tt = texit( & t, p.b, p.c, p.x, p.d, p.inv, & ax );
            const float dtau = ext * ( float ) tt;
            ++ cnt[ 0 ];
            ++ p.n_steps;
            int end = 0;
            if( dtau >= p.tau )
            {
                double ti = ( double ) ( p.tau / ext );
                ti = ti > tt ? tt : ti;
                tflux( & t, & p, ti );
                p.x[ 0 ] = fma( ti, ( double ) p.d.x, p.x[ 0 ] );
                p.x[ 1 ] = fma( ti, ( double ) p.d.y, p.x[ 1 ] );
                p.x[ 2 ] = fma( ti, ( double ) p.d.z, p.x[ 2 ] );
                ++ p.n_scat;
                ++ cnt[ 2 ];
                p.w = p.w * ( ss / ext );
                const int pix = t.img_n > 0 ? timage_pixel( & t, p.x ) : -1;
                if( pix >= 0 )
                {
                    const float tau = tpeel_tau( & t, p.b, p.c, p.x, & cnt[ 1 ], & cnt[ 8 ] );
                    if( tau <= t.tau_cut )
                    {
                        float Q, U, V;
                        const float I = om_peel_stokes( t.ph, p.d, p.e1, p.S, t.o, t.ev, t.eh,
                                                        & Q, & U, & V );
                        const float att = p.w * ( float ) om_exp_neg( -( double ) tau );
                        tdeposit_pixel( & t, pix, p.pid, att * I, att * Q, att * U, att * V );
                        ++ cnt[ 9 ];
                    }
                }
                if( p.n_scat >= t.max_scatter )
                    end = ST_SCATTER_CAP;
                else if( p.w < t.w_min )
                {
                    const om_u4 r = om_next( & p.rng );
                    if( om_u01( r.x ) < t.rr_survive ) p.w = p.w / t.rr_survive;
                    else end = ST_ABSORBED;
                }
                if( ! end )
                {
                    om_scatter( t.ph, & p.rng, & p.d, & p.e1, & p.S );
                    tset_inv( & p );
                    p.tau = tsample_tau( & p.rng );
                }
            }
            else
            {
                p.tau = p.tau - dtau;
                tflux( & t, & p, tt );
                for( int a = 0; a < 3; ++ a )
                    if( a != ax ) p.x[ a ] = fma( tt, ( double ) om_comp( p.d, a ), p.x[ a ] );
                int lost;
                const int b_old = p.b;
                if( ! tcross( & t, & p.b, p.c, p.x, ax, om_comp( p.d, ax ) > 0.0f, & lost ) )
                {
                    if( lost ) end = ST_LOST;
                    else { end = ST_ESCAPED; cnt[ 9 ] += ttally_escape( & t, & p ); }
                }
                else
                    cnt[ 8 ] += p.b != b_old;
            }
            if( ! end && p.n_steps >= t.max_steps ) end = ST_STEP_CAP;
            if( end )
            {
                trecord( c, rec, & p, end );
                cnt[ 3 ] += end == ST_ESCAPED;
                cnt[ 4 ] += end == ST_ABSORBED;
                cnt[ 5 ] += end == ST_SCATTER_CAP || end == ST_STEP_CAP;
                cnt[ 6 ] += end == ST_LOST;
                break;
            }
        }
    }
    if( counters )
        for( int k = 0; k < 10; ++ k ) counters[ k ] += cnt[ k ];
    free( t.inv_dx );
    return 0;
}

/* ====================================================================== */
/* Unit-test exports of the physics primitives                             */

void kpo_philox( const uint32_t * ctr, const uint32_t * key, uint32_t * out )
{
    om_u4 c = { ctr[ 0 ], ctr[ 1 ], ctr[ 2 ], ctr[ 3 ] };
    const om_u4 r = om_philox( c, key[ 0 ], key[ 1 ] );
    out[ 0 ] = r.x; out[ 1 ] = r.y; out[ 2 ] = r.z; out[ 3 ] = r.w;
}

void kpo_log_exp( long n, const double * x, double * ln_x, double * exp_negx )
{
    for( long i = 0; i < n; ++ i )
    {
        ln_x[ i ] = om_log( x[ i ] );
        exp_negx[ i ] = om_exp_neg( -x[ i ] );
    }
}

/* Scatters n packets travelling along +z (frame e1 = +x) with Stokes
 * (q, u, v); writes per packet the new direction, frame and Stokes. */
void kpo_scatter_sample( long n, uint32_t seed, int kind, float g, float pmax,
                         float q, float u, float v, float * out /* n*9 */ )
{
    om_phase ph = { kind, g, pmax };
    for( long i = 0; i < n; ++ i )
    {
        om_rng r = { seed, 7u, ( uint32_t ) i, 0u, 0u };
        om_v3 d = { 0.0f, 0.0f, 1.0f }, e1 = { 1.0f, 0.0f, 0.0f };
        om_stokes S = { q, u, v };
        om_scatter( ph, & r, & d, & e1, & S );
        float * o = out + 9 * i;
        o[ 0 ] = d.x; o[ 1 ] = d.y; o[ 2 ] = d.z;
        o[ 3 ] = e1.x; o[ 4 ] = e1.y; o[ 5 ] = e1.z;
        o[ 6 ] = S.q; o[ 7 ] = S.u; o[ 8 ] = S.v;
    }
}

/* ====================================================================== */
/* Path-replay adjoint restatement (same estimator and operation order as  */
/* the device kernel; sequential packets; int64 gradient tallies).         */

/* Optional per-cell sum of |term| and count of gradient deposits (both
 * tallies): what a float-atomic accumulation's rounding error is bounded by.
 * Set by kpo_set_abs_sink; process-global, for sequential test use. */
static double * s_abs_sink = NULL;

void kpo_set_abs_sink( double * sink ) { s_abs_sink = sink; }

static void tgadd( long long * base, long i, double v, double sc )
{
    base[ i ] += llrint( v * sc );
    if( s_abs_sink )
    {
        s_abs_sink[ 2 * i ] += fabs( v );
        s_abs_sink[ 2 * i + 1 ] += 1.0;
    }
}

static float tscore( const float * g, int pix, float I, float Q, float U, float V )
{
    const float * q = g + 4 * ( long ) pix;
    return ( ( q[ 0 ] * I + q[ 1 ] * Q ) + q[ 2 ] * U ) + q[ 3 ] * V;
}

/* Marches a peel-off ray like tpeel_tau and deposits -G * length per cell. */
static void tpeel_deposit( const tctx * t, int b, const int * c0, const double * x0, float G,
                           long long * g_len, double gsc, unsigned long long * steps )
{
    tray r;
    tray_start( t, & r, b, c0, x0 );
    float tau = 0.0f;
    unsigned long long hops = 0;
    for( int k = 0; k < ( 1 << 20 ); ++ k )
    {
        const long ci = tcell( t, r.b, r.c );
        const float ext = t->sig[ 2 * ci ] + t->sig[ 2 * ci + 1 ];
        int ax;
        const double dt = tray_segment( & r, & ax );
        tau = tau + ext * ( float ) dt;
        ++ * steps;
        if( tau > t->tau_cut ) return;
        tgadd( g_len, ci, -( double ) G * dt, gsc );
        if( ! tray_cross( t, & r, ax, & hops ) ) return;
    }
}

/* One replay of a packet.  pass 0 fills G0, Gs[] and *R (the sum of the
 * interaction terms, in vertex order); pass 1 deposits, starting from that
 * *R and subtracting each vertex's G after its peel-off ray.  Returns the
 * number of interaction vertices. */
static int tadjoint_pass( const tctx * t, const kpo_cfg_t * c, long long pid, int pass,
                          const float * g, float * G0, float * Gs, int gs_cap, double * Rp,
                          long long * g_len, long long * g_int, double gsc,
                          unsigned long long * cnt )
{
    tpk p;
    float peel_I;
    if( ! temit( t, c, pid, & p, & peel_I ) ) return -1;
    p.tau = tsample_tau( & p.rng );
    double R = pass == 1 ? * Rp : 0.0;
    int nv = 0;
    if( t->img_n > 0 && peel_I > 0.0f )
    {
        const int pix = timage_pixel( t, p.x );
        if( pix >= 0 )
        {
            if( pass == 0 )
            {
                const float tau = tpeel_tau( t, p.b, p.c, p.x, & cnt[ 1 ], & cnt[ 8 ] );
                float G = 0.0f;
                if( tau <= t->tau_cut )
                {
                    const float att = p.w * ( float ) om_exp_neg( -( double ) tau );
                    G = tscore( g, pix, att * peel_I, att * 0.0f, att * 0.0f, att * 0.0f );
                }
                * G0 = G;
            }
            else if( * G0 != 0.0f )
                tpeel_deposit( t, p.b, p.c, p.x, * G0, g_len, gsc, & cnt[ 1 ] );
        }
    }
    for( ;; )
    {
        const long ci = tcell( t, p.b, p.c );
        const float ss = t->sig[ 2 * ci ], sa = t->sig[ 2 * ci + 1 ];
        const float ext = ss + sa;
        int ax;
        const double tt = texit( t, p.b, p.c, p.x, p.d, p.inv, & ax );
        const float dtau = ext * ( float ) tt;
        ++ cnt[ 0 ];
        ++ p.n_steps;
        int end = 0;
        if( dtau >= p.tau )
        {
            double ti = ( double ) ( p.tau / ext );
            ti = ti > tt ? tt : ti;
            if( pass == 1 && R != 0.0 ) tgadd( g_len, ci, -R * ti, gsc );
            p.x[ 0 ] = fma( ti, ( double ) p.d.x, p.x[ 0 ] );
            p.x[ 1 ] = fma( ti, ( double ) p.d.y, p.x[ 1 ] );
            p.x[ 2 ] = fma( ti, ( double ) p.d.z, p.x[ 2 ] );
            ++ p.n_scat;
            ++ cnt[ 2 ];
            p.w = p.w * ( ss / ext );
            if( pass == 1 && R != 0.0 ) tgadd( g_int, ci, R / ( double ) ss, gsc );
            ++ nv;
            const int pix = t->img_n > 0 ? timage_pixel( t, p.x ) : -1;
            float pI = 0, pQ = 0, pU = 0, pV = 0, pw = 0;
            if( pix >= 0 )
            {
                pI = om_peel_stokes( t->ph, p.d, p.e1, p.S, t->o, t->ev, t->eh, & pQ, & pU, & pV );
                pw = p.w;
            }
            /* the peel-off ray of this vertex (before roulette and scattering,
             * whose random numbers it does not use) */
            if( pix >= 0 )
            {
                if( pass == 0 )
                {
                    const float tau = tpeel_tau( t, p.b, p.c, p.x, & cnt[ 1 ], & cnt[ 8 ] );
                    float G = 0.0f;
                    if( tau <= t->tau_cut )
                    {
                        const float att = pw * ( float ) om_exp_neg( -( double ) tau );
                        G = tscore( g, pix, att * pI, att * pQ, att * pU, att * pV );
                    }
                    R += ( double ) G;
                    if( nv <= gs_cap ) Gs[ nv - 1 ] = G;
                    else return -3;
                }
                else
                {
                    const float G = Gs[ nv - 1 ];
                    if( G != 0.0f )
                    {
                        tpeel_deposit( t, p.b, p.c, p.x, G, g_len, gsc, & cnt[ 1 ] );
                        R = R - ( double ) G;
                    }
                }
            }
            if( p.n_scat >= t->max_scatter ) end = ST_SCATTER_CAP;
            else if( p.w < t->w_min )
            {
                const om_u4 r = om_next( & p.rng );
                if( om_u01( r.x ) < t->rr_survive ) p.w = p.w / t->rr_survive;
                else end = ST_ABSORBED;
            }
            if( ! end )
            {
                om_scatter( t->ph, & p.rng, & p.d, & p.e1, & p.S );
                tset_inv( & p );
                p.tau = tsample_tau( & p.rng );
            }
        }
        else
        {
            p.tau = p.tau - dtau;
            if( pass == 1 && R != 0.0 ) tgadd( g_len, ci, -R * tt, gsc );
            for( int a = 0; a < 3; ++ a )
                if( a != ax ) p.x[ a ] = fma( tt, ( double ) om_comp( p.d, a ), p.x[ a ] );
            int lost;
            const int b_old = p.b;
            if( ! tcross( t, & p.b, p.c, p.x, ax, om_comp( p.d, ax ) > 0.0f, & lost ) )
                end = lost ? ST_LOST : ST_ESCAPED;
            else
                cnt[ 8 ] += p.b != b_old;
        }
        if( ! end && p.n_steps >= t->max_steps ) end = ST_STEP_CAP;
        if( end ) break;
    }
    if( pass == 0 ) * Rp = R;
    return nv;
}

int kpo_adjoint( const kpo_mesh_t * m, const float * sigma2, const int * lookup,
                 const int * lookup_n, const kpo_cfg_t * c, const float * adj_img,
                 int grad_shift, long long * g_len, long long * g_int,
                 unsigned long long * counters )
{
    tctx t;
    if( tsetup( & t, m, sigma2, lookup, lookup_n, c ) ) return -2;
    const double gsc = ldexp( 1.0, grad_shift );
    const int cap = 1 << 16;
    float * Gs = ( float * ) malloc( sizeof( float ) * cap );
    unsigned long long cnt[ 10 ] = { 0, 0, 0, 0, 0, 0, 0, 0, 0, 0 };
    int rc = 0;
    for( long long k = 0; k < c->n_packets && rc == 0; ++ k )
    {
        const long long pid = c->packet_offset + k;
        float G0 = 0.0f;
        double R = 0.0;
        const int n = tadjoint_pass( & t, c, pid, 0, adj_img, & G0, Gs, cap, & R, g_len, g_int,
                                     gsc, cnt );
        if( n < 0 ) { rc = n; break; }
        if( tadjoint_pass( & t, c, pid, 1, adj_img, & G0, Gs, cap, & R, g_len, g_int, gsc,
                           cnt ) < 0 )
            rc = -1;
    }
    if( counters )
        for( int k = 0; k < 10; ++ k ) counters[ k ] += cnt[ k ];
    free( Gs );
    free( t.inv_dx );
    return rc;
}
