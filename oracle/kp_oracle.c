/* Oracle: plain-C restatement of the transport path (test infrastructure;
 * see kp_oracle.h).  Compiled with -ffp-contract=off so that every float
 * operation rounds once, as the reference does on the host. */
#include "kp_oracle.h"

#include <float.h>
#include <math.h>
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
static void gl_fix_##S( const kpo_mesh_t * m, int b, const int * i,              \
                        const F * x, F * xl, F * xr )                            \
{   /* geo_loc_t::fix (particle_base.h:117-126): the cell index is left as is */ \
    for( int a = 0; a < 3; ++ a )                                                \
        if( x[ a ] > xr[ a ] )      gl_shift_##S( m, b, i, xl, xr, a, 1 );       \
        else if( x[ a ] < xl[ a ] ) gl_shift_##S( m, b, i, xl, xr, a, 0 );       \
}                                                                                \
static void walk_##S( const kpo_mesh_t * m, F * x, const F * dir, int * i,       \
                      int * ibp, F proper, int * stepp, int * todop,             \
                      double scale, double * flux_f, long long * flux_fx )       \
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
            gl_fix_##S( m, ib, i, x, xl, xr );                                   \
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
            gl_fix_##S( m, ib, i, x, xl, xr );                                   \
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
    const double scale = ldexp( 1.0, fx_shift );
    for( long p = 0; p < n; ++ p )
    {
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
                      todo + p, scale, flux_f, flux_fx );
            for( int a = 0; a < 3; ++ a ) x[ 3 * p + a ] = xf[ a ];
        }
        else
            walk_f64( m, x + 3 * p, dir + 3 * p, cell + 3 * p, ib + p, proper[ p ],
                      step + p, todo + p, scale, flux_f, flux_fx );
    }
    return 0;
}
