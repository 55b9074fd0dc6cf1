/* Oracle physics primitives (plain C restatement; test infrastructure).
 *
 * Same published methods and operation order as the device code, written
 * independently: Philox4x32-10 (Salmon et al., SC'11), ln by the atanh
 * series after binary range reduction, exp by Cody-Waite reduction and a
 * Taylor polynomial, the Rayleigh matrix and Stokes rotation of
 * Chandrasekhar (1960), Henyey-Greenstein (1941) with a Rayleigh-like
 * polarization term.  No reference code exists for these parts (the
 * reference's transport is the straight march of radiation/photon.h:73-125
 * and never calls its RNG, device/cuda/cuda.cpp:243-274).  Compiled with
 * -ffp-contract=off: each float/double operation rounds once; fma() is the
 * correctly rounded fused multiply-add.
 */
#ifndef KP_ORACLE_MATH_H
#define KP_ORACLE_MATH_H

#include <math.h>
#include <stdint.h>
#include <string.h>

/* Physical constants in the arithmetic type of the build (float here; the
 * FP64 build of the restatement, kp_oracle64.c, gives double values). */
#ifndef OM_INV4PI
#define OM_INV4PI 0x1.45f306p-4f          /* 1 / (4 pi)  */
#endif
#ifndef OM_3_16PI
#define OM_3_16PI 0x1.e8ec8ap-5f          /* 3 / (16 pi) */
#endif

typedef struct { uint32_t x, y, z, w; } om_u4;

static inline uint32_t om_mulhi( uint32_t a, uint32_t b )
{
    return ( uint32_t ) ( ( ( uint64_t ) a * b ) >> 32 );
}

static inline om_u4 om_philox( om_u4 c, uint32_t k0, uint32_t k1 )
{
    for( int r = 0; r < 10; ++ r )
    {
        if( r > 0 ) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        const uint32_t lo0 = 0xD2511F53u * c.x, hi0 = om_mulhi( 0xD2511F53u, c.x );
        const uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = om_mulhi( 0xCD9E8D57u, c.z );
        om_u4 n = { hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0 };
        c = n;
    }
    return c;
}

typedef struct { uint32_t k0, k1, pid_lo, pid_hi, draw; } om_rng;

static inline om_u4 om_next( om_rng * g )
{
    om_u4 c = { g->draw ++, g->pid_lo, g->pid_hi, 0x4B50u };
    return om_philox( c, g->k0, g->k1 );
}

static inline float om_u01( uint32_t r )
{
    return ( float ) ( ( r >> 9 ) * 2u + 1u ) * 0x1p-24f;
}
static inline float om_usym( uint32_t r ) { return 2.0f * om_u01( r ) - 1.0f; }

static inline double om_log( double x )
{
    int64_t bits;
    memcpy( & bits, & x, 8 );
    int e = ( int ) ( ( bits >> 52 ) & 0x7ff ) - 1023;
    int64_t mb = ( bits & 0x000fffffffffffffLL ) | 0x3ff0000000000000LL;
    double m;
    memcpy( & m, & mb, 8 );
    if( m > 0x1.6a09e667f3bcdp+0 ) { m = m * 0.5; e += 1; }
    const double s = ( m - 1.0 ) / ( m + 1.0 );
    const double z = s * s;
    double p = 0x1.af286bca1af28p-4;                  /* 2/19 */
    p = fma( p, z, 0x1.e1e1e1e1e1e1ep-4 );            /* 2/17 */
    p = fma( p, z, 0x1.1111111111111p-3 );            /* 2/15 */
    p = fma( p, z, 0x1.3b13b13b13b14p-3 );            /* 2/13 */
    p = fma( p, z, 0x1.745d1745d1746p-3 );
    p = fma( p, z, 0x1.c71c71c71c71cp-3 );
    p = fma( p, z, 0x1.2492492492492p-2 );
    p = fma( p, z, 0x1.999999999999ap-2 );
    p = fma( p, z, 0x1.5555555555555p-1 );
    p = fma( p, z, 2.0 );
    return fma( ( double ) e, 0x1.62e42fefa39efp-1, s * p );
}

static inline double om_exp_neg( double x )
{
    if( x < -700.0 ) return 0.0;
    const double k = rint( x * 0x1.71547652b82fep+0 );
    double r = fma( -k, 0x1.62e42fee00000p-1, x );
    r = fma( -k, 0x1.a39ef35793c76p-33, r );
    static const double c[ 14 ] = { 1.0, 1.0, 0.5, 0x1.5555555555555p-3,
        0x1.5555555555555p-5, 0x1.1111111111111p-7, 0x1.6c16c16c16c17p-10,
        0x1.a01a01a01a01ap-13, 0x1.a01a01a01a01ap-16, 0x1.71de3a556c734p-19,
        0x1.27e4fb7789f5cp-22, 0x1.ae64567f544e4p-26, 0x1.1eed8eff8d898p-29,
        0x1.6124613a86d09p-33 };
    double p = c[ 13 ];
    for( int n = 12; n >= 0; -- n ) p = fma( p, r, c[ n ] );
    const int64_t sb = ( ( int64_t ) k + 1023 ) << 52;
    double sc;
    memcpy( & sc, & sb, 8 );
    return p * sc;
}

typedef struct { float x, y, z; } om_v3;

static inline float om_dot( om_v3 a, om_v3 b ) { return ( a.x * b.x + a.y * b.y ) + a.z * b.z; }
static inline om_v3 om_cross( om_v3 a, om_v3 b )
{
    om_v3 r = { a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x };
    return r;
}
static inline om_v3 om_lin2( om_v3 a, float s, om_v3 b, float t )
{
    om_v3 r = { a.x * s + b.x * t, a.y * s + b.y * t, a.z * s + b.z * t };
    return r;
}
static inline om_v3 om_scale( om_v3 a, float s ) { om_v3 r = { a.x * s, a.y * s, a.z * s }; return r; }
static inline om_v3 om_normalize( om_v3 a ) { return om_scale( a, 1.0f / sqrtf( om_dot( a, a ) ) ); }
static inline float om_comp( om_v3 v, int a ) { return a == 0 ? v.x : ( a == 1 ? v.y : v.z ); }

static inline om_v3 om_frame_for( om_v3 d )
{
    om_v3 e;
    if( fabsf( d.z ) < 0.9f ) { e.x = -d.y; e.y = d.x; e.z = 0.0f; }
    else                      { e.x = 0.0f; e.y = -d.z; e.z = d.y; }
    return om_normalize( e );
}

static inline om_v3 om_dir_from( float mu, float c, float s )
{
    float t = 1.0f - mu * mu;
    t = t > 0.0f ? t : 0.0f;
    const float st = sqrtf( t );
    om_v3 r = { st * c, st * s, mu };
    return r;
}

typedef struct { float q, u, v; } om_stokes;
typedef struct { int kind; float g, pmax; } om_phase;
typedef struct { float f11, r12, r33; } om_smat;

static inline om_smat om_scatter_matrix( om_phase ph, float mu )
{
    const float mu2 = mu * mu, a = 1.0f + mu2;
    om_smat s;
    s.r33 = ( 2.0f * mu ) / a;
    if( ph.kind == 0 )
    {
        s.f11 = a * OM_3_16PI;
        s.r12 = ( mu2 - 1.0f ) / a;
    }
    else
    {
        const float g2 = ph.g * ph.g;
        const float den = ( 1.0f + g2 ) - ( 2.0f * ph.g ) * mu;
        const float sd = sqrtf( den );
        s.f11 = ( ( 1.0f - g2 ) * OM_INV4PI ) / ( den * sd );
        s.r12 = -ph.pmax * ( ( 1.0f - mu2 ) / a );
    }
    return s;
}

static inline void om_rotate( float * q, float * u, float c2, float s2 )
{
    const float qn = * q * c2 + * u * s2;
    const float un = * u * c2 - * q * s2;
    * q = qn;
    * u = un;
}

static inline void om_double_angle( float c, float s, float * c2, float * s2 )
{
    const float cc = c * c, ss = s * s, n2 = cc + ss;
    if( n2 > 1e-12f )
    {
        const float inv = 1.0f / n2;
        * c2 = ( cc - ss ) * inv;
        * s2 = ( ( 2.0f * c ) * s ) * inv;
    }
    else { * c2 = 1.0f; * s2 = 0.0f; }
}

static inline float om_hg_mu( float g, float xi )
{
    if( fabsf( g ) < 1e-3f ) return 2.0f * xi - 1.0f;
    const float g2 = g * g;
    const float t = ( 1.0f - g2 ) / ( ( 1.0f - g ) + ( 2.0f * g ) * xi );
    float mu = ( ( 1.0f + g2 ) - t * t ) / ( 2.0f * g );
    return mu > 1.0f ? 1.0f : ( mu < -1.0f ? -1.0f : mu );
}

static inline void om_scatter( om_phase ph, om_rng * rng, om_v3 * d, om_v3 * e1, om_stokes * S )
{
    float mu = 0.0f, a = 1.0f, b = 0.0f, r2 = 1.0f, c2 = 1.0f, s2 = 0.0f, qp = S->q;
    for( int trial = 0; trial < 64; ++ trial )
    {
        const om_u4 r = om_next( rng );
        mu = ph.kind == 0 ? om_usym( r.x ) : om_hg_mu( ph.g, om_u01( r.x ) );
        a = om_usym( r.y );
        b = om_usym( r.z );
        r2 = a * a + b * b;
        if( r2 > 1.0f || r2 == 0.0f ) { a = 1.0f; b = 0.0f; r2 = 1.0f; continue; }
        om_double_angle( a, b, & c2, & s2 );
        qp = S->q * c2 + S->u * s2;
        const float mu2 = mu * mu;
        if( ph.kind == 0 )
        {
            const float f = ( 1.0f + mu2 ) + ( mu2 - 1.0f ) * qp;
            if( 2.0f * om_u01( r.w ) < f ) break;
        }
        else
        {
            const float r12 = -ph.pmax * ( ( 1.0f - mu2 ) / ( 1.0f + mu2 ) );
            const float f = 1.0f + r12 * qp;
            if( om_u01( r.w ) * ( 1.0f + ph.pmax ) < f ) break;
        }
    }
    om_double_angle( a, b, & c2, & s2 );
    float q = S->q, u = S->u;
    om_rotate( & q, & u, c2, s2 );
    const om_smat sm = om_scatter_matrix( ph, mu );
    const float I = 1.0f + sm.r12 * q;
    const float Q = sm.r12 + q;
    const float U = sm.r33 * u;
    const float V = sm.r33 * S->v;
    const float iI = 1.0f / I;
    S->q = Q * iI;
    S->u = U * iI;
    S->v = V * iI;
    const float rr = sqrtf( r2 );
    const float cp = a / rr, sp = b / rr;
    const om_v3 e2 = om_cross( * d, * e1 );
    const om_v3 n = om_lin2( * e1, cp, e2, sp );
    float t = 1.0f - mu * mu;
    t = t > 0.0f ? t : 0.0f;
    const float st = sqrtf( t );
    const om_v3 dn = om_normalize( om_lin2( * d, mu, n, st ) );
    om_v3 en = om_lin2( n, mu, * d, -st );
    en = om_normalize( om_lin2( en, 1.0f, dn, -om_dot( en, dn ) ) );
    * d = dn;
    * e1 = en;
}

static inline float om_peel_stokes( om_phase ph, om_v3 d, om_v3 e1, om_stokes S, om_v3 o,
                                    om_v3 ev, om_v3 eh, float * Qo, float * Uo, float * Vo )
{
    const float mu = om_dot( d, o );
    const om_v3 e2 = om_cross( d, e1 );
    float c2, s2;
    om_double_angle( om_dot( o, e1 ), om_dot( o, e2 ), & c2, & s2 );
    float q = S.q, u = S.u;
    om_rotate( & q, & u, c2, s2 );
    const om_smat sm = om_scatter_matrix( ph, mu );
    const float I = 1.0f + sm.r12 * q;
    float Q = sm.r12 + q;
    float U = sm.r33 * u;
    const float V = sm.r33 * S.v;
    om_double_angle( om_dot( ev, d ), om_dot( eh, d ), & c2, & s2 );
    om_rotate( & Q, & U, c2, s2 );
    const float f = sm.f11 * 1.0f;
    * Qo = f * Q;
    * Uo = f * U;
    * Vo = f * V;
    return f * I;
}

#endif
