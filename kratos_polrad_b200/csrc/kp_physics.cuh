// Device physics of the polarized transport: RNG, portable elementary
// functions, Stokes-frame algebra and phase-matrix sampling.
//
// The reference has no scattering, no polarization and no RNG use on this
// path (its transport is the straight path-length march of
// modules/particle/radiation/photon.h:73-125; device::rand_dev in
// src/device/cuda/cuda.cpp:243-274 is never called).  Everything here is this
// project's own design from published methods:
//   - Philox4x32-10 counter-based RNG (Salmon, Moraes, Dror & Shaw, SC'11,
//     "Parallel random numbers: as easy as 1, 2, 3");
//   - natural log by the atanh series of s = (m-1)/(m+1) after binary
//     range reduction, and exp by Cody-Waite reduction with a Taylor
//     polynomial, both evaluated in double with fused multiply-adds;
//   - the Rayleigh (Thomson) scattering matrix and Stokes rotation of
//     Chandrasekhar, "Radiative Transfer" (1960), with the polarization
//     reference vector carried explicitly so that no trigonometric function
//     is needed;
//   - Henyey & Greenstein (1941) phase function with a Rayleigh-like linear
//     polarization term (White 1979, ApJ 229, 954).
// Every operation is written out in a fixed order with IEEE-rounded
// intrinsics (the file is compiled with --fmad=false), so that the plain-C
// restatement in the oracle reproduces each packet bit for bit.
#pragma once

#include <cstdint>

namespace kp
{
namespace phys
{

////////////////////////////////////////////////////////////
// Philox4x32-10

struct u4 { uint32_t x, y, z, w; };

__device__ __forceinline__ u4 philox( u4 c, uint32_t k0, uint32_t k1 )
{
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    #pragma unroll
    for( int r = 0; r < 10; ++ r )
    {
        if( r > 0 ) { k0 += W0; k1 += W1; }
        const uint32_t lo0 = M0 * c.x, hi0 = __umulhi( M0, c.x );
        const uint32_t lo1 = M1 * c.z, hi1 = __umulhi( M1, c.z );
        c = u4 { hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0 };
    }
    return c;
}

// Per-packet stream: key (seed, stream id), counter (draw, packet id lo/hi,
// tag).  `draw` is the packet's block counter; replaying a packet restarts
// it at zero, so no RNG state is ever stored.
struct rng_t
{
    uint32_t k0, k1, pid_lo, pid_hi, draw;
    __device__ __forceinline__ u4 next(  )
    {
        return philox( u4 { draw ++, pid_lo, pid_hi, 0x4B50u }, k0, k1 );
    }
};

// Uniform in (0,1): (2*(r>>9)+1) * 2^-24, exact in float, never 0 or 1.
__device__ __forceinline__ float u01( uint32_t r )
{
    return __fmul_rn( ( float ) ( ( r >> 9 ) * 2u + 1u ), 0x1p-24f );
}
// Uniform in (-1,1): 2*u01 - 1, exact.
__device__ __forceinline__ float usym( uint32_t r )
{
    return __fsub_rn( __fmul_rn( 2.0f, u01( r ) ), 1.0f );
}

////////////////////////////////////////////////////////////
// Elementary functions (double)

// ln(x) for x > 0 finite.
__device__ __forceinline__ double kp_log( double x )
{
    const long long bits = __double_as_longlong( x );
    int e = ( int ) ( ( bits >> 52 ) & 0x7ff ) - 1023;
    double m = __longlong_as_double( ( bits & 0x000fffffffffffffLL )
                                     | 0x3ff0000000000000LL );     // [1,2)
    if( m > 0x1.6a09e667f3bcdp+0 ) { m = __dmul_rn( m, 0.5 ); e += 1; }
    const double s = __ddiv_rn( __dsub_rn( m, 1.0 ), __dadd_rn( m, 1.0 ) );
    const double z = __dmul_rn( s, s );
    double p = 0x1.af286bca1af28p-4;                  // 2/19
    p = __fma_rn( p, z, 0x1.e1e1e1e1e1e1ep-4 );       // 2/17
    p = __fma_rn( p, z, 0x1.1111111111111p-3 );       // 2/15
    p = __fma_rn( p, z, 0x1.3b13b13b13b14p-3 );       // 2/13
    p = __fma_rn( p, z, 0x1.745d1745d1746p-3 );       // 2/11
    p = __fma_rn( p, z, 0x1.c71c71c71c71cp-3 );       // 2/9
    p = __fma_rn( p, z, 0x1.2492492492492p-2 );       // 2/7
    p = __fma_rn( p, z, 0x1.999999999999ap-2 );       // 2/5
    p = __fma_rn( p, z, 0x1.5555555555555p-1 );       // 2/3
    p = __fma_rn( p, z, 2.0 );
    return __fma_rn( ( double ) e, 0x1.62e42fefa39efp-1, __dmul_rn( s, p ) );
}

// exp(x) for x <= 0 (0 below -700).
__device__ __forceinline__ double kp_exp_neg( double x )
{
    if( x < -700.0 ) return 0.0;
    const double k = rint( __dmul_rn( x, 0x1.71547652b82fep+0 ) );
    double r = __fma_rn( -k, 0x1.62e42fee00000p-1, x );
    r = __fma_rn( -k, 0x1.a39ef35793c76p-33, r );
    double p = 0x1.6124613a86d09p-33;                 // 1/13!
    p = __fma_rn( p, r, 0x1.1eed8eff8d898p-29 );      // 1/12!
    p = __fma_rn( p, r, 0x1.ae64567f544e4p-26 );      // 1/11!
    p = __fma_rn( p, r, 0x1.27e4fb7789f5cp-22 );      // 1/10!
    p = __fma_rn( p, r, 0x1.71de3a556c734p-19 );      // 1/9!
    p = __fma_rn( p, r, 0x1.a01a01a01a01ap-16 );      // 1/8!
    p = __fma_rn( p, r, 0x1.a01a01a01a01ap-13 );      // 1/7!
    p = __fma_rn( p, r, 0x1.6c16c16c16c17p-10 );      // 1/6!
    p = __fma_rn( p, r, 0x1.1111111111111p-7 );       // 1/5!
    p = __fma_rn( p, r, 0x1.5555555555555p-5 );       // 1/4!
    p = __fma_rn( p, r, 0x1.5555555555555p-3 );       // 1/3!
    p = __fma_rn( p, r, 0.5 );                        // 1/2!
    p = __fma_rn( p, r, 1.0 );
    p = __fma_rn( p, r, 1.0 );
    const long long ki = ( long long ) k;
    return __dmul_rn( p, __longlong_as_double( ( ki + 1023 ) << 52 ) );
}

////////////////////////////////////////////////////////////
// Float vector helpers (explicit rounding, fixed order)

struct v3 { float x, y, z; };

__device__ __forceinline__ float dot( const v3 & a, const v3 & b )
{
    return __fadd_rn( __fadd_rn( __fmul_rn( a.x, b.x ), __fmul_rn( a.y, b.y ) ),
                      __fmul_rn( a.z, b.z ) );
}
__device__ __forceinline__ v3 cross( const v3 & a, const v3 & b )
{
    return v3 { __fsub_rn( __fmul_rn( a.y, b.z ), __fmul_rn( a.z, b.y ) ),
                __fsub_rn( __fmul_rn( a.z, b.x ), __fmul_rn( a.x, b.z ) ),
                __fsub_rn( __fmul_rn( a.x, b.y ), __fmul_rn( a.y, b.x ) ) };
}
// a*s + b*t, component-wise
__device__ __forceinline__ v3 lin2( const v3 & a, float s, const v3 & b, float t )
{
    return v3 { __fadd_rn( __fmul_rn( a.x, s ), __fmul_rn( b.x, t ) ),
                __fadd_rn( __fmul_rn( a.y, s ), __fmul_rn( b.y, t ) ),
                __fadd_rn( __fmul_rn( a.z, s ), __fmul_rn( b.z, t ) ) };
}
__device__ __forceinline__ v3 scale( const v3 & a, float s )
{
    return v3 { __fmul_rn( a.x, s ), __fmul_rn( a.y, s ), __fmul_rn( a.z, s ) };
}
__device__ __forceinline__ v3 normalize( const v3 & a )
{
    const float inv = __fdiv_rn( 1.0f, __fsqrt_rn( dot( a, a ) ) );
    return scale( a, inv );
}

// Unit vector perpendicular to d used as the polarization reference of an
// unpolarized packet: normalize(z x d), or normalize(x x d) near the poles.
__device__ __forceinline__ v3 frame_for( const v3 & d )
{
    v3 e;
    if( fabsf( d.z ) < 0.9f ) e = v3 { -d.y, d.x, 0.0f };
    else                      e = v3 { 0.0f, -d.z, d.y };
    return normalize( e );
}

// Direction from cos(theta) = mu and (cos phi, sin phi) about +z.
__device__ __forceinline__ v3 dir_from( float mu, float c, float s )
{
    float t = __fsub_rn( 1.0f, __fmul_rn( mu, mu ) );
    t = t > 0.0f ? t : 0.0f;
    const float st = __fsqrt_rn( t );
    return v3 { __fmul_rn( st, c ), __fmul_rn( st, s ), mu };
}

////////////////////////////////////////////////////////////
// Polarized packet and scattering

// Stokes vector normalized to I = 1 with its reference vector e1 (e1 _|_ d,
// e2 = d x e1; Q = I_e1 - I_e2, U = I_(e1+e2) - I_(e1-e2)).
struct stokes_t { float q, u, v; };

// Phase-matrix parameters: Rayleigh when hg_g == 0 and pol_max == 1.
struct phase_t
{
    int   kind;      // 0 Rayleigh (Thomson), 1 Henyey-Greenstein + Rayleigh-like pol.
    float g;         // HG asymmetry
    float pmax;      // peak linear polarization at 90 degrees (HG kind)
};

// Elements of the scattering matrix at cos(theta) = mu, scaled so that the
// intensity element is f11 and the polarized ones relative to it:
//   I' = f11 * ( 1 + r12 Q ),  Q' = f11 * ( r12 + Q ),  U' = f11 r33 U,
//   V' = f11 r33 V.   (Rayleigh: r12 = (mu^2-1)/(1+mu^2), r33 = 2mu/(1+mu^2).)
struct smat_t { float f11, r12, r33; };

__device__ __forceinline__ smat_t scatter_matrix( const phase_t & ph, float mu )
{
    const float mu2 = __fmul_rn( mu, mu );
    const float a   = __fadd_rn( 1.0f, mu2 );
    smat_t s;
    s.r33 = __fdiv_rn( __fmul_rn( 2.0f, mu ), a );
    if( ph.kind == 0 )
    {   // Rayleigh: f11 = (1+mu^2) * 3/(16 pi) per steradian
        s.f11 = __fmul_rn( a, 0x1.e8ec8ap-5f );
        s.r12 = __fdiv_rn( __fsub_rn( mu2, 1.0f ), a );
    }
    else
    {   // HG: (1-g^2) / (4 pi (1 + g^2 - 2 g mu)^1.5)
        const float g2 = __fmul_rn( ph.g, ph.g );
        const float den = __fsub_rn( __fadd_rn( 1.0f, g2 ),
                                     __fmul_rn( __fmul_rn( 2.0f, ph.g ), mu ) );
        const float sd = __fsqrt_rn( den );
        s.f11 = __fdiv_rn( __fmul_rn( __fsub_rn( 1.0f, g2 ), 0x1.45f306p-4f ),
                           __fmul_rn( den, sd ) );
        s.r12 = __fmul_rn( -ph.pmax, __fdiv_rn( __fsub_rn( 1.0f, mu2 ), a ) );
    }
    return s;
}

// Frame rotation: e1' = cos(psi) e1 + sin(psi) e2 given cos 2psi, sin 2psi.
__device__ __forceinline__ void rotate( float & q, float & u, float c2, float s2 )
{
    const float qn = __fadd_rn( __fmul_rn( q, c2 ), __fmul_rn( u, s2 ) );
    const float un = __fsub_rn( __fmul_rn( u, c2 ), __fmul_rn( q, s2 ) );
    q = qn;
    u = un;
}

// cos 2psi, sin 2psi of the angle whose (unnormalized) cosine and sine are
// (c, s); (1, 0) when the angle is undefined.
__device__ __forceinline__ void double_angle( float c, float s, float & c2, float & s2 )
{
    const float cc = __fmul_rn( c, c ), ss = __fmul_rn( s, s );
    const float n2 = __fadd_rn( cc, ss );
    if( n2 > 1e-12f )
    {
        const float inv = __fdiv_rn( 1.0f, n2 );
        c2 = __fmul_rn( __fsub_rn( cc, ss ), inv );
        s2 = __fmul_rn( __fmul_rn( __fmul_rn( 2.0f, c ), s ), inv );
    }
    else { c2 = 1.0f; s2 = 0.0f; }
}

// Henyey-Greenstein cos(theta) by inversion of its distribution.
__device__ __forceinline__ float hg_mu( float g, float xi )
{
    if( fabsf( g ) < 1e-3f )
        return __fsub_rn( __fmul_rn( 2.0f, xi ), 1.0f );
    const float g2 = __fmul_rn( g, g );
    const float t  = __fdiv_rn( __fsub_rn( 1.0f, g2 ),
                                __fadd_rn( __fsub_rn( 1.0f, g ),
                                           __fmul_rn( __fmul_rn( 2.0f, g ), xi ) ) );
    float mu = __fdiv_rn( __fsub_rn( __fadd_rn( 1.0f, g2 ), __fmul_rn( t, t ) ),
                          __fmul_rn( 2.0f, g ) );
    mu = mu > 1.0f ? 1.0f : ( mu < -1.0f ? -1.0f : mu );
    return mu;
}

// Samples a scattering event and updates direction, frame and Stokes vector.
// (mu, phi) are drawn jointly from the scattered intensity
// f11(mu) (1 + r12(mu) Q'(phi)) with Q' = q cos 2phi + u sin 2phi (phi from
// e1 toward e2), by rejection against a bound independent of (mu, phi):
// Rayleigh proposes mu uniform and accepts with (1+mu^2 + (mu^2-1) Q') / 2,
// HG proposes mu from HG and accepts with (1 + r12 Q') / (1 + pmax).
// (cos phi, sin phi) come from a point uniform in the unit disk.  At most 64
// proposals; the last one is kept if all are rejected.
__device__ __forceinline__ void scatter( const phase_t & ph, rng_t & rng, v3 & d,
                                         v3 & e1, stokes_t & S )
{
    float mu = 0.0f, a = 1.0f, b = 0.0f, r2 = 1.0f, c2 = 1.0f, s2 = 0.0f, qp = S.q;
    for( int trial = 0; trial < 64; ++ trial )
    {
        const u4 r = rng.next(  );
        mu = ph.kind == 0 ? usym( r.x ) : hg_mu( ph.g, u01( r.x ) );
        a  = usym( r.y );
        b  = usym( r.z );
        r2 = __fadd_rn( __fmul_rn( a, a ), __fmul_rn( b, b ) );
        if( r2 > 1.0f || r2 == 0.0f )
        {
            a = 1.0f; b = 0.0f; r2 = 1.0f;
            continue;
        }
        double_angle( a, b, c2, s2 );
        qp = __fadd_rn( __fmul_rn( S.q, c2 ), __fmul_rn( S.u, s2 ) );
        const float mu2 = __fmul_rn( mu, mu );
        if( ph.kind == 0 )
        {
            const float f = __fadd_rn( __fadd_rn( 1.0f, mu2 ),
                                       __fmul_rn( __fsub_rn( mu2, 1.0f ), qp ) );
            if( __fmul_rn( 2.0f, u01( r.w ) ) < f ) break;
        }
        else
        {
            const float r12 = __fmul_rn( -ph.pmax, __fdiv_rn( __fsub_rn( 1.0f, mu2 ),
                                                              __fadd_rn( 1.0f, mu2 ) ) );
            const float f = __fadd_rn( 1.0f, __fmul_rn( r12, qp ) );
            if( __fmul_rn( u01( r.w ), __fadd_rn( 1.0f, ph.pmax ) ) < f ) break;
        }
    }
    // Stokes: rotate into the scattering plane, apply the matrix, normalize.
    double_angle( a, b, c2, s2 );
    float q = S.q, u = S.u;
    rotate( q, u, c2, s2 );
    const smat_t sm = scatter_matrix( ph, mu );
    const float I  = __fadd_rn( 1.0f, __fmul_rn( sm.r12, q ) );
    const float Q  = __fadd_rn( sm.r12, q );
    const float U  = __fmul_rn( sm.r33, u );
    const float V  = __fmul_rn( sm.r33, S.v );
    const float iI = __fdiv_rn( 1.0f, I );
    S.q = __fmul_rn( Q, iI );
    S.u = __fmul_rn( U, iI );
    S.v = __fmul_rn( V, iI );
    // Geometry: n = cos phi e1 + sin phi e2; d' = mu d + st n; e1' = mu n - st d.
    const float rr = __fsqrt_rn( r2 );
    const float cp = __fdiv_rn( a, rr ), sp = __fdiv_rn( b, rr );
    const v3 e2 = cross( d, e1 );
    const v3 n  = lin2( e1, cp, e2, sp );
    float t = __fsub_rn( 1.0f, __fmul_rn( mu, mu ) );
    t = t > 0.0f ? t : 0.0f;
    const float st = __fsqrt_rn( t );
    v3 dn = normalize( lin2( d, mu, n, st ) );
    v3 en = lin2( n, mu, d, -st );
    en = normalize( lin2( en, 1.0f, dn, -dot( en, dn ) ) );
    d  = dn;
    e1 = en;
}

// Peel-off toward the observer direction o with image frame (ev, eh = ev x o):
// returns the intensity per steradian (times the packet's I = 1) and the
// Stokes (Q, U, V) in the image frame (Q > 0 along ev).
__device__ __forceinline__ float peel_stokes( const phase_t & ph, const v3 & d,
                                              const v3 & e1, const stokes_t & S,
                                              const v3 & o, const v3 & ev,
                                              const v3 & eh, float & Qo,
                                              float & Uo, float & Vo )
{
    const float mu = dot( d, o );
    const v3 e2 = cross( d, e1 );
    float c2, s2;
    double_angle( dot( o, e1 ), dot( o, e2 ), c2, s2 );
    float q = S.q, u = S.u;
    rotate( q, u, c2, s2 );
    const smat_t sm = scatter_matrix( ph, mu );
    const float I = __fadd_rn( 1.0f, __fmul_rn( sm.r12, q ) );
    float Q = __fadd_rn( sm.r12, q );
    float U = __fmul_rn( sm.r33, u );
    const float V = __fmul_rn( sm.r33, S.v );
    // outgoing frame e1' = (mu o - d)/s; to the image frame ev:
    // cos psi = -(ev.d)/s, sin psi = -(eh.d)/s
    double_angle( dot( ev, d ), dot( eh, d ), c2, s2 );
    rotate( Q, U, c2, s2 );
    const float f = __fmul_rn( sm.f11, 1.0f );
    Qo = __fmul_rn( f, Q );
    Uo = __fmul_rn( f, U );
    Vo = __fmul_rn( f, V );
    return __fmul_rn( f, I );
}

}   // namespace phys
}   // namespace kp
