/* Oracle: plain-C restatement of the transport path (test infrastructure).
 *
 * Only the tests, the smoke check and the bench's CPU-baseline leg use this
 * library (oracle/_ref/libkporacle.so); the product never links it.
 *
 * Geometric walk: restates photon::cart_t::proc and what it calls
 * (reference files modules/particle/radiation/photon.h:20-125,
 * types/particle_base.h:37-56,86-126, types/proxy.h:64-121,
 * mesh/geometry/geometry.h:206-256) over flat block tables, in float
 * (PRECISION=1) or double (PRECISION=2) arithmetic with the reference's
 * operation order.  Pinned bit-for-bit against the reference's own code
 * compiled on the host (oracle/ref_harness.cpp).
 */
#ifndef KP_ORACLE_H
#define KP_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Flat mesh tables, block-id order (see kp_mesh_geometry/_neighbors). */
typedef struct kpo_mesh
{
    int            n_blocks;
    int            nc[ 3 ];
    const double * xf0;       /* [nb][3] (float_t values widened)   */
    const double * dx0;       /* [nb][3]                             */
    const double * vol0;      /* [nb]                                */
    const int    * phybnd;    /* [nb][6]                             */
    const int    * nb_id;     /* [nb][24] slot ((a*2+s)*2+j0)*2+j1   */
    const int    * nb_shift;  /* [nb][48]                            */
    const int    * d_lvl;     /* [nb][6]                             */
    int            periodic[ 3 ];
    double         xlim[ 2 ][ 3 ];
    double         lbox[ 3 ];
} kpo_mesh_t;

/* Walks n packets in place (x, dir: 3n; cell: 3n; ib, step, todo: n).
 * precision 4: float_t = float, 8: double.  Deposits go to flux_f (float_t
 * sums in packet order, widened) and flux_fx (int64 round(v*2^fx_shift)),
 * both [n_blocks * cells_per_block]. */
int kpo_trace( const kpo_mesh_t * m, int precision, long n, double * x,
               const double * dir, int * cell, int * ib, const double * proper,
               int * step, int * todo, int fx_shift, double * flux_f,
               long long * flux_fx );
/* Same walk; fix_shifts[n] (may be null) adds, per packet, the number of
 * axes on which geo_loc_t::fix shifted the cached cell faces without moving
 * the cell index (particle_base.h:117-126).  A packet with none walks the
 * cells its position crosses; one with some deposits into cells other than
 * the ones it crosses, and on a collapsed axis no longer stops at faces. */
int kpo_trace_ex( const kpo_mesh_t * m, int precision, long n, double * x,
                  const double * dir, int * cell, int * ib, const double * proper,
                  int * step, int * todo, int fx_shift, double * flux_f,
                  long long * flux_fx, int * fix_shifts );

#ifdef __cplusplus
}
#endif

#endif

/* ---------------------------------------------------------------------- */
/* Polarized transport restatement (same algorithm and operation order as  */
/* the device kernels; sequential packets; int64 fixed-point tallies).    */
#ifndef KPO_TRANSPORT_DECLS
#define KPO_TRANSPORT_DECLS
#ifdef __cplusplus
extern "C" {
#endif

typedef struct kpo_source
{
    int    kind, emit;      /* 0 point / 1 plane at the lower z face; 0 iso / 1 up */
    double pos[ 3 ];
    int    ib;              /* block and cell of a point source              */
    int    cell[ 3 ];
} kpo_source_t;

/* A caller-made packet (the layout of kp_packet_init_t). */
typedef struct kpo_packet_init
{
    double x[ 3 ];
    float  d[ 3 ];
    float  w;
    float  stokes[ 3 ];
    int    ib;
    float  peel_I;
    int    pad;
} kpo_packet_init_t;

typedef struct kpo_cfg
{
    long long n_packets, packet_offset;
    uint32_t  seed, stream_id;
    int       phase;
    float     hg_g, pol_max;
    int       n_sources;
    const kpo_source_t * sources;
    int       n_mu_bins;
    float     mu_lo, mu_hi;
    int       image_n;
    double    inclination_deg, azimuth_deg;
    double    image_center[ 3 ];
    double    image_half_width;
    float     tau_peel_max;
    int       fx_shift;
    int       n_batches;
    int       image_batch_n;
    float     w_min, rr_survive;
    int       max_scatter;
    long long max_steps;
    long long n_record;
    int       flux_fx_shift;    /* flux tally scale 2^flux_fx_shift (0: fx_shift) */
    const kpo_packet_init_t * packets;  /* [n_packets] or NULL: the sources */
} kpo_cfg_t;

typedef struct kpo_record
{
    double    x[ 3 ];
    float     d[ 3 ];
    float     stokes[ 3 ];
    float     w;
    int       ib;
    int       cell[ 3 ];
    int       n_scatter;
    int       status;
    uint32_t  rng_draws;
    long long n_steps;
} kpo_record_t;

/* sigma2: [n_cells][2] (sca, abs); lookup: finest-level leaf ids.
 * Outputs are accumulated into (int64 fixed point); flux ([n_cells], may be
 * null) receives the path-length estimator w * dl / volume of every walk
 * segment. */
int kpo_transport( const kpo_mesh_t * m, const float * sigma2, const int * lookup,
                   const int * lookup_n, const kpo_cfg_t * c, long long * mu,
                   long long * image, long long * img_batch,
                   unsigned long long * counters, kpo_record_t * rec, long long * flux );

#ifdef __cplusplus
}
#endif
#endif

#ifndef KPO_ADJOINT_DECLS
#define KPO_ADJOINT_DECLS
#ifdef __cplusplus
extern "C" {
#endif
/* Path-replay adjoint of the peel-off image: adj_img [image_n][image_n][4]
 * float is dL/dimage; accumulates int64 round(v * 2^grad_shift) of the
 * path-length term into g_len and of the interaction term into g_int
 * (dL/dsigma_sca = g_len + g_int, dL/dsigma_abs = g_len). */
int kpo_adjoint( const kpo_mesh_t * m, const float * sigma2, const int * lookup,
                 const int * lookup_n, const kpo_cfg_t * c, const float * adj_img,
                 int grad_shift, long long * g_len, long long * g_int,
                 unsigned long long * counters );
/* While non-null, every adjoint deposit of value v into cell i also adds
 * |v| to sink[2 i] and 1 to sink[2 i + 1] (2 n_cells doubles); NULL switches
 * it off. */
void kpo_set_abs_sink( double * sink );
/* While n is non-null, every image deposit of kpo_transport is recorded:
 * pix[k] = its pixel, val[4 k .. 4 k + 3] = its (I, Q, U, V), for the first
 * `cap` deposits; *n counts all of them.  n = NULL switches it off. */
void kpo_set_pixel_sink( int * pix, float * val, long long cap, long long * n );
#ifdef __cplusplus
}
#endif
#endif
