/* kratos_polrad_b200 — C ABI of the B200 photon-packet transport path.
 *
 * Plain C: pointers, sizes and POD structs; no C++ or torch types.  Every
 * entry point returns an int status (KP_OK = 0); kp_last_error() gives the
 * calling thread's last message.  "device pointer" arguments are CUDA
 * global-memory addresses on the current device; "host pointer" arguments
 * are ordinary (pageable or pinned) host memory.  Streams and events are
 * passed as opaque `void *` holding a cudaStream_t / cudaEvent_t (NULL is
 * the legacy default stream).
 *
 * Each declaration names the reference interface it replaces
 * (paths relative to the reference project's tree).
 */
#ifndef KP_TRANSPORT_H
#define KP_TRANSPORT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KP_ABI_VERSION 2

enum kp_status
{
    KP_OK           = 0,
    KP_ERR_ARG      = 1,   /* invalid argument                         */
    KP_ERR_CUDA     = 2,   /* CUDA runtime error                        */
    KP_ERR_CONFIG   = 3,   /* bad mesh / transport configuration        */
    KP_ERR_CAPACITY = 4,   /* a size exceeds a documented maximum       */
    KP_ERR_DEVICE   = 5,   /* a kernel reported an error status word    */
    KP_ERR_ALLOC    = 6    /* allocation refused                        */
};

/* Message of the calling thread's last failed call ("" if none). */
const char * kp_last_error( void );
int          kp_abi_version( void );

/* ------------------------------------------------------------------ */
/* Device layer.  Replaces device::base_t's function objects and       */
/* virtuals (src/device/device.h:37-50,66-186) and their CUDA backend   */
/* (src/device/cuda/cuda.cpp:31-130,164-176).                           */

int kp_device_init( int idx_device );            /* cuda_t::init, cuda.cpp:108-130          */
int kp_device_count( int * n );
int kp_malloc( void ** p, size_t bytes );        /* f_malloc, device.h:37-50                */
int kp_malloc_host( void ** p, size_t bytes );   /* f_malloc_host (pinned), cuda.cpp:39-44  */
int kp_free( void * p );                         /* f_free                                  */
int kp_free_host( void * p );                    /* f_free_host                             */
int kp_memset_async( void * p, int value, size_t bytes, void * stream );  /* f_mset      */
int kp_memcpy( void * dst, const void * src, size_t bytes );              /* f_cp        */
int kp_memcpy_async( void * dst, const void * src, size_t bytes,
                     void * stream );                                     /* a_cp        */
int kp_stream_create( void ** stream );          /* yield_stream, cuda.cpp:164-176          */
int kp_stream_destroy( void * stream );
int kp_stream_sync( void * stream );             /* sync_stream, device.cpp:124-151         */
int kp_event_create( void ** event );            /* event_create                            */
int kp_event_destroy( void * event );            /* event_destroy                           */
int kp_event_record( void * event, void * stream );   /* event_record                       */
int kp_event_wait( void * stream, void * event );     /* event_wait                         */
int kp_event_sync( void * event );                    /* event_sync                         */
int kp_event_elapsed( float * ms, void * start, void * stop );
/* f_launch_host (device.cpp:101-119), without the reference's shared
 * static callback vector: each call carries its own (fn, arg). */
int kp_launch_host( void * stream, void ( * fn )( void * ), void * arg );

/* ------------------------------------------------------------------ */
/* Mesh.  Replaces meshgen::base_t (mesh/meshgen/meshgen.cpp:13-163,    */
/* 286-432), tree_t (mesh/tree/tree.cpp:177-230) and the proxy table    */
/* of particle::block_map_t (modules/particle/types/block_map.h:53-103, */
/* types/proxy.h:22-62).  Building a mesh needs no GPU; the tables are  */
/* copied to the current device on first use or by kp_mesh_upload.     */

typedef struct kp_mesh kp_mesh_t;

typedef struct kp_refine_box
{
    int    level;          /* [refine_region*] level                   */
    double x_min[ 3 ];     /* [refine_region*] x_min (or loc)           */
    double x_max[ 3 ];     /* [refine_region*] x_max                    */
} kp_refine_box_t;

typedef struct kp_mesh_desc
{
    double x_min[ 3 ];            /* [mesh] x_min                       */
    double x_max[ 3 ];            /* [mesh] x_max                       */
    int    n_cell_global[ 3 ];    /* [mesh] n_cell_global               */
    int    n_cell_block[ 3 ];     /* [mesh] n_cell_block                */
    int    periodic[ 3 ];         /* [boundary] kinds "per..." per axis */
    int    n_refine;
    const kp_refine_box_t * refine;
} kp_mesh_desc_t;

typedef struct kp_mesh_info
{
    int       n_blocks;
    int       n_cell_block[ 3 ];
    int       cells_per_block;
    int       max_level;
    long long n_cells;
    int       periodic[ 3 ];
    double    x_min[ 3 ];
    double    x_max[ 3 ];
} kp_mesh_info_t;

int kp_mesh_create( const kp_mesh_desc_t * desc, kp_mesh_t ** mesh );
/* Same, from an INI file with the reference's [mesh], [boundary] and
 * [refine_region*] keys (io/args/input.cpp:72-108). */
int kp_mesh_create_ini( const char * path, kp_mesh_t ** mesh );
int kp_mesh_destroy( kp_mesh_t * mesh );
int kp_mesh_info( const kp_mesh_t * mesh, kp_mesh_info_t * info );
/* Region key (level, logical block index) per block id; host arrays of
 * n_blocks and 3*n_blocks ints. */
int kp_mesh_blocks( const kp_mesh_t * mesh, int * level, int * reg3 );
/* Block geometry as the reference's geo_t holds it for float_t of
 * `precision` bytes (4 or 8), widened to double: face origin xf0[3],
 * spacing dx0[3], cell volume vol0, physical-boundary flags [6]. */
int kp_mesh_geometry( const kp_mesh_t * mesh, int precision, double * xf0,
                      double * dx0, double * vol0, int * phybnd );
/* Face-neighbour table per block, slot (((a*2+side)*2+j0)*2+j1):
 * ids [24], shift bits [48] (two per slot) and level deltas [6], with
 * proxy_base_t's layout (types/proxy.h:13-19). */
int kp_mesh_neighbors( const kp_mesh_t * mesh, int * nb_id, int * nb_shift,
                       int * d_lvl );
/* Host point location: block id and cell index of each of n points
 * (x: host, 3n doubles).  Points outside the domain get ib = -1. */
int kp_mesh_locate( const kp_mesh_t * mesh, long long n, const double * x,
                    int * ib, int * cell3 );
/* Copies the tables to the current device (idempotent). */
int kp_mesh_upload( kp_mesh_t * mesh );
/* Per-cell coefficients (sigma_sca, sigma_abs) as 2*n_cells floats in
 * block-id order, x-fastest within a block.  `src` is a host pointer, or a
 * device pointer when on_device != 0.  Replaces the per-block rad_t
 * inverse-mean-free-path field (modules/particle/radiation/rad_data.cpp:
 * 13-25). */
int kp_mesh_set_sigma( kp_mesh_t * mesh, const float * src, long long n_values,
                       int on_device, void * stream );
/* Device pointer of the mesh's coefficient array (2*n_cells floats). */
int kp_mesh_sigma_ptr( kp_mesh_t * mesh, float ** sigma );
/* Synchronizes `stream`, returns and clears the mesh's device error status
 * bits (out-of-range block or cell index, queue overflow, bad source); a
 * kernel that sets one skips the offending access instead of faulting.
 * Replaces the reference's debug flag (src/device/device.cpp:12-22,124-151). */
int kp_mesh_status( kp_mesh_t * mesh, void * stream, unsigned * flags );

/* ------------------------------------------------------------------ */
/* Spherical-polar meshes (axes r, theta, phi): meshgen::sph_t on       */
/* cyl_t's radial spacing (mesh/meshgen/spherical.h, cylindrical.h),    */
/* same tree and neighbour tables.  r_ratio as [mesh] r_ratio: 1 for    */
/* uniform radial cells, a ratio of successive radial widths, or < 0   */
/* for the ratio (r_max / r_min)^(1/n_r).                               */
int kp_mesh_create_sph( const kp_mesh_desc_t * desc, double r_ratio, kp_mesh_t ** mesh );
/* Same from an INI file ([mesh] r_ratio read as cyl_t::read does). */
int kp_mesh_create_sph_ini( const char * path, kp_mesh_t ** mesh );
/* Radial faces [n_blocks][nc0 + 1] (the block's dx0[0] is -1 when they are
 * not uniform) and cell volumes [n_cells], as geo_t holds them for float_t of
 * `precision` bytes, widened to double (sph_t::set_coord_axes, sph_t::volume). */
int kp_mesh_geometry_sph( const kp_mesh_t * mesh, int precision, double * r_faces,
                          double * vol );
/* photon::sph_t::proc (modules/particle/radiation/photon_sph.h) over a
 * packet pool on a spherical mesh, like kp_trace: x[3n] (r, theta, phi) and
 * x_car[3n] (its Cartesian copy), both updated, dir[3n], and the other
 * arrays as kp_trace's.  The walk evaluates cosf, sinf, sqrtf, acosf and
 * atan2f per step as the reference does, with CUDA's functions. */
int kp_trace_sph( kp_mesh_t * mesh, int precision, long long n, void * x, void * x_car,
                  const void * dir, int * cell, int * ib, const void * proper, int * step,
                  int8_t * todo, int flux_mode, int fx_shift, void * flux, void * stream );

/* ------------------------------------------------------------------ */
/* Runtime refinement.  The reference declares the hook and leaves it   */
/* empty: mesh_t::changed (mesh/mesh.cpp:86-89), meshgen::base_t::update */
/* (mesh/meshgen/meshgen.cpp:443-446); block_map_t::update              */
/* (modules/particle/types/block_map.h:53-103) would rebuild the        */
/* neighbour tables.                                                    */

/* Per-block flags (device int[n_blocks]) from the mesh's coefficients:  */
/* +1 where some cell's extinction depth across the block's widest cell */
/* side exceeds tau_refine, -1 where every cell's stays below           */
/* tau_coarsen, else 0. */
int kp_mesh_flag_tau( kp_mesh_t * mesh, float tau_refine, float tau_coarsen, int * flags,
                      void * stream );
/* New mesh (*out, coefficients not set) from `mesh` and host flags
 * int[n_blocks]: blocks flagged > 0 are replaced by their eight children,
 * families whose eight blocks are leaves flagged < 0 by their parent; the
 * 2:1 balance of static refinement is then restored, a refinement winning
 * over a coarsening it would break.  The result equals the mesh built from
 * one [refine_region*] box per resulting leaf. */
int kp_mesh_adapt( const kp_mesh_t * mesh, const int * flags, kp_mesh_t ** out );
/* Per-cell field of n_comp floats (device, block-id order) from mesh `from`
 * to mesh `to` of the same domain: a `to` cell inside one `from` cell takes
 * its value; a `to` cell covering several (coarsened) takes the mean of the
 * eight octant samples.  E.g. n_comp = 2 for the coefficients. */
int kp_mesh_remap( kp_mesh_t * from, kp_mesh_t * to, int n_comp, const float * src, float * dst,
                   void * stream );

/* ------------------------------------------------------------------ */
/* Geometric walk with the path-length flux estimator.  Replaces        */
/* integrate::base_t::intg / ker_itg (modules/particle/evolve/          */
/* integrator.h:11-17,47-63,80-106) running photon::cart_t::proc        */
/* (modules/particle/radiation/photon.h:20-125) over the packet pool,   */
/* with the same per-step arithmetic.  Packet state is structure-of-    */
/* arrays in device memory and is updated in place, as the pool is:   */
/*   x[3n], dir[3n]  float_t (float if precision == 4, double if 8)     */
/*   cell[3n], ib[n], step[n]  int;  todo[n]  int8 (to_keep -2,         */
/*   to_rm -3, as particle::todo_t, types/particle_base.h:12)           */
/*   proper[n] float_t                                                  */
/* flux_mode 0: `flux` is float_t[n_cells] summed with float atomics,   */
/* as the reference does (photon.h:81); 1: `flux` is int64[n_cells]     */
/* holding round(deposit * 2^fx_shift), order independent.              */

enum kp_flux_mode { KP_FLUX_FLOAT = 0, KP_FLUX_FIXED = 1 };

int kp_trace( kp_mesh_t * mesh, int precision, long long n,
              void * x, const void * dir, int * cell, int * ib,
              const void * proper, int * step, int8_t * todo,
              int flux_mode, int fx_shift, void * flux, void * stream );

/* ------------------------------------------------------------------ */
/* Polarized Monte-Carlo transport.  Replaces one cycle of the particle */
/* module (particle::base_t::integrate, modules/particle/driver.h:      */
/* 59-79): the generator launch (evolve/generate_par.h:51-62, ker_gen)  */
/* and the integrator launch running the packet walk (evolve/           */
/* integrator.h:47-63; radiation/photon.h:104-125), extended with the   */
/* physics the reference leaves to user hooks (photon.h:73-102,         */
/* proc_phys/proc_step): optical-depth sampling, albedo weighting,      */
/* Rayleigh or HG+polarization scattering of the Stokes vector,         */
/* peel-off imaging and escape tallies.  Packets have counter-based     */
/* Philox streams keyed by (seed, stream_id) and their global id, so a  */
/* packet's history does not depend on the launch, the GPU count or the */
/* thread that runs it.                                                 */

#define KP_MAX_SOURCES 64
#define KP_MAX_BATCHES 64

enum kp_phase       { KP_PHASE_RAYLEIGH = 0, KP_PHASE_HG_POL = 1 };
enum kp_source_kind { KP_SOURCE_POINT = 0, KP_SOURCE_PLANE_BASE = 1 };
enum kp_emit        { KP_EMIT_ISOTROPIC = 0, KP_EMIT_UP_UNIFORM = 1 };
enum kp_tally_mode  { KP_TALLY_FIXED = 0, KP_TALLY_FLOAT = 1 };
enum kp_counter
{
    KP_CNT_STEPS = 0,       /* packet-steps of the walk (segments)        */
    KP_CNT_PEEL_STEPS,      /* segments of peel-off rays                  */
    KP_CNT_SCATTER,         /* interactions                               */
    KP_CNT_ESCAPED,
    KP_CNT_ABSORBED,        /* ended by Russian roulette                  */
    KP_CNT_CAPPED,          /* ended by max_scatter or max_steps          */
    KP_CNT_LOST,            /* no neighbour across an inner face          */
    KP_CNT_EMITTED,
    KP_CNT_HOPS,            /* block-to-block hand-offs (walk and peel-off) */
    KP_CNT_DEPOSITS,        /* tally deposits (escape bins, image pixels)  */
    KP_NCOUNTERS
};

typedef struct kp_source
{
    int    kind;     /* KP_SOURCE_POINT at pos, or KP_SOURCE_PLANE_BASE:
                        uniform over the domain's lower z face            */
    int    emit;     /* KP_EMIT_ISOTROPIC, or KP_EMIT_UP_UNIFORM (mu = d.z
                        uniform in (0,1))                                  */
    double pos[ 3 ];
} kp_source_t;

/* One packet made by a user generator: what the reference's generator
 * functor writes into the pool for each packet (x, dir, cell, block,
 * proper; modules/particle/evolve/generate_par.h:10-15, launched by ker_gen
 * over n_par packets, generate_par.h:51-62).  64 bytes, device memory. */
typedef struct kp_packet_init
{
    double x[ 3 ];       /* position inside the mesh                          */
    float  d[ 3 ];       /* unit direction                                    */
    float  w;            /* weight (the reference's `proper`)                 */
    float  stokes[ 3 ];  /* q, u, v relative to I, reference vector e1 =
                            normalize(z x d) if |d.z| < 0.9 else
                            normalize(x x d); 0 for unpolarized light          */
    int    ib;           /* block id, or -1 to locate x on the device         */
    float  peel_I;       /* emitted intensity per steradian toward the
                            observer per unit weight (1/(4 pi) for isotropic
                            emission); 0: no peel-off ray at emission          */
    int    pad;
} kp_packet_init_t;

typedef struct kp_transport_cfg
{
    long long n_packets;       /* packets of this call                         */
    long long packet_offset;   /* global id of its first packet               */
    uint32_t  seed;
    uint32_t  stream_id;       /* second Philox key word (e.g. scene id)       */
    int       phase;           /* enum kp_phase                                */
    float     hg_g;            /* HG asymmetry (KP_PHASE_HG_POL)               */
    float     pol_max;         /* peak linear polarization at 90 deg (HG)      */
    int       n_sources;       /* 1..KP_MAX_SOURCES; packet p uses p % n       */
    const kp_source_t * sources;   /* host pointer                             */
    int       n_mu_bins;       /* escape tally bins in mu = d.z (0: off)       */
    float     mu_lo, mu_hi;
    int       image_n;         /* peel-off image side in pixels (0: off)       */
    double    inclination_deg; /* observer direction from +z                   */
    double    azimuth_deg;     /* ... and about +z from +x                     */
    double    image_center[ 3 ];
    double    image_half_width;
    float     tau_peel_max;    /* peel-off rays stop beyond this depth (<=0: 40) */
    int       tally_mode;      /* enum kp_tally_mode                           */
    int       fx_shift;        /* fixed point: round(value * 2^fx_shift)       */
    int       n_batches;       /* batch-means tallies: packet p -> p % n       */
    int       image_batch_n;   /* side of the per-batch coarse image (>=1)     */
    float     w_min;           /* Russian roulette below this weight (0: off)  */
    float     rr_survive;      /* roulette survival probability (<=0: 0.1)     */
    int       max_scatter;     /* interactions per packet before it is ended   */
    long long max_steps;       /* segments per packet before it is ended       */
    long long n_record;        /* final-state records for the first n packets  */
    int       lane_batch;      /* scheduling: lanes of a warp that wait for an
                                  interaction or emission batch (0: default 6)  */
    int       flux_fx_shift;   /* fixed point of the flux tally (kp_tallies_t::
                                  flux): round(value * 2^flux_fx_shift); 0 takes
                                  fx_shift.  A cell's sum must stay below
                                  2^(63 - flux_fx_shift).                       */
    const kp_packet_init_t * packets;  /* device [n_packets] or NULL: when set,
                                  packet k of the call (global id
                                  packet_offset + k) starts from packets[k]
                                  instead of a source (sources are then not
                                  used and n_sources may be 0); its RNG stream
                                  is still keyed by its global id              */
} kp_transport_cfg_t;

typedef struct kp_packet_record
{
    double    x[ 3 ];
    float     d[ 3 ];
    float     stokes[ 3 ];     /* q, u, v relative to I (frame vector below)   */
    float     w;
    int       ib;
    int       cell[ 3 ];
    int       n_scatter;
    int       status;          /* 1 escaped, 2 absorbed, 3/4 capped, 5 lost    */
    uint32_t  rng_draws;       /* Philox blocks consumed                       */
    long long n_steps;
} kp_packet_record_t;

/* Output buffers (device pointers), accumulated into: zero them before the
 * first call.  Element type int64 (KP_TALLY_FIXED) or float (KP_TALLY_FLOAT).
 *   mu          [n_batches][n_mu_bins][4]  escaping I,Q,U,V (meridian frame)
 *   image       [image_n][image_n][4]      peel-off I,Q,U,V (Q>0 vertical)
 *   image_batch [n_batches][image_batch_n][image_batch_n][4]  coarse image
 *                                          per batch (pixel i -> i*bn/n)
 *   counters    [KP_NCOUNTERS] uint64 (optional)
 *   records     [n_record] (optional)
 *   flux        [n_cells] (optional) path-length estimator of the mean
 *               intensity, the reference's rad_t::flx: every walk segment of
 *               length dl in cell i adds w * dl / volume(i), w the packet's
 *               weight along the segment (photon::cart_t::proc_phys,
 *               modules/particle/radiation/photon.h:73-83, and its field,
 *               radiation/rad_data.cpp:13-25).  Block-id order, x fastest in
 *               a block; int64 with scale 2^flux_fx_shift, or float.  Peel-off
 *               rays deposit nothing.  In a decomposed solve the array is the
 *               rank's own blocks in local order (kp_dd_round_t::block_local). */
typedef struct kp_tallies
{
    void * mu;
    void * image;
    void * image_batch;
    unsigned long long * counters;
    kp_packet_record_t * records;
    void * flux;
    float * carry;       /* KP_TALLY_FLOAT only, optional (NULL: plain float
                            atomics): device floats, zeroed before the first
                            call, that collect the rounding error of every
                            float atomic, laid out as the float tallies in
                            use one after another: image, image_batch (both
                            with an image), mu (n_mu_bins > 0), flux (flux
                            set; flux_n entries).  Each solve adds them into
                            the tallies at its end and zeroes them, so a
                            tally is the exact sum of its float deposits up
                            to about 2^-24 of its own value instead of 2^-24
                            of every partial sum.  The batched solve does not
                            take it. */
    long long flux_n;    /* entries of flux (needed with carry and flux)     */
} kp_tallies_t;

/* Asynchronous on `stream`.  Calls that share a mesh handle must not
 * overlap on the GPU (they share the mesh's packet counter and peel-off
 * queue).  With an image, the first solve of a mesh allocates its peel-off
 * queue: 64 B per ray, 12 rays per packet, at most kp_mesh_peel_queue_limit
 * rays (default 2^27, 8.6 GB); later solves reuse it, and the mesh frees it
 * with the mesh. */
int kp_transport_forward( kp_mesh_t * mesh, const kp_transport_cfg_t * cfg,
                          const kp_tallies_t * tallies, void * stream );

/* Packet state carried between calls, 128 bytes in device memory: a walk
 * that a step budget suspended (kp_transport_forward_resume), or one handed
 * to another rank (kp_transport_forward_dd's walk records have this
 * layout).  Everything the walk needs to go on bit for bit. */
typedef struct kp_packet_state
{
    double   x[ 3 ];
    float    d[ 3 ];
    float    e1[ 3 ];        /* Stokes reference vector                       */
    float    stokes[ 3 ];    /* q, u, v relative to I                         */
    float    w;              /* weight                                        */
    float    tau;            /* optical depth left to the next interaction    */
    int      ib, cell[ 3 ];
    int      n_scatter, n_steps;
    uint32_t stream_id;      /* RNG key word 2 (kp_transport_cfg_t::stream_id) */
    uint32_t pid_lo, pid_hi; /* global packet id                              */
    uint32_t rng_draws;      /* Philox blocks consumed                        */
    int      batch;          /* batch-means index (pid % n_batches)           */
    int      pad[ 4 ];
} kp_packet_state_t;

/* Step budget and packet queues of a resumable call. */
typedef struct kp_resume
{
    const kp_packet_state_t * in;   /* device [n_in]: packets an earlier call
                                       suspended, resumed before cfg's new ones */
    long long n_in;
    kp_packet_state_t * out;        /* device [cap_out]: packets this call
                                       suspends (must not overlap `in`)         */
    long long cap_out;
    unsigned long long * out_count; /* device: packets written to out, added to
                                       (zero it first); a count above cap_out
                                       means lost packets (kp_mesh_status:
                                       queue overflow)                          */
    int step_budget;                /* walk segments a packet may take in this
                                       call (>= 1)                              */
} kp_resume_t;

/* kp_transport_forward with a per-call step budget, as the reference walks
 * each packet for at most `step` segments per cycle (photon::cart_t::proc,
 * modules/particle/radiation/photon.h:104-125).  The reference then removes
 * a packet whose budget ran out (todo = to_rm, photon.h:122-123); here it is
 * kept, as the pool keeps unfinished particles across cycles (types/
 * particle_pool.h:191-248, evolve/integrator.h:80-106): its whole state goes
 * to rs->out, and a later call that passes it in rs->in continues its walk.
 * A call first resumes rs->in, then emits cfg's n_packets new packets (none
 * needed: n_packets may be 0 without sources).  cfg->max_steps still ends a
 * packet for good.  In fixed point, calls that carry every packet to its
 * end give the tallies, counters and records of one kp_transport_forward
 * with the same cfg, bit for bit (records: packet_offset and n_record as in
 * that solve).  The reference's behaviour, a budget that ends packets, is
 * kp_transport_forward with max_steps = the budget.  Out-of-place queues
 * (swap in and out between calls); worst case cap_out = n_in + n_packets. */
int kp_transport_forward_resume( kp_mesh_t * mesh, const kp_transport_cfg_t * cfg,
                                 const kp_resume_t * rs, const kp_tallies_t * tallies,
                                 void * stream );

/* Upper bound on the mesh's peel-off queue (device memory, 64 B per ray;
 * default 2^27 rays = 8.6 GB).  With an image, kp_transport_forward queues
 * the peel-off rays of its packets and marches them in a second kernel; the
 * queue holds 12 rays per packet, so solves of more than limit/12 packets
 * run in chunks of that many packets, and a chunk that queues more rays
 * than the queue holds marches the rest where they start (same tallies).
 * A queue larger than the new limit is freed now.  Limits below 1024 rays
 * are refused (KP_ERR_CONFIG).  No counterpart in the reference. */
int kp_mesh_peel_queue_limit( kp_mesh_t * mesh, long long max_rays );

/* The order in which kp_transport_forward marches the queued peel-off rays
 * of this mesh.  KP_PEEL_ORDER_QUEUE: as queued.  KP_PEEL_ORDER_CELL: sorted
 * by starting cell first (a counting sort over the mesh's cells: about 1.3 ms
 * per 1e8 rays, up to 10 ms when one cell starts most of them, as a point
 * source's does; 4 B per ray plus 8 B per cell of device memory), so that
 * a warp marches rays that cross nearly the same cells: this pays when the
 * extinction field (4 B per cell) does not stay in L2.  KP_PEEL_ORDER_AUTO
 * (the default): CELL when the field exceeds KP_PEEL_SORT_MIN_BYTES, else
 * QUEUE.  Fixed-point tallies are the same bit for bit in either order;
 * float tallies agree within rounding.  Other values are refused
 * (KP_ERR_CONFIG).  No counterpart in the reference. */
#define KP_PEEL_ORDER_AUTO  (-1)
#define KP_PEEL_ORDER_QUEUE 0
#define KP_PEEL_ORDER_CELL  1
#define KP_PEEL_SORT_MIN_BYTES ( 32ll << 20 )
int kp_mesh_peel_order( kp_mesh_t * mesh, int order );

/* Profiling hook.  With an image, kp_transport_forward runs two kernels:
 * the walk (which queues the peel-off rays) and the peel-off march.  Later
 * kp_transport_forward calls of this host thread record `event` (a
 * cudaEvent_t) on their stream between the two launches, so that a caller
 * can time them apart; without an image it is recorded after the only
 * kernel.  NULL turns it off.  No counterpart in the reference. */
int kp_transport_split_event( void * event );

/* ------------------------------------------------------------------ */
/* Batched solves: many independent scenes in one persistent launch.    */
/* The reference solves one mesh per process, one cycle at a time       */
/* (modules/particle/driver.h:59-79); there is no counterpart.  The     */
/* scenes' block tables are concatenated into one multi-scene mesh; a   */
/* scene's packets (seed from the cfg, its own stream_id, local ids     */
/* 0..n-1) are identical to those of a kp_transport_forward of that     */
/* scene alone with the same seed and stream_id.                        */

typedef struct kp_batch kp_batch_t;

typedef struct kp_scene
{
    kp_mesh_t * mesh;          /* uploaded mesh with its coefficients set      */
    long long   n_packets;
    uint32_t    stream_id;     /* RNG key word of the scene's packets          */
    kp_source_t source;        /* point source                                 */
} kp_scene_t;

typedef struct kp_tune_result
{
    int       threads;         /* threads per block (128 or 256)               */
    int       lane_batch;      /* event batch (see kp_transport_cfg_t)         */
    int       grid_pct;        /* persistent grid, percent of resident blocks  */
    float     sample_ms;       /* time of the best candidate on the sample     */
    long long sample_packets;
} kp_tune_result_t;

/* Builds the concatenated tables (the scenes must share the cells per block;
 * their meshes are uploaded and their coefficients copied). */
int kp_batch_create( int n_scenes, const kp_scene_t * scenes, kp_batch_t ** batch );
int kp_batch_destroy( kp_batch_t * batch );
/* Re-copies every scene's coefficients after kp_mesh_set_sigma. */
int kp_batch_refresh_sigma( kp_batch_t * batch, void * stream );
/* Synchronizes, returns and clears the batch's device error status. */
int kp_batch_status( kp_batch_t * batch, void * stream, unsigned * flags );
/* One launch over all scenes.  cfg gives the physics and tally settings
 * (n_packets, packet_offset is added to every local id, sources and images
 * are not used: image_n must be 0).  mu: device [n_scenes][n_batches]
 * [n_mu_bins][4], accumulated into. */
int kp_batch_forward( kp_batch_t * batch, const kp_transport_cfg_t * cfg, void * mu,
                      unsigned long long * counters, void * stream );
/* Same launch replayed from a CUDA graph: the first call (or one whose
 * arguments changed) captures the counter reset and the kernel on `stream`
 * (non-default), later calls replay it. */
int kp_batch_graph_launch( kp_batch_t * batch, const kp_transport_cfg_t * cfg, void * mu,
                           unsigned long long * counters, void * stream );
/* Autotuner: times candidate launch shapes (threads per block, event batch,
 * grid fill) on `fraction` of every scene's packets, tallying into
 * mu_scratch (same shape as mu), and keeps the fastest for later launches. */
int kp_batch_autotune( kp_batch_t * batch, const kp_transport_cfg_t * cfg, double fraction,
                       void * mu_scratch, void * stream, kp_tune_result_t * result );

/* Path-replay adjoint of the peel-off image.  No reference counterpart (the
 * reference's transport is not differentiable); it differentiates the
 * solve of kp_transport_forward with the same cfg (same seed, packet ids
 * and sources) with respect to the per-cell coefficients.  adj_image
 * (device, float [image_n][image_n][4]) is dL/dimage in the units of the
 * forward image tally.  Accumulates, as int64 round(v * 2^grad_fx_shift)
 * (cfg->tally_mode KP_TALLY_FIXED) or float, per cell:
 *     grad_len  the path-length term, grad_int  the interaction term, so
 *     dL/dsigma_sca = grad_len + grad_int,  dL/dsigma_abs = grad_len.
 * Each packet is replayed twice from its RNG counter.  Between the two
 * replays the peel-off rays of its vertices (start point, weight and Stokes
 * vector toward the observer) wait in the mesh's peel-off queue, where two
 * marches measure their scores and deposit along them; packets whose rays
 * do not fit the queue (kp_mesh_peel_queue_limit) are replayed with their
 * rays inline, with the same results.  counters (optional) receives the
 * KP_CNT_* counts of both replays.  Besides the queue, the mesh keeps the
 * adjoint's buffers from the first call on: 20 B per queued ray, 20 B per
 * packet of a chunk, and 8 private int64 path-length tallies (64 B per
 * cell). */
int kp_transport_adjoint( kp_mesh_t * mesh, const kp_transport_cfg_t * cfg,
                          const float * adj_image, int grad_fx_shift,
                          void * grad_len, void * grad_int,
                          unsigned long long * counters, void * stream );

/* A forward solve followed by gradients of it (an autograd step).  No
 * reference counterpart.  kp_transport_forward_tape is kp_transport_forward
 * (same tallies, bit for bit) that also keeps, in the mesh, each packet's
 * vertex peel-off rays in vertex order with their attenuation; *tape_id
 * receives an id (> 0), or 0 when the solve has more packets than one chunk
 * of the peel-off queue (kp_mesh_peel_queue_limit / 12) and was not taped.
 * kp_transport_adjoint_tape then computes kp_transport_adjoint's gradients
 * (bit for bit in fixed point) without its first replay and measuring
 * march; it may be called several times per tape (different adj_image).
 * The tape lasts until the next forward or adjoint solve on the mesh,
 * kp_mesh_set_sigma, kp_mesh_sigma_ptr or kp_mesh_peel_queue_limit; the
 * adjoint refuses (KP_ERR_CONFIG) a tape that is gone or a cfg that does
 * not describe the taped solve.  The coefficients must be those of the
 * taped solve.  counters receives the counts of the work done (the second
 * replay and the deposits). */
int kp_transport_forward_tape( kp_mesh_t * mesh, const kp_transport_cfg_t * cfg,
                               const kp_tallies_t * tallies, void * stream, long long * tape_id );
int kp_transport_adjoint_tape( kp_mesh_t * mesh, long long tape_id,
                               const kp_transport_cfg_t * cfg, const float * adj_image,
                               int grad_fx_shift, void * grad_len, void * grad_int,
                               unsigned long long * counters, void * stream );
/* Id of the mesh's current tape (0: none). */
int kp_mesh_tape_id( const kp_mesh_t * mesh, long long * tape_id );

/* Same solve as kp_transport_forward, for callers that must not allocate
 * device memory during the call: code that owns every device byte itself
 * (a fixed arena or pool it sized at start-up), or a step that has to run
 * in a region where cudaMalloc is not allowed.  It calls no cudaMalloc,
 * cudaFree or allocating library routine.  The kernel's only scratch, the
 * 64-bit counter that hands out packet indices, lives in a static device
 * array of KP_NOALLOC_SCRATCH_BYTES that the library holds on every GPU
 * that loads it, until the process exits.  With an image, the peel-off rays
 * are marched inside the walk kernel, where they start (kp_transport_forward
 * queues them for a second kernel, and the queue is an allocation): the
 * int64 tallies are the same bit for bit, float tallies agree within float
 * rounding (another summation order; kp_tallies_t::carry, the caller's
 * memory, folds in their rounding errors), and the solve is slower.  A
 * kp_transport_split_event event is recorded after the walk.  Like every
 * solve it first refreshes the mesh's per-cell extinction array from the
 * coefficients, a kernel into memory the mesh allocated with its
 * coefficients at upload.  Inputs and outputs are the
 * caller's: the mesh must already be on the current device (kp_mesh_upload,
 * or an earlier kp_mesh_set_sigma, at set-up time), else KP_ERR_CONFIG; a
 * solve whose scratch would not fit is rejected with KP_ERR_CAPACITY.  The
 * first call on a device looks up the array's device address, so make that
 * first call before any stream capture.  Every call uses the same array and
 * zeroes the counter at its start, so calls that overlap on the GPU race:
 * run them one after another.  This entry point has no counterpart in the
 * reference. */
#define KP_NOALLOC_SCRATCH_BYTES 256
int kp_transport_forward_noalloc( kp_mesh_t * mesh, const kp_transport_cfg_t * cfg,
                                  const kp_tallies_t * tallies, void * stream );

/* ------------------------------------------------------------------ */
/* Domain-decomposed solve: packet migration between ranks that each    */
/* own part of the blocks, for meshes too large to replicate.  Replaces */
/* the reference's off-rank registration and exchange loop              */
/* (modules/particle/boundary/comm.h:118-239, comm_t::reg/proc/cpy_d)   */
/* with device queues exchanged between rounds (kratos_polrad_b200/     */
/* decomp.py: NCCL all-to-all, or device copies for ranks emulated on   */
/* one GPU).  Every rank holds the block tables of the whole mesh and   */
/* the coefficients of its own blocks.                                  */

#define KP_DD_WALK_BYTES 128   /* one migrating walk (full packet state)       */
#define KP_DD_PEEL_BYTES 96    /* one migrating peel-off ray (and its deposit) */

typedef struct kp_dd_round
{
    int         rank, n_ranks;
    const int * owner;          /* device int[n_blocks]: owning rank            */
    const int * block_local;    /* device int[n_blocks]: index among this rank's
                                   blocks, -1 for other ranks' blocks           */
    const float * sigma_local;  /* device: (sigma_sca, sigma_abs) of this rank's
                                   blocks, local block order, x fastest         */
    const void * in_walk;       /* device records arriving from other ranks     */
    long long    n_in_walk;
    const void * in_peel;
    long long    n_in_peel;
    int          emit;          /* 1 in the first round: emit this rank's share  */
    void *       out_walk;      /* device [cap_walk] records leaving this rank   */
    int *        out_walk_rank; /* device [cap_walk] destination rank of each    */
    long long    cap_walk;
    void *       out_peel;      /* device [cap_peel] records                     */
    int *        out_peel_rank; /* device [cap_peel]                             */
    long long    cap_peel;
    unsigned long long * out_count;  /* device [2] (walks, peel-off rays written,
                                        in any order), zeroed by the caller; a
                                        count above its capacity means lost
                                        records (kp_mesh_status: queue overflow) */
} kp_dd_round_t;

/* One round on this rank: processes the incoming records and (emit) the
 * rank's emissions of cfg's packets (the same cfg on every rank: point-source
 * packets are emitted by the rank owning the source's block, plane-source
 * packets by the rank pid % n_ranks), and writes every ray that crosses into
 * another rank's block to that rank's out-queue.  Tallies accumulate on this
 * rank; summed over the ranks after the last round (no records left
 * anywhere) they equal kp_transport_forward's, bit for bit in fixed point.
 * cfg->n_record must be 0. */
int kp_transport_forward_dd( kp_mesh_t * mesh, const kp_transport_cfg_t * cfg,
                             const kp_dd_round_t * round, const kp_tallies_t * tallies,
                             void * stream );

/* ------------------------------------------------------------------ */
/* The particle radiation module's configuration: the [particle],        */
/* [particles] and [device] keys that particle::base_t and its drivers   */
/* read in their init() (reference defaults in parentheses).  The module */
/* layer above the ABI (include/kp_module.hpp) uses n_par (packets per   */
/* cycle), step_max (segments per packet), n_hv (flux fields; the walk   */
/* deposits into field 0 as photon.h:81 does), n_cycle_stp (cycles per   */
/* step), seed_rng, idx_device and n_th (generator threads per block);   */
/* max_round, static_proxy, output and f_par are read and kept for the  */
/* caller.                                                               */

typedef struct kp_particle_cfg
{
    double n_par;        /* [particle] n_par (1.0)        generate_par.h:38   */
    double f_par;        /* [particle] f_par (1.0)        generate_par.h:40   */
    int    step_max;     /* [particle] step_max (100)     generate_par.h:36   */
    int    n_hv;         /* [particle] n_hv (1)           radiation.h:26      */
    int    n_cycle_stp;  /* [particle] n_cycle_stp (1)    driver.cpp:18       */
    int    n_th;         /* [particle] n_th (64)          driver_base.h:30    */
    int    max_round;    /* [particle] max_round (16)     integrator.h:35     */
    int    static_proxy; /* [particle] static_proxy (0)   block_map.h:39      */
    int    output;       /* [particles] output (1)        particle_pool.h:50  */
    int    seed_rng;     /* [device] seed_rng (7)         device.cpp:69       */
    int    idx_device;   /* [device] idx_device (-1)      device.cpp:67       */
} kp_particle_cfg_t;

/* Reads those keys from an INI file with the reference's syntax (later
 * values override earlier ones, io/args/input.cpp:72-108). */
int kp_particle_read( const char * ini_path, kp_particle_cfg_t * out );

/* prob::cmd (user/probgen.cpp:8-16): reads the input files paths[0..n-1]
 * in order with the reference's syntax, a later file's value of a key
 * replacing an earlier one's (input::read, io/args/input.cpp:72-108,
 * 162-167), and writes the merged keys to out_path as one INI file for
 * kp_mesh_create_ini and kp_particle_read. */
int kp_ini_merge( int n, const char * const * paths, const char * out_path );

/* ------------------------------------------------------------------ */
/* Binary container of the reference's binary_io (io/binary/            */
/* binary_io.h:6-32; save/load in binary_io_base.cpp:89-131): a byte of */
/* (little-endian | sizeof(size_t)), the header size, a tag-sorted map  */
/* tag -> (size, unit size, offset), then the data.  Files written here */
/* are byte-identical to binary_io::base_t::save's for the same entries */
/* and readable by the reference's visual/binary_io.py:31-55; the       */
/* reader takes either writer's files.  Host memory only.  Replaces     */
/* mesh_t::save / the restart load (mesh/mesh.cpp:63-69,99-112) for the */
/* transport's fields and tallies.                                      */

typedef struct kp_bio_entry
{
    const char *       tag;
    const void *       data;       /* host pointer                          */
    unsigned long long count;      /* elements                              */
    int                unit_size;  /* bytes per element, 1..127             */
} kp_bio_entry_t;

/* Writes (truncates) `path`; a later entry with the same tag replaces an
 * earlier one, as binary_io::base_t::write does. */
int kp_bio_write( const char * path, int n_entries, const kp_bio_entry_t * entries );

typedef struct kp_bio kp_bio_t;
/* Opens a container and reads its header (checks size_t and endianness as
 * binary_io::base_t::load_header does, and every entry against the file). */
int kp_bio_open( const char * path, kp_bio_t ** file );
int kp_bio_close( kp_bio_t * file );
int kp_bio_n_entries( const kp_bio_t * file, int * n );
/* Entry i in file order: tag (NUL-terminated into tag[tag_cap]), size in
 * bytes, unit size.  Any output may be NULL. */
int kp_bio_entry( const kp_bio_t * file, int i, char * tag, size_t tag_cap,
                  unsigned long long * size, int * unit_size );
/* Copies entry `tag` into dst (cap bytes available; KP_ERR_ARG if the tag
 * is missing or the entry is larger); *size receives its size in bytes. */
int kp_bio_read( const kp_bio_t * file, const char * tag, void * dst, unsigned long long cap,
                 unsigned long long * size );

#ifdef __cplusplus
}
#endif

#endif /* KP_TRANSPORT_H */
