// Device building blocks of the polarized transport kernels: packet state,
// emission, the FP64 cell walk with AMR hand-off, peel-off and tallies.
//
// The walk keeps the reference's cell-by-cell structure (one segment per
// loop iteration, modules/particle/radiation/photon.h:104-125) and its
// face-neighbour hand-off (types/proxy.h:64-121: sub-face chosen by the
// transverse half when the neighbour is finer), with these differences of
// design: positions are FP64 with precomputed inverse directions, the
// crossing coordinate is snapped to the new block's face (this also performs
// the periodic wrap of par_base_t::regulate, particle_base.h:37-56), and the
// transverse cell indices are recomputed from the position after a block
// change.
#pragma once

#include "kp_common.cuh"
#include "kp_physics.cuh"

#include <cooperative_groups.h>

namespace kp
{

constexpr int MAX_SOURCES = KP_MAX_SOURCES;

struct src_dev_t
{
    double pos[ 3 ];
    int    ib;
    int    cell[ 3 ];
    int    kind;
    int    emit;
};

// One scene of a batched launch (all scenes share one concatenated mesh).
struct scene_dev_t
{
    src_dev_t src;
    uint32_t  stream;          // RNG key word 2 of the scene's packets
    uint32_t  pad;
};

// Walk segments per scheduling round of k_forward (but its decomposed rounds)
// and k_adj_walk: 3 (forward walk 58.5 -> 56.9 ms, gradient 252 -> 247 ms,
// batched launch 154.6 -> 151.5 ms against 2); the walk with the flux tally
// keeps 2 (119 against 134 ms with 3).
#ifndef KP_WALK_INNER
#define KP_WALK_INNER 3
#endif
#ifndef KP_WALK_INNER_FLUX
#define KP_WALK_INNER_FLUX 2
#endif

// Everything a transport launch reads, passed by value.
struct fwd_params_t
{
    mesh_view_t m;
    long long   n_packets;         // packets of this launch
    long long   pid0;              // global id of the first packet
    uint32_t    seed, stream;
    phys::phase_t ph;
    int         n_src;
    const kp_packet_init_t * pk_table;  // caller's packets (null: the sources)
    long long   pk_pid0;                // global id of pk_table[0]
    int         n_mu;
    float       mu_lo, mu_inv_w;
    int         img_n;
    phys::v3    o, ev, eh;         // observer direction, image frame
    double      inv_o[ 3 ];
    double      o_d[ 3 ], ev_d[ 3 ], eh_d[ 3 ], img_c[ 3 ];
    double      img_inv_pix;
    float       tau_cut;
    double      fx_scale;
    int         n_batch;
    int         img_bn;            // coarse per-batch image side
    float       w_min, rr_survive;
    int         max_scatter;
    long long   max_steps;
    int         ev_batch;          // lanes that must wait for an event batch
    int         emit_batch;        // lanes that must wait for an emission batch (0: ev_batch)
    int         hop_batch;         // lanes that must wait for a hand-off batch
    int         peel_batch;        // k_peel: lanes that must wait for a fetch batch
    double      lk_inv[ 3 ];       // lookup cells per unit length
    void      * mu_tally;
    void      * image;
    void      * img_batch;
    unsigned long long * counters;
    kp_packet_record_t * records;
    long long   n_record;
    long long   rec_pid0;          // global id of the packet that records[0] holds
    void      * flux;              // path-length flux tally [n_cells] (null: off)
    double      flux_scale;        // its fixed point scale
    // float tallies' rounding-error carries (kp_tallies_t::carry; null: none)
    float     * c_image, * c_img_batch, * c_mu, * c_flux;
    unsigned long long * work;     // scratch: next packet index
    // adjoint only
    const float4 * adj_img;        // dL/d(image) [img_n * img_n] (I, Q, U, V)
    void      * g_len;             // path-length term per cell
    void      * g_int;             // interaction term per cell (sigma_sca only)
    double      g_scale;           // fixed point scale of the gradient tallies
    // batched launch only (n_scenes > 0)
    int         n_scenes;
    const long long   * scene_prefix;   // [n_scenes + 1] packet index prefix
    const scene_dev_t * scenes;         // [n_scenes]
    long long   mu_scene_stride;        // mu tally elements per scene
    // domain-decomposed rounds only (kp_transport_forward_dd)
    int         dd_rank, dd_ranks;
    const int * dd_owner;               // [n_blocks] rank owning the block
    const int * dd_loc;                 // [n_blocks] local block index, -1 if foreign
    const struct dd_walk_t * dd_in_walk;
    const struct dd_peel_t * dd_in_peel;
    long long   dd_n_walk, dd_n_peel;   // incoming records
    int         dd_emit;                // emit this rank's packets in this round
    struct dd_walk_t * dd_out_walk;     // [dd_cap_walk] records leaving this rank
    struct dd_peel_t * dd_out_peel;     // [dd_cap_peel]
    int       * dd_out_walk_rank;       // destination rank of each record
    int       * dd_out_peel_rank;
    long long   dd_cap_walk, dd_cap_peel;
    unsigned long long * dd_out_count;  // [2]: walks, peel-off rays
    // resumable solves only (kp_transport_forward_resume): packets carried
    // across calls as whole walks
    const struct dd_walk_t * rs_in;     // [rs_n_in] suspended earlier, resumed first
    long long   rs_n_in;
    struct dd_walk_t * rs_out;          // [rs_cap] suspended by this launch
    long long   rs_cap;
    unsigned long long * rs_count;      // records written to rs_out (may exceed rs_cap)
    int         rs_budget;              // walk segments of a packet per launch
    // peel-off rays deferred to k_peel (plain forward solves)
    struct peel_task_t * pq;            // [pq_cap] tasks
    struct peel_link_t * pq_link;       // [pq_cap] per-packet links (tape, adjoint)
    unsigned long long * pq_count;      // tasks written (may exceed pq_cap: those ran inline)
    unsigned long long * pq_next;       // k_peel's task counter
    const int * pq_perm;                // k_peel: the tasks in march order (null: queue order)
    long long   pq_cap;
    // deferred adjoint (kp_transport_adjoint): the tasks are the vertices'
    // peel-off rays, linked in vertex order per packet of the launch
    float     * adj_G;                  // [pq_cap] G of each task's ray
    float     * adj_att;                // [pq_cap] taped solve: w exp(-tau) of each ray (-1: cut)
    int       * adj_head;               // [n_packets] first task of the packet, -1: none
    double    * adj_R0;                 // [n_packets] sum of G over its interactions
    int       * adj_flag;               // [n_packets] 1: the queue overflowed for it
    int       * adj_list;               // [n_packets] packets handed to k_adjoint
    unsigned long long * adj_list_n;    //   ... and their count
    int         adj_quiet;              // k_adjoint: its first replay counts nothing
    void      * adj_priv;               // k_peel mode 2: adj_npriv private path-length
    int         adj_npriv;              //   tallies (block b uses copy b % adj_npriv)
    src_dev_t   src[ MAX_SOURCES ];
};

// A peel-off ray waiting for k_peel: where it starts (the interaction or
// emission point, its block and cell) and its pending contribution.  64
// bytes, two whole 32-byte sectors, written and read as 16-byte vectors
// (store_task, load_task_ray, load_task_deposit); the cell indices are
// packed 10 bits each (blocks of at most 1024 cells a side).
struct __align__( 16 ) peel_task_t
{
    double   x[ 3 ];
    int      b;
    unsigned c;                    // c0 | c1 << 10 | c2 << 20
    float    w, I, Q, U, V;
    int      pix, cpix;
    int      pad;
};
static_assert( sizeof( peel_task_t ) == 64, "peel-off task: two sectors" );
constexpr int PQ_MAX_CELLS = 1024;   // cells per block side a task can hold

// When the rays are linked per packet (the deferred adjoint, a taped forward
// solve), the task's entry of this array, parallel to the queue, holds the
// packet's index in the launch (lp), the vertex (kv, 0: emission) and the
// packet's next task (next, -1: last).
struct peel_link_t
{
    int lp, kv, next;
};

__device__ __forceinline__ void store_task( peel_task_t * q, unsigned long long k,
                                            const double x[ 3 ], int b, const int c[ 3 ],
                                            float w, float I, float Q, float U, float V,
                                            int pix, int cpix )
{
    char * t = reinterpret_cast< char * >( q + k );
    const long long x2 = __double_as_longlong( x[ 2 ] );
    const unsigned cp = ( unsigned ) c[ 0 ] | ( ( unsigned ) c[ 1 ] << 10 )
                      | ( ( unsigned ) c[ 2 ] << 20 );
    * reinterpret_cast< double2 * >( t )     = make_double2( x[ 0 ], x[ 1 ] );
    * reinterpret_cast< int4 * >( t + 16 )   = make_int4( ( int ) x2, ( int ) ( x2 >> 32 ), b,
                                                          ( int ) cp );
    * reinterpret_cast< float4 * >( t + 32 ) = make_float4( w, I, Q, U );
    * reinterpret_cast< int4 * >( t + 48 )   = make_int4( __float_as_int( V ), pix, cpix, 0 );
}

// The ray's start: position, block, cell.
__device__ __forceinline__ void load_task_ray( const peel_task_t * q, long long k, double x[ 3 ],
                                               int & b, int c[ 3 ] )
{
    const char * t = reinterpret_cast< const char * >( q + k );
    const double2 a = * reinterpret_cast< const double2 * >( t );
    const int4    v = * reinterpret_cast< const int4 * >( t + 16 );
    x[ 0 ] = a.x;
    x[ 1 ] = a.y;
    x[ 2 ] = __hiloint2double( v.y, v.x );
    b = v.z;
    const unsigned cp = ( unsigned ) v.w;
    c[ 0 ] = ( int ) ( cp & 1023u );
    c[ 1 ] = ( int ) ( ( cp >> 10 ) & 1023u );
    c[ 2 ] = ( int ) ( cp >> 20 );
}

// The ray's pending contribution: weight, Stokes vector toward the observer,
// its pixel and coarse per-batch pixel.
struct task_dep_t
{
    float w, I, Q, U, V;
    int   pix, cpix;
};
__device__ __forceinline__ task_dep_t load_task_deposit( const peel_task_t * q, long long k )
{
    const char * t = reinterpret_cast< const char * >( q + k );
    const float4 f = * reinterpret_cast< const float4 * >( t + 32 );
    const int4   g = * reinterpret_cast< const int4 * >( t + 48 );
    return task_dep_t { f.x, f.y, f.z, f.w, __int_as_float( g.x ), g.y, g.z };
}

// A packet's walk crossing into a block of another rank (it has entered the
// block: position snapped to the face, cell and block set).  The inverse
// direction and the face cache are rebuilt from it, bit for bit.
struct __align__( 16 ) dd_walk_t
{
    double   x[ 3 ];
    float    d[ 3 ], e1[ 3 ], S[ 3 ];
    float    w, tau;
    int      b, c[ 3 ];
    int      n_scat, n_steps;
    uint32_t k1, pid_lo, pid_hi, draw;
    int      batch, pad[ 3 ];
};

// A peel-off ray crossing into a block of another rank, with its pending
// contribution (the deposit happens where the ray ends).
struct __align__( 16 ) dd_peel_t
{
    double x[ 3 ];                 // the ray's start
    int    b, c[ 3 ];              // the block entered, its cell
    float  ptau;
    int    pk;
    float  w, I, Q, U, V;
    int    pix, cpix;
    int    pad;
    double tc;                     // distance travelled from the start
};

enum pk_status { PK_ESCAPED = 1, PK_ABSORBED = 2, PK_SCATTER_CAP = 3, PK_STEP_CAP = 4,
                 PK_LOST = 5 };

struct packet_t
{
    double        x[ 3 ];
    double        inv[ 3 ];
    phys::v3      d, e1;
    phys::stokes_t S;
    float         w, tau;
    int           b;
    int           c[ 3 ];
    int           n_scat;
    int           n_steps;
    phys::rng_t   rng;
    __device__ __forceinline__ long long pid(  ) const
    {
        return ( long long ) ( ( ( unsigned long long ) rng.pid_hi << 32 ) | rng.pid_lo );
    }
};

struct local_counts_t
{
    unsigned long long steps = 0, peel = 0, scat = 0, esc = 0, absb = 0, cap = 0,
                       lost = 0, emit = 0, hops = 0, dep = 0;
};

__device__ __forceinline__ float comp( const phys::v3 & v, int a )
{
    return a == 0 ? v.x : ( a == 1 ? v.y : v.z );
}

__device__ __forceinline__ void set_inv( packet_t & p )
{
    #pragma unroll
    for( int a = 0; a < 3; ++ a )
    {
        const float da = comp( p.d, a );
        // the correctly rounded reciprocal: 1.0 / da, bit for bit
        p.inv[ a ] = da != 0.0f ? __drcp_rn( ( double ) da ) : 0.0;
    }
}

__device__ __forceinline__ size_t cell_index( const mesh_view_t & m, int b, const int c[ 3 ] )
{
    return ( size_t ) b * m.cpb + c[ 0 ] + m.nc[ 0 ] * ( c[ 1 ] + m.nc[ 1 ] * c[ 2 ] );
}

// Distance along d to the exit face of cell c of block b (first axis wins
// ties; axes with d == 0 never exit).
__device__ __forceinline__ double exit_dist( const mesh_view_t & m, int b, const int c[ 3 ],
                                             const double x[ 3 ], const phys::v3 & d,
                                             const double inv[ 3 ], int & ax )
{
    const double * g = m.geo_d + 16 * ( size_t ) b;
    double t = 1e300;
    ax = 0;
    #pragma unroll
    for( int a = 0; a < 3; ++ a )
    {
        const float da = comp( d, a );
        if( da == 0.0f ) continue;
        const double face = __fma_rn( ( double ) ( c[ a ] + ( da > 0.0f ? 1 : 0 ) ),
                                      g[ 3 + a ], g[ a ] );
        double ta = __dmul_rn( __dsub_rn( face, x[ a ] ), inv[ a ] );
        ta = ta < 0.0 ? 0.0 : ta;
        if( ta < t ) { t = ta; ax = a; }
    }
    return t;
}

// Steps into the neighbouring cell across face `ax` (x already advanced on
// the other axes).  Returns false when the packet leaves the domain
// (physical boundary) or finds no neighbour (lost = true).
__device__ __forceinline__ bool cross_face( const mesh_view_t & m, int & b, int c[ 3 ],
                                            double x[ 3 ], int ax, bool pos, bool & lost )
{
    lost = false;
    // select, not c[ ax ]: a runtime index would move c[] to local memory
    const int cax = ax == 0 ? c[ 0 ] : ( ax == 1 ? c[ 1 ] : c[ 2 ] );
    int cn = cax + ( pos ? 1 : -1 );
    const double * g = m.geo_d + 16 * ( size_t ) b;
    if( cn >= 0 && cn < m.nc[ ax ] )
    {
        #pragma unroll
        for( int a = 0; a < 3; ++ a )
            if( a == ax )
            {
                c[ a ] = cn;
                x[ a ] = __fma_rn( ( double ) ( pos ? cn : cn + 1 ), g[ 3 + a ], g[ a ] );
            }
        return true;
    }
    const int side = pos ? 1 : 0;
    // the face's four neighbour slots (16-byte aligned: 24 ints per block),
    // loaded together with the meta record, not after it
    const int4 q = reinterpret_cast< const int4 * >( m.nb + 24 * ( size_t ) b )[ ax * 2 + side ];
    const blk_meta_t md = m.meta[ b ];
    if( ( md.phybnd >> ( 2 * ax + side ) ) & 1 )
    {   // leaves the domain: the position ends on the boundary face
        #pragma unroll
        for( int a = 0; a < 3; ++ a )
            if( a == ax )
                x[ a ] = __fma_rn( ( double ) ( pos ? cax + 1 : cax ), g[ 3 + a ], g[ a ] );
        return false;
    }
    const int a1 = ax == 2 ? 0 : ax + 1;
    const int a2 = ax == 0 ? 2 : ax - 1;
    int ca1 = 0, ca2 = 0;
    #pragma unroll
    for( int a = 0; a < 3; ++ a ) { if( a == a1 ) ca1 = c[ a ]; if( a == a2 ) ca2 = c[ a ]; }
    int j0 = 0, j1 = 0;
    if( md.d_lvl[ 2 * ax + side ] > 0 )
    {
        j0 = ca1 >= m.nc[ a1 ] / 2;
        j1 = ca2 >= m.nc[ a2 ] / 2;
    }
    const int js = j0 * 2 + j1;
    const int nid = js == 0 ? q.x : ( js == 1 ? q.y : ( js == 2 ? q.z : q.w ) );
    if( nid < 0 || nid >= m.n_blocks )
    {
        lost = true;
        return false;
    }
    b = nid;
    const double * h = m.geo_d + 16 * ( size_t ) nid;
    #pragma unroll
    for( int a = 0; a < 3; ++ a )
    {
        if( a == ax )
        {
            c[ a ] = pos ? 0 : m.nc[ a ] - 1;
            x[ a ] = pos ? h[ a ] : __fma_rn( ( double ) m.nc[ a ], h[ 3 + a ], h[ a ] );
        }
        else
        {
            const double f = floor( __dmul_rn( __dsub_rn( x[ a ], h[ a ] ), h[ 8 + a ] ) );
            int ci = f < 0.0 ? 0 : ( f > ( double ) ( m.nc[ a ] - 1 ) ? m.nc[ a ] - 1 : ( int ) f );
            c[ a ] = ci;
        }
    }
    return true;
}

// Face cache of the active ray (forward kernel).  fx[a] is the coordinate of
// the face through which the ray leaves cell c along axis a, computed with
// exit_dist's expression, so distances from the cache are bit-identical to
// exit_dist's while a segment loads no geometry.  Refreshed for all axes when
// the direction or the block changes, for one axis after an in-block step.
__device__ __forceinline__ void faces_all( const mesh_view_t & m, int b, const int c[ 3 ],
                                           const phys::v3 & d, double fx[ 3 ] )
{
    const double * g = m.geo_d + 16 * ( size_t ) b;
    #pragma unroll
    for( int a = 0; a < 3; ++ a )
        fx[ a ] = __fma_rn( ( double ) ( c[ a ] + ( comp( d, a ) > 0.0f ? 1 : 0 ) ), g[ 3 + a ],
                            g[ a ] );
}

// exit_dist from the face cache.
__device__ __forceinline__ double exit_cached( const double x[ 3 ], const double fx[ 3 ],
                                               const phys::v3 & d, const double inv[ 3 ], int & ax )
{
    double t = 1e300;
    ax = 0;
    #pragma unroll
    for( int a = 0; a < 3; ++ a )
    {
        if( comp( d, a ) == 0.0f ) continue;
        double ta = __dmul_rn( __dsub_rn( fx[ a ], x[ a ] ), inv[ a ] );
        ta = ta < 0.0 ? 0.0 : ta;
        if( ta < t ) { t = ta; ax = a; }
    }
    return t;
}

// The in-block half of cross_cached: steps into the next cell across face
// `ax` when it lies in the same block (x snaps to the cached face, one new
// face is computed) and returns true; returns false, changing nothing, when
// the step leaves the block.
__device__ __forceinline__ bool step_in_block( const mesh_view_t & m, int b, int c[ 3 ],
                                               double x[ 3 ], double fx[ 3 ], int ax,
                                               const phys::v3 & d )
{
    const bool pos = comp( d, ax ) > 0.0f;
    const int cax = ax == 0 ? c[ 0 ] : ( ax == 1 ? c[ 1 ] : c[ 2 ] );
    const int cn = cax + ( pos ? 1 : -1 );
    if( cn < 0 || cn >= m.nc[ ax ] )
        return false;
    const double * g = m.geo_d + 16 * ( size_t ) b;
    const double nf = __fma_rn( ( double ) ( cn + ( pos ? 1 : 0 ) ), g[ 3 + ax ], g[ ax ] );
    #pragma unroll
    for( int a = 0; a < 3; ++ a )
        if( a == ax ) { c[ a ] = cn; x[ a ] = fx[ a ]; fx[ a ] = nf; }
    return true;
}

// cross_face with the face cache: inside the block the crossed face is the
// cached one (x snaps to it) and only that axis's next face is computed;
// a hand-off to a neighbour block refreshes all three.
__device__ __forceinline__ bool cross_cached( const mesh_view_t & m, int & b, int c[ 3 ],
                                              double x[ 3 ], double fx[ 3 ], int ax,
                                              const phys::v3 & d, bool & lost )
{
    const bool pos = comp( d, ax ) > 0.0f;
    const int cax = ax == 0 ? c[ 0 ] : ( ax == 1 ? c[ 1 ] : c[ 2 ] );
    const int cn = cax + ( pos ? 1 : -1 );
    if( cn >= 0 && cn < m.nc[ ax ] )
    {
        lost = false;
        const double * g = m.geo_d + 16 * ( size_t ) b;
        const double nf = __fma_rn( ( double ) ( cn + ( pos ? 1 : 0 ) ), g[ 3 + ax ], g[ ax ] );
        #pragma unroll
        for( int a = 0; a < 3; ++ a )
            if( a == ax ) { c[ a ] = cn; x[ a ] = fx[ a ]; fx[ a ] = nf; }
        return true;
    }
    if( ! cross_face( m, b, c, x, ax, pos, lost ) )
        return false;
    faces_all( m, b, c, d, fx );
    return true;
}

// Direction of the parked walk while a peel-off ray holds the direction
// registers (forward kernel).
template< int NT >
struct dir_park_t
{
    float  d[ 3 ][ NT ];
    double inv[ 3 ][ NT ];
    int    cpix[ NT ];             // coarse per-batch pixel of the pending deposit
};

template< class SD >
__device__ __forceinline__ void park_dir( SD & sd, packet_t & p, const phys::v3 & o,
                                          const double inv_o[ 3 ] )
{
    const int t = threadIdx.x;
    sd.d[ 0 ][ t ] = p.d.x; sd.d[ 1 ][ t ] = p.d.y; sd.d[ 2 ][ t ] = p.d.z;
    #pragma unroll
    for( int a = 0; a < 3; ++ a ) { sd.inv[ a ][ t ] = p.inv[ a ]; p.inv[ a ] = inv_o[ a ]; }
    p.d = o;
}
template< class SD >
__device__ __forceinline__ void unpark_dir( const SD & sd, packet_t & p )
{
    const int t = threadIdx.x;
    p.d = phys::v3 { sd.d[ 0 ][ t ], sd.d[ 1 ][ t ], sd.d[ 2 ][ t ] };
    #pragma unroll
    for( int a = 0; a < 3; ++ a ) p.inv[ a ] = sd.inv[ a ][ t ];
}

// Packet state that only interactions, emissions, tallies and records use
// (forward kernel): the Stokes frame, Stokes vector, weight, interaction
// count and RNG counter words live in shared memory between those events,
// so the segment loop keeps only the ray's geometry in registers.
template< int NT >
struct cold_park_t
{
    float    e1[ 3 ][ NT ];
    float    S[ 3 ][ NT ];
    float    w[ NT ];
    int      n_scat[ NT ];
    uint32_t k1[ NT ], pid_lo[ NT ], pid_hi[ NT ], draw[ NT ];
    int      batch[ NT ];          // pid % n_batches, set at emission
    double   wv[ NT ];             // flux tally: w / volume of the walk's block
};

template< class SC >
__device__ __forceinline__ void store_cold( SC & sc, const packet_t & p )
{
    const int t = threadIdx.x;
    sc.e1[ 0 ][ t ] = p.e1.x; sc.e1[ 1 ][ t ] = p.e1.y; sc.e1[ 2 ][ t ] = p.e1.z;
    sc.S[ 0 ][ t ] = p.S.q; sc.S[ 1 ][ t ] = p.S.u; sc.S[ 2 ][ t ] = p.S.v;
    sc.w[ t ] = p.w;
    sc.n_scat[ t ] = p.n_scat;
    sc.k1[ t ] = p.rng.k1; sc.pid_lo[ t ] = p.rng.pid_lo; sc.pid_hi[ t ] = p.rng.pid_hi;
    sc.draw[ t ] = p.rng.draw;
}
template< class SC >
__device__ __forceinline__ void load_cold( const SC & sc, packet_t & p, uint32_t seed )
{
    const int t = threadIdx.x;
    p.e1 = phys::v3 { sc.e1[ 0 ][ t ], sc.e1[ 1 ][ t ], sc.e1[ 2 ][ t ] };
    p.S = phys::stokes_t { sc.S[ 0 ][ t ], sc.S[ 1 ][ t ], sc.S[ 2 ][ t ] };
    p.w = sc.w[ t ];
    p.n_scat = sc.n_scat[ t ];
    p.rng = phys::rng_t { seed, sc.k1[ t ], sc.pid_lo[ t ], sc.pid_hi[ t ], sc.draw[ t ] };
}
template< class SC >
__device__ __forceinline__ long long cold_pid( const SC & sc )
{
    const int t = threadIdx.x;
    return ( long long ) ( ( ( unsigned long long ) sc.pid_hi[ t ] << 32 ) | sc.pid_lo[ t ] );
}

// Peel-off rays toward the observer are marched as a fixed-direction cell
// walk, block by block, measured from the point x0 where the ray entered its
// block (or started): tm[a] is the distance from x0 to the next face of the
// current cell on axis a ((face - x0[a]) times the inverse observer
// direction; 1e300 on an axis the direction does not move along), a segment
// ends at the nearest (the first axis wins ties), and its length is that
// distance less the distance tc already travelled from x0 (never negative).
// A block hand-off goes through the crossing point x0 + tc o (oray_point),
// which cross_face snaps to the new block's face (wrapping a periodic
// boundary), and that point becomes the new x0 with tc = 0 (oray_rebase).
// The position is not advanced segment by segment, so a segment costs one
// comparison chain and, inside a block, one new face.

// tm for every axis of cell c of block b.
__device__ __forceinline__ void oray_faces( const fwd_params_t & P, int b, const int c[ 3 ],
                                            const double x0[ 3 ], double tm[ 3 ] )
{
    const double * g = P.m.geo_d + 16 * ( size_t ) b;
    #pragma unroll
    for( int a = 0; a < 3; ++ a )
    {
        const float oa = comp( P.o, a );
        tm[ a ] = oa == 0.0f ? 1e300
                : __dmul_rn( __dsub_rn( __fma_rn( ( double ) ( c[ a ] + ( oa > 0.0f ? 1 : 0 ) ),
                                                  g[ 3 + a ], g[ a ] ), x0[ a ] ), P.inv_o[ a ] );
    }
}

// Length of the ray's next segment; ax receives its exit face's axis and tc
// moves to the face.
__device__ __forceinline__ double oray_segment( const double tm[ 3 ], double & tc, int & ax )
{
    int a0 = 0;
    double tn = tm[ 0 ];
    if( tm[ 1 ] < tn ) { tn = tm[ 1 ]; a0 = 1; }
    if( tm[ 2 ] < tn ) { tn = tm[ 2 ]; a0 = 2; }
    double dt = __dsub_rn( tn, tc );
    dt = dt < 0.0 ? 0.0 : dt;
    tc = tn > tc ? tn : tc;
    ax = a0;
    return dt;
}

// Into the next cell across face ax when it lies in the same block (the cell
// and that axis's face distance move) and true; false, changing nothing,
// when the step leaves the block.
__device__ __forceinline__ bool oray_step_in_block( const fwd_params_t & P, int b, int c[ 3 ],
                                                    const double x0[ 3 ], double tm[ 3 ], int ax )
{
    const bool pos = comp( P.o, ax ) > 0.0f;
    // selects, not c[ ax ] / x0[ ax ]: a runtime index would move the arrays
    // to local memory
    const int cax = ax == 0 ? c[ 0 ] : ( ax == 1 ? c[ 1 ] : c[ 2 ] );
    const int cn = cax + ( pos ? 1 : -1 );
    if( cn < 0 || cn >= P.m.nc[ ax ] )
        return false;
    const double * g = P.m.geo_d + 16 * ( size_t ) b;
    const double xa = ax == 0 ? x0[ 0 ] : ( ax == 1 ? x0[ 1 ] : x0[ 2 ] );
    const double nt = __dmul_rn( __dsub_rn( __fma_rn( ( double ) ( cn + ( pos ? 1 : 0 ) ),
                                                      g[ 3 + ax ], g[ ax ] ), xa ), P.inv_o[ ax ] );
    #pragma unroll
    for( int a = 0; a < 3; ++ a )
        if( a == ax ) { c[ a ] = cn; tm[ a ] = nt; }
    return true;
}

// The ray's point at distance tc from x0.
__device__ __forceinline__ void oray_point( const fwd_params_t & P, const double x0[ 3 ], double tc,
                                            double x[ 3 ] )
{
    #pragma unroll
    for( int a = 0; a < 3; ++ a ) x[ a ] = __fma_rn( tc, P.o_d[ a ], x0[ a ] );
}

// Block hand-off of a ray across face ax: through its crossing point into the
// neighbour (b, c move), which becomes its new x0 (tc = 0, tm refreshed).
// False when the ray leaves the domain or finds no neighbour.
__device__ __forceinline__ bool oray_rebase( const fwd_params_t & P, int & b, int c[ 3 ],
                                             double x0[ 3 ], double & tc, double tm[ 3 ], int ax,
                                             bool & lost )
{
    double x[ 3 ];
    oray_point( P, x0, tc, x );
    if( ! cross_face( P.m, b, c, x, ax, comp( P.o, ax ) > 0.0f, lost ) )
        return false;
    #pragma unroll
    for( int a = 0; a < 3; ++ a ) x0[ a ] = x[ a ];
    tc = 0.0;
    oray_faces( P, b, c, x0, tm );
    return true;
}

// A whole peel-off ray marched by one lane: the optical depth from x0 (cell
// c0 of block b) to the domain boundary, or the first value beyond tau_cut;
// segs and hops receive its segments and block hand-offs.  The segments are
// those of the scheduled march (k_peel, the inline rays), one by one.
__device__ __forceinline__ float oray_march( const fwd_params_t & P, int b, const int c0[ 3 ],
                                                 const double x0[ 3 ], unsigned & segs,
                                                 unsigned & hops )
{
    int c[ 3 ] = { c0[ 0 ], c0[ 1 ], c0[ 2 ] };
    double x[ 3 ] = { x0[ 0 ], x0[ 1 ], x0[ 2 ] };    // where the ray entered its block
    double tm[ 3 ], tc = 0.0;
    oray_faces( P, b, c, x, tm );
    float tau = 0.0f;
    for( int k = 0; k < ( 1 << 20 ); ++ k )
    {
        const float ext = P.m.ext[ cell_index( P.m, b, c ) ];
        int ax;
        const double dt = oray_segment( tm, tc, ax );
        tau = __fadd_rn( tau, __fmul_rn( ext, ( float ) dt ) );
        ++ segs;
        if( tau > P.tau_cut )
            return tau;
        if( ! oray_step_in_block( P, b, c, x, tm, ax ) )
        {
            bool lost;
            const int b_old = b;
            if( ! oray_rebase( P, b, c, x, tc, tm, ax, lost ) )
                return tau;
            hops += b != b_old;
        }
    }
    return tau;
}

// Carries of the float tallies and the fold that adds them in after a solve
// (kp_tallies_t::carry).
struct carry_seg_t
{
    float   * hi;                  // the tally
    float   * c;                   // its carry
    long long n;
};
struct carry_fold_t
{
    carry_seg_t seg[ 4 ];
    int         n_seg;
};
carry_fold_t carry_layout( const kp_transport_cfg_t & c, const kp_tallies_t & t );
void fold_carry( const kp_transport_cfg_t & c, const kp_tallies_t & t, cudaStream_t s );

// FP32 atomic add of v to base[i].  With a carry array, the rounding error
// of the sum that the atomic stored goes to carry[i]: atom.add.f32 rounds to
// nearest even, so the value it read (old) and v give that error exactly by
// the error-free transformation TwoSum (Knuth, TAOCP vol. 2, 4.2.2; Moller
// 1965): s = old + v, bv = s - old, e = (old - (s - bv)) + (v - bv), and
// old + v = s + e exactly.  base[i] + carry[i], folded after the solve, is
// then the float deposits' sum up to the carry's own rounding (of order
// 2^-24 of the sum of the errors, themselves 2^-24 of the partial sums).
// Subnormal operands, which the atomic flushes to zero, lose at most 2^-126.
__device__ __forceinline__ void atomic_add_carry( float * base, float * carry, size_t i, float v )
{
    if( carry == nullptr )
    {
        atomicAdd( base + i, v );
        return;
    }
    const float old = atomicAdd( base + i, v );
    const float s   = __fadd_rn( old, v );
    const float bv  = __fsub_rn( s, old );
    const float e   = __fadd_rn( __fsub_rn( old, __fsub_rn( s, bv ) ), __fsub_rn( v, bv ) );
    if( e != 0.0f )
        atomicAdd( carry + i, e );
}

template< int TALLY >
__device__ __forceinline__ void add_tally( void * base, float * carry, size_t i, float v,
                                           double sc )
{
    if( TALLY == KP_TALLY_FIXED )
        atomicAdd( ( unsigned long long * ) base + i,
                   ( unsigned long long ) __double2ll_rn( __dmul_rn( ( double ) v, sc ) ) );
    else
        atomic_add_carry( ( float * ) base, carry, i, v );
}

// Image pixel (iy * n + ix) under position x, or -1 outside the image.
__device__ __forceinline__ int image_pixel( const fwd_params_t & P, const double x[ 3 ] )
{
    double r[ 3 ];
    #pragma unroll
    for( int a = 0; a < 3; ++ a ) r[ a ] = __dsub_rn( x[ a ], P.img_c[ a ] );
    const double hp = __dadd_rn( __dadd_rn( __dmul_rn( r[ 0 ], P.eh_d[ 0 ] ),
                                            __dmul_rn( r[ 1 ], P.eh_d[ 1 ] ) ),
                                 __dmul_rn( r[ 2 ], P.eh_d[ 2 ] ) );
    const double vp = __dadd_rn( __dadd_rn( __dmul_rn( r[ 0 ], P.ev_d[ 0 ] ),
                                            __dmul_rn( r[ 1 ], P.ev_d[ 1 ] ) ),
                                 __dmul_rn( r[ 2 ], P.ev_d[ 2 ] ) );
    const double half = 0.5 * P.img_n;
    const double fx = floor( __fma_rn( hp, P.img_inv_pix, half ) );
    const double fy = floor( __fma_rn( vp, P.img_inv_pix, half ) );
    if( fx < 0.0 || fy < 0.0 || fx >= P.img_n || fy >= P.img_n )
        return -1;
    return ( int ) fy * P.img_n + ( int ) fx;
}

// Adds a peel-off contribution (intensity per steradian I and image-frame
// Q, U, V, already weighted) to image pixel `pix` (>= 0) and to the packet's
// batch image.
// Index of pixel `pixel` in the coarse per-batch image of batch `batch`
// (pixel i -> i * bn / n on each axis); computed once when a peel-off ray
// starts, so the deposit at its end is atomics only.
__device__ __forceinline__ int coarse_pixel( const fwd_params_t & P, int pixel, int batch )
{
    const int ix = pixel % P.img_n, iy = pixel / P.img_n;
    return ( batch * P.img_bn + iy * P.img_bn / P.img_n ) * P.img_bn + ix * P.img_bn / P.img_n;
}

template< int TALLY >
__device__ __forceinline__ void deposit_pixel( const fwd_params_t & P, int pixel, int cpix,
                                               float I, float Q, float U, float V )
{
    const size_t pix = ( size_t ) pixel * 4;
    add_tally< TALLY >( P.image, P.c_image, pix + 0, I, P.fx_scale );
    add_tally< TALLY >( P.image, P.c_image, pix + 1, Q, P.fx_scale );
    add_tally< TALLY >( P.image, P.c_image, pix + 2, U, P.fx_scale );
    add_tally< TALLY >( P.image, P.c_image, pix + 3, V, P.fx_scale );
    const size_t bp = ( size_t ) cpix * 4;
    add_tally< TALLY >( P.img_batch, P.c_img_batch, bp + 0, I, P.fx_scale );
    add_tally< TALLY >( P.img_batch, P.c_img_batch, bp + 1, Q, P.fx_scale );
    add_tally< TALLY >( P.img_batch, P.c_img_batch, bp + 2, U, P.fx_scale );
    add_tally< TALLY >( P.img_batch, P.c_img_batch, bp + 3, V, P.fx_scale );
}

// Double-valued deposit (adjoint gradients, flux): int64 fixed point, or the
// value rounded to float and added by float atomics (with a carry array,
// carrying their rounding error as atomic_add_carry does).
template< int TALLY >
__device__ __forceinline__ void add_grad( void * base, float * carry, size_t i, double v,
                                          double sc )
{
    if( TALLY == KP_TALLY_FIXED )
        atomicAdd( ( unsigned long long * ) base + i,
                   ( unsigned long long ) __double2ll_rn( __dmul_rn( v, sc ) ) );
    else
        atomic_add_carry( ( float * ) base, carry, i, ( float ) v );
}

template< int TALLY >
__device__ __forceinline__ void add_grad( void * base, size_t i, double v, double sc )
{
    add_grad< TALLY >( base, nullptr, i, v, sc );
}

// Adjoint score of a peel-off contribution: <dL/dimage[pix], (I, Q, U, V)>.
__device__ __forceinline__ float score( const fwd_params_t & P, int pix, float I, float Q,
                                        float U, float V )
{
    const float4 g = P.adj_img[ pix ];
    return __fadd_rn( __fadd_rn( __fadd_rn( __fmul_rn( g.x, I ), __fmul_rn( g.y, Q ) ),
                                 __fmul_rn( g.z, U ) ), __fmul_rn( g.w, V ) );
}

// Escape tally: mu = d.z bins, Stokes in the meridian frame (Q > 0 in the
// plane of d and +z).
template< int TALLY >
__device__ __forceinline__ bool tally_escape( const fwd_params_t & P, void * mu_base,
                                              float * carry, const packet_t & p, int batch )
{
    if( P.n_mu <= 0 ) return false;
    const float fb = floorf( __fmul_rn( __fsub_rn( p.d.z, P.mu_lo ), P.mu_inv_w ) );
    if( !( fb >= 0.0f && fb < ( float ) P.n_mu ) ) return false;
    const int bin = ( int ) fb;
    const phys::v3 e2 = phys::cross( p.d, p.e1 );
    float c2, s2;
    phys::double_angle( p.e1.z, e2.z, c2, s2 );
    float q = p.S.q, u = p.S.u;
    phys::rotate( q, u, c2, s2 );
    const size_t i = ( ( size_t ) batch * P.n_mu + bin ) * 4;
    add_tally< TALLY >( mu_base, carry, i + 0, p.w, P.fx_scale );
    add_tally< TALLY >( mu_base, carry, i + 1, __fmul_rn( p.w, q ), P.fx_scale );
    add_tally< TALLY >( mu_base, carry, i + 2, __fmul_rn( p.w, u ), P.fx_scale );
    add_tally< TALLY >( mu_base, carry, i + 3, __fmul_rn( p.w, p.S.v ), P.fx_scale );
    return true;
}

__device__ __forceinline__ float sample_tau( phys::rng_t & rng )
{
    const phys::u4 r = rng.next(  );
    return ( float ) ( -phys::kp_log( ( double ) phys::u01( r.x ) ) );
}

// Direction uniform on the sphere (emit 0) or with mu uniform in (0,1)
// about +z (emit 1); (cos phi, sin phi) from a point in the unit disk.
__device__ __forceinline__ phys::v3 sample_emission_dir( phys::rng_t & rng, int emit )
{
    float mu = 0.0f, a = 1.0f, b = 0.0f, r2 = 1.0f;
    for( int trial = 0; trial < 64; ++ trial )
    {
        const phys::u4 r = rng.next(  );
        mu = emit == KP_EMIT_UP_UNIFORM ? phys::u01( r.x ) : phys::usym( r.x );
        a  = phys::usym( r.y );
        b  = phys::usym( r.z );
        r2 = __fadd_rn( __fmul_rn( a, a ), __fmul_rn( b, b ) );
        if( r2 <= 1.0f && r2 > 0.0f ) break;
        a = 1.0f; b = 0.0f; r2 = 1.0f;
    }
    const float rr = __fsqrt_rn( r2 );
    return phys::dir_from( mu, __fdiv_rn( a, rr ), __fdiv_rn( b, rr ) );
}

// Cell of block b holding x: floor((x - xf0) / dx0) per axis, clamped to
// the block.
__device__ __forceinline__ void cell_of( const mesh_view_t & m, int b, const double x[ 3 ],
                                         int c[ 3 ] )
{
    const double * h = m.geo_d + 16 * ( size_t ) b;
    #pragma unroll
    for( int a = 0; a < 3; ++ a )
    {
        const double f = floor( __dmul_rn( __dsub_rn( x[ a ], h[ a ] ), h[ 8 + a ] ) );
        c[ a ] = f < 0.0 ? 0 : ( f > ( double ) ( m.nc[ a ] - 1 ) ? m.nc[ a ] - 1 : ( int ) f );
    }
}

// Block and cell holding x, through the finest-level lookup grid; false
// when no block is found there.
__device__ __forceinline__ bool locate_point( const fwd_params_t & P, const double x[ 3 ],
                                              int & b, int c[ 3 ] )
{
    int li[ 3 ];
    #pragma unroll
    for( int a = 0; a < 3; ++ a )
    {
        const double f = floor( __dmul_rn( __dsub_rn( x[ a ], P.m.xlim_d[ 0 ][ a ] ),
                                           P.lk_inv[ a ] ) );
        li[ a ] = f < 0.0 ? 0 : ( f >= P.m.lookup_n[ a ] ? P.m.lookup_n[ a ] - 1 : ( int ) f );
    }
    b = P.m.lookup[ ( ( size_t ) li[ 2 ] * P.m.lookup_n[ 1 ] + li[ 1 ] )
                    * P.m.lookup_n[ 0 ] + li[ 0 ] ];
    if( b < 0 || b >= P.m.n_blocks ) return false;
    cell_of( P.m, b, x, c );
    return true;
}

// Creates packet `pid` at source `s` with RNG key (seed, stream).  Returns
// false if the source position lies outside the mesh.
__device__ __forceinline__ bool emit_packet( const fwd_params_t & P, long long pid, packet_t & p,
                                             const src_dev_t & s, uint32_t stream )
{
    p.rng = phys::rng_t { P.seed, stream, ( uint32_t ) pid, ( uint32_t ) ( pid >> 32 ), 0u };
    if( s.kind == KP_SOURCE_POINT )
    {
        #pragma unroll
        for( int a = 0; a < 3; ++ a ) { p.x[ a ] = s.pos[ a ]; p.c[ a ] = s.cell[ a ]; }
        p.b = s.ib;
    }
    else
    {   // uniform over the domain's lower z face
        const phys::u4 r = p.rng.next(  );
        p.x[ 0 ] = __fma_rn( ( double ) phys::u01( r.x ), P.m.lbox_d[ 0 ], P.m.xlim_d[ 0 ][ 0 ] );
        p.x[ 1 ] = __fma_rn( ( double ) phys::u01( r.y ), P.m.lbox_d[ 1 ], P.m.xlim_d[ 0 ][ 1 ] );
        p.x[ 2 ] = P.m.xlim_d[ 0 ][ 2 ];
        if( ! locate_point( P, p.x, p.b, p.c ) ) return false;
    }
    if( p.b < 0 || p.b >= P.m.n_blocks ) return false;
    p.d  = sample_emission_dir( p.rng, s.emit );
    p.e1 = phys::frame_for( p.d );
    p.S  = phys::stokes_t { 0.0f, 0.0f, 0.0f };
    p.w  = 1.0f;
    p.n_scat  = 0;
    p.n_steps = 0;
    set_inv( p );
    return true;
}

// Packet (pid - pid0) that work index w of a launch of n packets walks:
// source-major order.  Packet pid starts from source pid % n_src, so the
// launch takes the packets of one source after another (slot j = 0 ..
// n_src - 1 holds k = j + m n_src, m = 0, 1, ...), and the packets in flight
// at any time start from one or two sources and share their part of the
// mesh in L2 instead of spreading over all of them.  The tallies (int64 sums)
// and the records (indexed by pid) do not depend on the order.  The
// identity for one source (and for a packet table, n_src = 1).
__device__ __forceinline__ long long source_major( long long w, long long n, int n_src )
{
    if( n_src <= 1 )
        return w;
    const long long q = n / n_src, r = n % n_src;
    long long j, m;
    if( w < r * ( q + 1 ) )
    {
        j = w / ( q + 1 );
        m = w % ( q + 1 );
    }
    else
    {
        const long long v = w - r * ( q + 1 );
        j = r + v / q;
        m = v % q;
    }
    return j + m * n_src;
}

// Creates packet `pid` of a single-mesh launch: from the caller's packet
// table when the launch has one (pid - pk_pid0 is its entry), else from
// source pid % n_src.  peel_I receives the emitted intensity per steradian
// toward the observer per unit weight, 0 for no peel-off ray at emission:
// 1 / (4 pi) for an isotropic point source, the entry's own for a table.
// Returns false when the packet's position lies in no block.
__device__ __forceinline__ bool emit_any( const fwd_params_t & P, long long pid, packet_t & p,
                                          float & peel_I )
{
    if( P.pk_table == nullptr )
    {
        const src_dev_t & s = P.src[ pid % P.n_src ];
        peel_I = s.kind == KP_SOURCE_POINT && s.emit == KP_EMIT_ISOTROPIC ? 0x1.45f306p-4f : 0.0f;
        return emit_packet( P, pid, p, s, P.stream );
    }
    const kp_packet_init_t & e = P.pk_table[ pid - P.pk_pid0 ];
    p.rng = phys::rng_t { P.seed, P.stream, ( uint32_t ) pid, ( uint32_t ) ( pid >> 32 ), 0u };
    #pragma unroll
    for( int a = 0; a < 3; ++ a ) p.x[ a ] = e.x[ a ];
    p.b = e.ib;
    if( p.b < 0 )
    {
        if( ! locate_point( P, p.x, p.b, p.c ) ) return false;
    }
    else
    {
        if( p.b >= P.m.n_blocks ) return false;
        cell_of( P.m, p.b, p.x, p.c );
    }
    p.d  = phys::v3 { e.d[ 0 ], e.d[ 1 ], e.d[ 2 ] };
    p.e1 = phys::frame_for( p.d );
    p.S  = phys::stokes_t { e.stokes[ 0 ], e.stokes[ 1 ], e.stokes[ 2 ] };
    p.w  = e.w;
    p.n_scat  = 0;
    p.n_steps = 0;
    set_inv( p );
    peel_I = e.peel_I;
    return true;
}

__device__ __forceinline__ void write_record( const fwd_params_t & P, const packet_t & p, int status )
{
    const long long k = p.pid(  ) - P.rec_pid0;
    if( P.records == nullptr || k < 0 || k >= P.n_record ) return;
    kp_packet_record_t * r = P.records + k;       // field by field: no local copy
    #pragma unroll
    for( int a = 0; a < 3; ++ a ) { r->x[ a ] = p.x[ a ]; r->cell[ a ] = p.c[ a ]; }
    r->d[ 0 ] = p.d.x; r->d[ 1 ] = p.d.y; r->d[ 2 ] = p.d.z;
    r->stokes[ 0 ] = p.S.q; r->stokes[ 1 ] = p.S.u; r->stokes[ 2 ] = p.S.v;
    r->w = p.w;
    r->ib = p.b;
    r->n_scatter = p.n_scat;
    r->status = status;
    r->rng_draws = p.rng.draw;
    r->n_steps = p.n_steps;
}

// Lane phases of the warp-synchronous transport kernels.
enum lane_phase { PH_EMIT = 0, PH_SEGMENT = 1, PH_EVENT = 2, PH_DONE = 3,
                  PH_HOP = 4 };          // waits for a batched block hand-off

// Segment counts stay in registers (32-bit: a thread walks far fewer than
// 2^32 segments in one launch); rare events are counted in shared memory.
struct counts32_t
{
    unsigned steps = 0, peel = 0;
};

constexpr int FWD_THREADS = 256;

// Rarely touched per-lane state kept in shared memory (structure of arrays):
// the parked walk position while a peel-off ray runs, and the pending
// peel-off contribution.
template< int NT = FWD_THREADS >
struct park_t
{
    double x[ 3 ][ NT ];
    int    c[ 3 ][ NT ];
    int    b[ NT ];
    float  w[ NT ], I[ NT ], Q[ NT ], U[ NT ], V[ NT ];
    int    pix[ NT ];
    unsigned long long cnt[ KP_NCOUNTERS ];
};

template< class SP >
__device__ __forceinline__ void park_walk( SP & sp, const packet_t & p )
{
    const int t = threadIdx.x;
    #pragma unroll
    for( int a = 0; a < 3; ++ a ) { sp.x[ a ][ t ] = p.x[ a ]; sp.c[ a ][ t ] = p.c[ a ]; }
    sp.b[ t ] = p.b;
}
template< class SP >
__device__ __forceinline__ void unpark_walk( const SP & sp, packet_t & p )
{
    const int t = threadIdx.x;
    #pragma unroll
    for( int a = 0; a < 3; ++ a ) { p.x[ a ] = sp.x[ a ][ t ]; p.c[ a ] = sp.c[ a ][ t ]; }
    p.b = sp.b[ t ];
}
// One event for counter k: the lanes that count the same k together add
// with one shared atomic (lanes of a batch would otherwise serialise on it).
template< class SP >
__device__ __forceinline__ void count( SP & sp, int k )
{
    const unsigned m = __match_any_sync( __activemask(  ), k );
    if( ( threadIdx.x & 31u ) == ( unsigned ) ( __ffs( m ) - 1 ) )
        atomicAdd( sp.cnt + k, ( unsigned long long ) __popc( m ) );
}
// v events per lane for counter k, all lanes of the warp together (after
// the scheduling loop).
template< class SP >
__device__ __forceinline__ void count_all( SP & sp, int k, unsigned v )
{
    const unsigned s = __reduce_add_sync( 0xffffffffu, v );
    if( ( threadIdx.x & 31u ) == 0 && s )
        atomicAdd( sp.cnt + k, ( unsigned long long ) s );
}

// Host helpers shared by the transport entry points (kp_transport.cu).
void make_fwd_params( kp_mesh_t * mesh, const kp_transport_cfg_t & c,
                      const kp_tallies_t & t, fwd_params_t & P );
void fill_common_params( const kp_transport_cfg_t & c, const kp_tallies_t & t,
                         fwd_params_t & P );
void make_source( kp_mesh_t * mesh, const kp_source_t & s, src_dev_t & d );
int  persistent_grid( const void * kernel, int threads );
void launch_peel_adjoint( const fwd_params_t & P, int tally_mode, int mode, cudaStream_t s );
constexpr int PQ_PER_PACKET = 12;    // peel-off queue rays per packet of a solve
void ensure_peel_queue( kp_mesh_t * mesh, long long n_packets );
// Points P's queue and deferred-adjoint fields at the mesh's buffers (grown
// for chunks of n_pk packets), with their own counters: P.work is set to
// them, so launches that use the mesh's workspace do not touch a tape.
void adjoint_buffers( kp_mesh_t * mesh, fwd_params_t & P, long long n_pk );
// The march order of the mesh's queue (kp_mesh_peel_order): whether to
// sort it by starting cell, the sort's buffers (returns the permutation),
// and the sort of the queue P describes into P.pq_perm.
bool peel_sorted( const kp_mesh_t * mesh );
int * ensure_task_sort( kp_mesh_t * mesh, long long pq_cap );
void task_sort( const kp_mesh_t * mesh, const fwd_params_t & P, cudaStream_t s );
// The walk of one chunk, then the march of its queue (in P.pq_perm's order
// when set, sorted first with the mesh's buffers).
template< int TALLY, bool TAPE, bool RESUME = false >
void launch_deferred_chunk( fwd_params_t & P, cudaStream_t s, const kp_mesh_t * mesh = nullptr );
// A forward solve with its peel-off rays queued for k_peel, in chunks (no tape).
void launch_deferred_solve( kp_mesh_t * mesh, const fwd_params_t & P, int tally_mode,
                            cudaStream_t s );
void launch_forward( const fwd_params_t & P, int tally_mode, cudaStream_t s, int threads,
                     int grid_pct );

}   // namespace kp
