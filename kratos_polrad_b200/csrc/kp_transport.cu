// Forward polarized transport: persistent kernel with packet regeneration.
//
// Replaces the reference's per-cycle generate + integrate launches
// (modules/particle/evolve/generate_par.h:51-62 -> ker_gen, then
// evolve/integrator.h:47-63 -> ker_itg running photon::cart_t::proc) by one
// persistent launch: every thread walks one packet at a time, segment by
// segment, and when its packet ends (escape, absorption) it takes the next
// packet index from a global counter.  Lanes that need new packets in the
// same iteration take them with one warp-aggregated atomic (the warp's
// coalesced group ballots, its leader adds the group size), so the warp
// stays full while packet lifetimes differ by orders of magnitude.
#include "kp_transport.cuh"

#include <cub/cub.cuh>

namespace kp
{
namespace
{
namespace cg = cooperative_groups;


// Warp-synchronous scheduler.  Each lane carries one packet through a small
// state machine: EMIT (needs a packet), SEGMENT (advance its active ray by
// one cell segment: the packet's own walk, or a peel-off ray toward the
// observer), EVENT (an interaction to process), HOP (its ray left the block:
// neighbour lookup and the new block's geometry).  Every iteration the warp
// ballots the lane phases and runs ONE phase for all lanes in it: events,
// emissions and hand-offs, which are long and rare, wait until at least
// `ev_batch` (hand-offs: `hop_batch`) lanes need them, or no lane can step,
// so their code runs with many lanes active and their dependent loads are
// paid once per batch; segments, which are short and frequent, run
// otherwise.  A hand-off left inline cost as much as 11 segments, because
// the whole warp waited on one lane's chain of dependent loads.  A peel-off
// ray starts at an emission or interaction point: the walk position is
// parked, the ray marches to the boundary (or beyond tau_cut), its
// contribution is deposited and the walk resumes.  Peel-off rays draw no
// random numbers, so each packet's history equals a sequential walk that
// marches every peel-off ray at the moment of its interaction.
#ifndef KP_PEEL_BATCH
#define KP_PEEL_BATCH 24             // k_peel: lanes that wait for a fetch batch
#endif
#ifndef KP_HOP_BATCH
#define KP_HOP_BATCH 6               // lanes that wait for a batched block hand-off
#endif
#ifndef KP_EMIT_BATCH
#define KP_EMIT_BATCH 0              // lanes that wait for an emission batch (0: the event batch)
#endif
#ifndef KP_PEEL_INNER
#define KP_PEEL_INNER 16             // k_peel: segments per scheduling round
#endif
#ifndef KP_PEEL_INNER_ADJ
#define KP_PEEL_INNER_ADJ 8          // ... in the adjoint's marches (modes 1, 2): 4
                                     // and 16 are slower there
#endif
#ifndef KP_PEEL_MINB
#define KP_PEEL_MINB 4               // k_peel: resident blocks of 256 the registers allow
#endif
#ifndef KP_FWD_RESIDENT
#define KP_FWD_RESIDENT 768          // resident threads per SM the register budget targets
#endif

// DD: one round of a domain-decomposed solve.  Work items are, in order, the
// incoming walks, the incoming peel-off rays (run alone: no walk parked) and
// this rank's emissions; a ray handed off into a block of another rank is
// written to that rank's out-queue instead of continuing.  Each packet's
// arithmetic is that of the replicated solve.
// DEFER: a peel-off ray is written to the task queue for k_peel (when it
// has room) instead of being marched here; the walk continues at once.
// TAPE (with DEFER): the rays are also linked per packet, in vertex order,
// for the adjoint of this solve (kp_transport_adjoint_tape); a packet with a
// ray that found the queue full is flagged and listed instead.
// FLUX: every walk segment adds w * dl / volume to its cell's flux tally,
// the path-length estimator of photon::cart_t::proc_phys
// (modules/particle/radiation/photon.h:73-83) with the packet's weight as
// its `proper`; w / volume of the walk's block waits in shared memory (set
// at emission, interactions and block hand-offs), so a segment adds one
// multiply and one atomic.
// RESUME (not with DD or TAPE): work items are first the packets an earlier
// call suspended (P.rs_in), then the call's new packets; a packet that has
// walked P.rs_budget segments in this launch (and is below max_steps) is
// written whole to P.rs_out and left for a later call instead of ending.
// Its arithmetic is that of an uninterrupted walk: the face cache and the
// inverse direction are rebuilt bit for bit from the stored state.
template< int TALLY, int NT, bool DD = false, bool DEFER = false, bool TAPE = false,
          bool FLUX = false, bool RESUME = false >
__global__ void __launch_bounds__( NT, KP_FWD_RESIDENT / NT )
k_forward( const __grid_constant__ fwd_params_t P )
{
    static_assert( ! ( RESUME && ( DD || TAPE ) ), "RESUME runs without DD and TAPE" );
    __shared__ park_t< NT > sp;
    __shared__ dir_park_t< NT > sd;
    __shared__ cold_park_t< NT > sc;
    // RESUME: the lane's packet stops (suspends or, at max_steps, ends) when
    // its n_steps reaches this
    __shared__ int s_stop[ RESUME ? NT : 1 ];
    const unsigned FULL = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31u;
    if( threadIdx.x < KP_NCOUNTERS ) sp.cnt[ threadIdx.x ] = 0;
    __syncthreads(  );
    counts32_t cnt;
    packet_t p;
    double fx[ 3 ];                               // face cache of the active ray
    int  phase = PH_EMIT;
    bool peel = false;            // the lane runs a peel-off ray: p.x holds its start,
    float ptau = 0;               // fx the distances to its cell's faces (oray_faces)
    double ptc = 0.0;             // ... and ptc the distance it has travelled
    int pk = 0, pend = 0;
    int si = 0;                                   // scene of a batched launch
    int hop_ax = 0;                               // face axis of a pending hand-off
    bool solo = false;                            // DD: peel-off ray without a parked walk
    int tlink = -1;                               // TAPE: the packet's last task (-2: flagged)

    // DEFER: appends the peel-off ray of vertex kv prepared in sp/sd
    // (starting at p's position) to the queue; false when the queue is full.
    // The lanes that append together take their slots with one atomic.
    auto defer_peel = [ & ]( int kv ) -> bool
    {
        const unsigned m = __activemask(  );
        const int leader = __ffs( m ) - 1;
        unsigned long long base = 0;
        if( ( int ) lane == leader )
            base = atomicAdd( P.pq_count, ( unsigned long long ) __popc( m ) );
        base = __shfl_sync( m, base, leader );
        const unsigned long long k = base + __popc( m & ( ( 1u << lane ) - 1u ) );
        const int lp = TAPE ? ( int ) ( p.pid(  ) - P.pid0 ) : 0;
        if( k >= ( unsigned long long ) P.pq_cap )
        {
            if constexpr( TAPE )
                if( tlink != -2 )
                {   // the adjoint replays this packet with its rays inline
                    tlink = -2;
                    P.adj_flag[ lp ] = 1;
                    P.adj_list[ atomicAdd( P.adj_list_n, 1ull ) ] = lp;
                }
            return false;
        }
        const int t = threadIdx.x;
        store_task( P.pq, k, p.x, p.b, p.c, sp.w[ t ], sp.I[ t ], sp.Q[ t ], sp.U[ t ], sp.V[ t ],
                    sp.pix[ t ], sd.cpix[ t ] );
        if constexpr( TAPE )
        {
            P.pq_link[ k ] = peel_link_t { lp, kv, -1 };
            if( tlink >= 0 ) P.pq_link[ tlink ].next = ( int ) k;
            else P.adj_head[ lp ] = ( int ) k;
            tlink = ( int ) k;
        }
        return true;
    };

    // A peel-off ray marched by this lane at once from the packet's position
    // (its contribution is in sp / sd): every ray of the single-kernel walk,
    // and the rays that find the queue full in the deferred one.  Only the
    // decomposed rounds schedule their rays segment by segment with the walk
    // (a ray may cross into another rank's block mid-way).
    auto peel_now = [ & ](  )
    {
        unsigned segs = 0, hops = 0;
        const float tau = oray_march( P, p.b, p.c, p.x, segs, hops );
        cnt.peel += segs;
        if( hops )
            atomicAdd( sp.cnt + KP_CNT_HOPS, ( unsigned long long ) hops );
        if( tau <= P.tau_cut )
        {
            const int th = threadIdx.x;
            const float att = __fmul_rn( sp.w[ th ], ( float ) phys::kp_exp_neg( -( double ) tau ) );
            deposit_pixel< TALLY >( P, sp.pix[ th ], sd.cpix[ th ], __fmul_rn( att, sp.I[ th ] ),
                                    __fmul_rn( att, sp.Q[ th ] ), __fmul_rn( att, sp.U[ th ] ),
                                    __fmul_rn( att, sp.V[ th ] ) );
            count( sp, KP_CNT_DEPOSITS );
        }
    };

    // coefficients of cell c of block b (DD: owned blocks stored compactly)
    auto sigma_at = [ & ]( int b, const int c[ 3 ] ) -> float2
    {
        if constexpr( DD )
        {
            const int l = P.dd_loc[ b ];
            if( l < 0 )
            {   // a block of another rank: never read here by construction
                atomicOr( P.m.status, ST_BAD_BLOCK );
                return make_float2( 0.0f, 0.0f );
            }
            return P.m.sigma[ ( size_t ) l * P.m.cpb + c[ 0 ]
                              + P.m.nc[ 0 ] * ( c[ 1 ] + P.m.nc[ 1 ] * c[ 2 ] ) ];
        }
        else
            return P.m.sigma[ cell_index( P.m, b, c ) ];
    };
    // extinction of cell c of block b (the float sum of its coefficients)
    auto ext_at = [ & ]( int b, const int c[ 3 ] ) -> float
    {
        if constexpr( DD )
        {
            const float2 sg = sigma_at( b, c );
            return __fadd_rn( sg.x, sg.y );
        }
        else
            return P.m.ext[ cell_index( P.m, b, c ) ];
    };

    // FLUX: w / volume of block b for the walk's later segments
    auto set_wv = [ & ]( float w, int b )
    {
        if constexpr( FLUX )
            sc.wv[ threadIdx.x ] = __ddiv_rn( ( double ) w, P.m.geo_d[ 16 * ( size_t ) b + 6 ] );
    };
    // FLUX: deposit of the walk's segment of length dl in its current cell
    // (DD: the rank's own blocks, stored compactly like the coefficients)
    auto add_flux = [ & ]( double dl )
    {
        if constexpr( FLUX )
        {
            size_t i;
            if constexpr( DD )
            {
                const int l = P.dd_loc[ p.b ];
                if( l < 0 ) return;                      // flagged by sigma_at
                i = ( size_t ) l * P.m.cpb + p.c[ 0 ] + P.m.nc[ 0 ] * ( p.c[ 1 ] + P.m.nc[ 1 ] * p.c[ 2 ] );
            }
            else
                i = cell_index( P.m, p.b, p.c );
            add_grad< TALLY >( P.flux, P.c_flux, i, __dmul_rn( dl, sc.wv[ threadIdx.x ] ),
                               P.flux_scale );
        }
    };

    // A whole walk (dd_walk_t) becomes the lane's packet: one arriving from
    // another rank (DD), or one an earlier call suspended (RESUME).
    auto load_walk = [ & ]( const dd_walk_t & o )
    {
        const int t = threadIdx.x;
        for( int a = 0; a < 3; ++ a ) { p.x[ a ] = o.x[ a ]; p.c[ a ] = o.c[ a ]; }
        p.d = phys::v3 { o.d[ 0 ], o.d[ 1 ], o.d[ 2 ] };
        p.e1 = phys::v3 { o.e1[ 0 ], o.e1[ 1 ], o.e1[ 2 ] };
        p.S = phys::stokes_t { o.S[ 0 ], o.S[ 1 ], o.S[ 2 ] };
        p.w = o.w; p.tau = o.tau; p.b = o.b;
        p.n_scat = o.n_scat; p.n_steps = o.n_steps;
        p.rng = phys::rng_t { P.seed, o.k1, o.pid_lo, o.pid_hi, o.draw };
        sc.batch[ t ] = o.batch;
        set_inv( p );
        store_cold( sc, p );
        set_wv( p.w, p.b );
        faces_all( P.m, p.b, p.c, p.d, fx );
    };
    // The lane's whole packet (its cold state loaded) into a walk record.
    auto store_walk = [ & ]( dd_walk_t & o )
    {
        for( int a = 0; a < 3; ++ a ) { o.x[ a ] = p.x[ a ]; o.c[ a ] = p.c[ a ]; }
        o.d[ 0 ] = p.d.x; o.d[ 1 ] = p.d.y; o.d[ 2 ] = p.d.z;
        o.e1[ 0 ] = p.e1.x; o.e1[ 1 ] = p.e1.y; o.e1[ 2 ] = p.e1.z;
        o.S[ 0 ] = p.S.q; o.S[ 1 ] = p.S.u; o.S[ 2 ] = p.S.v;
        o.w = p.w; o.tau = p.tau; o.b = p.b;
        o.n_scat = p.n_scat; o.n_steps = p.n_steps;
        o.k1 = p.rng.k1; o.pid_lo = p.rng.pid_lo; o.pid_hi = p.rng.pid_hi;
        o.draw = p.rng.draw; o.batch = sc.batch[ threadIdx.x ];
    };
    // RESUME: the packet (cold state loaded) leaves this launch unfinished.
    auto suspend = [ & ](  )
    {
        const unsigned long long k = atomicAdd( P.rs_count, 1ull );
        if( k < ( unsigned long long ) P.rs_cap )
            store_walk( P.rs_out[ k ] );
        else
            atomicOr( P.m.status, ST_QUEUE_FULL );
        phase = PH_EMIT;
    };

    // After the active ray crossed a face (or stopped): the end of a peel-off
    // ray (deposit, walk resumes) or of the packet's walk (escape, step cap,
    // or, RESUME, the end of this launch's step budget).
    // Shared by the segment phase and the hand-off phase.
    auto after_crossing = [ & ]( bool peel_cut, bool left, bool lost )
    {
        if( peel )
        {
            if( peel_cut || left || pk >= ( 1 << 20 ) )
            {
                if( ptau <= P.tau_cut )
                {
                    const int th = threadIdx.x;
                    const float att = __fmul_rn( sp.w[ th ],
                                                 ( float ) phys::kp_exp_neg( -( double ) ptau ) );
                    deposit_pixel< TALLY >( P, sp.pix[ th ], sd.cpix[ th ], __fmul_rn( att, sp.I[ th ] ),
                                            __fmul_rn( att, sp.Q[ th ] ), __fmul_rn( att, sp.U[ th ] ),
                                            __fmul_rn( att, sp.V[ th ] ) );
                    count( sp, KP_CNT_DEPOSITS );
                }
                if constexpr( DD )
                {
                    if( solo )
                    {
                        peel = false; solo = false;
                        phase = PH_EMIT;
                        return;
                    }
                }
                unpark_walk( sp, p );
                unpark_dir( sd, p );
                faces_all( P.m, p.b, p.c, p.d, fx );
                peel = false;
                if( pend )
                {
                    load_cold( sc, p, P.seed );
                    write_record( P, p, pend );
                    count( sp, pend == PK_ABSORBED ? KP_CNT_ABSORBED : KP_CNT_CAPPED );
                    phase = PH_EMIT;
                }
            }
            return;
        }
        int end = 0;
        if( left )
        {
            load_cold( sc, p, P.seed );
            if( lost )
                end = PK_LOST;
            else
            {
                end = PK_ESCAPED;
                if( tally_escape< TALLY >( P, ( char * ) P.mu_tally + ( size_t ) si * P.mu_scene_stride
                                             * ( TALLY == KP_TALLY_FIXED ? 8 : 4 ), P.c_mu, p,
                                             sc.batch[ threadIdx.x ] ) )
                    count( sp, KP_CNT_DEPOSITS );
            }
        }
        else if( p.n_steps >= ( RESUME ? ( long long ) s_stop[ threadIdx.x ] : P.max_steps ) )
        {
            load_cold( sc, p, P.seed );
            if( RESUME && p.n_steps < P.max_steps )
            {
                suspend(  );
                return;
            }
            end = PK_STEP_CAP;
        }
        if( end )
        {
            write_record( P, p, end );
            count( sp, end == PK_ESCAPED ? KP_CNT_ESCAPED
                     : ( end == PK_LOST ? KP_CNT_LOST : KP_CNT_CAPPED ) );
            phase = PH_EMIT;
        }
    };

    for( ;; )
    {
        const unsigned m_emit = __ballot_sync( FULL, phase == PH_EMIT );
        const unsigned m_seg  = __ballot_sync( FULL, phase == PH_SEGMENT );
        const unsigned m_ev   = __ballot_sync( FULL, phase == PH_EVENT );
        const unsigned m_hop  = __ballot_sync( FULL, phase == PH_HOP );
        if( ( m_emit | m_seg | m_ev | m_hop ) == 0u )
            break;
        const int n_seg = __popc( m_seg ), n_ev = __popc( m_ev ), n_emit = __popc( m_emit );
        const int n_hop = __popc( m_hop );
        int run;
        if( n_ev > 0 && ( n_ev >= P.ev_batch || n_seg == 0 ) )
            run = PH_EVENT;
        else if( n_emit > 0 && ( n_emit >= ( P.emit_batch > 0 ? P.emit_batch : P.ev_batch )
                                 || n_seg == 0 ) )
            run = PH_EMIT;
        else if( n_hop > 0 && ( n_hop >= P.hop_batch || n_seg == 0 ) )
            run = PH_HOP;
        else
            run = PH_SEGMENT;

        if( run == PH_HOP )
        {   // block hand-offs of the lanes that left their block, together:
            // neighbour lookup and the new block's geometry in one batch
            if( phase != PH_HOP ) continue;
            const int b_old = p.b;
            bool lost, left;
            if( peel )      // a peel-off ray: rebased at its crossing point
                left = ! oray_rebase( P, p.b, p.c, p.x, ptc, fx, hop_ax, lost );
            else
                left = ! cross_face( P.m, p.b, p.c, p.x, hop_ax, comp( p.d, hop_ax ) > 0.0f, lost );
            if( ! left )
            {
                if( p.b != b_old ) count( sp, KP_CNT_HOPS );
                if constexpr( DD )
                {
                    const int r = P.dd_owner[ p.b ];
                    // a ray that used its last segment ends here, as in the
                    // replicated solve (after_crossing below): no hand-over
                    const bool capped = peel ? pk >= ( 1 << 20 ) : p.n_steps >= P.max_steps;
                    if( r != P.dd_rank && ! capped )
                    {   // the ray continues on rank r
                        const int t = threadIdx.x;
                        if( peel )
                        {
                            const unsigned long long k = atomicAdd( P.dd_out_count + 1, 1ull );
                            if( k < ( unsigned long long ) P.dd_cap_peel )
                            {
                                P.dd_out_peel_rank[ k ] = r;
                                dd_peel_t & o = P.dd_out_peel[ k ];
                                for( int a = 0; a < 3; ++ a ) { o.x[ a ] = p.x[ a ]; o.c[ a ] = p.c[ a ]; }
                                o.b = p.b; o.ptau = ptau; o.pk = pk; o.tc = ptc;
                                o.w = sp.w[ t ]; o.I = sp.I[ t ]; o.Q = sp.Q[ t ]; o.U = sp.U[ t ];
                                o.V = sp.V[ t ]; o.pix = sp.pix[ t ]; o.cpix = sd.cpix[ t ];
                            }
                            else
                                atomicOr( P.m.status, ST_QUEUE_FULL );
                            peel = false;
                            if( solo )
                            {
                                solo = false;
                                phase = PH_EMIT;
                                continue;
                            }
                            unpark_walk( sp, p );
                            unpark_dir( sd, p );
                            faces_all( P.m, p.b, p.c, p.d, fx );
                            phase = PH_SEGMENT;
                            if( pend )
                            {
                                count( sp, pend == PK_ABSORBED ? KP_CNT_ABSORBED : KP_CNT_CAPPED );
                                phase = PH_EMIT;
                            }
                            continue;
                        }
                        const unsigned long long k = atomicAdd( P.dd_out_count, 1ull );
                        if( k < ( unsigned long long ) P.dd_cap_walk )
                        {
                            load_cold( sc, p, P.seed );
                            P.dd_out_walk_rank[ k ] = r;
                            store_walk( P.dd_out_walk[ k ] );
                        }
                        else
                            atomicOr( P.m.status, ST_QUEUE_FULL );
                        phase = PH_EMIT;
                        continue;
                    }
                }
                if( ! peel )
                {
                    if( p.b != b_old ) set_wv( sc.w[ threadIdx.x ], p.b );
                    faces_all( P.m, p.b, p.c, p.d, fx );
                }
            }
            phase = PH_SEGMENT;
            after_crossing( false, left, lost );
            continue;
        }

        if( run == PH_EMIT )
        {
            if( phase != PH_EMIT ) continue;
            const int leader = __ffs( m_emit ) - 1;
            const unsigned rank = __popc( m_emit & ( ( 1u << lane ) - 1u ) );
            unsigned long long base = 0;
            if( ( int ) lane == leader )
                base = atomicAdd( P.work, ( unsigned long long ) n_emit );
            base = __shfl_sync( m_emit, base, leader );
            unsigned long long idx = base + rank;
            if constexpr( DD )
            {
                const unsigned long long nw = P.dd_n_walk, npl = P.dd_n_peel;
                if( idx >= nw + npl + ( P.dd_emit ? ( unsigned long long ) P.n_packets : 0ull ) )
                {
                    phase = PH_DONE;
                    continue;
                }
                const int t = threadIdx.x;
                if( idx < nw )
                {   // a walk arriving from another rank
                    load_walk( P.dd_in_walk[ idx ] );
                    peel = false; solo = false;
                    phase = PH_SEGMENT;
                    continue;
                }
                if( idx < nw + npl )
                {   // a peel-off ray arriving from another rank
                    const dd_peel_t & o = P.dd_in_peel[ idx - nw ];
                    for( int a = 0; a < 3; ++ a )
                    {
                        p.x[ a ] = o.x[ a ]; p.c[ a ] = o.c[ a ]; p.inv[ a ] = P.inv_o[ a ];
                    }
                    p.b = o.b; p.d = P.o;
                    ptau = o.ptau; pk = o.pk; ptc = o.tc;
                    sp.w[ t ] = o.w; sp.I[ t ] = o.I; sp.Q[ t ] = o.Q; sp.U[ t ] = o.U;
                    sp.V[ t ] = o.V; sp.pix[ t ] = o.pix; sd.cpix[ t ] = o.cpix;
                    oray_faces( P, p.b, p.c, p.x, fx );
                    peel = true; solo = true; pend = 0;
                    phase = PH_SEGMENT;
                    continue;
                }
                idx -= nw + npl;
                // each packet is emitted once over the ranks: point sources by
                // the owner of the source's block, plane sources and the
                // caller's packets by pid modulo
                const long long pid = P.pid0 + ( long long ) idx;
                const bool point = P.pk_table == nullptr
                                && P.src[ pid % P.n_src ].kind == KP_SOURCE_POINT;
                if( point ? P.dd_owner[ P.src[ pid % P.n_src ].ib ] != P.dd_rank
                          : ( int ) ( pid % P.dd_ranks ) != P.dd_rank )
                    continue;
            }
            else
            {
                if constexpr( RESUME )
                {
                    if( idx < ( unsigned long long ) P.rs_n_in )
                    {   // a packet suspended by an earlier call goes on
                        load_walk( P.rs_in[ idx ] );
                        s_stop[ threadIdx.x ] = ( int ) min( P.max_steps,
                                                             ( long long ) p.n_steps + P.rs_budget );
                        phase = PH_SEGMENT;
                        continue;
                    }
                    idx -= ( unsigned long long ) P.rs_n_in;
                }
                if( idx >= ( unsigned long long ) P.n_packets )
                {
                    phase = PH_DONE;
                    continue;
                }
            }
            bool ok;
            float peel_I = 0.0f;          // emission's intensity toward the observer
            if( P.n_scenes > 0 )
            {   // batched launch: scene of this packet index, then its local id
                int lo = 0, hi = P.n_scenes;
                while( hi - lo > 1 )
                {
                    const int mid = ( lo + hi ) >> 1;
                    if( ( long long ) idx >= P.scene_prefix[ mid ] ) lo = mid; else hi = mid;
                }
                si = lo;
                const long long pid = P.pid0 + ( ( long long ) idx - P.scene_prefix[ si ] );
                const src_dev_t & s = P.scenes[ si ].src;
                ok = emit_packet( P, pid, p, s, P.scenes[ si ].stream );
                peel_I = s.kind == KP_SOURCE_POINT && s.emit == KP_EMIT_ISOTROPIC ? 0x1.45f306p-4f
                                                                                  : 0.0f;
            }
            else if constexpr( DD )
                ok = emit_any( P, P.pid0 + ( long long ) idx, p, peel_I );
            else
                ok = emit_any( P, P.pid0 + source_major( ( long long ) idx, P.n_packets, P.n_src ),
                               p, peel_I );
            if( ! ok )
            {
                atomicOr( P.m.status, ST_BAD_SOURCE );
                continue;
            }
            count( sp, KP_CNT_EMITTED );
            if constexpr( TAPE ) tlink = -1;     // a new packet: its list starts empty
            sc.batch[ threadIdx.x ] = ( int ) ( p.pid(  ) % P.n_batch );
            p.tau = sample_tau( p.rng );
            phase = PH_SEGMENT;
            if constexpr( DD )
            {
                const int r = P.dd_owner[ p.b ];
                if( r != P.dd_rank )
                {   // emitted into a block of rank r (plane sources, caller-made
                    // packets): hand it over, with the direct light of the
                    // emission as a peel-off ray that starts there
                    if( P.img_n > 0 && peel_I > 0.0f )
                    {
                        const int pix = image_pixel( P, p.x );
                        if( pix >= 0 )
                        {
                            const unsigned long long k = atomicAdd( P.dd_out_count + 1, 1ull );
                            if( k < ( unsigned long long ) P.dd_cap_peel )
                            {
                                P.dd_out_peel_rank[ k ] = r;
                                dd_peel_t & o = P.dd_out_peel[ k ];
                                for( int a = 0; a < 3; ++ a ) { o.x[ a ] = p.x[ a ]; o.c[ a ] = p.c[ a ]; }
                                o.b = p.b; o.ptau = 0.0f; o.pk = 0; o.tc = 0.0;
                                o.w = p.w; o.I = peel_I; o.Q = o.U = o.V = 0.0f;
                                o.pix = pix; o.cpix = coarse_pixel( P, pix, sc.batch[ threadIdx.x ] );
                            }
                            else
                                atomicOr( P.m.status, ST_QUEUE_FULL );
                        }
                    }
                    const unsigned long long k = atomicAdd( P.dd_out_count, 1ull );
                    if( k < ( unsigned long long ) P.dd_cap_walk )
                    {
                        P.dd_out_walk_rank[ k ] = r;
                        store_walk( P.dd_out_walk[ k ] );
                    }
                    else
                        atomicOr( P.m.status, ST_QUEUE_FULL );
                    phase = PH_EMIT;
                    continue;
                }
            }
            if( P.img_n > 0 && peel_I > 0.0f )
            {   // direct light of the emission (unpolarized)
                const int pix = image_pixel( P, p.x );
                if( pix >= 0 )
                {
                    const int t = threadIdx.x;
                    sp.w[ t ] = p.w; sp.I[ t ] = peel_I;
                    sp.Q[ t ] = sp.U[ t ] = sp.V[ t ] = 0.0f;
                    sp.pix[ t ] = pix;
                    sd.cpix[ t ] = coarse_pixel( P, pix, sc.batch[ t ] );
                    if constexpr( DEFER )
                    {
                        if( ! defer_peel( 0 ) )
                            peel_now(  );
                    }
                    else if constexpr( ! DD )
                        peel_now(  );
                    else
                    {
                        pend = 0; ptau = 0.0f; pk = 0; ptc = 0.0;
                        park_walk( sp, p );
                        park_dir( sd, p, P.o, P.inv_o );
                        peel = true;
                    }
                }
            }
            if( peel )
                oray_faces( P, p.b, p.c, p.x, fx );
            else
                faces_all( P.m, p.b, p.c, p.d, fx );
            store_cold( sc, p );
            set_wv( p.w, p.b );
            if constexpr( RESUME )
                s_stop[ threadIdx.x ] = ( int ) min( P.max_steps, ( long long ) P.rs_budget );
            continue;
        }

        if( run == PH_EVENT )
        {
            if( phase != PH_EVENT ) continue;
            load_cold( sc, p, P.seed );
            // interaction at p.x (already moved there by its segment)
            ++ p.n_scat;
            count( sp, KP_CNT_SCATTER );
            {
                const float2 sg = sigma_at( p.b, p.c );
                p.w = __fmul_rn( p.w, __fdiv_rn( sg.x, __fadd_rn( sg.x, sg.y ) ) );
            }   // survival weighting by the albedo
            bool do_peel = false;
            if( P.img_n > 0 )
            {
                const int pix = image_pixel( P, p.x );
                if( pix >= 0 )
                {
                    const int t = threadIdx.x;
                    float Q, U, V;
                    sp.I[ t ] = phys::peel_stokes( P.ph, p.d, p.e1, p.S, P.o, P.ev, P.eh, Q, U, V );
                    sp.Q[ t ] = Q; sp.U[ t ] = U; sp.V[ t ] = V;
                    sp.w[ t ] = p.w;
                    sp.pix[ t ] = pix;
                    sd.cpix[ t ] = coarse_pixel( P, pix, sc.batch[ t ] );
                    do_peel = true;
                }
            }
            int end = 0;
            if( p.n_scat >= P.max_scatter )
                end = PK_SCATTER_CAP;
            else if( p.w < P.w_min )
            {   // Russian roulette
                const phys::u4 r = p.rng.next(  );
                if( phys::u01( r.x ) < P.rr_survive )
                    p.w = __fdiv_rn( p.w, P.rr_survive );
                else
                    end = PK_ABSORBED;
            }
            if( ! end )
            {
                phys::scatter( P.ph, p.rng, p.d, p.e1, p.S );
                set_inv( p );
                p.tau = sample_tau( p.rng );
            }
            if( ! end && p.n_steps >= P.max_steps )
                end = PK_STEP_CAP;
            if constexpr( ! DD )
                if( do_peel )
                {   // queued, or marched here: the walk goes on (or ends) now
                    if( ! DEFER || ! defer_peel( p.n_scat ) )
                        peel_now(  );
                    do_peel = false;
                }
            if( do_peel )
            {
                park_walk( sp, p );
                park_dir( sd, p, P.o, P.inv_o );
                ptau = 0.0f; pk = 0; pend = end; ptc = 0.0;
                peel = true;
                phase = PH_SEGMENT;
            }
            else if( end )
            {
                write_record( P, p, end );
                count( sp, end == PK_ABSORBED ? KP_CNT_ABSORBED : KP_CNT_CAPPED );
                phase = PH_EMIT;
            }
            else if( RESUME && p.n_steps >= s_stop[ threadIdx.x ] )
                suspend(  );             // the budget ran out with this segment
            else
                phase = PH_SEGMENT;
            if( phase == PH_SEGMENT )
            {
                if( peel )
                    oray_faces( P, p.b, p.c, p.x, fx );
                else
                    faces_all( P.m, p.b, p.c, p.d, fx );
                store_cold( sc, p );
                set_wv( p.w, p.b );
            }
            continue;
        }

        // ---- PH_SEGMENT: segments of the active ray, up to KP_WALK_INNER
        // before the next scheduling round where no peel-off ray is
        // scheduled here (all but the decomposed rounds) ----
        if( phase != PH_SEGMENT ) continue;
        #pragma unroll 1
        for( int it = 0; it < ( DD ? 1 : ( FLUX ? KP_WALK_INNER_FLUX : KP_WALK_INNER ) ); ++ it )
        {
            // the active ray's direction is in p.d / p.inv (a peel-off ray
            // holds them while the walk's are parked)
            const float ext = ext_at( p.b, p.c );
            int ax;
            double t;
            if( peel )
                t = oray_segment( fx, ptc, ax );
            else
                t = exit_cached( p.x, fx, p.d, p.inv, ax );
            const float et = __fmul_rn( ext, ( float ) t );
            bool interact = false, peel_cut = false;
            if( peel )
            {
                ++ cnt.peel;
                ++ pk;
                ptau = __fadd_rn( ptau, et );
                peel_cut = ptau > P.tau_cut;
            }
            else
            {
                ++ cnt.steps;
                ++ p.n_steps;
                interact = et >= p.tau;
            }
            if( interact )
            {
                double ti = ( double ) __fdiv_rn( p.tau, ext );
                ti = ti > t ? t : ti;
                add_flux( ti );
                p.x[ 0 ] = __fma_rn( ti, ( double ) p.d.x, p.x[ 0 ] );
                p.x[ 1 ] = __fma_rn( ti, ( double ) p.d.y, p.x[ 1 ] );
                p.x[ 2 ] = __fma_rn( ti, ( double ) p.d.z, p.x[ 2 ] );
                phase = PH_EVENT;
                break;
            }
            if( ! peel_cut )
            {   // into the next cell
                bool in_block;
                if( peel )
                    in_block = oray_step_in_block( P, p.b, p.c, p.x, fx, ax );
                else
                {   // the walk advances to the exit face
                    p.tau = __fsub_rn( p.tau, et );
                    add_flux( t );
                    #pragma unroll
                    for( int a = 0; a < 3; ++ a )
                        if( a != ax ) p.x[ a ] = __fma_rn( t, ( double ) comp( p.d, a ), p.x[ a ] );
                    in_block = step_in_block( P.m, p.b, p.c, p.x, fx, ax, p.d );
                }
                if( ! in_block )
                {   // leaves the block: wait for a batched hand-off
                    hop_ax = ax;
                    phase = PH_HOP;
                    break;
                }
            }
            after_crossing( peel_cut, false, false );
            if( phase != PH_SEGMENT )
                break;
        }
    }
    count_all( sp, KP_CNT_STEPS, cnt.steps );
    count_all( sp, KP_CNT_PEEL_STEPS, cnt.peel );
    __syncthreads(  );
    if( P.counters && threadIdx.x < KP_NCOUNTERS && sp.cnt[ threadIdx.x ] )
        atomicAdd( P.counters + threadIdx.x, sp.cnt[ threadIdx.x ] );
}

// Marches the peel-off rays k_forward<..., DEFER> queued: each lane takes a
// task, walks it toward the observer segment by segment exactly as the
// forward kernel's inline peel-off ray does (same face cache, hand-off,
// tau cut, deposit), and takes the next.  Fetches (with the deposit of the
// finished ray) and block hand-offs wait for batches of lanes, as in
// k_forward; segments run up to KP_PEEL_INNER at a time between two
// scheduling rounds.  The direction is the launch's observer direction, so
// the face side and the cell-index step of each axis are the same for every
// lane, and a lane holds only the ray's position, faces, cell, optical depth
// and its block's origin and spacing (the next face is computed from them,
// with exit_dist's expression, without a load).
// MODE 0 deposits each ray into the image (forward solve); MODE 3 does the
// same and keeps, for the adjoint of a taped solve, each ray's attenuation
// w exp(-tau) (-1 beyond the cut) in adj_att and the number of its segments
// inside the depth cut in the task's cpix.  The deferred adjoint marches the
// same tasks twice: MODE 1 measures each ray's score G (what the image
// deposit would be worth to the loss) into adj_G and its segments inside the
// cut into cpix; MODE 2 walks exactly those segments again, by geometry
// alone, depositing -G * length into the path-length gradient.  Both skip
// the tasks of packets left to k_adjoint, and MODE 2 the rays with G = 0.
template< int TALLY, int MODE >
__global__ void __launch_bounds__( 256, MODE == 2 ? 3 : KP_PEEL_MINB )
k_peel( const __grid_constant__ fwd_params_t P )
{
    __shared__ unsigned long long cnt_s[ KP_NCOUNTERS ];
    const unsigned FULL = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31u;
    if( threadIdx.x < KP_NCOUNTERS ) cnt_s[ threadIdx.x ] = 0;
    __syncthreads(  );
    const unsigned long long n_queued = min( * P.pq_count, ( unsigned long long ) P.pq_cap );
    // in sorted order: the permutation's slots, whole groups of 32 (the
    // last group's unused slots hold -1)
    const unsigned long long n_tasks = P.pq_perm ? ( n_queued + 31 ) & ~31ull : n_queued;
    const int nc0 = P.m.nc[ 0 ], nc1 = P.m.nc[ 1 ];
    double x0[ 3 ], tm[ 3 ], g0[ 3 ], gd[ 3 ];    // ray start, distances to the next faces
    double tc = 0.0;                              // distance travelled from x0
    int    c[ 3 ] = { 0, 0, 0 }, b = 0, hop_ax = 0, pk = 0, ci = 0;
    const float * eb = P.m.ext;                   // this block's extinctions
    float  ptau = 0.0f;
    float  pG = 0.0f;                             // MODE 2: the ray's score
    int    n_dep = 0;                             // MODE 2: ... and its segments
    // MODE 2: every ray leaves toward the observer along the same corridor of
    // cells, so the blocks deposit into private copies (summed afterwards)
    // rather than all into one tally
    void * g_dep = P.g_len;
    if constexpr( MODE == 2 )
        if( P.adj_priv )
            g_dep = ( char * ) P.adj_priv + ( size_t ) ( blockIdx.x % P.adj_npriv )
                    * ( ( size_t ) P.m.n_blocks * P.m.cpb ) * ( TALLY == KP_TALLY_FIXED ? 8 : 4 );
    long long task = -1;
    unsigned n_seg_done = 0;
    int phase = PH_EMIT;
    // geometry of block b, the distances to the cell's faces (oray_faces's
    // expression) and the cell's index in the block
    auto enter = [ & ](  )
    {
        const double * g = P.m.geo_d + 16 * ( size_t ) b;
        #pragma unroll
        for( int a = 0; a < 3; ++ a )
        {
            g0[ a ] = g[ a ];
            gd[ a ] = g[ 3 + a ];
            const float oa = comp( P.o, a );
            tm[ a ] = oa == 0.0f ? 1e300
                    : __dmul_rn( __dsub_rn( __fma_rn( ( double ) ( c[ a ] + ( oa > 0.0f ? 1 : 0 ) ),
                                                      gd[ a ], g0[ a ] ), x0[ a ] ), P.inv_o[ a ] );
        }
        eb = P.m.ext + ( size_t ) b * P.m.cpb;
        ci = c[ 0 ] + nc0 * ( c[ 1 ] + nc1 * c[ 2 ] );
    };
    for( ;; )
    {
        const unsigned m_fetch = __ballot_sync( FULL, phase == PH_EMIT );
        const unsigned m_seg   = __ballot_sync( FULL, phase == PH_SEGMENT );
        const unsigned m_hop   = __ballot_sync( FULL, phase == PH_HOP );
        if( ( m_fetch | m_seg | m_hop ) == 0u )
            break;
        const int n_fetch = __popc( m_fetch ), n_seg = __popc( m_seg ), n_hop = __popc( m_hop );
        int run;
        if( n_fetch > 0 && ( n_fetch >= P.peel_batch || n_seg == 0 ) )
            run = PH_EMIT;
        else if( n_hop > 0 && ( n_hop >= P.hop_batch || n_seg == 0 ) )
            run = PH_HOP;
        else
            run = PH_SEGMENT;

        if( run == PH_EMIT )
        {
            if( phase != PH_EMIT ) continue;
            const int leader = __ffs( m_fetch ) - 1;
            if constexpr( MODE == 0 || MODE == 3 )
            {
                const bool dep = task >= 0 && ptau <= P.tau_cut;
                float att = -1.0f;                    // MODE 3: -1 marks a ray beyond the cut
                if( dep )
                {   // deposit of the ray that just ended (after_crossing's)
                    const task_dep_t o = load_task_deposit( P.pq, task );
                    att = __fmul_rn( o.w, ( float ) phys::kp_exp_neg( -( double ) ptau ) );
                    deposit_pixel< TALLY >( P, o.pix, o.cpix, __fmul_rn( att, o.I ),
                                            __fmul_rn( att, o.Q ), __fmul_rn( att, o.U ),
                                            __fmul_rn( att, o.V ) );
                }
                if constexpr( MODE == 3 )
                    if( task >= 0 )
                    {   // for the adjoint: attenuation, segments inside the cut
                        P.adj_att[ task ] = att;
                        P.pq[ task ].cpix = ptau > P.tau_cut ? pk - 1 : pk;
                    }
                const unsigned m_dep = __ballot_sync( m_fetch, dep );
                if( ( int ) lane == leader && m_dep )
                    atomicAdd( cnt_s + KP_CNT_DEPOSITS, ( unsigned long long ) __popc( m_dep ) );
            }
            if constexpr( MODE == 1 )
                if( task >= 0 )
                {   // score of the ray that just ended (k_adjoint's measure ray)
                    const task_dep_t o = load_task_deposit( P.pq, task );
                    float G = 0.0f;
                    if( ptau <= P.tau_cut )
                    {
                        const float att = __fmul_rn( o.w, ( float ) phys::kp_exp_neg( -( double ) ptau ) );
                        G = score( P, o.pix, __fmul_rn( att, o.I ), __fmul_rn( att, o.Q ),
                                   __fmul_rn( att, o.U ), __fmul_rn( att, o.V ) );
                    }
                    P.adj_G[ task ] = G;
                    // the segments inside the cut: what the depositing march walks
                    P.pq[ task ].cpix = ptau > P.tau_cut ? pk - 1 : pk;
                }
            task = -1;
            const unsigned rank = __popc( m_fetch & ( ( 1u << lane ) - 1u ) );
            unsigned long long base = 0;
            if( ( int ) lane == leader )
                base = atomicAdd( P.pq_next, ( unsigned long long ) n_fetch );
            base = __shfl_sync( m_fetch, base, leader );
            const unsigned long long idx = base + rank;
            if( idx >= n_tasks )
            {
                phase = PH_DONE;
                continue;
            }
            const long long tk = P.pq_perm ? ( long long ) P.pq_perm[ idx ] : ( long long ) idx;
            if( tk < 0 )
                continue;
            if constexpr( MODE == 1 || MODE == 2 )
            {   // rays of packets left to k_adjoint, and rays worth nothing
                if( P.adj_flag[ P.pq_link[ tk ].lp ] )
                    continue;
                if constexpr( MODE == 2 )
                {
                    pG = P.adj_G[ tk ];
                    n_dep = P.pq[ tk ].cpix;
                    if( pG == 0.0f || n_dep <= 0 )
                        continue;
                }
            }
            load_task_ray( P.pq, tk, x0, b, c );
            task = tk;
            ptau = 0.0f; pk = 0; tc = 0.0;
            enter(  );
            phase = PH_SEGMENT;
            continue;
        }

        if( run == PH_HOP )
        {
            if( phase != PH_HOP ) continue;
            const int b_old = b;
            bool lost;
            double x[ 3 ];                            // the crossing point: the new x0
            oray_point( P, x0, tc, x );
            const bool left = ! cross_face( P.m, b, c, x, hop_ax, comp( P.o, hop_ax ) > 0.0f, lost );
            const unsigned m_moved = __ballot_sync( m_hop, ! left && b != b_old );
            if( lane == ( unsigned ) ( __ffs( m_hop ) - 1 ) && m_moved )
                atomicAdd( cnt_s + KP_CNT_HOPS, ( unsigned long long ) __popc( m_moved ) );
            if( left )
            {
                phase = PH_EMIT;
                continue;
            }
            #pragma unroll
            for( int a = 0; a < 3; ++ a ) x0[ a ] = x[ a ];
            tc = 0.0;
            enter(  );
            phase = pk >= ( 1 << 20 ) ? PH_EMIT : PH_SEGMENT;
            continue;
        }

        if( phase != PH_SEGMENT ) continue;
        #pragma unroll 1
        for( int it = 0; it < ( MODE == 1 || MODE == 2 ? KP_PEEL_INNER_ADJ : KP_PEEL_INNER ); ++ it )
        {
            int ax;
            const double t = oray_segment( tm, tc, ax );
            ++ n_seg_done;
            ++ pk;
            if constexpr( MODE == 2 )
            {   // the measuring march counted the segments inside the cut:
                // geometry only, no coefficients
                add_grad< TALLY >( g_dep, ( size_t ) ( eb - P.m.ext ) + ci,
                                   __dmul_rn( -( double ) pG, t ), P.g_scale );
                if( pk >= n_dep )
                {
                    phase = PH_EMIT;
                    break;
                }
            }
            else
            {
                ptau = __fadd_rn( ptau, __fmul_rn( eb[ ci ], ( float ) t ) );
                if( ptau > P.tau_cut )
                {
                    phase = PH_EMIT;
                    break;
                }
            }
            // into the next cell of the block, with its geometry in registers
            const bool pos = comp( P.o, ax ) > 0.0f;
            const int cax = ax == 0 ? c[ 0 ] : ( ax == 1 ? c[ 1 ] : c[ 2 ] );
            const int cn = cax + ( pos ? 1 : -1 );
            if( cn < 0 || cn >= ( ax == 0 ? nc0 : ( ax == 1 ? nc1 : P.m.nc[ 2 ] ) ) )
            {
                hop_ax = ax;
                phase = PH_HOP;
                break;
            }
            const double nf = __fma_rn( ( double ) ( cn + ( pos ? 1 : 0 ) ),
                                        ax == 0 ? gd[ 0 ] : ( ax == 1 ? gd[ 1 ] : gd[ 2 ] ),
                                        ax == 0 ? g0[ 0 ] : ( ax == 1 ? g0[ 1 ] : g0[ 2 ] ) );
            const double ntm = __dmul_rn( __dsub_rn( nf, ax == 0 ? x0[ 0 ] : ( ax == 1 ? x0[ 1 ] : x0[ 2 ] ) ),
                                          P.inv_o[ ax ] );
            #pragma unroll
            for( int a = 0; a < 3; ++ a )
                if( a == ax ) { c[ a ] = cn; tm[ a ] = ntm; }
            const int st = ax == 0 ? 1 : ( ax == 1 ? nc0 : nc0 * nc1 );
            ci += pos ? st : -st;
            if( pk >= ( 1 << 20 ) )
            {
                phase = PH_EMIT;
                break;
            }
        }
    }
    {   // all lanes of the warp are here
        const unsigned v = __reduce_add_sync( FULL, n_seg_done );
        if( lane == 0 )
            atomicAdd( cnt_s + KP_CNT_PEEL_STEPS, ( unsigned long long ) v );
    }
    __syncthreads(  );
    if( P.counters && threadIdx.x < KP_NCOUNTERS && cnt_s[ threadIdx.x ] )
        atomicAdd( P.counters + threadIdx.x, cnt_s[ threadIdx.x ] );
}

// The starting cell of queued task k, as an index into the mesh's cells
// (block * cells per block + the cell's linear index in the block).
__device__ __forceinline__ unsigned task_cell( const fwd_params_t & P, unsigned long long k )
{
    const int4 v = * reinterpret_cast< const int4 * >(
        reinterpret_cast< const char * >( P.pq + k ) + 16 );
    const unsigned cp = ( unsigned ) v.w;
    return ( unsigned ) v.z * ( unsigned ) P.m.cpb + ( cp & 1023u )
         + ( unsigned ) P.m.nc[ 0 ] * ( ( ( cp >> 10 ) & 1023u ) + ( unsigned ) P.m.nc[ 1 ] * ( cp >> 20 ) );
}

// Counting sort of the queued tasks by starting cell, so that a warp of
// k_peel marches rays that start together and, all going the observer's
// way, cross nearly the same cells: their extinction gathers share cache
// lines.  PASS 0 counts the tasks per cell into cnt; PASS 1 (after an
// exclusive scan of cnt into off, passed as cnt) places each task's index
// in its cell's range.  Lanes of a warp with the same cell take one atomic.
// The order inside a cell is arbitrary: the march's fixed-point tallies do
// not depend on it.
// The sorted list is laid into perm by groups of 32 in a scrambled order
// (group g at (g * p) mod G of the G groups, p = 2^31 - 1, a prime above
// G: a bijection).  Rays that start together deposit into the same pixel;
// in plain sorted order every warp of the GPU would deposit into the same
// few pixels at once (measured 5x slower), scrambled only the lanes of a
// warp do.
template< int PASS >
__global__ void __launch_bounds__( 256 )
k_task_sort( const __grid_constant__ fwd_params_t P, unsigned * cnt, int * perm )
{
    const unsigned FULL = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned long long n = min( * P.pq_count, ( unsigned long long ) P.pq_cap );
    const unsigned long long stride = ( unsigned long long ) gridDim.x * blockDim.x;
    const unsigned long long n_grp = ( n + 31 ) >> 5;
    auto slot = [ & ]( unsigned long long pos )
    {
        return ( ( ( pos >> 5 ) * 2147483647ull ) % n_grp << 5 ) | ( pos & 31ull );
    };
    if constexpr( PASS == 1 )
        if( blockIdx.x == 0 && threadIdx.x < 32 && n > 0
            && threadIdx.x >= n - ( ( n_grp - 1 ) << 5 ) )
            perm[ slot( ( ( n_grp - 1 ) << 5 ) + threadIdx.x ) ] = -1;   // the last group's gaps
    for( unsigned long long i0 = ( unsigned long long ) blockIdx.x * blockDim.x; i0 < n; i0 += stride )
    {   // the loop bound is the same for the whole block
        const unsigned long long i = i0 + threadIdx.x;
        const unsigned act = __ballot_sync( FULL, i < n );
        if( i >= n )
            continue;
        const unsigned key = task_cell( P, i );
        const unsigned grp = __match_any_sync( act, key );
        const int leader = __ffs( grp ) - 1;
        if constexpr( PASS == 0 )
        {
            if( ( int ) lane == leader )
                atomicAdd( cnt + key, ( unsigned ) __popc( grp ) );
        }
        else
        {
            unsigned base = 0;
            if( ( int ) lane == leader )
                base = atomicAdd( cnt + key, ( unsigned ) __popc( grp ) );
            base = __shfl_sync( grp, base, leader );
            perm[ slot( base + __popc( grp & ( ( 1u << lane ) - 1u ) ) ) ] = ( int ) i;
        }
    }
}

}   // namespace

////////////////////////////////////////////////////////////
// Host side

// Fills the launch parameters that do not depend on the mesh or the
// sources (host work only).
void fill_common_params( const kp_transport_cfg_t & c, const kp_tallies_t & t,
                         fwd_params_t & P )
{
    require( c.n_packets >= 0 && c.packet_offset >= 0, "negative packet count" );
    require( c.phase == KP_PHASE_RAYLEIGH || c.phase == KP_PHASE_HG_POL, "unknown phase" );
    require( c.tally_mode == KP_TALLY_FIXED || c.tally_mode == KP_TALLY_FLOAT, "unknown tally mode" );
    require( c.fx_shift >= 0 && c.fx_shift <= 48, "fx_shift out of range" );
    require( c.flux_fx_shift >= 0 && c.flux_fx_shift <= 48, "flux_fx_shift out of range" );
    require( c.n_batches >= 1 && c.n_batches <= KP_MAX_BATCHES, "n_batches out of range",
             KP_ERR_CAPACITY );
    require( c.n_mu_bins >= 0 && ( c.n_mu_bins == 0 || ( t.mu && c.mu_hi > c.mu_lo ) ),
             "bad mu tally" );
    require( c.image_n >= 0 && ( c.image_n == 0 || ( t.image && t.image_batch &&
                                                     c.image_half_width > 0 ) ),
             "bad image" );
    require( c.n_record >= 0 && ( c.n_record == 0 || t.records ), "bad records" );
    require( c.max_scatter >= 1 && c.max_steps >= 1, "caps must be positive" );
    require( c.image_n == 0 || ( c.image_batch_n >= 1 && c.image_batch_n <= c.image_n ),
             "image_batch_n must be in 1..image_n" );
    require( c.lane_batch >= 0 && c.lane_batch <= 32, "lane_batch must be in 0..32" );
    require( c.image_n == 0 || ( long long ) c.n_batches * c.image_batch_n * c.image_batch_n
                                  < ( 1ll << 31 ), "per-batch image too large",
             KP_ERR_CAPACITY );
    std::memset( & P, 0, sizeof( P ) );
    P.n_packets = c.n_packets;
    P.pid0 = c.packet_offset;
    P.seed = c.seed;
    P.stream = c.stream_id;
    P.ph = phys::phase_t { c.phase, c.hg_g, c.pol_max };
    P.n_mu = c.n_mu_bins;
    P.mu_lo = c.mu_lo;
    P.mu_inv_w = c.n_mu_bins > 0 ? ( float ) ( c.n_mu_bins / ( ( double ) c.mu_hi - c.mu_lo ) ) : 0.f;
    P.img_n = c.image_n;
    // Observer at inclination i from +z and azimuth az about +z; image
    // vertical ev is the projection of +z, horizontal eh = ev x o.
    const double inc = c.inclination_deg * M_PI / 180.0, az = c.azimuth_deg * M_PI / 180.0;
    const float o[ 3 ]  = { ( float ) ( std::sin( inc ) * std::cos( az ) ),
                            ( float ) ( std::sin( inc ) * std::sin( az ) ),
                            ( float ) std::cos( inc ) };
    const float ev[ 3 ] = { ( float ) ( -std::cos( inc ) * std::cos( az ) ),
                            ( float ) ( -std::cos( inc ) * std::sin( az ) ),
                            ( float ) std::sin( inc ) };
    const float eh[ 3 ] = { ev[ 1 ] * o[ 2 ] - ev[ 2 ] * o[ 1 ],
                            ev[ 2 ] * o[ 0 ] - ev[ 0 ] * o[ 2 ],
                            ev[ 0 ] * o[ 1 ] - ev[ 1 ] * o[ 0 ] };
    P.o  = phys::v3 { o[ 0 ], o[ 1 ], o[ 2 ] };
    P.ev = phys::v3 { ev[ 0 ], ev[ 1 ], ev[ 2 ] };
    P.eh = phys::v3 { eh[ 0 ], eh[ 1 ], eh[ 2 ] };
    for( int a = 0; a < 3; ++ a )
    {
        P.o_d[ a ]  = o[ a ];
        P.ev_d[ a ] = ev[ a ];
        P.eh_d[ a ] = eh[ a ];
        P.inv_o[ a ] = o[ a ] != 0.0f ? 1.0 / ( double ) o[ a ] : 0.0;
        P.img_c[ a ] = c.image_center[ a ];
    }
    P.img_inv_pix = c.image_n > 0 ? c.image_n / ( 2.0 * c.image_half_width ) : 0.0;
    P.tau_cut = c.tau_peel_max > 0 ? c.tau_peel_max : 40.0f;
    P.fx_scale = std::ldexp( 1.0, c.fx_shift );
    P.n_batch = c.n_batches;
    P.img_bn = c.image_batch_n >= 1 ? c.image_batch_n : 1;
    P.w_min = c.w_min;
    P.rr_survive = c.rr_survive > 0 ? c.rr_survive : 0.1f;
    P.max_scatter = c.max_scatter;
    P.max_steps = std::min< long long >( c.max_steps, 0x7fffffff );
    P.ev_batch = c.lane_batch > 0 ? c.lane_batch : 6;
    // Block hand-offs wait for a batch of lanes (6 measured best for the
    // deferred walk and the peel-off march, 8 for the single-kernel walk
    // before it): the neighbour lookup and the new block's geometry are
    // dependent loads, paid once per batch.
    P.hop_batch = KP_HOP_BATCH;
    P.emit_batch = KP_EMIT_BATCH;
    P.peel_batch = KP_PEEL_BATCH;
    P.mu_tally = t.mu;
    P.image = t.image;
    P.img_batch = t.image_batch;
    P.counters = t.counters;
    P.records = t.records;
    P.n_record = c.n_record;
    P.rec_pid0 = c.packet_offset;
    P.flux = t.flux;
    P.flux_scale = std::ldexp( 1.0, c.flux_fx_shift > 0 ? c.flux_fx_shift : c.fx_shift );
    const carry_fold_t f = carry_layout( c, t );
    for( int k = 0; k < f.n_seg; ++ k )
    {
        if( f.seg[ k ].hi == t.image )       P.c_image = f.seg[ k ].c;
        if( f.seg[ k ].hi == t.image_batch ) P.c_img_batch = f.seg[ k ].c;
        if( f.seg[ k ].hi == t.mu )          P.c_mu = f.seg[ k ].c;
        if( f.seg[ k ].hi == t.flux )        P.c_flux = f.seg[ k ].c;
    }
}

// The float tallies' carries (kp_tallies_t::carry): image, image_batch, mu,
// flux, one after another, each as long as its tally.
carry_fold_t carry_layout( const kp_transport_cfg_t & c, const kp_tallies_t & t )
{
    carry_fold_t f {  };
    if( c.tally_mode != KP_TALLY_FLOAT || t.carry == nullptr )
        return f;
    float * q = t.carry;
    auto add = [ & ]( void * hi, long long n )
    {
        f.seg[ f.n_seg ++ ] = carry_seg_t { static_cast< float * >( hi ), q, n };
        q += n;
    };
    if( c.image_n > 0 )
    {
        const long long bn = c.image_batch_n;
        add( t.image, 4ll * c.image_n * c.image_n );
        add( t.image_batch, 4ll * c.n_batches * bn * bn );
    }
    if( c.n_mu_bins > 0 )
        add( t.mu, 4ll * c.n_batches * c.n_mu_bins );
    if( t.flux )
    {
        require( t.flux_n > 0, "a flux tally with a carry needs flux_n", KP_ERR_CONFIG );
        add( t.flux, t.flux_n );
    }
    return f;
}

__global__ void k_fold_carry( const carry_fold_t f )
{
    const long long stride = ( long long ) gridDim.x * blockDim.x;
    for( int k = 0; k < f.n_seg; ++ k )
        for( long long i = ( long long ) blockIdx.x * blockDim.x + threadIdx.x; i < f.seg[ k ].n;
             i += stride )
        {
            const float e = f.seg[ k ].c[ i ];
            if( e != 0.0f )
            {
                f.seg[ k ].hi[ i ] = __fadd_rn( f.seg[ k ].hi[ i ], e );
                f.seg[ k ].c[ i ] = 0.0f;
            }
        }
}

// Adds the carries into their tallies and zeroes them (after a solve's
// kernels, on its stream); nothing without a carry.
void fold_carry( const kp_transport_cfg_t & c, const kp_tallies_t & t, cudaStream_t s )
{
    const carry_fold_t f = carry_layout( c, t );
    long long n = 0;
    for( int k = 0; k < f.n_seg; ++ k ) n += f.seg[ k ].n;
    if( n == 0 ) return;
    const long long grid = std::min< long long >( ( n + 255 ) / 256, 4 * 148 );
    k_fold_carry<<< ( unsigned ) grid, 256, 0, s >>>( f );
    KP_CUDA( cudaGetLastError(  ) );
}

// Converts one C source to its device form; point sources are located in
// `mesh` (block id, cell).
void make_source( kp_mesh_t * mesh, const kp_source_t & s, src_dev_t & d )
{
    require( s.kind == KP_SOURCE_POINT || s.kind == KP_SOURCE_PLANE_BASE, "unknown source" );
    require( s.emit == KP_EMIT_ISOTROPIC || s.emit == KP_EMIT_UP_UNIFORM, "unknown emission" );
    d.kind = s.kind;
    d.emit = s.emit;
    for( int a = 0; a < 3; ++ a ) d.pos[ a ] = s.pos[ a ];
    d.ib = 0;
    d.cell[ 0 ] = d.cell[ 1 ] = d.cell[ 2 ] = 0;
    if( s.kind == KP_SOURCE_POINT )
        require( mesh->tree->locate( s.pos, d.ib, d.cell ), "source outside the mesh",
                 KP_ERR_CONFIG );
}

// Fills the launch parameters of a single-mesh solve (host work only).
void make_fwd_params( kp_mesh_t * mesh, const kp_transport_cfg_t & c,
                      const kp_tallies_t & t, fwd_params_t & P )
{
    const bool emits = c.packets == nullptr && c.n_packets > 0;
    if( emits )
        require( c.n_sources >= 1 && c.n_sources <= MAX_SOURCES && c.sources,
                 "need 1..KP_MAX_SOURCES sources", KP_ERR_CAPACITY );
    fill_common_params( c, t, P );
    const auto & tab = mesh->tree->tables(  );
    P.m = mesh->view(  );
    P.pk_table = c.packets;
    P.pk_pid0 = c.packet_offset;
    // P.src[ 0 ] is unused with a table or without new packets
    P.n_src = emits ? c.n_sources : 1;
    if( emits )
        for( int k = 0; k < c.n_sources; ++ k )
            make_source( mesh, c.sources[ k ], P.src[ k ] );
    for( int a = 0; a < 3; ++ a )
        P.lk_inv[ a ] = tab.lookup_n[ a ] / tab.l_box_d[ a ];
}

int persistent_grid( const void * kernel, int threads )
{
    int dev = 0, n_sm = 0, per_sm = 0;
    KP_CUDA( cudaGetDevice( & dev ) );
    KP_CUDA( cudaDeviceGetAttribute( & n_sm, cudaDevAttrMultiProcessorCount, dev ) );
    KP_CUDA( cudaOccupancyMaxActiveBlocksPerMultiprocessor( & per_sm, kernel, threads, 0 ) );
    return n_sm * std::max( per_sm, 1 );
}

template< int TALLY, int NT, bool FLUX, bool RESUME = false >
void launch_forward_k( const fwd_params_t & P, cudaStream_t s, int grid_pct )
{
    const void * k = ( const void * ) k_forward< TALLY, NT, false, false, false, FLUX, RESUME >;
    long long grid = persistent_grid( k, NT );
    grid = std::max< long long >( 1, grid * grid_pct / 100 );
    grid = std::min< long long >( grid, ( P.n_packets + P.rs_n_in + NT - 1 ) / NT );
    KP_CUDA( cudaMemsetAsync( P.work, 0, sizeof( unsigned long long ), s ) );
    // whole warps only: the scheduler ballots over full warps
    k_forward< TALLY, NT, false, false, false, FLUX, RESUME ><<< ( unsigned ) grid, NT, 0, s >>>( P );
    KP_CUDA( cudaGetLastError(  ) );
}

template< int NT >
void launch_forward_nt( const fwd_params_t & P, int tally_mode, cudaStream_t s, int grid_pct )
{
    const bool fl = P.flux != nullptr;
    if( tally_mode == KP_TALLY_FIXED )
        fl ? launch_forward_k< KP_TALLY_FIXED, NT, true  >( P, s, grid_pct )
           : launch_forward_k< KP_TALLY_FIXED, NT, false >( P, s, grid_pct );
    else
        fl ? launch_forward_k< KP_TALLY_FLOAT, NT, true  >( P, s, grid_pct )
           : launch_forward_k< KP_TALLY_FLOAT, NT, false >( P, s, grid_pct );
}

// Launches the forward kernel with `threads` per block (128 or 256) and a
// persistent grid of grid_pct percent of the resident-block capacity.
void launch_forward( const fwd_params_t & P, int tally_mode, cudaStream_t s, int threads,
                     int grid_pct )
{
    if( P.n_packets == 0 ) return;
    if( threads == 128 )
        launch_forward_nt< 128 >( P, tally_mode, s, grid_pct );
    else
        launch_forward_nt< 256 >( P, tally_mode, s, grid_pct );
}

}   // namespace kp

namespace kp
{
// Event recorded between the two kernels of a solve (kp_transport_split_event).
thread_local cudaEvent_t split_event = nullptr;

// Solve with peel-off rays deferred: k_forward<..., DEFER> walks the packets
// and queues their peel-off rays (marching them inline only if the queue is
// full), then k_peel marches the queue.  The queue belongs to the mesh and
// holds 12 rays per packet, at most the mesh's limit (default 2^27 rays,
// 8.6 GB); larger solves run in chunks of packets (cap / 12 packets each,
// walk then march), so the queue is sized for the chunk, not the solve.

// Grows the mesh's peel-off queue to 12 rays per packet of a solve of
// n_packets (at least 2^16 rays, at most the mesh's limit).
void ensure_peel_queue( kp_mesh_t * mesh, long long n_packets )
{
    const auto v = mesh->view(  );
    require( v.nc[ 0 ] <= PQ_MAX_CELLS && v.nc[ 1 ] <= PQ_MAX_CELLS && v.nc[ 2 ] <= PQ_MAX_CELLS,
             "peel-off queue: blocks of at most 1024 cells a side", KP_ERR_CAPACITY );
    const long long want = std::min( std::max< long long >( PQ_PER_PACKET * n_packets, 1 << 16 ),
                                     mesh->pq_limit );
    if( mesh->pq_cap < want )
    {
        cudaFree( mesh->d_pq );
        mesh->d_pq = nullptr;
        mesh->pq_cap = 0;
        KP_CUDA( cudaMalloc( & mesh->d_pq, ( size_t ) want * sizeof( peel_task_t ) ) );
        mesh->pq_cap = want;
    }
}

template< int TALLY, bool TAPE, bool FLUX, bool RESUME >
void launch_deferred_walk( const fwd_params_t & P, cudaStream_t s )
{
    const void * kf = ( const void * ) k_forward< TALLY, 256, false, true, TAPE, FLUX, RESUME >;
    long long grid = persistent_grid( kf, 256 );
    grid = std::min< long long >( grid, ( P.n_packets + P.rs_n_in + 255 ) / 256 );
    k_forward< TALLY, 256, false, true, TAPE, FLUX, RESUME ><<< ( unsigned ) grid, 256, 0, s >>>( P );
    KP_CUDA( cudaGetLastError(  ) );
}

// Whether the forward solve marches the mesh's queue sorted by starting
// cell (kp_mesh_peel_order).  Measured: the 2-level clump scene (9.3 MB of
// extinction, in L2) march took 59 + 10 ms sorted against 52 ms; the
// 3-level large scene (83 MB) forward solve took 1.96 against 2.15 s.
bool peel_sorted( const kp_mesh_t * mesh )
{
    if( mesh->peel_order != KP_PEEL_ORDER_AUTO )
        return mesh->peel_order == KP_PEEL_ORDER_CELL;
    const auto v = mesh->view(  );
    return ( long long ) v.n_blocks * v.cpb * ( long long ) sizeof( float ) > KP_PEEL_SORT_MIN_BYTES;
}

// Makes room on the mesh for sorting a queue of pq_cap tasks (a permutation
// of pq_cap + 32 slots: whole groups of 32); returns the permutation.
int * ensure_task_sort( kp_mesh_t * mesh, long long pq_cap )
{
    const auto v = mesh->view(  );
    const size_t nk = ( size_t ) v.n_blocks * v.cpb;
    const size_t n_slots = ( size_t ) pq_cap + 32;
    require( n_slots < ( 1ull << 31 ) && nk < ( 1ull << 31 ),
             "peel-off sort: at most 2^31 rays and cells", KP_ERR_CAPACITY );
    if( mesh->sort_cells < nk )
    {
        cudaFree( mesh->d_sort_cnt ); cudaFree( mesh->d_sort_off ); cudaFree( mesh->d_sort_tmp );
        mesh->d_sort_cnt = mesh->d_sort_off = nullptr;
        mesh->d_sort_tmp = nullptr;
        mesh->sort_cells = mesh->sort_tmp_bytes = 0;
        KP_CUDA( cudaMalloc( & mesh->d_sort_cnt, nk * sizeof( unsigned ) ) );
        KP_CUDA( cudaMalloc( & mesh->d_sort_off, nk * sizeof( unsigned ) ) );
        size_t tb = 0;
        KP_CUDA( cub::DeviceScan::ExclusiveSum( nullptr, tb, mesh->d_sort_cnt, mesh->d_sort_off,
                                                ( int ) nk ) );
        KP_CUDA( cudaMalloc( & mesh->d_sort_tmp, tb ) );
        mesh->sort_tmp_bytes = tb;
        mesh->sort_cells = nk;
    }
    if( mesh->sort_perm < n_slots )
    {
        cudaFree( mesh->d_sort_perm );
        mesh->d_sort_perm = nullptr;
        mesh->sort_perm = 0;
        KP_CUDA( cudaMalloc( & mesh->d_sort_perm, n_slots * sizeof( int ) ) );
        mesh->sort_perm = n_slots;
    }
    return mesh->d_sort_perm;
}

// Sorts the queued tasks by starting cell into P.pq_perm (k_task_sort).
void task_sort( const kp_mesh_t * mesh, const fwd_params_t & P, cudaStream_t s )
{
    const size_t nk = ( size_t ) P.m.n_blocks * P.m.cpb;
    int dev = 0, n_sm = 0;
    KP_CUDA( cudaGetDevice( & dev ) );
    KP_CUDA( cudaDeviceGetAttribute( & n_sm, cudaDevAttrMultiProcessorCount, dev ) );
    const unsigned grid = ( unsigned ) n_sm * 8;
    KP_CUDA( cudaMemsetAsync( mesh->d_sort_cnt, 0, nk * sizeof( unsigned ), s ) );
    k_task_sort< 0 ><<< grid, 256, 0, s >>>( P, mesh->d_sort_cnt, nullptr );
    KP_CUDA( cudaGetLastError(  ) );
    size_t tb = mesh->sort_tmp_bytes;
    KP_CUDA( cub::DeviceScan::ExclusiveSum( mesh->d_sort_tmp, tb, mesh->d_sort_cnt,
                                            mesh->d_sort_off, ( int ) nk, s ) );
    k_task_sort< 1 ><<< grid, 256, 0, s >>>( P, mesh->d_sort_off, mesh->d_sort_perm );
    KP_CUDA( cudaGetLastError(  ) );
}

template< int TALLY, bool TAPE, bool RESUME >
void launch_deferred_chunk( fwd_params_t & P, cudaStream_t s, const kp_mesh_t * mesh )
{
    require( P.pq_perm == nullptr || mesh, "peel-off sort without its mesh" );
    P.pq_count = P.work + 1;
    P.pq_next = P.work + 2;
    KP_CUDA( cudaMemsetAsync( P.work, 0, 3 * sizeof( unsigned long long ), s ) );
    if( P.flux ) launch_deferred_walk< TALLY, TAPE, true,  RESUME >( P, s );
    else         launch_deferred_walk< TALLY, TAPE, false, RESUME >( P, s );
    if( split_event ) KP_CUDA( cudaEventRecord( split_event, s ) );
    if( P.pq_perm ) task_sort( mesh, P, s );
    constexpr int MODE = TAPE ? 3 : 0;
    const long long gp = persistent_grid( ( const void * ) k_peel< TALLY, MODE >, 256 );
    k_peel< TALLY, MODE ><<< ( unsigned ) gp, 256, 0, s >>>( P );
    KP_CUDA( cudaGetLastError(  ) );
}
template void launch_deferred_chunk< KP_TALLY_FIXED, true, false >( fwd_params_t &, cudaStream_t,
                                                                     const kp_mesh_t * );
template void launch_deferred_chunk< KP_TALLY_FLOAT, true, false >( fwd_params_t &, cudaStream_t,
                                                                     const kp_mesh_t * );

// The deferred adjoint's marches of the queued vertex rays: mode 1 measures
// their scores, mode 2 deposits along them (k_peel).
void launch_peel_adjoint( const fwd_params_t & P, int tally_mode, int mode, cudaStream_t s )
{
    KP_CUDA( cudaMemsetAsync( P.pq_next, 0, sizeof( unsigned long long ), s ) );
    const bool fx = tally_mode == KP_TALLY_FIXED;
    const void * k = mode == 1 ? ( fx ? ( const void * ) k_peel< KP_TALLY_FIXED, 1 >
                                      : ( const void * ) k_peel< KP_TALLY_FLOAT, 1 > )
                               : ( fx ? ( const void * ) k_peel< KP_TALLY_FIXED, 2 >
                                      : ( const void * ) k_peel< KP_TALLY_FLOAT, 2 > );
    const unsigned gp = ( unsigned ) persistent_grid( k, 256 );
    if( mode == 1 )
    {
        if( fx ) k_peel< KP_TALLY_FIXED, 1 ><<< gp, 256, 0, s >>>( P );
        else     k_peel< KP_TALLY_FLOAT, 1 ><<< gp, 256, 0, s >>>( P );
    }
    else
    {
        if( fx ) k_peel< KP_TALLY_FIXED, 2 ><<< gp, 256, 0, s >>>( P );
        else     k_peel< KP_TALLY_FLOAT, 2 ><<< gp, 256, 0, s >>>( P );
    }
    KP_CUDA( cudaGetLastError(  ) );
}

template< int TALLY >
void launch_deferred( kp_mesh_t * mesh, const fwd_params_t & P, cudaStream_t s )
{
    mesh->tape_id = 0;                      // the queue is overwritten
    ensure_peel_queue( mesh, P.n_packets );
    const long long chunk = std::max< long long >( mesh->pq_cap / PQ_PER_PACKET, 1 );
    int * perm = peel_sorted( mesh ) ? ensure_task_sort( mesh, mesh->pq_cap ) : nullptr;
    static thread_local fwd_params_t C;
    for( long long done = 0; done < P.n_packets; done += chunk )
    {
        C = P;
        C.pq = static_cast< peel_task_t * >( mesh->d_pq );
        C.pq_cap = mesh->pq_cap;
        C.pq_perm = perm;
        C.pid0 = P.pid0 + done;
        C.n_packets = std::min( chunk, P.n_packets - done );
        launch_deferred_chunk< TALLY, false, false >( C, s, mesh );
    }
}

void launch_deferred_solve( kp_mesh_t * mesh, const fwd_params_t & P, int tally_mode,
                            cudaStream_t s )
{
    if( tally_mode == KP_TALLY_FIXED ) launch_deferred< KP_TALLY_FIXED >( mesh, P, s );
    else                               launch_deferred< KP_TALLY_FLOAT >( mesh, P, s );
}
}   // namespace kp

extern "C" int kp_transport_forward( kp_mesh_t * mesh, const kp_transport_cfg_t * cfg,
                                     const kp_tallies_t * tallies, void * stream )
{
    return kp::guarded( "kp_transport_forward", [ & ]
    {
        kp::require( mesh && cfg && tallies, "null argument" );
        mesh->upload(  );
        mesh->refresh_ext( ( cudaStream_t ) stream );
        static thread_local kp::fwd_params_t P;
        kp::make_fwd_params( mesh, * cfg, * tallies, P );
        P.work = mesh->workspace(  );
        if( cfg->image_n > 0 && P.n_packets > 0 )
        {   // peel-off rays through their own kernel; without them the walk
            // kernel's interactions run best in batches of 12 lanes (measured)
            if( cfg->lane_batch == 0 ) P.ev_batch = 12;
            if( cfg->tally_mode == KP_TALLY_FIXED )
                kp::launch_deferred< KP_TALLY_FIXED >( mesh, P, ( cudaStream_t ) stream );
            else
                kp::launch_deferred< KP_TALLY_FLOAT >( mesh, P, ( cudaStream_t ) stream );
        }
        else
        {
            kp::launch_forward( P, cfg->tally_mode, ( cudaStream_t ) stream, 256, 100 );
            if( kp::split_event )
                KP_CUDA( cudaEventRecord( kp::split_event, ( cudaStream_t ) stream ) );
        }
        kp::fold_carry( * cfg, * tallies, ( cudaStream_t ) stream );
    } );
}

extern "C" int kp_mesh_peel_queue_limit( kp_mesh_t * mesh, long long max_rays )
{
    return kp::guarded( "kp_mesh_peel_queue_limit", [ & ]
    {
        kp::require( mesh, "null mesh" );
        kp::require( max_rays >= 1024, "the peel-off queue limit must be at least 1024 rays",
                     KP_ERR_CONFIG );
        if( mesh->pq_cap > max_rays )
        {   // the next solve allocates a queue within the new limit
            KP_CUDA( cudaFree( mesh->d_pq ) );
            mesh->d_pq = nullptr;
            mesh->pq_cap = 0;
            KP_CUDA( cudaFree( mesh->d_adj ) );
            mesh->d_adj = nullptr;
            mesh->adj_bytes = 0;
            mesh->tape_id = 0;
        }
        mesh->pq_limit = max_rays;
    } );
}

extern "C" int kp_mesh_peel_order( kp_mesh_t * mesh, int order )
{
    return kp::guarded( "kp_mesh_peel_order", [ & ]
    {
        kp::require( mesh, "null mesh" );
        kp::require( order == KP_PEEL_ORDER_AUTO || order == KP_PEEL_ORDER_QUEUE
                     || order == KP_PEEL_ORDER_CELL, "unknown peel-off order", KP_ERR_CONFIG );
        mesh->peel_order = order;
    } );
}

extern "C" int kp_transport_split_event( void * event )
{
    kp::split_event = static_cast< cudaEvent_t >( event );
    return KP_OK;
}

////////////////////////////////////////////////////////////
// Resumable solve: the step budget of one call (k_forward<..., RESUME>).

static_assert( sizeof( kp_packet_state_t ) == sizeof( kp::dd_walk_t ), "packet state size" );
static_assert( offsetof( kp_packet_state_t, n_steps ) == offsetof( kp::dd_walk_t, n_steps )
               && offsetof( kp_packet_state_t, rng_draws ) == offsetof( kp::dd_walk_t, draw )
               && offsetof( kp_packet_state_t, batch ) == offsetof( kp::dd_walk_t, batch ),
               "packet state layout" );

namespace kp
{
// With an image: work items (the resumed packets, then the new ones) in
// chunks of the queue's capacity / 12, each walked and then marched, as
// launch_deferred does for new packets alone.
template< int TALLY >
void launch_resume_deferred( kp_mesh_t * mesh, const fwd_params_t & P, cudaStream_t s )
{
    const long long n_in = P.rs_n_in, items = n_in + P.n_packets;
    mesh->tape_id = 0;                      // the queue is overwritten
    ensure_peel_queue( mesh, items );
    const long long chunk = std::max< long long >( mesh->pq_cap / PQ_PER_PACKET, 1 );
    int * perm = peel_sorted( mesh ) ? ensure_task_sort( mesh, mesh->pq_cap ) : nullptr;
    static thread_local fwd_params_t C;
    for( long long lo = 0; lo < items; lo += chunk )
    {
        const long long hi = std::min( items, lo + chunk );
        C = P;
        C.pq = static_cast< peel_task_t * >( mesh->d_pq );
        C.pq_cap = mesh->pq_cap;
        C.pq_perm = perm;
        C.rs_in = P.rs_in + std::min( lo, n_in );
        C.rs_n_in = std::max< long long >( std::min( hi, n_in ) - lo, 0 );
        const long long first = std::max( lo, n_in );   // first new packet's item
        C.pid0 = P.pid0 + ( first - n_in );
        C.n_packets = std::max< long long >( hi - first, 0 );
        launch_deferred_chunk< TALLY, false, true >( C, s, mesh );
    }
}
}   // namespace kp

extern "C" int kp_transport_forward_resume( kp_mesh_t * mesh, const kp_transport_cfg_t * cfg,
                                            const kp_resume_t * rs, const kp_tallies_t * tallies,
                                            void * stream )
{
    return kp::guarded( "kp_transport_forward_resume", [ & ]
    {
        kp::require( mesh && cfg && rs && tallies, "null argument" );
        kp::require( rs->step_budget >= 1, "step_budget must be at least 1" );
        kp::require( rs->n_in >= 0 && rs->cap_out >= 0, "negative queue size" );
        kp::require( ( rs->n_in == 0 || rs->in ) && ( rs->cap_out == 0 || rs->out ) && rs->out_count,
                     "null queue" );
        {   // the kernel reads `in` while it writes `out`
            const auto a0 = reinterpret_cast< uintptr_t >( rs->in );
            const auto b0 = reinterpret_cast< uintptr_t >( rs->out );
            const auto a1 = a0 + ( uintptr_t ) rs->n_in * sizeof( kp_packet_state_t );
            const auto b1 = b0 + ( uintptr_t ) rs->cap_out * sizeof( kp_packet_state_t );
            kp::require( rs->n_in == 0 || rs->cap_out == 0 || a1 <= b0 || b1 <= a0,
                         "the in and out packet queues overlap" );
        }
        mesh->upload(  );
        mesh->refresh_ext( ( cudaStream_t ) stream );
        static thread_local kp::fwd_params_t P;
        kp::make_fwd_params( mesh, * cfg, * tallies, P );
        P.work = mesh->workspace(  );
        P.rs_in = reinterpret_cast< const kp::dd_walk_t * >( rs->in );
        P.rs_n_in = rs->n_in;
        P.rs_out = reinterpret_cast< kp::dd_walk_t * >( rs->out );
        P.rs_cap = rs->cap_out;
        P.rs_count = rs->out_count;
        P.rs_budget = rs->step_budget;
        cudaStream_t s = ( cudaStream_t ) stream;
        if( P.n_packets + P.rs_n_in > 0 )
        {
            const bool fx = cfg->tally_mode == KP_TALLY_FIXED, fl = P.flux != nullptr;
            if( cfg->image_n > 0 )
            {   // the deferred walk's interaction batch, as kp_transport_forward
                if( cfg->lane_batch == 0 ) P.ev_batch = 12;
                fx ? kp::launch_resume_deferred< KP_TALLY_FIXED >( mesh, P, s )
                   : kp::launch_resume_deferred< KP_TALLY_FLOAT >( mesh, P, s );
            }
            else
            {
                if( fx ) fl ? kp::launch_forward_k< KP_TALLY_FIXED, 256, true,  true >( P, s, 100 )
                            : kp::launch_forward_k< KP_TALLY_FIXED, 256, false, true >( P, s, 100 );
                else     fl ? kp::launch_forward_k< KP_TALLY_FLOAT, 256, true,  true >( P, s, 100 )
                            : kp::launch_forward_k< KP_TALLY_FLOAT, 256, false, true >( P, s, 100 );
                if( kp::split_event ) KP_CUDA( cudaEventRecord( kp::split_event, s ) );
            }
        }
        kp::fold_carry( * cfg, * tallies, s );
    } );
}

////////////////////////////////////////////////////////////
// One round of a domain-decomposed solve (k_forward<..., DD = true>).

static_assert( sizeof( kp::dd_walk_t ) == KP_DD_WALK_BYTES, "walk record size" );

namespace kp
{
template< int TALLY, bool FLUX >
void launch_dd( const fwd_params_t & P, long long items, cudaStream_t s )
{
    const void * k = ( const void * ) k_forward< TALLY, 256, true, false, false, FLUX >;
    long long grid = persistent_grid( k, 256 );
    grid = std::min< long long >( grid, ( items + 255 ) / 256 );
    k_forward< TALLY, 256, true, false, false, FLUX ><<< ( unsigned ) grid, 256, 0, s >>>( P );
    KP_CUDA( cudaGetLastError(  ) );
}
}   // namespace kp
static_assert( sizeof( kp::dd_peel_t ) == KP_DD_PEEL_BYTES, "peel-off record size" );

extern "C" int kp_transport_forward_dd( kp_mesh_t * mesh, const kp_transport_cfg_t * cfg,
                                        const kp_dd_round_t * r, const kp_tallies_t * tallies,
                                        void * stream )
{
    return kp::guarded( "kp_transport_forward_dd", [ & ]
    {
        kp::require( mesh && cfg && r && tallies, "null argument" );
        kp::require( cfg->n_record == 0, "records are not kept in decomposed solves" );
        kp::require( r->n_ranks >= 1 && r->rank >= 0 && r->rank < r->n_ranks, "bad rank" );
        kp::require( r->owner && r->block_local && r->sigma_local && r->out_count,
                     "null decomposition array" );
        kp::require( r->n_in_walk >= 0 && r->n_in_peel >= 0 && r->cap_walk >= 0
                     && r->cap_peel >= 0, "negative queue size" );
        kp::require( ( r->n_in_walk == 0 || r->in_walk ) && ( r->n_in_peel == 0 || r->in_peel )
                     && ( r->cap_walk == 0 || ( r->out_walk && r->out_walk_rank ) )
                     && ( r->cap_peel == 0 || ( r->out_peel && r->out_peel_rank ) ),
                     "null queue" );
        mesh->upload( false );                    // tables only: sigma is per rank
        static thread_local kp::fwd_params_t P;
        kp::make_fwd_params( mesh, * cfg, * tallies, P );
        P.m.sigma = reinterpret_cast< const float2 * >( r->sigma_local );
        P.work = mesh->workspace(  );
        P.dd_rank = r->rank; P.dd_ranks = r->n_ranks;
        P.dd_owner = r->owner; P.dd_loc = r->block_local;
        P.dd_in_walk = static_cast< const kp::dd_walk_t * >( r->in_walk );
        P.dd_in_peel = static_cast< const kp::dd_peel_t * >( r->in_peel );
        P.dd_n_walk = r->n_in_walk; P.dd_n_peel = r->n_in_peel;
        P.dd_emit = r->emit != 0;
        P.dd_out_walk = static_cast< kp::dd_walk_t * >( r->out_walk );
        P.dd_out_peel = static_cast< kp::dd_peel_t * >( r->out_peel );
        P.dd_out_walk_rank = r->out_walk_rank;
        P.dd_out_peel_rank = r->out_peel_rank;
        P.dd_cap_walk = r->cap_walk; P.dd_cap_peel = r->cap_peel;
        P.dd_out_count = r->out_count;
        const long long items = r->n_in_walk + r->n_in_peel + ( r->emit ? cfg->n_packets : 0 );
        if( items == 0 ) return;
        cudaStream_t s = ( cudaStream_t ) stream;
        KP_CUDA( cudaMemsetAsync( P.work, 0, sizeof( unsigned long long ), s ) );
        const bool fx = cfg->tally_mode == KP_TALLY_FIXED;
        if( P.flux )
            fx ? kp::launch_dd< KP_TALLY_FIXED, true  >( P, items, s )
               : kp::launch_dd< KP_TALLY_FLOAT, true  >( P, items, s );
        else
            fx ? kp::launch_dd< KP_TALLY_FIXED, false >( P, items, s )
               : kp::launch_dd< KP_TALLY_FLOAT, false >( P, items, s );
        kp::fold_carry( * cfg, * tallies, s );
    } );
}

////////////////////////////////////////////////////////////
// No-allocation entry point: the forward solve with its packet counter in a
// static device array instead of the mesh's workspace.

#include <mutex>

namespace kp
{
namespace
{

// Scratch of kp_transport_forward_noalloc.  In host code this name is only a
// stand-in for the symbol: kernels receive the device address looked up
// below, never the name itself.
static __device__ __align__( 256 ) unsigned char g_noalloc_scratch[ KP_NOALLOC_SCRATCH_BYTES ];

constexpr int NOALLOC_MAX_DEVICES = 64;
std::mutex    g_noalloc_mutex;
void        * g_noalloc_addr[ NOALLOC_MAX_DEVICES ] = {  };

// Device address of the scratch array on the current device, looked up once
// per device (with that device current) and cached.
void * noalloc_scratch(  )
{
    int dev = 0;
    KP_CUDA( cudaGetDevice( & dev ) );
    require( dev >= 0 && dev < NOALLOC_MAX_DEVICES, "device index too large for the scratch table",
             KP_ERR_CAPACITY );
    std::lock_guard< std::mutex > lock( g_noalloc_mutex );
    if( g_noalloc_addr[ dev ] == nullptr )
    {
        void * p = nullptr;
        KP_CUDA( cudaGetSymbolAddress( & p, g_noalloc_scratch ) );
        g_noalloc_addr[ dev ] = p;
    }
    return g_noalloc_addr[ dev ];
}

}   // namespace
}   // namespace kp

extern "C" int kp_transport_forward_noalloc( kp_mesh_t * mesh, const kp_transport_cfg_t * cfg,
                                             const kp_tallies_t * tallies, void * stream )
{
    return kp::guarded( "kp_transport_forward_noalloc", [ & ]
    {
        kp::require( mesh && cfg && tallies, "null argument" );
        kp::require( mesh->uploaded && mesh->d_sigma != nullptr,
                     "mesh is not on the device: call kp_mesh_upload at set-up",
                     KP_ERR_CONFIG );
        int dev = 0;
        KP_CUDA( cudaGetDevice( & dev ) );
        kp::require( dev == mesh->device, "mesh was uploaded to another device", KP_ERR_CONFIG );
        // Scratch needed by one forward launch: one 64-bit packet counter.
        const size_t need = sizeof( unsigned long long );
        kp::require( need <= KP_NOALLOC_SCRATCH_BYTES,
                     "forward scratch exceeds KP_NOALLOC_SCRATCH_BYTES", KP_ERR_CAPACITY );
        static thread_local kp::fwd_params_t P;
        kp::make_fwd_params( mesh, * cfg, * tallies, P );
        P.work = static_cast< unsigned long long * >( kp::noalloc_scratch(  ) );
        mesh->refresh_ext( ( cudaStream_t ) stream );    // a kernel into mesh memory
        kp::launch_forward( P, cfg->tally_mode, ( cudaStream_t ) stream, 256, 100 );
        if( kp::split_event ) KP_CUDA( cudaEventRecord( kp::split_event, ( cudaStream_t ) stream ) );
        kp::fold_carry( * cfg, * tallies, ( cudaStream_t ) stream );
    } );
}
