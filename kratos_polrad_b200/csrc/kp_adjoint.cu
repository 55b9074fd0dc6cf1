// Path-replay adjoint of the peel-off image (gradient of an image loss with
// respect to the per-cell scattering and absorption coefficients).
//
// The reference has no differentiable transport.  The estimator follows path
// replay backpropagation (Vicini, Speierer & Jakob, SIGGRAPH 2021) for the
// volumetric case with tau-threshold sampling: for a sampled path held fixed,
// the peel-off contribution C_k of vertex k (k = 0 the emission, k >= 1 the
// interactions) has
//     d ln f_k / d sigma_sca(c) = n_k(c) / sigma_sca(c) - L_k(c) - L_obs,k(c)
//     d ln f_k / d sigma_abs(c) =                      - L_k(c) - L_obs,k(c)
// where n_k(c) counts interactions in cell c among vertices 1..k, L_k(c) is
// the walk's path length in c up to vertex k and L_obs,k(c) the peel-off
// ray's.  With G_k = <dL/dimage[pixel_k], C_k>, the gradient is
// sum_k G_k d ln f_k.  Every packet is replayed twice from its RNG counter:
// pass 0 computes each G_k and R = sum_{k>=1} G_k; pass 1 deposits
// -R * length along walk segments (R the suffix sum of the vertices still
// ahead), +R / sigma_sca at interactions, and -G_k * length along each
// peel-off ray, subtracting G_k from R after vertex k.
// kp_transport_adjoint runs this in five launches per chunk of packets
// (k_adj_walk pass 0, k_peel measuring, k_adj_fold, k_adj_walk pass 1,
// k_peel depositing), the vertices' rays queued between them; k_adjoint
// does both passes in one launch with the rays inline (G_k kept in a
// 32-entry per-lane array, later vertices re-measured in pass 1) and takes
// the packets whose rays did not fit the queue.
// Outputs: g_len (length term, shared by both coefficients) and g_int
// (interaction term, scattering only):
//     dL/dsigma_sca = g_len + g_int,  dL/dsigma_abs = g_len.
#include "kp_transport.cuh"

namespace kp
{
namespace
{

// Private copies of the path-length tally for the depositing march.
#ifndef KP_ADJ_PRIV
#define KP_ADJ_PRIV 8
#endif

constexpr int ADJ_KMAX = 32;
enum ray_kind { RAY_WALK = 0, RAY_MEASURE = 1, RAY_DEPOSIT = 2 };

template< int TALLY >
__global__ void __launch_bounds__( FWD_THREADS, 3 )
k_adjoint( const __grid_constant__ fwd_params_t P )
{
    __shared__ park_t<  > sp;
    __shared__ dir_park_t< FWD_THREADS > sd;
    __shared__ cold_park_t< FWD_THREADS > sc;
    const unsigned FULL = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31u;
    const int th = threadIdx.x;
    if( threadIdx.x < KP_NCOUNTERS ) sp.cnt[ threadIdx.x ] = 0;
    __syncthreads(  );
    counts32_t cnt;
    packet_t p;
    double fx[ 3 ];                               // face cache of the active ray
    int   phase = PH_EMIT, ray = RAY_WALK, pass = 0;
    float ptau = 0.f, pG = 0.f, G0 = 0.f;
    double ptc = 0.0;             // a peel-off ray: distance travelled from its start
    int   pk = 0, pend = 0, nv = 0;   // (p.x), fx its face distances (oray_faces)
    bool  remeasure = false;
    double R = 0.0;
    float gk[ ADJ_KMAX ];
    // packets of a list (the deferred adjoint's overflow), whose first
    // replay the deferred walk has counted already
    const unsigned long long n_items = P.adj_list ? * P.adj_list_n
                                                  : ( unsigned long long ) P.n_packets;
    auto counting = [ & ](  ) { return pass == 1 || ! P.adj_quiet; };

    // Starts pass 1 of the lane's packet (same id, RNG from its start).
    auto begin_pass1 = [ & ](  )
    {
        const long long pid = cold_pid( sc );
        float peel_I;
        emit_any( P, pid, p, peel_I );
        p.tau = sample_tau( p.rng );
        store_cold( sc, p );
        pass = 1;
        nv = 0;
        phase = PH_SEGMENT;
        ray = RAY_WALK;
        if( P.img_n > 0 && peel_I > 0.0f && G0 != 0.0f )
        {
            park_walk( sp, p );
            park_dir( sd, p, P.o, P.inv_o );
            pG = G0; ptau = 0.f; pk = 0; pend = 0; ptc = 0.0;
            ray = RAY_DEPOSIT;
            oray_faces( P, p.b, p.c, p.x, fx );
        }
        else
            faces_all( P.m, p.b, p.c, p.d, fx );
    };
    // The lane's packet has ended (in the current pass).
    auto end_packet = [ & ](  )
    {
        if( pass == 0 )
            begin_pass1(  );
        else
        {
            phase = PH_EMIT;
            pass = 0;
        }
    };

    // After the active ray crossed a face (or stopped): the end of a peel-off
    // ray (measure / deposit bookkeeping, walk resumes) or of the walk.
    // Shared by the segment phase and the hand-off phase.
    auto after_crossing = [ & ]( bool peel_cut, bool left, bool lost )
    {
        if( ray != RAY_WALK )
        {
            if( !( peel_cut || left || pk >= ( 1 << 20 ) ) )
                return;
            if( ray == RAY_MEASURE )
            {
                float G = 0.0f;
                if( ptau <= P.tau_cut )
                {
                    const float att = __fmul_rn( sp.w[ th ],
                                                 ( float ) phys::kp_exp_neg( -( double ) ptau ) );
                    G = score( P, sp.pix[ th ], __fmul_rn( att, sp.I[ th ] ),
                               __fmul_rn( att, sp.Q[ th ] ), __fmul_rn( att, sp.U[ th ] ),
                               __fmul_rn( att, sp.V[ th ] ) );
                }
                if( remeasure )
                {   // pass 1, vertex beyond the stored ones: now deposit along it
                    remeasure = false;
                    unpark_walk( sp, p );
                    if( G != 0.0f )
                    {
                        pG = G; ptau = 0.f; pk = 0; ptc = 0.0;
                        ray = RAY_DEPOSIT;          // the walk position stays parked
                        oray_faces( P, p.b, p.c, p.x, fx );    // p.d is still o
                        return;
                    }
                }
                else if( nv == 0 )
                    G0 = G;                          // emission
                else
                {
                    R = __dadd_rn( R, ( double ) G );
                    if( nv <= ADJ_KMAX ) gk[ nv - 1 ] = G;
                }
            }
            else if( nv > 0 )
                R = __dsub_rn( R, ( double ) pG );   // deposit ray of vertex nv done
            unpark_walk( sp, p );
            unpark_dir( sd, p );
            ray = RAY_WALK;
            if( pend )
                end_packet(  );
            else
                faces_all( P.m, p.b, p.c, p.d, fx );
            return;
        }
        if( left || p.n_steps >= P.max_steps )
        {
            if( counting(  ) )
            {
                if( left )
                    count( sp, lost ? KP_CNT_LOST : KP_CNT_ESCAPED );
                else
                    count( sp, KP_CNT_CAPPED );
            }
            end_packet(  );
        }
    };
    int hop_ax = 0;                               // face axis of a pending hand-off

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
        else if( n_emit > 0 && ( n_emit >= P.ev_batch || n_seg == 0 ) )
            run = PH_EMIT;
        else if( n_hop > 0 && ( n_hop >= P.hop_batch || n_seg == 0 ) )
            run = PH_HOP;
        else
            run = PH_SEGMENT;

        if( run == PH_HOP )
        {   // batched block hand-offs (see k_forward)
            if( phase != PH_HOP ) continue;
            const int b_old = p.b;
            bool lost, left;
            if( ray != RAY_WALK )   // a peel-off ray: rebased at its crossing point
                left = ! oray_rebase( P, p.b, p.c, p.x, ptc, fx, hop_ax, lost );
            else
                left = ! cross_face( P.m, p.b, p.c, p.x, hop_ax, comp( p.d, hop_ax ) > 0.0f, lost );
            if( ! left )
            {
                if( ray == RAY_WALK )
                    faces_all( P.m, p.b, p.c, p.d, fx );
                if( p.b != b_old && counting(  ) ) count( sp, KP_CNT_HOPS );
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
            const unsigned long long idx = base + rank;
            if( idx >= n_items )
            {
                phase = PH_DONE;
                continue;
            }
            const long long pid = P.pid0 + ( P.adj_list ? ( long long ) P.adj_list[ idx ]
                                                        : source_major( ( long long ) idx,
                                                                        ( long long ) n_items,
                                                                        P.n_src ) );
            float peel_I;
            if( ! emit_any( P, pid, p, peel_I ) )
            {
                atomicOr( P.m.status, ST_BAD_SOURCE );
                continue;
            }
            if( ! P.adj_quiet ) count( sp, KP_CNT_EMITTED );
            p.tau = sample_tau( p.rng );
            store_cold( sc, p );
            pass = 0; nv = 0; R = 0.0; G0 = 0.f;
            phase = PH_SEGMENT;
            ray = RAY_WALK;
            if( P.img_n > 0 && peel_I > 0.0f )
            {
                const int pix = image_pixel( P, p.x );
                if( pix >= 0 )
                {
                    sp.w[ th ] = p.w; sp.I[ th ] = peel_I;
                    sp.Q[ th ] = sp.U[ th ] = sp.V[ th ] = 0.0f;
                    sp.pix[ th ] = pix;
                    pend = 0; ptau = 0.0f; pk = 0; ptc = 0.0;
                    park_walk( sp, p );
                    park_dir( sd, p, P.o, P.inv_o );
                    ray = RAY_MEASURE;
                }
            }
            if( ray != RAY_WALK )
                oray_faces( P, p.b, p.c, p.x, fx );
            else
                faces_all( P.m, p.b, p.c, p.d, fx );
            continue;
        }

        if( run == PH_EVENT )
        {
            if( phase != PH_EVENT ) continue;
            load_cold( sc, p, P.seed );
            ++ p.n_scat;
            if( counting(  ) ) count( sp, KP_CNT_SCATTER );
            const size_t ci = cell_index( P.m, p.b, p.c );
            {
                const float2 sg = P.m.sigma[ ci ];
                p.w = __fmul_rn( p.w, __fdiv_rn( sg.x, __fadd_rn( sg.x, sg.y ) ) );
                if( pass == 1 && R != 0.0 )
                    add_grad< TALLY >( P.g_int, ci, __ddiv_rn( R, ( double ) sg.x ), P.g_scale );
            }
            ++ nv;
            bool do_peel = false;
            if( P.img_n > 0 )
            {
                const int pix = image_pixel( P, p.x );
                if( pix >= 0 )
                {
                    float Q, U, V;
                    sp.I[ th ] = phys::peel_stokes( P.ph, p.d, p.e1, p.S, P.o, P.ev, P.eh, Q, U, V );
                    sp.Q[ th ] = Q; sp.U[ th ] = U; sp.V[ th ] = V;
                    sp.w[ th ] = p.w;
                    sp.pix[ th ] = pix;
                    do_peel = true;
                }
            }
            int end = 0;
            if( p.n_scat >= P.max_scatter )
                end = PK_SCATTER_CAP;
            else if( p.w < P.w_min )
            {
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
            store_cold( sc, p );
            phase = PH_SEGMENT;
            if( do_peel )
            {
                pend = end;
                ptau = 0.f; pk = 0; ptc = 0.0;
                if( pass == 0 || nv > ADJ_KMAX )
                {
                    park_walk( sp, p );
                    park_dir( sd, p, P.o, P.inv_o );
                    oray_faces( P, p.b, p.c, p.x, fx );
                    ray = RAY_MEASURE;
                    remeasure = pass == 1;
                    continue;
                }
                pG = gk[ nv - 1 ];
                if( pG != 0.0f )
                {
                    park_walk( sp, p );
                    park_dir( sd, p, P.o, P.inv_o );
                    oray_faces( P, p.b, p.c, p.x, fx );
                    ray = RAY_DEPOSIT;
                    continue;
                }
            }
            if( end )
                end_packet(  );
            else
                faces_all( P.m, p.b, p.c, p.d, fx );
            continue;
        }

        // ---- PH_SEGMENT ----
        if( phase != PH_SEGMENT ) continue;
        const bool peel = ray != RAY_WALK;
        const size_t ci = cell_index( P.m, p.b, p.c );
        const float ext = P.m.ext[ ci ];
        int ax;                                   // p.d / p.inv: the active ray's
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
            if( ray == RAY_DEPOSIT && ! peel_cut )
                add_grad< TALLY >( P.g_len, ci, __dmul_rn( -( double ) pG, t ), P.g_scale );
        }
        else
        {
            if( counting(  ) ) ++ cnt.steps;
            ++ p.n_steps;
            interact = et >= p.tau;
        }
        if( interact )
        {
            double ti = ( double ) __fdiv_rn( p.tau, ext );
            ti = ti > t ? t : ti;
            if( pass == 1 && R != 0.0 )
                add_grad< TALLY >( P.g_len, ci, __dmul_rn( -R, ti ), P.g_scale );
            p.x[ 0 ] = __fma_rn( ti, ( double ) p.d.x, p.x[ 0 ] );
            p.x[ 1 ] = __fma_rn( ti, ( double ) p.d.y, p.x[ 1 ] );
            p.x[ 2 ] = __fma_rn( ti, ( double ) p.d.z, p.x[ 2 ] );
            phase = PH_EVENT;
            continue;
        }
        if( ! peel_cut )
        {
            bool in_block;
            if( peel )
                in_block = oray_step_in_block( P, p.b, p.c, p.x, fx, ax );
            else
            {
                p.tau = __fsub_rn( p.tau, et );
                if( pass == 1 && R != 0.0 )
                    add_grad< TALLY >( P.g_len, ci, __dmul_rn( -R, t ), P.g_scale );
                #pragma unroll
                for( int a = 0; a < 3; ++ a )
                    if( a != ax ) p.x[ a ] = __fma_rn( t, ( double ) comp( p.d, a ), p.x[ a ] );
                in_block = step_in_block( P.m, p.b, p.c, p.x, fx, ax, p.d );
            }
            if( ! in_block )
            {   // leaves the block: wait for a batched hand-off
                hop_ax = ax;
                phase = PH_HOP;
                continue;
            }
        }
        after_crossing( peel_cut, false, false );
    }
    count_all( sp, KP_CNT_STEPS, cnt.steps );
    count_all( sp, KP_CNT_PEEL_STEPS, cnt.peel );
    __syncthreads(  );
    if( P.counters && threadIdx.x < KP_NCOUNTERS && sp.cnt[ threadIdx.x ] )
        atomicAdd( P.counters + threadIdx.x, sp.cnt[ threadIdx.x ] );
}

// Deferred adjoint, the walks.  PASS 0 walks every packet of the launch and
// queues the peel-off ray of each vertex (the emission of an isotropic point
// source and every interaction, when its point projects into the image) as
// a task, linked in vertex order per packet; a packet whose ray finds the
// queue full is flagged and listed for k_adjoint.  k_peel (mode 1) then
// measures each ray's score G, k_adj_fold sums them per packet.  PASS 1
// replays the walks with R, the sum of the scores of the interactions still
// ahead (adj_R0 at the start, minus each vertex's G after it), and deposits
// -R * length along the walk and R / sigma_sca at interactions; k_peel
// (mode 2) deposits along the rays.  Per packet this is k_adjoint's
// arithmetic in k_adjoint's order, so the int64 gradients are the same.
template< int TALLY, int PASS >
__global__ void __launch_bounds__( FWD_THREADS, 3 )
k_adj_walk( const __grid_constant__ fwd_params_t P )
{
    struct cnt_park_t { unsigned long long cnt[ KP_NCOUNTERS ]; };
    __shared__ cnt_park_t sp;
    __shared__ cold_park_t< FWD_THREADS > sc;
    const unsigned FULL = 0xffffffffu;
    const unsigned lane = threadIdx.x & 31u;
    if( threadIdx.x < KP_NCOUNTERS ) sp.cnt[ threadIdx.x ] = 0;
    __syncthreads(  );
    counts32_t cnt;
    packet_t p;
    double fx[ 3 ];
    int phase = PH_EMIT, hop_ax = 0;
    int lp = 0;        // the packet's index in the launch
    int link = -1;     // PASS 0: its last task (-1 none, -2 the queue overflowed);
                       // PASS 1: its next task
    double R = 0.0;    // PASS 1

    // PASS 0: queues the ray of vertex kv (toward the observer, weight w,
    // Stokes I, Q, U, V), the lanes together with one atomic.
    auto queue_ray = [ & ]( int pix, float w, float I, float Q, float U, float V, int kv )
    {
        const unsigned m = __activemask(  );
        const int leader = __ffs( m ) - 1;
        unsigned long long base = 0;
        if( ( int ) lane == leader )
            base = atomicAdd( P.pq_count, ( unsigned long long ) __popc( m ) );
        base = __shfl_sync( m, base, leader );
        const unsigned long long k = base + __popc( m & ( ( 1u << lane ) - 1u ) );
        if( k >= ( unsigned long long ) P.pq_cap )
        {   // the whole packet goes to k_adjoint
            link = -2;
            P.adj_flag[ lp ] = 1;
            P.adj_list[ atomicAdd( P.adj_list_n, 1ull ) ] = lp;
            return;
        }
        store_task( P.pq, k, p.x, p.b, p.c, w, I, Q, U, V, pix, 0 );
        P.pq_link[ k ] = peel_link_t { lp, kv, -1 };
        if( link >= 0 ) P.pq_link[ link ].next = ( int ) k;
        else P.adj_head[ lp ] = ( int ) k;
        link = ( int ) k;
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
        else if( n_emit > 0 && ( n_emit >= P.ev_batch || n_seg == 0 ) )
            run = PH_EMIT;
        else if( n_hop > 0 && ( n_hop >= P.hop_batch || n_seg == 0 ) )
            run = PH_HOP;
        else
            run = PH_SEGMENT;

        if( run == PH_HOP )
        {
            if( phase != PH_HOP ) continue;
            const int b_old = p.b;
            bool lost;
            const bool left = ! cross_face( P.m, p.b, p.c, p.x, hop_ax,
                                            comp( p.d, hop_ax ) > 0.0f, lost );
            if( left )
            {
                count( sp, lost ? KP_CNT_LOST : KP_CNT_ESCAPED );
                phase = PH_EMIT;
                continue;
            }
            faces_all( P.m, p.b, p.c, p.d, fx );
            if( p.b != b_old ) count( sp, KP_CNT_HOPS );
            if( p.n_steps >= P.max_steps )
            {
                count( sp, KP_CNT_CAPPED );
                phase = PH_EMIT;
            }
            else
                phase = PH_SEGMENT;
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
            const unsigned long long idx = base + rank;
            if( idx >= ( unsigned long long ) P.n_packets )
            {
                phase = PH_DONE;
                continue;
            }
            lp = ( int ) source_major( ( long long ) idx, P.n_packets, P.n_src );
            if constexpr( PASS == 1 )
                if( P.adj_flag[ lp ] )
                    continue;                     // replayed by k_adjoint
            const long long pid = P.pid0 + ( long long ) lp;
            float peel_I;
            if( ! emit_any( P, pid, p, peel_I ) )
            {
                atomicOr( P.m.status, ST_BAD_SOURCE );
                continue;
            }
            if constexpr( PASS == 0 )
            {
                count( sp, KP_CNT_EMITTED );
                link = -1;
            }
            else
            {
                link = P.adj_head[ lp ];
                R = P.adj_R0[ lp ];
            }
            p.tau = sample_tau( p.rng );
            store_cold( sc, p );
            if( P.img_n > 0 && peel_I > 0.0f )
            {   // direct light of the emission (unpolarized)
                const int pix = image_pixel( P, p.x );
                if( pix >= 0 )
                {
                    if constexpr( PASS == 0 )
                        queue_ray( pix, p.w, peel_I, 0.0f, 0.0f, 0.0f, 0 );
                    else if( link >= 0 )
                        link = P.pq_link[ link ].next;     // its ray is deposited by k_peel
                }
            }
            faces_all( P.m, p.b, p.c, p.d, fx );
            phase = PH_SEGMENT;
            continue;
        }

        if( run == PH_EVENT )
        {
            if( phase != PH_EVENT ) continue;
            load_cold( sc, p, P.seed );
            ++ p.n_scat;
            count( sp, KP_CNT_SCATTER );
            const size_t ci = cell_index( P.m, p.b, p.c );
            {
                const float2 sg = P.m.sigma[ ci ];
                p.w = __fmul_rn( p.w, __fdiv_rn( sg.x, __fadd_rn( sg.x, sg.y ) ) );
                if constexpr( PASS == 1 )
                    if( R != 0.0 )
                        add_grad< TALLY >( P.g_int, ci, __ddiv_rn( R, ( double ) sg.x ), P.g_scale );
            }
            if( P.img_n > 0 )
            {
                const int pix = image_pixel( P, p.x );
                if( pix >= 0 )
                {
                    if constexpr( PASS == 0 )
                    {
                        if( link != -2 )
                        {
                            float Q, U, V;
                            const float I = phys::peel_stokes( P.ph, p.d, p.e1, p.S, P.o, P.ev,
                                                               P.eh, Q, U, V );
                            queue_ray( pix, p.w, I, Q, U, V, p.n_scat );
                        }
                    }
                    else if( link >= 0 )
                    {   // this vertex's score leaves R once its ray is deposited
                        const float G = P.adj_G[ link ];
                        link = P.pq_link[ link ].next;
                        if( G != 0.0f )
                            R = __dsub_rn( R, ( double ) G );
                    }
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
            if( end )
                phase = PH_EMIT;
            else
            {
                store_cold( sc, p );
                faces_all( P.m, p.b, p.c, p.d, fx );
                phase = PH_SEGMENT;
            }
            continue;
        }

        // ---- PH_SEGMENT: walk segments, up to KP_WALK_INNER per round ----
        if( phase != PH_SEGMENT ) continue;
        #pragma unroll 1
        for( int it = 0; it < KP_WALK_INNER; ++ it )
        {
            const size_t ci = cell_index( P.m, p.b, p.c );
            const float ext = P.m.ext[ ci ];
            int ax;
            const double t = exit_cached( p.x, fx, p.d, p.inv, ax );
            const float et = __fmul_rn( ext, ( float ) t );
            ++ cnt.steps;
            ++ p.n_steps;
            if( et >= p.tau )
            {
                double ti = ( double ) __fdiv_rn( p.tau, ext );
                ti = ti > t ? t : ti;
                if constexpr( PASS == 1 )
                    if( R != 0.0 )
                        add_grad< TALLY >( P.g_len, ci, __dmul_rn( -R, ti ), P.g_scale );
                p.x[ 0 ] = __fma_rn( ti, ( double ) p.d.x, p.x[ 0 ] );
                p.x[ 1 ] = __fma_rn( ti, ( double ) p.d.y, p.x[ 1 ] );
                p.x[ 2 ] = __fma_rn( ti, ( double ) p.d.z, p.x[ 2 ] );
                phase = PH_EVENT;
                break;
            }
            p.tau = __fsub_rn( p.tau, et );
            if constexpr( PASS == 1 )
                if( R != 0.0 )
                    add_grad< TALLY >( P.g_len, ci, __dmul_rn( -R, t ), P.g_scale );
            #pragma unroll
            for( int a = 0; a < 3; ++ a )
                if( a != ax ) p.x[ a ] = __fma_rn( t, ( double ) comp( p.d, a ), p.x[ a ] );
            if( ! step_in_block( P.m, p.b, p.c, p.x, fx, ax, p.d ) )
            {   // leaves the block: wait for a batched hand-off
                hop_ax = ax;
                phase = PH_HOP;
                break;
            }
            if( p.n_steps >= P.max_steps )
            {
                count( sp, KP_CNT_CAPPED );
                phase = PH_EMIT;
                break;
            }
        }
    }
    count_all( sp, KP_CNT_STEPS, cnt.steps );
    __syncthreads(  );
    if( P.counters && threadIdx.x < KP_NCOUNTERS && sp.cnt[ threadIdx.x ] )
        atomicAdd( P.counters + threadIdx.x, sp.cnt[ threadIdx.x ] );
}

// Deferred adjoint: R of each packet, the sum of its interactions' scores in
// vertex order (k_adjoint's first replay).  Task indices grow along a
// packet's list, which bounds the walk through it.
__global__ void k_adj_fold( const __grid_constant__ fwd_params_t P )
{
    for( long long lp = blockIdx.x * ( long long ) blockDim.x + threadIdx.x; lp < P.n_packets;
         lp += ( long long ) gridDim.x * blockDim.x )
    {
        if( P.adj_flag[ lp ] ) continue;
        double R = 0.0;
        for( int t = P.adj_head[ lp ]; t >= 0; )
        {
            const peel_link_t o = P.pq_link[ t ];
            if( o.kv > 0 )
                R = __dadd_rn( R, ( double ) P.adj_G[ t ] );
            const int nx = o.next;
            t = nx > t ? nx : -1;
        }
        P.adj_R0[ lp ] = R;
    }
}

// Adjoint of a taped solve: the score of every queued ray from the
// attenuation the solve's march kept (k_peel mode 3), with the expression of
// the measuring march (k_peel mode 1).  Rays of flagged packets are skipped.
__global__ void k_adj_score( const __grid_constant__ fwd_params_t P )
{
    const long long n = min( * P.pq_count, ( unsigned long long ) P.pq_cap );
    for( long long t = blockIdx.x * ( long long ) blockDim.x + threadIdx.x; t < n;
         t += ( long long ) gridDim.x * blockDim.x )
    {
        if( P.adj_flag[ P.pq_link[ t ].lp ] ) continue;
        const task_dep_t o = load_task_deposit( P.pq, t );
        const float att = P.adj_att[ t ];
        float G = 0.0f;
        if( att >= 0.0f )
            G = score( P, o.pix, __fmul_rn( att, o.I ), __fmul_rn( att, o.Q ),
                       __fmul_rn( att, o.U ), __fmul_rn( att, o.V ) );
        P.adj_G[ t ] = G;
    }
}

// Deferred adjoint: adds the private path-length tallies of the depositing
// march into grad_len (integer sums: the same result in any order).
template< int TALLY >
__global__ void k_adj_reduce( const __grid_constant__ fwd_params_t P )
{
    const long long n = ( long long ) P.m.n_blocks * P.m.cpb;
    for( long long i = blockIdx.x * ( long long ) blockDim.x + threadIdx.x; i < n;
         i += ( long long ) gridDim.x * blockDim.x )
    {
        if constexpr( TALLY == KP_TALLY_FIXED )
        {
            const unsigned long long * q = static_cast< const unsigned long long * >( P.adj_priv );
            unsigned long long v = 0;
            for( int k = 0; k < P.adj_npriv; ++ k ) v += q[ k * n + i ];
            if( v ) static_cast< unsigned long long * >( P.g_len )[ i ] += v;
        }
        else
        {
            const float * q = static_cast< const float * >( P.adj_priv );
            float v = 0.0f;
            for( int k = 0; k < P.adj_npriv; ++ k ) v = __fadd_rn( v, q[ k * n + i ] );
            if( v != 0.0f ) static_cast< float * >( P.g_len )[ i ] += v;
        }
    }
}

}   // namespace
}   // namespace kp

namespace kp
{
void adjoint_buffers( kp_mesh_t * mesh, fwd_params_t & P, long long n_pk )
{
    const long long cap = mesh->pq_cap;
    const long long n_cells = ( long long ) P.m.n_blocks * P.m.cpb;
    const int n_priv = KP_ADJ_PRIV;
    const size_t priv_bytes = n_priv > 1 ? ( size_t ) n_priv * n_cells * 8 : 0;
    // 256 B of counters, the per-packet and per-task arrays, then the private
    // tallies (256-byte aligned)
    const size_t adj_bytes = ( 256 + ( size_t ) n_pk * ( sizeof( double ) + 3 * sizeof( int ) )
                               + ( size_t ) cap * ( 2 * sizeof( float ) + sizeof( peel_link_t ) )
                               + 255 ) & ~( size_t ) 255;
    if( mesh->adj_bytes < adj_bytes + priv_bytes )
    {
        cudaFree( mesh->d_adj );
        mesh->d_adj = nullptr;
        mesh->adj_bytes = 0;
        mesh->tape_id = 0;
        KP_CUDA( cudaMalloc( & mesh->d_adj, adj_bytes + priv_bytes ) );
        mesh->adj_bytes = adj_bytes + priv_bytes;
    }
    char * a = static_cast< char * >( mesh->d_adj );
    P.work     = reinterpret_cast< unsigned long long * >( a );
    P.pq_count = P.work + 1;
    P.pq_next  = P.work + 2;
    P.adj_list_n = P.work + 3;
    a += 256;
    P.adj_R0   = reinterpret_cast< double * >( a );
    P.adj_G    = reinterpret_cast< float * >( a + n_pk * sizeof( double ) );
    P.adj_att  = P.adj_G + cap;
    P.adj_head = reinterpret_cast< int * >( P.adj_att + cap );
    P.adj_flag = P.adj_head + n_pk;
    P.adj_list = P.adj_flag + n_pk;
    P.pq_link  = reinterpret_cast< peel_link_t * >( P.adj_list + n_pk );
    P.adj_priv = n_priv > 1 ? static_cast< char * >( mesh->d_adj ) + adj_bytes : nullptr;
    P.adj_npriv = n_priv > 1 ? n_priv : 0;
    P.pq = static_cast< peel_task_t * >( mesh->d_pq );
    P.pq_cap = cap;
}
}   // namespace kp

namespace
{
// Launch parameters of an adjoint: the forward's, with the image tallies
// replaced by the gradient outputs.
void adjoint_params( kp_mesh_t * mesh, const kp_transport_cfg_t * cfg, const float * adj_image,
                     int grad_fx_shift, void * grad_len, void * grad_int,
                     unsigned long long * counters, kp::fwd_params_t & P )
{
    kp::require( mesh && cfg && adj_image && grad_len && grad_int, "null argument" );
    kp::require( cfg->image_n > 0, "the adjoint needs a peel-off image (image_n > 0)" );
    kp::require( grad_fx_shift >= 0 && grad_fx_shift <= 48, "grad_fx_shift out of range" );
    mesh->upload(  );
    kp_tallies_t none {  };
    none.counters = counters;
    // the forward's image buffers are not written by the adjoint; any
    // non-null placeholders pass the configuration checks
    none.image = grad_len;
    none.image_batch = grad_len;
    none.mu = grad_len;
    kp_transport_cfg_t c = * cfg;
    c.n_record = 0;
    kp::make_fwd_params( mesh, c, none, P );
    P.image = P.img_batch = P.mu_tally = nullptr;
    P.adj_img = reinterpret_cast< const float4 * >( adj_image );
    P.g_len = grad_len;
    P.g_int = grad_int;
    P.g_scale = std::ldexp( 1.0, grad_fx_shift );
}

// The adjoint once every queued ray of the chunk C has its score in adj_G:
// R per packet, the second replay, the deposits along the rays, and the
// packets left to k_adjoint (whose first replay counts nothing).
void adjoint_second_half( kp::fwd_params_t & C, int tally_mode, cudaStream_t s )
{
    const bool fx = tally_mode == KP_TALLY_FIXED;
    const int threads = kp::FWD_THREADS;
    const long long n_cells = ( long long ) C.m.n_blocks * C.m.cpb;
    const void * kw = fx ? ( const void * ) kp::k_adj_walk< KP_TALLY_FIXED, 1 >
                         : ( const void * ) kp::k_adj_walk< KP_TALLY_FLOAT, 1 >;
    const void * ka = fx ? ( const void * ) kp::k_adjoint< KP_TALLY_FIXED >
                         : ( const void * ) kp::k_adjoint< KP_TALLY_FLOAT >;
    const long long blocks = ( C.n_packets + threads - 1 ) / threads;
    const unsigned gw = ( unsigned ) std::min< long long >( kp::persistent_grid( kw, threads ), blocks );
    const unsigned ga = ( unsigned ) std::min< long long >( kp::persistent_grid( ka, threads ), blocks );
    const unsigned gf = ( unsigned ) std::min< long long >( 4096, ( C.n_packets + 255 ) / 256 );
    kp::k_adj_fold<<< gf, 256, 0, s >>>( C );                           // R per packet
    KP_CUDA( cudaGetLastError(  ) );
    KP_CUDA( cudaMemsetAsync( C.work, 0, sizeof( unsigned long long ), s ) );
    if( fx ) kp::k_adj_walk< KP_TALLY_FIXED, 1 ><<< gw, threads, 0, s >>>( C );
    else     kp::k_adj_walk< KP_TALLY_FLOAT, 1 ><<< gw, threads, 0, s >>>( C );
    KP_CUDA( cudaGetLastError(  ) );
    if( C.adj_priv )
        KP_CUDA( cudaMemsetAsync( C.adj_priv, 0, ( size_t ) C.adj_npriv * n_cells * ( fx ? 8 : 4 ), s ) );
    kp::launch_peel_adjoint( C, tally_mode, 2, s );
    if( C.adj_priv )
    {
        const unsigned gr = ( unsigned ) std::min< long long >( 4096, ( n_cells + 255 ) / 256 );
        if( fx ) kp::k_adj_reduce< KP_TALLY_FIXED ><<< gr, 256, 0, s >>>( C );
        else     kp::k_adj_reduce< KP_TALLY_FLOAT ><<< gr, 256, 0, s >>>( C );
        KP_CUDA( cudaGetLastError(  ) );
    }
    // packets whose rays found the queue full: both replays inline
    KP_CUDA( cudaMemsetAsync( C.work, 0, sizeof( unsigned long long ), s ) );
    C.adj_quiet = 1;
    if( fx ) kp::k_adjoint< KP_TALLY_FIXED ><<< ga, threads, 0, s >>>( C );
    else     kp::k_adjoint< KP_TALLY_FLOAT ><<< ga, threads, 0, s >>>( C );
    KP_CUDA( cudaGetLastError(  ) );
}

// The fields of two solve configurations that decide the packets' paths and
// their peel-off rays.
bool same_solve( const kp_transport_cfg_t & a, const kp_source_t * sa, const kp_transport_cfg_t & b )
{
    bool eq = a.n_packets == b.n_packets && a.packet_offset == b.packet_offset
           && a.seed == b.seed && a.stream_id == b.stream_id && a.phase == b.phase
           && a.hg_g == b.hg_g && a.pol_max == b.pol_max && a.n_sources == b.n_sources
           && a.image_n == b.image_n && a.inclination_deg == b.inclination_deg
           && a.azimuth_deg == b.azimuth_deg && a.image_half_width == b.image_half_width
           && a.tau_peel_max == b.tau_peel_max && a.w_min == b.w_min
           && a.rr_survive == b.rr_survive && a.max_scatter == b.max_scatter
           && a.max_steps == b.max_steps && a.packets == b.packets
           && ( b.sources != nullptr || b.packets != nullptr );
    for( int k = 0; eq && k < 3; ++ k ) eq = a.image_center[ k ] == b.image_center[ k ];
    for( int k = 0; eq && k < b.n_sources; ++ k )
    {
        const kp_source_t & x = sa[ k ], & y = b.sources[ k ];
        eq = x.kind == y.kind && x.emit == y.emit && x.pos[ 0 ] == y.pos[ 0 ]
          && x.pos[ 1 ] == y.pos[ 1 ] && x.pos[ 2 ] == y.pos[ 2 ];
    }
    return eq;
}
}   // namespace

extern "C" int kp_transport_adjoint( kp_mesh_t * mesh, const kp_transport_cfg_t * cfg,
                                     const float * adj_image, int grad_fx_shift,
                                     void * grad_len, void * grad_int,
                                     unsigned long long * counters, void * stream )
{
    return kp::guarded( "kp_transport_adjoint", [ & ]
    {
        static thread_local kp::fwd_params_t P;
        adjoint_params( mesh, cfg, adj_image, grad_fx_shift, grad_len, grad_int, counters, P );
        if( P.n_packets == 0 ) return;
        auto s = ( cudaStream_t ) stream;
        mesh->refresh_ext( s );
        const bool fx = cfg->tally_mode == KP_TALLY_FIXED;
        const int threads = kp::FWD_THREADS;
        mesh->tape_id = 0;                  // the queue is overwritten
        // The vertices' peel-off rays go through the mesh's queue (12 rays per
        // packet, chunks of packets beyond that) and are marched by k_peel.
        kp::ensure_peel_queue( mesh, P.n_packets );
        const long long chunk = std::max< long long >( mesh->pq_cap / kp::PQ_PER_PACKET, 1 );
        kp::adjoint_buffers( mesh, P, std::min( chunk, P.n_packets ) );
        // both marches read the queue in the forward solve's order
        int * perm = kp::peel_sorted( mesh ) ? kp::ensure_task_sort( mesh, mesh->pq_cap ) : nullptr;
        const void * kw0 = fx ? ( const void * ) kp::k_adj_walk< KP_TALLY_FIXED, 0 >
                              : ( const void * ) kp::k_adj_walk< KP_TALLY_FLOAT, 0 >;
        const long long grid_w = kp::persistent_grid( kw0, threads );
        static thread_local kp::fwd_params_t C;
        for( long long done = 0; done < P.n_packets; done += chunk )
        {
            C = P;
            C.pq_perm = perm;
            C.pid0 = P.pid0 + done;
            C.n_packets = std::min( chunk, P.n_packets - done );
            const unsigned gw = ( unsigned ) std::min< long long >( grid_w,
                                                                   ( C.n_packets + threads - 1 ) / threads );
            KP_CUDA( cudaMemsetAsync( C.work, 0, 4 * sizeof( unsigned long long ), s ) );
            KP_CUDA( cudaMemsetAsync( C.adj_head, 0xff, C.n_packets * sizeof( int ), s ) );
            KP_CUDA( cudaMemsetAsync( C.adj_flag, 0, C.n_packets * sizeof( int ), s ) );
            // first replay: walks, vertex rays queued
            if( fx ) kp::k_adj_walk< KP_TALLY_FIXED, 0 ><<< gw, threads, 0, s >>>( C );
            else     kp::k_adj_walk< KP_TALLY_FLOAT, 0 ><<< gw, threads, 0, s >>>( C );
            KP_CUDA( cudaGetLastError(  ) );
            if( perm ) kp::task_sort( mesh, C, s );                     // by starting cell
            kp::launch_peel_adjoint( C, cfg->tally_mode, 1, s );       // scores G
            adjoint_second_half( C, cfg->tally_mode, s );
        }
    } );
}

extern "C" int kp_transport_forward_tape( kp_mesh_t * mesh, const kp_transport_cfg_t * cfg,
                                          const kp_tallies_t * tallies, void * stream,
                                          long long * tape_id )
{
    return kp::guarded( "kp_transport_forward_tape", [ & ]
    {
        kp::require( mesh && cfg && tallies && tape_id, "null argument" );
        * tape_id = 0;
        kp::require( cfg->image_n > 0, "a taped solve needs a peel-off image (image_n > 0)" );
        mesh->upload(  );
        mesh->tape_id = 0;
        static thread_local kp::fwd_params_t P;
        kp::make_fwd_params( mesh, * cfg, * tallies, P );
        if( P.n_packets == 0 ) return;
        mesh->refresh_ext( ( cudaStream_t ) stream );
        if( cfg->lane_batch == 0 ) P.ev_batch = 12;
        kp::ensure_peel_queue( mesh, P.n_packets );
        if( P.n_packets > std::max< long long >( mesh->pq_cap / kp::PQ_PER_PACKET, 1 ) )
        {   // more packets than one chunk of the queue: an untaped solve
            P.work = mesh->workspace(  );
            kp::launch_deferred_solve( mesh, P, cfg->tally_mode, ( cudaStream_t ) stream );
            kp::fold_carry( * cfg, * tallies, ( cudaStream_t ) stream );
            return;
        }
        kp::adjoint_buffers( mesh, P, P.n_packets );
        // the march order; the gradient's depositing march reads the same
        // permutation, which lives as long as the tape (every solve that
        // overwrites the queue drops the tape)
        const bool sorted = kp::peel_sorted( mesh );
        P.pq_perm = sorted ? kp::ensure_task_sort( mesh, mesh->pq_cap ) : nullptr;
        auto s = ( cudaStream_t ) stream;
        KP_CUDA( cudaMemsetAsync( P.work, 0, 4 * sizeof( unsigned long long ), s ) );
        KP_CUDA( cudaMemsetAsync( P.adj_head, 0xff, P.n_packets * sizeof( int ), s ) );
        KP_CUDA( cudaMemsetAsync( P.adj_flag, 0, P.n_packets * sizeof( int ), s ) );
        if( cfg->tally_mode == KP_TALLY_FIXED )
            kp::launch_deferred_chunk< KP_TALLY_FIXED, true >( P, s, mesh );
        else
            kp::launch_deferred_chunk< KP_TALLY_FLOAT, true >( P, s, mesh );
        kp::fold_carry( * cfg, * tallies, s );
        mesh->tape_cfg = * cfg;
        mesh->tape_cfg.sources = nullptr;
        for( int k = 0; k < cfg->n_sources; ++ k ) mesh->tape_src[ k ] = cfg->sources[ k ];
        mesh->tape_n = P.n_packets;
        mesh->tape_sorted = sorted;
        mesh->tape_id = ++ mesh->tape_serial;
        * tape_id = mesh->tape_id;
    } );
}

extern "C" int kp_transport_adjoint_tape( kp_mesh_t * mesh, long long tape_id,
                                          const kp_transport_cfg_t * cfg, const float * adj_image,
                                          int grad_fx_shift, void * grad_len, void * grad_int,
                                          unsigned long long * counters, void * stream )
{
    return kp::guarded( "kp_transport_adjoint_tape", [ & ]
    {
        kp::require( mesh && cfg, "null argument" );
        kp::require( tape_id > 0 && tape_id == mesh->tape_id,
                     "no taped solve with this id on the mesh (a later solve or new "
                     "coefficients replaced it)", KP_ERR_CONFIG );
        kp::require( same_solve( mesh->tape_cfg, mesh->tape_src, * cfg ),
                     "cfg differs from the taped solve's", KP_ERR_CONFIG );
        static thread_local kp::fwd_params_t P;
        adjoint_params( mesh, cfg, adj_image, grad_fx_shift, grad_len, grad_int, counters, P );
        kp::adjoint_buffers( mesh, P, mesh->tape_n );      // the taped solve's layout
        P.pq_perm = mesh->tape_sorted ? mesh->d_sort_perm : nullptr;   // ... and order
        auto s = ( cudaStream_t ) stream;
        mesh->refresh_ext( s );
        const unsigned gs = 4 * 148;
        kp::k_adj_score<<< gs, 256, 0, s >>>( P );                        // G from the tape
        KP_CUDA( cudaGetLastError(  ) );
        adjoint_second_half( P, cfg->tally_mode, s );
    } );
}

extern "C" int kp_mesh_tape_id( const kp_mesh_t * mesh, long long * tape_id )
{
    return kp::guarded( "kp_mesh_tape_id", [ & ]
    {
        kp::require( mesh && tape_id, "null argument" );
        * tape_id = mesh->tape_id;
    } );
}
