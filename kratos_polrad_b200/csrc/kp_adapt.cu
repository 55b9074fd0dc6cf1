// Runtime refinement of the block tree: per-block flags from the coefficient
// field, the adapted mesh, and the remapping of per-cell fields onto it.
//
// The reference declares the hook and leaves it empty: mesh_t::changed
// returns false (mesh/mesh.cpp:86-89), meshgen::base_t::update does nothing
// (mesh/meshgen/meshgen.cpp:443-446), and block_map_t::update
// (modules/particle/types/block_map.h:53-103) would rebuild the neighbour
// tables.  Here an adapted mesh is a new tree built from the desired leaves
// with the static-refinement 2:1 closure, so its blocks and tables are those
// the reference builds from one refine box per leaf.
#include "kp_common.cuh"

#include <vector>

using kp::guarded;
using kp::require;

namespace kp
{
namespace
{

// +1 where some cell's extinction depth across the block's widest cell side
// exceeds tau_refine, -1 where every cell's stays below tau_coarsen, else 0.
// One CTA per block; the max is order-independent.
__global__ void k_flag_tau( const mesh_view_t m, float tau_refine, float tau_coarsen, int * flags )
{
    __shared__ float red[ 32 ];
    const int b = blockIdx.x;
    const double * g = m.geo_d + 16 * ( size_t ) b;
    const float dx = ( float ) fmax( g[ 3 ], fmax( g[ 4 ], g[ 5 ] ) );
    float mx = 0.0f;
    for( int i = threadIdx.x; i < m.cpb; i += blockDim.x )
    {
        const float2 s = m.sigma[ ( size_t ) b * m.cpb + i ];
        mx = fmaxf( mx, __fmul_rn( __fadd_rn( s.x, s.y ), dx ) );
    }
    for( int o = 16; o > 0; o >>= 1 )
        mx = fmaxf( mx, __shfl_xor_sync( 0xffffffffu, mx, o ) );
    if( ( threadIdx.x & 31 ) == 0 ) red[ threadIdx.x >> 5 ] = mx;
    __syncthreads(  );
    if( threadIdx.x == 0 )
    {
        float v = 0.0f;
        for( int w = 0; w < ( int ) ( blockDim.x + 31 ) / 32; ++ w ) v = fmaxf( v, red[ w ] );
        flags[ b ] = v > tau_refine ? 1 : ( v < tau_coarsen ? -1 : 0 );
    }
}

struct remap_params_t
{
    mesh_view_t from, to;
    double      lk_inv[ 3 ];     // from's lookup cells per unit length
    int         n_comp;
    const float * src;
    float       * dst;
};

// Flat cell index in `m` holding x, or -1.
__device__ __forceinline__ long long locate_flat( const mesh_view_t & m, const double lk_inv[ 3 ],
                                                  const double x[ 3 ] )
{
    int li[ 3 ];
    #pragma unroll
    for( int a = 0; a < 3; ++ a )
    {
        const double f = floor( __dmul_rn( __dsub_rn( x[ a ], m.xlim_d[ 0 ][ a ] ), lk_inv[ a ] ) );
        li[ a ] = f < 0.0 ? 0 : ( f >= m.lookup_n[ a ] ? m.lookup_n[ a ] - 1 : ( int ) f );
    }
    const int b = m.lookup[ ( ( size_t ) li[ 2 ] * m.lookup_n[ 1 ] + li[ 1 ] ) * m.lookup_n[ 0 ] + li[ 0 ] ];
    if( b < 0 || b >= m.n_blocks ) return -1;
    const double * h = m.geo_d + 16 * ( size_t ) b;
    int c[ 3 ];
    #pragma unroll
    for( int a = 0; a < 3; ++ a )
    {
        const double f = floor( __dmul_rn( __dsub_rn( x[ a ], h[ a ] ), h[ 8 + a ] ) );
        c[ a ] = f < 0.0 ? 0 : ( f > ( double ) ( m.nc[ a ] - 1 ) ? m.nc[ a ] - 1 : ( int ) f );
    }
    return ( long long ) b * m.cpb + c[ 0 ] + m.nc[ 0 ] * ( c[ 1 ] + m.nc[ 1 ] * c[ 2 ] );
}

// Each cell of `to` samples `from` at the centres of its eight octants: a
// cell inside one source cell (same level or refined) copies it, a cell
// covering several (coarsened) takes their mean, summed in octant order.
__global__ void k_remap( const __grid_constant__ remap_params_t R )
{
    const long long n = ( long long ) R.to.n_blocks * R.to.cpb;
    for( long long i = blockIdx.x * ( long long ) blockDim.x + threadIdx.x; i < n;
         i += ( long long ) gridDim.x * blockDim.x )
    {
        const int b = ( int ) ( i / R.to.cpb ), l = ( int ) ( i % R.to.cpb );
        const int c[ 3 ] = { l % R.to.nc[ 0 ], ( l / R.to.nc[ 0 ] ) % R.to.nc[ 1 ],
                             l / ( R.to.nc[ 0 ] * R.to.nc[ 1 ] ) };
        const double * h = R.to.geo_d + 16 * ( size_t ) b;
        long long idx[ 8 ];
        bool same = true, bad = false;
        for( int s = 0; s < 8; ++ s )
        {
            double x[ 3 ];
            #pragma unroll
            for( int a = 0; a < 3; ++ a )
                x[ a ] = __fma_rn( ( double ) c[ a ] + ( ( s >> a ) & 1 ? 0.75 : 0.25 ), h[ 3 + a ],
                                   h[ a ] );
            idx[ s ] = locate_flat( R.from, R.lk_inv, x );
            bad  = bad  || idx[ s ] < 0;
            same = same && idx[ s ] == idx[ 0 ];
        }
        if( bad )
        {
            atomicOr( R.to.status, ST_BAD_CELL );
            for( int k = 0; k < R.n_comp; ++ k ) R.dst[ i * R.n_comp + k ] = 0.0f;
            continue;
        }
        for( int k = 0; k < R.n_comp; ++ k )
        {
            float v = R.src[ idx[ 0 ] * R.n_comp + k ];
            if( ! same )
            {
                for( int s = 1; s < 8; ++ s ) v = __fadd_rn( v, R.src[ idx[ s ] * R.n_comp + k ] );
                v = __fmul_rn( v, 0.125f );
            }
            R.dst[ i * R.n_comp + k ] = v;
        }
    }
}

}   // namespace
}   // namespace kp

int kp_mesh_flag_tau( kp_mesh_t * mesh, float tau_refine, float tau_coarsen, int * flags,
                      void * stream )
{
    return guarded( "kp_mesh_flag_tau", [ & ]
    {
        require( mesh && flags, "null argument" );
        require( tau_coarsen <= tau_refine, "tau_coarsen must not exceed tau_refine" );
        mesh->upload(  );
        const kp::mesh_view_t v = mesh->view(  );
        kp::k_flag_tau<<< v.n_blocks, 256, 0, ( cudaStream_t ) stream >>>( v, tau_refine,
                                                                          tau_coarsen, flags );
        KP_CUDA( cudaGetLastError(  ) );
    } );
}

int kp_mesh_adapt( const kp_mesh_t * mesh, const int * flags, kp_mesh_t ** out )
{
    return guarded( "kp_mesh_adapt", [ & ]
    {
        require( mesh && flags && out, "null argument" );
        * out = nullptr;
        const auto & t = mesh->tree->tables(  );
        const int nb = t.n_blocks;
        std::map< kp::region_key_t, int > id;
        for( int b = 0; b < nb; ++ b )
            id[ { t.level[ b ], { t.reg[ 3 * b ], t.reg[ 3 * b + 1 ], t.reg[ 3 * b + 2 ] } } ] = b;
        std::vector< kp::region_key_t > keys;
        keys.reserve( nb );
        for( int b = 0; b < nb; ++ b )
        {
            const kp::region_key_t k { t.level[ b ], { t.reg[ 3 * b ], t.reg[ 3 * b + 1 ],
                                                       t.reg[ 3 * b + 2 ] } };
            if( flags[ b ] > 0 )
            {
                require( k.level < 20, "refinement level would exceed 20", KP_ERR_CAPACITY );
                for( int c = 0; c < 8; ++ c )
                    keys.push_back( { k.level + 1, { 2 * k.i[ 0 ] + ( c & 1 ),
                                                     2 * k.i[ 1 ] + ( ( c >> 1 ) & 1 ),
                                                     2 * k.i[ 2 ] + ( ( c >> 2 ) & 1 ) } } );
                continue;
            }
            if( flags[ b ] < 0 && k.level > 0 )
            {   // the parent, if all eight siblings are leaves asking to coarsen
                const kp::region_key_t p { k.level - 1, { k.i[ 0 ] >> 1, k.i[ 1 ] >> 1,
                                                          k.i[ 2 ] >> 1 } };
                bool all = true;
                for( int c = 0; c < 8 && all; ++ c )
                {
                    auto it = id.find( { k.level, { 2 * p.i[ 0 ] + ( c & 1 ),
                                                    2 * p.i[ 1 ] + ( ( c >> 1 ) & 1 ),
                                                    2 * p.i[ 2 ] + ( ( c >> 2 ) & 1 ) } } );
                    all = it != id.end(  ) && flags[ it->second ] < 0;
                }
                if( all )
                {
                    keys.push_back( p );
                    continue;
                }
            }
            keys.push_back( k );
        }
        auto m = std::make_unique< kp_mesh >(  );
        m->tree = std::make_unique< kp::block_tree_t >( mesh->tree->desc(  ), keys );
        * out = m.release(  );
    } );
}

int kp_mesh_remap( kp_mesh_t * from, kp_mesh_t * to, int n_comp, const float * src, float * dst,
                   void * stream )
{
    return guarded( "kp_mesh_remap", [ & ]
    {
        require( from && to && src && dst, "null argument" );
        require( n_comp >= 1 && n_comp <= 64, "n_comp must be in 1..64" );
        const auto & a = from->tree->desc(  );
        const auto & b = to->tree->desc(  );
        for( int k = 0; k < 3; ++ k )
            require( a.x_min[ k ] == b.x_min[ k ] && a.x_max[ k ] == b.x_max[ k ]
                     && a.n_cell_global[ k ] == b.n_cell_global[ k ]
                     && a.n_cell_block[ k ] == b.n_cell_block[ k ]
                     && a.periodic[ k ] == b.periodic[ k ],
                     "meshes of different domains", KP_ERR_CONFIG );
        from->upload(  );
        to->upload(  );
        kp::remap_params_t R {  };
        R.from = from->view(  );
        R.to = to->view(  );
        const auto & ft = from->tree->tables(  );
        for( int k = 0; k < 3; ++ k ) R.lk_inv[ k ] = ft.lookup_n[ k ] / ft.l_box_d[ k ];
        R.n_comp = n_comp;
        R.src = src;
        R.dst = dst;
        const long long n = ( long long ) R.to.n_blocks * R.to.cpb;
        const int grid = ( int ) std::min< long long >( ( n + 255 ) / 256, 148 * 16 );
        kp::k_remap<<< grid, 256, 0, ( cudaStream_t ) stream >>>( R );
        KP_CUDA( cudaGetLastError(  ) );
    } );
}
