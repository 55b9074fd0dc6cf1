// Mesh entry points of the C ABI: build on the host, upload block tables.
#include "kp_common.cuh"
#include "host/ini.h"

#include <algorithm>
#include <cstring>
#include <vector>

using kp::guarded;
using kp::require;

kp::mesh_view_t kp_mesh::view(  ) const
{
    const auto & t = tree->tables(  );
    kp::mesh_view_t v {  };
    v.n_blocks = t.n_blocks;
    for( int a = 0; a < 3; ++ a ) v.nc[ a ] = t.nc[ a ];
    v.cpb   = t.cells_per_block;
    v.nb    = d_nb;
    v.meta  = d_meta;
    v.geo_d = d_geo_d;
    v.geo_f = d_geo_f;
    v.sigma = d_sigma;
    v.ext   = d_ext;
    v.lookup = d_lookup;
    for( int a = 0; a < 3; ++ a ) v.lookup_n[ a ] = t.lookup_n[ a ];
    v.max_level = t.max_level;
    v.periodic = 0;
    for( int a = 0; a < 3; ++ a )
    {
        if( t.periodic[ a ] ) v.periodic |= 1u << a;
        for( int l = 0; l < 2; ++ l )
        {
            v.xlim_d[ l ][ a ] = t.xlim_d[ l ][ a ];
            v.xlim_f[ l ][ a ] = t.xlim_f[ l ][ a ];
        }
        v.lbox_d[ a ] = t.l_box_d[ a ];
        v.lbox_f[ a ] = t.l_box_f[ a ];
    }
    v.status = d_status;
    v.rf_f = d_rf_f; v.rf_d = d_rf_d; v.vol_f = d_vol_f; v.vol_d = d_vol_d;
    return v;
}

namespace
{
__global__ void k_extinction( const float2 * __restrict__ sigma, float * __restrict__ ext,
                              long long n )
{
    const long long stride = ( long long ) gridDim.x * blockDim.x;
    for( long long i = ( long long ) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride )
    {
        const float2 s = sigma[ i ];
        ext[ i ] = __fadd_rn( s.x, s.y );
    }
}
}   // namespace

void kp::extinction( const float2 * sigma, float * ext, long long n, cudaStream_t s )
{
    if( n <= 0 ) return;
    int dev = 0, n_sm = 0;
    KP_CUDA( cudaGetDevice( & dev ) );
    KP_CUDA( cudaDeviceGetAttribute( & n_sm, cudaDevAttrMultiProcessorCount, dev ) );
    const long long grid = std::min< long long >( ( n + 255 ) / 256, 8ll * n_sm );
    k_extinction<<< ( unsigned ) grid, 256, 0, s >>>( sigma, ext, n );
    KP_CUDA( cudaGetLastError(  ) );
}

void kp_mesh::refresh_ext( cudaStream_t s )
{
    kp::require( d_sigma != nullptr && d_ext != nullptr, "mesh coefficients not on the device",
                 KP_ERR_CONFIG );
    const auto & t = tree->tables(  );
    kp::extinction( d_sigma, d_ext, ( long long ) t.n_blocks * t.cells_per_block, s );
}

void kp_mesh::upload( bool with_sigma )
{
    int dev = 0;
    KP_CUDA( cudaGetDevice( & dev ) );
    if( uploaded )
    {
        kp::require( dev == device, "mesh was uploaded to another device",
                     KP_ERR_CONFIG );
        if( with_sigma && d_sigma == nullptr )
        {
            const auto & t = tree->tables(  );
            const size_t n = ( size_t ) t.n_blocks * t.cells_per_block;
            KP_CUDA( cudaMalloc( & d_sigma, n * sizeof( float2 ) ) );
            KP_CUDA( cudaMemset( d_sigma, 0, n * sizeof( float2 ) ) );
            KP_CUDA( cudaMalloc( & d_ext, n * sizeof( float ) ) );
            KP_CUDA( cudaMemset( d_ext, 0, n * sizeof( float ) ) );
        }
        return;
    }
    const auto & t = tree->tables(  );
    const size_t nb = t.n_blocks;
    std::vector< kp::blk_meta_t > meta( nb );
    std::vector< double > gd( nb * 16, 0. );
    std::vector< float  > gf( nb * 8, 0.f );
    for( size_t b = 0; b < nb; ++ b )
    {
        auto & m = meta[ b ];
        std::memset( & m, 0, sizeof( m ) );
        for( int f = 0; f < 6; ++ f )
        {
            m.d_lvl[ f ] = t.d_lvl[ 6 * b + f ];
            m.shift[ f ] = t.nb_shift[ 24 * b + 4 * f ];   // slot [a][s][0][0]
        }
        m.phybnd = t.phybnd[ b ];
        for( int a = 0; a < 3; ++ a )
        {
            gd[ 16 * b + a ]     = t.xf0_d[ 3 * b + a ];
            gd[ 16 * b + 3 + a ] = t.dx0_d[ 3 * b + a ];
            gd[ 16 * b + 8 + a ] = 1.0 / t.dx0_d[ 3 * b + a ];
            gf[ 8 * b + a ]     = t.xf0_f[ 3 * b + a ];
            gf[ 8 * b + 3 + a ] = t.dx0_f[ 3 * b + a ];
        }
        gd[ 16 * b + 6 ] = t.vol0_d[ b ];
        gf[ 8 * b + 6 ] = t.vol0_f[ b ];
    }
    const size_t n_cells = nb * ( size_t ) t.cells_per_block;
    try
    {
        KP_CUDA( cudaMalloc( & d_nb,     nb * 24 * sizeof( int ) ) );
        KP_CUDA( cudaMalloc( & d_meta,   nb * sizeof( kp::blk_meta_t ) ) );
        KP_CUDA( cudaMalloc( & d_geo_d,  nb * 16 * sizeof( double ) ) );
        KP_CUDA( cudaMalloc( & d_lookup, t.lookup.size(  ) * sizeof( int ) ) );
        KP_CUDA( cudaMemcpy( d_lookup, t.lookup.data(  ), t.lookup.size(  ) * sizeof( int ),
                             cudaMemcpyHostToDevice ) );
        KP_CUDA( cudaMalloc( & d_geo_f,  nb * 8 * sizeof( float ) ) );
        if( with_sigma )
        {
            KP_CUDA( cudaMalloc( & d_sigma,  n_cells * sizeof( float2 ) ) );
            KP_CUDA( cudaMalloc( & d_ext,    n_cells * sizeof( float ) ) );
        }
        KP_CUDA( cudaMalloc( & d_status, 4 * sizeof( unsigned ) ) );
        KP_CUDA( cudaMalloc( & d_work, 32 * sizeof( unsigned long long ) ) );
        if( t.coord == 1 )
        {
            KP_CUDA( cudaMalloc( & d_rf_f, t.rf_f.size(  ) * sizeof( float ) ) );
            KP_CUDA( cudaMalloc( & d_rf_d, t.rf_d.size(  ) * sizeof( double ) ) );
            KP_CUDA( cudaMalloc( & d_vol_f, t.vol_f.size(  ) * sizeof( float ) ) );
            KP_CUDA( cudaMalloc( & d_vol_d, t.vol_d.size(  ) * sizeof( double ) ) );
            KP_CUDA( cudaMemcpy( d_rf_f, t.rf_f.data(  ), t.rf_f.size(  ) * sizeof( float ),
                                 cudaMemcpyHostToDevice ) );
            KP_CUDA( cudaMemcpy( d_rf_d, t.rf_d.data(  ), t.rf_d.size(  ) * sizeof( double ),
                                 cudaMemcpyHostToDevice ) );
            KP_CUDA( cudaMemcpy( d_vol_f, t.vol_f.data(  ), t.vol_f.size(  ) * sizeof( float ),
                                 cudaMemcpyHostToDevice ) );
            KP_CUDA( cudaMemcpy( d_vol_d, t.vol_d.data(  ), t.vol_d.size(  ) * sizeof( double ),
                                 cudaMemcpyHostToDevice ) );
        }
        KP_CUDA( cudaMemset( d_work, 0, 32 * sizeof( unsigned long long ) ) );
        KP_CUDA( cudaMemcpy( d_nb, t.nb_id.data(  ), nb * 24 * sizeof( int ),
                             cudaMemcpyHostToDevice ) );
        KP_CUDA( cudaMemcpy( d_meta, meta.data(  ), nb * sizeof( kp::blk_meta_t ),
                             cudaMemcpyHostToDevice ) );
        KP_CUDA( cudaMemcpy( d_geo_d, gd.data(  ), gd.size(  ) * sizeof( double ),
                             cudaMemcpyHostToDevice ) );
        KP_CUDA( cudaMemcpy( d_geo_f, gf.data(  ), gf.size(  ) * sizeof( float ),
                             cudaMemcpyHostToDevice ) );
        if( with_sigma )
        {
            KP_CUDA( cudaMemset( d_sigma, 0, n_cells * sizeof( float2 ) ) );
            KP_CUDA( cudaMemset( d_ext, 0, n_cells * sizeof( float ) ) );
        }
        KP_CUDA( cudaMemset( d_status, 0, 4 * sizeof( unsigned ) ) );
    }
    catch( ... )
    {
        release(  );
        throw;
    }
    device   = dev;
    uploaded = true;
}

void kp_mesh::release(  )
{
    cudaFree( d_nb );     d_nb     = nullptr;
    cudaFree( d_meta );   d_meta   = nullptr;
    cudaFree( d_geo_d );  d_geo_d  = nullptr;
    cudaFree( d_geo_f );  d_geo_f  = nullptr;
    cudaFree( d_sigma );  d_sigma  = nullptr;
    cudaFree( d_ext );    d_ext    = nullptr;
    cudaFree( d_lookup ); d_lookup = nullptr;
    cudaFree( d_status ); d_status = nullptr;
    cudaFree( d_work );   d_work   = nullptr;
    cudaFree( d_pq );     d_pq     = nullptr; pq_cap = 0;
    cudaFree( d_sort_cnt );  d_sort_cnt  = nullptr;
    cudaFree( d_sort_off );  d_sort_off  = nullptr;
    cudaFree( d_sort_perm ); d_sort_perm = nullptr;
    cudaFree( d_sort_tmp );  d_sort_tmp  = nullptr;
    sort_cells = sort_perm = sort_tmp_bytes = 0;
    cudaFree( d_adj );    d_adj    = nullptr; adj_bytes = 0; tape_id = 0;
    cudaFree( d_rf_f );   d_rf_f   = nullptr;
    cudaFree( d_rf_d );   d_rf_d   = nullptr;
    cudaFree( d_vol_f );  d_vol_f  = nullptr;
    cudaFree( d_vol_d );  d_vol_d  = nullptr;
    uploaded = false;
}

extern "C" {

static kp::mesh_desc_t desc_from_c( const kp_mesh_desc_t * desc )
{
    require( desc->n_refine >= 0 && ( desc->n_refine == 0 || desc->refine ), "bad refine list" );
    kp::mesh_desc_t d {  };
    for( int a = 0; a < 3; ++ a )
    {
        d.x_min[ a ] = desc->x_min[ a ];
        d.x_max[ a ] = desc->x_max[ a ];
        d.n_cell_global[ a ] = desc->n_cell_global[ a ];
        d.n_cell_block [ a ] = desc->n_cell_block [ a ];
        d.periodic[ a ] = desc->periodic[ a ] != 0;
    }
    for( int r = 0; r < desc->n_refine; ++ r )
    {
        kp::refine_box_t b {  };
        b.level = desc->refine[ r ].level;
        for( int a = 0; a < 3; ++ a )
        {
            b.x_min[ a ] = desc->refine[ r ].x_min[ a ];
            b.x_max[ a ] = desc->refine[ r ].x_max[ a ];
        }
        d.refine.push_back( b );
    }
    return d;
}

int kp_mesh_create( const kp_mesh_desc_t * desc, kp_mesh_t ** mesh )
{
    return guarded( "kp_mesh_create", [ & ]
    {
        require( desc != nullptr && mesh != nullptr, "null argument" );
        auto m = std::make_unique< kp_mesh >(  );
        m->tree = std::make_unique< kp::block_tree_t >( desc_from_c( desc ) );
        * mesh = m.release(  );
    } );
}

int kp_mesh_create_sph( const kp_mesh_desc_t * desc, double r_ratio, kp_mesh_t ** mesh )
{
    return guarded( "kp_mesh_create_sph", [ & ]
    {
        require( desc != nullptr && mesh != nullptr, "null argument" );
        kp::mesh_desc_t d = desc_from_c( desc );
        d.coord = 1;
        d.r_ratio = r_ratio;
        auto m = std::make_unique< kp_mesh >(  );
        m->tree = std::make_unique< kp::block_tree_t >( d );
        * mesh = m.release(  );
    } );
}

int kp_mesh_create_sph_ini( const char * path, kp_mesh_t ** mesh )
{
    return guarded( "kp_mesh_create_sph_ini", [ & ]
    {
        require( path != nullptr && mesh != nullptr, "null argument" );
        kp::ini_t ini;
        require( ini.read_file( path ), "cannot read INI file", KP_ERR_CONFIG );
        kp::mesh_desc_t d = kp::mesh_desc_from_ini( ini );
        d.coord = 1;
        d.r_ratio = ini.get_or< double >( "mesh", "r_ratio", 1.0 );   // cyl_t::read
        auto m = std::make_unique< kp_mesh >(  );
        m->tree = std::make_unique< kp::block_tree_t >( d );
        * mesh = m.release(  );
    } );
}

int kp_mesh_geometry_sph( const kp_mesh_t * mesh, int precision, double * r_faces, double * vol )
{
    return guarded( "kp_mesh_geometry_sph", [ & ]
    {
        require( mesh && r_faces && vol, "null argument" );
        require( precision == 4 || precision == 8, "precision must be 4 or 8" );
        const auto & t = mesh->tree->tables(  );
        require( t.coord == 1, "not a spherical mesh", KP_ERR_CONFIG );
        const int n0 = t.nc[ 0 ];
        for( int b = 0; b < t.n_blocks; ++ b )
            for( int i = 0; i <= n0; ++ i )
            {
                const size_t k = ( size_t ) b * ( n0 + 3 ) + i + 1;
                r_faces[ ( size_t ) b * ( n0 + 1 ) + i ] = precision == 4 ? t.rf_f[ k ] : t.rf_d[ k ];
            }
        for( size_t k = 0; k < t.vol_d.size(  ); ++ k )
            vol[ k ] = precision == 4 ? t.vol_f[ k ] : t.vol_d[ k ];
    } );
}

int kp_mesh_create_ini( const char * path, kp_mesh_t ** mesh )
{
    return guarded( "kp_mesh_create_ini", [ & ]
    {
        require( path != nullptr && mesh != nullptr, "null argument" );
        kp::ini_t ini;
        require( ini.read_file( path ), "cannot read INI file", KP_ERR_CONFIG );
        auto m = std::make_unique< kp_mesh >(  );
        m->tree = std::make_unique< kp::block_tree_t >( kp::mesh_desc_from_ini( ini ) );
        * mesh = m.release(  );
    } );
}

int kp_mesh_destroy( kp_mesh_t * mesh )
{
    return guarded( "kp_mesh_destroy", [ & ]
    {
        if( ! mesh ) return;
        if( mesh->uploaded )
        {
            int cur = 0;
            cudaGetDevice( & cur );
            cudaSetDevice( mesh->device );
            mesh->release(  );
            cudaSetDevice( cur );
        }
        delete mesh;
    } );
}

int kp_mesh_info( const kp_mesh_t * mesh, kp_mesh_info_t * info )
{
    return guarded( "kp_mesh_info", [ & ]
    {
        require( mesh && info, "null argument" );
        const auto & t = mesh->tree->tables(  );
        const auto & d = mesh->tree->desc(  );
        info->n_blocks = t.n_blocks;
        for( int a = 0; a < 3; ++ a )
        {
            info->n_cell_block[ a ] = t.nc[ a ];
            info->periodic[ a ] = t.periodic[ a ];
            info->x_min[ a ] = d.x_min[ a ];
            info->x_max[ a ] = d.x_max[ a ];
        }
        info->cells_per_block = t.cells_per_block;
        info->max_level = t.max_level;
        info->n_cells = ( long long ) t.n_blocks * t.cells_per_block;
    } );
}

int kp_mesh_blocks( const kp_mesh_t * mesh, int * level, int * reg3 )
{
    return guarded( "kp_mesh_blocks", [ & ]
    {
        require( mesh && level && reg3, "null argument" );
        const auto & t = mesh->tree->tables(  );
        std::copy( t.level.begin(  ), t.level.end(  ), level );
        std::copy( t.reg.begin(  ), t.reg.end(  ), reg3 );
    } );
}

int kp_mesh_geometry( const kp_mesh_t * mesh, int precision, double * xf0,
                      double * dx0, double * vol0, int * phybnd )
{
    return guarded( "kp_mesh_geometry", [ & ]
    {
        require( mesh && xf0 && dx0 && vol0 && phybnd, "null argument" );
        require( precision == 4 || precision == 8, "precision must be 4 or 8" );
        const auto & t = mesh->tree->tables(  );
        for( int b = 0; b < t.n_blocks; ++ b )
        {
            for( int a = 0; a < 3; ++ a )
            {
                xf0[ 3 * b + a ] = precision == 4 ? t.xf0_f[ 3 * b + a ] : t.xf0_d[ 3 * b + a ];
                dx0[ 3 * b + a ] = precision == 4 ? t.dx0_f[ 3 * b + a ] : t.dx0_d[ 3 * b + a ];
            }
            vol0[ b ] = precision == 4 ? t.vol0_f[ b ] : t.vol0_d[ b ];
            for( int f = 0; f < 6; ++ f )
                phybnd[ 6 * b + f ] = ( t.phybnd[ b ] >> f ) & 1;
        }
    } );
}

int kp_mesh_neighbors( const kp_mesh_t * mesh, int * nb_id, int * nb_shift,
                       int * d_lvl )
{
    return guarded( "kp_mesh_neighbors", [ & ]
    {
        require( mesh && nb_id && nb_shift && d_lvl, "null argument" );
        const auto & t = mesh->tree->tables(  );
        for( size_t k = 0; k < t.nb_id.size(  ); ++ k )
        {
            nb_id[ k ] = t.nb_id[ k ];
            nb_shift[ 2 * k ]     = t.nb_shift[ k ] & 1;
            nb_shift[ 2 * k + 1 ] = ( t.nb_shift[ k ] >> 1 ) & 1;
        }
        for( size_t k = 0; k < t.d_lvl.size(  ); ++ k )
            d_lvl[ k ] = t.d_lvl[ k ];
    } );
}

int kp_mesh_locate( const kp_mesh_t * mesh, long long n, const double * x,
                    int * ib, int * cell3 )
{
    return guarded( "kp_mesh_locate", [ & ]
    {
        require( mesh && ( n == 0 || ( x && ib && cell3 ) ), "null argument" );
        for( long long p = 0; p < n; ++ p )
            if( ! mesh->tree->locate( x + 3 * p, ib[ p ], cell3 + 3 * p ) )
            {
                ib[ p ] = -1;
                cell3[ 3 * p ] = cell3[ 3 * p + 1 ] = cell3[ 3 * p + 2 ] = -1;
            }
    } );
}

int kp_mesh_upload( kp_mesh_t * mesh )
{
    return guarded( "kp_mesh_upload", [ & ]
    {
        require( mesh != nullptr, "null mesh" );
        mesh->upload(  );
    } );
}

int kp_mesh_set_sigma( kp_mesh_t * mesh, const float * src, long long n_values,
                       int on_device, void * stream )
{
    return guarded( "kp_mesh_set_sigma", [ & ]
    {
        require( mesh && src, "null argument" );
        const auto & t = mesh->tree->tables(  );
        const long long n_cells = ( long long ) t.n_blocks * t.cells_per_block;
        require( n_values == 2 * n_cells, "sigma needs 2*n_cells values" );
        mesh->upload(  );
        mesh->tape_id = 0;                  // new coefficients: a taped solve is stale
        KP_CUDA( cudaMemcpyAsync( mesh->d_sigma, src, n_values * sizeof( float ),
                                  on_device ? cudaMemcpyDeviceToDevice
                                            : cudaMemcpyHostToDevice,
                                  ( cudaStream_t ) stream ) );
        if( ! on_device )
            KP_CUDA( cudaStreamSynchronize( ( cudaStream_t ) stream ) );
    } );
}

int kp_mesh_sigma_ptr( kp_mesh_t * mesh, float ** sigma )
{
    return guarded( "kp_mesh_sigma_ptr", [ & ]
    {
        require( mesh && sigma, "null argument" );
        mesh->upload(  );
        mesh->tape_id = 0;                  // the caller may write new coefficients
        * sigma = reinterpret_cast< float * >( mesh->d_sigma );
    } );
}

int kp_mesh_status( kp_mesh_t * mesh, void * stream, unsigned * flags )
{
    return guarded( "kp_mesh_status", [ & ]
    {
        require( mesh && flags, "null argument" );
        * flags = 0;
        if( ! mesh->uploaded ) return;
        unsigned h[ 4 ];
        KP_CUDA( cudaMemcpyAsync( h, mesh->d_status, sizeof( h ),
                                  cudaMemcpyDeviceToHost, ( cudaStream_t ) stream ) );
        KP_CUDA( cudaStreamSynchronize( ( cudaStream_t ) stream ) );
        * flags = h[ 0 ];
        KP_CUDA( cudaMemsetAsync( mesh->d_status, 0, sizeof( h ),
                                  ( cudaStream_t ) stream ) );
    } );
}

}   // extern "C"
