#include "block_tree.h"
#include "ini.h"

#include <cmath>
#include <stdexcept>

namespace kp
{

////////////////////////////////////////////////////////////
// Configuration

mesh_desc_t mesh_desc_from_ini( const ini_t & ini )
{
    mesh_desc_t d {  };
    if( ! ini.get3( "mesh", "x_min", d.x_min ) ||
        ! ini.get3( "mesh", "x_max", d.x_max ) ||
        ! ini.get3( "mesh", "n_cell_global", d.n_cell_global ) )
        throw std::runtime_error( "[mesh] needs x_min, x_max, n_cell_global" );
    if( ! ini.get3( "mesh", "n_cell_block", d.n_cell_block ) )
        for( int a = 0; a < 3; ++ a )
            d.n_cell_block[ a ] = d.n_cell_global[ a ];
    // [boundary] kinds: one word per side; "per..." marks a periodic axis
    // (the later side of an axis decides, as meshgen.cpp:52-55 does).
    const auto kinds = ini.values( "boundary", "kinds" );
    for( int a = 0; a < 3; ++ a ) d.periodic[ a ] = false;
    for( size_t s = 0; s < kinds.size(  ) && s < 6; ++ s )
        d.periodic[ s / 2 ] = kinds[ s ].find( "per" ) != std::string::npos;
    for( const auto & sec : ini.sections(  ) )
    {
        if( sec.find( "refine_region" ) == std::string::npos )
            continue;
        refine_box_t r {  };
        r.level = ini.get_or< int >( sec, "level", 0 );
        double lo[ 3 ] = { 0, 0, 0 };
        ini.get3( sec, "loc", lo );
        ini.get3( sec, "x_min", lo );
        double hi[ 3 ] = { lo[ 0 ], lo[ 1 ], lo[ 2 ] };
        ini.get3( sec, "x_max", hi );
        for( int a = 0; a < 3; ++ a )
        {
            r.x_min[ a ] = lo[ a ];
            r.x_max[ a ] = hi[ a ];
        }
        d.refine.push_back( r );
    }
    return d;
}

////////////////////////////////////////////////////////////
// Tree construction

void block_tree_t::init_domain(  )
{
    const mesh_desc_t & desc = desc_;
    n_dim_ = 0;
    for( int a = 0; a < 3; ++ a )
        if( desc.n_cell_global[ a ] > 1 )
            n_dim_ = a + 1;
    if( n_dim_ != 3 )
        throw std::runtime_error( "only 3-D meshes are supported" );
    for( int a = 0; a < 3; ++ a )
    {
        const int ng = desc.n_cell_global[ a ], nb = desc.n_cell_block[ a ];
        if( ng <= 0 || nb <= 0 || ng % nb != 0 )
            throw std::runtime_error( "Mesh size indivisible by sub-mesh." );
        if( nb < 2 || nb % 2 != 0 )
            throw std::runtime_error( "cells per block must be even" );
        if( ! ( desc.x_max[ a ] > desc.x_min[ a ] ) )
            throw std::runtime_error( "x_max must exceed x_min" );
        lim_[ a ] = ng / nb;
    }
    // cyl_t::read (mesh/meshgen/cylindrical.h): geometric radial spacing
    ratio_ = 1.0; dr0_ = -1.0;
    if( desc.coord == 1 )
    {
        if( ! ( desc.x_min[ 0 ] > 0.0 ) )
            throw std::runtime_error( "spherical meshes need r_min > 0" );
        ratio_ = desc.r_ratio;
        const int n_r = desc.n_cell_global[ 0 ];
        if( ! ( std::fabs( ratio_ - 1 ) < 1e-6 ) )
        {
            if( ratio_ < 0 )
                ratio_ = std::pow( desc.x_max[ 0 ] / desc.x_min[ 0 ], 1. / n_r );
            dr0_  = desc.x_max[ 0 ] - desc.x_min[ 0 ];
            dr0_ /= ( std::pow( ratio_, n_r ) - 1 ) / ( ratio_ - 1 );
        }
    }
    else if( desc.coord != 0 )
        throw std::runtime_error( "unknown coordinate system" );
}

block_tree_t::block_tree_t( const mesh_desc_t & desc ) : desc_( desc )
{
    init_domain(  );
    // Static refinement: every block of every box is forced to the box's
    // level (meshgen.cpp:144-163); insert() keeps the 2:1 balance.
    for( const auto & r : desc.refine )
    {
        if( r.level <= 0 )
            continue;
        if( r.level > 20 )
            throw std::runtime_error( "refinement level too deep" );
        int lo[ 3 ], hi[ 3 ];
        for( int a = 0; a < 3; ++ a )
        {
            lo[ a ] = block_index( r.x_min[ a ], r.level, a );
            hi[ a ] = block_index( r.x_max[ a ], r.level, a );
            if( lo[ a ] < 0 || hi[ a ] < 0 )
                throw std::runtime_error( "Incorrect SMR region" );
        }
        for( int k = lo[ 2 ]; k <= hi[ 2 ]; ++ k )
            for( int j = lo[ 1 ]; j <= hi[ 1 ]; ++ j )
                for( int i = lo[ 0 ]; i <= hi[ 0 ]; ++ i )
                    insert( { r.level, { i, j, k } } );
    }
    for( int k = 0; k < lim_[ 2 ]; ++ k )
        for( int j = 0; j < lim_[ 1 ]; ++ j )
            for( int i = 0; i < lim_[ 0 ]; ++ i )
                nodes_[ { 0, { i, j, k } } ];
    build_tables(  );
}

block_tree_t::block_tree_t( const mesh_desc_t & desc, const std::vector< region_key_t > & keys )
    : desc_( desc )
{
    desc_.refine.clear(  );
    init_domain(  );
    for( const auto & k0 : keys )
    {
        if( k0.level < 0 || k0.level > 20 )
            throw std::runtime_error( "refinement level outside 0..20" );
        region_key_t k = k0;
        for( int a = 0; a < 3; ++ a )
            if( k.i[ a ] < 0 || k.i[ a ] >= blocks_at( k.level, a ) )
                throw std::runtime_error( "block index outside the domain" );
        if( k.level > 0 )
            insert( k );
    }
    for( int k = 0; k < lim_[ 2 ]; ++ k )
        for( int j = 0; j < lim_[ 1 ]; ++ j )
            for( int i = 0; i < lim_[ 0 ]; ++ i )
                nodes_[ { 0, { i, j, k } } ];
    build_tables(  );
}

int block_tree_t::blocks_at( int level, int a ) const
{
    return lim_[ a ] << level;
}

double block_tree_t::location( double x_logic, int a ) const
{
    if( a == 0 && ! radial_uniform(  ) )
    {   // cyl_t::location: geometric radial faces
        const double n_logic( x_logic * desc_.n_cell_global[ 0 ] );
        return desc_.x_min[ 0 ] + dr0_ / ( ratio_ - 1 ) * ( std::pow( ratio_, n_logic ) - 1 );
    }
    return desc_.x_min[ a ] + x_logic * ( desc_.x_max[ a ] - desc_.x_min[ a ] );
}

// Largest block index i at `level` whose lower face lies strictly below
// `loc` (0 if none); -1 outside the domain.  Same predicate and search as
// meshgen::base_t::search_blk_idx (meshgen.cpp:448-468).
int block_tree_t::block_index( double loc, int level, int a ) const
{
    if( loc > desc_.x_max[ a ] || loc < desc_.x_min[ a ] )
        return -1;
    const int    n  = blocks_at( level, a );
    const double nf = n;
    int lo = 0, hi = n;
    while( hi - lo > 1 )
    {
        const int m = ( lo + hi ) / 2;
        if( location( m / nf, a ) < loc ) lo = m;
        else                              hi = m;
    }
    return lo;
}

// Wraps periodic axes into range; false if the region lies outside.
bool block_tree_t::inside( region_key_t & k ) const
{
    for( int a = 0; a < 3; ++ a )
    {
        const int n = blocks_at( k.level, a );
        if( desc_.periodic[ a ] )
            k.i[ a ] = ( ( k.i[ a ] % n ) + n ) % n;
        else if( k.i[ a ] < 0 || k.i[ a ] >= n )
            return false;
    }
    return true;
}

static region_key_t parent_of( const region_key_t & k )
{
    region_key_t p = k;
    p.level -= 1;
    for( auto & v : p.i )
        v = v >= 0 ? v / 2 : -( ( 1 - v ) / 2 );    // floor division
    return p;
}

// Refining a block creates all its siblings and requires every block that
// touches its parent (faces, edges, corners) to exist at the parent's level
// (the 2:1 balance of tree_t::insert, tree.cpp:202-218).
void block_tree_t::insert( const region_key_t & k )
{
    if( nodes_.count( k ) )
        return;
    if( k.level > 0 )
    {
        const region_key_t p = parent_of( k );
        insert( p );
        nodes_[ p ].refined = true;
        for( int c = 0; c < 8; ++ c )
            nodes_[ { k.level, { 2 * p.i[ 0 ] + ( c & 1 ),
                                 2 * p.i[ 1 ] + ( ( c >> 1 ) & 1 ),
                                 2 * p.i[ 2 ] + ( ( c >> 2 ) & 1 ) } } ];
        for( int dz = -1; dz <= 1; ++ dz )
            for( int dy = -1; dy <= 1; ++ dy )
                for( int dx = -1; dx <= 1; ++ dx )
                {
                    if( dx == 0 && dy == 0 && dz == 0 )
                        continue;
                    region_key_t q { p.level, { p.i[ 0 ] + dx, p.i[ 1 ] + dy,
                                                p.i[ 2 ] + dz } };
                    if( inside( q ) )
                        insert( q );
                }
    }
    nodes_[ k ];
}

int block_tree_t::find( const region_key_t & k ) const
{
    auto it = nodes_.find( k );
    if( it == nodes_.end(  ) || it->second.refined )
        return -1;
    return it->second.id;
}

////////////////////////////////////////////////////////////
// Flat tables

void block_tree_t::build_tables(  )
{
    auto & t = tab_;
    int id = 0;
    for( auto & [ k, n ] : nodes_ )
        if( ! n.refined )
            n.id = id ++;
    t.n_blocks = id;
    t.n_dim    = n_dim_;
    for( int a = 0; a < 3; ++ a )
        t.nc[ a ] = desc_.n_cell_block[ a ];
    t.cells_per_block = t.nc[ 0 ] * t.nc[ 1 ] * t.nc[ 2 ];

    const int nb = t.n_blocks;
    t.level .assign( nb, 0 );
    t.reg   .assign( 3 * nb, 0 );
    t.xf0_d .assign( 3 * nb, 0 );  t.dx0_d .assign( 3 * nb, 0 );
    t.xf0_f .assign( 3 * nb, 0 );  t.dx0_f .assign( 3 * nb, 0 );
    t.vol0_d.assign( nb, 0 );      t.vol0_f.assign( nb, 0 );
    t.phybnd.assign( nb, 0 );
    t.nb_id .assign( 24 * nb, -1 );
    t.d_lvl .assign( 6 * nb, 0 );
    t.nb_shift.assign( 24 * nb, 0 );
    t.max_level = 0;

    for( const auto & [ k, n ] : nodes_ )
    {
        if( n.refined )
            continue;
        const int b = n.id;
        t.level[ b ] = k.level;
        t.max_level  = std::max( t.max_level, k.level );
        double vd = 1., vf = 1.;
        for( int a = 0; a < 3; ++ a )
        {
            t.reg[ 3 * b + a ] = k.i[ a ];
            // Face coordinate of logical cell offset c within the block,
            // evaluated in double as set_coord_axes does (meshgen.cpp:
            // 386-399); the FP32 copy rounds xf0 first and then takes the
            // spacing against the rounded origin.
            const double nl = blocks_at( k.level, a );
            const double l0 = location( ( k.i[ a ] + 0.0 / t.nc[ a ] ) / nl, a );
            const double l1 = location( ( k.i[ a ] + 1.0 / t.nc[ a ] ) / nl, a );
            t.xf0_d[ 3 * b + a ] = l0;
            t.dx0_d[ 3 * b + a ] = l1 - l0;
            const float x0f = ( float ) l0;
            t.xf0_f[ 3 * b + a ] = x0f;
            t.dx0_f[ 3 * b + a ] = ( float ) ( l1 - ( double ) x0f );
            vd *= t.dx0_d[ 3 * b + a ];
            vf *= ( double ) t.dx0_f[ 3 * b + a ];
            if( ! desc_.periodic[ a ] )
            {
                if( k.i[ a ] == 0 )
                    t.phybnd[ b ] |= 1u << ( 2 * a );
                if( k.i[ a ] == blocks_at( k.level, a ) - 1 )
                    t.phybnd[ b ] |= 1u << ( 2 * a + 1 );
            }
        }
        t.vol0_d[ b ] = vd;
        t.vol0_f[ b ] = ( float ) vf;

        // Face neighbours: finer (4 sub-faces), same level, or coarser.
        for( int a = 0; a < 3; ++ a )
        {
            const int ap0 = ( a + 1 ) % 3, ap1 = ( a + 2 ) % 3;
            for( int s = 0; s < 2; ++ s )
            {
                region_key_t q = k;
                q.i[ a ] += s ? 1 : -1;
                if( ! inside( q ) )
                    continue;
                auto it = nodes_.find( q );
                if( it != nodes_.end(  ) && ! it->second.refined )
                {
                    t.nb_id[ 24 * b + nb_slot( a, s, 0, 0 ) ] = it->second.id;
                }
                else if( it != nodes_.end(  ) )
                {
                    t.d_lvl[ 6 * b + 2 * a + s ] = 1;
                    for( int j0 = 0; j0 < 2; ++ j0 )
                        for( int j1 = 0; j1 < 2; ++ j1 )
                        {
                            region_key_t c { q.level + 1, { 0, 0, 0 } };
                            c.i[ a ]   = 2 * q.i[ a ]   + ( s ? 0 : 1 );
                            c.i[ ap0 ] = 2 * q.i[ ap0 ] + j0;
                            c.i[ ap1 ] = 2 * q.i[ ap1 ] + j1;
                            const int cid = find( c );
                            if( cid < 0 )
                                throw std::runtime_error( "2:1 balance violated" );
                            t.nb_id[ 24 * b + nb_slot( a, s, j0, j1 ) ] = cid;
                        }
                }
                else
                {
                    const int pid = find( parent_of( q ) );
                    if( pid < 0 )
                        throw std::runtime_error( "2:1 balance violated" );
                    const int sl = nb_slot( a, s, 0, 0 );
                    t.nb_id[ 24 * b + sl ]    = pid;
                    t.d_lvl[ 6 * b + 2 * a + s ] = -1;
                    t.nb_shift[ 24 * b + sl ] =
                        ( k.i[ ap0 ] & 1 ) | ( ( k.i[ ap1 ] & 1 ) << 1 );
                }
            }
        }
    }
    build_sph_tables(  );
    const int L = t.max_level;
    double n_lookup = 1.0;
    for( int a = 0; a < 3; ++ a )
        n_lookup *= std::ldexp( ( double ) lim_[ a ], L );
    if( n_lookup > ( double ) ( 1 << 28 ) )
        throw std::runtime_error( "finest-level lookup grid too large (more than 2^28 "
                                  "block positions): too many refinement levels" );
    for( int a = 0; a < 3; ++ a )
        t.lookup_n[ a ] = blocks_at( L, a );
    t.lookup.assign( ( size_t ) t.lookup_n[ 0 ] * t.lookup_n[ 1 ] * t.lookup_n[ 2 ], -1 );
    for( const auto & [ k, n ] : nodes_ )
    {
        if( n.refined )
            continue;
        const int f = 1 << ( L - k.level );
        for( int dz = 0; dz < f; ++ dz )
            for( int dy = 0; dy < f; ++ dy )
                for( int dx = 0; dx < f; ++ dx )
                {
                    const size_t i = k.i[ 0 ] * f + dx, j = k.i[ 1 ] * f + dy,
                                 l = k.i[ 2 ] * f + dz;
                    t.lookup[ ( l * t.lookup_n[ 1 ] + j ) * t.lookup_n[ 0 ] + i ] = n.id;
                }
    }
    for( int a = 0; a < 3; ++ a )
    {
        t.periodic[ a ]  = desc_.periodic[ a ];
        t.xlim_d[ 0 ][ a ] = desc_.x_min[ a ];
        t.xlim_d[ 1 ][ a ] = desc_.x_max[ a ];
        t.xlim_f[ 0 ][ a ] = ( float ) desc_.x_min[ a ];
        t.xlim_f[ 1 ][ a ] = ( float ) desc_.x_max[ a ];
        t.l_box_d[ a ]   = desc_.x_max[ a ] - desc_.x_min[ a ];
        t.l_box_f[ a ]   = ( float ) t.l_box_d[ a ];
    }
}

// Spherical tables: sph_t::set_coord_axes (radial faces loc_f(i) in double,
// stored as float_t when the spacing is not uniform) and sph_t::volume
// (mesh/meshgen/spherical.h), whose face coordinates come from geo_t::x_fc
// in float_t (geometry.h) and whose arithmetic is double.
namespace
{
template< class F >
struct sph_geo_t
{
    const F * xf0; const F * dx0; const F * rf;
    bool r_table;
    F x_fc( int a, int i ) const
    {
        if( a == 0 && r_table ) return rf[ i + 1 ];      // one ghost face below
        return xf0[ a ] + ( F ) i * dx0[ a ];
    }
};

template< class F >
double sph_volume( const sph_geo_t< F > & g, int c0, int c1, int c2 )
{
    const F r_l  = g.x_fc( 0, c0 ), r_r = g.x_fc( 0, c0 + 1 );
    const F th_l = g.x_fc( 1, c1 ), th_r = g.x_fc( 1, c1 + 1 );
    const F d_phi = g.x_fc( 2, c2 + 1 ) - g.x_fc( 2, c2 );
    return ( std::pow( ( double ) r_r, 3. ) - std::pow( ( double ) r_l, 3. ) ) / 3.
         * std::fabs( std::cos( ( double ) th_l ) - std::cos( ( double ) th_r ) ) * d_phi;
}
}   // namespace

void block_tree_t::build_sph_tables(  )
{
    auto & t = tab_;
    t.coord = desc_.coord;
    t.rf_d.clear(  ); t.rf_f.clear(  ); t.vol_d.clear(  ); t.vol_f.clear(  );
    if( desc_.coord != 1 )
        return;
    const int nb = t.n_blocks, n0 = t.nc[ 0 ], cpb = t.cells_per_block;
    const bool table = ! radial_uniform(  );
    const int nf = n0 + 3;                       // faces -1 .. n0 + 1 (one ghost each side)
    t.rf_d.assign( ( size_t ) nb * nf, 0. );
    t.rf_f.assign( ( size_t ) nb * nf, 0.f );
    t.vol_d.assign( ( size_t ) nb * cpb, 0. );
    t.vol_f.assign( ( size_t ) nb * cpb, 0.f );
    for( int b = 0; b < nb; ++ b )
    {
        const double nl = blocks_at( t.level[ b ], 0 );
        for( int i = -1; i <= n0 + 1; ++ i )
        {
            const double l = location( ( t.reg[ 3 * b ] + ( double ) i / n0 ) / nl, 0 );
            t.rf_d[ ( size_t ) b * nf + i + 1 ] = l;
            t.rf_f[ ( size_t ) b * nf + i + 1 ] = ( float ) l;
        }
        if( table )
        {
            t.dx0_d[ 3 * b ] = -1.0;
            t.dx0_f[ 3 * b ] = -1.0f;
        }
        t.vol0_d[ b ] = -1.0;
        t.vol0_f[ b ] = -1.0f;
        const sph_geo_t< double > gd { & t.xf0_d[ 3 * b ], & t.dx0_d[ 3 * b ],
                                       & t.rf_d[ ( size_t ) b * nf ], table };
        const sph_geo_t< float >  gf { & t.xf0_f[ 3 * b ], & t.dx0_f[ 3 * b ],
                                       & t.rf_f[ ( size_t ) b * nf ], table };
        size_t k = ( size_t ) b * cpb;
        for( int c2 = 0; c2 < t.nc[ 2 ]; ++ c2 )
            for( int c1 = 0; c1 < t.nc[ 1 ]; ++ c1 )
                for( int c0 = 0; c0 < n0; ++ c0, ++ k )
                {
                    t.vol_d[ k ] = sph_volume( gd, c0, c1, c2 );
                    t.vol_f[ k ] = ( float ) sph_volume( gf, c0, c1, c2 );
                }
    }
}

bool block_tree_t::locate( const double x[ 3 ], int & ib, int cell[ 3 ] ) const
{
    // logical coordinate in [0, 1] (the inverse of location)
    auto logic = [ & ]( int a ) -> double
    {
        if( a == 0 && ! radial_uniform(  ) )
            return std::log1p( ( x[ 0 ] - desc_.x_min[ 0 ] ) * ( ratio_ - 1 ) / dr0_ )
                 / std::log( ratio_ ) / desc_.n_cell_global[ 0 ];
        return ( x[ a ] - desc_.x_min[ a ] ) / ( desc_.x_max[ a ] - desc_.x_min[ a ] );
    };
    region_key_t k { 0, { 0, 0, 0 } };
    for( int a = 0; a < 3; ++ a )
    {
        if( ! ( x[ a ] >= desc_.x_min[ a ] && x[ a ] <= desc_.x_max[ a ] ) )
            return false;
        k.i[ a ] = std::max( 0, std::min( lim_[ a ] - 1,
                                          ( int ) std::floor( logic( a ) * lim_[ a ] ) ) );
    }
    for( ;; )
    {
        auto it = nodes_.find( k );
        if( it == nodes_.end(  ) )
            return false;
        if( ! it->second.refined )
        {
            ib = it->second.id;
            break;
        }
        region_key_t c { k.level + 1, { 0, 0, 0 } };
        for( int a = 0; a < 3; ++ a )
        {
            const double n  = blocks_at( c.level, a );
            int i = ( int ) std::floor( logic( a ) * n );
            i = std::max( 2 * k.i[ a ], std::min( 2 * k.i[ a ] + 1, i ) );
            c.i[ a ] = i;
        }
        k = c;
    }
    const auto & t = tab_;
    for( int a = 0; a < 3; ++ a )
    {
        int i;
        if( a == 0 && t.coord == 1 && t.dx0_d[ 3 * ib ] < 0 )
        {   // radial face table: last face not above x
            const double * f = & t.rf_d[ ( size_t ) ib * ( t.nc[ 0 ] + 3 ) + 1 ];
            i = 0;
            while( i + 1 < t.nc[ 0 ] && f[ i + 1 ] <= x[ 0 ] ) ++ i;
        }
        else
            i = ( int ) std::floor( ( x[ a ] - t.xf0_d[ 3 * ib + a ] ) / t.dx0_d[ 3 * ib + a ] );
        cell[ a ] = std::max( 0, std::min( t.nc[ a ] - 1, i ) );
    }
    return true;
}

}   // namespace kp
