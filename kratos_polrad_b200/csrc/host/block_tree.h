// Block-structured AMR tree and the flat tables the transport kernels read.
//
// Replaces, for the transport path, the reference's mesh generator and tree
// (mesh/meshgen/meshgen.cpp:13-163,286-351,378-400; mesh/tree/tree.cpp:
// 112-230) and the proxy table that particle::block_map_t uploads
// (modules/particle/types/proxy.h:22-62, types/block_map.h:53-103).
// Refinement is static: boxes of [refine_region*] sections, each forcing its
// blocks to a level, with 2:1 balance across faces, edges and corners.
#pragma once

#include <array>
#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace kp
{

struct refine_box_t
{
    int    level;
    double x_min[ 3 ];
    double x_max[ 3 ];
};

struct mesh_desc_t
{
    double x_min[ 3 ];
    double x_max[ 3 ];
    int    n_cell_global[ 3 ];
    int    n_cell_block [ 3 ];
    bool   periodic     [ 3 ];
    std::vector< refine_box_t > refine;
    // Coordinates: 0 Cartesian (meshgen::base_t); 1 spherical-polar
    // (r, theta, phi) of meshgen::sph_t, whose radius follows cyl_t's
    // geometric spacing ([mesh] r_ratio: 1 uniform, < 0 from the radii).
    int    coord   = 0;
    double r_ratio = 1.0;
};

// Region key: (level, logical block index) with the reference's lexical
// order (level first, then axis 0, 1, 2; geometry/region.h:318-334).
struct region_key_t
{
    int level;
    std::array< int, 3 > i;
    bool operator < ( const region_key_t & o ) const
    {
        if( level != o.level ) return level < o.level;
        return i < o.i;
    }
    bool operator == ( const region_key_t & o ) const
    {
        return level == o.level && i == o.i;
    }
};

// One face-neighbour slot per [axis][side][j0][j1] (j0 along axis+1,
// j1 along axis+2), the layout of proxy_base_t::neighbors (proxy.h:13-19).
inline int nb_slot( int a, int s, int j0, int j1 )
{
    return ( ( a * 2 + s ) * 2 + j0 ) * 2 + j1;
}

struct block_tables_t
{
    int n_blocks = 0;
    int n_dim    = 3;
    int nc[ 3 ]  = { 0, 0, 0 };            // cells per block and axis
    int cells_per_block = 0;
    int max_level = 0;

    std::vector< int >      level;         // [nb]
    std::vector< int >      reg;           // [nb][3]
    // Geometry: face origin and spacing.  The *_f arrays hold the values
    // the reference computes with float_t = float, *_d with double.
    std::vector< double >   xf0_d, dx0_d, vol0_d;   // [nb][3], [nb][3], [nb]
    std::vector< float  >   xf0_f, dx0_f, vol0_f;
    std::vector< uint8_t >  phybnd;        // [nb] bit (2a+s)
    // Spherical meshes: radial faces [nb][nc0+3] (faces -1..nc0+1: one ghost
    // each side, as geo_t keeps them; when the radial spacing
    // is not uniform, dx0[0] is then -1) and cell volumes [n_cells], as
    // sph_t::set_coord_axes and sph_t::volume give them (FP64 and FP32).
    int coord = 0;
    std::vector< double >   rf_d;  std::vector< float > rf_f;
    std::vector< double >   vol_d; std::vector< float > vol_f;
    std::vector< int >      nb_id;         // [nb][24]
    std::vector< int8_t >   d_lvl;         // [nb][6]
    std::vector< uint8_t >  nb_shift;      // [nb][24] bit0: shift[0], bit1: shift[1]

    // Finest-level lookup grid: leaf block id of every finest-level block
    // position, x fastest (device-side point location of plane sources).
    int lookup_n[ 3 ] = { 0, 0, 0 };
    std::vector< int >      lookup;

    double xlim_d[ 2 ][ 3 ];
    double l_box_d[ 3 ];
    float  xlim_f[ 2 ][ 3 ];
    float  l_box_f[ 3 ];
    bool   periodic[ 3 ];
};

class block_tree_t
{
public:
    explicit block_tree_t( const mesh_desc_t & desc );
    // Tree whose leaves include `keys` (each inserted with the 2:1 closure,
    // as a refine box covering one block at its level would insert it);
    // desc.refine is not used.  The runtime refinement path.
    block_tree_t( const mesh_desc_t & desc, const std::vector< region_key_t > & keys );

    const block_tables_t & tables(  ) const { return tab_; }
    const mesh_desc_t    & desc  (  ) const { return desc_; }

    // Block id of a region key, -1 if it is not a leaf.
    int find( const region_key_t & k ) const;

    // Host-side point location: block id and cell index holding x
    // (half-open cells, the upper domain face belongs to the last cell).
    // Returns false if x lies outside the domain.
    bool locate( const double x[ 3 ], int & ib, int cell[ 3 ] ) const;

private:
    struct node_t { bool refined = false; int id = -1; };

    void   init_domain(  );                          // checks desc_, sets lim_
    void   insert( const region_key_t & k );
    bool   inside( region_key_t & k ) const;         // wraps periodic axes
    int    blocks_at( int level, int a ) const;      // blocks per axis
    double location( double x_logic, int a ) const;
    int    block_index( double loc, int level, int a ) const;
    void   build_tables(  );
    void   build_sph_tables(  );
    bool   radial_uniform(  ) const { return dr0_ <= 0.0; }

    mesh_desc_t                        desc_;
    int                                n_dim_ = 3;
    double                             ratio_ = 1.0, dr0_ = -1.0;   // cyl_t::read
    int                                lim_[ 3 ];    // root blocks per axis
    std::map< region_key_t, node_t >   nodes_;
    block_tables_t                     tab_;
};

// Reads [mesh], [boundary] and [refine_region*] with the reference's key
// names (meshgen.cpp:13-42,44-55,111-142).
mesh_desc_t mesh_desc_from_ini( const class ini_t & ini );

}   // namespace kp
