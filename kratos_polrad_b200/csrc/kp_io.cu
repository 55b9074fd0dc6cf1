// C ABI of the binary container (host code; see host/bio.h for the format).
#include "kp_common.cuh"
#include "host/bio.h"

#include <vector>

struct kp_bio
{
    kp::bio::reader_t r;
    explicit kp_bio( const char * path ) : r( path ) {  }
};

int kp_bio_write( const char * path, int n_entries, const kp_bio_entry_t * entries )
{
    return kp::guarded( "kp_bio_write", [ & ]
    {
        kp::require( path != nullptr && n_entries >= 0 && ( n_entries == 0 || entries ),
                     "bad arguments" );
        std::vector< std::pair< std::string, kp::bio::view_t > > v;
        v.reserve( n_entries );
        for( int i = 0; i < n_entries; ++ i )
        {
            kp::require( entries[ i ].tag != nullptr, "entry without a tag" );
            v.emplace_back( entries[ i ].tag, kp::bio::view_t { entries[ i ].data,
                                                                 entries[ i ].count,
                                                                 entries[ i ].unit_size } );
        }
        try { kp::bio::write_file( path, v ); }
        catch( const std::runtime_error & e ) { throw kp::error_t( KP_ERR_ARG, e.what(  ) ); }
    } );
}

int kp_bio_open( const char * path, kp_bio_t ** file )
{
    return kp::guarded( "kp_bio_open", [ & ]
    {
        kp::require( path != nullptr && file != nullptr, "bad arguments" );
        * file = nullptr;
        try { * file = new kp_bio( path ); }
        catch( const std::runtime_error & e ) { throw kp::error_t( KP_ERR_ARG, e.what(  ) ); }
    } );
}

int kp_bio_close( kp_bio_t * file )
{
    return kp::guarded( "kp_bio_close", [ & ] { delete file; } );
}

int kp_bio_n_entries( const kp_bio_t * file, int * n )
{
    return kp::guarded( "kp_bio_n_entries", [ & ]
    {
        kp::require( file && n, "bad arguments" );
        * n = ( int ) file->r.entries(  ).size(  );
    } );
}

int kp_bio_entry( const kp_bio_t * file, int i, char * tag, size_t tag_cap,
                  unsigned long long * size, int * unit_size )
{
    return kp::guarded( "kp_bio_entry", [ & ]
    {
        kp::require( file != nullptr, "bad arguments" );
        const auto & e = file->r.entries(  );
        kp::require( i >= 0 && i < ( int ) e.size(  ), "entry index out of range" );
        if( tag )
        {
            kp::require( tag_cap > e[ i ].first.size(  ), "tag buffer too small", KP_ERR_CAPACITY );
            std::memcpy( tag, e[ i ].first.c_str(  ), e[ i ].first.size(  ) + 1 );
        }
        if( size ) * size = e[ i ].second.size;
        if( unit_size ) * unit_size = e[ i ].second.u_size;
    } );
}

int kp_bio_read( const kp_bio_t * file, const char * tag, void * dst, unsigned long long cap,
                 unsigned long long * size )
{
    return kp::guarded( "kp_bio_read", [ & ]
    {
        kp::require( file != nullptr && tag != nullptr, "bad arguments" );
        unsigned long long n = 0;
        try { n = file->r.read( tag, dst, cap ); }
        catch( const std::runtime_error & e ) { throw kp::error_t( KP_ERR_ARG, e.what(  ) ); }
        if( size ) * size = n;
    } );
}
