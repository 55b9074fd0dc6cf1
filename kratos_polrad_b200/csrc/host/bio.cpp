#include "bio.h"

#include <algorithm>
#include <cstring>
#include <fstream>
#include <stdexcept>

namespace kp::bio
{
namespace
{

static_assert( sizeof( std::size_t ) == 8, "the container stores 8-byte size_t" );

bool host_is_little(  )
{
    const std::uint16_t one = 1;
    unsigned char b;
    std::memcpy( & b, & one, 1 );
    return b == 1;
}

void put_u64( std::string & s, std::uint64_t v )
{
    s.append( reinterpret_cast< const char * >( & v ), 8 );
}

}   // namespace

void write_file( const std::string & path, const std::vector< std::pair< std::string, view_t > > & entries )
{
    if( ! host_is_little(  ) )
        throw std::runtime_error( "binary container: big-endian host" );
    std::map< std::string, view_t > m;
    for( const auto & e : entries )
    {
        if( e.second.u_size < 1 || e.second.u_size > 127 )
            throw std::runtime_error( "binary container: unit size of '" + e.first
                                      + "' outside 1..127" );
        if( e.second.count > 0 && e.second.data == nullptr )
            throw std::runtime_error( "binary container: null data for '" + e.first + "'" );
        if( e.second.count > UINT64_MAX / ( std::uint64_t ) e.second.u_size )
            throw std::runtime_error( "binary container: size of '" + e.first + "' overflows" );
        m[ e.first ] = e.second;
    }
    // serialized map: count, then per entry tag, size, unit size, offset
    std::string map_bytes;
    put_u64( map_bytes, m.size(  ) );
    std::uint64_t offset = 0;
    for( const auto & p : m )
    {
        const std::uint64_t size = p.second.count * ( std::uint64_t ) p.second.u_size;
        put_u64( map_bytes, p.first.size(  ) );
        map_bytes += p.first;
        put_u64( map_bytes, size );
        map_bytes.push_back( ( char ) p.second.u_size );
        put_u64( map_bytes, offset );
        offset += size;
    }
    std::ofstream f( path, std::ios::binary | std::ios::trunc );
    if( ! f )
        throw std::runtime_error( "Cannot open file " + path );
    const char first = ( char ) ( 1 | ( int ) sizeof( std::size_t ) );
    const std::uint64_t header_size = 1 + 8 + map_bytes.size(  );
    f.write( & first, 1 );
    f.write( reinterpret_cast< const char * >( & header_size ), 8 );
    f.write( map_bytes.data(  ), ( std::streamsize ) map_bytes.size(  ) );
    for( const auto & p : m )
        f.write( static_cast< const char * >( p.second.data ),
                 ( std::streamsize ) ( p.second.count * ( std::uint64_t ) p.second.u_size ) );
    if( ! f )
        throw std::runtime_error( "binary container: write failed on " + path );
}

reader_t::reader_t( const std::string & path ) : path_( path )
{
    std::ifstream f( path, std::ios::binary | std::ios::ate );
    if( ! f )
        throw std::runtime_error( "Cannot open file " + path );
    file_size_ = ( std::uint64_t ) f.tellg(  );
    f.seekg( 0 );
    std::vector< char > head( ( std::size_t ) std::min< std::uint64_t >( file_size_, 9 ) );
    f.read( head.data(  ), ( std::streamsize ) head.size(  ) );
    if( head.size(  ) < 9 )
        throw std::runtime_error( "binary container: file too short" );
    const int first = ( unsigned char ) head[ 0 ];
    if( ( first & ~1 ) != ( int ) sizeof( std::size_t ) )
        throw std::runtime_error( "Inconsistent size_t " );
    if( ( ( first & 1 ) != 0 ) != host_is_little(  ) )
        throw std::runtime_error( "Inconsistent endian " );
    std::memcpy( & header_size_, head.data(  ) + 1, 8 );
    if( header_size_ < 17 || header_size_ > file_size_ )
        throw std::runtime_error( "binary container: bad header size" );
    std::string h( ( std::size_t ) ( header_size_ - 9 ), '\0' );
    f.read( & h[ 0 ], ( std::streamsize ) h.size(  ) );
    std::size_t pos = 0;
    auto get = [ & ]( void * dst, std::size_t n )
    {
        if( pos + n > h.size(  ) )
            throw std::runtime_error( "binary container: truncated header" );
        std::memcpy( dst, h.data(  ) + pos, n );
        pos += n;
    };
    std::uint64_t n = 0;
    get( & n, 8 );
    if( n > h.size(  ) / 26 )
        throw std::runtime_error( "binary container: bad entry count" );
    const std::uint64_t bulk = file_size_ - header_size_;
    for( std::uint64_t i = 0; i < n; ++ i )
    {
        std::uint64_t len = 0;
        get( & len, 8 );
        if( len > h.size(  ) - pos )
            throw std::runtime_error( "binary container: bad tag length" );
        std::string tag( h.data(  ) + pos, ( std::size_t ) len );
        pos += ( std::size_t ) len;
        info_t in;
        char u = 0;
        get( & in.size, 8 );
        get( & u, 1 );
        get( & in.offset, 8 );
        in.u_size = ( unsigned char ) u;
        if( in.offset > bulk || in.size > bulk - in.offset )
            throw std::runtime_error( "binary container: entry '" + tag + "' beyond the file" );
        index_[ tag ] = entries_.size(  );
        entries_.emplace_back( std::move( tag ), in );
    }
}

const info_t & reader_t::info( const std::string & tag ) const
{
    const auto it = index_.find( tag );
    if( it == index_.end(  ) )
        throw std::runtime_error( "Read cannot find tag: " + tag );
    return entries_[ it->second ].second;
}

std::uint64_t reader_t::read( const std::string & tag, void * dst, std::uint64_t cap ) const
{
    const info_t & in = info( tag );
    if( in.size > cap )
        throw std::runtime_error( "binary container: buffer too small for '" + tag + "'" );
    if( in.size == 0 )
        return 0;
    if( dst == nullptr )
        throw std::runtime_error( "nullptr in binary r" );
    std::ifstream f( path_, std::ios::binary );
    if( ! f )
        throw std::runtime_error( "Cannot open file " + path_ );
    f.seekg( ( std::streamoff ) ( header_size_ + in.offset ) );
    f.read( static_cast< char * >( dst ), ( std::streamsize ) in.size );
    if( ! f )
        throw std::runtime_error( "binary container: read failed for '" + tag + "'" );
    return in.size;
}

}   // namespace kp::bio
