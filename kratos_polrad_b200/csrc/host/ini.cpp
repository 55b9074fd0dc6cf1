#include "ini.h"

#include <fstream>

namespace kp
{

static std::string trim( const std::string & s )
{
    const char * ws = " \t\r\n";
    const auto b = s.find_first_not_of( ws );
    if( b == std::string::npos ) return "";
    const auto e = s.find_last_not_of( ws );
    return s.substr( b, e - b + 1 );
}

bool ini_t::parse( const std::string & text )
{
    std::istringstream in( text );
    std::string line, sec;
    while( std::getline( in, line ) )
    {
        line = trim( line.substr( 0, line.find( '#' ) ) );
        if( line.empty(  ) ) continue;
        if( line[ 0 ] == '[' )
        {
            const auto e = line.find( ']' );
            if( e == std::string::npos ) return false;
            sec = line.substr( 1, e - 1 );
            secs_.insert( sec );
            continue;
        }
        const auto eq = line.find( '=' );
        const std::string key = trim( line.substr( 0, eq ) );
        const std::string val = eq == std::string::npos ? ""
                              : trim( line.substr( eq + 1 ) );
        map_[ sec + "|" + key ] = val;
    }
    return true;
}

bool ini_t::read_file( const std::string & path )
{
    std::ifstream f( path );
    if( ! f ) return false;
    std::stringstream ss;
    ss << f.rdbuf(  );
    return parse( ss.str(  ) );
}

bool ini_t::found( const std::string & sec, const std::string & key ) const
{
    return map_.count( sec + "|" + key ) > 0;
}

std::vector< std::string > ini_t::values( const std::string & sec,
                                          const std::string & key ) const
{
    std::vector< std::string > out;
    auto it = map_.find( sec + "|" + key );
    if( it == map_.end(  ) ) return out;
    std::stringstream ss( it->second );
    for( std::string t; ss >> t; ) out.push_back( t );
    return out;
}

std::string ini_t::text(  ) const
{
    std::map< std::string, std::vector< std::pair< std::string, std::string > > > by_sec;
    for( const auto & kv : map_ )
    {
        const auto bar = kv.first.find( '|' );
        by_sec[ kv.first.substr( 0, bar ) ].emplace_back( kv.first.substr( bar + 1 ), kv.second );
    }
    for( const auto & s : secs_ )
        by_sec[ s ];                                // sections without keys
    std::ostringstream out;
    for( const auto & [ sec, keys ] : by_sec )
    {
        if( ! sec.empty(  ) )
            out << "[" << sec << "]\n";
        for( const auto & [ k, v ] : keys )
            out << k << " = " << v << "\n";
        out << "\n";
    }
    return out.str(  );
}

void ini_t::set( const std::string & sec, const std::string & key,
                 const std::string & val )
{
    map_[ sec + "|" + key ] = val;
    if( ! sec.empty(  ) ) secs_.insert( sec );
}

}   // namespace kp
