// INI configuration reader with the reference's syntax and key names.
//
// Follows io/args/input.cpp:72-108 (read_ascii): `[section]` headers,
// `key = value` lines, `#` starts a comment, later files override earlier
// ones (user/probgen.cpp:8-16), values are whitespace-separated lists.
// Keys are stored as "section|key" like input::key_expand (input.cpp).
#pragma once

#include <map>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace kp
{

class ini_t
{
public:
    // Parses `text` (file contents); returns false on a malformed section.
    bool parse( const std::string & text );
    bool read_file( const std::string & path );

    bool found( const std::string & sec, const std::string & key ) const;
    const std::set< std::string > & sections(  ) const { return secs_; }

    // Whitespace-separated values of one key; empty if absent.
    std::vector< std::string > values( const std::string & sec,
                                       const std::string & key ) const;

    template< class T >
    bool get( const std::string & sec, const std::string & key, T & out ) const
    {
        auto it = map_.find( sec + "|" + key );
        if( it == map_.end(  ) ) return false;
        std::stringstream ss( it->second );
        ss >> out;
        return ! ss.fail(  );
    }
    template< class T >
    T get_or( const std::string & sec, const std::string & key, T def ) const
    {
        T v;
        return get( sec, key, v ) ? v : def;
    }
    template< class T >
    bool get3( const std::string & sec, const std::string & key, T out[ 3 ] ) const
    {
        auto it = map_.find( sec + "|" + key );
        if( it == map_.end(  ) ) return false;
        std::stringstream ss( it->second );
        for( int a = 0; a < 3; ++ a ) ss >> out[ a ];
        return ! ss.fail(  );
    }
    template< class T >
    T require( const std::string & sec, const std::string & key ) const
    {
        T v;
        if( ! get( sec, key, v ) )
            throw std::runtime_error( "missing [" + sec + "] " + key );
        return v;
    }
    void set( const std::string & sec, const std::string & key,
              const std::string & val );
    // The keys as INI text: keys outside any section first, then one
    // [section] block per section in name order, keys in name order.
    std::string text(  ) const;

private:
    std::map< std::string, std::string > map_;
    std::set< std::string >              secs_;
};

}   // namespace kp
