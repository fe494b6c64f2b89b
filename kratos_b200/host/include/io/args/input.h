// Parameter files: the `[section]` / `key = value` format of Kratos
// (src/io/args/input.h:37-197, input.cpp:70-230 of the reference).  Lines are
// cut at '#', trimmed; a line starting with '[' opens a section; later files
// (and later lines) override earlier keys.  A snapshot file given instead of a
// text file contributes its stored `input_args` map (restart).  Values are
// read with stream extraction: numbers, bools as 0/1, 3-vectors as three
// numbers, sequences as whitespace-separated lists.
#pragma once

#include <cctype>
#include <fstream>
#include <iostream>
#include <map>
#include <memory>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../../types.h"

namespace comm { struct base_t; }

class input
{
    std::map< std::string, std::string > items_;
    std::set< std::string > prefixes_;
    std::vector< std::string > files_;
    std::shared_ptr< comm::base_t > p_com_;

    static std::string trim( const std::string & s )
    {
        size_t a = 0, b = s.size(  );
        while( a < b && std::isspace( ( unsigned char ) s[ a ] ) ) ++ a;
        while( b > a && std::isspace( ( unsigned char ) s[ b - 1 ] ) ) -- b;
        return s.substr( a, b - a );
    }
    static std::string key( const std::string & pre, const std::string & k )
    {
        return ( pre.empty(  ) ? "" : pre + "|" ) + k;
    }

    template< class T > static void assign( std::stringstream & ss, T & t ) { ss >> t; }
    static void assign( std::stringstream & ss, std::string & t ) { ss >> t; }
    template< class T > static void assign( std::stringstream & ss, type::v3_base_t< T > & t )
    {   for( int a = 0; a < 3; ++ a ) ss >> t[ a ]; }
    template< class T > static void assign( std::stringstream & ss, std::vector< T > & t )
    {
        t.clear(  );
        T v;
        while( ss >> v ) t.push_back( v );
    }

public:
    input(  ) {}
    explicit input( const std::string & file ) { set_file( file ); read(  ); }

    void set_comm( std::shared_ptr< comm::base_t > p ) { p_com_ = p; }
    void set_file( const std::string & file, bool = true ) { files_.push_back( file ); }

    // Parse the last file given to set_file (text, or a snapshot's input_args).
    bool read(  );
    bool read_text( std::istream & in );

    void set( const std::string & pre, const std::string & k, const std::string & v )
    {
        items_[ key( pre, k ) ] = v;
        if( ! pre.empty(  ) ) prefixes_.insert( pre );
    }
    bool found( const std::string & pre, const std::string & k ) const
    {
        return items_.count( key( pre, k ) ) > 0;
    }
    template< class T >
    bool operator(  )( const std::string & pre, const std::string & k, T & res ) const
    {
        const auto it = items_.find( key( pre, k ) );
        if( it == items_.end(  ) ) return false;
        std::stringstream ss( it->second );
        assign( ss, res );
        return true;
    }
    template< class T > T get( const std::string & pre, const std::string & k ) const
    {
        T res{};
        if( ! ( * this )( pre, k, res ) )
        {
            std::cerr << "Entry \"[" << pre << "]: " << k << "\" not found.\n";
            throw std::runtime_error( "input::get" );
        }
        return res;
    }
    template< class T, class D > T get( const std::string & pre, const std::string & k, const D & def ) const
    {
        T res = T( def );
        ( * this )( pre, k, res );
        return res;
    }
    const std::map< std::string, std::string > & get_item_map(  ) const { return items_; }
    const std::set< std::string > & get_prefixes(  ) const { return prefixes_; }
};
