// kratos_b200 host layer: the problem-generator-facing types of Kratos
// (src/types.h of the reference: float_t / float2_t, 3-vectors idx_t /
// coord_t).  The device step always keeps its state in FP64, so both
// float types are double here.
#pragma once

#include <cmath>
#include <cstddef>

namespace type
{
typedef double float_t;
typedef double float2_t;
typedef int    int_t;

template< class T >
struct v3_base_t
{
    T x[ 3 ];
    v3_base_t(  ) : x{ T( 0 ), T( 0 ), T( 0 ) } {}
    v3_base_t( const T & t ) : x{ t, t, t } {}
    v3_base_t( const T & a, const T & b, const T & c ) : x{ a, b, c } {}
    static constexpr int size(  ) { return 3; }
    T & operator[]( int i ) { return x[ i ]; }
    const T & operator[]( int i ) const { return x[ i ]; }
    bool operator==( const v3_base_t & o ) const
    {   return x[ 0 ] == o.x[ 0 ] && x[ 1 ] == o.x[ 1 ] && x[ 2 ] == o.x[ 2 ]; }
    bool operator!=( const v3_base_t & o ) const { return ! ( * this == o ); }
    T prod(  ) const { return x[ 0 ] * x[ 1 ] * x[ 2 ]; }
    static v3_base_t null(  ) { return v3_base_t( T( 0 ) ); }
};

typedef v3_base_t< int >      idx_t;
typedef v3_base_t< float_t >  coord_t;
typedef v3_base_t< float2_t > coord2_t;
}   // namespace type
