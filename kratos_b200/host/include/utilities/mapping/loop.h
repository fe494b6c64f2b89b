// utils::loop: iterate a 3-D index box, x fastest (utilities/mapping/loop.h
// of the reference: loop(i_max), loop(i_min, i_max, include_max)).
#pragma once

#include "../../types.h"

namespace utils
{
class loop_t
{
    type::idx_t lo_, hi_;         // half-open box [lo_, hi_)
public:
    loop_t( const type::idx_t & lo, const type::idx_t & hi ) : lo_( lo ), hi_( hi ) {}
    struct iterator
    {
        type::idx_t i, lo, hi;
        bool end;
        const type::idx_t & operator*(  ) const { return i; }
        iterator & operator++(  )
        {
            for( int a = 0; a < 3; ++ a )
            {
                if( ++ i[ a ] < hi[ a ] ) return * this;
                i[ a ] = lo[ a ];
            }
            end = true;
            return * this;
        }
        bool operator!=( const iterator & o ) const { return end != o.end; }
    };
    iterator begin(  ) const
    {
        bool empty = false;
        for( int a = 0; a < 3; ++ a ) empty |= hi_[ a ] <= lo_[ a ];
        return iterator{ lo_, lo_, hi_, empty };
    }
    iterator end(  ) const { return iterator{ lo_, lo_, hi_, true }; }
};

inline loop_t loop( const type::idx_t & i_max )
{
    return loop_t( type::idx_t( 0 ), i_max );
}
inline loop_t loop( const type::idx_t & i_min, const type::idx_t & i_max, bool include_max = false )
{
    type::idx_t hi = i_max;
    if( include_max ) for( int a = 0; a < 3; ++ a ) hi[ a ] += 1;
    return loop_t( i_min, hi );
}
}   // namespace utils
