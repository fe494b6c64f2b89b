// Per-block host arrays with the reference's layout (src/mesh/types/dat_3d.h:
// field index fastest, then x, y, z; n_cell includes 2 * n_gh ghosts).
#pragma once

#include <vector>
#include "../../types.h"

namespace mesh
{
using type::idx_t;

template< class T >
struct dat_3d_t
{
    using f_t = T;
    std::vector< T > buf;
    T * dat = nullptr;
    int n_int = 1, n_step = 1;
    idx_t n_cell, n_gh;
    size_t n_ctot = 0;

    void init( const idx_t & n_ceff, const idx_t & gh, int nint )
    {
        n_int = nint;
        n_gh = gh;
        n_ctot = size_t( nint );
        for( int a = 0; a < 3; ++ a )
        {
            n_cell[ a ] = n_ceff[ a ] + 2 * gh[ a ];
            n_ctot *= size_t( n_cell[ a ] );
        }
        buf.assign( n_ctot, T( 0 ) );
        dat = buf.data(  );
    }
    size_t idx( const idx_t & i ) const
    {
        return ( size_t( i[ 0 ] + n_gh[ 0 ] ) + size_t( n_cell[ 0 ] ) *
               ( size_t( i[ 1 ] + n_gh[ 1 ] ) + size_t( n_cell[ 1 ] ) *
                 size_t( i[ 2 ] + n_gh[ 2 ] ) ) ) * n_int;
    }
    T * at( const idx_t & i ) const { return const_cast< T * >( dat ) + idx( i ); }
    T & operator(  )( const idx_t & i ) const { return * at( i ); }
    explicit operator bool(  ) const { return dat != nullptr; }
};
}   // namespace mesh
