// Uniform Cartesian block geometry (src/mesh/geometry/geometry.h:23-173 and
// meshgen.cpp:252-363 of the reference): face origin xf0, spacing dx0 = loc(1)
// - loc(0), face areas and cell volume as products of spacings.
#pragma once

#include "../../types.h"

namespace mesh
{
using type::idx_t;

struct geo_t
{
    idx_t  n_ceff;
    int    n_dim = 3, n_gh = 2;
    bool   is_uniform[ 3 ] = { true, true, true };
    double xf0[ 3 ] = { 0, 0, 0 }, dx0[ 3 ] = { 1, 1, 1 }, sfc0[ 3 ] = { 1, 1, 1 }, vol0 = 1;
    bool   phybnd_flag[ 3 ][ 2 ] = { { false, false }, { false, false }, { false, false } };

    double x_cc( int ax, int i ) const { return xf0[ ax ] + ( i + 0.5f ) * dx0[ ax ]; }
    double x_fc( int ax, int i ) const { return xf0[ ax ] + i * dx0[ ax ]; }
    template< class I > double dx_f( int a, const I & ) const { return dx0[ a ]; }
    template< class I > double surface( const I &, int a ) const { return sfc0[ a ]; }
    template< class I > double volume( const I & ) const { return vol0; }
};
}   // namespace mesh
