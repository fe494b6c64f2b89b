// Per-cell and per-face arithmetic of the hydro / ideal-MHD step, as device
// functions templated on the reconstruction / Riemann real type R (double for
// the plain FP64 step, float for the mixed step whose conserved state, CT face
// update, dt reduction and cons-to-prim stay in double).
//
// Each function restates the reference expression by expression (paths relative
// to the Kratos source tree); the compiler may fuse multiply-adds, so results
// agree with the reference to rounding, not bit for bit.
#pragma once

#include <cfloat>
#include <cstdint>

namespace kr
{
enum { RHO = 0, ENE = 1, MOM = 2, BCC = 5 };              // dynamics/indices.h:5-13

__device__ __forceinline__ int mod3( int a ) { return a < 3 ? a : a - 3; }

template< class R > __device__ __forceinline__ R rmax( R a, R b ) { return a > b ? a : b; }
template< class R > __device__ __forceinline__ R rmin( R a, R b ) { return a < b ? a : b; }
template< class R > __device__ __forceinline__ R uabs( R a ) { return a > 0 ? a : -a; }
template< class R > __device__ __forceinline__ int sgn( R a ) { return a > 0 ? 1 : ( a < 0 ? -1 : 0 ); }

// Cyclic rotation of a 3-vector (utilities/mapping/mapping.h idx_swap).
template< class R > __device__ __forceinline__ void idx_swap( R * x, int axis )
{
    if( axis == 1 )      { const R t = x[ 0 ]; x[ 0 ] = x[ 1 ]; x[ 1 ] = x[ 2 ]; x[ 2 ] = t; }
    else if( axis == 2 ) { const R t = x[ 2 ]; x[ 2 ] = x[ 1 ]; x[ 1 ] = x[ 0 ]; x[ 0 ] = t; }
}

////////////////////////////////////////////////////////////
// EOS (hydro/eos/adiabatic.h:62-85, 159-206; mhd/eos/adiabatic.h:84-98)

// Fast magnetosonic speed along `axis` from squared field components b_2.
template< class R > __device__ __forceinline__
R c_fms( const R * w, const R * b_2, R gam, int axis )
{
    const R rho   = w[ RHO ];
    const R cs_2  = w[ ENE ] * gam / rho;
    const R v_ax2 = b_2[ axis ] / rho;
    const R v_t2  = ( b_2[ mod3( axis + 1 ) ] + b_2[ mod3( axis + 2 ) ] ) / rho;
    const R q_2   = v_ax2 + v_t2 + cs_2;
    const R r_2   = v_ax2 + v_t2 - cs_2;
    return sqrt( R( 0.5f ) * ( q_2 + sqrt( r_2 * r_2 + R( 4 ) * cs_2 * v_t2 ) ) );
}

// Fast magnetosonic speed along `axis` with 1 / rho given (c_fms with its three
// divisions by rho replaced by products).
template< class R > __device__ __forceinline__
R c_fms_ri( const R * w, const R * b_2, R gam, int axis, R rho_inv )
{
    const R cs_2  = w[ ENE ] * gam * rho_inv;
    const R v_ax2 = b_2[ axis ] * rho_inv;
    const R v_t2  = ( b_2[ mod3( axis + 1 ) ] + b_2[ mod3( axis + 2 ) ] ) * rho_inv;
    const R q_2   = v_ax2 + v_t2 + cs_2;
    const R r_2   = v_ax2 + v_t2 - cs_2;
    return sqrt( R( 0.5f ) * ( q_2 + sqrt( r_2 * r_2 + R( 4 ) * cs_2 * v_t2 ) ) );
}

// Conserved -> primitive with density / pressure floors (always FP64).
// cons[0..4] in; prim[0..4] out; floor corrections are written back to cons
// and flagged in the return's low bits (1: rho floored, 2: energy healed).
// cs2 receives the squared sound speed.
__device__ __forceinline__
int c2p( const double * cons_in, double * prim, double * cons_out, double gamma,
         double d_floor, double t_floor, double & cs2 )
{
    int healed = 0;
    double rho = cons_in[ RHO ];
    cons_out[ RHO ] = rho;
    cons_out[ ENE ] = cons_in[ ENE ];
    if( isnan( rho ) || rho < d_floor )
    {
        rho = d_floor;
        cons_out[ RHO ] = d_floor;
        healed |= 1;
    }
    prim[ RHO ] = rho;
    const double rho_inv = 1 / rho;
    double e_k = 0.;
    for( int n = MOM; n < MOM + 3; ++ n )
    {
        prim[ n ] = rho_inv * cons_in[ n ];
        e_k += cons_in[ n ] * cons_in[ n ];
    }
    e_k *= rho_inv / 2;
    const double e_g   = cons_in[ ENE ] - e_k;
    // the reference divides by cv = 1 / (gamma - 1) and by rho; multiplying by
    // gamma - 1 and 1 / rho differs in rounding only
    prim[ ENE ] = e_g * ( gamma - 1 );
    cs2 = gamma * prim[ ENE ] * rho_inv;
    const double pre_floor = t_floor * prim[ RHO ];
    if( isnan( prim[ ENE ] ) || prim[ ENE ] < pre_floor )
    {
        const double pre = pre_floor;
        prim[ ENE ] = pre;
        cons_out[ ENE ] = e_k + pre / ( gamma - 1 );
        cs2 = gamma * pre / rho;
        healed |= 2;
    }
    return healed;
}

////////////////////////////////////////////////////////////
// Physical flux of a rotated hydro state (hydro/riemann/hllc.h:239-250
// f_lr_hyd) and of an MHD state (mhd/riemann/hlld.h:49-80 f_flux), used by
// the solvers in kr_fast.cuh.

template< class R > __device__ __forceinline__
void f_lr_hyd( R * f, const R * w, R v, R e )
{
    const R rho = w[ RHO ];
    const R pre = w[ ENE ];
    f[ RHO ] = rho * v;
    f[ ENE ] = pre * w[ MOM ] + e * v;
    for( int a = MOM; a < MOM + 3; ++ a )
        f[ a ] = rho * w[ a ] * v;
    f[ MOM ] += pre;
}

template< class R > __device__ __forceinline__
void hlld_f_flux( R * flux, const R * u, const R * w, R p_tot, R b_x )
{
    const R bx_2 = b_x * b_x;
    flux[ RHO ] = u[ MOM ];
    flux[ ENE ] = w[ MOM ] * ( p_tot + u[ ENE ] - bx_2 ) - b_x
                * ( w[ MOM + 1 ] * u[ BCC + 1 ] + w[ MOM + 2 ] * u[ BCC + 2 ] );
    flux[ MOM ]     = p_tot - bx_2 + u[ MOM ] * w[ MOM ];
    flux[ MOM + 1 ] = -b_x * u[ BCC + 1 ] + u[ MOM + 1 ] * w[ MOM ];
    flux[ MOM + 2 ] = -b_x * u[ BCC + 2 ] + u[ MOM + 2 ] * w[ MOM ];
    flux[ BCC + 1 ] = -b_x * w[ MOM + 1 ] + u[ BCC + 1 ] * w[ MOM ];
    flux[ BCC + 2 ] = -b_x * w[ MOM + 2 ] + u[ BCC + 2 ] * w[ MOM ];
}

}   // namespace kr
