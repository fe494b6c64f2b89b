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

__device__ __forceinline__ double rsqrt_rn( double x ) { return __dsqrt_rn( x ); }
__device__ __forceinline__ float  rsqrt_rn( float x )  { return __fsqrt_rn( x ); }

// Cyclic rotation of a 3-vector (utilities/mapping/mapping.h idx_swap).
template< class R > __device__ __forceinline__ void idx_swap( R * x, int axis )
{
    if( axis == 1 )      { const R t = x[ 0 ]; x[ 0 ] = x[ 1 ]; x[ 1 ] = x[ 2 ]; x[ 2 ] = t; }
    else if( axis == 2 ) { const R t = x[ 2 ]; x[ 2 ] = x[ 1 ]; x[ 1 ] = x[ 0 ]; x[ 0 ] = t; }
}

////////////////////////////////////////////////////////////
// EOS (hydro/eos/adiabatic.h:62-85, 159-206; mhd/eos/adiabatic.h:84-98)

// Total energy and sound speed of a primitive state; returns 1 / (gamma - 1).
template< class R > __device__ __forceinline__
R et_cs( R gamma, R & e_tot, R & c_s, const R * w )
{
    const R pre = w[ ENE ], rho = w[ RHO ];
    const R cv_kb = R( 1 ) / ( gamma - R( 1 ) );
    R v2 = 0;
    for( int a = 0; a < 3; ++ a )
        v2 += w[ MOM + a ] * w[ MOM + a ];
    e_tot = pre * cv_kb + rho * v2 / R( 2 );
    c_s   = rsqrt_rn( gamma * rmax( pre / rho, R( 0 ) ) );
    return cv_kb;
}

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
// PLM, van Leer harmonic limiter (hydro/reconstruct/plm.h:116-153).  For float
// the differences are first normalised by their largest magnitude.

template< class R > __device__ __forceinline__
void plm_face( R q_ll, R q_l, R q_r, R q_rr, R & ql, R & qr )
{
    const R dql = ( q_l  - q_ll );
    const R dqc = ( q_r  - q_l  );
    const R dqr = ( q_rr - q_r  );
    R norm( 1 );
    if constexpr( sizeof( R ) == 4 )
        if( uabs( dqc ) > R( 1e-24f ) || uabs( dqr ) > R( 1e-24f ) || uabs( dql ) > R( 1e-24f ) )
        {
            norm = rmax( uabs( dqr ), uabs( dql ) );
            norm = R( 1 ) / rmax( uabs( dqc ), norm );
        }
    const R dqr2  = norm * dqr * dqr;
    const R dql2  = norm * dql * dql;
    const R dqc2  = norm * dqc * dqc;
    const R dq2_l = norm * dql * dqc;
    const R dq2_r = norm * dqr * dqc;
    const R ql_coef = dq2_l <= 0 ? R( 0 ) :  dq2_l / ( dql2 + dqc2 + dq2_l * R( 2 ) );
    const R qr_coef = dq2_r <= 0 ? R( 0 ) : -dq2_r / ( dqr2 + dqc2 + dq2_r * R( 2 ) );
    ql = q_l + ( dq2_l <= 0 ? R( 0 ) : ql_coef * ( dql + dqc ) );
    qr = q_r + ( dq2_r <= 0 ? R( 0 ) : qr_coef * ( dqc + dqr ) );
}

////////////////////////////////////////////////////////////
// HLLC (hydro/riemann/hllc.h:239-250 f_lr_hyd, 262-379 eval) on rotated
// primitive states wl / wr (overwritten as scratch).

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
void hllc_eval( R * flx, R * wli, R * wri, R gamma )
{
    R el, er, cl, cr;
    const R gm1i_l = et_cs( gamma, el, cl, wli );
    const R gm1i_r = et_cs( gamma, er, cr, wri );
    R wroe[ 5 ];
    const R sqrtdl  = rsqrt_rn( wli[ RHO ] );
    const R sqrtdr  = rsqrt_rn( wri[ RHO ] );
    const R isdlpdr = R( 1 ) / ( sqrtdl + sqrtdr );
    wroe[ RHO ] = sqrtdl * sqrtdr;
    for( int n = MOM; n < MOM + 3; ++ n )
        wroe[ n ] = ( sqrtdl * wli[ n ] + sqrtdr * wri[ n ] ) * isdlpdr;
    const R hroe = isdlpdr * ( ( el + wli[ ENE ] ) / sqrtdl + ( er + wri[ ENE ] ) / sqrtdr );
    const R gam1_roe = R( 1 ) / ( isdlpdr * ( sqrtdl * gm1i_l + sqrtdr * gm1i_r ) );
    const R v2roe = wroe[ MOM ] * wroe[ MOM ] + wroe[ MOM + 1 ] * wroe[ MOM + 1 ]
                  + wroe[ MOM + 2 ] * wroe[ MOM + 2 ];
    const R q = hroe - R( 0.5f ) * v2roe;
    const R a = ( q <= 0 ) ? R( 0 ) : rsqrt_rn( gam1_roe * q );
    const R al = rmin( wroe[ MOM ] - a, wli[ MOM ] - cl );
    const R ar = rmax( wroe[ MOM ] + a, wri[ MOM ] + cr );
    const R bp = ar > 0 ? ar : R( 0 );
    const R bm = al < 0 ? al : R( 0 );
    const R vxl = wli[ MOM ] - al;
    const R vxr = wri[ MOM ] - ar;
    const R tl  = wli[ ENE ] + vxl * wli[ RHO ] * wli[ MOM ];
    const R tr  = wri[ ENE ] + vxr * wri[ RHO ] * wri[ MOM ];
    const R ml  =  wli[ RHO ] * vxl;
    const R mr  = -wri[ RHO ] * vxr;
    R cp, am;
    const R f_max = R( FLT_MAX / 1e1f );
    const R f_min = R( FLT_MIN * 1e1f );
    if( uabs( ml + mr ) < f_min )
    {
        cp = 0;
        am = 0;
    }
    else if( ( tr != 0 && uabs( ml ) > f_max / uabs( tr ) ) ||
             ( tl != 0 && uabs( mr ) > f_max / uabs( tl ) ) )
    {
        const R mli = R( sgn( ml ) ) / rmax( uabs( ml ), f_min );
        const R mri = R( sgn( mr ) ) / rmax( uabs( mr ), f_min );
        am = ( tl - tr ) / ( ml + mr );
        cp = rmax( ( mri * tr + mli * tl ) / ( mli + mri ), R( 0 ) );
    }
    else
    {
        am = ( tl - tr ) / ( ml + mr );
        cp = rmax( ( ml * tr + mr * tl ) / ( ml + mr ), R( 0 ) );
    }
    const R d_am_bm = rmax( uabs( am - bm ), f_min ) * R( am > bm ? 1 : -1 );
    const R d_am_bp = rmax( uabs( am - bp ), f_min ) * R( am > bp ? 1 : -1 );
    const R sl = ( am >= 0 ? am / d_am_bm : R( 0 ) );
    const R sr = ( am <  0 ? am / d_am_bp : R( 0 ) );
    const R sm = ( am >  0 ? -bm / d_am_bm : -bp / d_am_bp );
    R fl[ 5 ], fr[ 5 ];
    f_lr_hyd( fl, wli, wli[ MOM ] - bm, el );
    f_lr_hyd( fr, wri, wri[ MOM ] - bp, er );
    for( int n = RHO; n < MOM + 3; ++ n )
        flx[ n ] = sl * fl[ n ] + sr * fr[ n ];
    flx[ MOM ] += sm * cp;
    flx[ ENE ] += sm * cp * am;
}

////////////////////////////////////////////////////////////
// HLLE: the two-wave flux with the HLLD outer (fast magnetosonic) speed
// bounds (mhd/riemann/hlld.h:132-140 for the bounds; Harten, Lax & van Leer
// 1983 / Einfeldt 1988 for the flux).  No reference counterpart: it is the cheap
// flux of the learned face selector.  Rotated primitive states in, rotated
// flux out (B flux in slots BCC+1, BCC+2; slot BCC zero).

template< class R > __device__ __forceinline__
R hlld_cons( R * u, const R * w, R bx_2, R b_x, R gamma, R & gam1 )
{
    R p_m = bx_2 / R( 2 ), cs;
    for( int a = 1; a <= 2; ++ a )
    {
        const int n = BCC + a;
        p_m += w[ n ] * w[ n ] / R( 2 );
        u[ n ] = w[ n ];
    }
    gam1 = R( 1 ) / et_cs( gamma, u[ ENE ], cs, w );
    for( int n = MOM; n < MOM + 3; ++ n )
        u[ n ] = w[ RHO ] * w[ n ];
    u[ RHO ] = w[ RHO ];
    u[ ENE ] += p_m;
    u[ BCC ] = b_x;
    return p_m;
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

template< class R > __device__ __forceinline__
void hlle_eval( R * flx, const R * wli, const R * wri, R gamma )
{
    R u_l[ 8 ], u_r[ 8 ], f_l[ 8 ], f_r[ 8 ];
    const R b_x = wli[ BCC ], bx_2 = b_x * b_x;
    R gam1_l, gam1_r;
    const R pm_l = hlld_cons( u_l, wli, bx_2, b_x, gamma, gam1_l );
    const R pm_r = hlld_cons( u_r, wri, bx_2, b_x, gamma, gam1_r );
    R b2_l[ 3 ] = { bx_2, wli[ BCC + 1 ] * wli[ BCC + 1 ], wli[ BCC + 2 ] * wli[ BCC + 2 ] };
    R b2_r[ 3 ] = { bx_2, wri[ BCC + 1 ] * wri[ BCC + 1 ], wri[ BCC + 2 ] * wri[ BCC + 2 ] };
    const R cfm_l = c_fms( wli, b2_l, gam1_l + R( 1 ), 0 );
    const R cfm_r = c_fms( wri, b2_r, gam1_r + R( 1 ), 0 );
    const R s_l = rmin( rmin( wli[ MOM ] - cfm_l, wri[ MOM ] - cfm_r ), R( 0 ) );
    const R s_r = rmax( rmax( wli[ MOM ] + cfm_l, wri[ MOM ] + cfm_r ), R( 0 ) );
    hlld_f_flux( f_l, u_l, wli, wli[ ENE ] + pm_l, b_x );
    hlld_f_flux( f_r, u_r, wri, wri[ ENE ] + pm_r, b_x );
    f_l[ BCC ] = f_r[ BCC ] = 0;
    const R inv = R( 1 ) / ( s_r - s_l );
    for( int n = 0; n < 8; ++ n )
        flx[ n ] = ( s_r * f_l[ n ] - s_l * f_r[ n ] + s_r * s_l * ( u_r[ n ] - u_l[ n ] ) ) * inv;
    flx[ BCC ] = 0;
}

////////////////////////////////////////////////////////////
// HLLD (mhd/riemann/hlld.h:81-298 eval) on rotated primitive states.

template< class R > __device__ __forceinline__
R hlld_star( R * u_star, const R * u, const R * w, R rhos, R sd, R sdm, R p_tot,
             R b_x, R bx_2, R ptot_s, R spd0, R f_tiny )
{
    u_star[ RHO ] = rhos;
    u_star[ MOM ] = rhos * spd0;
    u_star[ BCC ] = b_x;
    const R denom = u[ RHO ] * sd * sdm - bx_2;
    if( uabs( denom ) < f_tiny * ptot_s )
        for( int a = 1; a <= 2; ++ a )
        {
            u_star[ MOM + a ] = rhos * w[ MOM + a ];
            u_star[ BCC + a ] = u[ BCC + a ];
        }
    else
    {
        const R tmp_v = b_x * ( sd - sdm ) / denom;
        const R tmp_b = ( u[ RHO ] * sd * sd - bx_2 ) / denom;
        for( int a = 1; a <= 2; ++ a )
        {
            u_star[ MOM + a ] = rhos * ( w[ MOM + a ] - u[ BCC + a ] * tmp_v );
            u_star[ BCC + a ] = u[ BCC + a ] * tmp_b;
        }
    }
    R u_dot_b = 0, w_dot_b = 0;
    for( int a = 0; a < 3; ++ a )
    {
        u_dot_b += u_star[ MOM + a ] * u_star[ BCC + a ];
        w_dot_b += w[ MOM + a ] * u[ BCC + a ];
    }
    u_dot_b /= rhos;
    u_star[ ENE ] = b_x * ( w_dot_b - u_dot_b ) - p_tot * w[ MOM ] + sd * u[ ENE ] + ptot_s * spd0;
    u_star[ ENE ] /= sdm;
    return u_dot_b;
}

template< class R > __device__ __forceinline__
void hlld_eval( R * flx, const R * wli, const R * wri, R gamma )
{
    flx[ BCC ] = 0;
    R u_l[ 8 ], u_r[ 8 ];
    const R b_x  = wli[ BCC ];
    const R bx_2 = b_x * b_x;
    R gam1_l, gam1_r;
    const R pm_l = hlld_cons( u_l, wli, bx_2, b_x, gamma, gam1_l );
    const R pm_r = hlld_cons( u_r, wri, bx_2, b_x, gamma, gam1_r );
    const R ptot_l = wli[ ENE ] + pm_l;
    const R ptot_r = wri[ ENE ] + pm_r;
    R b2_l[ 3 ] = { b_x, wli[ BCC + 1 ], wli[ BCC + 2 ] };
    R b2_r[ 3 ] = { b_x, wri[ BCC + 1 ], wri[ BCC + 2 ] };
    for( int a = 0; a < 3; ++ a )
    {
        b2_l[ a ] *= b2_l[ a ];
        b2_r[ a ] *= b2_r[ a ];
    }
    const R cfm_l = c_fms( wli, b2_l, gam1_l + R( 1 ), 0 );
    const R cfm_r = c_fms( wri, b2_r, gam1_r + R( 1 ), 0 );
    const R spd_m2 = rmin( wli[ MOM ] - cfm_l, wri[ MOM ] - cfm_r );
    const R spd_p2 = rmax( wli[ MOM ] + cfm_l, wri[ MOM ] + cfm_r );
    if( spd_m2 >= 0 || spd_p2 <= 0 )
    {
        const bool is_left = spd_m2 >= 0;
        hlld_f_flux( flx, is_left ? u_l : u_r, is_left ? wli : wri,
                     is_left ? ptot_l : ptot_r, b_x );
        return;
    }
    const R sd_l = spd_m2 - wli[ MOM ];
    const R sd_r = spd_p2 - wri[ MOM ];
    const R spd0 = ( sd_r * u_r[ MOM ] - ptot_r - sd_l * u_l[ MOM ] + ptot_l )
                 / ( sd_r * u_r[ RHO ] - sd_l * u_l[ RHO ] );
    const R sdm_l  = spd_m2 - spd0;
    const R sdm_r  = spd_p2 - spd0;
    const R rhos_l = u_l[ RHO ] * sd_l / sdm_l;
    const R rhos_r = u_r[ RHO ] * sd_r / sdm_r;
    const R rhos_l_sqrt = sqrt( rhos_l );
    const R rhos_r_sqrt = sqrt( rhos_r );
    const R spd_m1 = spd0 - uabs( b_x ) / rhos_l_sqrt;
    const R spd_p1 = spd0 + uabs( b_x ) / rhos_r_sqrt;
    const R f_tiny = R( 1.00e-4f );
    const R ptot_s = ptot_l + u_l[ RHO ] * sd_l * ( sd_l - sdm_l );
    R us_l[ 8 ], us_r[ 8 ];
    const R u_dot_b_l = hlld_star( us_l, u_l, wli, rhos_l, sd_l, sdm_l, ptot_l,
                                   b_x, bx_2, ptot_s, spd0, f_tiny );
    const R u_dot_b_r = hlld_star( us_r, u_r, wri, rhos_r, sd_r, sdm_r, ptot_r,
                                   b_x, bx_2, ptot_s, spd0, f_tiny );
    if( spd_m1 >= 0 )
    {
        hlld_f_flux( flx, u_l, wli, ptot_l, b_x );
        for( int n = 0; n < 8; ++ n )
            flx[ n ] += spd_m2 * ( us_l[ n ] - u_l[ n ] );
        return;
    }
    if( spd_p1 <= 0 )
    {
        hlld_f_flux( flx, u_r, wri, ptot_r, b_x );
        for( int n = 0; n < 8; ++ n )
            flx[ n ] += spd_p2 * ( us_r[ n ] - u_r[ n ] );
        return;
    }
    R uss_l[ 8 ], uss_r[ 8 ];
    for( int n = 0; n < 8; ++ n )
    {
        uss_l[ n ] = us_l[ n ];
        uss_r[ n ] = us_r[ n ];
    }
    if( bx_2 > ptot_s * f_tiny )
    {
        const R bx_sgn = b_x > 0 ? R( 1 ) : R( -1 );
        const R rhos_norm_inv = R( 1.f ) / ( rhos_l_sqrt + rhos_r_sqrt );
        for( int a = 1; a <= 2; ++ a )
        {
            R tmp = rhos_norm_inv *
                ( us_l[ MOM + a ] / rhos_l_sqrt + us_r[ MOM + a ] / rhos_r_sqrt
                + bx_sgn * ( us_r[ BCC + a ] - us_l[ BCC + a ] ) );
            uss_l[ MOM + a ] = uss_l[ RHO ] * tmp;
            uss_r[ MOM + a ] = uss_r[ RHO ] * tmp;
            tmp = rhos_norm_inv *
                ( rhos_l_sqrt * us_r[ BCC + a ] + rhos_r_sqrt * us_l[ BCC + a ]
                + bx_sgn * rhos_l_sqrt * rhos_r_sqrt
                * ( us_r[ MOM + a ] / rhos_r - us_l[ MOM + a ] / rhos_l ) );
            uss_l[ BCC + a ] = tmp;
            uss_r[ BCC + a ] = tmp;
        }
        const R tmp = spd0 * b_x + ( uss_l[ MOM + 1 ] * uss_l[ BCC + 1 ]
                                   + uss_l[ MOM + 2 ] * uss_l[ BCC + 2 ] ) / uss_l[ RHO ];
        uss_l[ ENE ] -= rhos_l_sqrt * bx_sgn * ( u_dot_b_l - tmp );
        uss_r[ ENE ] += rhos_r_sqrt * bx_sgn * ( u_dot_b_r - tmp );
    }
    if( spd0 >= 0 )
    {
        hlld_f_flux( flx, u_l, wli, ptot_l, b_x );
        const R d_v = spd_m1 - spd_m2;
        for( int n = 0; n < 8; ++ n )
            flx[ n ] += -spd_m2 * u_l[ n ] - d_v * us_l[ n ] + spd_m1 * uss_l[ n ];
    }
    else
    {
        hlld_f_flux( flx, u_r, wri, ptot_r, b_x );
        const R d_v = spd_p1 - spd_p2;
        for( int n = 0; n < 8; ++ n )
            flx[ n ] += -spd_p2 * u_r[ n ] - d_v * us_r[ n ] + spd_p1 * uss_r[ n ];
    }
}

}   // namespace kr
