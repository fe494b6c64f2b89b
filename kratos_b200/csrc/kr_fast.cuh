// Face arithmetic of the step, arranged for the FP64 / FP32 pipes of sm_100a.
//
// Same mathematics as kr_math.cuh (which restates the reference expression by
// expression), with every division by a shared denominator replaced by one
// reciprocal: 1 / rho per state, 1 / (gamma - 1) and gamma - 1 from the host,
// rsqrt for the star-state densities, one reciprocal per HLLD star denominator,
// and the van Leer PLM slope (dl dc / (dl + dc), algebraically the reference's
// dl dc (dl + dc) / (dl^2 + dc^2 + 2 dl dc)) with one reciprocal for both faces.
// Results differ from the reference by rounding only; the GPU parity tests state
// the bound.  FP64 divides are long dependent DFMA sequences, so this is what
// moves the FP64 flux kernel off its latency floor.
#pragma once

#include "kr_math.cuh"

namespace kr
{
template< class R > struct eos_c
{
    R gamma, gm1, cv;        // gamma, gamma - 1, 1 / (gamma - 1)
};

// FP64: correctly rounded reciprocal / IEEE square root.  FP32 (the mixed
// step, whose error budget is 1e-4 in density): the SFU approximations, one
// MUFU instruction each instead of an IEEE refinement sequence.
__device__ __forceinline__ double rcp( double x ) { return __drcp_rn( x ); }
__device__ __forceinline__ float  rcp( float x )  { return __fdividef( 1.0f, x ); }
__device__ __forceinline__ double rsq( double x ) { return rsqrt( x ); }
__device__ __forceinline__ float  rsq( float x )  { return rsqrtf( x ); }
__device__ __forceinline__ double fsqrt( double x ) { return sqrt( x ); }
__device__ __forceinline__ float  fsqrt( float x )  { return x > 0.f ? x * rsqrtf( x ) : 0.f; }

// PLM on one face from the four cells around it (plm.h:116-153 mathematics).
template< class R > __device__ __forceinline__
void plm_face_fast( R q_ll, R q_l, R q_r, R q_rr, R & ql, R & qr )
{
    R dql = q_l - q_ll, dqc = q_r - q_l, dqr = q_rr - q_r;
    if constexpr( sizeof( R ) == 4 )
    {   // Scale-free form of the same limiter: dl dr / ( dl + dr ) =
        // dl * ( dr / ( dl + dr ) ), whose quotient lies in ( 0, 1 ) when dl
        // and dr share a sign, so the slope never forms the product of two
        // differences -- no FP32 overflow for huge differences (the
        // reference's FP32 path rescales by max |d| for the same purpose).
        // Same sign is a positive product of the two differences (the limited
        // slope itself is formed scale-free below).  A positive product needs
        // one difference of normal size, so the sum is normal and its SFU
        // reciprocal finite (a subnormal sum would give 1 / 0 = inf); two
        // differences whose product underflows (both below ~1e-23) give no
        // slope.  plm_face_fast2 makes the same test on pairs.
        const bool lpos = dql * dqc > R( 0 );
        const bool rpos = dqr * dqc > R( 0 );
        ql = lpos ? q_l + dql * ( dqc * rcp( dql + dqc ) ) : q_l;
        qr = rpos ? q_r - dqr * ( dqc * rcp( dqc + dqr ) ) : q_r;
        return;
    }
    const R scale = R( 1 );
    const R dq2_l = dql * dqc;
    const R dq2_r = dqr * dqc;
    const bool lpos = dq2_l > 0, rpos = dq2_r > 0;
    const R sl = lpos ? dql + dqc : R( 1 );
    const R sr = rpos ? dqc + dqr : R( 1 );
    const R inv = rcp( sl * sr );
    ql = lpos ? q_l + dq2_l * sr * inv * scale : q_l;
    qr = rpos ? q_r - dq2_r * sl * inv * scale : q_r;
}

// The FP32 limiter of plm_face_fast on two variables at once (.x, .y): the
// differences, sums and products as paired FP32 instructions (sm_100's
// FADD2 / FMUL2 / FFMA2), the sign tests and reciprocals per element.  Same
// operations per element as the scalar form.
__device__ __forceinline__
void plm_face_fast2( float2 q_ll, float2 q_l, float2 q_r, float2 q_rr, float2 & ql, float2 & qr )
{
    const float2 m1 = make_float2( -1.f, -1.f );
    const float2 dql = __ffma2_rn( q_ll, m1, q_l );      // q_l - q_ll, exact
    const float2 dqc = __ffma2_rn( q_l, m1, q_r );
    const float2 dqr = __ffma2_rn( q_r, m1, q_rr );
    // same sign: a positive product (paired multiply, one compare each).  A
    // positive product needs one difference of normal size, so the sum below
    // is normal and its SFU reciprocal finite; differences whose product
    // underflows (both below ~1e-23) give no slope
    const float2 pl = __fmul2_rn( dql, dqc ), pr = __fmul2_rn( dqr, dqc );
    const bool lx = pl.x > 0.f, ly = pl.y > 0.f, rx = pr.x > 0.f, ry = pr.y > 0.f;
    const float2 sl = __fadd2_rn( dql, dqc ), sr = __fadd2_rn( dqc, dqr );
    const float2 il = make_float2( rcp( sl.x ), rcp( sl.y ) ), ir = make_float2( rcp( sr.x ), rcp( sr.y ) );
    const float2 tl = __fmul2_rn( dqc, il );
    const float2 tr = __fmul2_rn( __fmul2_rn( dqc, ir ), m1 );
    const float2 cl = __ffma2_rn( dql, tl, q_l );        // q_l + dql ( dqc / ( dql + dqc ) )
    const float2 cr = __ffma2_rn( dqr, tr, q_r );        // q_r - dqr ( dqc / ( dqc + dqr ) )
    ql = make_float2( lx ? cl.x : q_l.x, ly ? cl.y : q_l.y );
    qr = make_float2( rx ? cr.x : q_r.x, ry ? cr.y : q_r.y );
}

// Fast magnetosonic speed from squared field components and 1 / rho.
template< class R > __device__ __forceinline__
R c_fms_fast( R pre, R inv_rho, R bn2, R bt2, R gam )
{
    const R cs_2  = gam * pre * inv_rho;
    const R v_ax2 = bn2 * inv_rho;
    const R v_t2  = bt2 * inv_rho;
    const R q_2   = v_ax2 + v_t2 + cs_2;
    const R r_2   = v_ax2 + v_t2 - cs_2;
    return fsqrt( R( 0.5f ) * ( q_2 + fsqrt( r_2 * r_2 + R( 4 ) * cs_2 * v_t2 ) ) );
}

////////////////////////////////////////////////////////////
// HLLC on rotated primitive states (hllc.h:262-379 mathematics).

template< class R > __device__ __forceinline__
void hllc_fast( R * flx, const R * wl, const R * wr, const eos_c< R > & e )
{
    const R irl = rcp( wl[ RHO ] ), irr = rcp( wr[ RHO ] );
    R v2l = wl[ MOM ] * wl[ MOM ] + wl[ MOM + 1 ] * wl[ MOM + 1 ] + wl[ MOM + 2 ] * wl[ MOM + 2 ];
    R v2r = wr[ MOM ] * wr[ MOM ] + wr[ MOM + 1 ] * wr[ MOM + 1 ] + wr[ MOM + 2 ] * wr[ MOM + 2 ];
    const R el = wl[ ENE ] * e.cv + wl[ RHO ] * v2l * R( 0.5f );
    const R er = wr[ ENE ] * e.cv + wr[ RHO ] * v2r * R( 0.5f );
    const R cl = fsqrt( e.gamma * rmax( wl[ ENE ] * irl, R( 0 ) ) );
    const R cr = fsqrt( e.gamma * rmax( wr[ ENE ] * irr, R( 0 ) ) );
    const R rsl = rsq( wl[ RHO ] ), rsr = rsq( wr[ RHO ] );
    const R sqrtdl = wl[ RHO ] * rsl, sqrtdr = wr[ RHO ] * rsr;
    const R isdlpdr = rcp( sqrtdl + sqrtdr );
    R wroe[ 5 ];
    for( int n = MOM; n < MOM + 3; ++ n )
        wroe[ n ] = ( sqrtdl * wl[ n ] + sqrtdr * wr[ n ] ) * isdlpdr;
    const R hroe = isdlpdr * ( ( el + wl[ ENE ] ) * rsl + ( er + wr[ ENE ] ) * rsr );
    const R gam1_roe = e.gm1;            // constant gamma: the Roe average is gamma - 1
    const R v2roe = wroe[ MOM ] * wroe[ MOM ] + wroe[ MOM + 1 ] * wroe[ MOM + 1 ]
                  + wroe[ MOM + 2 ] * wroe[ MOM + 2 ];
    const R q = hroe - R( 0.5f ) * v2roe;
    const R a = ( q <= 0 ) ? R( 0 ) : fsqrt( gam1_roe * q );
    const R al = rmin( wroe[ MOM ] - a, wl[ MOM ] - cl );
    const R ar = rmax( wroe[ MOM ] + a, wr[ MOM ] + cr );
    const R bp = ar > 0 ? ar : R( 0 );
    const R bm = al < 0 ? al : R( 0 );
    const R vxl = wl[ MOM ] - al, vxr = wr[ MOM ] - ar;
    const R tl  = wl[ ENE ] + vxl * wl[ RHO ] * wl[ MOM ];
    const R tr  = wr[ ENE ] + vxr * wr[ RHO ] * wr[ MOM ];
    const R ml  =  wl[ RHO ] * vxl;
    const R mr  = -wr[ RHO ] * vxr;
    R cp, am;
    const R f_max = R( FLT_MAX / 1e1f ), f_min = R( FLT_MIN * 1e1f );
    if( uabs( ml + mr ) < f_min )
        cp = am = 0;
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
        const R im = rcp( ml + mr );
        am = ( tl - tr ) * im;
        cp = rmax( ( ml * tr + mr * tl ) * im, R( 0 ) );
    }
    const R d_am_bm = rmax( uabs( am - bm ), f_min ) * R( am > bm ? 1 : -1 );
    const R d_am_bp = rmax( uabs( am - bp ), f_min ) * R( am > bp ? 1 : -1 );
    const R i_bm = rcp( d_am_bm ), i_bp = rcp( d_am_bp );
    const R sl = am >= 0 ? am * i_bm : R( 0 );
    const R sr = am <  0 ? am * i_bp : R( 0 );
    const R sm = am >  0 ? -bm * i_bm : -bp * i_bp;
    R fl[ 5 ], fr[ 5 ];
    f_lr_hyd( fl, wl, wl[ MOM ] - bm, el );
    f_lr_hyd( fr, wr, wr[ MOM ] - bp, er );
    for( int n = RHO; n < MOM + 3; ++ n )
        flx[ n ] = sl * fl[ n ] + sr * fr[ n ];
    flx[ MOM ] += sm * cp;
    flx[ ENE ] += sm * cp * am;
}

////////////////////////////////////////////////////////////
// HLLD on rotated primitive states (hlld.h:81-298 mathematics).

template< class R > __device__ __forceinline__
R hlld_cons_fast( R * u, const R * w, R bx_2, R b_x, const eos_c< R > & e )
{
    const R p_m = ( bx_2 + w[ BCC + 1 ] * w[ BCC + 1 ] + w[ BCC + 2 ] * w[ BCC + 2 ] ) * R( 0.5f );
    const R v2 = w[ MOM ] * w[ MOM ] + w[ MOM + 1 ] * w[ MOM + 1 ] + w[ MOM + 2 ] * w[ MOM + 2 ];
    u[ RHO ] = w[ RHO ];
    u[ ENE ] = w[ ENE ] * e.cv + w[ RHO ] * v2 * R( 0.5f ) + p_m;
    for( int n = MOM; n < MOM + 3; ++ n )
        u[ n ] = w[ RHO ] * w[ n ];
    u[ BCC ] = b_x;
    u[ BCC + 1 ] = w[ BCC + 1 ];
    u[ BCC + 2 ] = w[ BCC + 2 ];
    return p_m;
}

template< class R > __device__ __forceinline__
R hlld_star_fast( R * us, const R * u, const R * w, R rhos, R inv_rhos, R sd, R inv_sdm,
                  R p_tot, R b_x, R bx_2, R ptot_s, R spd0, R f_tiny, R sdm )
{
    us[ RHO ] = rhos;
    us[ MOM ] = rhos * spd0;
    us[ BCC ] = b_x;
    const R denom = u[ RHO ] * sd * sdm - bx_2;
    if( uabs( denom ) < f_tiny * ptot_s )
        for( int a = 1; a <= 2; ++ a )
        {
            us[ MOM + a ] = rhos * w[ MOM + a ];
            us[ BCC + a ] = u[ BCC + a ];
        }
    else
    {
        const R id = rcp( denom );
        const R tmp_v = b_x * ( sd - sdm ) * id;
        const R tmp_b = ( u[ RHO ] * sd * sd - bx_2 ) * id;
        for( int a = 1; a <= 2; ++ a )
        {
            us[ MOM + a ] = rhos * ( w[ MOM + a ] - u[ BCC + a ] * tmp_v );
            us[ BCC + a ] = u[ BCC + a ] * tmp_b;
        }
    }
    R u_dot_b = 0, w_dot_b = 0;
    for( int a = 0; a < 3; ++ a )
    {
        u_dot_b += us[ MOM + a ] * us[ BCC + a ];
        w_dot_b += w[ MOM + a ] * u[ BCC + a ];
    }
    u_dot_b *= inv_rhos;
    us[ ENE ] = ( b_x * ( w_dot_b - u_dot_b ) - p_tot * w[ MOM ] + sd * u[ ENE ] + ptot_s * spd0 ) * inv_sdm;
    return u_dot_b;
}

// What HLLD and HLLE (the learned mode's cheap flux) both start from: the
// conserved states, total pressures and the outer wave speeds.
template< class R > struct hll_prefix
{
    R u_l[ 8 ], u_r[ 8 ];
    R b_x, bx_2, pm_l, pm_r, spd_m2, spd_p2;
};

template< class R > __device__ __forceinline__
void hll_prefix_fast( hll_prefix< R > & h, const R * wl, const R * wr, const eos_c< R > & e )
{
    h.b_x = wl[ BCC ];
    h.bx_2 = h.b_x * h.b_x;
    h.pm_l = hlld_cons_fast( h.u_l, wl, h.bx_2, h.b_x, e );
    h.pm_r = hlld_cons_fast( h.u_r, wr, h.bx_2, h.b_x, e );
    const R irl = rcp( wl[ RHO ] ), irr = rcp( wr[ RHO ] );
    const R cfm_l = c_fms_fast( wl[ ENE ], irl, h.bx_2,
                                wl[ BCC + 1 ] * wl[ BCC + 1 ] + wl[ BCC + 2 ] * wl[ BCC + 2 ], e.gamma );
    const R cfm_r = c_fms_fast( wr[ ENE ], irr, h.bx_2,
                                wr[ BCC + 1 ] * wr[ BCC + 1 ] + wr[ BCC + 2 ] * wr[ BCC + 2 ], e.gamma );
    h.spd_m2 = rmin( wl[ MOM ] - cfm_l, wr[ MOM ] - cfm_r );
    h.spd_p2 = rmax( wl[ MOM ] + cfm_l, wr[ MOM ] + cfm_r );
}

// HLLD from the prefix (mhd/riemann/hlld.h:31-298).
template< class R > __device__ __forceinline__
void hlld_tail( R * flx, const R * wl, const R * wr, const hll_prefix< R > & h )
{
    const R * u_l = h.u_l, * u_r = h.u_r;
    const R b_x = h.b_x, bx_2 = h.bx_2, spd_m2 = h.spd_m2, spd_p2 = h.spd_p2;
    const R ptot_l = wl[ ENE ] + h.pm_l, ptot_r = wr[ ENE ] + h.pm_r;
    flx[ BCC ] = 0;
    if( spd_m2 >= 0 || spd_p2 <= 0 )
    {
        const bool is_left = spd_m2 >= 0;
        hlld_f_flux( flx, is_left ? u_l : u_r, is_left ? wl : wr, is_left ? ptot_l : ptot_r, b_x );
        flx[ BCC ] = 0;
        return;
    }
    const R sd_l = spd_m2 - wl[ MOM ];
    const R sd_r = spd_p2 - wr[ MOM ];
    const R spd0 = ( sd_r * u_r[ MOM ] - ptot_r - sd_l * u_l[ MOM ] + ptot_l )
                 * rcp( sd_r * u_r[ RHO ] - sd_l * u_l[ RHO ] );
    const R sdm_l = spd_m2 - spd0, sdm_r = spd_p2 - spd0;
    const R isdm = rcp( sdm_l * sdm_r );
    const R inv_sdm_l = sdm_r * isdm, inv_sdm_r = sdm_l * isdm;
    const R rhos_l = u_l[ RHO ] * sd_l * inv_sdm_l;
    const R rhos_r = u_r[ RHO ] * sd_r * inv_sdm_r;
    const R rs_l = rsq( rhos_l ), rs_r = rsq( rhos_r );       // 1 / sqrt(rho*)
    const R rhos_l_sqrt = rhos_l * rs_l, rhos_r_sqrt = rhos_r * rs_r;
    const R irs_l = rs_l * rs_l, irs_r = rs_r * rs_r;          // 1 / rho*
    const R spd_m1 = spd0 - uabs( b_x ) * rs_l;
    const R spd_p1 = spd0 + uabs( b_x ) * rs_r;
    const R f_tiny = R( 1.00e-4f );
    const R ptot_s = ptot_l + u_l[ RHO ] * sd_l * ( sd_l - sdm_l );
    R us_l[ 8 ], us_r[ 8 ];
    const R udb_l = hlld_star_fast( us_l, u_l, wl, rhos_l, irs_l, sd_l, inv_sdm_l, ptot_l,
                                    b_x, bx_2, ptot_s, spd0, f_tiny, sdm_l );
    const R udb_r = hlld_star_fast( us_r, u_r, wr, rhos_r, irs_r, sd_r, inv_sdm_r, ptot_r,
                                    b_x, bx_2, ptot_s, spd0, f_tiny, sdm_r );
    if( spd_m1 >= 0 )
    {
        hlld_f_flux( flx, u_l, wl, ptot_l, b_x );
        for( int n = 0; n < 8; ++ n )
            flx[ n ] += spd_m2 * ( us_l[ n ] - u_l[ n ] );
        flx[ BCC ] = 0;
        return;
    }
    if( spd_p1 <= 0 )
    {
        hlld_f_flux( flx, u_r, wr, ptot_r, b_x );
        for( int n = 0; n < 8; ++ n )
            flx[ n ] += spd_p2 * ( us_r[ n ] - u_r[ n ] );
        flx[ BCC ] = 0;
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
        const R rni = rcp( rhos_l_sqrt + rhos_r_sqrt );
        for( int a = 1; a <= 2; ++ a )
        {
            R tmp = rni * ( us_l[ MOM + a ] * rs_l + us_r[ MOM + a ] * rs_r
                          + bx_sgn * ( us_r[ BCC + a ] - us_l[ BCC + a ] ) );
            uss_l[ MOM + a ] = uss_l[ RHO ] * tmp;
            uss_r[ MOM + a ] = uss_r[ RHO ] * tmp;
            tmp = rni * ( rhos_l_sqrt * us_r[ BCC + a ] + rhos_r_sqrt * us_l[ BCC + a ]
                        + bx_sgn * rhos_l_sqrt * rhos_r_sqrt
                        * ( us_r[ MOM + a ] * irs_r - us_l[ MOM + a ] * irs_l ) );
            uss_l[ BCC + a ] = tmp;
            uss_r[ BCC + a ] = tmp;
        }
        const R tmp = spd0 * b_x + ( uss_l[ MOM + 1 ] * uss_l[ BCC + 1 ]
                                   + uss_l[ MOM + 2 ] * uss_l[ BCC + 2 ] ) * irs_l;
        uss_l[ ENE ] -= rhos_l_sqrt * bx_sgn * ( udb_l - tmp );
        uss_r[ ENE ] += rhos_r_sqrt * bx_sgn * ( udb_r - tmp );
    }
    if( spd0 >= 0 )
    {
        hlld_f_flux( flx, u_l, wl, ptot_l, b_x );
        const R d_v = spd_m1 - spd_m2;
        for( int n = 0; n < 8; ++ n )
            flx[ n ] += -spd_m2 * u_l[ n ] - d_v * us_l[ n ] + spd_m1 * uss_l[ n ];
    }
    else
    {
        hlld_f_flux( flx, u_r, wr, ptot_r, b_x );
        const R d_v = spd_p1 - spd_p2;
        for( int n = 0; n < 8; ++ n )
            flx[ n ] += -spd_p2 * u_r[ n ] - d_v * us_r[ n ] + spd_p1 * uss_r[ n ];
    }
    flx[ BCC ] = 0;
}

// HLLE with the HLLD outer speeds, from the prefix.
template< class R > __device__ __forceinline__
void hlle_tail( R * flx, const R * wl, const R * wr, const hll_prefix< R > & h )
{
    R f_l[ 8 ], f_r[ 8 ];
    const R s_l = rmin( h.spd_m2, R( 0 ) );
    const R s_r = rmax( h.spd_p2, R( 0 ) );
    hlld_f_flux( f_l, h.u_l, wl, wl[ ENE ] + h.pm_l, h.b_x );
    hlld_f_flux( f_r, h.u_r, wr, wr[ ENE ] + h.pm_r, h.b_x );
    f_l[ BCC ] = f_r[ BCC ] = 0;
    const R inv = rcp( s_r - s_l );
    for( int n = 0; n < 8; ++ n )
        flx[ n ] = ( s_r * f_l[ n ] - s_l * f_r[ n ] + s_r * s_l * ( h.u_r[ n ] - h.u_l[ n ] ) ) * inv;
    flx[ BCC ] = 0;
}

template< class R > __device__ __forceinline__
void hlld_fast( R * flx, const R * wl, const R * wr, const eos_c< R > & e )
{
    hll_prefix< R > h;
    hll_prefix_fast( h, wl, wr, e );
    hlld_tail( flx, wl, wr, h );
}

// HLLE with the HLLD outer speeds (cheap flux of the learned selector).
template< class R > __device__ __forceinline__
void hlle_fast( R * flx, const R * wl, const R * wr, const eos_c< R > & e )
{
    hll_prefix< R > h;
    hll_prefix_fast( h, wl, wr, e );
    hlle_tail( flx, wl, wr, h );
}

// The learned mode's solver of one face, HLLE where `cheap`, else HLLD, from
// one shared prefix (one copy of it in the kernel).
template< class R > __device__ __forceinline__
void hll_pick_fast( R * flx, const R * wl, const R * wr, const eos_c< R > & e, bool cheap )
{
    hll_prefix< R > h;
    hll_prefix_fast( h, wl, wr, e );
    if( cheap ) hlle_tail( flx, wl, wr, h );
    else        hlld_tail( flx, wl, wr, h );
}

}   // namespace kr
