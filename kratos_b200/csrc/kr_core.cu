// kratos_b200 device engine: storage, kernels and the C ABI of
// include/kratos_b200.h.
//
// HBM layout (one pool per array, blocks back to back, component-major within
// a block, x fastest -- every kernel below maps consecutive threads to
// consecutive x, so all global traffic is coalesced):
//   U [slot][block][5][n2][n1][n0]           conserved rho, E, m0..2 (double)
//   BF[slot][block][3][n2+5][n1+5][n0+5]     face B, 2 ghost layers (double)
//   W [block][nw][n2+4][n1+4][n0+4]          primitives, 2 ghost layers (R)
//   F [axis][block][nf][n2+3][n1+3][n0+3]    face fluxes, 1 ghost layer (R);
//                                            nf = 5 hydro, 7 MHD (5 + edge E)
//   EE[block][3][n2+3][n1+3][n0+3]           edge EMF (R)
// R is double for the FP64 step and float for the mixed step.  One Heun step
// is 2 x (c2p, ghost, flux z, flux y, flux x, [emf], update) plus two scalar
// kernels, captured once into a CUDA graph and replayed.  On a uniform MHD mesh
// stage 0's two updates and stage 1's c2p are one launch (k_update_c2p).
#include "../../include/kratos_b200.h"
#include "kr_fast.cuh"
#include "kr_mlp.cuh"
#include "problems.h"
#include "smr_tree.h"

#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nccl.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <type_traits>
#include <unordered_map>
#include <vector>

namespace kr
{
////////////////////////////////////////////////////////////
// Device-side scalars of the time loop (cycle.cpp:77-115 semantics)

struct scal_t
{
    unsigned long long dt_bits;   // running CFL minimum (positive double bits)
    double dt_bound;              // value a step's minimum starts from
    double dt_last;               // dt of the last completed step
    double t;
    long long n_steps;
    int status;                   // sticky error bits
    int sel_force;                // learned mode: run the network at the next step
    int heal_count;               // floor corrections (diagnostic)
};

struct geo_t
{
    double dx[ 3 ], sfc[ 3 ], vol;
    double idx[ 3 ];              // 1 / dx
    double isfc[ 3 ];             // 1 / sfc (0 for an empty face)
    int phys;                     // bit 2a+s: side (a, s) is a non-periodic domain side
    int fine;                     // bit 2a+s: the neighbours across side (a, s) are finer
    int fitem[ 6 ];               // refined side: first of its 4 flux-average items
    int xlev;                     // bit 2a+s: the neighbours across side (a, s) are on another level
};

// Static refinement: one (block, face) pair across a level jump.  dst / src:
// the block written / read; face: the written block's side 2a+s; o1, o2: the
// cell offsets (along (a+1)%3, (a+2)%3) of the fine block's half inside the
// coarse block.
struct smr_item_t
{
    int dst, src, face, o1, o2;
};

// Kernel parameters (by value).
template< class R >
struct args_t
{
    int n0, n1, n2, nblk;
    long long nc, ngw, nbf, nfb;      // per-component sizes: U, W, BF, F/EE
    int sw1, sw2, sb1, sb2, sf1, sf2; // strides of W, BF, F/EE boxes
    double gamma, cfl, d_floor, t_floor, dt_expand;
    double gm1, cv;                   // gamma - 1 and 1 / (gamma - 1)
    double * u[ 2 ];
    double * bf[ 2 ];
    R * w;
    R * f[ 3 ];
    R * ee;
    const geo_t * geo;
    int boxes;                        // 1: every block an independent box, scalars s[ block ]
    // learned face selector (riemann == KR_RIEMANN_LEARNED)
    const unsigned * sel_w;           // [32 lanes][MLP_BFRAG] bf16 pairs
    const float * sel_b;              // b1, b2, b3
    float sel_thr;                    // logit threshold for HLLE
    unsigned long long * sel_cnt;     // [0] faces, [1] faces given HLLE
    unsigned * sel_dec;               // per (axis, block, warp of 32 faces): bit l = lane l on HLLE
    long long sel_wcap;               // warps of faces per (axis, block)
    int sel_period;                   // steps between evaluations of the network
    // face sampling for selector training (collect steps only)
    float * smp;                      // [max][17]: 16 features + flux gap
    unsigned long long * smp_n;
    long long smp_max;
    unsigned smp_stride, smp_seed;
    const int * nbr;                  // [block][27]: local block, -1 past a physical
                                      // boundary, -2 filled by the halo exchange
    const int * gid;                  // [block] global (lexicographic) block id
    int nbk[ 3 ];                     // blocks per axis (global mesh)
    int bc[ 6 ];                      // kr_bc_t per side
    double w_fix[ 5 ];
    double b_fix[ 3 ];
    int emf_out;                      // bit a: high side of axis a is out / fre (MHD)
    int vl2;                          // 1: VL2 integrator (donor-cell predictor)
    double * favg;                    // refined mesh: averaged fine face fluxes,
    int favg_n;                       //   [item][5][favg_n] (FP64 in both precisions)
    int mh_smr;                       // 1: refined MHD mesh (ghost-line normal B rule)
    scal_t * s;
};

template< class R > __device__ __forceinline__
long long iw( const args_t< R > & a, int b, int c, int nw, int i0, int i1, int i2 )
{
    return ( long long )( b * nw + c ) * a.ngw + ( i0 + 2 ) + a.sw1 * ( i1 + 2 ) + a.sw2 * ( i2 + 2 );
}
template< class R > __device__ __forceinline__
long long iuc( const args_t< R > & a, int b, int c, int i0, int i1, int i2 )
{
    return ( long long )( b * 5 + c ) * a.nc + i0 + a.n0 * ( i1 + a.n1 * i2 );
}
template< class R > __device__ __forceinline__
long long ibf( const args_t< R > & a, int b, int c, int i0, int i1, int i2 )
{
    return ( long long )( b * 3 + c ) * a.nbf + ( i0 + 2 ) + a.sb1 * ( i1 + 2 ) + a.sb2 * ( i2 + 2 );
}
template< class R > __device__ __forceinline__
long long ifx( const args_t< R > & a, int b, int c, int nf, int i0, int i1, int i2 )
{
    return ( long long )( b * nf + c ) * a.nfb + ( i0 + 1 ) + a.sf1 * ( i1 + 1 ) + a.sf2 * ( i2 + 1 );
}

// Quotient of a non-negative n by a fixed d >= 2 with one multiply-high:
// q = umulhi( n, ceil( 2^32 / d ) ), exact while n * d < 2^32 (the rounding
// error of the multiplier, below d, times n stays under 2^32).
struct udiv_t { unsigned d, m; };
static inline udiv_t make_udiv( unsigned d )
{
    return { d, unsigned( ( ( 1ull << 32 ) + d - 1 ) / d ) };
}
__device__ __forceinline__ unsigned udiv_q( unsigned n, const udiv_t & v ) { return __umulhi( n, v.m ); }

__device__ __forceinline__ double warp_min( double v )
{
    for( int o = 16; o > 0; o >>= 1 )
        v = fmin( v, __shfl_xor_sync( 0xffffffffu, v, o ) );
    return v;
}

////////////////////////////////////////////////////////////
// Scalars: step begin / end (cycle.cpp:77-115)

__device__ __forceinline__ bool sel_eval_step( const scal_t * s, int period )
{   // learned mode: the network runs at stage 0 of this step
    return s->sel_force || s->n_steps % period == 0;
}

// ns: 1, or one scalar set per block (independent boxes, KR_FLAG_BOXES); the
// status word of set 0 collects every set's.
__global__ void k_step_begin( scal_t * s, int ns )
{
    for( int k = 0; k < ns; ++ k )
        s[ k ].dt_bits = __double_as_longlong( s[ k ].dt_bound );
}

__global__ void k_step_end( scal_t * s, double dt_expand, int ns )
{
    for( int k = 0; k < ns; ++ k )
    {
        scal_t & r = s[ k ];
        const double dt = __longlong_as_double( r.dt_bits );
        if( ! ( dt > 0 ) || ! isfinite( dt ) )
            s[ 0 ].status |= 1;
        r.dt_last  = dt;
        r.t       += dt;
        r.dt_bound = dt * dt_expand;
        r.n_steps += 1;
        r.sel_force = 0;
    }
}

////////////////////////////////////////////////////////////
// cons -> prim over the interior of every block, CFL dt at stage 0
// (hydro/eos/adiabatic.h:211-258; mhd/eos/adiabatic.h:127-234).

// cons -> prim of interior cell (i0, i1, i2) of block b from its conserved
// words (cons, changed) and, MHD, the face B on its low and high side per axis
// (b_l, b_r): stores the W words into W (the primitives and the cell E),
// pushes them into the ghost shells of the same-level neighbours, and writes
// floored words back to U.  prim, bc_2, b_max, cs2 return what the CFL dt needs.
template< bool MHD, class R > __device__ __forceinline__
void c2p_point( const args_t< R > & a, R * W, double * U, int b, int i0, int i1, int i2,
                double * cons, const double * b_l, const double * b_r,
                double * prim, double * bc_2, double * b_max, double & cs2 )
{
    constexpr int NW = MHD ? 11 : 5;   // stored W words: prim (8) + cell E (3)
    double cout[ 5 ];
    double bc[ 3 ], e_m = 0;
    if( MHD )
    {
        for( int d = 0; d < 3; ++ d )
        {
            const double bc_m = ( b_l[ d ] + b_r[ d ] ) / 2;
            bc[ d ] = bc_m;
            bc_2[ d ] = bc_m * bc_m;
            e_m += bc_2[ d ];
            b_max[ d ] = fmax( fabs( b_l[ d ] ), fabs( b_r[ d ] ) );
        }
        e_m /= 2;
        cons[ ENE ] -= e_m;
    }
    const int healed = c2p( cons, prim, cout, a.gamma, a.d_floor, a.t_floor, cs2 );
    if( healed )
    {
        U[ iuc( a, b, RHO, i0, i1, i2 ) ] = cout[ RHO ];
        U[ iuc( a, b, ENE, i0, i1, i2 ) ] = MHD ? cout[ ENE ] + e_m : cout[ ENE ];
        atomicAdd( & a.s->heal_count, 1 );
    }
    R wv[ NW ];
    for( int k = 0; k < 5; ++ k )
        wv[ k ] = R( prim[ k ] );
    if( MHD )
        for( int d = 0; d < 3; ++ d )
        {   // cell-centred E = B x v (mhd/eos/adiabatic.h:216-220), from the
            // stored (R-rounded) primitives so ghost copies agree bit for bit
            const int d1 = mod3( d + 1 ), d2 = mod3( d + 2 );
            wv[ BCC + d ] = R( bc[ d ] );
            wv[ 8 + d ] = R( bc[ d1 ] ) * R( prim[ MOM + d2 ] ) - R( bc[ d2 ] ) * R( prim[ MOM + d1 ] );
        }
    const int ngw = int( a.ngw );
    {
        R * o = W + iw( a, b, 0, NW, i0, i1, i2 );
#pragma unroll
        for( int k = 0; k < NW; ++ k )
            o[ k * ngw ] = wv[ k ];
    }
    // Same-level ghost fill by push: a cell within two cells of a side is a
    // ghost cell of the block across it (faces, edges, corners).  The block
    // that holds this cell's position at i + sh n in its ghost shell is the
    // neighbour in direction -sh, the one whose k_ghost pull in direction sh
    // reads this cell; past a physical side (-1), on another rank (-2, the
    // halo exchange) or across a level jump (-3) nothing is written here.
    // Per axis the shift is +1 within two cells of the low side, -1 of the
    // high side (n >= 4: never both); the targets are the nonempty subsets.
    const int sx = i0 < 2 ? 1 : ( i0 >= a.n0 - 2 ? -1 : 0 );
    const int sy = i1 < 2 ? 1 : ( i1 >= a.n1 - 2 ? -1 : 0 );
    const int sz = i2 < 2 ? 1 : ( i2 >= a.n2 - 2 ? -1 : 0 );
    const int mask = ( sx != 0 ) | ( sy != 0 ) << 1 | ( sz != 0 ) << 2;
    if( mask )
        for( int m = 1; m < 8; ++ m )
        {
            if( m & ~mask )
                continue;
            const int dx = m & 1 ? sx : 0, dy = m & 2 ? sy : 0, dz = m & 4 ? sz : 0;
            const int dst = a.nbr[ b * 27 + ( 1 - dx ) + 3 * ( 1 - dy ) + 9 * ( 1 - dz ) ];
            if( dst < 0 )
                continue;
            R * o = W + iw( a, dst, 0, NW, i0 + dx * a.n0, i1 + dy * a.n1, i2 + dz * a.n2 );
#pragma unroll
            for( int k = 0; k < NW; ++ k )
                o[ k * ngw ] = wv[ k ];
        }
}

// DT: stage 0's launch, which also reduces the CFL dt; stage 1's launch has none
// of that code (fewer registers).
// One CTA's cells: block b, z plane i2, cell c of the (x, y) plane (every
// thread of the CTA calls it: the dt reduction is CTA-wide).
template< bool MHD, class R, bool DT > __device__ __forceinline__
void c2p_cells( const args_t< R > & a, int step, udiv_t dv, int b, int i2, unsigned c )
{
    double dt = FLT_MAX;
    if( c < unsigned( a.n0 * a.n1 ) )
    {
        const unsigned q = udiv_q( c, dv );
        const int i0 = int( c - q * unsigned( a.n0 ) );
        const int i1 = int( q );
        double * U = a.u[ step ];
        double cons[ 5 ], prim[ 5 ];
        for( int k = 0; k < 5; ++ k )
            cons[ k ] = U[ iuc( a, b, k, i0, i1, i2 ) ];
        double b_l[ 3 ], b_r[ 3 ], bc_2[ 3 ], b_max[ 3 ], cs2;
        if( MHD )
        {
            const double * BF = a.bf[ step ];
            const int ii[ 3 ] = { i0, i1, i2 };
            for( int d = 0; d < 3; ++ d )
            {
                int jj[ 3 ] = { ii[ 0 ], ii[ 1 ], ii[ 2 ] };
                b_l[ d ] = BF[ ibf( a, b, d, jj[ 0 ], jj[ 1 ], jj[ 2 ] ) ];
                ++ jj[ d ];
                b_r[ d ] = BF[ ibf( a, b, d, jj[ 0 ], jj[ 1 ], jj[ 2 ] ) ];
            }
        }
        c2p_point< MHD, R >( a, a.w, U, b, i0, i1, i2, cons, b_l, b_r, prim, bc_2, b_max, cs2 );
        if( DT )
        {   // cfl * min_a dx_a / s_a as cfl / max_a ( s_a / dx_a ): one division
            // (the reference divides per axis; rounding differs only); like
            // fmin, fmax drops a NaN candidate
            const geo_t & g = a.geo[ b ];
            double smax = 0;
            if( ! MHD )
            {
                const double cs = sqrt( cs2 );
                for( int d = 0; d < 3; ++ d )
                    smax = fmax( smax, ( cs + fabs( prim[ MOM + d ] ) ) * g.idx[ d ] );
            }
            else
            {
                const double rho_inv = 1 / prim[ RHO ];
                double bm_2[ 3 ] = { bc_2[ 0 ], bc_2[ 1 ], bc_2[ 2 ] };
                for( int d = 0; d < 3; ++ d )
                {
                    bm_2[ d ] = b_max[ d ] * b_max[ d ];
                    const double cf = c_fms_ri< double >( prim, bm_2, a.gamma, d, rho_inv );
                    smax = fmax( smax, ( cf + fabs( prim[ MOM + d ] ) ) * g.idx[ d ] );
                    bm_2[ d ] = bc_2[ d ];
                }
            }
            dt = smax > 0 ? a.cfl / smax : FLT_MAX;
            // fmax drops a NaN speed, so a NaN velocity would leave dt finite:
            // flag it in the status word (bit 1) instead
            if( isnan( prim[ MOM ] + prim[ MOM + 1 ] + prim[ MOM + 2 ] ) )
                dt = -1;
        }
    }
    if( DT )
    {
        __shared__ double red[ 8 ];
        if( __any_sync( 0xffffffffu, dt < 0 ) )
        {
            if( ( threadIdx.x & 31 ) == 0 )
                atomicOr( & a.s[ 0 ].status, 2 );
            dt = dt < 0 ? FLT_MAX : dt;
        }
        dt = warp_min( dt );
        if( ( threadIdx.x & 31 ) == 0 )
            red[ threadIdx.x >> 5 ] = dt;
        __syncthreads(  );
        if( threadIdx.x < 32 )
        {
            dt = threadIdx.x < ( blockDim.x >> 5 ) ? red[ threadIdx.x ] : FLT_MAX;
            dt = warp_min( dt );
            if( threadIdx.x == 0 )
                atomicMin( & a.s[ a.boxes ? b : 0 ].dt_bits, ( unsigned long long ) __double_as_longlong( dt ) );
        }
    }
}

template< bool MHD, class R, bool DT >
__global__ void __launch_bounds__( 256, ( MHD && DT ) ? 3 : 4 ) k_c2p( const args_t< R > a, int step, udiv_t dv )
{
    // grid: x over the cells of one (x, y) plane, y over z, z over blocks
    c2p_cells< MHD, R, DT >( a, step, dv, blockIdx.z, blockIdx.y, blockIdx.x * blockDim.x + threadIdx.x );
}

////////////////////////////////////////////////////////////
// Ghost fill between same-level blocks: every ghost cell of W and every
// non-owned slot of BF takes the value held by the block that owns it.

__device__ __forceinline__ int wrap_axis( int i, int n, int & sh )
{
    if( i < 0 )  { sh = -1; return i + n; }
    if( i >= n ) { sh = +1; return i - n; }
    sh = 0;
    return i;
}

// Site t of the ghost shell [-g, n+g)^3 \ [0, n)^3, enumerated as z slabs, then
// y slabs (interior z), then x slabs (interior y, z).
__device__ __forceinline__ void shell_site( long long t, int n0, int n1, int n2, int g,
                                            int & i0, int & i1, int & i2 )
{
    const int e0 = n0 + 2 * g, e1 = n1 + 2 * g, l2 = 2 * g;
    const long long zs = ( long long ) l2 * e0 * e1;
    if( t < zs )
    {
        i0 = int( t % e0 ) - g;
        i1 = int( ( t / e0 ) % e1 ) - g;
        const int l = int( t / ( ( long long ) e0 * e1 ) );
        i2 = l < g ? l - g : n2 + l - g;
        return;
    }
    t -= zs;
    const long long ys = ( long long ) l2 * e0 * n2;
    if( t < ys )
    {
        i0 = int( t % e0 ) - g;
        const int l = int( ( t / e0 ) % l2 );
        i2 = int( t / ( ( long long ) e0 * l2 ) );
        i1 = l < g ? l - g : n1 + l - g;
        return;
    }
    t -= ys;
    const int l = int( t % l2 );
    i1 = int( ( t / l2 ) % n1 );
    i2 = int( t / ( ( long long ) l2 * n1 ) );
    i0 = l < g ? l - g : n0 + l - g;
}

__host__ __device__ __forceinline__ long long shell_count( int n0, int n1, int n2, int g )
{
    return ( long long ) 2 * g * ( ( long long )( n0 + 2 * g ) * ( n1 + 2 * g )
                                 + ( long long )( n0 + 2 * g ) * n2 + ( long long ) n1 * n2 );
}

// Face-B ghost slots the flux sweeps read: component c on its own faces
// (0..n_c) at the first transverse ghost line (-1 or n) of one transverse axis.
__host__ __device__ __forceinline__ long long bf_strip_count( int n0, int n1, int n2 )
{
    const int nn[ 3 ] = { n0, n1, n2 };
    long long s = 0;
    for( int c = 0; c < 3; ++ c )
        s += 2LL * ( nn[ c ] + 1 ) * ( nn[ ( c + 1 ) % 3 ] + nn[ ( c + 2 ) % 3 ] );
    return s;
}

// Divisors of the shell and strip enumerations (multiply-high quotients).
struct ghost_div_t { udiv_t e0, e1, n1, f[ 3 ]; };

static ghost_div_t make_ghost_div( const int * n )
{
    ghost_div_t g;
    g.e0 = make_udiv( unsigned( n[ 0 ] + 4 ) );
    g.e1 = make_udiv( unsigned( n[ 1 ] + 4 ) );
    g.n1 = make_udiv( unsigned( n[ 1 ] ) );
    for( int c = 0; c < 3; ++ c )
        g.f[ c ] = make_udiv( unsigned( n[ c ] + 1 ) );
    return g;
}

template< bool MHD, class R >
__global__ void __launch_bounds__( 256 ) k_ghost( const args_t< R > a, int step, ghost_div_t gd )
{
    constexpr int NW = MHD ? 11 : 5;   // stored W words: prim (8) + cell E (3)
    const int b = blockIdx.y;
    unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
    const int e0 = a.n0 + 4, e1 = a.n1 + 4;
    const unsigned zs = 4u * e0 * e1, ys = 4u * e0 * a.n2, xs = 4u * a.n1 * a.n2;
    if( t < zs + ys + xs )
    {   // shell [-2, n+2)^3 \ [0, n)^3: z slabs, y slabs (interior z), x slabs
        int i0, i1, i2;
        if( t < zs )
        {
            const unsigned q = udiv_q( t, gd.e0 ), q2 = udiv_q( q, gd.e1 );
            i0 = int( t - q * e0 ) - 2;
            i1 = int( q - q2 * e1 ) - 2;
            i2 = q2 < 2 ? int( q2 ) - 2 : a.n2 + int( q2 ) - 2;
        }
        else if( ( t -= zs ) < ys )
        {
            const unsigned q = udiv_q( t, gd.e0 ), l = q & 3u;
            i0 = int( t - q * e0 ) - 2;
            i2 = int( q >> 2 );
            i1 = l < 2 ? int( l ) - 2 : a.n1 + int( l ) - 2;
        }
        else
        {
            t -= ys;
            const unsigned l = t & 3u, q = t >> 2, q2 = udiv_q( q, gd.n1 );
            i1 = int( q - q2 * a.n1 );
            i2 = int( q2 );
            i0 = l < 2 ? int( l ) - 2 : a.n0 + int( l ) - 2;
        }
        int s0, s1, s2;
        const int j0 = wrap_axis( i0, a.n0, s0 );
        const int j1 = wrap_axis( i1, a.n1, s1 );
        const int j2 = wrap_axis( i2, a.n2, s2 );
        const int src = a.nbr[ b * 27 + ( s0 + 1 ) + 3 * ( s1 + 1 ) + 9 * ( s2 + 1 ) ];
        if( src < 0 )
            return;                              // physical side or another rank
        const int ngw = int( a.ngw );
        R * dst = a.w + ( size_t ) b * NW * a.ngw + ( ( i0 + 2 ) + a.sw1 * ( i1 + 2 ) + a.sw2 * ( i2 + 2 ) );
        const R * srcp = a.w + ( size_t ) src * NW * a.ngw + ( ( j0 + 2 ) + a.sw1 * ( j1 + 2 ) + a.sw2 * ( j2 + 2 ) );
        R v[ NW ];
        for( int k = 0; k < NW; ++ k )
            v[ k ] = srcp[ k * ngw ];
        for( int k = 0; k < NW; ++ k )
            dst[ k * ngw ] = v[ k ];
        return;
    }
    if( ! MHD )
        return;
    t -= zs + ys + xs;
    const int nn[ 3 ] = { a.n0, a.n1, a.n2 };
    for( int c = 0; c < 3; ++ c )
    {
        const int a1 = ( c + 1 ) % 3, a2 = ( c + 2 ) % 3;
        const unsigned cnt = 2u * ( nn[ c ] + 1 ) * ( nn[ a1 ] + nn[ a2 ] );
        if( t >= cnt )
        {
            t -= cnt;
            continue;
        }
        // t -> (face index along c, side, transverse position along the other axis)
        const unsigned q = udiv_q( t, gd.f[ c ] );
        const int fc = int( t - q * unsigned( nn[ c ] + 1 ) );
        const int side = int( q & 1u );
        const int r = int( q >> 1 );
        int ii[ 3 ];
        ii[ c ] = fc;
        if( r < nn[ a2 ] )
        {   // ghost line along a1
            ii[ a1 ] = side ? nn[ a1 ] : -1;
            ii[ a2 ] = r;
        }
        else
        {
            ii[ a2 ] = side ? nn[ a2 ] : -1;
            ii[ a1 ] = r - nn[ a2 ];
        }
        int sh[ 3 ] = { 0, 0, 0 }, jj[ 3 ] = { ii[ 0 ], ii[ 1 ], ii[ 2 ] };
        for( int d = 0; d < 3; ++ d )
            if( d != c )
                jj[ d ] = wrap_axis( ii[ d ], nn[ d ], sh[ d ] );
        const int src = a.nbr[ b * 27 + ( sh[ 0 ] + 1 ) + 3 * ( sh[ 1 ] + 1 ) + 9 * ( sh[ 2 ] + 1 ) ];
        if( src < 0 )
            return;
        double * BF = a.bf[ step ];
        BF[ ibf( a, b, c, ii[ 0 ], ii[ 1 ], ii[ 2 ] ) ] = BF[ ibf( a, src, c, jj[ 0 ], jj[ 1 ], jj[ 2 ] ) ];
        return;
    }
}

////////////////////////////////////////////////////////////
// Physical boundaries on the primitives (hydro/boundary/phys.h:95-139,
// phys_functors.h:11-91).  One thread per transverse interior position of a
// domain-edge side of a block: the two cells next to the boundary (index 0 =
// adjacent) feed the two ghost cells.  Hydro only.

template< class R >
__global__ void __launch_bounds__( 128 ) k_phys( const args_t< R > a )
{
    const int b = blockIdx.z, side = blockIdx.y;
    const int axis = side >> 1, right = side & 1;
    const int kind = a.bc[ side ];
    if( ! ( ( a.geo[ b ].phys >> side ) & 1 ) )
        return;                              // periodic, or not on this domain side
    const int nn[ 3 ] = { a.n0, a.n1, a.n2 };
    const int a1 = mod3( axis + 1 ), a2 = mod3( axis + 2 );
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if( t >= nn[ a1 ] * nn[ a2 ] )
        return;
    int ii[ 3 ];
    ii[ a1 ] = t % nn[ a1 ];
    ii[ a2 ] = t / nn[ a1 ];
    const int i_mom = MOM + axis;
    R c0[ 5 ], c1[ 5 ];
    ii[ axis ] = right ? nn[ axis ] - 1 : 0;
    for( int k = 0; k < 5; ++ k ) c0[ k ] = a.w[ iw( a, b, k, 5, ii[ 0 ], ii[ 1 ], ii[ 2 ] ) ];
    ii[ axis ] = right ? nn[ axis ] - 2 : 1;
    for( int k = 0; k < 5; ++ k ) c1[ k ] = a.w[ iw( a, b, k, 5, ii[ 0 ], ii[ 1 ], ii[ 2 ] ) ];
    if( kind == KR_BC_OUT && c0[ i_mom ] * R( right ? -1 : 1 ) > 0 )
        c0[ i_mom ] = 0;                     // no inflow through an outflow side
    for( int g = 1; g <= 2; ++ g )           // ghost g: -g (left) or n - 1 + g (right)
    {
        ii[ axis ] = right ? nn[ axis ] - 1 + g : -g;
        for( int k = 0; k < 5; ++ k )
        {
            R v;
            if( kind == KR_BC_REF )
                v = ( g == 1 ? c0[ k ] : c1[ k ] ) * R( k == i_mom ? -1 : 1 );
            else if( kind == KR_BC_FIXD )
                v = R( a.w_fix[ k ] );
            else
                v = c0[ k ];                 // outflow, free: zero gradient
            a.w[ iw( a, b, k, 5, ii[ 0 ], ii[ 1 ], ii[ 2 ] ) ] = v;
        }
    }
}

////////////////////////////////////////////////////////////
// Static refinement, hydro (hydro/boundary/comm_functions.h:329-505,
// keeper.cpp:148-166): ghost cells across a level jump and the coarse side's
// face flux.  Arithmetic in FP64 from the stored words, in the reference's
// order; one item per (coarse block, face, fine child) or (fine block, face).

__device__ __forceinline__ void smr_axes( int face, int & ax, int & a1, int & a2, int & s )
{
    ax = face >> 1; s = face & 1; a1 = mod3( ax + 1 ); a2 = mod3( ax + 2 );
}

// to_coarser: each of the 2 ghost layers x (n1/2) x (n2/2) coarse cells that a
// fine child covers is the volume average of its 8 fine cells, accumulated
// fine layer by layer, (d1, d2) with d1 outer.
template< class R >
__global__ void __launch_bounds__( 128 ) k_restrict( const args_t< R > a, const smr_item_t * items )
{
    const smr_item_t it = items[ blockIdx.y ];
    int ax, a1, a2, s;
    smr_axes( it.face, ax, a1, a2, s );
    const int nn[ 3 ] = { a.n0, a.n1, a.n2 };
    const int h1 = nn[ a1 ] >> 1, h2 = nn[ a2 ] >> 1;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if( t >= 2 * h1 * h2 )
        return;
    const int t1 = t % h1, t2 = ( t / h1 ) % h2, gl = t / ( h1 * h2 );
    const double dv = a.geo[ it.src ].vol;
    double p[ 5 ] = { 0, 0, 0, 0, 0 }, norm = 0;
    for( int kk = 0; kk < 2; ++ kk )
        for( int e1 = 0; e1 < 2; ++ e1 )
            for( int e2 = 0; e2 < 2; ++ e2 )
            {
                const int k = 2 * gl + kk;
                int jj[ 3 ];
                jj[ ax ] = s ? k : nn[ ax ] - 4 + k;
                jj[ a1 ] = 2 * t1 + e1;
                jj[ a2 ] = 2 * t2 + e2;
                for( int c = 0; c < 5; ++ c )
                    p[ c ] += double( a.w[ iw( a, it.src, c, 5, jj[ 0 ], jj[ 1 ], jj[ 2 ] ) ] ) * dv;
                norm += dv;
            }
    int ii[ 3 ];
    ii[ ax ] = s ? nn[ ax ] + gl : gl - 2;
    ii[ a1 ] = it.o1 + t1;
    ii[ a2 ] = it.o2 + t2;
    for( int c = 0; c < 5; ++ c )
        a.w[ iw( a, it.dst, c, 5, ii[ 0 ], ii[ 1 ], ii[ 2 ] ) ] = R( p[ c ] / norm );
}

__device__ __forceinline__ double minmod( double x, double y )
{   // utilities/functions.h:159-170
    return ( ( x < 0 ) ^ ( y < 0 ) ) ? 0. : ( fabs( x ) < fabs( y ) ? x : y );
}

// to_finer: every coarse cell next to the face gives its 2 x 2 x 2 fine ghost
// cells q_c + sum over the axes (normal, (a+1)%3, (a+2)%3) of
// +-minmod(q_r - q_c, q_c - q_l) / 4.  Reads the coarse block's ghosts, so it
// runs after the restriction, the same-level fill and the physical sides.
template< class R >
__global__ void __launch_bounds__( 128 ) k_prolong( const args_t< R > a, const smr_item_t * items )
{
    const smr_item_t it = items[ blockIdx.y ];
    int ax, a1, a2, s;
    smr_axes( it.face, ax, a1, a2, s );
    const int nn[ 3 ] = { a.n0, a.n1, a.n2 };
    const int h1 = nn[ a1 ] >> 1, h2 = nn[ a2 ] >> 1;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if( t >= h1 * h2 )
        return;
    const int t1 = t % h1, t2 = t / h1;
    int jc[ 3 ];
    jc[ ax ] = s ? 0 : nn[ ax ] - 1;
    jc[ a1 ] = it.o1 + t1;
    jc[ a2 ] = it.o2 + t2;
    for( int c = 0; c < 5; ++ c )
    {
        const double qc = double( a.w[ iw( a, it.src, c, 5, jc[ 0 ], jc[ 1 ], jc[ 2 ] ) ] );
        double dq[ 3 ];
        for( int d = 0; d < 3; ++ d )
        {
            int jr[ 3 ] = { jc[ 0 ], jc[ 1 ], jc[ 2 ] }, jl[ 3 ] = { jc[ 0 ], jc[ 1 ], jc[ 2 ] };
            ++ jr[ d ];
            -- jl[ d ];
            const double qr = double( a.w[ iw( a, it.src, c, 5, jr[ 0 ], jr[ 1 ], jr[ 2 ] ) ] );
            const double ql = double( a.w[ iw( a, it.src, c, 5, jl[ 0 ], jl[ 1 ], jl[ 2 ] ) ] );
            dq[ d ] = minmod( qr - qc, qc - ql ) * 0.25;
        }
        for( int k = 0; k < 2; ++ k )
            for( int e1 = 0; e1 < 2; ++ e1 )
                for( int e2 = 0; e2 < 2; ++ e2 )
                {
                    int ii[ 3 ];
                    ii[ ax ] = s ? nn[ ax ] + k : k - 2;
                    ii[ a1 ] = 2 * t1 + e1;
                    ii[ a2 ] = 2 * t2 + e2;
                    const double q = qc + dq[ ax ] * double( 2 * ( k & 1 ) - 1 )
                                   + dq[ a1 ] * double( 2 * e1 - 1 )
                                   + dq[ a2 ] * double( 2 * e2 - 1 );
                    a.w[ iw( a, it.dst, c, 5, ii[ 0 ], ii[ 1 ], ii[ 2 ] ) ] = R( q );
                }
    }
}

// flux_to_buf / flux_from_buf: the coarse face flux over a refined side is the
// area average of the 4 fine face fluxes it covers ((d1, d2), d1 outer).  Kept
// in FP64 (a.favg) in both precisions, so the coarse correction carries the
// fine fluxes without a rounding to the flux word type.
template< class R, int NF = 5 >        // NF: flux words per face (5 hydro, 7 MHD)
__global__ void __launch_bounds__( 128 ) k_flux_avg( const args_t< R > a, const smr_item_t * items )
{
    const smr_item_t it = items[ blockIdx.y ];
    int ax, a1, a2, s;
    smr_axes( it.face, ax, a1, a2, s );
    const int nn[ 3 ] = { a.n0, a.n1, a.n2 };
    const int h1 = nn[ a1 ] >> 1, h2 = nn[ a2 ] >> 1;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if( t >= h1 * h2 )
        return;
    const int t1 = t % h1, t2 = t / h1;
    const double ds = a.geo[ it.src ].sfc[ ax ];
    double acc[ 5 ] = { 0, 0, 0, 0, 0 }, norm = 0;
    for( int e1 = 0; e1 < 2; ++ e1 )
        for( int e2 = 0; e2 < 2; ++ e2 )
        {
            int jj[ 3 ];
            jj[ ax ] = s ? 0 : nn[ ax ];
            jj[ a1 ] = 2 * t1 + e1;
            jj[ a2 ] = 2 * t2 + e2;
            for( int c = 0; c < 5; ++ c )
                acc[ c ] += double( a.f[ ax ][ ifx( a, it.src, c, NF, jj[ 0 ], jj[ 1 ], jj[ 2 ] ) ] ) * ds;
            norm += ds;
        }
    for( int c = 0; c < 5; ++ c )
        a.favg[ ( ( size_t ) blockIdx.y * 5 + c ) * a.favg_n + t ] = acc[ c ] / norm;
}

////////////////////////////////////////////////////////////
// MHD physical boundaries (mhd/boundary/phys.h:118-250, phys_functors.h:9-132).
// One launch per non-periodic side (sides in order, so cells shared by two
// sides take the later side's values); one thread per transverse row of the
// ghost shell, ghost rows included.  The source row is clamped into the
// interior only along transverse axes that end at a physical side there; the
// three cells (primitives, cell-centred B) and faces (normal B on the face
// lattice, tangential B on the cell lattice) next to the boundary go through
// the functor into the two ghost layers.  The ghost cells' E = B x v is
// stored with them, as the edge EMF reads it (integrator.h:201-213).  Runs
// after the same-level fill: the reference also runs it once before, with
// face B, but those values from not-yet-filled rows land only in ghost-shell
// corner slots that no stencil reads.

// field: 1 writes the face B of the ghost layers too, 0 the primitives only
// (the second pass of a refined mesh's exchange, phys.h:199-249 step < 0).
template< class R >
__global__ void __launch_bounds__( 128 ) k_phys_mhd( const args_t< R > a, int side, int step, int field = 1 )
{
    const int b = blockIdx.y;
    const int axis = side >> 1, right = side & 1;
    const int kind = a.bc[ side ];
    const int ph = a.geo[ b ].phys;          // bit 2d+s: side (d, s) is a domain side here
    if( ! ( ( ph >> side ) & 1 ) )
        return;
    const int nn[ 3 ] = { a.n0, a.n1, a.n2 };
    const int a1 = mod3( axis + 1 ), a2 = mod3( axis + 2 );
    const int e1 = nn[ a1 ] + 4;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if( t >= e1 * ( nn[ a2 ] + 4 ) )
        return;
    int i_tgt[ 3 ], i_src[ 3 ], i_sfc[ 3 ];
    i_tgt[ a1 ] = t % e1 - 2;
    i_tgt[ a2 ] = t / e1 - 2;
    for( int h = 0; h < 2; ++ h )
    {
        const int d = h ? a2 : a1;
        int r = i_tgt[ d ], f = i_tgt[ d ];
        if( ( ph >> ( 2 * d ) ) & 1 )
        {   r = max( r, 0 ); f = max( f, 0 ); }
        if( ( ph >> ( 2 * d + 1 ) ) & 1 )
        {   r = min( r, nn[ d ] - 1 ); f = min( f, nn[ d ] ); }
        i_src[ d ] = r;
        i_sfc[ d ] = f;
    }
    const int n = nn[ axis ];
    const double * BF = a.bf[ step ];
    R hyd[ 5 ][ 8 ], bc[ 5 ][ 3 ];          // index i + 2, i = -2..2
    double bfb[ 5 ][ 3 ];
    for( int i = 0; i <= 2; ++ i )
    {
        i_src[ axis ] = right ? n - i - 1 : i;
        i_sfc[ axis ] = right ? n - i : i;
        for( int k = 0; k < 8; ++ k )
            hyd[ 2 + i ][ k ] = a.w[ iw( a, b, k, 11, i_src[ 0 ], i_src[ 1 ], i_src[ 2 ] ) ];
        for( int q = 0; q < 3; ++ q )
        {
            bc[ 2 + i ][ q ] = hyd[ 2 + i ][ BCC + q ];
            bfb[ 2 + i ][ q ] = q == axis ? BF[ ibf( a, b, q, i_sfc[ 0 ], i_sfc[ 1 ], i_sfc[ 2 ] ) ]
                                          : BF[ ibf( a, b, q, i_src[ 0 ], i_src[ 1 ], i_src[ 2 ] ) ];
        }
    }
    const int i_mom = MOM + axis;
    if( kind == KR_BC_OUT && hyd[ 2 ][ i_mom ] * R( right ? -1 : 1 ) > 0 )
        hyd[ 2 ][ i_mom ] = 0;                   // no inflow through an outflow side
    for( int i = -2; i < 0; ++ i )
    {
        for( int k = 0; k < 8; ++ k )
        {
            if( kind == KR_BC_REF )
                hyd[ 2 + i ][ k ] = hyd[ 2 - i - 1 ][ k ] * R( k == i_mom ? -1 : 1 );
            else if( kind == KR_BC_FIXD )
                hyd[ 2 + i ][ k ] = R( k < 5 ? a.w_fix[ k ] : a.b_fix[ k - 5 ] );
            else
                hyd[ 2 + i ][ k ] = hyd[ 2 ][ k ];
        }
        for( int q = 0; q < 3; ++ q )
        {
            if( kind == KR_BC_REF )
            {   // faces mirror at -i, cells at -i-1; tangential components flip
                bfb[ 2 + i ][ q ] = ( q != axis ? -1. : 1. ) * bfb[ 2 - i ][ q ];
                bc [ 2 + i ][ q ] = R( q != axis ? -1 : 1 ) * bc[ 2 - i - 1 ][ q ];
            }
            else if( kind == KR_BC_FIXD )
            {
                bfb[ 2 + i ][ q ] = a.b_fix[ q ];
                bc [ 2 + i ][ q ] = R( a.b_fix[ q ] );
            }
            else
            {
                bfb[ 2 + i ][ q ] = bfb[ 2 ][ q ];
                bc [ 2 + i ][ q ] = bc [ 2 ][ q ];
            }
        }
    }
    double * BFw = a.bf[ step ];
    for( int i = -2; i < 0; ++ i )
    {
        i_tgt[ axis ] = right ? n - i - 1 : i;
        int i_fbc[ 3 ] = { i_tgt[ 0 ], i_tgt[ 1 ], i_tgt[ 2 ] };
        i_fbc[ axis ] = right ? n - i : i;
        R * p = hyd[ 2 + i ];
        for( int q = 0; q < 3; ++ q )
            p[ BCC + q ] = bc[ 2 + i ][ q ];
        for( int k = 0; k < 8; ++ k )
            a.w[ iw( a, b, k, 11, i_tgt[ 0 ], i_tgt[ 1 ], i_tgt[ 2 ] ) ] = p[ k ];
        for( int d = 0; d < 3; ++ d )
        {
            const int d1 = mod3( d + 1 ), d2 = mod3( d + 2 );
            a.w[ iw( a, b, 8 + d, 11, i_tgt[ 0 ], i_tgt[ 1 ], i_tgt[ 2 ] ) ] =
                p[ BCC + d1 ] * p[ MOM + d2 ] - p[ BCC + d2 ] * p[ MOM + d1 ];
        }
        for( int q = 0; q < 3 && field; ++ q )
        {
            if( q == axis )
                BFw[ ibf( a, b, q, i_fbc[ 0 ], i_fbc[ 1 ], i_fbc[ 2 ] ) ] = bfb[ 2 + i ][ q ];
            else
                BFw[ ibf( a, b, q, i_tgt[ 0 ], i_tgt[ 1 ], i_tgt[ 2 ] ) ] = bfb[ 2 + i ][ q ];
        }
    }
}

////////////////////////////////////////////////////////////
// Face fluxes along one axis: PLM + HLLC / HLLD / HLLE per face.
// One thread per face; consecutive threads take consecutive x.  MHD also covers
// the transverse ghost lines that the corner EMF reads
// (mhd/integrator/integrator.h:138-168, mhd/integrator/data.h:106-144).

// MODE: KR_RIEMANN_DEFAULT, KR_RIEMANN_HLLE, KR_RIEMANN_LEARNED, or FLUX_SAMPLE
// (HLLD step that also logs selector training samples).  Compile-time, so the
// plain step carries none of the selector's registers.
constexpr int FLUX_SAMPLE = 3;
// Learned mode, the sweeps without the network: each warp of faces runs the
// solver the last evaluation chose for it.
constexpr int FLUX_APPLY = 4;

// Riemann solve of one face from its reconstructed states and store of the
// flux (and, for MHD, the two edge EMFs: hlld.h:42-46 -- slot 5 holds
// E_{(axis+1)%3}, slot 6 E_{(axis+2)%3}).  (The learned mode goes through
// learned_solve below.)
template< bool MHD, class R, int MODE > __device__ __forceinline__
void solve_store( const args_t< R > & a, int b, int axis, const int * ii, bool valid,
                  R * ql, R * qr, int warp, unsigned long long key, bool cheap = false )
{
    constexpr bool SAMPLE = MODE == FLUX_SAMPLE;
    constexpr int rsel = MODE == FLUX_SAMPLE ? KR_RIEMANN_DEFAULT : MODE;
    constexpr int NF = MHD ? 7 : 5;
    R flx[ 8 ];
    const eos_c< R > e = { R( a.gamma ), R( a.gm1 ), R( a.cv ) };
    if( ! valid )
        for( int k = 0; k < 8; ++ k )
            ql[ k ] = qr[ k ] = ( k == RHO || k == ENE ) ? R( 1 ) : R( 0 );
    idx_swap( ql + MOM, axis );
    idx_swap( qr + MOM, axis );
    if( ! MHD )
    {
        if( ! valid ) return;
        hllc_fast< R >( flx, ql, qr, e );
    }
    else
    {
        idx_swap( ql + BCC, axis );
        idx_swap( qr + BCC, axis );
        if( ! valid ) return;
        if( rsel == KR_RIEMANN_HLLE )
            hlle_fast< R >( flx, ql, qr, e );
        else if( MODE == FLUX_APPLY )      // learned mode: this warp's choice
            hll_pick_fast< R >( flx, ql, qr, e, cheap );
        else
            hlld_fast< R >( flx, ql, qr, e );
        if constexpr( SAMPLE )
        {   // training sample: features, and the HLLE-HLLD gap of this face
            key = ( key + a.smp_seed ) * 0xBF58476D1CE4E5B9ull;
            if( ( unsigned )( ( key ^ ( key >> 29 ) ) % a.smp_stride ) == 0 )
            {
                R fe[ 8 ], fd[ 8 ];
                hlle_fast< R >( fe, ql, qr, e );
                hlld_fast< R >( fd, ql, qr, e );
                const unsigned long long slot = atomicAdd( a.smp_n, 1ull );
                if( ( long long ) slot < a.smp_max )
                {
                    float f[ MLP_IN ];
                    face_features< R >( ql, qr, e.gamma, f );
                    float * o = a.smp + slot * ( MLP_IN + 1 );
                    for( int k = 0; k < MLP_IN; ++ k ) o[ k ] = f[ k ];
                    o[ MLP_IN ] = flux_gap< R >( fe, fd, ql, qr, e.gamma );
                }
            }
        }
    }
    idx_swap( flx + MOM, 3 - axis );
    // block base once in 64 bits, offsets inside the block in 32
    R * F = a.f[ axis ] + ( size_t ) b * NF * a.nfb;
    const int off = ( ii[ 0 ] + 1 ) + a.sf1 * ( ii[ 1 ] + 1 ) + a.sf2 * ( ii[ 2 ] + 1 );
    const int nfb = int( a.nfb );
    for( int k = 0; k < 5; ++ k )
        F[ k * nfb + off ] = flx[ k ];
    if( MHD )
    {
        F[ 5 * nfb + off ] =  flx[ BCC + 2 ];
        F[ 6 * nfb + off ] = -flx[ BCC + 1 ];
    }
}

// One thread per face: every face of the sweep, the MHD transverse ghost lines
// included (mhd/integrator/integrator.h:138-168).
// Learned mode (no reference counterpart).  The network runs at stage 0 of
// every sel_period-th step (and the step after new weights): this sweep
// evaluates it for every face.  A face that only this block computes follows
// its warp: the warp's such faces go to HLLE together, only when the network
// passes every one of them (a face it flags keeps them all on HLLD), so most
// warps run one solver.  A face that more than one block computes -- on a
// block side along the sweep, or within one cell of a transverse side, where
// the neighbours' ghost lines (the edge EMFs' inputs) hold it too -- follows
// its own logit instead: every block that computes it reconstructs the same
// states from the same (ghost-copied) primitives and so takes the same
// decision, and the face gets one flux, so the update keeps telescoping.
// The choice is kept as one 32-bit mask per warp (sel_dec, wid: the warp's
// number in the sweep's chunk order), which the other sweeps of the period
// read (FLUX_APPLY) on the same face grid.
template< bool MHD, class R > __device__ __forceinline__
void learned_solve( const args_t< R > & a, int b, int axis, const int * ii, bool valid,
                    R * ql, R * qr, unsigned wid )
{
    constexpr int NF = 7;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const eos_c< R > e = { R( a.gamma ), R( a.gm1 ), R( a.cv ) };
    if( ! valid )
        for( int k = 0; k < 8; ++ k )
            ql[ k ] = qr[ k ] = ( k == RHO || k == ENE ) ? R( 1 ) : R( 0 );
    idx_swap( ql + MOM, axis ); idx_swap( qr + MOM, axis );
    idx_swap( ql + BCC, axis ); idx_swap( qr + BCC, axis );
    __shared__ __nv_bfloat16 xs[ 4 ][ 32 * MLP_IN ];
    // the network: every lane of the warp takes part in the MMAs
    float f[ MLP_IN ];
    face_features< R >( ql, qr, e.gamma, f );
    const float z = mlp_logit( f, a.sel_w, a.sel_b, xs[ warp ] );
    // faces that a neighbouring block computes too (see above)
    const int nn[ 3 ] = { a.n0, a.n1, a.n2 };
    const int a1 = mod3( axis + 1 ), a2 = mod3( axis + 2 );
    const bool shared = ii[ axis ] == 0 || ii[ axis ] == nn[ axis ]
                     || ii[ a1 ] <= 0 || ii[ a1 ] >= nn[ a1 ] - 1
                     || ii[ a2 ] <= 0 || ii[ a2 ] >= nn[ a2 ] - 1;
    const bool pass = z > a.sel_thr;
    const unsigned mv = __ballot_sync( 0xffffffffu, valid && ! shared );
    const unsigned mc = __ballot_sync( 0xffffffffu, valid && ! shared && pass );
    const bool cheap = shared ? pass : ( mv != 0u && mc == mv );
    const unsigned mask = __ballot_sync( 0xffffffffu, valid && cheap );
    const unsigned mvalid = __ballot_sync( 0xffffffffu, valid );
    if( lane == 0 )
    {
        a.sel_dec[ ( ( size_t ) axis * a.nblk + b ) * a.sel_wcap + wid ] = mask;
        if( mvalid )
        {
            atomicAdd( a.sel_cnt, ( unsigned long long ) __popc( mvalid ) );
            if( mask )
                atomicAdd( a.sel_cnt + 1, ( unsigned long long ) __popc( mask ) );
        }
    }
    if( ! valid )
        return;
    R flx[ 8 ];
    hll_pick_fast< R >( flx, ql, qr, e, cheap );
    idx_swap( flx + MOM, 3 - axis );
    R * F = a.f[ axis ] + ( size_t ) b * NF * a.nfb;
    const int off = ( ii[ 0 ] + 1 ) + a.sf1 * ( ii[ 1 ] + 1 ) + a.sf2 * ( ii[ 2 ] + 1 );
    const int nfb = int( a.nfb );
    for( int k = 0; k < 5; ++ k )
        F[ k * nfb + off ] = flx[ k ];
    F[ 5 * nfb + off ] =  flx[ BCC + 2 ];
    F[ 6 * nfb + off ] = -flx[ BCC + 1 ];
}

// Resident CTAs per SM the per-face sweep is compiled for: register budgets
// that ptxas meets without spilling (FP32 default / HLLE: 64 registers, 8 CTAs;
// learned with the network: 6; FP64: 4).  The learned sweep without the network
// holds both solvers: at 64 registers it spills 12 bytes and still ran 0.5%
// faster per step than at 72 (7 CTAs).
template< class R, int MODE > constexpr int flux_min_ctas(  )
{
    return sizeof( R ) == 4 ? ( ( MODE <= KR_RIEMANN_HLLE || MODE == FLUX_APPLY ) ? 8
                                : ( MODE == KR_RIEMANN_LEARNED ? 6 : 4 ) )
                            : ( MODE == KR_RIEMANN_HLLE ? 5 : 4 );
}

// PLM of the NP primitive words of one face from the four cells around it
// (wb: the right cell's first word, st: stride along the sweep, ngw: word
// stride); the normal B of an MHD face comes from the face lattice instead.
// FP32: words k and k + NP / 2 in pairs (plm_face_fast2).
// The normal B of a face for the reconstruction: the face lattice's value;
// on a refined MHD mesh, along a transverse ghost line next to a side whose
// neighbours are on another level, the cell-centred B of the cell above the
// face instead (mhd/integrator/data.h:98-130 load_primative; no holder
// carries face B onto those lines).  wb: that cell's first W word.
template< class R, bool XL > __device__ __forceinline__
R normal_b( const args_t< R > & a, int b, int axis, int step, const int * ii, const R * wb )
{
    if constexpr( XL )
    {
        const int nn[ 3 ] = { a.n0, a.n1, a.n2 };
        const int x = a.geo[ b ].xlev;
        bool cross = false;
        for( int q = 1; q <= 2; ++ q )
        {
            const int t = mod3( axis + q );
            if( ii[ t ] < 0 )
                cross |= ( x >> ( 2 * t ) ) & 1;
            else if( ii[ t ] >= nn[ t ] )
                cross |= ( x >> ( 2 * t + 1 ) ) & 1;
        }
        if( cross )
            return wb[ ( BCC + axis ) * a.ngw ];
    }
    return R( a.bf[ step ][ ibf( a, b, axis, ii[ 0 ], ii[ 1 ], ii[ 2 ] ) ] );
}

template< bool MHD, class R, bool XL = false > __device__ __forceinline__
void plm_stencil( const args_t< R > & a, int b, int axis, int step, const int * ii, const R * wb,
                  int st, R * ql, R * qr )
{
    constexpr int NP = MHD ? 8 : 5;
    const int ngw = int( a.ngw );
    if( a.vl2 && step == 0 )
    {   // VL2 predictor: piecewise-constant (donor-cell) states
        for( int k = 0; k < NP; ++ k )
        {
            const R * p = wb + k * ngw;
            ql[ k ] = p[ -st ];
            qr[ k ] = p[ 0 ];
        }
        if constexpr( MHD )
            ql[ BCC + axis ] = qr[ BCC + axis ] = normal_b< R, XL >( a, b, axis, step, ii, wb );
        return;
    }
    if constexpr( sizeof( R ) == 4 )
    {
        constexpr int H = NP / 2;
        for( int k = 0; k < H; ++ k )
        {
            const R * p = wb + k * ngw, * p2 = wb + ( k + H ) * ngw;
            float2 l2, r2;
            plm_face_fast2( make_float2( p[ -2 * st ], p2[ -2 * st ] ), make_float2( p[ -st ], p2[ -st ] ),
                            make_float2( p[ 0 ], p2[ 0 ] ), make_float2( p[ st ], p2[ st ] ), l2, r2 );
            ql[ k ] = l2.x; ql[ k + H ] = l2.y;
            qr[ k ] = r2.x; qr[ k + H ] = r2.y;
        }
        if constexpr( NP % 2 )
        {
            const R * p = wb + ( NP - 1 ) * ngw;
            plm_face_fast< R >( p[ -2 * st ], p[ -st ], p[ 0 ], p[ st ], ql[ NP - 1 ], qr[ NP - 1 ] );
        }
        if constexpr( MHD )
            ql[ BCC + axis ] = qr[ BCC + axis ] = normal_b< R, XL >( a, b, axis, step, ii, wb );
    }
    else
        for( int k = 0; k < NP; ++ k )
        {
            if( MHD && k == BCC + axis )
            {
                ql[ k ] = qr[ k ] = normal_b< R, XL >( a, b, axis, step, ii, wb );
                continue;
            }
            const R * p = wb + k * ngw;
            plm_face_fast< R >( p[ -2 * st ], p[ -st ], p[ 0 ], p[ st ], ql[ k ], qr[ k ] );
        }
}

// One CTA's 128 faces of a sweep: bx = CTA along the faces of one (x, y)
// plane, by = z plane, blockIdx.z = block; dv
// divides by the row length.
template< bool MHD, class R, int MODE, bool XL = false > __device__ __forceinline__
void flux_faces( const args_t< R > & a, int axis, int step, udiv_t dv, int b, unsigned bx, unsigned by,
                 bool hlle_warp = false )
{
    constexpr int NW = MHD ? 11 : 5;   // stored W words: prim (8) + cell E (3)
    constexpr bool learned = MHD && MODE == KR_RIEMANN_LEARNED;
    const int nn[ 3 ] = { a.n0, a.n1, a.n2 };
    unsigned t = bx * blockDim.x + threadIdx.x;
    int ii[ 3 ];
    int outside = 0;
    unsigned total;
    long long t_lin;                  // face number within the sweep (sampling keys)
    const int lo = MHD ? -1 : 0;
    int ext[ 3 ];
    for( int d = 0; d < 3; ++ d )
        ext[ d ] = d == axis ? nn[ d ] + 1 : nn[ d ] - 2 * lo;
    total = unsigned( ext[ 0 ] * ext[ 1 ] );
    if constexpr( XL )
    {   // refined MHD: one index over the whole block's faces (its blocks are
        // small, and per-plane rows of 128 faces left a fifth of the lanes idle)
        by = t / total;
        t -= by * total;
        if( by >= unsigned( ext[ 2 ] ) )
            return;
    }
    const unsigned q = udiv_q( t, dv );
    ii[ 0 ] = int( t - q * unsigned( ext[ 0 ] ) );
    ii[ 1 ] = int( q );
    ii[ 2 ] = int( by );
    t_lin = ( long long ) t + ( long long ) total * by;
    for( int d = 0; d < 3; ++ d )
        if( d != axis )
        {
            ii[ d ] += lo;
            outside += ( ii[ d ] < 0 || ii[ d ] >= nn[ d ] );
        }
    // corner lines are never read; lanes past the end idle.  Lanes stay alive
    // until the (warp-collective) selector has run.
    const bool valid = t < total && outside <= 1;
    if( ! valid && ! learned )
        return;
    // learned mode: the warp's place in the sweep's chunk order (chunks of 128
    // faces, z plane outer, 4 warps each)
    const unsigned wid = ( by * ( ( total + 127u ) >> 7 ) + bx ) * 4u + ( threadIdx.x >> 5 );
    const int st = axis == 0 ? 1 : ( axis == 1 ? a.sw1 : a.sw2 );
    R ql[ 8 ], qr[ 8 ];
    if( valid )
    {
        const R * wb = a.w + ( size_t ) b * NW * a.ngw
                     + ( ( ii[ 0 ] + 2 ) + a.sw1 * ( ii[ 1 ] + 2 ) + a.sw2 * ( ii[ 2 ] + 2 ) );
        plm_stencil< MHD, R, XL >( a, b, axis, step, ii, wb, st, ql, qr );
    }
    if constexpr( learned || MODE == FLUX_APPLY )
    {
        if constexpr( learned )
            learned_solve< MHD, R >( a, b, axis, ii, valid, ql, qr, wid );
        else
            solve_store< MHD, R, FLUX_APPLY >( a, b, axis, ii, true, ql, qr, 0, 0ull, hlle_warp );
        return;
    }
    const unsigned long long key = ( ( unsigned long long ) b * 3 + axis ) * 0x9E3779B97F4A7C15ull
                                 + ( unsigned long long ) t_lin;
    solve_store< MHD, R, MODE >( a, b, axis, ii, valid, ql, qr, threadIdx.x >> 5, key );
}

// XL: a refined MHD mesh (the ghost-line normal-B rule, normal_b).  AXIS: the
// sweep direction as a compile-time constant, so the stencil stride, the
// component permutation and the face extents fold into the code (one kernel
// per axis; the sweep is bound by instruction issue).
template< bool MHD, class R, int MODE, bool XL, int AXIS >
__global__ void __launch_bounds__( 128, ( flux_min_ctas< R, MODE >(  ) ) ) k_flux( const args_t< R > a, int step, udiv_t dv )
{
    constexpr int axis = AXIS;
    bool hlle_warp = false;
    if constexpr( MODE == FLUX_APPLY )
    {   // learned mode, sweeps without the network: this warp's solver choice,
        // loaded first (gridDim.x: 128-face chunks per z plane)
        if( step == 0 && sel_eval_step( a.s, a.sel_period ) )
            return;                   // the network's sweep (k_flux_eval) solves this one
        hlle_warp = ( a.sel_dec[ ( ( size_t ) axis * a.nblk + blockIdx.z ) * a.sel_wcap
                                 + ( blockIdx.y * gridDim.x + blockIdx.x ) * 4u + ( threadIdx.x >> 5 ) ]
                      >> ( threadIdx.x & 31 ) ) & 1u;
    }
    flux_faces< MHD, R, MODE, XL >( a, axis, step, dv, blockIdx.z, blockIdx.x, blockIdx.y, hlle_warp );
}

// Learned mode, the network's sweep: a fixed grid strides over the 128-face
// chunks (cpp per z plane, nz planes), so on the stages where the network does
// not run (k_flux<FLUX_APPLY> solves them) only this small grid launches and
// exits.
template< bool MHD, class R, int AXIS >
__global__ void __launch_bounds__( 128, ( flux_min_ctas< R, KR_RIEMANN_LEARNED >(  ) ) )
k_flux_eval( const args_t< R > a, int step, udiv_t dv, unsigned cpp, unsigned nz )
{
    constexpr int axis = AXIS;
    if( step != 0 || ! sel_eval_step( a.s, a.sel_period ) )
        return;
    for( unsigned ch = blockIdx.x; ch < cpp * nz; ch += gridDim.x )
        flux_faces< MHD, R, KR_RIEMANN_LEARNED >( a, axis, step, dv, blockIdx.z, ch % cpp, ch / cpp );
}

////////////////////////////////////////////////////////////
// Edge EMF (mhd/integrator/integrator.h:189-327 calc_field): face EMF average
// plus the upwinded corner terms chosen by the sign of the mass flux.

template< class R > __device__ __forceinline__
R e_cell( const args_t< R > & a, int b, const int * j, int ax )
{
    return a.w[ iw( a, b, 8 + ax, 11, j[ 0 ], j[ 1 ], j[ 2 ] ) ];   // cell E, stored by k_c2p
}

template< class R > __device__ __forceinline__
R face_emf( const args_t< R > & a, int b, int fa, int ax, const int * i )
{   // E_ax held by the flux of axis fa
    const int slot = ( ax == mod3( fa + 1 ) ) ? 5 : 6;
    return a.f[ fa ][ ifx( a, b, slot, 7, i[ 0 ], i[ 1 ], i[ 2 ] ) ];
}

// Edge site t of the (x, y) plane i2 of block b.
template< class R > __device__ __forceinline__
void emf_site( const args_t< R > & a, udiv_t dv, int b, int i2, unsigned t )
{
    const int e0 = a.n0 + 1, e1 = a.n1 + 1;
    if( t >= unsigned( e0 * e1 ) )
        return;
    const unsigned q = udiv_q( t, dv );
    int i[ 3 ] = { int( t - q * unsigned( e0 ) ), int( q ), i2 };
    const int nn[ 3 ] = { a.n0, a.n1, a.n2 };
    const R w_e = R( 0.25f );
    // one base offset per site (cell E in W, the fluxes, the edge EMF); the
    // neighbours by constant strides
    const long long oW = iw( a, b, 8, 11, i[ 0 ], i[ 1 ], i[ 2 ] );
    const long long oF = ifx( a, b, 0, 7, i[ 0 ], i[ 1 ], i[ 2 ] );
    const long long oE = ifx( a, b, 0, 3, i[ 0 ], i[ 1 ], i[ 2 ] );
    const int sw[ 3 ] = { 1, a.sw1, a.sw2 }, sf[ 3 ] = { 1, a.sf1, a.sf2 };
    for( int ax = 0; ax < 3; ++ ax )
    {
        if( i[ ax ] >= nn[ ax ] )
            continue;
        const int ax1 = mod3( 1 + ax ), ax2 = mod3( 2 + ax );
        const R * we = a.w + oW + ( long long ) ax * a.ngw;   // cell E_ax, stored by k_c2p
        R ec[ 2 ][ 2 ];
        ec[ 1 ][ 1 ] = we[ 0 ];
        ec[ 1 ][ 0 ] = we[ -sw[ ax1 ] ];
        ec[ 0 ][ 0 ] = we[ -sw[ ax1 ] - sw[ ax2 ] ];
        ec[ 0 ][ 1 ] = we[ -sw[ ax2 ] ];
        R e = 0;
        for( int it = 0; it < 2; ++ it )
        {
            const int a_para = it == 0 ? ax1 : ax2;
            const int a_perp = it == 0 ? ax2 : ax1;
            // E_ax held by the flux of axis a_para (face_emf's slot)
            const R * fe = a.f[ a_para ] + oF + ( long long )( ( ax == mod3( a_para + 1 ) ) ? 5 : 6 ) * a.nfb;
            const R ef_m = fe[ -sf[ a_perp ] ];
            const R ef_p = fe[ 0 ];
            e += w_e * ( ef_m + ef_p );
            const R * fr = a.f[ a_perp ] + oF;                   // mass flux (RHO = 0)
            const R frho_p = fr[ 0 ];
            const R frho_m = fr[ -sf[ a_para ] ];
            const R de_p = frho_p > 0 ?  ( ec[ 0 ][ 1 ] - ef_m ) :  ( ec[ 1 ][ 1 ] - ef_p );
            const R de_m = frho_m > 0 ? -( ec[ 0 ][ 0 ] - ef_m ) : -( ec[ 1 ][ 0 ] - ef_p );
            e += w_e * ( de_m - de_p );
            if( it == 0 )
            {
                const R swp = ec[ 0 ][ 1 ];
                ec[ 0 ][ 1 ] = ec[ 1 ][ 0 ];
                ec[ 1 ][ 0 ] = swp;
            }
        }
        a.ee[ oE + ( long long ) ax * a.nfb ] = e;
    }
    if( ! a.emf_out )
        return;
    // boundary-plane edges of a high out / fre side: the interior cell's
    // advective E, with the reference's velocity scaling (w holds v, which it
    // multiplies by 1 / rho once more) -- integrator.h:329-382
    const int ph = a.geo[ b ].phys;
    for( int d = 0; d < 3; ++ d )
    {
        if( ! ( a.emf_out >> d & 1 ) || i[ d ] != nn[ d ] || nn[ d ] < 2 || ! ( ( ph >> ( 2 * d + 1 ) ) & 1 ) )
            continue;
        int jc[ 3 ] = { i[ 0 ], i[ 1 ], i[ 2 ] };
        -- jc[ d ];
        const R irho = R( 1 ) / fmax( a.w[ iw( a, b, RHO, 11, jc[ 0 ], jc[ 1 ], jc[ 2 ] ) ], R( 1e-30 ) );
        R v_c[ 3 ], b_c[ 3 ];
        for( int q = 0; q < 3; ++ q )
        {
            v_c[ q ] = a.w[ iw( a, b, MOM + q, 11, jc[ 0 ], jc[ 1 ], jc[ 2 ] ) ] * irho;
            b_c[ q ] = a.w[ iw( a, b, BCC + q, 11, jc[ 0 ], jc[ 1 ], jc[ 2 ] ) ];
        }
        const int d1 = mod3( d + 1 ), d2 = mod3( d + 2 );
        a.ee[ ifx( a, b, d1, 3, i[ 0 ], i[ 1 ], i[ 2 ] ) ] = v_c[ d ] * b_c[ d2 ] - v_c[ d2 ] * b_c[ d ];
        a.ee[ ifx( a, b, d2, 3, i[ 0 ], i[ 1 ], i[ 2 ] ) ] = v_c[ d1 ] * b_c[ d ] - v_c[ d ] * b_c[ d1 ];
    }
}

template< class R >
__global__ void __launch_bounds__( 256 ) k_emf( const args_t< R > a, udiv_t dv )
{
    // grid: x over the edges of one (x, y) plane, y over z, z over blocks
    emf_site< R >( a, dv, blockIdx.z, blockIdx.y, blockIdx.x * blockDim.x + threadIdx.x );
}

////////////////////////////////////////////////////////////
// Conserved update (hydro/integrator/integrator.h:241-265 add_flux with
// hydro/integrator/rk2.h:20-34 load) and CT face update
// (mhd/integrator/integrator.h:387-462, mhd/integrator/rk2.h:49-63 set_field).
// One thread per lattice site.

// Static refinement (SMR): the face of a refined side is left out of the
// update (load_flux_sfc, f_a = -1), and afterwards the cell takes the
// averaged fine flux of that face, sides z, y, x and low before high
// (hydro/integrator/integrator.h:343-382 intg_flx / add_flux):
// u += ( dt * ds / ( +-vol ) ) * f.
template< class R > __device__ __forceinline__
double smr_correct( const args_t< R > & a, const geo_t & g, int b, const int * i, const int * nn,
                    int k, double dt, double v )
{
    for( int ax = 2; ax >= 0; -- ax )
        for( int side = 0; side <= 1; ++ side )
            if( ( ( g.fine >> ( 2 * ax + side ) ) & 1 ) && i[ ax ] == ( side ? nn[ ax ] - 1 : 0 ) )
            {
                const int a1 = mod3( ax + 1 ), a2 = mod3( ax + 2 );
                const int h1 = nn[ a1 ] >> 1, h2 = nn[ a2 ] >> 1;
                const int d1 = i[ a1 ] >= h1, d2 = i[ a2 ] >= h2;
                const int item = g.fitem[ 2 * ax + side ] + 2 * d1 + d2;
                const int t = ( i[ a2 ] - d2 * h2 ) * h1 + ( i[ a1 ] - d1 * h1 );
                const double conv = dt * g.sfc[ ax ] / ( g.vol * ( side ? -1 : 1 ) );
                v += conv * a.favg[ ( ( size_t ) item * 5 + k ) * a.favg_n + t ];
            }
    return v;
}

// The same for all five components (sides outer, components inner: each
// component still takes its sides in the order above).
template< class R > __device__ __forceinline__
void smr_correct5( const args_t< R > & a, const geo_t & g, int b, const int * i, const int * nn,
                   double dt, double * v )
{
#pragma unroll
    for( int ax = 2; ax >= 0; -- ax )
#pragma unroll
        for( int side = 0; side <= 1; ++ side )
            if( ( ( g.fine >> ( 2 * ax + side ) ) & 1 ) && i[ ax ] == ( side ? nn[ ax ] - 1 : 0 ) )
            {
                const int a1 = mod3( ax + 1 ), a2 = mod3( ax + 2 );
                const int h1 = nn[ a1 ] >> 1, h2 = nn[ a2 ] >> 1;
                const int d1 = i[ a1 ] >= h1, d2 = i[ a2 ] >= h2;
                const int item = g.fitem[ 2 * ax + side ] + 2 * d1 + d2;
                const int t = ( i[ a2 ] - d2 * h2 ) * h1 + ( i[ a1 ] - d1 * h1 );
                const double conv = dt * g.sfc[ ax ] / ( g.vol * ( side ? -1 : 1 ) );
                const double * f = a.favg + ( size_t ) item * 5 * a.favg_n + t;
#pragma unroll
                for( int k = 0; k < 5; ++ k )
                    v[ k ] += conv * f[ ( size_t ) k * a.favg_n ];
            }
}

// dt of the stage's update: Heun U* = U + dt L(U), U' = (U + U*) / 2 + dt / 2
// L(U*); VL2 U* = U + dt / 2 L1(U), U' = U + dt L(U*).
template< class R > __device__ __forceinline__
double stage_dt( const args_t< R > & a, int step, int b )
{
    return __longlong_as_double( a.s[ a.boxes ? b : 0 ].dt_bits )
         * ( ( step == 0 ) != bool( a.vl2 ) ? 1.0 : double( 0.5f ) );
}

// Stage 0's conserved update of interior cell i of a uniform MHD block from its
// six face fluxes (update_site's PART 1 arithmetic, term for term), written to
// slot 1; v returns the five new words.
template< class R > __device__ __forceinline__
void update_cell( const args_t< R > & a, int b, const int * i, double dt, double * v )
{
    constexpr int NF = 7;
    const geo_t & g = a.geo[ b ];
    const R * __restrict__ F[ 3 ] = { a.f[ 0 ], a.f[ 1 ], a.f[ 2 ] };
    const double * __restrict__ us = a.u[ 0 ];
    double * __restrict__ ut = a.u[ 1 ];
    const double dt_dv = dt / g.vol;
    const long long o = ifx( a, b, 0, NF, i[ 0 ], i[ 1 ], i[ 2 ] );
    const long long c0 = iuc( a, b, 0, i[ 0 ], i[ 1 ], i[ 2 ] );
    const long long s1[ 3 ] = { 1, a.sf1, a.sf2 };
    if constexpr( sizeof( R ) == 4 )
    {   // all loads first (30 flux words, 5 state words), then the sums
        R fl[ 3 ][ 5 ], fr[ 3 ][ 5 ];
        for( int d = 0; d < 3; ++ d )
            for( int k = 0; k < 5; ++ k )
            {
                fl[ d ][ k ] = F[ d ][ o + k * a.nfb ];
                fr[ d ][ k ] = F[ d ][ o + k * a.nfb + s1[ d ] ];
            }
        for( int k = 0; k < 5; ++ k )
            v[ k ] = us[ c0 + k * a.nc ];
        for( int k = 0; k < 5; ++ k )
        {
            for( int d = 0; d < 3; ++ d )
            {
                const double f_a = g.sfc[ d ] * dt_dv;
                double res = 0;
                res += f_a * double( fl[ d ][ k ] );
                res -= f_a * double( fr[ d ][ k ] );
                v[ k ] += res;
            }
            ut[ c0 + k * a.nc ] = v[ k ];
        }
    }
    else
        for( int k = 0; k < 5; ++ k )
        {   // FP64 fluxes: one component at a time keeps the registers low
            const long long c = c0 + k * a.nc;
            double w = us[ c ];
            for( int d = 0; d < 3; ++ d )
            {
                const double f_a = g.sfc[ d ] * dt_dv;
                double res = 0;
                res += f_a * double( F[ d ][ o + k * a.nfb ] );
                res -= f_a * double( F[ d ][ o + k * a.nfb + s1[ d ] ] );
                w += res;
            }
            ut[ c ] = w;
            v[ k ] = w;
        }
}

// CT update of face B component c at lattice site i of block b from its four
// edge EMFs (update_site's PART 2 arithmetic, term for term): e1 = E_ax1 at i,
// e1p at i + e_ax2, e2 = E_ax2 at i, e2p at i + e_ax1 (ax1, ax2 = c + 1, c + 2).
// WRITE: store it, and push it into the ghost strip of the same-level block
// across a transverse side it lies next to (for the next stage: that block's
// sweeps read it); -1 / -2 neighbours as for W.
// k: the face's index in BF (ibf( a, b, c, i )).
template< class R, bool WRITE > __device__ __forceinline__
double ct_face( const args_t< R > & a, const geo_t & g, int b, int c, const int * i, long long k, int step,
                double dt, R e1, R e1p, R e2, R e2p )
{
    const int nn[ 3 ] = { a.n0, a.n1, a.n2 };
    const int sb[ 3 ] = { 1, a.sb1, a.sb2 };
    const double * __restrict__ bs = a.bf[ step ];
    double * __restrict__ bt = a.bf[ 1 - step ];
    const int ax1 = mod3( c + 1 ), ax2 = mod3( c + 2 );
    double db;
    db  = double( e1 ) * g.dx[ ax1 ];
    db -= double( e2 ) * g.dx[ ax2 ];
    db += double( e2p ) * g.dx[ ax2 ];
    db -= double( e1p ) * g.dx[ ax1 ];
    // the reference scales by -dt / sfc; -dt * (1 / sfc) differs in rounding only
    db *= -dt * g.isfc[ c ];
    const double nb = db + ( step == 0 ? bs[ k ] : ( a.vl2 ? bt[ k ] : ( bs[ k ] + bt[ k ] ) / 2 ) );
    if constexpr( WRITE )
    {
        bt[ k ] = nb;
        for( int l = 0; l < 2; ++ l )
        {
            const int t = l ? ax2 : ax1;
            if( i[ t ] != 0 && i[ t ] != nn[ t ] - 1 )
                continue;
            const int s = i[ t ] == 0 ? -1 : 1;
            const int dst = a.nbr[ b * 27 + 13 + s * ( t == 0 ? 1 : ( t == 1 ? 3 : 9 ) ) ];
            if( dst < 0 )
                continue;
            const int dj = ( s < 0 ? nn[ t ] : -1 ) - i[ t ];
            bt[ k + ( long long )( dst - b ) * 3 * a.nbf + ( long long ) dj * sb[ t ] ] = nb;
        }
    }
    return nb;
}

// PART 0: cells and faces in one launch; 1: the conserved update only; 2: the
// CT face update only (MHD: two launches, each with fewer registers).
// Lattice site t of the (x, y) plane i2 of block b.
template< bool MHD, class R, bool SMR, int PART > __device__ __forceinline__
void update_site( const args_t< R > & a, int step, udiv_t dv, int b, int i2, unsigned t )
{
    constexpr int NF = MHD ? 7 : 5;
    const int e0 = a.n0 + 1, e1 = a.n1 + 1;
    if( t >= unsigned( e0 * e1 ) )
        return;
    const unsigned q = udiv_q( t, dv );
    int i[ 3 ] = { int( t - q * unsigned( e0 ) ), int( q ), i2 };
    const int nn[ 3 ] = { a.n0, a.n1, a.n2 };
    // Heun: U* = U + dt L(U), U' = (U + U*) / 2 + dt / 2 L(U*); VL2:
    // U* = U + dt / 2 L1(U), U' = U + dt L(U*)
    const double dt = __longlong_as_double( a.s[ a.boxes ? b : 0 ].dt_bits )
                    * ( ( step == 0 ) != bool( a.vl2 ) ? 1.0 : double( 0.5f ) );
    const geo_t & g = a.geo[ b ];
    // The arrays never overlap: restrict lets the loads of later components
    // issue ahead of the stores of earlier ones.
    const R * __restrict__ F[ 3 ] = { a.f[ 0 ], a.f[ 1 ], a.f[ 2 ] };
    const R * __restrict__ EE = a.ee;
    if( PART != 2 && i[ 0 ] < nn[ 0 ] && i[ 1 ] < nn[ 1 ] && i[ 2 ] < nn[ 2 ] )
    {
        const double * __restrict__ us = a.u[ step ];
        double * __restrict__ ut = a.u[ 1 - step ];
        const double dt_dv = dt / g.vol;
        const long long o = ifx( a, b, 0, NF, i[ 0 ], i[ 1 ], i[ 2 ] );
        const long long c0 = iuc( a, b, 0, i[ 0 ], i[ 1 ], i[ 2 ] );
        const long long s1[ 3 ] = { 1, a.sf1, a.sf2 };
        if constexpr( sizeof( R ) == 4 )
        {   // all loads first (30 flux words, 5 or 10 state words), then the sums
            R fl[ 3 ][ 5 ], fr[ 3 ][ 5 ];
            for( int d = 0; d < 3; ++ d )
                for( int k = 0; k < 5; ++ k )
                {
                    fl[ d ][ k ] = F[ d ][ o + k * a.nfb ];
                    fr[ d ][ k ] = F[ d ][ o + k * a.nfb + s1[ d ] ];
                }
            double v[ 5 ];
            for( int k = 0; k < 5; ++ k )
                v[ k ] = step == 0 ? us[ c0 + k * a.nc ]
                       : ( a.vl2 ? ut[ c0 + k * a.nc ] : ( us[ c0 + k * a.nc ] + ut[ c0 + k * a.nc ] ) * 0.5f );
            if constexpr( ! SMR )
                for( int k = 0; k < 5; ++ k )
                {
                    for( int d = 0; d < 3; ++ d )
                    {
                        const double f_a = g.sfc[ d ] * dt_dv;
                        double res = 0;
                        res += f_a * double( fl[ d ][ k ] );
                        res -= f_a * double( fr[ d ][ k ] );
                        v[ k ] += res;
                    }
                    ut[ c0 + k * a.nc ] = v[ k ];
                }
            else
            {
                bool nl[ 3 ], nr[ 3 ];
                for( int d = 0; d < 3; ++ d )
                {
                    nl[ d ] = ( ( g.fine >> ( 2 * d ) ) & 1 ) && i[ d ] == 0;
                    nr[ d ] = ( ( g.fine >> ( 2 * d + 1 ) ) & 1 ) && i[ d ] == nn[ d ] - 1;
                }
#pragma unroll
                for( int k = 0; k < 5; ++ k )
#pragma unroll
                    for( int d = 0; d < 3; ++ d )
                    {
                        const double f_a = g.sfc[ d ] * dt_dv;
                        double res = 0;
                        if( ! nl[ d ] )
                            res += f_a * double( fl[ d ][ k ] );
                        if( ! nr[ d ] )
                            res -= f_a * double( fr[ d ][ k ] );
                        v[ k ] += res;
                    }
                if( g.fine )
                    smr_correct5( a, g, b, i, nn, dt, v );
#pragma unroll
                for( int k = 0; k < 5; ++ k )
                    ut[ c0 + k * a.nc ] = v[ k ];
            }
        }
        else
            for( int k = 0; k < 5; ++ k )
            {   // FP64 fluxes: one component at a time keeps the registers low
                const long long c = c0 + k * a.nc;
                double v = step == 0 ? us[ c ] : ( a.vl2 ? ut[ c ] : ( us[ c ] + ut[ c ] ) * 0.5f );
                for( int d = 0; d < 3; ++ d )
                {
                    const double f_a = g.sfc[ d ] * dt_dv;
                    double res = 0;
                    if( ! SMR || ! ( ( ( g.fine >> ( 2 * d ) ) & 1 ) && i[ d ] == 0 ) )
                        res += f_a * double( F[ d ][ o + k * a.nfb ] );
                    if( ! SMR || ! ( ( ( g.fine >> ( 2 * d + 1 ) ) & 1 ) && i[ d ] == nn[ d ] - 1 ) )
                        res -= f_a * double( F[ d ][ o + k * a.nfb + s1[ d ] ] );
                    v += res;
                }
                if constexpr( SMR )
                    v = smr_correct( a, g, b, i, nn, k, dt, v );
                ut[ c ] = v;
            }
    }
    if( ! MHD || PART == 1 )
        return;
    const double * __restrict__ bs = a.bf[ step ];
    double * __restrict__ bt = a.bf[ 1 - step ];
    // one base offset per site; components and neighbours by constant strides
    const long long oe = ifx( a, b, 0, 3, i[ 0 ], i[ 1 ], i[ 2 ] );
    const long long ob = ibf( a, b, 0, i[ 0 ], i[ 1 ], i[ 2 ] );
    const int se[ 3 ] = { 1, a.sf1, a.sf2 };
    const int sb[ 3 ] = { 1, a.sb1, a.sb2 };
    for( int c = 0; c < 3; ++ c )
    {
        const int ax1 = mod3( c + 1 ), ax2 = mod3( c + 2 );
        if( i[ ax1 ] >= nn[ ax1 ] || i[ ax2 ] >= nn[ ax2 ] )
            continue;
        const R * e1 = EE + oe + ( long long ) ax1 * a.nfb;
        const R * e2 = EE + oe + ( long long ) ax2 * a.nfb;
        double db;
        db  = double( e1[ 0 ] ) * g.dx[ ax1 ];
        db -= double( e2[ 0 ] ) * g.dx[ ax2 ];
        db += double( e2[ se[ ax1 ] ] ) * g.dx[ ax2 ];
        db -= double( e1[ se[ ax2 ] ] ) * g.dx[ ax1 ];
        // the reference scales by -dt / sfc; -dt * (1 / sfc) differs in rounding only
        db *= -dt * g.isfc[ c ];
        const long long k = ob + ( long long ) c * a.nbf;
        const double nb = db + ( step == 0 ? bs[ k ] : ( a.vl2 ? bt[ k ] : ( bs[ k ] + bt[ k ] ) / 2 ) );
        bt[ k ] = nb;
        // Same-level face-B ghost strips by push, for the next stage: a face
        // next to a transverse side is a ghost face of the block across it
        // (the one whose pull along that axis reads it); -1 / -2 as for W.
        for( int l = 0; l < 2; ++ l )
        {
            const int t = l ? ax2 : ax1;
            if( i[ t ] != 0 && i[ t ] != nn[ t ] - 1 )
                continue;
            const int s = i[ t ] == 0 ? -1 : 1;
            const int dst = a.nbr[ b * 27 + 13 + s * ( t == 0 ? 1 : ( t == 1 ? 3 : 9 ) ) ];
            if( dst < 0 )
                continue;
            const int dj = ( s < 0 ? nn[ t ] : -1 ) - i[ t ];
            bt[ k + ( long long )( dst - b ) * 3 * a.nbf + ( long long ) dj * sb[ t ] ] = nb;
        }
    }
}

template< bool MHD, class R, bool SMR = false, int PART = 0 >
__global__ void __launch_bounds__( 256, ( SMR && sizeof( R ) == 4 ) ? 4 : ( PART == 2 ? 6 : 4 ) ) k_update( const args_t< R > a, int step, udiv_t dv )
{
    // grid: x over the lattice sites of one (x, y) plane, y over z, z over blocks
    update_site< MHD, R, SMR, PART >( a, step, dv, blockIdx.z, blockIdx.y, blockIdx.x * blockDim.x + threadIdx.x );
}

////////////////////////////////////////////////////////////
// Stage 0 of a uniform MHD step after the edge EMF, in one launch: the cell
// update, the CT update of the cell's six faces and cons -> prim of (U*, B*)
// for stage 1 -- what k_update's two parts and stage 1's k_c2p do, with the
// same arithmetic term for term (c2p_point is shared with k_c2p), one thread
// per cell with no shared memory.  A face is written
// by the cell above it (its low face) and, at the block's high end, by the last
// cell; the cell below computes it again for its own cell-centred B.  At stage
// 0 both computations read only slot 0 of B and the edge EMFs and the writes go
// to slot 1, so they agree bit for bit.  (Stage 1 updates B in place, so there
// the faces keep one writer each and c2p stays at the start of the next step.)
// Nothing here reads W, so the new primitives go straight to it.
template< class R > __device__ __forceinline__
void update_c2p_cell( const args_t< R > & a, int b, int i0, int i1, int i2 )
{
    const int i[ 3 ] = { i0, i1, i2 };
    const int nn[ 3 ] = { a.n0, a.n1, a.n2 };
    const geo_t & g = a.geo[ b ];
    const double dt = stage_dt( a, 0, b );
    double v[ 5 ];
    update_cell< R >( a, b, i, dt, v );
    const R * __restrict__ EE = a.ee;
    const int se[ 3 ] = { 1, a.sf1, a.sf2 };
    const int sb[ 3 ] = { 1, a.sb1, a.sb2 };
    const long long ob = ibf( a, b, 0, i0, i1, i2 );
    double b_l[ 3 ], b_r[ 3 ];
#pragma unroll
    for( int c = 0; c < 3; ++ c )
    {
        const int ax1 = mod3( c + 1 ), ax2 = mod3( c + 2 );
#pragma unroll
        for( int side = 0; side < 2; ++ side )
        {
            int j[ 3 ] = { i0, i1, i2 };
            j[ c ] += side;
            const long long oe = ifx( a, b, 0, 3, j[ 0 ], j[ 1 ], j[ 2 ] );
            const R * e1 = EE + oe + ( long long ) ax1 * a.nfb;
            const R * e2 = EE + oe + ( long long ) ax2 * a.nfb;
            const R e1a = e1[ 0 ], e1b = e1[ se[ ax2 ] ], e2a = e2[ 0 ], e2b = e2[ se[ ax1 ] ];
            const long long k = ob + ( long long ) c * a.nbf + ( side ? sb[ c ] : 0 );
            const bool own = side == 0 || i[ c ] == nn[ c ] - 1;
            const double nb = own ? ct_face< R, true >( a, g, b, c, j, k, 0, dt, e1a, e1b, e2a, e2b )
                                  : ct_face< R, false >( a, g, b, c, j, k, 0, dt, e1a, e1b, e2a, e2b );
            ( side ? b_r : b_l )[ c ] = nb;
        }
    }
    double prim[ 5 ], bc_2[ 3 ], b_max[ 3 ], cs2;
    c2p_point< true, R >( a, a.w, a.u[ 1 ], b, i0, i1, i2, v, b_l, b_r, prim, bc_2, b_max, cs2 );
}

template< class R >
__global__ void __launch_bounds__( 256, 4 ) k_update_c2p( const args_t< R > a, udiv_t dv )
{
    // grid: x over the cells of one (x, y) plane, y over z, z over blocks
    const unsigned c = blockIdx.x * blockDim.x + threadIdx.x;
    if( c >= unsigned( a.n0 * a.n1 ) )
        return;
    const unsigned q = udiv_q( c, dv );
    update_c2p_cell< R >( a, blockIdx.z, int( c - q * unsigned( a.n0 ) ), int( q ), blockIdx.y );
}

template< bool MHD, class R >
__global__ void k_scatter( const args_t< R > a, const double * hu, const double * hbf )
{
    constexpr int NWR = MHD ? 8 : 5;
    const int b = blockIdx.y;
    const long long t = ( long long ) blockIdx.x * blockDim.x + threadIdx.x;
    if( t < a.nc )
        for( int k = 0; k < 5; ++ k )
            a.u[ 0 ][ ( long long )( b * 5 + k ) * a.nc + t ] = hu[ ( ( long long ) b * a.nc + t ) * NWR + k ];
    if( MHD && t < a.nbf )
        for( int c = 0; c < 3; ++ c )
            a.bf[ 0 ][ ( long long )( b * 3 + c ) * a.nbf + t ] = hbf[ ( ( long long ) b * a.nbf + t ) * 3 + c ];
}

template< bool MHD, class R >
__global__ void k_gather( const args_t< R > a, double * hu, double * hbf )
{
    constexpr int NWR = MHD ? 8 : 5;
    const int b = blockIdx.y;
    const long long t = ( long long ) blockIdx.x * blockDim.x + threadIdx.x;
    if( t < a.nc )
    {
        for( int k = 0; k < 5; ++ k )
            hu[ ( ( long long ) b * a.nc + t ) * NWR + k ] = a.u[ 0 ][ ( long long )( b * 5 + k ) * a.nc + t ];
        if( MHD )
        {
            const int i0 = int( t % a.n0 ), i1 = int( ( t / a.n0 ) % a.n1 ), i2 = int( t / ( ( long long ) a.n0 * a.n1 ) );
            const int ii[ 3 ] = { i0, i1, i2 };
            for( int d = 0; d < 3; ++ d )
            {
                int jj[ 3 ] = { ii[ 0 ], ii[ 1 ], ii[ 2 ] };
                const double bl = a.bf[ 0 ][ ibf( a, b, d, jj[ 0 ], jj[ 1 ], jj[ 2 ] ) ];
                ++ jj[ d ];
                const double br = a.bf[ 0 ][ ibf( a, b, d, jj[ 0 ], jj[ 1 ], jj[ 2 ] ) ];
                hu[ ( ( long long ) b * a.nc + t ) * NWR + BCC + d ] = ( bl + br ) / 2;
            }
        }
    }
    if( MHD && t < a.nbf )
        for( int c = 0; c < 3; ++ c )
            hbf[ ( ( long long ) b * a.nbf + t ) * 3 + c ] = a.bf[ 0 ][ ( long long )( b * 3 + c ) * a.nbf + t ];
}

////////////////////////////////////////////////////////////
// Diagnostics: max |div B| (owned cells) and domain totals.

template< bool MHD, class R >
__global__ void __launch_bounds__( 256 ) k_diag( const args_t< R > a, double * out )
{
    // per thread: one cell's contributions; then a CTA reduction and one
    // atomic per CTA and quantity (not one per cell: the per-cell atomics on
    // six addresses serialised the whole grid)
    const int b = blockIdx.y;
    const long long t = ( long long ) blockIdx.x * blockDim.x + threadIdx.x;
    double v[ 5 ] = { 0, 0, 0, 0, 0 }, div = 0;
    if( t < a.nc )
    {
        const int i0 = int( t % a.n0 ), i1 = int( ( t / a.n0 ) % a.n1 ), i2 = int( t / ( ( long long ) a.n0 * a.n1 ) );
        const geo_t & g = a.geo[ b ];
        for( int k = 0; k < 5; ++ k )
            v[ k ] = a.u[ 0 ][ iuc( a, b, k, i0, i1, i2 ) ] * g.vol;
        if( MHD )
        {
            const int ii[ 3 ] = { i0, i1, i2 };
            for( int d = 0; d < 3; ++ d )
            {
                int jj[ 3 ] = { ii[ 0 ], ii[ 1 ], ii[ 2 ] };
                const double bl = a.bf[ 0 ][ ibf( a, b, d, jj[ 0 ], jj[ 1 ], jj[ 2 ] ) ];
                ++ jj[ d ];
                const double br = a.bf[ 0 ][ ibf( a, b, d, jj[ 0 ], jj[ 1 ], jj[ 2 ] ) ];
                div += ( br - bl ) * g.sfc[ d ];
            }
            div = fabs( div ) / g.vol;
        }
    }
    __shared__ double red[ 6 ][ 8 ];
    for( int o = 16; o > 0; o >>= 1 )
    {
        for( int k = 0; k < 5; ++ k )
            v[ k ] += __shfl_xor_sync( 0xffffffffu, v[ k ], o );
        div = fmax( div, __shfl_xor_sync( 0xffffffffu, div, o ) );
    }
    const int w = threadIdx.x >> 5;
    if( ( threadIdx.x & 31 ) == 0 )
    {
        for( int k = 0; k < 5; ++ k )
            red[ k ][ w ] = v[ k ];
        red[ 5 ][ w ] = div;
    }
    __syncthreads(  );
    if( threadIdx.x < 6 )
    {
        double r = red[ threadIdx.x ][ 0 ];
        for( int k = 1; k < int( blockDim.x >> 5 ); ++ k )
            r = threadIdx.x < 5 ? r + red[ threadIdx.x ][ k ] : fmax( r, red[ threadIdx.x ][ k ] );
        if( threadIdx.x < 5 )
            atomicAdd( out + 1 + threadIdx.x, r );
        else if( MHD )
            atomicMax( ( unsigned long long * ) out, ( unsigned long long ) __double_as_longlong( r ) );
    }
}

////////////////////////////////////////////////////////////
// Halo exchange between ranks: pack / unpack of the ghost values one block
// takes from a neighbour in direction `dir` (k_ghost's sources, per item).
// Item layout in the buffers: primitive words component-major over the
// destination's ghost box (x fastest), then for a face direction along d the
// face-B strips of components (d+1)%3 and (d+2)%3.  PACK runs on the rank
// owning the source block (blk = source, coordinates shifted by -dir * n),
// !PACK on the rank owning the destination block (blk = destination).

struct halo_item_t
{
    int blk, dir;
    long long woff, boff;
};

template< bool MHD, class R, bool PACK >
__global__ void __launch_bounds__( 256 ) k_halo( const args_t< R > a, const halo_item_t * items,
                                                 R * wbuf, double * bbuf, int step )
{
    constexpr int NW = MHD ? 11 : 5;
    const halo_item_t m = items[ blockIdx.y ];
    const int s[ 3 ] = { m.dir % 3 - 1, ( m.dir / 3 ) % 3 - 1, m.dir / 9 - 1 };
    const int nn[ 3 ] = { a.n0, a.n1, a.n2 };
    int org[ 3 ], ext[ 3 ];
    for( int d = 0; d < 3; ++ d )
    {
        ext[ d ] = s[ d ] ? 2 : nn[ d ];
        org[ d ] = s[ d ] < 0 ? -2 : ( s[ d ] > 0 ? nn[ d ] : 0 );
    }
    const int sh[ 3 ] = { PACK ? s[ 0 ] * nn[ 0 ] : 0, PACK ? s[ 1 ] * nn[ 1 ] : 0, PACK ? s[ 2 ] * nn[ 2 ] : 0 };
    const long long cells = ( long long ) ext[ 0 ] * ext[ 1 ] * ext[ 2 ];
    const long long stride = ( long long ) gridDim.x * blockDim.x;
    const long long t0 = ( long long ) blockIdx.x * blockDim.x + threadIdx.x;
    for( long long t = t0; t < cells; t += stride )
    {
        const int i0 = org[ 0 ] + int( t % ext[ 0 ] ) - sh[ 0 ];
        const int i1 = org[ 1 ] + int( ( t / ext[ 0 ] ) % ext[ 1 ] ) - sh[ 1 ];
        const int i2 = org[ 2 ] + int( t / ( ( long long ) ext[ 0 ] * ext[ 1 ] ) ) - sh[ 2 ];
        for( int k = 0; k < NW; ++ k )
        {
            R * p = wbuf + m.woff + k * cells + t;
            R * q = a.w + iw( a, m.blk, k, NW, i0, i1, i2 );
            if( PACK ) * p = * q;
            else       * q = * p;
        }
    }
    if( ! MHD || abs( s[ 0 ] ) + abs( s[ 1 ] ) + abs( s[ 2 ] ) != 1 )
        return;
    const int d = s[ 0 ] ? 0 : ( s[ 1 ] ? 1 : 2 );
    double * BF = a.bf[ step ];
    long long off = m.boff;
    for( int h = 0; h < 2; ++ h )
    {
        const int c = ( d + 1 + h ) % 3, o = 3 - d - c;
        const long long cnt = ( long long )( nn[ c ] + 1 ) * nn[ o ];
        for( long long t = t0; t < cnt; t += stride )
        {
            int ii[ 3 ];
            ii[ c ] = int( t % ( nn[ c ] + 1 ) );
            ii[ o ] = int( t / ( nn[ c ] + 1 ) );
            ii[ d ] = ( s[ d ] < 0 ? -1 : nn[ d ] ) - sh[ d ];
            double * p = bbuf + off + t;
            double * q = BF + ibf( a, m.blk, c, ii[ 0 ], ii[ 1 ], ii[ 2 ] );
            if( PACK ) * p = * q;
            else       * q = * p;
        }
        off += cnt;
    }
}

// dt of a mesh split over several contexts in one process: the minimum of
// their stage-0 CFL minima, written back to each.
constexpr int KR_GROUP_MAX = 64;
struct group_scal_t { scal_t * s[ KR_GROUP_MAX ]; int n; };

__global__ void k_group_dt_min( group_scal_t g )
{
    unsigned long long m = ~0ull;
    for( int r = 0; r < g.n; ++ r )
    {
        const unsigned long long v = g.s[ r ]->dt_bits;
        m = v < m ? v : m;
    }
    for( int r = 0; r < g.n; ++ r )
        g.s[ r ]->dt_bits = m;
}

}   // namespace kr

////////////////////////////////////////////////////////////
// Context

using namespace kr;

////////////////////////////////////////////////////////////
// Sharding plan (host): block owners, neighbour ids, halo items

static int ranks_of( const kr_cfg & g ) { return g.n_ranks > 1 ? g.n_ranks : 1; }

// owner[g] for every global block: recursive coordinate bisection of the
// block grid into n_ranks boxes (largest extent first, ties to the outer axis;
// the lower part gets floor(ranks / 2) ranks and a proportional share).
static bool shard_owner( const kr_cfg & g, std::vector< int > & owner, std::string & err )
{
    const int R = ranks_of( g );
    const int nb0 = g.nb[ 0 ], nb1 = g.nb[ 1 ], nb2 = g.nb[ 2 ];
    owner.assign( size_t( nb0 ) * nb1 * nb2, 0 );
    struct box_t { int lo[ 3 ], hi[ 3 ], r0, r1; };
    std::vector< box_t > todo{ { { 0, 0, 0 }, { nb0, nb1, nb2 }, 0, R } };
    while( ! todo.empty(  ) )
    {
        const box_t b = todo.back(  );
        todo.pop_back(  );
        const int nr = b.r1 - b.r0;
        long long nblk = 1;
        for( int a = 0; a < 3; ++ a ) nblk *= b.hi[ a ] - b.lo[ a ];
        if( nblk < nr )
        {
            err = "kr_shard_owner: fewer blocks than ranks in a bisection box";
            return false;
        }
        if( nr == 1 )
        {
            for( int k = b.lo[ 2 ]; k < b.hi[ 2 ]; ++ k )
            for( int j = b.lo[ 1 ]; j < b.hi[ 1 ]; ++ j )
            for( int i = b.lo[ 0 ]; i < b.hi[ 0 ]; ++ i )
                owner[ i + size_t( nb0 ) * ( j + size_t( nb1 ) * k ) ] = b.r0;
            continue;
        }
        int ax = 2;
        for( int a = 1; a >= 0; -- a )
            if( b.hi[ a ] - b.lo[ a ] > b.hi[ ax ] - b.lo[ ax ] ) ax = a;
        const int ext = b.hi[ ax ] - b.lo[ ax ];
        const int k = nr / 2;
        int cut = b.lo[ ax ] + int( ( ( long long ) ext * k + nr / 2 ) / nr );
        cut = std::min( std::max( cut, b.lo[ ax ] + 1 ), b.hi[ ax ] - 1 );
        box_t lo = b, hi = b;
        lo.hi[ ax ] = cut; lo.r1 = b.r0 + k;
        hi.lo[ ax ] = cut; hi.r0 = b.r0 + k;
        todo.push_back( hi );
        todo.push_back( lo );
    }
    return true;
}

// Global neighbour of global block gb in direction k (0..26, x fastest), or
// -1 past a non-periodic side.
static int nbr_global( const kr_cfg & g, int gb, int k )
{
    const int reg[ 3 ] = { gb % g.nb[ 0 ], ( gb / g.nb[ 0 ] ) % g.nb[ 1 ], gb / ( g.nb[ 0 ] * g.nb[ 1 ] ) };
    const int sh[ 3 ] = { k % 3 - 1, ( k / 3 ) % 3 - 1, k / 9 - 1 };
    int r[ 3 ];
    for( int a = 0; a < 3; ++ a )
    {
        r[ a ] = reg[ a ] + sh[ a ];
        const bool periodic = g.bc[ 2 * a ] == KR_BC_PER && g.bc[ 2 * a + 1 ] == KR_BC_PER;
        if( ( r[ a ] < 0 || r[ a ] >= g.nb[ a ] ) && ! periodic )
            return -1;
        r[ a ] = ( r[ a ] + g.nb[ a ] ) % g.nb[ a ];
    }
    return r[ 0 ] + g.nb[ 0 ] * ( r[ 1 ] + g.nb[ 1 ] * r[ 2 ] );
}

// Words of one halo item: primitives over the ghost box of direction k, and
// for MHD face directions the two face-B strips.
static long long halo_w_words( const kr_cfg & g, int k )
{
    const int sh[ 3 ] = { k % 3 - 1, ( k / 3 ) % 3 - 1, k / 9 - 1 };
    long long cells = 1;
    for( int a = 0; a < 3; ++ a ) cells *= sh[ a ] ? 2 : g.n[ a ];
    return cells * ( g.mhd ? 11 : 5 );
}
static long long halo_b_words( const kr_cfg & g, int k )
{
    const int sh[ 3 ] = { k % 3 - 1, ( k / 3 ) % 3 - 1, k / 9 - 1 };
    if( ! g.mhd || std::abs( sh[ 0 ] ) + std::abs( sh[ 1 ] ) + std::abs( sh[ 2 ] ) != 1 )
        return 0;
    const int d = sh[ 0 ] ? 0 : ( sh[ 1 ] ? 1 : 2 );
    const int c1 = ( d + 1 ) % 3, c2 = ( d + 2 ) % 3;
    return ( long long )( g.n[ c1 ] + 1 ) * g.n[ c2 ] + ( long long )( g.n[ c2 ] + 1 ) * g.n[ c1 ];
}

// One side (send or receive) of a rank's exchange: items grouped by peer in
// the order both ends enumerate them -- destination blocks by ascending global
// id, directions 0..26.
struct halo_side_t
{
    std::vector< halo_item_t > items;
    std::vector< long long > w_off, w_cnt, b_off, b_cnt;   // per peer, words
    long long w_tot = 0, b_tot = 0;
};

static void halo_plan( const kr_cfg & g, const std::vector< int > & owner, const std::vector< int > & local,
                       bool all, halo_side_t & snd, halo_side_t & rcv )
{
    const int R = ranks_of( g ), me = ranks_of( g ) > 1 ? g.rank : 0;
    const int nglob = int( owner.size(  ) );
    for( halo_side_t * h : { & snd, & rcv } )
    {
        h->items.clear(  );
        h->w_off.assign( R, 0 ); h->w_cnt.assign( R, 0 );
        h->b_off.assign( R, 0 ); h->b_cnt.assign( R, 0 );
        h->w_tot = h->b_tot = 0;
    }
    for( int q = 0; q < R; ++ q )
    {
        if( q == me && ! all )
            continue;
        snd.w_off[ q ] = snd.w_tot; snd.b_off[ q ] = snd.b_tot;
        rcv.w_off[ q ] = rcv.w_tot; rcv.b_off[ q ] = rcv.b_tot;
        for( int gb = 0; gb < nglob; ++ gb )
        {
            const bool to_q = owner[ gb ] == q, mine = owner[ gb ] == me;
            if( ! to_q && ! mine )
                continue;
            for( int k = 0; k < 27; ++ k )
            {
                const int src = k == 13 ? -1 : nbr_global( g, gb, k );
                if( src < 0 )
                    continue;
                const long long wn = halo_w_words( g, k ), bn = halo_b_words( g, k );
                if( to_q && owner[ src ] == me )      // q's block gb reads my block src
                {
                    snd.items.push_back( { local[ src ], k, snd.w_tot, snd.b_tot } );
                    snd.w_tot += wn; snd.b_tot += bn;
                }
                if( mine && owner[ src ] == q )       // my block gb reads q's block src
                {
                    rcv.items.push_back( { local[ gb ], k, rcv.w_tot, rcv.b_tot } );
                    rcv.w_tot += wn; rcv.b_tot += bn;
                }
            }
        }
        snd.w_cnt[ q ] = snd.w_tot - snd.w_off[ q ]; snd.b_cnt[ q ] = snd.b_tot - snd.b_off[ q ];
        rcv.w_cnt[ q ] = rcv.w_tot - rcv.w_off[ q ]; rcv.b_cnt[ q ] = rcv.b_tot - rcv.b_off[ q ];
    }
}

////////////////////////////////////////////////////////////
// NCCL, loaded at run time: the library has no link dependency on it.  A copy
// of libnccl.so.2 already in the process (e.g. the one torch links) is used;
// else the file named by $KRATOS_B200_NCCL; else the one the dynamic linker
// finds.  Opened with local symbol scope.  A process holds one libnccl.so.2
// (one soname): a framework loaded later that links a newer NCCL than the one
// opened here fails to load, so name that framework's copy in the variable.

struct nccl_api_t
{
    bool ok = false;
    std::string err;
    decltype( & ncclGetUniqueId ) GetUniqueId = nullptr;
    decltype( & ncclCommInitRank ) CommInitRank = nullptr;
    decltype( & ncclCommDestroy ) CommDestroy = nullptr;
    decltype( & ncclGroupStart ) GroupStart = nullptr;
    decltype( & ncclGroupEnd ) GroupEnd = nullptr;
    decltype( & ncclSend ) Send = nullptr;
    decltype( & ncclRecv ) Recv = nullptr;
    decltype( & ncclAllReduce ) AllReduce = nullptr;
    decltype( & ncclGetErrorString ) GetErrorString = nullptr;
};

static nccl_api_t & nccl(  )
{
    static nccl_api_t api;
    static std::once_flag once;
    std::call_once( once, [](  )
    {
        void * h = dlopen( "libnccl.so.2", RTLD_NOW | RTLD_NOLOAD );
        const char * path = std::getenv( "KRATOS_B200_NCCL" );
        if( ! h && path && * path )
            h = dlopen( path, RTLD_NOW | RTLD_LOCAL );
        if( ! h )
            h = dlopen( "libnccl.so.2", RTLD_NOW | RTLD_LOCAL );
        if( ! h )
        {
            api.err = std::string( "dlopen libnccl.so.2: " ) + dlerror(  );
            return;
        }
        bool ok = true;
        auto sym = [ & ]( auto & fn, const char * name )
        {
            fn = reinterpret_cast< std::remove_reference_t< decltype( fn ) > >( dlsym( h, name ) );
            if( ! fn ) { ok = false; api.err = std::string( "libnccl.so.2 lacks " ) + name; }
        };
        sym( api.GetUniqueId, "ncclGetUniqueId" );
        sym( api.CommInitRank, "ncclCommInitRank" );
        sym( api.CommDestroy, "ncclCommDestroy" );
        sym( api.GroupStart, "ncclGroupStart" );
        sym( api.GroupEnd, "ncclGroupEnd" );
        sym( api.Send, "ncclSend" );
        sym( api.Recv, "ncclRecv" );
        sym( api.AllReduce, "ncclAllReduce" );
        sym( api.GetErrorString, "ncclGetErrorString" );
        api.ok = ok;
    } );
    return api;
}

#include "kr_smr_mhd.cuh"

struct kr_ctx
{
    kr_cfg cfg;
    std::string err;
    int nblk = 0, nw = 0, nws = 0, nf = 0;   // nw: host words / cell; nws: stored W words
    long long nc = 0, ngw = 0, nbf = 0, nfb = 0;
    size_t rsize = 8;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    // device memory
    double * u[ 2 ] = { nullptr, nullptr };
    double * bf[ 2 ] = { nullptr, nullptr };
    void * w = nullptr;
    // uniform MHD: stage 0's update and stage 1's c2p in one launch, in the
    // step graph (FP64, where it measured faster) and in batched launches
    bool fuse = false, fuse_batch = false;
    void * f[ 3 ] = { nullptr, nullptr, nullptr };
    void * ee = nullptr;
    geo_t * geo = nullptr;
    int * nbr = nullptr;
    scal_t * s = nullptr;
    double * stage = nullptr;          // host-layout staging buffer (device)
    size_t stage_bytes = 0;
    double * diag = nullptr;
    // learned selector
    unsigned * sel_w = nullptr;
    float * sel_b = nullptr;
    unsigned long long * sel_cnt = nullptr;
    float sel_thr = 0.f;
    bool sel_ready = false;
    unsigned * sel_dec = nullptr;     // learned mode: solver per face, a mask per warp
    long long sel_wcap = 0;
    // selector training samples (only during kr_selector_collect)
    float * smp = nullptr;
    unsigned long long * smp_n = nullptr;
    long long smp_max = 0;
    unsigned smp_stride = 1, smp_seed = 0;
    // graph of one step
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    cudaStream_t graph_stream = nullptr;
    std::vector< geo_t > geo_h;
    int n_sm = 148;                    // multiprocessors of the device
    // sharding: this rank's blocks and the halo exchange with the others
    int nranks = 1, rank = 0;
    std::vector< int > gid_h;          // global id of each local block
    int * gid = nullptr;
    halo_side_t hsend, hrecv;
    halo_item_t * send_items = nullptr;
    halo_item_t * recv_items = nullptr;
    void * send_w = nullptr;           // R words
    void * recv_w = nullptr;
    double * send_b = nullptr;
    double * recv_b = nullptr;
    int halo_grid = 1;                 // CTAs per item of k_halo
    ncclComm_t comm = nullptr;
    // static refinement (hydro, one rank): blocks are the tree's leaves
    bool smr = false;
    int max_level = 0;
    bool boxes = false;                // KR_FLAG_BOXES: independent periodic boxes
    int nscal = 1;                     // scalar sets (one per box in that mode)
    std::vector< int > lvl_h, reg_h;   // per block: level, logical position (3)
    smr_item_t * smr_items = nullptr;  // [restriction / flux-average items | prolongation items by level]
    double * favg = nullptr;           // averaged fine fluxes of the flux-average items
    int n_restrict = 0;
    std::vector< int > prolong_off;    // prolongation items of level l: [prolong_off[l - 1], prolong_off[l])
    // refined MHD: the exchange holders (kr_smr_mhd.cuh)
    mh_t * mh_list = nullptr;
    uint2 * mh_work = nullptr;         // (holder, item) per thread, phase by phase
    int mh_restrict[ 2 ] = { 0, 0 };   // work-item range
    std::vector< int > mh_prolong, mh_waves;
};

static thread_local std::string g_create_error;

// FP32 selector parameters -> per-lane bf16 fragment words + biases (kr_learn.cu)
void kr_mlp_pack( const float * w, std::vector< unsigned > & words, std::vector< float > & bias );

static bool ck( kr_ctx * c, cudaError_t e, const char * what )
{
    if( e == cudaSuccess )
        return true;
    if( c )
        c->err = std::string( what ) + ": " + cudaGetErrorString( e );
    else
        g_create_error = std::string( what ) + ": " + cudaGetErrorString( e );
    return false;
}

static long long smr_half_sites( const kr_ctx * c )
{   // largest (n1 / 2) x (n2 / 2) over the three face orientations
    const int * n = c->cfg.n;
    return std::max( { ( long long )( n[ 1 ] / 2 ) * ( n[ 2 ] / 2 ), ( long long )( n[ 0 ] / 2 ) * ( n[ 2 ] / 2 ),
                       ( long long )( n[ 0 ] / 2 ) * ( n[ 1 ] / 2 ) } );
}

template< class R >
static args_t< R > make_args( kr_ctx * c )
{
    args_t< R > a;
    const int * n = c->cfg.n;
    a.n0 = n[ 0 ]; a.n1 = n[ 1 ]; a.n2 = n[ 2 ]; a.nblk = c->nblk;
    a.nc = c->nc; a.ngw = c->ngw; a.nbf = c->nbf; a.nfb = c->nfb;
    a.sw1 = n[ 0 ] + 4; a.sw2 = ( n[ 0 ] + 4 ) * ( n[ 1 ] + 4 );
    a.sb1 = n[ 0 ] + 5; a.sb2 = ( n[ 0 ] + 5 ) * ( n[ 1 ] + 5 );
    a.sf1 = n[ 0 ] + 3; a.sf2 = ( n[ 0 ] + 3 ) * ( n[ 1 ] + 3 );
    a.gamma = c->cfg.gamma; a.cfl = c->cfg.cfl;
    a.gm1 = c->cfg.gamma - 1; a.cv = 1 / ( c->cfg.gamma - 1 );
    a.d_floor = c->cfg.rho_floor; a.t_floor = c->cfg.tmp_floor;
    a.dt_expand = c->cfg.dt_expand;
    for( int s = 0; s < 2; ++ s ) { a.u[ s ] = c->u[ s ]; a.bf[ s ] = c->bf[ s ]; }
    a.w = ( R * ) c->w;
    for( int d = 0; d < 3; ++ d ) a.f[ d ] = ( R * ) c->f[ d ];
    a.ee = ( R * ) c->ee;
    a.geo = c->geo; a.nbr = c->nbr; a.gid = c->gid; a.s = c->s; a.boxes = c->boxes;
    a.favg = c->favg; a.favg_n = int( smr_half_sites( c ) );
    a.mh_smr = c->smr && c->cfg.mhd;
    for( int d = 0; d < 3; ++ d ) a.nbk[ d ] = c->cfg.nb[ d ];
    for( int k = 0; k < 6; ++ k ) a.bc[ k ] = c->cfg.bc[ k ];
    for( int k = 0; k < 5; ++ k ) a.w_fix[ k ] = c->cfg.w_fix[ k ];
    for( int k = 0; k < 3; ++ k ) a.b_fix[ k ] = c->cfg.b_fix[ k ];
    a.vl2 = c->cfg.integrator == KR_INTEGRATOR_VL2;
    a.emf_out = 0;
    for( int d = 0; d < 3; ++ d )
        if( c->cfg.bc[ 2 * d + 1 ] == KR_BC_OUT || c->cfg.bc[ 2 * d + 1 ] == KR_BC_FRE )
            a.emf_out |= 1 << d;
    a.sel_w = c->sel_w; a.sel_b = c->sel_b; a.sel_thr = c->sel_thr; a.sel_cnt = c->sel_cnt;
    a.sel_dec = c->sel_dec; a.sel_wcap = c->sel_wcap;
    a.sel_period = c->cfg.sel_period > 1 ? c->cfg.sel_period : 1;
    a.smp = c->smp; a.smp_n = c->smp_n; a.smp_max = c->smp_max;
    a.smp_stride = c->smp_stride; a.smp_seed = c->smp_seed;
    return a;
}

static inline unsigned blocks_for( long long n, int th ) { return unsigned( ( n + th - 1 ) / th ); }

static bool has_phys( const kr_ctx * c )
{
    for( int k = 0; k < 6; ++ k )
        if( c->cfg.bc[ k ] != KR_BC_PER )
            return true;
    return false;
}

static long long phys_sites( const kr_ctx * c )
{   // largest transverse face count of a side
    const int * n = c->cfg.n;
    return std::max( { ( long long ) n[ 1 ] * n[ 2 ], ( long long ) n[ 0 ] * n[ 2 ], ( long long ) n[ 0 ] * n[ 1 ] } );
}

template< bool MHD, class R, int MODE, int axis >
static void launch_flux_axis( kr_ctx * c, cudaStream_t st, const args_t< R > & a, int stage )
{
    // one thread per face of the sweep, the MHD transverse ghost lines included
    const int * n = c->cfg.n;
    int ext[ 3 ];
    for( int d = 0; d < 3; ++ d )
        ext[ d ] = ( d == axis ) ? n[ d ] + 1 : n[ d ] + ( MHD ? 2 : 0 );
    if constexpr( MODE == KR_RIEMANN_LEARNED && MHD )
    {
        const unsigned cpp = blocks_for( ( long long ) ext[ 0 ] * ext[ 1 ], 128 );
        const unsigned ge = unsigned( std::max< long long >( 1, std::min< long long >(
            ( long long ) cpp * ext[ 2 ], ( 2LL * c->n_sm * flux_min_ctas< R, KR_RIEMANN_LEARNED >(  ) ) / c->nblk ) ) );
        k_flux_eval< MHD, R, axis ><<< dim3( ge, 1, c->nblk ), 128, 0, st >>>(
            a, stage, make_udiv( unsigned( ext[ 0 ] ) ), cpp, unsigned( ext[ 2 ] ) );
    }
    // sweeps without the network: each warp of faces runs the solver chosen
    // for it (exits at once on the network's sweep)
    constexpr int M = ( MODE == KR_RIEMANN_LEARNED && MHD ) ? FLUX_APPLY : MODE;
    const dim3 grid( blocks_for( ( long long ) ext[ 0 ] * ext[ 1 ], 128 ), ext[ 2 ], c->nblk );
    if constexpr( MHD && ( MODE == KR_RIEMANN_DEFAULT || MODE == KR_RIEMANN_HLLE ) )
        if( c->smr )
        {   // one flat index over each block's faces (flux_faces, XL)
            const dim3 flat( blocks_for( ( long long ) ext[ 0 ] * ext[ 1 ] * ext[ 2 ], 128 ), 1, c->nblk );
            k_flux< MHD, R, M, true, axis ><<< flat, 128, 0, st >>>( a, stage, make_udiv( unsigned( ext[ 0 ] ) ) );
            return;
        }
    k_flux< MHD, R, M, false, axis ><<< grid, 128, 0, st >>>( a, stage, make_udiv( unsigned( ext[ 0 ] ) ) );
}

template< bool MHD, class R, int MODE >
static void launch_flux( kr_ctx * c, cudaStream_t st, const args_t< R > & a, int axis, int stage )
{
    if( axis == 0 )      launch_flux_axis< MHD, R, MODE, 0 >( c, st, a, stage );
    else if( axis == 1 ) launch_flux_axis< MHD, R, MODE, 1 >( c, st, a, stage );
    else                 launch_flux_axis< MHD, R, MODE, 2 >( c, st, a, stage );
}

template< bool MHD, class R >
static void launch_flux_mode( kr_ctx * c, cudaStream_t st, const args_t< R > & a, int axis,
                              int stage, int mode )
{
    if( mode == FLUX_SAMPLE )                   launch_flux< MHD, R, FLUX_SAMPLE >( c, st, a, axis, stage );
    else if( mode == KR_RIEMANN_LEARNED && MHD ) launch_flux< MHD, R, KR_RIEMANN_LEARNED >( c, st, a, axis, stage );
    else if( mode == KR_RIEMANN_HLLE && MHD )    launch_flux< MHD, R, KR_RIEMANN_HLLE >( c, st, a, axis, stage );
    else                                          launch_flux< MHD, R, KR_RIEMANN_DEFAULT >( c, st, a, axis, stage );
}

// One stage is front (cons -> prim, CFL dt at stage 0, pack of the halo other
// ranks read), exchange (NCCL send / receive by peer; at stage 0 the dt
// all-reduce), back (unpack, same-rank ghosts, physical sides, flux sweeps,
// EMF, update).  `timed( kind, launch )` wraps each piece (profiling: kinds
// 0 c2p, 1 ghost and halo, 2..4 flux z, y, x, 5 emf, 6 update).
struct untimed_t { template< class F > void operator(  )( int, F && f ) const { f(  ); } };

// One phase of the refined-MHD exchange: work items [i0, i1) of the plan.
template< class R, int KIND >
static void launch_mh( kr_ctx * c, cudaStream_t st, const args_t< R > & a, int i0, int i1, int stage )
{
    if( i1 > i0 )
        k_mh< R, KIND ><<< blocks_for( i1 - i0, 256 ), 256, 0, st >>>( a, c->mh_list, c->mh_work + i0, i1 - i0, stage );
}

template< bool MHD, class R, class T >
static void enqueue_front( kr_ctx * c, cudaStream_t st, const args_t< R > & a, int stage, T && timed )
{
    const unsigned nb = unsigned( c->nblk );
    const int * n = c->cfg.n;
    if( ! ( c->fuse && stage == 1 ) )        // (fused: stage 0's update did stage 1's c2p)
        timed( 0, [ & ] { ( stage == 0 ? k_c2p< MHD, R, true > : k_c2p< MHD, R, false > )<<< dim3( blocks_for( ( long long ) n[ 0 ] * n[ 1 ], 256 ), n[ 2 ], nb ), 256, 0, st >>>(
            a, stage, make_udiv( unsigned( n[ 0 ] ) ) ); } );
    if( ! c->hsend.items.empty(  ) )
        timed( 1, [ & ] {
            k_halo< MHD, R, true ><<< dim3( c->halo_grid, unsigned( c->hsend.items.size(  ) ) ), 256, 0, st >>>(
                a, c->send_items, ( R * ) c->send_w, c->send_b, stage ); } );
}

template< bool MHD, class R, class T >
static void enqueue_back( kr_ctx * c, cudaStream_t st, const args_t< R > & a, int stage, int mode, T && timed )
{
    const int * n = c->cfg.n;
    const unsigned nb = unsigned( c->nblk );
    timed( 1, [ & ] {
        if( ! c->hrecv.items.empty(  ) )
            k_halo< MHD, R, false ><<< dim3( c->halo_grid, unsigned( c->hrecv.items.size(  ) ) ), 256, 0, st >>>(
                a, c->recv_items, ( R * ) c->recv_w, c->recv_b, stage );
        // (the same-level ghost fill happens in k_c2p and k_update: push)
        if( MHD && c->mh_list )
        {   // refined MHD: every ghost by the exchange holders (keeper.cpp:148-160
            // act_bnd: restrictions, same-level copies, prolongations by the
            // coarser host's level, the restrictions' second pass)
            auto sides = [ & ]( int field )
            {   // keeper.cpp:148-157 and mhd/boundary/keeper.h:304-309
                for( int side = 0; side < 6; ++ side )
                    if( c->cfg.bc[ side ] != KR_BC_PER )
                    {
                        const int ax = side / 2;
                        const long long rows = ( long long )( n[ ( ax + 1 ) % 3 ] + 4 ) * ( n[ ( ax + 2 ) % 3 ] + 4 );
                        k_phys_mhd< R ><<< dim3( blocks_for( rows, 128 ), nb ), 128, 0, st >>>( a, side, stage, field );
                    }
            };
            // (the same-level copies were pushed by k_c2p and the CT update)
            launch_mh< R, MH_RESTRICT >( c, st, a, c->mh_restrict[ 0 ], c->mh_restrict[ 1 ], stage );
            sides( 1 );
            for( size_t l = 0; l + 1 < c->mh_prolong.size(  ); ++ l )
                launch_mh< R, MH_PROLONG >( c, st, a, c->mh_prolong[ l ], c->mh_prolong[ l + 1 ], stage );
            // (the reference's second restriction pass, keeper.cpp:121-127,
            // rewrites the same values: its inputs are finer interiors, which
            // nothing in between changes, with blocks of >= 4 cells per axis)
            sides( 0 );
            return;
        }
        if( c->n_restrict )            // finer -> coarser ghosts
            k_restrict< R ><<< dim3( blocks_for( 2 * smr_half_sites( c ), 128 ), c->n_restrict ), 128, 0, st >>>( a, c->smr_items );
        if( ! MHD && has_phys( c ) )
            k_phys< R ><<< dim3( blocks_for( phys_sites( c ), 128 ), 6, nb ), 128, 0, st >>>( a );
        for( int l = 1; l <= c->max_level; ++ l )
        {   // coarser -> finer ghosts, coarser levels first
            const int i0 = c->prolong_off[ l - 1 ], cnt = c->prolong_off[ l ] - i0;
            if( cnt )
                k_prolong< R ><<< dim3( blocks_for( smr_half_sites( c ), 128 ), cnt ), 128, 0, st >>>( a, c->smr_items + i0 );
        }
        if( MHD )
            for( int side = 0; side < 6; ++ side )
                if( c->cfg.bc[ side ] != KR_BC_PER )
                {
                    const int ax = side / 2;
                    const long long rows = ( long long )( n[ ( ax + 1 ) % 3 ] + 4 ) * ( n[ ( ax + 2 ) % 3 ] + 4 );
                    k_phys_mhd< R ><<< dim3( blocks_for( rows, 128 ), nb ), 128, 0, st >>>( a, side, stage );
                } } );
    for( int axis = 2; axis >= 0; -- axis )
        timed( 4 - axis, [ & ] { launch_flux_mode< MHD, R >( c, st, a, axis, stage, mode ); } );
    if( MHD )
        timed( 5, [ & ] { k_emf< R ><<< dim3( blocks_for( ( long long )( n[ 0 ] + 1 ) * ( n[ 1 ] + 1 ), 256 ), n[ 2 ] + 1, nb ), 256, 0, st >>>(
            a, make_udiv( unsigned( n[ 0 ] + 1 ) ) ); } );
    const dim3 ug( blocks_for( ( long long )( n[ 0 ] + 1 ) * ( n[ 1 ] + 1 ), 256 ), n[ 2 ] + 1, nb );
    if constexpr( MHD )
        if( c->smr )
        {   // refined MHD (dynamics.h:80-99): the coarse face flux over a
            // refined side, the edge-E correction in waves, then the update
            timed( 6, [ & ] {
                if( c->n_restrict )
                    k_flux_avg< R, 7 ><<< dim3( blocks_for( smr_half_sites( c ), 128 ), c->n_restrict ), 128, 0, st >>>( a, c->smr_items );
                for( size_t w = 0; w + 1 < c->mh_waves.size(  ); ++ w )
                    launch_mh< R, MH_FLUX >( c, st, a, c->mh_waves[ w ], c->mh_waves[ w + 1 ], stage );
                k_update< MHD, R, true, 1 ><<< ug, 256, 0, st >>>( a, stage, make_udiv( unsigned( n[ 0 ] + 1 ) ) );
                k_update< MHD, R, false, 2 ><<< ug, 256, 0, st >>>( a, stage, make_udiv( unsigned( n[ 0 ] + 1 ) ) ); } );
            return;
        }
    if constexpr( ! MHD )
        if( c->smr )
        {
            timed( 6, [ & ] {
                if( c->n_restrict )      // coarse face flux over a refined side
                    k_flux_avg< R ><<< dim3( blocks_for( smr_half_sites( c ), 128 ), c->n_restrict ), 128, 0, st >>>( a, c->smr_items );
                k_update< MHD, R, true ><<< ug, 256, 0, st >>>( a, stage, make_udiv( unsigned( n[ 0 ] + 1 ) ) ); } );
            return;
        }
    timed( 6, [ & ] {
        if( MHD && c->fuse && stage == 0 )      // update, CT and stage 1's c2p
            k_update_c2p< R ><<< dim3( blocks_for( ( long long ) n[ 0 ] * n[ 1 ], 256 ), n[ 2 ], nb ), 256, 0, st >>>(
                a, make_udiv( unsigned( n[ 0 ] ) ) );
        else if( MHD )
        {
            k_update< MHD, R, false, 1 ><<< ug, 256, 0, st >>>( a, stage, make_udiv( unsigned( n[ 0 ] + 1 ) ) );
            k_update< MHD, R, false, 2 ><<< ug, 256, 0, st >>>( a, stage, make_udiv( unsigned( n[ 0 ] + 1 ) ) );
        }
        else
            k_update< MHD, R ><<< ug, 256, 0, st >>>( a, stage, make_udiv( unsigned( n[ 0 ] + 1 ) ) ); } );
}

// Halo transfer of one stage between this rank and its peers, and at stage 0
// the global dt minimum.  Same-rank items without a communicator (the
// KR_FLAG_HALO_ALL check of one unsharded context) are device copies.
static bool enqueue_exchange( kr_ctx * c, cudaStream_t st, int stage )
{
    const size_t rs = c->rsize;
    if( ! c->comm && c->hsend.items.empty(  ) && c->hrecv.items.empty(  ) )
        return true;                     // nothing to move; NCCL never loaded
    nccl_api_t * api = c->comm ? & nccl(  ) : nullptr;
    bool grouped = false;
    ncclResult_t r = ncclSuccess;
    for( int q = 0; q < c->nranks; ++ q )
    {
        const long long sw = c->hsend.w_cnt[ q ], sb = c->hsend.b_cnt[ q ];
        const long long rw = c->hrecv.w_cnt[ q ], rb = c->hrecv.b_cnt[ q ];
        if( ! ( sw || sb || rw || rb ) )
            continue;
        char * sW = ( char * ) c->send_w + c->hsend.w_off[ q ] * rs;
        char * rW = ( char * ) c->recv_w + c->hrecv.w_off[ q ] * rs;
        double * sB = c->send_b + c->hsend.b_off[ q ];
        double * rB = c->recv_b + c->hrecv.b_off[ q ];
        if( q == c->rank && ! c->comm )
        {   // send and receive lists to oneself coincide item by item
            if( sw && ! ck( c, cudaMemcpyAsync( rW, sW, sw * rs, cudaMemcpyDeviceToDevice, st ), "halo copy" ) ) return false;
            if( sb && ! ck( c, cudaMemcpyAsync( rB, sB, sb * 8, cudaMemcpyDeviceToDevice, st ), "halo copy" ) ) return false;
            continue;
        }
        if( ! c->comm )
        {
            c->err = "sharded context without a communicator (call kr_comm_init)";
            return false;
        }
        if( ! grouped ) { r = api->GroupStart(  ); grouped = true; }
        const ncclDataType_t tw = rs == 4 ? ncclFloat32 : ncclFloat64;
        if( sw && r == ncclSuccess ) r = api->Send( sW, size_t( sw ), tw, q, c->comm, st );
        if( sb && r == ncclSuccess ) r = api->Send( sB, size_t( sb ), ncclFloat64, q, c->comm, st );
        if( rw && r == ncclSuccess ) r = api->Recv( rW, size_t( rw ), tw, q, c->comm, st );
        if( rb && r == ncclSuccess ) r = api->Recv( rB, size_t( rb ), ncclFloat64, q, c->comm, st );
    }
    if( grouped )
    {
        const ncclResult_t e = api->GroupEnd(  );
        if( r == ncclSuccess ) r = e;
    }
    if( stage == 0 && c->comm && r == ncclSuccess )   // cycle.cpp:77-95 reduce_all(min)
        r = api->AllReduce( & c->s->dt_bits, & c->s->dt_bits, 1, ncclUint64, ncclMin, c->comm, st );
    if( r != ncclSuccess )
    {
        c->err = std::string( "NCCL: " ) + api->GetErrorString( r );
        return false;
    }
    return true;
}

// Enqueue one Heun step on stream st (SAMPLE: also log selector training samples).
template< bool MHD, class R, bool SAMPLE = false >
static bool enqueue_step( kr_ctx * c, cudaStream_t st )
{
    const args_t< R > a = make_args< R >( c );
    k_step_begin<<< 1, 1, 0, st >>>( c->s, c->nscal );
    for( int stage = 0; stage < 2; ++ stage )
    {
        enqueue_front< MHD, R >( c, st, a, stage, untimed_t(  ) );
        if( ! enqueue_exchange( c, st, stage ) )
            return false;
        enqueue_back< MHD, R >( c, st, a, stage, SAMPLE ? FLUX_SAMPLE : c->cfg.riemann, untimed_t(  ) );
    }
    k_step_end<<< 1, 1, 0, st >>>( c->s, c->cfg.dt_expand, c->nscal );
    return true;
}

// One step launched eagerly with CUDA events around every kernel; per kind
// the summed milliseconds of the step are added to ms[kind].
template< bool MHD, class R >
static bool profile_step( kr_ctx * c, double * ms )
{
    const args_t< R > a = make_args< R >( c );
    cudaStream_t st = c->stream;
    cudaEvent_t ev[ 2 ];
    cudaEventCreate( & ev[ 0 ] );
    cudaEventCreate( & ev[ 1 ] );
    auto timed = [ & ]( int kind, auto && launch )
    {
        cudaEventRecord( ev[ 0 ], st );
        launch(  );
        cudaEventRecord( ev[ 1 ], st );
        cudaEventSynchronize( ev[ 1 ] );
        float t = 0;
        cudaEventElapsedTime( & t, ev[ 0 ], ev[ 1 ] );
        ms[ kind ] += t;
    };
    bool ok = true;
    k_step_begin<<< 1, 1, 0, st >>>( c->s, c->nscal );
    for( int stage = 0; stage < 2 && ok; ++ stage )
    {
        enqueue_front< MHD, R >( c, st, a, stage, timed );
        timed( 1, [ & ] { ok = enqueue_exchange( c, st, stage ); } );
        if( ok )
            enqueue_back< MHD, R >( c, st, a, stage, c->cfg.riemann, timed );
    }
    k_step_end<<< 1, 1, 0, st >>>( c->s, c->cfg.dt_expand, c->nscal );
    cudaEventDestroy( ev[ 0 ] );
    cudaEventDestroy( ev[ 1 ] );
    return ck( c, cudaStreamSynchronize( st ), "profile" ) && ok;
}

static bool enqueue_step_any( kr_ctx * c, cudaStream_t st )
{
    if( c->cfg.mhd )
        return c->cfg.precision == 1 ? enqueue_step< true, float >( c, st ) : enqueue_step< true, double >( c, st );
    return c->cfg.precision == 1 ? enqueue_step< false, float >( c, st ) : enqueue_step< false, double >( c, st );
}

static void drop_graph( kr_ctx * c )
{
    if( c->graph_exec ) cudaGraphExecDestroy( c->graph_exec );
    if( c->graph ) cudaGraphDestroy( c->graph );
    c->graph_exec = nullptr;
    c->graph = nullptr;
    c->graph_stream = nullptr;
}

static bool build_graph( kr_ctx * c )
{
    drop_graph( c );
    if( ! ck( c, cudaStreamBeginCapture( c->stream, cudaStreamCaptureModeThreadLocal ), "capture begin" ) )
        return false;
    const bool ok = enqueue_step_any( c, c->stream );
    const bool ended = ck( c, cudaStreamEndCapture( c->stream, & c->graph ), "capture end" );
    if( ! ok || ! ended )
    {
        const std::string e = c->err;
        drop_graph( c );
        c->err = e;
        return false;
    }
    if( ! ck( c, cudaGraphInstantiate( & c->graph_exec, c->graph, 0 ), "graph instantiate" ) )
        return false;
    c->graph_stream = c->stream;
    return true;
}

// The configuration the block geometry follows: independent boxes are each
// the whole domain (one block per axis).
static kr_cfg geo_cfg( const kr_ctx * c )
{
    kr_cfg g = c->cfg;
    if( c->boxes )
        g.nb[ 0 ] = g.nb[ 1 ] = g.nb[ 2 ] = 1;
    return g;
}

// Geometry exactly as meshgen computes it (meshgen.cpp:252-363).
static void set_geometry( kr_ctx * c )
{
    const kr_cfg g = geo_cfg( c );
    c->geo_h.resize( c->nblk );
    for( int b = 0; b < c->nblk; ++ b )
    {
        const int * reg = & c->reg_h[ 3 * b ];
        const int lvl = c->lvl_h[ b ];
        geo_t & o = c->geo_h[ b ];
        o.phys = o.fine = o.xlev = 0;
        for( int f = 0; f < 6; ++ f ) o.fitem[ f ] = -1;
        for( int side = 0; side < 6; ++ side )
            if( g.bc[ side ] != KR_BC_PER && reg[ side / 2 ] == ( side & 1 ? ( g.nb[ side / 2 ] << lvl ) - 1 : 0 ) )
                o.phys |= 1 << side;
        for( int a = 0; a < 3; ++ a )
        {   // loc(i) = location( ( reg + i / n ) / ( i_logic_lim << level ) )
            const double lim = double( g.nb[ a ] << lvl );
            const double x0 = ( reg[ a ] + 0.0 / g.n[ a ] ) / lim;
            const double x1 = ( reg[ a ] + 1.0 / g.n[ a ] ) / lim;
            const double l0 = g.x_min[ a ] + x0 * ( g.x_max[ a ] - g.x_min[ a ] );
            const double l1 = g.x_min[ a ] + x1 * ( g.x_max[ a ] - g.x_min[ a ] );
            o.dx[ a ] = l1 - l0;
            o.idx[ a ] = 1 / o.dx[ a ];
        }
        double vol = 1.;
        for( int a = 0; a < 3; ++ a )
        {
            double s = 1.;
            s *= o.dx[ ( a + 1 ) % 3 ];
            s *= o.dx[ ( a + 2 ) % 3 ];
            o.sfc[ a ] = s;
            o.isfc[ a ] = s > 0 ? 1 / s : 0.;
            vol *= o.dx[ a ];
        }
        o.vol = vol;
    }
}

// Cell centre of cell i along axis a of a block at `reg` on level lvl.
static double x_cc( const kr_cfg & g, const int * reg, int lvl, int a, int i )
{
    const double lim = double( g.nb[ a ] << lvl );
    const double x0 = ( reg[ a ] + 0.0 / g.n[ a ] ) / lim;
    const double x1 = ( reg[ a ] + 1.0 / g.n[ a ] ) / lim;
    const double l0 = g.x_min[ a ] + x0 * ( g.x_max[ a ] - g.x_min[ a ] );
    const double l1 = g.x_min[ a ] + x1 * ( g.x_max[ a ] - g.x_min[ a ] );
    return l0 + ( i + 0.5f ) * ( l1 - l0 );
}

extern "C" {

void kr_cfg_default( kr_cfg * g )
{
    std::memset( g, 0, sizeof( * g ) );
    g->abi_version = KR_ABI_VERSION;
    g->precision = 2;
    for( int a = 0; a < 3; ++ a ) { g->nb[ a ] = 1; g->n[ a ] = 16; g->x_max[ a ] = 1; }
    g->gamma = 1.66667;
    g->cfl = 0.3;
    g->rho_floor = 1e-9;
    g->tmp_floor = 1e-9;
    g->dt_expand = 2;
}

const char * kr_last_error( const kr_ctx * c )
{
    return c ? c->err.c_str(  ) : g_create_error.c_str(  );
}

}   // extern "C"

// The tree of a refined mesh (meshgen.cpp:111-160 load_refinement /
// generate_tree); false with g_create_error set on a bad region or setup.
static bool build_tree( const kr_cfg * cfg, int n_regions, const kr_region * regions, kr_tree & tree )
{
    int per[ 3 ];
    for( int a = 0; a < 3; ++ a )
        per[ a ] = cfg->bc[ 2 * a ] == KR_BC_PER && cfg->bc[ 2 * a + 1 ] == KR_BC_PER;
    std::vector< kr_tree_region > rg( std::max( 1, n_regions ) );
    for( int k = 0; k < n_regions; ++ k )
    {
        rg[ k ].level = regions[ k ].level;
        for( int a = 0; a < 3; ++ a )
        {
            rg[ k ].x_min[ a ] = regions[ k ].x_min[ a ];
            rg[ k ].x_max[ a ] = regions[ k ].x_max[ a ];
        }
    }
    char err[ 128 ] = { 0 };
    if( kr_tree_build( & tree, cfg->nb, per, cfg->x_min, cfg->x_max, n_regions, rg.data(  ), err, sizeof( err ) - 1 ) != 0 )
    {
        g_create_error = std::string( "kr_ctx_create_refined: " ) + err;
        return false;
    }
    if( tree.max_level == 0 )
        return true;
    const char * why = nullptr;
    if( cfg->mhd && cfg->riemann == KR_RIEMANN_LEARNED )
        why = "the learned face selector runs on uniform meshes";
    else if( ranks_of( * cfg ) > 1 || ( cfg->flags & KR_FLAG_HALO_ALL ) )
        why = "static refinement runs on one rank, without KR_FLAG_HALO_ALL";
    else if( cfg->n[ 0 ] % 2 || cfg->n[ 1 ] % 2 || cfg->n[ 2 ] % 2 )
        why = "static refinement needs an even number of cells per block along every axis";
    if( why )
    {
        g_create_error = std::string( "kr_ctx_create_refined: " ) + why;
        kr_tree_free( & tree );
        return false;
    }
    return true;
}

// Restriction / flux-average items (coarse block, side, child) and the
// prolongation items (fine block, side) of each level, from the tree.
static void smr_plan( const kr_tree & t, const int * n, std::vector< smr_item_t > & items, int & n_restrict,
                      std::vector< int > & prolong_off )
{
    items.clear(  );
    for( int b = 0; b < t.nblk; ++ b )
        for( int f = 0; f < 6; ++ f )
            if( t.face[ 6 * b + f ] == KR_FACE_FINE )
            {
                const int a = f / 2, h1 = n[ ( a + 1 ) % 3 ] / 2, h2 = n[ ( a + 2 ) % 3 ] / 2;
                for( int d = 0; d < 4; ++ d )
                    items.push_back( { b, t.fnb[ ( 6 * b + f ) * 4 + d ], f, ( d >> 1 ) * h1, ( d & 1 ) * h2 } );
            }
    n_restrict = int( items.size(  ) );
    prolong_off.assign( 1, n_restrict );
    for( int l = 1; l <= t.max_level; ++ l )
    {
        for( int b = 0; b < t.nblk; ++ b )
        {
            if( t.level[ b ] != l )
                continue;
            for( int f = 0; f < 6; ++ f )
                if( t.face[ 6 * b + f ] == KR_FACE_COARSE )
                {
                    const int a = f / 2, a1 = ( a + 1 ) % 3, a2 = ( a + 2 ) % 3;
                    const int * r = t.reg + 3 * b;
                    items.push_back( { b, t.fnb[ ( 6 * b + f ) * 4 ], f, ( r[ a1 ] & 1 ) * ( n[ a1 ] / 2 ),
                                       ( r[ a2 ] & 1 ) * ( n[ a2 ] / 2 ) } );
                }
        }
        prolong_off.push_back( int( items.size(  ) ) );
    }
}

static kr_ctx * create_ctx( const kr_cfg * cfg, int n_regions, const kr_region * regions )
{
    g_create_error.clear(  );
    if( ! cfg || cfg->abi_version != KR_ABI_VERSION )
    {
        g_create_error = "kr_ctx_create: missing config or ABI version mismatch";
        return nullptr;
    }
    for( int a = 0; a < 3; ++ a )
        if( cfg->n[ a ] < 4 || cfg->nb[ a ] < 1 )
        {
            g_create_error = "kr_ctx_create: need n >= 4 cells and nb >= 1 blocks per axis";
            return nullptr;
        }
    if( cfg->precision != 1 && cfg->precision != 2 )
    {
        g_create_error = "kr_ctx_create: precision must be 1 (mixed) or 2 (FP64)";
        return nullptr;
    }
    for( int k = 0; k < 6; ++ k )
        if( cfg->bc[ k ] < KR_BC_PER || cfg->bc[ k ] > KR_BC_FIXD )
        {
            g_create_error = "kr_ctx_create: boundary kinds must be kr_bc_t";
            return nullptr;
        }
    for( int a = 0; a < 3; ++ a )
        if( ( cfg->bc[ 2 * a ] == KR_BC_PER ) != ( cfg->bc[ 2 * a + 1 ] == KR_BC_PER ) )
        {
            g_create_error = "kr_ctx_create: a periodic axis needs both sides periodic";
            return nullptr;
        }
    if( cfg->riemann != KR_RIEMANN_DEFAULT && ! cfg->mhd )
    {
        g_create_error = "kr_ctx_create: HLLE / learned selection is MHD only";
        return nullptr;
    }
    if( cfg->integrator != KR_INTEGRATOR_RK2 && cfg->integrator != KR_INTEGRATOR_VL2 )
    {
        g_create_error = "kr_ctx_create: integrator must be KR_INTEGRATOR_RK2 or KR_INTEGRATOR_VL2";
        return nullptr;
    }
    if( cfg->n_ranks < 0 || cfg->n_ranks > 65536 || ( cfg->n_ranks > 1 && ( cfg->rank < 0 || cfg->rank >= cfg->n_ranks ) ) )
    {
        g_create_error = "kr_ctx_create: need 0 <= rank < n_ranks";
        return nullptr;
    }
    if( n_regions < 0 || ( n_regions > 0 && ! regions ) )
    {
        g_create_error = "kr_ctx_create_refined: bad region list";
        return nullptr;
    }
    if( cfg->flags & KR_FLAG_BOXES )
    {
        bool ok = cfg->mhd && ranks_of( * cfg ) <= 1 && n_regions == 0 && ! ( cfg->flags & KR_FLAG_HALO_ALL )
               && cfg->nb[ 1 ] == 1 && cfg->nb[ 2 ] == 1;
        for( int k = 0; k < 6; ++ k )
            ok = ok && cfg->bc[ k ] == KR_BC_PER;
        if( ! ok )
        {
            g_create_error = "kr_ctx_create: KR_FLAG_BOXES needs MHD, one rank, periodic sides, "
                             "no refinement and nb = (boxes, 1, 1)";
            return nullptr;
        }
    }
    kr_tree tree;
    std::memset( & tree, 0, sizeof( tree ) );
    if( n_regions > 0 && ! build_tree( cfg, n_regions, regions, tree ) )
        return nullptr;
    struct tree_guard { kr_tree & t; ~tree_guard(  ) { kr_tree_free( & t ); } } guard{ tree };
    const bool smr = tree.max_level > 0;
    std::vector< int > owner;
    if( ! smr && ! shard_owner( * cfg, owner, g_create_error ) )
        return nullptr;
    int ndev = 0;
    if( ! ck( nullptr, cudaGetDeviceCount( & ndev ), "cudaGetDeviceCount" ) )
        return nullptr;
    if( cfg->device < 0 || cfg->device >= ndev )
    {
        g_create_error = "kr_ctx_create: no such CUDA device";
        return nullptr;
    }
    if( ! ck( nullptr, cudaSetDevice( cfg->device ), "cudaSetDevice" ) )
        return nullptr;
    int n_sm = 148;
    cudaDeviceGetAttribute( & n_sm, cudaDevAttrMultiProcessorCount, cfg->device );

    kr_ctx * c = new kr_ctx;
    c->cfg = * cfg;
    c->n_sm = n_sm;
    c->boxes = ( cfg->flags & KR_FLAG_BOXES ) != 0;
    // The shared-memory tiled sweep is opt-in: on the 256^3 OT step it measured
    // slower than the per-face kernel (more registers per thread, long per-thread
    // face loops, a tail of partial CTAs), so the per-face kernel is the default.
    const int * n = cfg->n;
    c->nranks = ranks_of( * cfg );
    c->rank = c->nranks > 1 ? cfg->rank : 0;
    std::vector< int > local( owner.size(  ), -1 );
    for( int gb = 0; gb < int( owner.size(  ) ); ++ gb )
        if( owner[ gb ] == c->rank )
        {
            local[ gb ] = int( c->gid_h.size(  ) );
            c->gid_h.push_back( gb );
        }
    const bool halo_all = ( cfg->flags & KR_FLAG_HALO_ALL ) != 0;
    std::vector< smr_item_t > smr_items;
    std::vector< mh_t > mh_plan_h;
    std::vector< uint2 > mh_work_h;
    std::vector< int > mh_same_h;      // (block, direction, neighbour) of same-level pairs
    if( smr )
    {   // the tree's leaves, one rank, no halo exchange
        c->smr = true;
        c->max_level = tree.max_level;
        for( int b = 0; b < tree.nblk; ++ b )
        {
            c->gid_h.push_back( b );
            c->lvl_h.push_back( tree.level[ b ] );
            for( int a = 0; a < 3; ++ a )
                c->reg_h.push_back( tree.reg[ 3 * b + a ] );
        }
        for( halo_side_t * h : { & c->hsend, & c->hrecv } )
        {
            h->w_off.assign( 1, 0 ); h->w_cnt.assign( 1, 0 );
            h->b_off.assign( 1, 0 ); h->b_cnt.assign( 1, 0 );
        }
        smr_plan( tree, cfg->n, smr_items, c->n_restrict, c->prolong_off );
        if( cfg->mhd )
        {
            mh_plan_t mp = mh_plan( tree, cfg->n );
            c->mh_restrict[ 0 ] = mp.restrict_[ 0 ]; c->mh_restrict[ 1 ] = mp.restrict_[ 1 ];
            c->mh_prolong = mp.prolong;
            c->mh_waves = mp.waves;
            mh_plan_h.swap( mp.list );
            mh_work_h.swap( mp.work );
            mh_same_h.swap( mp.same_nbr );
        }
        if( smr_items.size(  ) > 65535 )
        {   // one grid row per item
            g_create_error = "kr_ctx_create_refined: more than 65535 level-jump items";
            delete c;
            return nullptr;
        }
    }
    else
    {
        for( int gb : c->gid_h )
        {   // an independent box sits at the origin of its own domain
            c->lvl_h.push_back( 0 );
            c->reg_h.push_back( c->boxes ? 0 : gb % cfg->nb[ 0 ] );
            c->reg_h.push_back( c->boxes ? 0 : ( gb / cfg->nb[ 0 ] ) % cfg->nb[ 1 ] );
            c->reg_h.push_back( c->boxes ? 0 : gb / ( cfg->nb[ 0 ] * cfg->nb[ 1 ] ) );
        }
        halo_plan( * cfg, owner, local, halo_all, c->hsend, c->hrecv );
    }
    c->nblk = int( c->gid_h.size(  ) );
    if( c->hsend.items.size(  ) > 65535 || c->hrecv.items.size(  ) > 65535 )
    {   // one grid row per item
        g_create_error = "kr_ctx_create: more than 65535 halo items on one rank";
        delete c;
        return nullptr;
    }
    c->nw = cfg->mhd ? 8 : 5;
    c->nws = cfg->mhd ? 11 : 5;
    c->nf = cfg->mhd ? 7 : 5;
    c->nc  = ( long long ) n[ 0 ] * n[ 1 ] * n[ 2 ];
    c->ngw = ( long long )( n[ 0 ] + 4 ) * ( n[ 1 ] + 4 ) * ( n[ 2 ] + 4 );
    c->nbf = ( long long )( n[ 0 ] + 5 ) * ( n[ 1 ] + 5 ) * ( n[ 2 ] + 5 );
    c->nfb = ( long long )( n[ 0 ] + 3 ) * ( n[ 1 ] + 3 ) * ( n[ 2 ] + 3 );
    c->rsize = cfg->precision == 1 ? 4 : 8;
    const size_t nb = size_t( c->nblk );
    bool ok = ck( c, cudaStreamCreateWithFlags( & c->stream, cudaStreamNonBlocking ), "stream" );
    c->own_stream = ok;
    for( int s = 0; s < 2 && ok; ++ s )
    {
        ok = ok && ck( c, cudaMalloc( & c->u[ s ], nb * 5 * c->nc * 8 ), "malloc u" );
        if( cfg->mhd )
            ok = ok && ck( c, cudaMalloc( & c->bf[ s ], nb * 3 * c->nbf * 8 ), "malloc bf" );
    }
    ok = ok && ck( c, cudaMalloc( & c->w, nb * c->nws * c->ngw * c->rsize ), "malloc w" );
    // In the FP32 step graph the three separate launches measured 0.07 ms per
    // 256^3 step faster than the fused one (the FP32 c2p and cell update each
    // run at 64 registers, 4 CTAs per SM, and the face update at 38 / 6); the
    // FP64 step and the batched launches are faster fused.
    c->fuse_batch = cfg->mhd && ! c->smr && ! ( cfg->flags & KR_FLAG_UNFUSED );
    c->fuse = c->fuse_batch && cfg->precision == 2;
    for( int d = 0; d < 3 && ok; ++ d )
        ok = ck( c, cudaMalloc( & c->f[ d ], nb * c->nf * c->nfb * c->rsize ), "malloc f" );
    if( cfg->mhd && ok )
        ok = ck( c, cudaMalloc( & c->ee, nb * 3 * c->nfb * c->rsize ), "malloc ee" );
    ok = ok && ck( c, cudaMalloc( & c->geo, nb * sizeof( geo_t ) ), "malloc geo" );
    ok = ok && ck( c, cudaMalloc( & c->nbr, nb * 27 * sizeof( int ) ), "malloc nbr" );
    ok = ok && ck( c, cudaMalloc( & c->gid, nb * sizeof( int ) ), "malloc gid" );
    if( ok && ! smr_items.empty(  ) )
        ok = ck( c, cudaMalloc( & c->favg, std::max( 1, c->n_restrict ) * 5 * smr_half_sites( c ) * sizeof( double ) ), "malloc refinement fluxes" )
          && ck( c, cudaMalloc( & c->smr_items, smr_items.size(  ) * sizeof( smr_item_t ) ), "malloc refinement items" )
          && ck( c, cudaMemcpyAsync( c->smr_items, smr_items.data(  ), smr_items.size(  ) * sizeof( smr_item_t ),
                                     cudaMemcpyHostToDevice, c->stream ), "upload refinement items" );
    if( ok && ! mh_plan_h.empty(  ) )
        ok = ck( c, cudaMalloc( & c->mh_list, mh_plan_h.size(  ) * sizeof( mh_t ) ), "malloc exchange holders" )
          && ck( c, cudaMemcpyAsync( c->mh_list, mh_plan_h.data(  ), mh_plan_h.size(  ) * sizeof( mh_t ),
                                     cudaMemcpyHostToDevice, c->stream ), "upload exchange holders" )
          && ck( c, cudaMalloc( & c->mh_work, mh_work_h.size(  ) * sizeof( uint2 ) ), "malloc exchange items" )
          && ck( c, cudaMemcpyAsync( c->mh_work, mh_work_h.data(  ), mh_work_h.size(  ) * sizeof( uint2 ),
                                     cudaMemcpyHostToDevice, c->stream ), "upload exchange items" );
    // halo exchange: item lists and buffers (1-word minimum keeps pointers valid)
    {
        const halo_side_t * hs[ 2 ] = { & c->hsend, & c->hrecv };
        halo_item_t ** di[ 2 ] = { & c->send_items, & c->recv_items };
        void ** wb[ 2 ] = { & c->send_w, & c->recv_w };
        double ** bb[ 2 ] = { & c->send_b, & c->recv_b };
        for( int k = 0; k < 2 && ok; ++ k )
        {
            ok = ck( c, cudaMalloc( di[ k ], std::max< size_t >( 1, hs[ k ]->items.size(  ) ) * sizeof( halo_item_t ) ), "malloc halo items" )
              && ck( c, cudaMalloc( wb[ k ], std::max< long long >( 1, hs[ k ]->w_tot ) * c->rsize ), "malloc halo buffer" )
              && ck( c, cudaMalloc( bb[ k ], std::max< long long >( 1, hs[ k ]->b_tot ) * sizeof( double ) ), "malloc halo buffer" );
            if( ok && ! hs[ k ]->items.empty(  ) )
                ok = ck( c, cudaMemcpyAsync( * di[ k ], hs[ k ]->items.data(  ), hs[ k ]->items.size(  ) * sizeof( halo_item_t ),
                                             cudaMemcpyHostToDevice, c->stream ), "upload halo items" );
        }
        long long mx = 0;
        for( int a = 0; a < 3; ++ a )
            mx = std::max( mx, 2LL * n[ ( a + 1 ) % 3 ] * n[ ( a + 2 ) % 3 ] );
        c->halo_grid = int( std::min< long long >( 64, blocks_for( mx, 256 ) ) );
    }
    c->nscal = c->boxes ? c->nblk : 1;
    ok = ok && ck( c, cudaMalloc( & c->s, c->nscal * sizeof( scal_t ) ), "malloc scalars" );
    ok = ok && ck( c, cudaMalloc( & c->diag, 8 * sizeof( double ) ), "malloc diag" );
    if( cfg->mhd )
        ok = ok && ck( c, cudaMalloc( & c->sel_w, 32 * MLP_BFRAG * sizeof( unsigned ) ), "malloc selector" )
                && ck( c, cudaMalloc( & c->sel_b, ( 2 * MLP_H + 1 ) * sizeof( float ) ), "malloc selector" )
                && ck( c, cudaMalloc( & c->sel_cnt, 2 * sizeof( unsigned long long ) ), "malloc selector" )
                && ck( c, cudaMemset( c->sel_cnt, 0, 2 * sizeof( unsigned long long ) ), "memset selector" );
    if( cfg->mhd && cfg->riemann == KR_RIEMANN_LEARNED && ok )
    {   // per (axis, block): one byte per warp of the per-face sweep's grid
        // (128-face chunks per z plane x z planes x 4 warps)
        for( int ax = 0; ax < 3; ++ ax )
        {
            long long ext[ 3 ];
            for( int d = 0; d < 3; ++ d )
                ext[ d ] = d == ax ? n[ d ] + 1 : n[ d ] + 2;
            c->sel_wcap = std::max( c->sel_wcap, blocks_for( ext[ 0 ] * ext[ 1 ], 128 ) * ext[ 2 ] * 4 );
        }
        const size_t bytes = size_t( 3 ) * nb * c->sel_wcap * sizeof( unsigned );
        ok = ck( c, cudaMalloc( & c->sel_dec, bytes ), "malloc selector choices" )
          && ck( c, cudaMemset( c->sel_dec, 0, bytes ), "memset selector choices" );
    }
    c->stage_bytes = nb * ( size_t( c->nc ) * c->nw + ( cfg->mhd ? size_t( c->nbf ) * 3 : 0 ) ) * 8;
    ok = ok && ck( c, cudaMalloc( & c->stage, c->stage_bytes ), "malloc staging" );
    if( ! ok )
    {
        g_create_error = c->err;
        kr_ctx_destroy( c );
        return nullptr;
    }
    // zero everything that a kernel may read before writing it
    for( int s = 0; s < 2; ++ s )
    {
        cudaMemsetAsync( c->u[ s ], 0, nb * 5 * c->nc * 8, c->stream );
        if( cfg->mhd ) cudaMemsetAsync( c->bf[ s ], 0, nb * 3 * c->nbf * 8, c->stream );
    }
    cudaMemsetAsync( c->w, 0, nb * c->nws * c->ngw * c->rsize, c->stream );
    for( int d = 0; d < 3; ++ d )
        cudaMemsetAsync( c->f[ d ], 0, nb * c->nf * c->nfb * c->rsize, c->stream );
    if( cfg->mhd ) cudaMemsetAsync( c->ee, 0, nb * 3 * c->nfb * c->rsize, c->stream );

    set_geometry( c );
    // neighbour table of the local blocks: local index of a same-rank
    // neighbour, -1 past a physical side, -2 where the halo exchange fills,
    // -3 across a level jump (refined mesh: only face neighbours of the same
    // level are copied; hydro reads no edge or corner ghost)
    std::vector< int > nbr( nb * 27 );
    for( int b = 0; b < c->nblk; ++ b )
        for( int k = 0; k < 27; ++ k )
        {
            if( smr )
            {   // refined MHD: same-level neighbours in all 26 directions by push
                // (below, from the holders), the level jumps by the exchange
                const int sh[ 3 ] = { k % 3 - 1, ( k / 3 ) % 3 - 1, k / 9 - 1 };
                const int nz = ( sh[ 0 ] != 0 ) + ( sh[ 1 ] != 0 ) + ( sh[ 2 ] != 0 );
                int v = k == 13 ? b : -3;
                if( nz == 1 )
                {
                    const int a = sh[ 0 ] ? 0 : ( sh[ 1 ] ? 1 : 2 );
                    const int f = 2 * a + ( sh[ a ] > 0 );
                    const int kind = tree.face[ 6 * b + f ];
                    v = kind == KR_FACE_SAME ? tree.fnb[ ( 6 * b + f ) * 4 ] : ( kind == KR_FACE_PHYS ? -1 : -3 );
                    if( cfg->mhd && kind == KR_FACE_SAME )
                        v = -3;
                    if( kind == KR_FACE_FINE || kind == KR_FACE_COARSE )
                        c->geo_h[ b ].xlev |= 1 << f;
                    if( kind == KR_FACE_FINE )
                        c->geo_h[ b ].fine |= 1 << f;
                    if( kind == KR_FACE_FINE )
                        for( int it = 0; it < c->n_restrict; it += 4 )
                            if( smr_items[ it ].dst == b && smr_items[ it ].face == f )
                                c->geo_h[ b ].fitem[ f ] = it;
                }
                nbr[ b * 27 + k ] = v;
                continue;
            }
            if( c->boxes )
            {   // periodic onto itself in every direction
                nbr[ b * 27 + k ] = b;
                continue;
            }
            const int src = nbr_global( * cfg, c->gid_h[ b ], k );
            nbr[ b * 27 + k ] = src < 0 ? -1 : ( owner[ src ] == c->rank && ! ( halo_all && k != 13 ) ? local[ src ] : -2 );
        }
    for( const int * h = mh_same_h.data(  ); h < mh_same_h.data(  ) + mh_same_h.size(  ); h += 3 )
        nbr[ h[ 0 ] * 27 + h[ 1 ] ] = h[ 2 ];
    std::vector< scal_t > s0( c->nscal, scal_t{} );
    for( scal_t & r : s0 )
        r.dt_bound = cfg->dt_init >= FLT_MIN ? cfg->dt_init : FLT_MAX / 10;   // cycle.cpp:163-166
    ok = ck( c, cudaMemcpyAsync( c->geo, c->geo_h.data(  ), nb * sizeof( geo_t ), cudaMemcpyHostToDevice, c->stream ), "upload geo" )
      && ck( c, cudaMemcpyAsync( c->nbr, nbr.data(  ), nbr.size(  ) * sizeof( int ), cudaMemcpyHostToDevice, c->stream ), "upload nbr" )
      && ck( c, cudaMemcpyAsync( c->gid, c->gid_h.data(  ), nb * sizeof( int ), cudaMemcpyHostToDevice, c->stream ), "upload gid" )
      && ck( c, cudaMemcpyAsync( c->s, s0.data(  ), s0.size(  ) * sizeof( scal_t ), cudaMemcpyHostToDevice, c->stream ), "upload scalars" )
      && ck( c, cudaStreamSynchronize( c->stream ), "sync" );
    if( ! ok )
    {
        g_create_error = c->err;
        kr_ctx_destroy( c );
        return nullptr;
    }
    return c;
}

extern "C" {

kr_ctx * kr_ctx_create( const kr_cfg * cfg )
{
    return create_ctx( cfg, 0, nullptr );
}

kr_ctx * kr_ctx_create_refined( const kr_cfg * cfg, int n_regions, const kr_region * regions )
{
    return create_ctx( cfg, n_regions, regions );
}

int kr_block_info( kr_ctx * c, int * level, int * reg )
{
    if( ! c ) return -1;
    if( level ) std::copy( c->lvl_h.begin(  ), c->lvl_h.end(  ), level );
    if( reg ) std::copy( c->reg_h.begin(  ), c->reg_h.end(  ), reg );
    return c->nblk;
}

void kr_ctx_destroy( kr_ctx * c )
{
    if( ! c ) return;
    cudaSetDevice( c->cfg.device );
    if( c->stream ) cudaStreamSynchronize( c->stream );
    drop_graph( c );                   // before the communicator its graph uses
    if( c->comm ) nccl(  ).CommDestroy( c->comm );
    cudaFree( c->gid ); cudaFree( c->smr_items ); cudaFree( c->favg ); cudaFree( c->mh_list ); cudaFree( c->mh_work );
    cudaFree( c->send_items ); cudaFree( c->recv_items );
    cudaFree( c->send_w ); cudaFree( c->recv_w ); cudaFree( c->send_b ); cudaFree( c->recv_b );
    for( int s = 0; s < 2; ++ s ) { cudaFree( c->u[ s ] ); cudaFree( c->bf[ s ] ); }
    cudaFree( c->w );
    for( int d = 0; d < 3; ++ d ) cudaFree( c->f[ d ] );
    cudaFree( c->ee ); cudaFree( c->geo ); cudaFree( c->nbr ); cudaFree( c->s );
    cudaFree( c->stage ); cudaFree( c->diag );
    cudaFree( c->sel_w ); cudaFree( c->sel_b ); cudaFree( c->sel_cnt ); cudaFree( c->sel_dec );
    if( c->own_stream && c->stream ) cudaStreamDestroy( c->stream );
    delete c;
}

int kr_set_stream( kr_ctx * c, void * stream )
{
    if( ! c ) return -1;
    cudaStreamSynchronize( c->stream );
    if( c->own_stream ) cudaStreamDestroy( c->stream );
    c->own_stream = stream == nullptr;
    if( stream ) c->stream = ( cudaStream_t ) stream;
    else if( ! ck( c, cudaStreamCreateWithFlags( & c->stream, cudaStreamNonBlocking ), "stream" ) )
        return -1;
    drop_graph( c );
    return 0;
}

}   // extern "C"

template< bool MHD, class R >
static void launch_scatter( kr_ctx * c )
{
    const args_t< R > a = make_args< R >( c );
    const long long nmax = MHD ? std::max( c->nc, c->nbf ) : c->nc;
    const double * hu = c->stage;
    const double * hb = c->stage + size_t( c->nblk ) * c->nc * c->nw;
    k_scatter< MHD, R ><<< dim3( blocks_for( nmax, 256 ), c->nblk ), 256, 0, c->stream >>>( a, hu, hb );
    if( MHD )
    {   // the face-B ghost strips of slot 0 for the first stage (later stages
        // get them pushed by the face update)
        const int * n = c->cfg.n;
        const long long nghost = shell_count( n[ 0 ], n[ 1 ], n[ 2 ], 2 ) + bf_strip_count( n[ 0 ], n[ 1 ], n[ 2 ] );
        k_ghost< MHD, R ><<< dim3( blocks_for( nghost, 256 ), c->nblk ), 256, 0, c->stream >>>( a, 0, make_ghost_div( n ) );
    }
}
template< bool MHD, class R >
static void launch_gather( kr_ctx * c )
{
    const args_t< R > a = make_args< R >( c );
    const long long nmax = MHD ? std::max( c->nc, c->nbf ) : c->nc;
    double * hu = c->stage;
    double * hb = c->stage + size_t( c->nblk ) * c->nc * c->nw;
    k_gather< MHD, R ><<< dim3( blocks_for( nmax, 256 ), c->nblk ), 256, 0, c->stream >>>( a, hu, hb );
}

extern "C" {

int kr_set_state( kr_ctx * c, const double * u, const double * bf )
{
    if( ! c || ! u || ( c->cfg.mhd && ! bf ) ) { if( c ) c->err = "kr_set_state: null array"; return -1; }
    cudaSetDevice( c->cfg.device );
    const size_t su = size_t( c->nblk ) * c->nc * c->nw * 8;
    const size_t sb = c->cfg.mhd ? size_t( c->nblk ) * c->nbf * 3 * 8 : 0;
    if( ! ck( c, cudaMemcpyAsync( c->stage, u, su, cudaMemcpyHostToDevice, c->stream ), "upload u" ) )
        return -1;
    if( sb && ! ck( c, cudaMemcpyAsync( ( char * ) c->stage + su, bf, sb, cudaMemcpyHostToDevice, c->stream ), "upload bf" ) )
        return -1;
    if( c->cfg.mhd ) { if( c->cfg.precision == 1 ) launch_scatter< true, float >( c ); else launch_scatter< true, double >( c ); }
    else             { if( c->cfg.precision == 1 ) launch_scatter< false, float >( c ); else launch_scatter< false, double >( c ); }
    return ck( c, cudaGetLastError(  ), "scatter" ) && ck( c, cudaStreamSynchronize( c->stream ), "sync" ) ? 0 : -1;
}

int kr_get_state( kr_ctx * c, double * u, double * bf )
{
    if( ! c || ! u || ( c->cfg.mhd && ! bf ) ) { if( c ) c->err = "kr_get_state: null array"; return -1; }
    cudaSetDevice( c->cfg.device );
    const size_t su = size_t( c->nblk ) * c->nc * c->nw * 8;
    const size_t sb = c->cfg.mhd ? size_t( c->nblk ) * c->nbf * 3 * 8 : 0;
    if( c->cfg.mhd ) { if( c->cfg.precision == 1 ) launch_gather< true, float >( c ); else launch_gather< true, double >( c ); }
    else             { if( c->cfg.precision == 1 ) launch_gather< false, float >( c ); else launch_gather< false, double >( c ); }
    if( ! ck( c, cudaGetLastError(  ), "gather" ) ) return -1;
    if( ! ck( c, cudaMemcpyAsync( u, c->stage, su, cudaMemcpyDeviceToHost, c->stream ), "download u" ) )
        return -1;
    if( sb && ! ck( c, cudaMemcpyAsync( bf, ( char * ) c->stage + su, sb, cudaMemcpyDeviceToHost, c->stream ), "download bf" ) )
        return -1;
    return ck( c, cudaStreamSynchronize( c->stream ), "sync" ) ? 0 : -1;
}

int kr_init_problem( kr_ctx * c, const char * name, uint64_t seed )
{
    if( ! c || ! name ) return -1;
    const bool shock = ! std::strcmp( name, "shock" ), turb = ! std::strcmp( name, "turb" );
    const bool blast = ! std::strcmp( name, "blast" );
    const bool ot = ! std::strcmp( name, "ot" ) || turb || blast;     // the MHD workloads
    if( ( ! shock && ! ot ) || ( ot != bool( c->cfg.mhd ) ) || c->boxes )
    {
        c->err = std::string( "kr_init_problem: unknown workload '" ) + name + "' for this mesh";
        return -1;
    }
    const kr_cfg & g = c->cfg;
    const int * n = g.n;
    const int nw = c->nw;
    std::vector< double > hu( size_t( c->nblk ) * c->nc * nw, 0.0 );
    std::vector< double > hb( ot ? size_t( c->nblk ) * c->nbf * 3 : 0, 0.0 );
    int nglob[ 3 ];
    for( int a = 0; a < 3; ++ a ) nglob[ a ] = n[ a ] * g.nb[ a ];
    const long long sb1 = n[ 0 ] + 5, sb2 = ( long long )( n[ 0 ] + 5 ) * ( n[ 1 ] + 5 );
    auto bidx = [ & ]( int b, int i0, int i1, int i2 )
    {   return ( ( size_t ) b * c->nbf + ( i0 + 2 ) + sb1 * ( i1 + 2 ) + sb2 * ( i2 + 2 ) ) * 3; };
    kr_turb_t modes;
    if( turb )
        kr_turb_modes( & modes, seed );
    double centre[ 3 ];
    for( int a = 0; a < 3; ++ a )
        centre[ a ] = ( g.x_min[ a ] + g.x_max[ a ] ) / 2;
    auto work = [ & ]( int b )
    {
        const int * reg = & c->reg_h[ 3 * b ];
        const int lvl = c->lvl_h[ b ];
        if( ot )
            for( int i2 = 0; i2 <= n[ 2 ]; ++ i2 )
            for( int i1 = 0; i1 <= n[ 1 ]; ++ i1 )
            for( int i0 = 0; i0 <= n[ 0 ]; ++ i0 )
            {
                double * p = hb.data(  ) + bidx( b, i0, i1, i2 );
                if( blast )
                    for( int a = 0; a < 3; ++ a )
                        p[ a ] = kr_blast_b( a );
                else
                {
                    p[ 0 ] = turb ? kr_turb_bx( g.gamma ) : kr_ot_bx( x_cc( g, reg, lvl, 1, i1 ) );
                    p[ 1 ] = turb ? 0.0 : kr_ot_by( x_cc( g, reg, lvl, 0, i0 ) );
                    p[ 2 ] = turb ? 0.0 : kr_ot_bz(  );
                }
            }
        for( int i2 = 0; i2 < n[ 2 ]; ++ i2 )
        for( int i1 = 0; i1 < n[ 1 ]; ++ i1 )
        for( int i0 = 0; i0 < n[ 0 ]; ++ i0 )
        {
            const int ii[ 3 ] = { i0, i1, i2 };
            int ig[ 3 ];
            for( int a = 0; a < 3; ++ a ) ig[ a ] = reg[ a ] * n[ a ] + ii[ a ];
            const uint64_t key = kr_cell_key( lvl, ig, nglob );
            double * u = hu.data(  ) + ( ( size_t ) b * c->nc + i0 + ( size_t ) n[ 0 ] * ( i1 + ( size_t ) n[ 1 ] * i2 ) ) * nw;
            if( shock )
                kr_shock_cell( u, x_cc( g, reg, lvl, 0, i0 ), g.gamma, seed, key );
            else
            {
                double x[ 3 ], bc[ 3 ];
                for( int a = 0; a < 3; ++ a )
                {
                    int jj[ 3 ] = { i0, i1, i2 };
                    x[ a ] = x_cc( g, reg, lvl, a, ii[ a ] );
                    const double bl = hb[ bidx( b, jj[ 0 ], jj[ 1 ], jj[ 2 ] ) + a ];
                    ++ jj[ a ];
                    bc[ a ] = ( bl + hb[ bidx( b, jj[ 0 ], jj[ 1 ], jj[ 2 ] ) + a ] ) / 2;
                }
                if( turb )
                    kr_turb_cell( u, x, bc, g.gamma, & modes );
                else if( blast )
                    kr_blast_cell( u, x, bc, centre, g.gamma );
                else
                    kr_ot_cell( u, x, bc, g.gamma, seed, key );
            }
        }
    };
    const int nt = std::max( 1, std::min( c->nblk, int( std::thread::hardware_concurrency(  ) ) ) );
    std::vector< std::thread > th;
    for( int t = 0; t < nt; ++ t )
        th.emplace_back( [ & , t ] (  ) { for( int b = t; b < c->nblk; b += nt ) work( b ); } );
    for( auto & x : th ) x.join(  );
    return kr_set_state( c, hu.data(  ), ot ? hb.data(  ) : nullptr );
}

int kr_box_params( uint64_t seed, int box, double gamma, double * out )
{
    if( ! out || box < 0 ) return -1;
    kr_box_t p;
    kr_box_params( & p, seed, box, gamma );
    const double v[ 8 ] = { double( p.n ), p.rho, p.pre, p.amp, p.beta, p.b[ 0 ], p.b[ 1 ], p.b[ 2 ] };
    std::copy( v, v + 8, out );
    return 0;
}

int kr_init_boxes( kr_ctx * c, uint64_t seed, const int * ids )
{
    if( ! c || ! ids ) return -1;
    bool periodic = true;
    for( int k = 0; k < 6; ++ k )
        periodic = periodic && c->cfg.bc[ k ] == KR_BC_PER;
    if( ! c->cfg.mhd || c->smr || ( ! c->boxes && ! ( c->nblk == 1 && c->nranks == 1 && periodic ) ) )
    {
        c->err = "kr_init_boxes: needs a KR_FLAG_BOXES context or a periodic one-block MHD mesh";
        return -1;
    }
    const kr_cfg g = geo_cfg( c );
    const int * n = g.n;
    std::vector< kr_box_t > box( c->nblk );
    for( int b = 0; b < c->nblk; ++ b )
    {
        if( ids[ b ] < 0 )
        {
            c->err = "kr_init_boxes: negative box index";
            return -1;
        }
        kr_box_params( & box[ b ], seed, ids[ b ], g.gamma );
        if( box[ b ].n != n[ 0 ] || box[ b ].n != n[ 1 ] || box[ b ].n != n[ 2 ] )
        {
            c->err = "kr_init_boxes: box " + std::to_string( ids[ b ] ) + " has " + std::to_string( box[ b ].n )
                   + " cells per axis, the context's blocks " + std::to_string( n[ 0 ] ) + "x"
                   + std::to_string( n[ 1 ] ) + "x" + std::to_string( n[ 2 ] );
            return -1;
        }
    }
    const int nw = c->nw;
    std::vector< double > hu( size_t( c->nblk ) * c->nc * nw, 0.0 );
    std::vector< double > hb( size_t( c->nblk ) * c->nbf * 3, 0.0 );
    const long long sb1 = n[ 0 ] + 5, sb2 = ( long long )( n[ 0 ] + 5 ) * ( n[ 1 ] + 5 );
    auto bidx = [ & ]( int b, int i0, int i1, int i2 )
    {   return ( ( size_t ) b * c->nbf + ( i0 + 2 ) + sb1 * ( i1 + 2 ) + sb2 * ( i2 + 2 ) ) * 3; };
    const int reg0[ 3 ] = { 0, 0, 0 };
    auto work = [ & ]( int b )
    {   // the box is its own domain: cell keys and centres of a one-block mesh
        const kr_box_t & p = box[ b ];
        for( int i2 = 0; i2 <= n[ 2 ]; ++ i2 )
        for( int i1 = 0; i1 <= n[ 1 ]; ++ i1 )
        for( int i0 = 0; i0 <= n[ 0 ]; ++ i0 )
            for( int a = 0; a < 3; ++ a )
                hb[ bidx( b, i0, i1, i2 ) + a ] = p.b[ a ];
        for( int i2 = 0; i2 < n[ 2 ]; ++ i2 )
        for( int i1 = 0; i1 < n[ 1 ]; ++ i1 )
        for( int i0 = 0; i0 < n[ 0 ]; ++ i0 )
        {
            const int ii[ 3 ] = { i0, i1, i2 };
            double x[ 3 ], bc[ 3 ];
            for( int a = 0; a < 3; ++ a )
            {
                int jj[ 3 ] = { i0, i1, i2 };
                x[ a ] = x_cc( g, reg0, 0, a, ii[ a ] );
                const double bl = hb[ bidx( b, jj[ 0 ], jj[ 1 ], jj[ 2 ] ) + a ];
                ++ jj[ a ];
                bc[ a ] = ( bl + hb[ bidx( b, jj[ 0 ], jj[ 1 ], jj[ 2 ] ) + a ] ) / 2;
            }
            double * u = hu.data(  ) + ( ( size_t ) b * c->nc + i0 + ( size_t ) n[ 0 ] * ( i1 + ( size_t ) n[ 1 ] * i2 ) ) * nw;
            kr_box_cell( u, x, bc, g.gamma, & p, kr_cell_key( 0, ii, n ) );
        }
    };
    const int nt = std::max( 1, std::min( c->nblk, int( std::thread::hardware_concurrency(  ) ) ) );
    std::vector< std::thread > th;
    for( int t = 0; t < nt; ++ t )
        th.emplace_back( [ & , t ] (  ) { for( int b = t; b < c->nblk; b += nt ) work( b ); } );
    for( auto & x : th ) x.join(  );
    return kr_set_state( c, hu.data(  ), hb.data(  ) );
}

int kr_step( kr_ctx * c, int n_steps )
{
    if( ! c || n_steps < 0 ) return -1;
    if( c->cfg.riemann == KR_RIEMANN_LEARNED && ! c->sel_ready )
    {
        c->err = "kr_step: learned face selector configured but no weights set (kr_set_selector)";
        return -1;
    }
    if( c->nranks > 1 && ! c->comm )
    {
        c->err = "kr_step: sharded context without a communicator (kr_comm_init, or kr_group_step)";
        return -1;
    }
    cudaSetDevice( c->cfg.device );
    if( ! c->graph_exec || c->graph_stream != c->stream )
        if( ! build_graph( c ) )
            return -1;
    for( int s = 0; s < n_steps; ++ s )
        if( ! ck( c, cudaGraphLaunch( c->graph_exec, c->stream ), "graph launch" ) )
            return -1;
    return 0;
}

int kr_get_time( kr_ctx * c, double * t, double * dt_last, double * dt_bound, long long * n )
{
    if( ! c ) return -1;
    scal_t s;
    if( ! ck( c, cudaMemcpyAsync( & s, c->s, sizeof( s ), cudaMemcpyDeviceToHost, c->stream ), "read scalars" )
        || ! ck( c, cudaStreamSynchronize( c->stream ), "sync" ) )
        return -1;
    if( t ) * t = s.t;
    if( dt_last ) * dt_last = s.dt_last;
    if( dt_bound ) * dt_bound = s.dt_bound;
    if( n ) * n = s.n_steps;
    return 0;
}

int kr_set_time( kr_ctx * c, double t, double dt_bound )
{   // independent boxes: every box
    if( ! c ) return -1;
    std::vector< scal_t > s( c->nscal );
    if( ! ck( c, cudaMemcpyAsync( s.data(  ), c->s, s.size(  ) * sizeof( scal_t ), cudaMemcpyDeviceToHost, c->stream ), "read scalars" )
        || ! ck( c, cudaStreamSynchronize( c->stream ), "sync" ) )
        return -1;
    for( scal_t & r : s )
    {
        r.t = t;
        r.dt_bound = dt_bound;
    }
    return ck( c, cudaMemcpyAsync( c->s, s.data(  ), s.size(  ) * sizeof( scal_t ), cudaMemcpyHostToDevice, c->stream ), "write scalars" )
        && ck( c, cudaStreamSynchronize( c->stream ), "sync" ) ? 0 : -1;
}

int kr_box_times( kr_ctx * c, double * t, double * dt_last, long long * n_steps )
{
    if( ! c ) return -1;
    std::vector< scal_t > s( c->nscal );
    if( ! ck( c, cudaMemcpyAsync( s.data(  ), c->s, s.size(  ) * sizeof( scal_t ), cudaMemcpyDeviceToHost, c->stream ), "read scalars" )
        || ! ck( c, cudaStreamSynchronize( c->stream ), "sync" ) )
        return -1;
    for( int b = 0; b < c->nblk; ++ b )
    {   // one shared set unless the blocks are independent boxes
        const scal_t & r = s[ c->boxes ? b : 0 ];
        if( t ) t[ b ] = r.t;
        if( dt_last ) dt_last[ b ] = r.dt_last;
        if( n_steps ) n_steps[ b ] = r.n_steps;
    }
    return 0;
}

int kr_status( kr_ctx * c )
{
    if( ! c ) return -1;
    scal_t s;
    if( ! ck( c, cudaMemcpyAsync( & s, c->s, sizeof( s ), cudaMemcpyDeviceToHost, c->stream ), "read scalars" )
        || ! ck( c, cudaStreamSynchronize( c->stream ), "sync" ) )
        return -1;
    const cudaError_t e = cudaGetLastError(  );
    if( e != cudaSuccess ) { ck( c, e, "device" ); return -1; }
    return s.status;
}

int kr_set_selector( kr_ctx * c, const float * w, float threshold )
{
    if( ! c || ! w ) return -1;
    if( ! c->cfg.mhd ) { c->err = "kr_set_selector: MHD only"; return -1; }
    cudaSetDevice( c->cfg.device );
    std::vector< unsigned > words;
    std::vector< float > bias;
    kr_mlp_pack( w, words, bias );
    if( ! ck( c, cudaMemcpyAsync( c->sel_w, words.data(  ), words.size(  ) * 4, cudaMemcpyHostToDevice, c->stream ), "upload selector" )
        || ! ck( c, cudaMemcpyAsync( c->sel_b, bias.data(  ), bias.size(  ) * 4, cudaMemcpyHostToDevice, c->stream ), "upload selector" )
        || ! ck( c, cudaStreamSynchronize( c->stream ), "sync" ) )
        return -1;
    if( c->sel_thr != threshold )
        drop_graph( c );                 // the threshold is a kernel argument
    c->sel_thr = threshold;
    c->sel_ready = true;
    const int one = 1;                   // the network runs at the next step
    if( ! ck( c, cudaMemcpyAsync( ( char * ) c->s + offsetof( scal_t, sel_force ), & one, sizeof( one ),
                                  cudaMemcpyHostToDevice, c->stream ), "selector force" )
        || ! ck( c, cudaStreamSynchronize( c->stream ), "sync" ) )
        return -1;
    return 0;
}

int kr_selector_stats( kr_ctx * c, long long * faces, long long * cheap, int reset )
{
    if( ! c || ! c->sel_cnt ) return -1;
    unsigned long long h[ 2 ];
    if( ! ck( c, cudaMemcpyAsync( h, c->sel_cnt, sizeof( h ), cudaMemcpyDeviceToHost, c->stream ), "read counters" )
        || ! ck( c, cudaStreamSynchronize( c->stream ), "sync" ) )
        return -1;
    if( faces ) * faces = ( long long ) h[ 0 ];
    if( cheap ) * cheap = ( long long ) h[ 1 ];
    if( reset && ! ck( c, cudaMemsetAsync( c->sel_cnt, 0, sizeof( h ), c->stream ), "reset counters" ) )
        return -1;
    return 0;
}

int kr_selector_collect( kr_ctx * c, int n_steps, unsigned stride, uint64_t seed,
                         long long max_samples, float * out, long long * n_out )
{
    if( ! c || ! out || max_samples <= 0 || stride == 0 || n_steps < 0 ) return -1;
    if( ! c->cfg.mhd ) { c->err = "kr_selector_collect: MHD only"; return -1; }
    if( c->smr ) { c->err = "kr_selector_collect: the learned face selector runs on uniform meshes"; return -1; }
    cudaSetDevice( c->cfg.device );
    const size_t bytes = size_t( max_samples ) * ( MLP_IN + 1 ) * sizeof( float );
    if( ! ck( c, cudaMalloc( & c->smp, bytes ), "malloc samples" )
        || ! ck( c, cudaMalloc( & c->smp_n, sizeof( unsigned long long ) ), "malloc samples" )
        || ! ck( c, cudaMemsetAsync( c->smp_n, 0, sizeof( unsigned long long ), c->stream ), "memset" ) )
        return -1;
    c->smp_max = max_samples;
    c->smp_stride = stride;
    bool ok = true;
    for( int k = 0; k < n_steps && ok; ++ k )
    {
        c->smp_seed = unsigned( seed * 0x9E3779B9u + k );
        ok = c->cfg.precision == 1 ? enqueue_step< true, float, true >( c, c->stream )
                                   : enqueue_step< true, double, true >( c, c->stream );
        ok = ok && ck( c, cudaGetLastError(  ), "collect step" );
    }
    unsigned long long n = 0;
    ok = ok && ck( c, cudaMemcpyAsync( & n, c->smp_n, sizeof( n ), cudaMemcpyDeviceToHost, c->stream ), "read count" )
            && ck( c, cudaStreamSynchronize( c->stream ), "sync" );
    const long long got = std::min( ( long long ) n, max_samples );
    ok = ok && ck( c, cudaMemcpy( out, c->smp, size_t( got ) * ( MLP_IN + 1 ) * sizeof( float ), cudaMemcpyDeviceToHost ), "download samples" );
    cudaFree( c->smp );
    cudaFree( c->smp_n );
    c->smp = nullptr;
    c->smp_n = nullptr;
    c->smp_max = 0;
    if( n_out ) * n_out = got;
    return ok ? 0 : -1;
}

int kr_profile_step( kr_ctx * c, int n_kinds, double * ms )
{
    if( ! c || ! ms || n_kinds < 7 ) { if( c ) c->err = "kr_profile_step: need 7 slots"; return -1; }
    cudaSetDevice( c->cfg.device );
    for( int k = 0; k < n_kinds; ++ k ) ms[ k ] = 0;
    bool ok;
    if( c->cfg.mhd ) ok = c->cfg.precision == 1 ? profile_step< true, float >( c, ms ) : profile_step< true, double >( c, ms );
    else             ok = c->cfg.precision == 1 ? profile_step< false, float >( c, ms ) : profile_step< false, double >( c, ms );
    return ok ? 0 : -1;
}

int kr_launches_per_step( kr_ctx * c )
{
    if( ! c ) return -1;
    int flux = 3;                     // one per-face sweep per axis
    if( c->cfg.mhd && c->cfg.riemann == KR_RIEMANN_LEARNED )
        flux = 6;                     // per sweep: the network's kernel and the list kernel
    const int halo = ( c->hsend.items.empty(  ) ? 0 : 1 ) + ( c->hrecv.items.empty(  ) ? 0 : 1 );
    int phys = ! c->cfg.mhd && has_phys( c ) ? 1 : 0;
    if( c->cfg.mhd )
        for( int s = 0; s < 6; ++ s )
            phys += ( c->cfg.bc[ s ] != KR_BC_PER ) * ( c->mh_list ? 2 : 1 );   // refined MHD: two passes
    int smr = 0;
    if( c->smr && c->mh_list )
    {   // refined MHD: restrictions (two passes), copies, prolongations by
        // level, the flux average and the edge-E waves
        smr = ( c->mh_restrict[ 1 ] > c->mh_restrict[ 0 ] )
            + ( c->n_restrict ? 1 : 0 ) + int( c->mh_waves.size(  ) ) - 1;
        for( size_t l = 0; l + 1 < c->mh_prolong.size(  ); ++ l )
            smr += c->mh_prolong[ l + 1 ] > c->mh_prolong[ l ];
    }
    else if( c->smr )
    {
        smr = c->n_restrict ? 2 : 0;     // restriction, flux average
        for( int l = 1; l <= c->max_level; ++ l )
            smr += c->prolong_off[ l ] > c->prolong_off[ l - 1 ];
    }
    // fused: stage 0's two updates and stage 1's c2p are one launch
    return 2 + 2 * ( ( c->cfg.mhd ? 4 : 2 ) + flux + phys + halo + smr ) - ( c->fuse ? 2 : 0 );
}

int kr_diagnostics( kr_ctx * c, double * max_div_b, double * totals5 )
{
    if( ! c ) return -1;
    cudaSetDevice( c->cfg.device );
    cudaMemsetAsync( c->diag, 0, 8 * sizeof( double ), c->stream );
    const long long nmax = c->nc;
    if( c->cfg.mhd )
    {
        if( c->cfg.precision == 1 ) k_diag< true, float ><<< dim3( blocks_for( nmax, 256 ), c->nblk ), 256, 0, c->stream >>>( make_args< float >( c ), c->diag );
        else                        k_diag< true, double ><<< dim3( blocks_for( nmax, 256 ), c->nblk ), 256, 0, c->stream >>>( make_args< double >( c ), c->diag );
    }
    else
    {
        if( c->cfg.precision == 1 ) k_diag< false, float ><<< dim3( blocks_for( nmax, 256 ), c->nblk ), 256, 0, c->stream >>>( make_args< float >( c ), c->diag );
        else                        k_diag< false, double ><<< dim3( blocks_for( nmax, 256 ), c->nblk ), 256, 0, c->stream >>>( make_args< double >( c ), c->diag );
    }
    double h[ 8 ];
    if( ! ck( c, cudaMemcpyAsync( h, c->diag, sizeof( h ), cudaMemcpyDeviceToHost, c->stream ), "diag" )
        || ! ck( c, cudaStreamSynchronize( c->stream ), "sync" ) )
        return -1;
    if( max_div_b ) * max_div_b = h[ 0 ];
    if( totals5 ) for( int k = 0; k < 5; ++ k ) totals5[ k ] = h[ 1 + k ];
    return 0;
}

////////////////////////////////////////////////////////////
// Sharding

int kr_shard_owner( const kr_cfg * cfg, int * owner )
{
    g_create_error.clear(  );
    if( ! cfg || cfg->nb[ 0 ] < 1 || cfg->nb[ 1 ] < 1 || cfg->nb[ 2 ] < 1
        || cfg->n_ranks < 0 || ( cfg->n_ranks > 1 && ( cfg->rank < 0 || cfg->rank >= cfg->n_ranks ) ) )
    {
        g_create_error = "kr_shard_owner: need nb >= 1 and 0 <= rank < n_ranks";
        return -1;
    }
    std::vector< int > o;
    if( ! shard_owner( * cfg, o, g_create_error ) )
        return -1;
    const int me = ranks_of( * cfg ) > 1 ? cfg->rank : 0;
    if( owner )
        std::copy( o.begin(  ), o.end(  ), owner );
    return int( std::count( o.begin(  ), o.end(  ), me ) );
}

int kr_halo_counts( const kr_cfg * cfg, long long * send, long long * recv )
{
    if( kr_shard_owner( cfg, nullptr ) < 0 || ! send || ! recv )
        return -1;
    std::vector< int > owner;
    shard_owner( * cfg, owner, g_create_error );
    const int me = ranks_of( * cfg ) > 1 ? cfg->rank : 0;
    std::vector< int > local( owner.size(  ), -1 );
    int nl = 0;
    for( size_t gb = 0; gb < owner.size(  ); ++ gb )
        if( owner[ gb ] == me ) local[ gb ] = nl ++;
    halo_side_t hs, hr;
    halo_plan( * cfg, owner, local, ( cfg->flags & KR_FLAG_HALO_ALL ) != 0, hs, hr );
    for( int q = 0; q < ranks_of( * cfg ); ++ q )
    {
        send[ 2 * q ] = hs.w_cnt[ q ]; send[ 2 * q + 1 ] = hs.b_cnt[ q ];
        recv[ 2 * q ] = hr.w_cnt[ q ]; recv[ 2 * q + 1 ] = hr.b_cnt[ q ];
    }
    return 0;
}

int kr_shard_blocks( kr_ctx * c, int * gid )
{
    if( ! c ) return -1;
    if( gid ) std::copy( c->gid_h.begin(  ), c->gid_h.end(  ), gid );
    return c->nblk;
}

int kr_comm_unique_id( unsigned char id[ 128 ] )
{
    static_assert( sizeof( ncclUniqueId ) == 128, "NCCL unique id size" );
    nccl_api_t & api = nccl(  );
    if( ! api.ok ) { g_create_error = api.err; return -1; }
    ncclUniqueId uid;
    const ncclResult_t r = api.GetUniqueId( & uid );
    if( r != ncclSuccess ) { g_create_error = std::string( "ncclGetUniqueId: " ) + api.GetErrorString( r ); return -1; }
    std::memcpy( id, & uid, sizeof( uid ) );
    return 0;
}

int kr_comm_init( kr_ctx * c, const unsigned char id[ 128 ] )
{
    if( ! c || ! id ) return -1;
    nccl_api_t & api = nccl(  );
    if( ! api.ok ) { c->err = api.err; return -1; }
    if( c->comm ) { c->err = "kr_comm_init: communicator already set"; return -1; }
    if( c->smr ) { c->err = "kr_comm_init: a refined mesh runs on one rank"; return -1; }
    cudaSetDevice( c->cfg.device );
    ncclUniqueId uid;
    std::memcpy( & uid, id, sizeof( uid ) );
    const ncclResult_t r = api.CommInitRank( & c->comm, c->nranks, uid, c->rank );
    if( r != ncclSuccess )
    {
        c->comm = nullptr;
        c->err = std::string( "ncclCommInitRank: " ) + api.GetErrorString( r );
        return -1;
    }
    drop_graph( c );                   // the next step captures the exchange
    return 0;
}

}   // extern "C"

template< bool MHD, class R >
static void group_front( kr_ctx * c, cudaStream_t st, int stage )
{
    enqueue_front< MHD, R >( c, st, make_args< R >( c ), stage, untimed_t(  ) );
}
template< bool MHD, class R >
static void group_back( kr_ctx * c, cudaStream_t st, int stage )
{
    enqueue_back< MHD, R >( c, st, make_args< R >( c ), stage, c->cfg.riemann, untimed_t(  ) );
}

extern "C" {

int kr_group_step( kr_ctx * const * ctxs, int n, int n_steps )
{
    g_create_error.clear(  );
    if( ! ctxs || n < 1 || n > KR_GROUP_MAX || n_steps < 0 || ! ctxs[ 0 ] )
    {
        g_create_error = "kr_group_step: need 1..64 contexts and n_steps >= 0";
        return -1;
    }
    const kr_cfg & g0 = ctxs[ 0 ]->cfg;
    std::vector< kr_ctx * > by( n, nullptr );
    for( int k = 0; k < n; ++ k )
    {
        kr_ctx * c = ctxs[ k ];
        if( ! c || c->boxes || c->nranks != n || by[ c->rank ] || c->cfg.device != g0.device || c->cfg.mhd != g0.mhd
            || c->cfg.precision != g0.precision || ( c->cfg.riemann == KR_RIEMANN_LEARNED && ! c->sel_ready ) )
        {
            g_create_error = "kr_group_step: need the n_ranks contexts of one mesh, one per rank, on one device";
            return -1;
        }
        by[ c->rank ] = c;
    }
    for( int p = 0; p < n; ++ p )
        for( int q = 0; q < n; ++ q )
            if( by[ p ]->hsend.w_cnt[ q ] != by[ q ]->hrecv.w_cnt[ p ]
                || by[ p ]->hsend.b_cnt[ q ] != by[ q ]->hrecv.b_cnt[ p ] )
            {
                g_create_error = "kr_group_step: halo plans of the contexts disagree (different meshes?)";
                return -1;
            }
    cudaSetDevice( g0.device );
    cudaStream_t st = ctxs[ 0 ]->stream;
    for( kr_ctx * c : by )
        cudaStreamSynchronize( c->stream );
    group_scal_t gs;
    gs.n = n;
    for( int r = 0; r < n; ++ r ) gs.s[ r ] = by[ r ]->s;
    const size_t rs = by[ 0 ]->rsize;
    const bool mhd = g0.mhd, fp32 = g0.precision == 1;
    for( int step = 0; step < n_steps; ++ step )
    {
        for( kr_ctx * c : by ) k_step_begin<<< 1, 1, 0, st >>>( c->s, c->nscal );
        for( int stage = 0; stage < 2; ++ stage )
        {
            for( kr_ctx * c : by )
            {
                if( mhd ) fp32 ? group_front< true, float >( c, st, stage ) : group_front< true, double >( c, st, stage );
                else      fp32 ? group_front< false, float >( c, st, stage ) : group_front< false, double >( c, st, stage );
            }
            for( int p = 0; p < n; ++ p )
                for( int q = 0; q < n; ++ q )
                {
                    const kr_ctx * P = by[ p ];
                    const kr_ctx * Q = by[ q ];
                    const long long w = P->hsend.w_cnt[ q ], b = P->hsend.b_cnt[ q ];
                    if( w ) cudaMemcpyAsync( ( char * ) Q->recv_w + Q->hrecv.w_off[ p ] * rs,
                                             ( char * ) P->send_w + P->hsend.w_off[ q ] * rs, w * rs, cudaMemcpyDeviceToDevice, st );
                    if( b ) cudaMemcpyAsync( Q->recv_b + Q->hrecv.b_off[ p ], P->send_b + P->hsend.b_off[ q ],
                                             b * sizeof( double ), cudaMemcpyDeviceToDevice, st );
                }
            if( stage == 0 )
                k_group_dt_min<<< 1, 1, 0, st >>>( gs );
            for( kr_ctx * c : by )
            {
                if( mhd ) fp32 ? group_back< true, float >( c, st, stage ) : group_back< true, double >( c, st, stage );
                else      fp32 ? group_back< false, float >( c, st, stage ) : group_back< false, double >( c, st, stage );
            }
        }
        for( kr_ctx * c : by ) k_step_end<<< 1, 1, 0, st >>>( c->s, c->cfg.dt_expand, c->nscal );
    }
    const cudaError_t e = cudaStreamSynchronize( st );
    const cudaError_t l = cudaGetLastError(  );
    if( e != cudaSuccess || l != cudaSuccess )
    {
        g_create_error = std::string( "kr_group_step: " ) + cudaGetErrorString( e != cudaSuccess ? e : l );
        return -1;
    }
    return 0;
}

}   // extern "C"

////////////////////////////////////////////////////////////
// Allocation-free cons -> prim + CFL dt for one block.
//
// For callers that cannot allocate device memory themselves: code that runs
// under another framework's memory pool or inside a region where cudaMalloc is
// not allowed (a real-time loop, a plugin whose host forbids allocation).  The
// caller passes device inputs (u, bf) and outputs (w, dt); the only scratch the
// kernel needs -- the per-CTA partial minima of the CFL dt and a completion
// counter -- lives in the file-scope array below, which every GPU that loads
// the library holds until the process exits.
//
// The array is shared by every call: calls that overlap on the GPU (two
// streams, or two host threads) race on it and give wrong results; serialise
// them.  The counter is cleared on the caller's stream at the start of every
// call, and the partials need no clearing (each CTA writes its own slot before
// the last CTA reads them all).

namespace kr
{
constexpr int NOALLOC_THREADS   = 256;
constexpr int NOALLOC_MAX_CTAS  = 16384;
constexpr long long NOALLOC_MAX_CELLS = ( long long ) NOALLOC_THREADS * NOALLOC_MAX_CTAS;

// [0]: completion counter; [32 ..]: one partial minimum per CTA (bit patterns)
static __device__ __align__( 256 ) unsigned long long g_noalloc_scratch[ 32 + NOALLOC_MAX_CTAS ];

template< bool MHD >
__global__ void __launch_bounds__( NOALLOC_THREADS )
k_c2p_dt_noalloc( const double * u, const double * bf, double * w, double * dt_out,
                  unsigned long long * scratch, int n0, int n1, int n2,
                  double gamma, double cfl, double d_floor, double t_floor,
                  double dx0, double dx1, double dx2 )
{
    constexpr int NW = MHD ? 8 : 5;
    const long long nc = ( long long ) n0 * n1 * n2;
    const long long c = ( long long ) blockIdx.x * blockDim.x + threadIdx.x;
    const long long ngw = ( long long )( n0 + 4 ) * ( n1 + 4 ) * ( n2 + 4 );
    const long long nbf = ( long long )( n0 + 5 ) * ( n1 + 5 ) * ( n2 + 5 );
    const double dx[ 3 ] = { dx0, dx1, dx2 };
    double dt = FLT_MAX;
    if( c < nc )
    {
        const int i0 = int( c % n0 ), i1 = int( ( c / n0 ) % n1 ), i2 = int( c / ( ( long long ) n0 * n1 ) );
        double cons[ 5 ], cout[ 5 ], prim[ 5 ];
        for( int k = 0; k < 5; ++ k )
            cons[ k ] = u[ k * nc + c ];
        double bc[ 3 ] = { 0, 0, 0 }, bc_2[ 3 ] = { 0, 0, 0 }, b_max[ 3 ] = { 0, 0, 0 }, e_m = 0;
        if( MHD )
        {
            const int ii[ 3 ] = { i0, i1, i2 };
            for( int d = 0; d < 3; ++ d )
            {
                int jj[ 3 ] = { ii[ 0 ], ii[ 1 ], ii[ 2 ] };
                auto at = [ & ]( const int * j )
                {   return bf[ d * nbf + ( j[ 0 ] + 2 ) + ( long long )( n0 + 5 ) * ( ( j[ 1 ] + 2 ) + ( long long )( n1 + 5 ) * ( j[ 2 ] + 2 ) ) ]; };
                const double b_l = at( jj );
                ++ jj[ d ];
                const double b_r = at( jj );
                bc[ d ] = ( b_l + b_r ) / 2;
                bc_2[ d ] = bc[ d ] * bc[ d ];
                e_m += bc_2[ d ];
                b_max[ d ] = fmax( fabs( b_l ), fabs( b_r ) );
            }
            e_m /= 2;
            cons[ ENE ] -= e_m;
        }
        double cs2;
        c2p( cons, prim, cout, gamma, d_floor, t_floor, cs2 );
        const long long iw0 = ( i0 + 2 ) + ( long long )( n0 + 4 ) * ( ( i1 + 2 ) + ( long long )( n1 + 4 ) * ( i2 + 2 ) );
        for( int k = 0; k < 5; ++ k )
            w[ k * ngw + iw0 ] = prim[ k ];
        if( MHD )
            for( int d = 0; d < 3; ++ d )
                w[ ( BCC + d ) * ngw + iw0 ] = bc[ d ];
        if( ! MHD )
        {
            const double cs = sqrt( cs2 );
            for( int d = 0; d < 3; ++ d )
                dt = fmin( dt, dx[ d ] / ( cs + fabs( prim[ MOM + d ] ) ) );
        }
        else
        {
            double bm_2[ 3 ] = { bc_2[ 0 ], bc_2[ 1 ], bc_2[ 2 ] };
            for( int d = 0; d < 3; ++ d )
            {
                bm_2[ d ] = b_max[ d ] * b_max[ d ];
                const double cf = c_fms< double >( prim, bm_2, gamma, d );
                dt = fmin( dt, dx[ d ] / ( cf + fabs( prim[ MOM + d ] ) ) );
                bm_2[ d ] = bc_2[ d ];
            }
        }
        dt *= cfl;
        ( void ) NW;
    }
    // CTA minimum -> this CTA's scratch slot; the last CTA to finish reduces
    // all slots into dt_out and re-arms the counter.
    __shared__ double red[ NOALLOC_THREADS / 32 ];
    __shared__ bool last;
    dt = warp_min( dt );
    if( ( threadIdx.x & 31 ) == 0 )
        red[ threadIdx.x >> 5 ] = dt;
    __syncthreads(  );
    if( threadIdx.x == 0 )
    {
        double m = red[ 0 ];
        for( int k = 1; k < NOALLOC_THREADS / 32; ++ k )
            m = fmin( m, red[ k ] );
        scratch[ 32 + blockIdx.x ] = ( unsigned long long ) __double_as_longlong( m );
        __threadfence(  );
        const unsigned long long done = atomicAdd( & scratch[ 0 ], 1ull );
        last = ( done == gridDim.x - 1 );
    }
    __syncthreads(  );
    if( ! last )
        return;
    __threadfence(  );
    double m = FLT_MAX;
    for( unsigned k = threadIdx.x; k < gridDim.x; k += blockDim.x )
        m = fmin( m, __longlong_as_double( ( long long ) ( ( volatile unsigned long long * ) scratch )[ 32 + k ] ) );
    m = warp_min( m );
    if( ( threadIdx.x & 31 ) == 0 )
        red[ threadIdx.x >> 5 ] = m;
    __syncthreads(  );
    if( threadIdx.x == 0 )
    {
        for( int k = 1; k < NOALLOC_THREADS / 32; ++ k )
            red[ 0 ] = fmin( red[ 0 ], red[ k ] );
        * dt_out = red[ 0 ];
        scratch[ 0 ] = 0;
    }
}

// Per-device address of the scratch array, looked up once per device.
static unsigned long long * g_noalloc_ptr[ 64 ] = { nullptr };
static std::mutex g_noalloc_mx;
}   // namespace kr

extern "C" int kr_c2p_dt_noalloc( const kr_cfg * cfg, const double * u, const double * bf,
                                  double * w, double * dt_out, void * stream )
{
    using namespace kr;
    g_create_error.clear(  );
    if( ! cfg || cfg->abi_version != KR_ABI_VERSION )
    {
        g_create_error = "kr_c2p_dt_noalloc: missing configuration or ABI version mismatch";
        return -1;
    }
    if( ! u || ! w || ! dt_out || ( cfg->mhd && ! bf ) )
    {
        g_create_error = "kr_c2p_dt_noalloc: null argument";
        return -1;
    }
    // the same lower bound as kr_ctx_create: every axis holds a PLM stencil, so
    // each cell's face B has both faces inside the block
    for( int a = 0; a < 3; ++ a )
        if( cfg->n[ a ] < 4 )
        {
            g_create_error = "kr_c2p_dt_noalloc: need n >= 4 cells per axis";
            return -1;
        }
    const long long nc = ( long long ) cfg->n[ 0 ] * cfg->n[ 1 ] * cfg->n[ 2 ];
    if( nc > NOALLOC_MAX_CELLS )
    {
        g_create_error = "kr_c2p_dt_noalloc: block of " + std::to_string( nc ) + " cells exceeds the "
                         "scratch limit of " + std::to_string( NOALLOC_MAX_CELLS ) + " cells "
                         "(16384 CTAs of 256 threads)";
        return -2;
    }
    int dev = 0;
    if( ! ck( nullptr, cudaGetDevice( & dev ), "cudaGetDevice" ) )
        return -1;
    if( dev < 0 || dev >= 64 )
    {
        g_create_error = "kr_c2p_dt_noalloc: device ordinal out of range";
        return -1;
    }
    unsigned long long * scratch;
    {
        std::lock_guard< std::mutex > lk( g_noalloc_mx );
        if( ! g_noalloc_ptr[ dev ] )
        {   // first call on this device: resolve the array's device address
            void * p = nullptr;
            if( ! ck( nullptr, cudaGetSymbolAddress( & p, g_noalloc_scratch ), "cudaGetSymbolAddress" ) )
                return -1;
            g_noalloc_ptr[ dev ] = ( unsigned long long * ) p;
        }
        scratch = g_noalloc_ptr[ dev ];
    }
    cudaStream_t st = ( cudaStream_t ) stream;
    if( ! ck( nullptr, cudaMemsetAsync( scratch, 0, sizeof( unsigned long long ), st ), "clear counter" ) )
        return -1;
    // uniform block geometry as meshgen computes it for a single-block mesh
    double dx[ 3 ];
    for( int a = 0; a < 3; ++ a )
    {
        const double l0 = cfg->x_min[ a ] + ( 0 + 0.0 / cfg->n[ a ] ) / 1.0 * ( cfg->x_max[ a ] - cfg->x_min[ a ] );
        const double l1 = cfg->x_min[ a ] + ( 0 + 1.0 / cfg->n[ a ] ) / 1.0 * ( cfg->x_max[ a ] - cfg->x_min[ a ] );
        dx[ a ] = l1 - l0;
    }
    const unsigned grid = unsigned( ( nc + NOALLOC_THREADS - 1 ) / NOALLOC_THREADS );
    if( cfg->mhd )
        k_c2p_dt_noalloc< true ><<< grid, NOALLOC_THREADS, 0, st >>>( u, bf, w, dt_out, scratch,
            cfg->n[ 0 ], cfg->n[ 1 ], cfg->n[ 2 ], cfg->gamma, cfg->cfl, cfg->rho_floor, cfg->tmp_floor,
            dx[ 0 ], dx[ 1 ], dx[ 2 ] );
    else
        k_c2p_dt_noalloc< false ><<< grid, NOALLOC_THREADS, 0, st >>>( u, bf, w, dt_out, scratch,
            cfg->n[ 0 ], cfg->n[ 1 ], cfg->n[ 2 ], cfg->gamma, cfg->cfl, cfg->rho_floor, cfg->tmp_floor,
            dx[ 0 ], dx[ 1 ], dx[ 2 ] );
    return ck( nullptr, cudaGetLastError(  ), "kr_c2p_dt_noalloc launch" ) ? 0 : -1;
}
#include "kr_batch.cuh"
