/* CPU restatement (FP64) of the Kratos hydro / ideal-MHD step.  TEST
 * INFRASTRUCTURE ONLY -- see kr_oracle.h for scope, layout and conventions.
 * Build: oracle/Makefile (gcc, no fused multiply-add). */
#define _GNU_SOURCE                      /* qsort_r */
#include "kr_oracle.h"
#include "../../kratos_b200/csrc/problems.h"
#include "../../kratos_b200/csrc/smr_tree.h"

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

enum { RHO = 0, ENE = 1, MOM = 2, BCC = 5 };       /* dynamics/indices.h:5-13 */

struct kro_mesh
{
    kro_cfg c;
    int     nw, nblk;
    long    ncell;                       /* interior cells per block        */
    int     gw[ 3 ];                     /* w extents with 2 ghosts         */
    long    nw_cells;
    int     gb[ 3 ];                     /* bf lattice extents (n+1+4)      */
    long    nbf;
    int     gf[ 3 ][ 3 ];                /* flux extents per axis, 1 ghost  */
    long    nf[ 3 ];
    int     ge[ 3 ];                     /* edge lattice extents (n+1+2)    */
    long    nee;
    /* per block geometry (meshgen.cpp:286-363) */
    double *xf0, *dx0, *sfc0, *vol0;     /* [nblk*3], [nblk*3], [nblk*3], [nblk] */
    double *u[ 2 ], *bf[ 2 ], *w, *f[ 3 ], *ee;
    double *dtc;                         /* per block CFL minimum           */
    kr_tree tree;                        /* blocks: levels, positions, faces */
    int     smr;                         /* more than one level             */
    struct mh_holder * hold;             /* MHD refined meshes: the exchange */
    int     n_hold;                      /* holders, in the reference's order */
};

static void build_holders( kro_mesh * m );   /* refined MHD meshes, below */

/* logical position and per-axis block count of block b's level */
static inline const int * blk_reg( const kro_mesh * m, int b ) { return m->tree.reg + 3 * b; }
static inline int blk_lim( const kro_mesh * m, int b, int a ) { return m->c.nb[ a ] << m->tree.level[ b ]; }

/* ------------------------------------------------------------------ */
/* indexing                                                             */

static inline long iw( const kro_mesh * m, int i0, int i1, int i2 )
{
    return ( ( i0 + 2 ) + m->gw[ 0 ] * ( ( long )( i1 + 2 ) + m->gw[ 1 ] * ( long )( i2 + 2 ) ) )
           * m->nw;
}
static inline long iu( const kro_mesh * m, int i0, int i1, int i2 )
{
    return ( i0 + m->c.n[ 0 ] * ( ( long ) i1 + m->c.n[ 1 ] * ( long ) i2 ) ) * m->nw;
}
static inline long ib( const kro_mesh * m, int i0, int i1, int i2 )
{
    return ( ( i0 + 2 ) + m->gb[ 0 ] * ( ( long )( i1 + 2 ) + m->gb[ 1 ] * ( long )( i2 + 2 ) ) ) * 3;
}
static inline long ifl( const kro_mesh * m, int a, int i0, int i1, int i2 )
{
    const int * g = m->gf[ a ];
    return ( ( i0 + 1 ) + g[ 0 ] * ( ( long )( i1 + 1 ) + g[ 1 ] * ( long )( i2 + 1 ) ) ) * m->nw;
}
static inline long ie( const kro_mesh * m, int i0, int i1, int i2 )
{
    return ( ( i0 + 1 ) + m->ge[ 0 ] * ( ( long )( i1 + 1 ) + m->ge[ 1 ] * ( long )( i2 + 1 ) ) ) * 3;
}
static inline int mod3( int a ) { return a < 3 ? a : a - 3; }

/* utilities/functions.h:51-64 (PRECISION == 2) */
static inline double dmax( double a, double b ) { return a > b ? a : b; }
static inline double dmin( double a, double b ) { return a < b ? a : b; }
static inline double uabs( double a ) { return a > 0 ? a : -a; }   /* functions.h:32-36 */
static inline int    sgn ( double a ) { return a > 0 ? 1 : ( a < 0 ? -1 : 0 ); }

/* utilities/mapping/mapping.h idx_swap: cyclic rotation of a 3-vector */
static inline void idx_swap( double * x, int axis )
{
    if( mod3( axis ) != 0 )
    {
        double s[ 3 ];
        for( int i = 0; i < 3; ++ i )
            s[ i ] = x[ mod3( i + axis ) ];
        for( int i = 0; i < 3; ++ i )
            x[ i ] = s[ i ];
    }
}

/* ------------------------------------------------------------------ */
/* thread helper: run fn(m, b, aux) for every block                      */

typedef void ( * blk_fn )( kro_mesh *, int, void * );
typedef struct { kro_mesh * m; blk_fn fn; void * aux; int next; pthread_mutex_t mx; } pf_t;

static void * pf_worker( void * p )
{
    pf_t * pf = ( pf_t * ) p;
    for( ;; )
    {
        pthread_mutex_lock( & pf->mx );
        const int b = pf->next ++;
        pthread_mutex_unlock( & pf->mx );
        if( b >= pf->m->nblk )
            break;
        pf->fn( pf->m, b, pf->aux );
    }
    return NULL;
}

static void par_blocks( kro_mesh * m, blk_fn fn, void * aux )
{
    int nt = m->c.n_threads > 0 ? m->c.n_threads : ( int ) sysconf( _SC_NPROCESSORS_ONLN );
    if( nt > m->nblk ) nt = m->nblk;
    if( nt <= 1 )
    {
        for( int b = 0; b < m->nblk; ++ b )
            fn( m, b, aux );
        return;
    }
    pf_t pf = { m, fn, aux, 0 };
    pthread_mutex_init( & pf.mx, NULL );
    pthread_t th[ 256 ];
    if( nt > 256 ) nt = 256;
    for( int t = 0; t < nt; ++ t )
        pthread_create( & th[ t ], NULL, pf_worker, & pf );
    for( int t = 0; t < nt; ++ t )
        pthread_join( th[ t ], NULL );
    pthread_mutex_destroy( & pf.mx );
}

/* ------------------------------------------------------------------ */
/* geometry (mesh/meshgen/meshgen.cpp:252-363, geometry/geometry.h:73-150) */

static void set_geometry( kro_mesh * m )
{
    for( int b = 0; b < m->nblk; ++ b )
    {
        const int * reg = blk_reg( m, b );
        for( int a = 0; a < 3; ++ a )
        {
            /* loc(i) = location( ( reg + i / n ) / ( i_logic_lim << level ) ) */
            const double lim = ( double ) blk_lim( m, b, a );
            const double x0 = ( reg[ a ] + 0.0 / m->c.n[ a ] ) / lim;
            const double x1 = ( reg[ a ] + 1.0 / m->c.n[ a ] ) / lim;
            const double l0 = m->c.x_min[ a ] + x0 * ( m->c.x_max[ a ] - m->c.x_min[ a ] );
            const double l1 = m->c.x_min[ a ] + x1 * ( m->c.x_max[ a ] - m->c.x_min[ a ] );
            m->xf0[ b * 3 + a ] = l0;
            m->dx0[ b * 3 + a ] = l1 - l0;
        }
        /* surface(): res = 1; res *= dx_f( (a+1)%3 ); res *= dx_f( (a+2)%3 ) */
        double vol = 1.;
        for( int a = 0; a < 3; ++ a )
        {
            double s = 1.;
            s *= m->dx0[ b * 3 + ( a + 1 ) % 3 ];
            s *= m->dx0[ b * 3 + ( a + 2 ) % 3 ];
            m->sfc0[ b * 3 + a ] = s;
            vol *= m->dx0[ b * 3 + a ];
        }
        m->vol0[ b ] = vol;
    }
}

double kro_x_cc( const kro_mesh * m, int b, int a, int i )
{
    return m->xf0[ b * 3 + a ] + ( i + 0.5f ) * m->dx0[ b * 3 + a ];   /* geometry.h:73-79 */
}
double kro_x_fc( const kro_mesh * m, int b, int a, int i )
{
    return m->xf0[ b * 3 + a ] + i * m->dx0[ b * 3 + a ];              /* geometry.h:80-95 */
}
double kro_dx( const kro_mesh * m, int b, int a ) { return m->dx0[ b * 3 + a ]; }

/* ------------------------------------------------------------------ */
/* create / destroy / state                                             */

kro_mesh * kro_create( const kro_cfg * cfg )
{
    return kro_create_tree( cfg, 0, NULL );
}

kro_mesh * kro_create_tree( const kro_cfg * cfg, int n_regions, const kro_region * regions )
{
    kro_mesh * m = ( kro_mesh * ) calloc( 1, sizeof( kro_mesh ) );
    m->c    = * cfg;
    m->nw   = cfg->mhd ? 8 : 5;
    {   /* meshgen.cpp:51-55: an axis is periodic when its kinds say "per" */
        int per[ 3 ];
        kr_tree_region * rg = ( kr_tree_region * ) calloc( n_regions > 0 ? n_regions : 1, sizeof( * rg ) );
        for( int a = 0; a < 3; ++ a )
            per[ a ] = cfg->bc[ 2 * a ] == KRO_PER && cfg->bc[ 2 * a + 1 ] == KRO_PER;
        for( int k = 0; k < n_regions; ++ k )
        {
            rg[ k ].level = regions[ k ].level;
            for( int a = 0; a < 3; ++ a )
            {
                rg[ k ].x_min[ a ] = regions[ k ].x_min[ a ];
                rg[ k ].x_max[ a ] = regions[ k ].x_max[ a ];
            }
        }
        const int r = kr_tree_build( & m->tree, cfg->nb, per, cfg->x_min, cfg->x_max,
                                     n_regions, rg, NULL, 0 );
        free( rg );
        if( r != 0 )
        {
            kr_tree_free( & m->tree );
            free( m );
            return NULL;
        }
    }
    m->smr  = m->tree.max_level > 0;
    m->nblk = m->tree.nblk;
    m->ncell = ( long ) cfg->n[ 0 ] * cfg->n[ 1 ] * cfg->n[ 2 ];
    m->nw_cells = 1; m->nbf = 3; m->nee = 3;
    for( int a = 0; a < 3; ++ a )
    {
        m->gw[ a ] = cfg->n[ a ] + 4;
        m->gb[ a ] = cfg->n[ a ] + 5;
        m->ge[ a ] = cfg->n[ a ] + 3;
        m->nw_cells *= m->gw[ a ];
        m->nbf *= m->gb[ a ];
        m->nee *= m->ge[ a ];
    }
    for( int a = 0; a < 3; ++ a )
    {
        m->nf[ a ] = m->nw;
        for( int d = 0; d < 3; ++ d )
        {
            m->gf[ a ][ d ] = cfg->n[ d ] + ( d == a ) + 2;
            m->nf[ a ] *= m->gf[ a ][ d ];
        }
    }
    m->xf0  = ( double * ) calloc( m->nblk * 3, sizeof( double ) );
    m->dx0  = ( double * ) calloc( m->nblk * 3, sizeof( double ) );
    m->sfc0 = ( double * ) calloc( m->nblk * 3, sizeof( double ) );
    m->vol0 = ( double * ) calloc( m->nblk, sizeof( double ) );
    m->dtc  = ( double * ) calloc( m->nblk, sizeof( double ) );
    for( int s = 0; s < 2; ++ s )
    {
        m->u [ s ] = ( double * ) calloc( ( size_t ) m->nblk * m->ncell * m->nw, sizeof( double ) );
        m->bf[ s ] = ( double * ) calloc( ( size_t ) m->nblk * m->nbf, sizeof( double ) );
    }
    m->w = ( double * ) calloc( ( size_t ) m->nblk * m->nw_cells * m->nw, sizeof( double ) );
    for( int a = 0; a < 3; ++ a )
        m->f[ a ] = ( double * ) calloc( ( size_t ) m->nblk * m->nf[ a ], sizeof( double ) );
    m->ee = ( double * ) calloc( ( size_t ) m->nblk * m->nee, sizeof( double ) );
    set_geometry( m );
    if( m->smr && cfg->mhd )
        build_holders( m );
    return m;
}

int kro_nblk( const kro_mesh * m ) { return m->nblk; }

void kro_block_info( const kro_mesh * m, int * level, int * reg )
{
    for( int b = 0; b < m->nblk; ++ b )
    {
        if( level ) level[ b ] = m->tree.level[ b ];
        if( reg )
            for( int a = 0; a < 3; ++ a )
                reg[ 3 * b + a ] = m->tree.reg[ 3 * b + a ];
    }
}

void kro_destroy( kro_mesh * m )
{
    if( ! m ) return;
    kr_tree_free( & m->tree );
    free( m->xf0 ); free( m->dx0 ); free( m->sfc0 ); free( m->vol0 ); free( m->dtc );
    for( int s = 0; s < 2; ++ s ) { free( m->u[ s ] ); free( m->bf[ s ] ); }
    free( m->w );
    for( int a = 0; a < 3; ++ a ) free( m->f[ a ] );
    free( m->ee );
    free( m->hold );
    free( m );
}

int  kro_nw   ( const kro_mesh * m ) { return m->nw; }
long kro_ncell( const kro_mesh * m ) { return m->ncell; }
long kro_nface( const kro_mesh * m ) { return m->nbf / 3; }

void kro_set_state( kro_mesh * m, const double * u, const double * bf )
{
    memcpy( m->u[ 0 ], u, sizeof( double ) * m->nblk * m->ncell * m->nw );
    if( m->c.mhd && bf )
        memcpy( m->bf[ 0 ], bf, sizeof( double ) * m->nblk * m->nbf );
}
void kro_get_state( const kro_mesh * m, double * u, double * bf )
{
    memcpy( u, m->u[ 0 ], sizeof( double ) * m->nblk * m->ncell * m->nw );
    if( m->c.mhd && bf )
        memcpy( bf, m->bf[ 0 ], sizeof( double ) * m->nblk * m->nbf );
}

/* ------------------------------------------------------------------ */
/* EOS                                                                  */

/* hydro/eos/adiabatic.h:62-76 et_cs: total energy and sound speed of a
 * primitive state; returns cv_kb = 1 / ( gamma - 1 ). */
static inline double et_cs( double gamma, double * e_tot, double * c_s, const double * w )
{
    const double pre = w[ ENE ], rho = w[ RHO ];
    const double cv_kb = 1 / ( gamma - 1 );
    double v2 = 0;
    for( int a = 0; a < 3; ++ a )
        v2 += w[ MOM + a ] * w[ MOM + a ];
    * e_tot = pre * cv_kb + rho * v2 / 2;
    * c_s   = sqrt( gamma * dmax( pre / rho, 0 ) );
    return cv_kb;
}

/* hydro/eos/adiabatic.h:159-206 c2p (+ pre_cs2 77-85).  cons: the cell's
 * conserved state (floor corrections are written back); prim: output.
 * Returns the squared sound speed. */
static double c2p( const kro_mesh * m, double * prim, double * cons )
{
    const double gamma = m->c.gamma;
    double rho = cons[ RHO ];
    if( isnan( rho ) || rho < m->c.d_floor )
    {
        rho = m->c.d_floor;
        cons[ RHO ] = m->c.d_floor;
    }
    prim[ RHO ] = rho;
    const double rho_inv = 1 / rho;
    double e_k = 0.;
    for( int n = MOM; n < MOM + 3; ++ n )
    {
        prim[ n ] = rho_inv * cons[ n ];
        e_k += cons[ n ] * cons[ n ];
    }
    e_k *= rho_inv / 2;
    const double e_g = cons[ ENE ] - e_k;
    const double cv_kb = 1 / ( gamma - 1 );
    prim[ ENE ] = e_g / cv_kb;
    double cs2 = gamma * prim[ ENE ] / prim[ RHO ];
    double pre = prim[ ENE ];
    const double pre_floor = m->c.t_floor * prim[ RHO ];
    if( isnan( pre ) || pre < pre_floor )
    {
        pre = pre_floor;
        prim[ ENE ] = pre;
        cons[ ENE ] = e_k + pre / ( gamma - 1 );
        cs2 = gamma * pre / rho;
    }
    return cs2;
}

/* mhd/eos/adiabatic.h:84-98 fast magnetosonic speed along axis */
static inline double c_fms( const double * w, const double * b_2, double gam, int axis )
{
    const double rho  = w[ RHO ];
    const double cs_2 = w[ ENE ] * gam / rho;
    const double v_ax2 = b_2[ axis ] / rho;
    const double v_t2 = ( b_2[ mod3( axis + 1 ) ] + b_2[ mod3( axis + 2 ) ] ) / rho;
    const double q_2 = v_ax2 + v_t2 + cs_2;
    const double r_2 = v_ax2 + v_t2 - cs_2;
    return sqrt( 0.5f * ( q_2 + sqrt( r_2 * r_2 + 4 * cs_2 * v_t2 ) ) );
}

/* Per-block cons -> prim over the interior, from RK slot `step`.
 * hydro: hydro/eos/adiabatic.h:211-258; MHD: mhd/eos/adiabatic.h:127-234.
 * Stage 0 also takes the per-cell CFL dt (adiabatic.h:146-157 /
 * mhd/eos/adiabatic.h:105-122) into m->dtc[b]. */
typedef struct { int step; } c2p_arg;

static void c2p_block( kro_mesh * m, int b, void * aux )
{
    const int step = ( ( c2p_arg * ) aux )->step;
    const int nw = m->nw;
    const int * n = m->c.n;
    double * u  = m->u[ step ] + ( size_t ) b * m->ncell * nw;
    double * bf = m->c.mhd ? m->bf[ step ] + ( size_t ) b * m->nbf : NULL;
    double * w  = m->w + ( size_t ) b * m->nw_cells * nw;
    const double * dx = m->dx0 + b * 3;
    double dt_min = FLT_MAX;
    for( int i2 = 0; i2 < n[ 2 ]; ++ i2 )
    for( int i1 = 0; i1 < n[ 1 ]; ++ i1 )
    for( int i0 = 0; i0 < n[ 0 ]; ++ i0 )
    {
        double * c = u + iu( m, i0, i1, i2 );
        double * p = w + iw( m, i0, i1, i2 );
        double prim[ 8 ], cons[ 8 ];
        double dt = FLT_MAX;
        if( ! m->c.mhd )
        {
            for( int k = 0; k < 5; ++ k ) cons[ k ] = c[ k ];
            const double cs2 = c2p( m, prim, cons );
            c[ RHO ] = cons[ RHO ];
            c[ ENE ] = cons[ ENE ];
            for( int k = 0; k < 5; ++ k ) p[ k ] = prim[ k ];
            if( step == 0 )
            {
                const double cs = sqrt( cs2 );
                for( int a = 0; a < 3; ++ a )
                    dt = dmin( dt, dx[ a ] / ( cs + fabs( prim[ MOM + a ] ) ) );
                dt = dt * m->c.cfl;
            }
        }
        else
        {
            const int ii[ 3 ] = { i0, i1, i2 };
            double bc[ 3 ], bc_2[ 3 ], b_max[ 3 ];
            double e_m = 0;
            for( int a = 0; a < 3; ++ a )
            {
                int jj[ 3 ] = { ii[ 0 ], ii[ 1 ], ii[ 2 ] };
                const double b_l = bf[ ib( m, jj[ 0 ], jj[ 1 ], jj[ 2 ] ) + a ];
                ++ jj[ a ];
                const double b_r = bf[ ib( m, jj[ 0 ], jj[ 1 ], jj[ 2 ] ) + a ];
                const double bc_m = ( b_l + b_r ) / 2;
                bc[ a ] = bc_m;
                const double bcs2 = bc_m * bc_m;
                e_m += bcs2;
                bc_2 [ a ] = bcs2;
                b_max[ a ] = dmax( fabs( b_l ), fabs( b_r ) );
            }
            e_m /= 2;
            c[ ENE ] -= e_m;
            for( int k = 0; k < 8; ++ k ) cons[ k ] = c[ k ];
            ( void ) c2p( m, prim, cons );
            c[ RHO ] = cons[ RHO ];
            c[ ENE ] = cons[ ENE ];
            c[ ENE ] += e_m;
            for( int k = 0; k < 5; ++ k ) p[ k ] = prim[ k ];
            for( int a = 0; a < 3; ++ a )
            {
                p[ BCC + a ] = bc[ a ];
                c[ BCC + a ] = bc[ a ];
            }
            if( step == 0 )
            {
                double bm_2[ 3 ] = { bc_2[ 0 ], bc_2[ 1 ], bc_2[ 2 ] };
                for( int a = 0; a < 3; ++ a )
                {
                    bm_2[ a ] = b_max[ a ] * b_max[ a ];
                    const double cf = c_fms( prim, bm_2, m->c.gamma, a );
                    dt = dmin( dt, dx[ a ] / ( cf + fabs( prim[ MOM + a ] ) ) );
                    bm_2[ a ] = bc_2[ a ];
                }
                dt = dt * m->c.cfl;
            }
        }
        if( step == 0 )
            dt_min = dmin( dt_min, dt );
    }
    m->dtc[ b ] = dt_min;
}

/* cons -> prim (with floors) and the CFL dt of the state in slot 0, without
 * stepping: w_out [nblk][n2][n1][n0][nw] interior primitives (MHD: rho, p,
 * v0..2, B_cc0..2), dt_out [nblk] each block's cfl * min dx / signal speed.
 * Floor corrections heal slot 0's conserved state as the step's c2p does. */
void kro_c2p_dt( kro_mesh * m, double * w_out, double * dt_out )
{
    c2p_arg ca = { 0 };
    for( int b = 0; b < m->nblk; ++ b )
    {
        c2p_block( m, b, & ca );
        dt_out[ b ] = m->dtc[ b ];
        const int * n = m->c.n;
        const double * w = m->w + ( size_t ) b * m->nw_cells * m->nw;
        double * o = w_out + ( size_t ) b * m->ncell * m->nw;
        for( int i2 = 0; i2 < n[ 2 ]; ++ i2 )
        for( int i1 = 0; i1 < n[ 1 ]; ++ i1 )
        for( int i0 = 0; i0 < n[ 0 ]; ++ i0 )
            for( int k = 0; k < m->nw; ++ k )
                o[ iu( m, i0, i1, i2 ) + k ] = w[ iw( m, i0, i1, i2 ) + k ];
    }
}

/* ------------------------------------------------------------------ */
/* ghost fill (same level, periodic): every ghost cell of w and every  */
/* non-owned face slot of bf takes the value of the block that owns it */
/* (hydro/boundary/comm_functions.h:306-327, 456-483; MHD              */
/* mhd/boundary/comm_functions.h:433-465, 786-815).                   */

static inline int wrap( int i, int n, int * shift )
{
    if( i < 0 )       { * shift = -1; return i + n; }
    if( i >= n )      { * shift = +1; return i - n; }
    * shift = 0; return i;
}

static inline int periodic_axis( const kro_mesh * m, int a )
{   /* meshgen.cpp:51-55: an axis is periodic when its kinds say "per" */
    return m->c.bc[ 2 * a ] == KRO_PER && m->c.bc[ 2 * a + 1 ] == KRO_PER;
}

/* Neighbour block in direction sh, or -1 past a non-periodic domain edge
 * (no tree neighbour there: tree.cpp neighbour search). */
static inline int nbr_block( const kro_mesh * m, int b, const int sh[ 3 ] )
{
    int reg[ 3 ] = { b % m->c.nb[ 0 ], ( b / m->c.nb[ 0 ] ) % m->c.nb[ 1 ],
                     b / ( m->c.nb[ 0 ] * m->c.nb[ 1 ] ) };
    for( int a = 0; a < 3; ++ a )
    {
        reg[ a ] += sh[ a ];
        if( reg[ a ] < 0 || reg[ a ] >= m->c.nb[ a ] )
        {
            if( ! periodic_axis( m, a ) )
                return -1;
            reg[ a ] = ( reg[ a ] + m->c.nb[ a ] ) % m->c.nb[ a ];
        }
    }
    return reg[ 0 ] + m->c.nb[ 0 ] * ( reg[ 1 ] + m->c.nb[ 1 ] * reg[ 2 ] );
}

typedef struct { int step; int no_field; } ghost_arg;   /* no_field: MHD sides, primitives only */

static void ghost_block( kro_mesh * m, int b, void * aux )
{
    const int step = ( ( ghost_arg * ) aux )->step;
    const int nw = m->nw;
    const int * n = m->c.n;
    double * w = m->w + ( size_t ) b * m->nw_cells * nw;
    for( int i2 = -2; i2 < n[ 2 ] + 2; ++ i2 )
    for( int i1 = -2; i1 < n[ 1 ] + 2; ++ i1 )
    for( int i0 = -2; i0 < n[ 0 ] + 2; ++ i0 )
    {
        int sh[ 3 ], j[ 3 ];
        j[ 0 ] = wrap( i0, n[ 0 ], & sh[ 0 ] );
        j[ 1 ] = wrap( i1, n[ 1 ], & sh[ 1 ] );
        j[ 2 ] = wrap( i2, n[ 2 ], & sh[ 2 ] );
        if( ! sh[ 0 ] && ! sh[ 1 ] && ! sh[ 2 ] )
            continue;
        const int s = nbr_block( m, b, sh );
        if( s < 0 )
            continue;                        /* physical boundary: bc_block */
        const double * src = m->w + ( size_t ) s * m->nw_cells * nw + iw( m, j[ 0 ], j[ 1 ], j[ 2 ] );
        memcpy( w + iw( m, i0, i1, i2 ), src, sizeof( double ) * nw );
    }
    if( ! m->c.mhd )
        return;
    double * bf = m->bf[ step ] + ( size_t ) b * m->nbf;
    for( int c = 0; c < 3; ++ c )
    for( int i2 = -2; i2 <= n[ 2 ] + 2; ++ i2 )
    for( int i1 = -2; i1 <= n[ 1 ] + 2; ++ i1 )
    for( int i0 = -2; i0 <= n[ 0 ] + 2; ++ i0 )
    {
        const int ii[ 3 ] = { i0, i1, i2 };
        int own = 1, sh[ 3 ], j[ 3 ];
        for( int a = 0; a < 3; ++ a )
        {
            const int hi = ( a == c ) ? n[ a ] : n[ a ] - 1;
            own &= ii[ a ] >= 0 && ii[ a ] <= hi;
        }
        if( own )
            continue;
        int ok = 1;
        for( int a = 0; a < 3; ++ a )
        {
            if( a == c )
            {   /* face index: owned 0..n; wrap outside that range */
                if( ii[ a ] < 0 )          { sh[ a ] = -1; j[ a ] = ii[ a ] + n[ a ]; }
                else if( ii[ a ] > n[ a ] ) { sh[ a ] = +1; j[ a ] = ii[ a ] - n[ a ]; }
                else                        { sh[ a ] = 0;  j[ a ] = ii[ a ]; }
            }
            else
                j[ a ] = wrap( ii[ a ], n[ a ], & sh[ a ] );
            ok &= j[ a ] >= -2 && j[ a ] <= n[ a ] + 2;
        }
        if( ! ok )
            continue;
        const int s = nbr_block( m, b, sh );
        bf[ ib( m, i0, i1, i2 ) + c ]
            = m->bf[ step ][ ( size_t ) s * m->nbf + ib( m, j[ 0 ], j[ 1 ], j[ 2 ] ) + c ];
    }
}

/* ------------------------------------------------------------------ */
/* Physical boundaries on the primitives (hydro/boundary/phys.h:95-139,  */
/* phys_functors.h:11-91): for every transverse interior position of a   */
/* domain-edge side, the n_gh cells next to the boundary are copied to a */
/* buffer (index 0 = adjacent cell), the functor fills the ghost part of */
/* the buffer, and the ghosts are written back.                          */

static void bc_block( kro_mesh * m, int b, void * aux )
{
    ( void ) aux;
    const int nw = m->nw;
    const int * n = m->c.n;
    const int * reg = blk_reg( m, b );
    double * w = m->w + ( size_t ) b * m->nw_cells * nw;
    for( int side = 0; side < 6; ++ side )
    {
        const int axis = side / 2, right = side & 1;
        const int kind = m->c.bc[ side ];
        if( kind == KRO_PER )
            continue;
        if( reg[ axis ] != ( right ? blk_lim( m, b, axis ) - 1 : 0 ) )
            continue;                        /* not on this domain edge */
        const int a1 = mod3( axis + 1 ), a2 = mod3( axis + 2 );
        const int i_mom = MOM + axis;
        for( int t2 = 0; t2 < n[ a2 ]; ++ t2 )
        for( int t1 = 0; t1 < n[ a1 ]; ++ t1 )
        {
            double buf[ 4 ][ 8 ];            /* rows -2, -1, 0, 1 */
            int ii[ 3 ];
            ii[ a1 ] = t1;
            ii[ a2 ] = t2;
            for( int i = 0; i < 2; ++ i )
            {
                ii[ axis ] = right ? n[ axis ] - i - 1 : i;
                memcpy( buf[ 2 + i ], w + iw( m, ii[ 0 ], ii[ 1 ], ii[ 2 ] ), sizeof( double ) * nw );
            }
            if( kind == KRO_OUT )
            {
                if( buf[ 2 ][ i_mom ] * ( right ? -1 : 1 ) > 0 )
                    buf[ 2 ][ i_mom ] = 0;
                for( int i = -2; i < 0; ++ i )
                    memcpy( buf[ 2 + i ], buf[ 2 ], sizeof( double ) * nw );
            }
            else if( kind == KRO_FRE )
                for( int i = -2; i < 0; ++ i )
                    memcpy( buf[ 2 + i ], buf[ 2 ], sizeof( double ) * nw );
            else if( kind == KRO_REF )
                for( int i = -2; i < 0; ++ i )
                    for( int k = 0; k < nw; ++ k )
                        buf[ 2 + i ][ k ] = buf[ 2 - i - 1 ][ k ] * ( k == i_mom ? -1 : 1 );
            else if( kind == KRO_FIXD )
                for( int i = -2; i < 0; ++ i )
                    for( int k = 0; k < nw; ++ k )
                        buf[ 2 + i ][ k ] = m->c.w_fix[ k ];
            for( int i = -2; i < 0; ++ i )
            {
                ii[ axis ] = right ? n[ axis ] - i - 1 : i;
                memcpy( w + iw( m, ii[ 0 ], ii[ 1 ], ii[ 2 ] ), buf[ 2 + i ], sizeof( double ) * nw );
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* Static refinement, hydro: the ghost cells of a face whose neighbour   */
/* is on another level (hydro/boundary/comm_functions.h:268-380         */
/* to_same / to_coarser / to_finer; face neighbours only,               */
/* keeper.cpp:86-89 desired_mode).  keeper.cpp:148-160 act_bnd runs the  */
/* restrictions (finer -> coarser ghosts), the physical sides, the       */
/* same-level copies and then the prolongations (coarser -> finer        */
/* ghosts), which read the coarse block's ghosts filled before.          */

static void smr_same_block( kro_mesh * m, int b, void * aux )
{
    ( void ) aux;
    const int nw = m->nw;
    const int * n = m->c.n;
    double * w = m->w + ( size_t ) b * m->nw_cells * nw;
    for( int f = 0; f < 6; ++ f )
    {
        if( m->tree.face[ 6 * b + f ] != KR_FACE_SAME )
            continue;
        const int a = f / 2, s = f & 1, a1 = mod3( a + 1 ), a2 = mod3( a + 2 );
        const int src = m->tree.fnb[ ( 6 * b + f ) * 4 ];
        const double * ws = m->w + ( size_t ) src * m->nw_cells * nw;
        for( int g = 0; g < 2; ++ g )
        for( int t2 = 0; t2 < n[ a2 ]; ++ t2 )
        for( int t1 = 0; t1 < n[ a1 ]; ++ t1 )
        {
            int ii[ 3 ], jj[ 3 ];
            ii[ a1 ] = jj[ a1 ] = t1;
            ii[ a2 ] = jj[ a2 ] = t2;
            ii[ a ] = s ? n[ a ] + g : g - 2;
            jj[ a ] = s ? g : n[ a ] - 2 + g;
            memcpy( w + iw( m, ii[ 0 ], ii[ 1 ], ii[ 2 ] ), ws + iw( m, jj[ 0 ], jj[ 1 ], jj[ 2 ] ),
                    sizeof( double ) * nw );
        }
    }
}

/* comm_functions.h:329-380 to_coarser: a coarse ghost cell is the volume
 * average of the 8 fine cells it covers, accumulated fine layer by fine
 * layer in increasing index, (d1, d2) with d1 outer in each layer. */
static void smr_restrict_block( kro_mesh * m, int b, void * aux )
{
    ( void ) aux;
    const int nw = m->nw;
    const int * n = m->c.n;
    double * w = m->w + ( size_t ) b * m->nw_cells * nw;
    for( int f = 0; f < 6; ++ f )
    {
        if( m->tree.face[ 6 * b + f ] != KR_FACE_FINE )
            continue;
        const int a = f / 2, s = f & 1, a1 = mod3( a + 1 ), a2 = mod3( a + 2 );
        const int h1 = n[ a1 ] / 2, h2 = n[ a2 ] / 2;
        for( int d1 = 0; d1 < 2; ++ d1 )
        for( int d2 = 0; d2 < 2; ++ d2 )
        {
            const int fb = m->tree.fnb[ ( 6 * b + f ) * 4 + d1 * 2 + d2 ];
            const double * wf = m->w + ( size_t ) fb * m->nw_cells * nw;
            const double dv = m->vol0[ fb ];
            for( int gl = 0; gl < 2; ++ gl )
            for( int t2 = 0; t2 < h2; ++ t2 )
            for( int t1 = 0; t1 < h1; ++ t1 )
            {
                double p[ 8 ] = { 0 }, norm = 0;
                for( int kk = 0; kk < 2; ++ kk )
                {
                    const int k = 2 * gl + kk;       /* fine layer from offset_s */
                    for( int e1 = 0; e1 < 2; ++ e1 )
                    for( int e2 = 0; e2 < 2; ++ e2 )
                    {
                        int jj[ 3 ];
                        jj[ a ] = s ? k : n[ a ] - 4 + k;
                        jj[ a1 ] = 2 * t1 + e1;
                        jj[ a2 ] = 2 * t2 + e2;
                        const double * q = wf + iw( m, jj[ 0 ], jj[ 1 ], jj[ 2 ] );
                        for( int c = 0; c < nw; ++ c )
                            p[ c ] += q[ c ] * dv;
                        norm += dv;
                    }
                }
                int ii[ 3 ];
                ii[ a ] = s ? n[ a ] + gl : gl - 2;
                ii[ a1 ] = d1 * h1 + t1;
                ii[ a2 ] = d2 * h2 + t2;
                double * o = w + iw( m, ii[ 0 ], ii[ 1 ], ii[ 2 ] );
                for( int c = 0; c < nw; ++ c )
                    o[ c ] = p[ c ] / norm;
            }
        }
    }
}

static inline double minmod( double a, double b )
{   /* utilities/functions.h:159-170 */
    return ( ( a < 0 ) ^ ( b < 0 ) ) ? 0 : ( fabs( a ) < fabs( b ) ? a : b );
}

/* comm_functions.h:382-447 to_finer: each coarse cell next to the face
 * gives its 2 x 2 x 2 fine ghost cells q_c + sum over axes of
 * +-minmod(q_r - q_c, q_c - q_l) / 4 (normal axis first, then (a+1)%3,
 * (a+2)%3).  Blocks of one level per call (aux: the level), coarser
 * levels first, since a coarse block's own ghosts feed its slopes. */
typedef struct { int level; } prol_arg;

static void smr_prolong_block( kro_mesh * m, int b, void * aux )
{
    if( m->tree.level[ b ] != ( ( const prol_arg * ) aux )->level )
        return;
    const int nw = m->nw;
    const int * n = m->c.n;
    double * w = m->w + ( size_t ) b * m->nw_cells * nw;
    const int * rf = blk_reg( m, b );
    for( int f = 0; f < 6; ++ f )
    {
        if( m->tree.face[ 6 * b + f ] != KR_FACE_COARSE )
            continue;
        const int a = f / 2, s = f & 1, a1 = mod3( a + 1 ), a2 = mod3( a + 2 );
        const int h1 = n[ a1 ] / 2, h2 = n[ a2 ] / 2;
        const int cb = m->tree.fnb[ ( 6 * b + f ) * 4 ];
        const double * wc = m->w + ( size_t ) cb * m->nw_cells * nw;
        const int o1 = ( rf[ a1 ] & 1 ) * h1, o2 = ( rf[ a2 ] & 1 ) * h2;
        for( int t2 = 0; t2 < h2; ++ t2 )
        for( int t1 = 0; t1 < h1; ++ t1 )
        {
            int jc[ 3 ];
            jc[ a ] = s ? 0 : n[ a ] - 1;
            jc[ a1 ] = o1 + t1;
            jc[ a2 ] = o2 + t2;
            const double * qc = wc + iw( m, jc[ 0 ], jc[ 1 ], jc[ 2 ] );
            double dq[ 3 ][ 8 ];
            for( int d = 0; d < 3; ++ d )
            {
                int jr[ 3 ] = { jc[ 0 ], jc[ 1 ], jc[ 2 ] }, jl[ 3 ] = { jc[ 0 ], jc[ 1 ], jc[ 2 ] };
                ++ jr[ d ];
                -- jl[ d ];
                const double * qr = wc + iw( m, jr[ 0 ], jr[ 1 ], jr[ 2 ] );
                const double * ql = wc + iw( m, jl[ 0 ], jl[ 1 ], jl[ 2 ] );
                for( int c = 0; c < nw; ++ c )
                    dq[ d ][ c ] = minmod( qr[ c ] - qc[ c ], qc[ c ] - ql[ c ] ) * 0.25f;
            }
            for( int k = 0; k < 2; ++ k )
            for( int e1 = 0; e1 < 2; ++ e1 )
            for( int e2 = 0; e2 < 2; ++ e2 )
            {
                int ii[ 3 ];
                ii[ a ] = s ? n[ a ] + k : k - 2;
                ii[ a1 ] = 2 * t1 + e1;
                ii[ a2 ] = 2 * t2 + e2;
                double * o = w + iw( m, ii[ 0 ], ii[ 1 ], ii[ 2 ] );
                for( int c = 0; c < nw; ++ c )
                    o[ c ] = qc[ c ] + dq[ a ][ c ] * ( 2 * ( k & 1 ) - 1 )
                           + dq[ a1 ][ c ] * ( 2 * e1 - 1 )
                           + dq[ a2 ][ c ] * ( 2 * e2 - 1 );
            }
        }
    }
}

/* comm_functions.h:469-505 flux_to_buf / flux_from_buf: the coarse face
 * flux over a refined face becomes the area average of the 4 fine face
 * fluxes it covers ((d1, d2), d1 outer). */
static void smr_flux_block( kro_mesh * m, int b, void * aux )
{
    ( void ) aux;
    const int nw = m->nw;
    const int * n = m->c.n;
    for( int f = 0; f < 6; ++ f )
    {
        if( m->tree.face[ 6 * b + f ] != KR_FACE_FINE )
            continue;
        const int a = f / 2, s = f & 1, a1 = mod3( a + 1 ), a2 = mod3( a + 2 );
        const int h1 = n[ a1 ] / 2, h2 = n[ a2 ] / 2;
        double * fc = m->f[ a ] + ( size_t ) b * m->nf[ a ];
        for( int d1 = 0; d1 < 2; ++ d1 )
        for( int d2 = 0; d2 < 2; ++ d2 )
        {
            const int fb = m->tree.fnb[ ( 6 * b + f ) * 4 + d1 * 2 + d2 ];
            const double * ff = m->f[ a ] + ( size_t ) fb * m->nf[ a ];
            const double ds = m->sfc0[ fb * 3 + a ];
            for( int t2 = 0; t2 < h2; ++ t2 )
            for( int t1 = 0; t1 < h1; ++ t1 )
            {
                double acc[ 8 ] = { 0 }, norm = 0;
                for( int e1 = 0; e1 < 2; ++ e1 )
                for( int e2 = 0; e2 < 2; ++ e2 )
                {
                    int jj[ 3 ];
                    jj[ a ] = s ? 0 : n[ a ];
                    jj[ a1 ] = 2 * t1 + e1;
                    jj[ a2 ] = 2 * t2 + e2;
                    const double * fm = ff + ifl( m, a, jj[ 0 ], jj[ 1 ], jj[ 2 ] );
                    for( int c = 0; c < nw; ++ c )
                        acc[ c ] += fm[ c ] * ds;
                    norm += ds;
                }
                int ii[ 3 ];
                ii[ a ] = s ? n[ a ] : 0;
                ii[ a1 ] = d1 * h1 + t1;
                ii[ a2 ] = d2 * h2 + t2;
                double * o = fc + ifl( m, a, ii[ 0 ], ii[ 1 ], ii[ 2 ] );
                for( int c = 0; c < nw; ++ c )
                    o[ c ] = acc[ c ] / norm;
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* Static refinement, MHD: the reference's exchange holders, one per     */
/* (host block, neighbour) pair with faces, edges and vertices enrolled   */
/* (mhd/boundary/keeper.h:280-285 desired_mode).  Each holder pushes from */
/* its host into its guest: same-level copies (to_same), restrictions     */
/* (finer host, to_coarser) and prolongations (coarser host, to_finer) of */
/* the primitives, with the tangential face B of face holders; after the  */
/* flux sweeps the finer hosts' face holders average the fluxes and edge  */
/* E of a refined face into the coarser guest and edge holders the edge E */
/* of a refined edge, both writing the average back onto their own edges. */
/* Every holder's index space is restated as the reference launches it   */
/* (grids of resource_pack / resource_flux / resource_edge, the dispatch  */
/* of a CTA row, BND_TH threads per CTA and the last CTA's second pass),  */
/* and the holders run in the reference's order: hosts by level, then     */
/* logical position (x most significant; region.h lex_ord_t), each       */
/* host's neighbours by their direction flags in the same order.          */

enum { BND_TH = 64, ORD = 2, NGH = 2 };  /* [dynamics] bnd_thread_limit (its default); PLM order; ghosts */

typedef struct mh_holder
{
    int host, guest;
    int x[ 3 ], xr[ 3 ];         /* direction flags, seen from host and from guest */
    int mode, d_lvl, rhs, ax[ 3 ];
    int os[ 3 ], oc[ 3 ];        /* offset_s, offset_c: primitives            */
    int obs[ 3 ], obc[ 3 ], obr[ 3 ];   /* offset_bs / bc / br: face B        */
    int oes[ 3 ], oec[ 3 ];      /* offset_es / ec: edge E                    */
    int n1;                      /* the exchange grid's extent along axis[ 1 ] */
} mh_holder;

/* region.h:110-145 neighbor_t: flags of g (level lg) seen from h (level lh) */
static void nb_flags( const int * h, int lh, const int * g, int lg, int * x )
{
    const int d = lg - lh;
    for( int a = 0; a < 3; ++ a )
    {
        const int base = d >= 0 ? h[ a ] * ( 1 << d ) : ( h[ a ] >> -d );
        x[ a ] = g[ a ] - base;
        if( x[ a ] > 0 && d <= 0 )
            x[ a ] *= 2;
    }
}

static int leaf_at( const kro_mesh * m, int l, const int * r )
{   /* the block index of the leaf at (l, r), or -1 */
    const unsigned char * nd = m->tree.node[ l ];
    if( ! nd || nd[ kr_tree_idx( & m->tree, l, r ) ] != 1 )
        return -1;
    for( int b = 0; b < m->nblk; ++ b )
        if( m->tree.level[ b ] == l && ! memcmp( m->tree.reg + 3 * b, r, sizeof( int ) * 3 ) )
            return b;
    return -1;
}

static int cmp_host( const void * pa, const void * pb, void * pm )
{   /* region.h:17-34 lex_ord_t: level, then x[0], x[1], x[2] */
    const kro_mesh * m = ( const kro_mesh * ) pm;
    const int a = * ( const int * ) pa, b = * ( const int * ) pb;
    if( m->tree.level[ a ] != m->tree.level[ b ] )
        return m->tree.level[ a ] - m->tree.level[ b ];
    for( int k = 0; k < 3; ++ k )
        if( m->tree.reg[ 3 * a + k ] != m->tree.reg[ 3 * b + k ] )
            return m->tree.reg[ 3 * a + k ] - m->tree.reg[ 3 * b + k ];
    return 0;
}

static int cmp_flags( const void * pa, const void * pb )
{
    const mh_holder * a = ( const mh_holder * ) pa, * b = ( const mh_holder * ) pb;
    for( int k = 0; k < 3; ++ k )
        if( a->x[ k ] != b->x[ k ] )
            return a->x[ k ] - b->x[ k ];
    return 0;
}

/* boundary.cpp:33-60 comm_base_t::set_geo (axis, rhs) and
 * mhd/boundary/comm_functions.h:58-122 set_geo (offsets; one rank) */
static void holder_geo( const kro_mesh * m, mh_holder * h )
{
    const int * n = m->c.n;
    h->rhs = 0;
    for( int a = 0; a < 3; ++ a )
    {
        h->ax[ a ] = 0;
        const int out = h->x[ a ] < 0 || h->x[ a ] > 1;
        if( ( h->mode != 0 ) ^ out )
        {
            h->rhs = h->x[ a ] > 0;
            for( int k = 0; k < 3; ++ k )
                h->ax[ ( h->mode + k ) % 3 ] = ( a + k ) % 3;
            break;
        }
        else if( h->mode == 2 )
            h->ax[ a ] = a;
    }
    const int ax = h->ax[ 0 ];
    const int sh = h->d_lvl == 0 ? ORD : ( h->d_lvl > 0 ? ORD >> 1 : ORD << 1 );   /* shift(ord, -d_lvl) */
    for( int a = 0; a < 3; ++ a )
    {
        const int n2 = n[ a ] / 2;
        const int xp = h->x[ a ] > 0 ? h->x[ a ] : 0, rp = h->xr[ a ] > 0 ? h->xr[ a ] : 0;
        h->oes[ a ] = xp * n2;
        h->oec[ a ] = rp * n2;
        h->obs[ a ] = xp * n2;
        h->obc[ a ] = rp * n2;
        h->obr[ a ] = xp * n2;
        h->os[ a ] = xp * n2 - sh * ( h->x[ a ] > 0 );
        h->oc[ a ] = rp * n2 - ORD * ( h->x[ a ] > 0 );
    }
    h->obs[ ax ] -= h->x [ ax ] > 1;
    h->obr[ ax ] -= h->xr[ ax ] > 1;
    h->obc[ ax ] -= h->x [ ax ] > 1;
    if( h->mode == 1 )
    {
        const int a1 = h->ax[ 1 ];
        h->os[ a1 ] = h->x [ a1 ] * ( n[ a1 ] / 2 );
        h->oc[ a1 ] = h->xr[ a1 ] * ( n[ a1 ] / 2 );
    }
}

static void holder_extent( const kro_mesh * m, mh_holder * h );

/* tree.cpp:176-197 neighbors: for every level-(l+1) site around the block
 * (offsets -1..2 per axis, the block's own 2 x 2 x 2 excluded), wrapped on
 * periodic axes, the first leaf on the way down to level l - 1 */
static void build_holders( kro_mesh * m )
{
    int * order = ( int * ) malloc( sizeof( int ) * m->nblk );
    for( int b = 0; b < m->nblk; ++ b )
        order[ b ] = b;
    qsort_r( order, m->nblk, sizeof( int ), cmp_host, m );
    mh_holder * hs = ( mh_holder * ) calloc( ( size_t ) m->nblk * 64, sizeof( mh_holder ) );
    int nh = 0;
    for( int k = 0; k < m->nblk; ++ k )
    {
        const int b = order[ k ], l = m->tree.level[ b ];
        const int * r = m->tree.reg + 3 * b;
        const int first = nh;
        int di[ 3 ];
        for( di[ 0 ] = -1; di[ 0 ] < 3; ++ di[ 0 ] )
        for( di[ 1 ] = -1; di[ 1 ] < 3; ++ di[ 1 ] )
        for( di[ 2 ] = -1; di[ 2 ] < 3; ++ di[ 2 ] )
        {
            if( di[ 0 ] >= 0 && di[ 0 ] <= 1 && di[ 1 ] >= 0 && di[ 1 ] <= 1 && di[ 2 ] >= 0 && di[ 2 ] <= 1 )
                continue;
            int t[ 3 ], t0[ 3 ];
            for( int a = 0; a < 3; ++ a )
                t[ a ] = t0[ a ] = 2 * r[ a ] + di[ a ];
            if( ! kr_tree_regularize( & m->tree, l + 1, t ) )
                continue;
            for( int lt = l + 1; lt >= ( l > 0 ? l - 1 : 0 ); -- lt )
            {
                const int g = leaf_at( m, lt, t );
                if( g >= 0 )
                {
                    mh_holder h;
                    memset( & h, 0, sizeof( h ) );
                    h.host = b;
                    h.guest = g;
                    h.d_lvl = lt - l;
                    nb_flags( r, l, t0, lt, h.x );
                    nb_flags( t0, lt, r, l, h.xr );
                    int dup = 0;
                    for( int q = first; q < nh; ++ q )
                        dup |= ! memcmp( hs[ q ].x, h.x, sizeof( h.x ) );
                    if( ! dup )
                    {
                        h.mode = -1;
                        for( int a = 0; a < 3; ++ a )
                            h.mode += h.x[ a ] != 0 && h.x[ a ] != 1;
                        holder_geo( m, & h );
                        holder_extent( m, & h );
                        hs[ nh ++ ] = h;
                    }
                    break;
                }
                for( int a = 0; a < 3; ++ a )   /* region.h:61-69 coarsen */
                {
                    t [ a ] = ( t [ a ] > 0 ? t [ a ] : t [ a ] - 1 ) / 2;
                    t0[ a ] = ( t0[ a ] > 0 ? t0[ a ] : t0[ a ] - 1 ) / 2;
                }
            }
        }
        qsort( hs + first, nh - first, sizeof( mh_holder ), cmp_flags );
    }
    free( order );
    m->hold = hs;
    m->n_hold = nh;
}

static inline double * w_at( const kro_mesh * m, int b, const int * i )
{
    return m->w + ( size_t ) b * m->nw_cells * m->nw + iw( m, i[ 0 ], i[ 1 ], i[ 2 ] );
}
static inline double * bf_at( const kro_mesh * m, int step, int b, const int * i )
{
    return m->bf[ step ] + ( size_t ) b * m->nbf + ib( m, i[ 0 ], i[ 1 ], i[ 2 ] );
}
static inline double * ee_at( const kro_mesh * m, int b, const int * i )
{
    return m->ee + ( size_t ) b * m->nee + ie( m, i[ 0 ], i[ 1 ], i[ 2 ] );
}
static inline double * f_at( const kro_mesh * m, int a, int b, const int * i )
{
    return m->f[ a ] + ( size_t ) b * m->nf[ a ] + ifl( m, a, i[ 0 ], i[ 1 ], i[ 2 ] );
}

/* a launch of one holder: grid (nbx, nby), nth threads per CTA */
typedef struct { int nbx, nby, nth; } mh_grid;

static mh_grid grid_of( int n1, int nby )
{   /* boundary.cpp:10-16 resource_thbl, along axis[ 1 ] */
    mh_grid g;
    g.nth = n1 < BND_TH ? n1 : BND_TH;
    g.nbx = ( g.nth - 1 + n1 ) / g.nth;
    g.nby = nby;
    return g;
}

/* mhd/boundary/comm_functions.h:323-368 resource_pack */
static mh_grid grid_pack( const kro_mesh * m, const mh_holder * h )
{
    int nc[ 3 ] = { m->c.n[ 0 ], m->c.n[ 1 ], m->c.n[ 2 ] };
    const int a1 = h->ax[ 1 ], a2 = h->ax[ 2 ];
    if( h->d_lvl >= 0 )
    {
        if( h->mode > 0 ) nc[ a2 ] = ORD;
        if( h->mode > 1 ) nc[ a1 ] = ORD;
    }
    for( int a = 0; a < 3; ++ a )
        nc[ a ] /= 1 + ( h->d_lvl != 0 );
    if( h->d_lvl < 0 && h->mode > 0 )
    {
        nc[ a2 ] = NGH;
        if( h->mode > 1 ) nc[ a1 ] = NGH;
    }
    int nby = nc[ a2 ];
    if( h->mode == 0 )
        nby += h->d_lvl > 0 ? NGH / 2 : ( h->d_lvl < 0 ? h->xr[ a2 ] > 0 : 1 );
    return grid_of( nc[ a1 ], nby );
}

static void holder_extent( const kro_mesh * m, mh_holder * h )
{   /* grid_pack's n_cell along axis[ 1 ] */
    const int a1 = h->ax[ 1 ];
    int e = m->c.n[ a1 ];
    if( h->d_lvl >= 0 && h->mode > 1 ) e = ORD;
    e /= 1 + ( h->d_lvl != 0 );
    if( h->d_lvl < 0 && h->mode > 1 ) e = NGH;
    h->n1 = e;
}

/* comm_functions.h:160-174 dispatch: axis[0] 0, axis[1] along the CTA row */
static inline void dispatch( const mh_holder * h, const mh_grid * g, int bx, int by, int tx, int * i )
{
    i[ h->ax[ 0 ] ] = 0;
    i[ h->ax[ 1 ] ] = bx * g->nth + tx;
    i[ h->ax[ 2 ] ] = by;
}

/* hydro/boundary/comm_functions.h:306-327 to_same and
 * mhd/boundary/comm_functions.h:422-465 to_same (face B of face holders) */
static void mh_to_same( kro_mesh * m, const mh_holder * h, int step )
{
    const int * n = m->c.n, nw = m->nw;
    const int ax = h->ax[ 0 ], a1 = h->ax[ 1 ], a2 = h->ax[ 2 ];
    const mh_grid g = grid_pack( m, h );
    for( int by = 0; by < g.nby; ++ by )
    for( int bx = 0; bx < g.nbx; ++ bx )
    for( int tx = 0; tx < g.nth; ++ tx )
    {
        int i0[ 3 ], im[ 3 ], ibb[ 3 ];
        dispatch( h, & g, bx, by, tx, i0 );
        /* the CTA row covers exactly its extent along axis[ 1 ] while that is
         * at most BND_TH (the reference's threads past it would step out of
         * the arrays); the guard keeps larger extents in bounds */
        if( i0[ a2 ] < n[ a2 ] && i0[ a1 ] < h->n1 )
        {
            for( int a = 0; a < 3; ++ a )
            {
                im[ a ] = h->os[ a ] + i0[ a ];
                ibb[ a ] = h->oc[ a ] + i0[ a ];
            }
            for( int k = 0; k < ORD; ++ k )
            {
                im[ ax ] = k + h->os[ ax ];
                ibb[ ax ] = k + h->oc[ ax ];
                memcpy( w_at( m, h->guest, ibb ), w_at( m, h->host, im ), sizeof( double ) * nw );
            }
        }
        if( h->mode != 0 )
            continue;
        for( int a = 0; a < 3; ++ a )
        {
            im[ a ] = h->obs[ a ] + i0[ a ];
            ibb[ a ] = h->obc[ a ] + i0[ a ];
        }
        const int jmax = ( bx == g.nbx - 1 ) + 1;
        for( int j = 0; j < jmax && ibb[ a1 ] < n[ a1 ] + 1; ++ j )
        {
            double * bt = bf_at( m, step, h->guest, ibb );
            const double * bs = bf_at( m, step, h->host, im );
            bt[ a1 ] = bs[ a1 ];
            bt[ a2 ] = bs[ a2 ];
            ibb[ a1 ] += g.nth;
            im[ a1 ] += g.nth;
        }
    }
}

/* mhd/boundary/comm_functions.h:446-452 in_band_axis */
static inline int in_band( int i, int off )
{
    return off == 0 || ( i - off >= 0 && i - off < ORD );
}

/* mhd/boundary/comm_functions.h:467-691 to_finer: the primitives of the
 * coarser host's cells next to the face, limited-slope prolongation into
 * the finer guest's ghosts (face holders: the whole receiver slab with its
 * tangential ghost extensions; edge / vertex holders: ORD-wide bands), and
 * for face holders the tangential face B of the guest's first ghost layer
 * by Toth & Roe's divergence-preserving prolongation. */
static void mh_to_finer( kro_mesh * m, const mh_holder * h, int step )
{
    const int * n = m->c.n, nw = m->nw;
    const int ax = h->ax[ 0 ], a1 = h->ax[ 1 ], a2 = h->ax[ 2 ];
    const mh_grid g = grid_pack( m, h );
    for( int by = 0; by < g.nby; ++ by )
    for( int bx = 0; bx < g.nbx; ++ bx )
    for( int tx = 0; tx < g.nth; ++ tx )
    {
        int i0[ 3 ], im[ 3 ], ibb[ 3 ];
        dispatch( h, & g, bx, by, tx, i0 );
        for( int a = 0; a < 3; ++ a )
        {
            ibb[ a ] = h->oc[ a ] + 2 * i0[ a ];
            im[ a ] = h->os[ a ] + i0[ a ];
        }
        const int im_max = ( h->mode > 0 && h->oc[ a1 ] != 0 ) ? 1 : ( n[ a1 ] + ORD ) / 2;
        const int jmax = ( bx == g.nbx - 1 ) + 1;
        for( int j = 0; j < jmax && i0[ a1 ] < im_max; ++ j )
        {
            double qc[ 8 ], dq[ 3 ][ 8 ];
            for( int k = 0; k < ORD; ++ k )
            {
                im[ ax ] = h->os[ ax ] + k / 2;
                ibb[ ax ] = h->oc[ ax ] + k;
                if( ( k & 1 ) == 0 )
                {
                    memcpy( qc, w_at( m, h->host, im ), sizeof( double ) * nw );
                    for( int q = 0; q < 3; ++ q )
                    {
                        const int aq = h->ax[ q ];
                        ++ im[ aq ];
                        const double * qr = w_at( m, h->host, im );
                        im[ aq ] -= 2;
                        const double * ql = w_at( m, h->host, im );
                        ++ im[ aq ];
                        for( int c = 0; c < nw; ++ c )
                            dq[ aq ][ c ] = minmod( qr[ c ] - qc[ c ], qc[ c ] - ql[ c ] ) * 0.25f;
                    }
                }
                for( int d1 = 0; d1 < 2; ++ d1 )
                for( int d2 = 0; d2 < 2; ++ d2 )
                {
                    ibb[ a1 ] += d1;
                    ibb[ a2 ] += d2;
                    if( h->mode == 0 || ( in_band( ibb[ a1 ], h->oc[ a1 ] ) && in_band( ibb[ a2 ], h->oc[ a2 ] ) ) )
                    {
                        double * q = w_at( m, h->guest, ibb );
                        for( int c = 0; c < nw; ++ c )
                            q[ c ] = qc[ c ] + dq[ ax ][ c ] * ( 2 * ( k & 1 ) - 1 )
                                   + dq[ a1 ][ c ] * ( 2 * d1 - 1 )
                                   + dq[ a2 ][ c ] * ( 2 * d2 - 1 );
                    }
                    ibb[ a1 ] -= d1;
                    ibb[ a2 ] -= d2;
                }
            }
            ibb[ a1 ] += 2 * g.nth;
            im[ a1 ] += g.nth;
            i0[ a1 ] += g.nth;
        }
        if( h->mode != 0 )
            continue;
        /* face B (comm_functions.h:588-690) */
        dispatch( h, & g, bx, by, tx, i0 );
        for( int a = 0; a < 3; ++ a )
        {
            ibb[ a ] = 2 * i0[ a ] + h->obc[ a ];
            im[ a ] = i0[ a ] + h->obr[ a ];
        }
        if( ibb[ a2 ] > n[ a2 ] - 2 || ibb[ a1 ] > n[ a1 ] - 2 )
            continue;
        ibb[ ax ] = h->rhs ? -1 : n[ ax ];
        im[ ax ] = h->rhs ? n[ ax ] - 1 : 0;
        double bb[ 3 ][ 3 ][ 2 ][ 2 ], db1[ 2 ], db2[ 3 ], db3[ 3 ];
        for( int a = 0; a < 3; ++ a )
        {
            const int ap[ 2 ] = { mod3( a + 1 ), mod3( a + 2 ) };
            for( int d = 0; d < 2; ++ d )
            {
                im[ a ] += d;
                const double bc = bf_at( m, step, h->host, im )[ a ];
                for( int q = 0; q < 2; ++ q )
                {
                    im[ ap[ q ] ] -= 1;
                    const double bl = bf_at( m, step, h->host, im )[ a ];
                    im[ ap[ q ] ] += 2;
                    const double br = bf_at( m, step, h->host, im )[ a ];
                    im[ ap[ q ] ] -= 1;
                    db1[ q ] = minmod( br - bc, bc - bl ) / 4;
                }
                bb[ a ][ 2 * d ][ 0 ][ 0 ] = bc - db1[ 0 ] - db1[ 1 ];
                bb[ a ][ 2 * d ][ 0 ][ 1 ] = bc - db1[ 0 ] + db1[ 1 ];
                bb[ a ][ 2 * d ][ 1 ][ 0 ] = bc + db1[ 0 ] - db1[ 1 ];
                bb[ a ][ 2 * d ][ 1 ][ 1 ] = bc + db1[ 0 ] + db1[ 1 ];
                im[ a ] -= d;
            }
        }
        for( int a = 0; a < 3; ++ a )
        {
            const int b1 = mod3( a + 1 ), b2 = mod3( a + 2 );
            db2[ a ] = 0;
            for( int l = 0; l < 2; ++ l )
                for( int q = 0; q < 2; ++ q )   /* the reference divides only the second term by 8 */
                    db2[ a ] += ( 2 * q - 1 ) * ( bb[ b1 ][ 2 ][ l ][ q ] - bb[ b1 ][ 0 ][ l ][ q ] )
                              + ( 2 * l - 1 ) * ( bb[ b2 ][ 2 ][ l ][ q ] - bb[ b2 ][ 0 ][ l ][ q ] ) / 8;
            db3[ a ] = 0;
            for( int k = 0; k < 2; ++ k )
                for( int l = 0; l < 2; ++ l )
                    for( int q = 0; q < 2; ++ q )
                        db3[ a ] += ( 2 * k - 1 ) / 16.f * ( 2 * l - 1 ) * ( 2 * q - 1 ) * bb[ a ][ 2 * k ][ l ][ q ];
        }
        for( int a = 0; a < 3; ++ a )
        {
            const int b1 = mod3( a + 1 ), b2 = mod3( a + 2 );
            for( int l = 0; l < 2; ++ l )
                for( int q = 0; q < 2; ++ q )
                    bb[ a ][ 1 ][ l ][ q ] = db2[ a ] + ( bb[ a ][ 2 ][ l ][ q ] + bb[ a ][ 0 ][ l ][ q ] ) / 2
                                           + db3[ b1 ] * ( 2 * l - 1 ) + db3[ b2 ] * ( 2 * q - 1 );
        }
        const int l_max = ( ibb[ a1 ] == n[ a1 ] - 2 ) + 2;
        const int q_max = ( ibb[ a2 ] == n[ a2 ] - 2 ) + 2;
        for( int l = 0; l < l_max; ++ l )
            for( int q = 0; q < q_max; ++ q )
            {
                ibb[ a1 ] += l;
                ibb[ a2 ] += q;
                double * bt = bf_at( m, step, h->guest, ibb );
                if( q < 2 )
                    bt[ a1 ] = bb[ a1 ][ l ][ q ][ h->rhs ];
                if( l < 2 )
                    bt[ a2 ] = bb[ a2 ][ q ][ h->rhs ][ l ];
                ibb[ a1 ] -= l;
                ibb[ a2 ] -= q;
            }
    }
}

/* hydro/boundary/comm_functions.h:329-380 to_coarser (volume averages of
 * the finer host's cells) inside mhd/boundary/comm_functions.h:693-780
 * to_coarser, which limits edge / vertex holders to the NGH-wide band and
 * adds, for face holders, the area average of the tangential face B over
 * the two finer cell rows next to the face. */
static void mh_to_coarser( kro_mesh * m, const mh_holder * h, int step )
{
    const int * n = m->c.n, nw = m->nw;
    const int ax = h->ax[ 0 ], a1 = h->ax[ 1 ], a2 = h->ax[ 2 ];
    const mh_grid g = grid_pack( m, h );
    const double dv = m->vol0[ h->host ];
    for( int by = 0; by < g.nby; ++ by )
    for( int bx = 0; bx < g.nbx; ++ bx )
    for( int tx = 0; tx < g.nth; ++ tx )
    {
        int i0[ 3 ], im[ 3 ], ibb[ 3 ];
        dispatch( h, & g, bx, by, tx, i0 );
        const int lim2 = h->mode > 0 ? NGH : n[ a2 ] / 2;
        const int lim1 = h->mode > 1 ? NGH : n[ a1 ] / 2;
        if( i0[ a2 ] < lim2 && i0[ a1 ] < lim1 )
        {
            for( int a = 0; a < 3; ++ a )
            {
                im[ a ] = h->os[ a ] + 2 * i0[ a ];
                ibb[ a ] = i0[ a ] + h->oc[ a ];
            }
            double p[ 8 ], norm = 0;
            for( int k = 0; k < 2 * ORD; ++ k )
            {
                im[ ax ] = k + h->os[ ax ];
                if( ( k & 1 ) == 0 )
                {
                    ibb[ ax ] = k / 2 + h->oc[ ax ];
                    norm = 0;
                    for( int c = 0; c < nw; ++ c )
                        p[ c ] = 0;
                }
                const int s1 = im[ a1 ], s2 = im[ a2 ];
                for( int d1 = 0; d1 < 2; ++ d1 )
                for( int d2 = 0; d2 < 2; ++ d2 )
                {
                    im[ a1 ] = s1 + d1;
                    im[ a2 ] = s2 + d2;
                    const double * q = w_at( m, h->host, im );
                    for( int c = 0; c < nw; ++ c )
                        p[ c ] += q[ c ] * dv;
                    norm += dv;
                }
                im[ a1 ] = s1;
                im[ a2 ] = s2;
                if( k & 1 )
                {
                    double * o = w_at( m, h->guest, ibb );
                    for( int c = 0; c < nw; ++ c )
                        o[ c ] = p[ c ] / norm;
                }
            }
        }
        if( h->mode != 0 )
            continue;
        for( int a = 0; a < 3; ++ a )
        {
            im[ a ] = 2 * i0[ a ] + h->obs[ a ];
            ibb[ a ] = i0[ a ] + h->obc[ a ];
        }
        if( h->obs[ ax ] > 0 )
            -- im[ ax ];
        const int jmax = ( bx == g.nbx - 1 ) + 1;
        const int ib_max = n[ a1 ] / 2 + ( h->obc[ a1 ] > 1 );
        for( int j = 0; j < jmax && i0[ a1 ] < ib_max; ++ j )
        {
            im[ a1 ] = 2 * i0[ a1 ] + h->obs[ a1 ];
            double * bt = bf_at( m, step, h->guest, ibb );
            for( int l = 0; l < 2; ++ l )
            {
                const int a = h->ax[ 1 + l ], ap = h->ax[ 2 - l ];
                if( im[ ap ] >= n[ ap ] )
                    continue;
                double bsum = 0, s = 0;
                const double ds = m->sfc0[ h->host * 3 + a ];
                for( int k = 0; k < 2; ++ k )
                {
                    bsum += ds * bf_at( m, step, h->host, im )[ a ];
                    s += ds;
                    ++ im[ ap ];
                    bsum += ds * bf_at( m, step, h->host, im )[ a ];
                    s += ds;
                    -- im[ ap ];
                    ++ im[ ax ];
                }
                im[ ax ] -= 2;
                bt[ a ] = s > 0 ? bsum / s : 0;
            }
            i0[ a1 ] += g.nth;
            ibb[ a1 ] += g.nth;
        }
    }
}

/* act_flx, a finer host's face holder (mhd/boundary/comm_functions.h:818-884
 * flux_to_buf over hydro/boundary/comm_functions.h:469-505): the coarser
 * guest's flux on the refined face is the area average of the 4 finer
 * fluxes; its tangential edge E the length average of the 2 finer edges,
 * written back onto both. */
static void mh_flux_to_buf( kro_mesh * m, const mh_holder * h )
{
    const int * n = m->c.n, nw = m->nw;
    const int ax = h->ax[ 0 ], a1 = h->ax[ 1 ], a2 = h->ax[ 2 ];
    /* resource_flux (comm_functions.h:384-399) */
    const mh_grid g = grid_of( n[ a1 ] / 2, n[ a2 ] / 2 + ( h->xr[ a2 ] > 0 ) );
    const double ds = m->sfc0[ h->host * 3 + ax ];
    for( int by = 0; by < g.nby; ++ by )
    for( int bx = 0; bx < g.nbx; ++ bx )
    for( int tx = 0; tx < g.nth; ++ tx )
    {
        int i0[ 3 ], im[ 3 ], ibb[ 3 ];
        dispatch( h, & g, bx, by, tx, i0 );
        if( i0[ a2 ] < n[ a2 ] / 2 && i0[ a1 ] < n[ a1 ] / 2 )
        {
            for( int a = 0; a < 3; ++ a )
                ibb[ a ] = i0[ a ] + h->oc[ a ];
            ibb[ ax ] = h->rhs ? 0 : n[ ax ];
            im[ ax ] = h->rhs ? n[ ax ] : 0;
            double * fb = f_at( m, ax, h->guest, ibb );
            for( int c = 0; c < nw; ++ c )
                fb[ c ] = 0;
            double norm = 0;
            for( int d1 = 0; d1 < 2; ++ d1 )
            for( int d2 = 0; d2 < 2; ++ d2 )
            {
                im[ a1 ] = 2 * i0[ a1 ] + d1;
                im[ a2 ] = 2 * i0[ a2 ] + d2;
                const double * fm = f_at( m, ax, h->host, im );
                for( int c = 0; c < nw; ++ c )
                    fb[ c ] += fm[ c ] * ds;
                norm += ds;
            }
            for( int c = 0; c < nw; ++ c )
                fb[ c ] /= norm;
        }
        for( int a = 0; a < 3; ++ a )
        {
            im[ a ] = 2 * i0[ a ] + h->oes[ a ];
            ibb[ a ] = i0[ a ] + h->oec[ a ];
        }
        const int jmax = ( bx == g.nbx - 1 ) + 1;
        const int ib_max = n[ a1 ] / 2 + ( h->oec[ a1 ] > 1 );
        for( int j = 0; j < jmax && i0[ a1 ] < ib_max; ++ j )
        {
            im[ a1 ] = 2 * i0[ a1 ] + h->oes[ a1 ];
            double * eb = ee_at( m, h->guest, ibb );
            double * em = ee_at( m, h->host, im );
            for( int q = 0; q < 3; ++ q )
            {
                const int am = h->ax[ mod3( ax + q ) ];
                if( am == ax )
                    continue;
                const double dl_l = m->dx0[ h->host * 3 + am ];
                const double e_l = em[ am ] * dl_l;
                ++ im[ am ];
                double * ep = ee_at( m, h->host, im );
                const double dl_r = m->dx0[ h->host * 3 + am ];
                const double e_r = ep[ am ] * dl_r;
                -- im[ am ];
                eb[ am ] = ( e_l + e_r ) / ( dl_l + dl_r );
                em[ am ] = eb[ am ];
                ep[ am ] = eb[ am ];
            }
            ibb[ a1 ] += g.nth;
            i0[ a1 ] += g.nth;
        }
    }
}

/* act_flx, a finer host's edge holder (mhd/boundary/comm_functions.h:918-954
 * edge_efield): the coarser guest's E along the refined edge is the length
 * average of the 2 finer edges, written back onto both. */
static void mh_edge_efield( kro_mesh * m, const mh_holder * h )
{
    const int a1 = h->ax[ 1 ];
    const int ne = m->c.n[ a1 ] / 2;                  /* resource_edge */
    const mh_grid g = grid_of( ne, 1 );
    for( int bx = 0; bx < g.nbx; ++ bx )
    for( int tx = 0; tx < g.nth; ++ tx )
    {
        int i0[ 3 ], im[ 3 ], ibb[ 3 ];
        dispatch( h, & g, bx, 0, tx, i0 );
        if( i0[ a1 ] >= ne )
            continue;
        for( int a = 0; a < 3; ++ a )
        {
            im[ a ] = h->oes[ a ] + 2 * i0[ a ];
            ibb[ a ] = h->oec[ a ] + i0[ a ];
        }
        double * el = ee_at( m, h->host, im );
        const double dl_l = m->dx0[ h->host * 3 + a1 ];
        double et = el[ a1 ] * dl_l;
        ++ im[ a1 ];
        double * er = ee_at( m, h->host, im );
        const double dl_r = m->dx0[ h->host * 3 + a1 ];
        et += er[ a1 ] * dl_r;
        const double ea = et / ( dl_l + dl_r );
        ee_at( m, h->guest, ibb )[ a1 ] = ea;
        el[ a1 ] = ea;
        er[ a1 ] = ea;
    }
}

/* keeper.cpp:148-160 act_bnd with mhd/boundary/keeper.h:304-326: the
 * restrictions, the same-level copies, the prolongations (which read the
 * coarser hosts' ghosts filled before), the restrictions again (their
 * second pass, keeper.cpp:121-127 q_plgt.unpk), each in holder order. */
static void bc_block_mhd( kro_mesh * m, int b, void * aux );

static void mh_act_bnd( kro_mesh * m, int step )
{
    ghost_arg pass1 = { step, 0 }, pass2 = { step, 1 };
    for( int k = 0; k < m->n_hold; ++ k )
        if( m->hold[ k ].d_lvl < 0 ) mh_to_coarser( m, m->hold + k, step );
    par_blocks( m, bc_block_mhd, & pass1 );      /* keeper.cpp:148-157: the sides, then the copies */
    for( int k = 0; k < m->n_hold; ++ k )
        if( m->hold[ k ].d_lvl == 0 ) mh_to_same( m, m->hold + k, step );
    for( int k = 0; k < m->n_hold; ++ k )
        if( m->hold[ k ].d_lvl > 0 ) mh_to_finer( m, m->hold + k, step );
    for( int k = 0; k < m->n_hold; ++ k )
        if( m->hold[ k ].d_lvl < 0 ) mh_to_coarser( m, m->hold + k, step );
    par_blocks( m, bc_block_mhd, & pass2 );      /* mhd/boundary/keeper.h:304-309: primitives again */
}

/* keeper.cpp:162-166 act_flx: the finer hosts' face and edge holders */
static void mh_act_flx( kro_mesh * m )
{
    for( int k = 0; k < m->n_hold; ++ k )
    {
        const mh_holder * h = m->hold + k;
        if( h->d_lvl >= 0 )
            continue;
        if( h->mode == 0 )
            mh_flux_to_buf( m, h );
        else if( h->mode == 1 )
            mh_edge_efield( m, h );
    }
}

/* ------------------------------------------------------------------ */
/* MHD physical boundaries (mhd/boundary/phys.h:118-250 operator(),      */
/* phys_functors.h:9-132 free / fixed / outflow / reflect).  Per side on  */
/* the domain edge, every transverse row of the ghost shell (ghost rows   */
/* included) takes its source row clamped into the interior only along    */
/* transverse axes that end at a physical side there; the n_gh + 1 cells  */
/* (primitives, cell-centred B) and faces (normal B on the face lattice,  */
/* tangential B on the cell lattice) next to the boundary go through the  */
/* functor into the ghost slots.  Sides in order x-, x+, y-, y+, z-, z+.  */
/* The reference runs this once before and once after the same-level     */
/* exchange (keeper_t::act_bnd, face B only in the first pass); this      */
/* restatement runs it once after the exchange: the first pass's face-B   */
/* values from not-yet-exchanged rows land only in ghost-shell corner     */
/* slots, which no later stencil reads.                                   */

static void bc_block_mhd( kro_mesh * m, int b, void * aux )
{
    const int step = ( ( ghost_arg * ) aux )->step;
    const int field = ! ( ( ghost_arg * ) aux )->no_field;  /* phys.h:199-249: step >= 0 */
    const int * n = m->c.n;
    const int nw = m->nw;
    const int * reg = blk_reg( m, b );
    double * w = m->w + ( size_t ) b * m->nw_cells * nw;
    double * bf = m->bf[ step ] + ( size_t ) b * m->nbf;
    int phy[ 3 ][ 2 ];                       /* geo.phybnd_flag */
    for( int a = 0; a < 3; ++ a )
    {
        phy[ a ][ 0 ] = m->c.bc[ 2 * a ] != KRO_PER && reg[ a ] == 0;
        phy[ a ][ 1 ] = m->c.bc[ 2 * a + 1 ] != KRO_PER && reg[ a ] == blk_lim( m, b, a ) - 1;
    }
    for( int side = 0; side < 6; ++ side )
    {
        const int axis = side / 2, right = side & 1;
        const int kind = m->c.bc[ side ];
        if( kind == KRO_PER || ! phy[ axis ][ right ] )
            continue;
        const int a1 = mod3( axis + 1 ), a2 = mod3( axis + 2 );
        const int i_mom = MOM + axis;
        const int nn = n[ axis ];
        for( int t2 = -2; t2 < n[ a2 ] + 2; ++ t2 )
        for( int t1 = -2; t1 < n[ a1 ] + 2; ++ t1 )
        {
            int i_tgt[ 3 ], i_src[ 3 ], i_sfc[ 3 ];
            i_tgt[ a1 ] = t1;
            i_tgt[ a2 ] = t2;
            for( int h = 0; h < 2; ++ h )
            {
                const int a = h ? a2 : a1;
                int r = i_tgt[ a ], f = i_tgt[ a ];
                if( phy[ a ][ 0 ] ) { r = r < 0 ? 0 : r; f = f < 0 ? 0 : f; }
                if( phy[ a ][ 1 ] ) { r = r > n[ a ] - 1 ? n[ a ] - 1 : r; f = f > n[ a ] ? n[ a ] : f; }
                i_src[ a ] = r;
                i_sfc[ a ] = f;
            }
            double hyd[ 5 ][ 8 ], bc[ 5 ][ 3 ], bfb[ 5 ][ 3 ];   /* index i + 2, i = -2..2 */
            for( int i = 0; i <= 2; ++ i )
            {
                i_src[ axis ] = right ? nn - i - 1 : i;
                i_sfc[ axis ] = right ? nn - i : i;
                const double * hs = w + iw( m, i_src[ 0 ], i_src[ 1 ], i_src[ 2 ] );
                for( int k = 0; k < 8; ++ k )
                    hyd[ 2 + i ][ k ] = hs[ k ];
                for( int q = 0; q < 3; ++ q )
                {
                    bc[ 2 + i ][ q ] = hs[ BCC + q ];
                    bfb[ 2 + i ][ q ] = q == axis ? bf[ ib( m, i_sfc[ 0 ], i_sfc[ 1 ], i_sfc[ 2 ] ) + q ]
                                                  : bf[ ib( m, i_src[ 0 ], i_src[ 1 ], i_src[ 2 ] ) + q ];
                }
            }
            /* hydro part of the functor (n_int = 8: the B_cc slots ride along and
             * are replaced by the field part below) */
            if( kind == KRO_OUT && hyd[ 2 ][ i_mom ] * ( right ? -1 : 1 ) > 0 )
                hyd[ 2 ][ i_mom ] = 0;
            for( int i = -2; i < 0; ++ i )
                for( int k = 0; k < 8; ++ k )
                {
                    if( kind == KRO_REF )
                        hyd[ 2 + i ][ k ] = hyd[ 2 - i - 1 ][ k ] * ( k == i_mom ? -1 : 1 );
                    else if( kind == KRO_FIXD )
                        hyd[ 2 + i ][ k ] = k < 5 ? m->c.w_fix[ k ] : m->c.b_fix[ k - 5 ];
                    else
                        hyd[ 2 + i ][ k ] = hyd[ 2 ][ k ];
                }
            /* field part */
            for( int i = -2; i < 0; ++ i )
                for( int q = 0; q < 3; ++ q )
                {
                    if( kind == KRO_REF )
                    {   /* faces mirror at -i, cells at -i-1; tangential components
                         * flip sign (phys_functors.h:120-131) */
                        const double sg = q != axis ? -1 : 1;
                        bfb[ 2 + i ][ q ] = sg * bfb[ 2 - i ][ q ];
                        bc [ 2 + i ][ q ] = sg * bc [ 2 - i - 1 ][ q ];
                    }
                    else if( kind == KRO_FIXD )
                        bfb[ 2 + i ][ q ] = bc[ 2 + i ][ q ] = m->c.b_fix[ q ];
                    else
                    {
                        bc [ 2 + i ][ q ] = bc [ 2 ][ q ];
                        bfb[ 2 + i ][ q ] = bfb[ 2 ][ q ];
                    }
                }
            for( int i = -2; i < 0; ++ i )
            {
                i_tgt[ axis ] = right ? nn - i - 1 : i;
                int i_fbc[ 3 ] = { i_tgt[ 0 ], i_tgt[ 1 ], i_tgt[ 2 ] };
                i_fbc[ axis ] = right ? nn - i : i;
                double * ht = w + iw( m, i_tgt[ 0 ], i_tgt[ 1 ], i_tgt[ 2 ] );
                for( int k = 0; k < 8; ++ k )
                    ht[ k ] = hyd[ 2 + i ][ k ];
                for( int q = 0; q < 3; ++ q )
                {
                    ht[ BCC + q ] = bc[ 2 + i ][ q ];
                    if( ! field )
                        continue;
                    if( q == axis )
                        bf[ ib( m, i_fbc[ 0 ], i_fbc[ 1 ], i_fbc[ 2 ] ) + q ] = bfb[ 2 + i ][ q ];
                    else
                        bf[ ib( m, i_tgt[ 0 ], i_tgt[ 1 ], i_tgt[ 2 ] ) + q ] = bfb[ 2 + i ][ q ];
                }
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* PLM (hydro/reconstruct/plm.h:116-153, uniform mesh, FP64: norm = 1)  */

static inline void plm_face( double q_ll, double q_l, double q_r, double q_rr,
                             double * ql, double * qr )
{
    const double norm = 1;
    const double dql = ( q_l  - q_ll );
    const double dqc = ( q_r  - q_l  );
    const double dqr = ( q_rr - q_r  );
    const double dqr2  = norm * dqr * dqr;
    const double dql2  = norm * dql * dql;
    const double dqc2  = norm * dqc * dqc;
    const double dq2_l = norm * dql * dqc;
    const double dq2_r = norm * dqr * dqc;
    const double ql_coef = dq2_l <= 0 ? 0 :  dq2_l / ( dql2 + dqc2 + dq2_l * 2 );
    const double qr_coef = dq2_r <= 0 ? 0 : -dq2_r / ( dqr2 + dqc2 + dq2_r * 2 );
    * ql = q_l + ( dq2_l <= 0 ? 0 : ql_coef * ( dql + dqc ) );
    * qr = q_r + ( dq2_r <= 0 ? 0 : qr_coef * ( dqc + dqr ) );
}

void kro_plm( const double * q4, double * ql, double * qr )
{
    plm_face( q4[ 0 ], q4[ 1 ], q4[ 2 ], q4[ 3 ], ql, qr );
}

/* ------------------------------------------------------------------ */
/* HLLC (hydro/riemann/hllc.h:239-250 f_lr_hyd, 262-379 eval), on the   */
/* rotated states; wli / wri are overwritten (the reference reuses them */
/* as flux scratch).                                                    */

static inline void f_lr_hyd( double * f, const double * w, double v, double e )
{
    const double rho = w[ RHO ];
    const double pre = w[ ENE ];
    f[ RHO ] = rho * v;
    f[ ENE ] = pre * w[ MOM ] + e * v;
    for( int a = MOM; a < MOM + 3; ++ a )
        f[ a ] = rho * w[ a ] * v;
    f[ MOM ] += pre;
}

static void hllc_eval( double * flx, double * wli, double * wri, double gamma )
{
    double * fl = wli, * fr = wri, * wroe = flx;
    double el, er, cl, cr;
    const double gm1i_l = et_cs( gamma, & el, & cl, wli );
    const double gm1i_r = et_cs( gamma, & er, & cr, wri );

    const double sqrtdl  = sqrt( wli[ RHO ] );
    const double sqrtdr  = sqrt( wri[ RHO ] );
    const double isdlpdr = ( double ) 1 / ( sqrtdl + sqrtdr );
    wroe[ RHO ] = sqrtdl * sqrtdr;
    for( int n = MOM; n < MOM + 3; ++ n )
        wroe[ n ] = ( sqrtdl * wli[ n ] + sqrtdr * wri[ n ] ) * isdlpdr;
    const double hroe = isdlpdr *
        ( ( el + wli[ ENE ] ) / sqrtdl + ( er + wri[ ENE ] ) / sqrtdr );
    const double gam1_roe = ( double ) 1 /
        ( isdlpdr * ( sqrtdl * gm1i_l + sqrtdr * gm1i_r ) );

    const double v2roe = wroe[ MOM ] * wroe[ MOM ] + wroe[ MOM + 1 ] * wroe[ MOM + 1 ]
                       + wroe[ MOM + 2 ] * wroe[ MOM + 2 ];
    const double q = hroe - 0.5f * v2roe;
    const double a = ( q <= 0 ) ? 0 : sqrt( gam1_roe * q );

    const double al = dmin( wroe[ MOM ] - a, wli[ MOM ] - cl );
    const double ar = dmax( wroe[ MOM ] + a, wri[ MOM ] + cr );
    const double bp = ar > 0 ? ar : 0;
    const double bm = al < 0 ? al : 0;

    const double vxl = wli[ MOM ] - al;
    const double vxr = wri[ MOM ] - ar;
    const double tl  = wli[ ENE ] + vxl * wli[ RHO ] * wli[ MOM ];
    const double tr  = wri[ ENE ] + vxr * wri[ RHO ] * wri[ MOM ];
    const double ml  =  wli[ RHO ] * vxl;
    const double mr  = -wri[ RHO ] * vxr;

    double cp, am;
    const double f_max = FLT_MAX / 1e1f;     /* float constants, as hllc.h:326-327 */
    const double f_min = FLT_MIN * 1e1f;
    if( fabs( ml + mr ) < f_min )
    {
        cp = 0;
        am = 0;
    }
    else if( ( tr != 0 && fabs( ml ) > f_max / fabs( tr ) ) ||
             ( tl != 0 && fabs( mr ) > f_max / fabs( tl ) ) )
    {
        const double mli = sgn( ml ) / dmax( fabs( ml ), f_min );
        const double mri = sgn( mr ) / dmax( fabs( mr ), f_min );
        am = ( tl - tr ) / ( ml + mr );
        cp = dmax( ( mri * tr + mli * tl ) / ( mli + mri ), ( double ) 0 );
    }
    else
    {
        am = ( tl - tr ) / ( ml + mr );
        cp = dmax( ( ml * tr + mr * tl ) / ( ml + mr ), ( double ) 0 );
    }

    const double d_am_bm = dmax( fabs( am - bm ), f_min ) * ( am > bm ? 1 : -1 );
    const double d_am_bp = dmax( fabs( am - bp ), f_min ) * ( am > bp ? 1 : -1 );
    const double sl = ( am >= 0 ? am / d_am_bm : 0 );
    const double sr = ( am <  0 ? am / d_am_bp : 0 );
    const double sm = ( am >  0 ? -bm / d_am_bm : -bp / d_am_bp );

    f_lr_hyd( fl, wli, wli[ MOM ] - bm, el );
    f_lr_hyd( fr, wri, wri[ MOM ] - bp, er );
    for( int n = RHO; n < MOM + 3; ++ n )
        flx[ n ] = sl * fl[ n ] + sr * fr[ n ];
    flx[ MOM ] += sm * cp;
    flx[ ENE ] += sm * cp * am;
}

/* hydro/riemann/hllc.h:218-229 calc: rotate, solve, rotate back */
static void hllc_calc( double * flx, double * ql, double * qr, int axis, double gamma )
{
    idx_swap( ql + MOM, axis );
    idx_swap( qr + MOM, axis );
    hllc_eval( flx, ql, qr, gamma );
    idx_swap( flx + MOM, 3 - axis );
}

void kro_hllc( const double * ql_in, const double * qr_in, int axis, double gamma, double * flx )
{
    double ql[ 5 ], qr[ 5 ];
    memcpy( ql, ql_in, sizeof ql );
    memcpy( qr, qr_in, sizeof qr );
    hllc_calc( flx, ql, qr, axis, gamma );
}

/* ------------------------------------------------------------------ */
/* HLLD (mhd/riemann/hlld.h:49-69 f_flux, 81-298 eval)                 */

static inline void hlld_f_flux( double * flux, const double * u, const double * w,
                                double p_tot, double b_x )
{
    const double bx_2 = b_x * b_x;
    flux[ RHO ] = u[ MOM ];
    flux[ ENE ] = w[ MOM ] * ( p_tot + u[ ENE ] - bx_2 ) - b_x
                * ( w[ MOM + 1 ] * u[ BCC + 1 ] + w[ MOM + 2 ] * u[ BCC + 2 ] );
    flux[ MOM ]     = p_tot - bx_2 + u[ MOM ] * w[ MOM ];
    flux[ MOM + 1 ] = -b_x * u[ BCC + 1 ] + u[ MOM + 1 ] * w[ MOM ];
    flux[ MOM + 2 ] = -b_x * u[ BCC + 2 ] + u[ MOM + 2 ] * w[ MOM ];
    flux[ BCC + 1 ] = -b_x * w[ MOM + 1 ] + u[ BCC + 1 ] * w[ MOM ];
    flux[ BCC + 2 ] = -b_x * w[ MOM + 2 ] + u[ BCC + 2 ] * w[ MOM ];
}

static inline double hlld_cons( double * u, const double * w, double bx_2, double b_x,
                                double gamma, double * gam1 )
{
    double p_m = bx_2 / 2, cs;
    for( int a = 1; a <= 2; ++ a )
    {
        const int n = BCC + a;
        p_m += w[ n ] * w[ n ] / 2;
        u[ n ] = w[ n ];
    }
    * gam1 = 1 / et_cs( gamma, & u[ ENE ], & cs, w );
    for( int n = MOM; n < MOM + 3; ++ n )
        u[ n ] = w[ RHO ] * w[ n ];
    u[ RHO ] = w[ RHO ];
    u[ ENE ] += p_m;
    u[ BCC ] = b_x;
    return p_m;
}

typedef struct { double b_x, bx_2, ptot_s, spd0; } hlld_ctx;

static double hlld_star( const hlld_ctx * h, double * u_star, const double * u,
                         const double * w, double rhos, double sd, double sdm,
                         double p_tot, double f_tiny )
{
    const double b_x = h->b_x, bx_2 = h->bx_2;
    u_star[ RHO ] = rhos;
    u_star[ MOM ] = rhos * h->spd0;
    u_star[ BCC ] = b_x;
    const double denom = u[ RHO ] * sd * sdm - bx_2;
    if( uabs( denom ) < f_tiny * h->ptot_s )
        for( int a = 1; a <= 2; ++ a )
        {
            u_star[ MOM + a ] = rhos * w[ MOM + a ];
            u_star[ BCC + a ] = u[ BCC + a ];
        }
    else
    {
        const double tmp_v = b_x * ( sd - sdm ) / denom;
        const double tmp_b = ( u[ RHO ] * sd * sd - bx_2 ) / denom;
        for( int a = 1; a <= 2; ++ a )
        {
            u_star[ MOM + a ] = rhos * ( w[ MOM + a ] - u[ BCC + a ] * tmp_v );
            u_star[ BCC + a ] = u[ BCC + a ] * tmp_b;
        }
    }
    double u_dot_b = 0, w_dot_b = 0;
    for( int a = 0; a < 3; ++ a )
    {
        u_dot_b += u_star[ MOM + a ] * u_star[ BCC + a ];
        w_dot_b += w[ MOM + a ] * u[ BCC + a ];
    }
    u_dot_b /= rhos;
    u_star[ ENE ] = b_x * ( w_dot_b - u_dot_b )
        - p_tot * w[ MOM ] + sd * u[ ENE ]
        + h->ptot_s * h->spd0;
    u_star[ ENE ] /= sdm;
    return u_dot_b;
}

static void hlld_eval( double * flx, const double * wli, const double * wri, double gamma )
{
    flx[ BCC ] = 0;
    double spd_m2, spd_m1, spd0, spd_p1, spd_p2;
    double u_l[ 8 ], u_r[ 8 ];
    const double b_x  = wli[ BCC ];
    const double bx_2 = b_x * b_x;
    double gam1_l, gam1_r;
    const double pm_l = hlld_cons( u_l, wli, bx_2, b_x, gamma, & gam1_l );
    const double pm_r = hlld_cons( u_r, wri, bx_2, b_x, gamma, & gam1_r );
    const double ptot_l = wli[ ENE ] + pm_l;
    const double ptot_r = wri[ ENE ] + pm_r;

    double b2_eff_l[ 3 ] = { b_x, wli[ BCC + 1 ], wli[ BCC + 2 ] };
    double b2_eff_r[ 3 ] = { b_x, wri[ BCC + 1 ], wri[ BCC + 2 ] };
    for( int a = 0; a < 3; ++ a )
    {
        b2_eff_l[ a ] *= b2_eff_l[ a ];
        b2_eff_r[ a ] *= b2_eff_r[ a ];
    }
    const double cfm_l = c_fms( wli, b2_eff_l, gam1_l + 1, 0 );
    const double cfm_r = c_fms( wri, b2_eff_r, gam1_r + 1, 0 );

    spd_m2 = dmin( wli[ MOM ] - cfm_l, wri[ MOM ] - cfm_r );
    spd_p2 = dmax( wli[ MOM ] + cfm_l, wri[ MOM ] + cfm_r );

    if( spd_m2 >= 0 || spd_p2 <= 0 )
    {
        const int is_left = spd_m2 >= 0;
        hlld_f_flux( flx, is_left ? u_l : u_r, is_left ? wli : wri,
                     is_left ? ptot_l : ptot_r, b_x );
        return;
    }

    const double sd_l = spd_m2 - wli[ MOM ];
    const double sd_r = spd_p2 - wri[ MOM ];
    spd0 = ( sd_r * u_r[ MOM ] - ptot_r - sd_l * u_l[ MOM ] + ptot_l )
         / ( sd_r * u_r[ RHO ] - sd_l * u_l[ RHO ] );

    const double sdm_l  = spd_m2 - spd0;
    const double sdm_r  = spd_p2 - spd0;
    const double rhos_l = u_l[ RHO ] * sd_l / sdm_l;
    const double rhos_r = u_r[ RHO ] * sd_r / sdm_r;
    const double rhos_l_sqrt = sqrt( rhos_l );
    const double rhos_r_sqrt = sqrt( rhos_r );
    spd_m1 = spd0 - uabs( b_x ) / rhos_l_sqrt;
    spd_p1 = spd0 + uabs( b_x ) / rhos_r_sqrt;

    const double f_tiny = ( double )( 1.00e-4f );
    const double ptot_s = ptot_l + u_l[ RHO ] * sd_l * ( sd_l - sdm_l );
    const hlld_ctx h = { b_x, bx_2, ptot_s, spd0 };

    double us_l[ 8 ], us_r[ 8 ];
    const double u_dot_b_l = hlld_star( & h, us_l, u_l, wli, rhos_l, sd_l, sdm_l, ptot_l, f_tiny );
    const double u_dot_b_r = hlld_star( & h, us_r, u_r, wri, rhos_r, sd_r, sdm_r, ptot_r, f_tiny );
    if( spd_m1 >= 0 )
    {
        hlld_f_flux( flx, u_l, wli, ptot_l, b_x );
        for( int n = 0; n < 8; ++ n )
            flx[ n ] += spd_m2 * ( us_l[ n ] - u_l[ n ] );
        return;
    }
    else if( spd_p1 <= 0 )
    {
        hlld_f_flux( flx, u_r, wri, ptot_r, b_x );
        for( int n = 0; n < 8; ++ n )
            flx[ n ] += spd_p2 * ( us_r[ n ] - u_r[ n ] );
        return;
    }

    double uss_l[ 8 ], uss_r[ 8 ];
    for( int n = 0; n < 8; ++ n )
    {
        uss_l[ n ] = us_l[ n ];
        uss_r[ n ] = us_r[ n ];
    }
    if( bx_2 > ptot_s * f_tiny )
    {
        const int bx_sgn = b_x > 0 ? 1 : -1;
        const double rhos_norm_inv = 1.f / ( rhos_l_sqrt + rhos_r_sqrt );
        for( int a = 1; a <= 2; ++ a )
        {
            double tmp = rhos_norm_inv *
                ( us_l[ MOM + a ] / rhos_l_sqrt
                + us_r[ MOM + a ] / rhos_r_sqrt
                + bx_sgn * ( us_r[ BCC + a ] - us_l[ BCC + a ] ) );
            uss_l[ MOM + a ] = uss_l[ RHO ] * tmp;
            uss_r[ MOM + a ] = uss_r[ RHO ] * tmp;

            tmp = rhos_norm_inv *
                ( rhos_l_sqrt * us_r[ BCC + a ]
                + rhos_r_sqrt * us_l[ BCC + a ]
                + bx_sgn * rhos_l_sqrt * rhos_r_sqrt
                * ( us_r[ MOM + a ] / rhos_r - us_l[ MOM + a ] / rhos_l ) );
            uss_l[ BCC + a ] = tmp;
            uss_r[ BCC + a ] = tmp;
        }
        const double tmp = spd0 * b_x +
            ( uss_l[ MOM + 1 ] * uss_l[ BCC + 1 ]
            + uss_l[ MOM + 2 ] * uss_l[ BCC + 2 ] ) / uss_l[ RHO ];
        uss_l[ ENE ] -= rhos_l_sqrt * bx_sgn * ( u_dot_b_l - tmp );
        uss_r[ ENE ] += rhos_r_sqrt * bx_sgn * ( u_dot_b_r - tmp );
    }
    if( spd0 >= 0 )
    {
        hlld_f_flux( flx, u_l, wli, ptot_l, b_x );
        const double d_v = spd_m1 - spd_m2;
        for( int n = 0; n < 8; ++ n )
            flx[ n ] += -spd_m2 * u_l[ n ] - d_v * us_l[ n ] + spd_m1 * uss_l[ n ];
    }
    else
    {
        hlld_f_flux( flx, u_r, wri, ptot_r, b_x );
        const double d_v = spd_p1 - spd_p2;
        for( int n = 0; n < 8; ++ n )
            flx[ n ] += -spd_p2 * u_r[ n ] - d_v * us_r[ n ] + spd_p1 * uss_r[ n ];
    }
}

/* mhd/riemann/hlld.h:29-47 calc: rotate momenta and B, solve, rotate the
 * momentum flux back, remap the transverse B fluxes to edge EMFs. */
static void hlld_calc( double * flx, double * ql, double * qr, int axis, double gamma )
{
    idx_swap( ql + MOM, axis );
    idx_swap( qr + MOM, axis );
    idx_swap( ql + BCC, axis );
    idx_swap( qr + BCC, axis );
    hlld_eval( flx, ql, qr, gamma );
    idx_swap( flx + MOM, 3 - axis );
    const double ef[ 2 ] = { flx[ BCC + 2 ], -flx[ BCC + 1 ] };
    flx[ BCC + mod3( axis + 1 ) ] = ef[ 0 ];
    flx[ BCC + mod3( axis + 2 ) ] = ef[ 1 ];
    flx[ BCC + axis ] = 0;
}

void kro_hlld( const double * ql_in, const double * qr_in, int axis, double gamma, double * flx )
{
    double ql[ 8 ], qr[ 8 ];
    memcpy( ql, ql_in, sizeof ql );
    memcpy( qr, qr_in, sizeof qr );
    hlld_calc( flx, ql, qr, axis, gamma );
}

/* ------------------------------------------------------------------ */
/* Face fluxes along one axis for one block: PLM + Riemann on every    */
/* face of every pencil (integrator.h:14-32 flux_kernel; pencil gather  */
/* hydro/integrator/data.h:139-157, MHD mhd/integrator/data.h:146-194;  */
/* MHD also covers the transverse ghost lines, mhd/integrator/         */
/* integrator.h:138-168 and data.h:106-144).                           */

typedef struct { int step; int axis; } flux_arg;

static void flux_pencil( kro_mesh * m, int b, int axis, int step, int t1, int t2 )
{
    const int nw = m->nw;
    const int a1 = mod3( axis + 1 ), a2 = mod3( axis + 2 );
    const int nax = m->c.n[ axis ];
    const double * w  = m->w + ( size_t ) b * m->nw_cells * nw;
    const double * bf = m->c.mhd ? m->bf[ step ] + ( size_t ) b * m->nbf : NULL;
    double * f = m->f[ axis ] + ( size_t ) b * m->nf[ axis ];
    /* mhd/integrator/data.h:98-130 load_primative: on a transverse ghost
     * line next to a side whose neighbour is on another level, the normal
     * B of a face is the cell-centred B of the cell above it */
    int cross = 0;
    if( m->c.mhd && m->smr )
        for( int q = 0; q < 2; ++ q )
        {
            const int a = q ? a2 : a1, t = q ? t2 : t1;
            const int side = t < 0 ? 0 : ( t >= m->c.n[ a ] ? 1 : -1 );
            if( side >= 0 )
            {
                const int fk = m->tree.face[ 6 * b + 2 * a + side ];
                cross |= fk == KR_FACE_FINE || fk == KR_FACE_COARSE;
            }
        }
    for( int fc = 0; fc <= nax; ++ fc )
    {
        double ql[ 8 ], qr[ 8 ], flx[ 8 ];
        int ii[ 3 ];
        ii[ a1 ] = t1;
        ii[ a2 ] = t2;
        for( int k = 0; k < nw; ++ k )
        {
            if( m->c.mhd && k == BCC + axis )
            {
                ii[ axis ] = fc;
                ql[ k ] = qr[ k ] = cross ? w[ iw( m, ii[ 0 ], ii[ 1 ], ii[ 2 ] ) + k ]
                                          : bf[ ib( m, ii[ 0 ], ii[ 1 ], ii[ 2 ] ) + axis ];
                continue;
            }
            double q4[ 4 ];
            for( int s = 0; s < 4; ++ s )
            {
                ii[ axis ] = fc - 2 + s;
                q4[ s ] = w[ iw( m, ii[ 0 ], ii[ 1 ], ii[ 2 ] ) + k ];
            }
            if( m->c.integrator == 1 && step == 0 )
            {   /* VL2 predictor: piecewise-constant (donor-cell) states */
                ql[ k ] = q4[ 1 ];
                qr[ k ] = q4[ 2 ];
            }
            else
                plm_face( q4[ 0 ], q4[ 1 ], q4[ 2 ], q4[ 3 ], & ql[ k ], & qr[ k ] );
        }
        if( m->c.mhd )
            hlld_calc( flx, ql, qr, axis, m->c.gamma );
        else
            hllc_calc( flx, ql, qr, axis, m->c.gamma );
        ii[ axis ] = fc;
        memcpy( f + ifl( m, axis, ii[ 0 ], ii[ 1 ], ii[ 2 ] ), flx, sizeof( double ) * nw );
    }
}

static void flux_block( kro_mesh * m, int b, void * aux )
{
    const flux_arg * fa = ( const flux_arg * ) aux;
    const int axis = fa->axis;
    const int a1 = mod3( axis + 1 ), a2 = mod3( axis + 2 );
    const int n1 = m->c.n[ a1 ], n2 = m->c.n[ a2 ];
    for( int t2 = 0; t2 < n2; ++ t2 )
        for( int t1 = 0; t1 < n1; ++ t1 )
            flux_pencil( m, b, axis, fa->step, t1, t2 );
    if( ! m->c.mhd )
        return;
    for( int t2 = 0; t2 < n2; ++ t2 )
    {
        flux_pencil( m, b, axis, fa->step, -1, t2 );
        flux_pencil( m, b, axis, fa->step, n1, t2 );
    }
    for( int t1 = 0; t1 < n1; ++ t1 )
    {
        flux_pencil( m, b, axis, fa->step, t1, -1 );
        flux_pencil( m, b, axis, fa->step, t1, n2 );
    }
}

/* ------------------------------------------------------------------ */
/* Conserved update (hydro/integrator/integrator.h:58-67 flux_to_du,    */
/* 156-182 load_flux_sfc, 241-265 add_flux; rk2.h:404-425 load).        */

typedef struct { int step; double dt; } upd_arg;

static void update_block( kro_mesh * m, int b, void * aux )
{
    const upd_arg * ua = ( const upd_arg * ) aux;
    const int step = ua->step, nw = m->nw;
    const int * n = m->c.n;
    const double * us = m->u[ step ]     + ( size_t ) b * m->ncell * nw;
    double       * ut = m->u[ 1 - step ] + ( size_t ) b * m->ncell * nw;
    const double vol  = m->vol0[ b ];
    const double dt_dv = ua->dt / vol;
    double f_a[ 3 ];
    for( int a = 0; a < 3; ++ a )
        f_a[ a ] = m->sfc0[ b * 3 + a ] * dt_dv;
    int fine[ 6 ];                       /* geometry.h refine_flag per side */
    for( int k = 0; k < 6; ++ k )
        fine[ k ] = m->smr && m->tree.face[ 6 * b + k ] == KR_FACE_FINE;
    for( int i2 = 0; i2 < n[ 2 ]; ++ i2 )
    for( int i1 = 0; i1 < n[ 1 ]; ++ i1 )
    for( int i0 = 0; i0 < n[ 0 ]; ++ i0 )
    {
        const long c = iu( m, i0, i1, i2 );
        double v[ 8 ];
        for( int k = 0; k < nw; ++ k )
            v[ k ] = step == 0 ? us[ c + k ]
                   : ( m->c.integrator == 1 ? ut[ c + k ] : ( us[ c + k ] + ut[ c + k ] ) * 0.5f );
        for( int a = 0; a < 3; ++ a )
        {
            int ii[ 3 ] = { i0, i1, i2 };
            const double * fl = m->f[ a ] + ( size_t ) b * m->nf[ a ]
                              + ifl( m, a, ii[ 0 ], ii[ 1 ], ii[ 2 ] );
            ++ ii[ a ];
            const double * fr = m->f[ a ] + ( size_t ) b * m->nf[ a ]
                              + ifl( m, a, ii[ 0 ], ii[ 1 ], ii[ 2 ] );
            /* load_flux_sfc: f_a = -1 (skipped) on a refined side's face */
            const int i_a = a == 0 ? i0 : ( a == 1 ? i1 : i2 );
            const int null_l = fine[ 2 * a ] && i_a == 0;
            const int null_r = fine[ 2 * a + 1 ] && i_a == n[ a ] - 1;
            for( int k = 0; k < nw; ++ k )
            {
                double res = 0;
                if( f_a[ a ] > 0 && ! null_l )
                    res += f_a[ a ] * fl[ k ];
                if( f_a[ a ] > 0 && ! null_r )
                    res -= f_a[ a ] * fr[ k ];
                v[ k ] += res;
            }
        }
        /* hydro/integrator/integrator.h:343-382 intg_flx / add_flux, after
         * the update: the cells next to a refined side take the averaged
         * fine flux, sides in the order z, y, x and low before high:
         * u += ( dt * ds / ( +-vol ) ) * f */
        for( int ax = 2; ax >= 0; -- ax )
            for( int side = 0; side <= 1; ++ side )
            {
                const int i_ax = ax == 0 ? i0 : ( ax == 1 ? i1 : i2 );
                if( ! fine[ 2 * ax + side ] || i_ax != ( side ? n[ ax ] - 1 : 0 ) )
                    continue;
                int jj[ 3 ] = { i0, i1, i2 };
                jj[ ax ] = side * n[ ax ];
                const double * fx = m->f[ ax ] + ( size_t ) b * m->nf[ ax ]
                                  + ifl( m, ax, jj[ 0 ], jj[ 1 ], jj[ 2 ] );
                const double ds = m->sfc0[ b * 3 + ax ];
                const double dv = vol * ( side ? -1 : 1 );
                const double conv = ua->dt * ds / dv;
                for( int k = 0; k < nw; ++ k )
                    v[ k ] += conv * fx[ k ];
            }
        for( int k = 0; k < nw; ++ k )
            ut[ c + k ] = v[ k ];
    }
}

/* ------------------------------------------------------------------ */
/* CT: edge EMF (mhd/integrator/integrator.h:189-327 calc_field) and   */
/* face update (385-462 intg_field; rk2.h:244-258 set_field).          */

static inline double e_cell( const kro_mesh * m, const double * w, const int * j, int ax )
{
    /* ec = B x v, from the cell's primitives (mhd/eos/adiabatic.h:216-220;
     * ghost cells: integrator.h:201-213) */
    const double * p = w + iw( m, j[ 0 ], j[ 1 ], j[ 2 ] );
    const int ax1 = mod3( ax + 1 ), ax2 = mod3( ax + 2 );
    return p[ BCC + ax1 ] * p[ MOM + ax2 ] - p[ BCC + ax2 ] * p[ MOM + ax1 ];
}

static void emf_block( kro_mesh * m, int b, void * aux )
{
    ( void ) aux;
    const int nw = m->nw;
    const int * n = m->c.n;
    const double * w = m->w + ( size_t ) b * m->nw_cells * nw;
    const double * F[ 3 ];
    for( int a = 0; a < 3; ++ a )
        F[ a ] = m->f[ a ] + ( size_t ) b * m->nf[ a ];
    double * ee = m->ee + ( size_t ) b * m->nee;
    const double w_e = 0.25f;
    for( int i2 = 0; i2 <= n[ 2 ]; ++ i2 )
    for( int i1 = 0; i1 <= n[ 1 ]; ++ i1 )
    for( int i0 = 0; i0 <= n[ 0 ]; ++ i0 )
    {
        int i[ 3 ] = { i0, i1, i2 };
        for( int ax = 0; ax < 3; ++ ax )
        {
            if( i[ ax ] >= n[ ax ] )
                continue;
            const int ax1 = mod3( 1 + ax ), ax2 = mod3( 2 + ax );
            double ec[ 2 ][ 2 ];
            ec[ 1 ][ 1 ] = e_cell( m, w, i, ax );
            -- i[ ax1 ];
            ec[ 1 ][ 0 ] = e_cell( m, w, i, ax );
            -- i[ ax2 ];
            ec[ 0 ][ 0 ] = e_cell( m, w, i, ax );
            ++ i[ ax1 ];
            ec[ 0 ][ 1 ] = e_cell( m, w, i, ax );
            ++ i[ ax2 ];
            double e = 0;
            for( int it = 0; it < 2; ++ it )
            {
                const int a_para = it == 0 ? ax1 : ax2;
                const int a_perp = it == 0 ? ax2 : ax1;
                -- i[ a_perp ];
                const double ef_m = F[ a_para ][ ifl( m, a_para, i[ 0 ], i[ 1 ], i[ 2 ] ) + BCC + ax ];
                ++ i[ a_perp ];
                const double ef_p = F[ a_para ][ ifl( m, a_para, i[ 0 ], i[ 1 ], i[ 2 ] ) + BCC + ax ];
                e += w_e * ( ef_m + ef_p );
                const double frho_p = F[ a_perp ][ ifl( m, a_perp, i[ 0 ], i[ 1 ], i[ 2 ] ) + RHO ];
                -- i[ a_para ];
                const double frho_m = F[ a_perp ][ ifl( m, a_perp, i[ 0 ], i[ 1 ], i[ 2 ] ) + RHO ];
                ++ i[ a_para ];
                const double de_p = frho_p > 0 ?  ( ec[ 0 ][ 1 ] - ef_m ) :  ( ec[ 1 ][ 1 ] - ef_p );
                const double de_m = frho_m > 0 ? -( ec[ 0 ][ 0 ] - ef_m ) : -( ec[ 1 ][ 0 ] - ef_p );
                e += w_e * ( de_m - de_p );
                if( it == 0 )
                {
                    const double swp = ec[ 0 ][ 1 ];
                    ec[ 0 ][ 1 ] = ec[ 1 ][ 0 ];
                    ec[ 1 ][ 0 ] = swp;
                }
            }
            ee[ ie( m, i0, i1, i2 ) + ax ] = e;
        }
        /* boundary-plane edges of a high out / fre side: the interior cell's
         * advective E, with the reference's velocity scaling (w holds v, which
         * it multiplies by 1 / rho once more) -- integrator.h:329-382 */
        for( int a = 0; a < 3; ++ a )
        {
            if( i[ a ] != n[ a ] || n[ a ] < 2 )
                continue;
            const int kind = m->c.bc[ 2 * a + 1 ];
            const int reg_a = blk_reg( m, b )[ a ];
            if( kind == KRO_PER || reg_a != blk_lim( m, b, a ) - 1 || ( kind != KRO_OUT && kind != KRO_FRE ) )
                continue;
            int jc[ 3 ] = { i[ 0 ], i[ 1 ], i[ 2 ] };
            -- jc[ a ];
            const double * p = w + iw( m, jc[ 0 ], jc[ 1 ], jc[ 2 ] );
            const double irho = 1.0 / fmax( p[ RHO ], 1e-30 );
            double v_c[ 3 ], b_c[ 3 ];
            for( int q = 0; q < 3; ++ q )
            {
                v_c[ q ] = p[ MOM + q ] * irho;
                b_c[ q ] = p[ BCC + q ];
            }
            const int a1 = mod3( a + 1 ), a2 = mod3( a + 2 );
            ee[ ie( m, i0, i1, i2 ) + a1 ] = v_c[ a ] * b_c[ a2 ] - v_c[ a2 ] * b_c[ a ];
            ee[ ie( m, i0, i1, i2 ) + a2 ] = v_c[ a1 ] * b_c[ a ] - v_c[ a ] * b_c[ a1 ];
        }
    }
}

typedef struct { int step; double dt; } ct_arg;

static void ct_block( kro_mesh * m, int b, void * aux )
{
    const ct_arg * ca = ( const ct_arg * ) aux;
    const int step = ca->step;
    const int * n = m->c.n;
    const double * ee = m->ee + ( size_t ) b * m->nee;
    const double * bs = m->bf[ step ]     + ( size_t ) b * m->nbf;
    double       * bt = m->bf[ 1 - step ] + ( size_t ) b * m->nbf;
    const double * dx = m->dx0 + b * 3;
    for( int i2 = 0; i2 <= n[ 2 ]; ++ i2 )
    for( int i1 = 0; i1 <= n[ 1 ]; ++ i1 )
    for( int i0 = 0; i0 <= n[ 0 ]; ++ i0 )
    {
        int i[ 3 ] = { i0, i1, i2 };
        for( int a = 0; a < 3; ++ a )
        {
            const int ax1 = mod3( a + 1 ), ax2 = mod3( a + 2 );
            if( i[ ax1 ] >= n[ ax1 ] || i[ ax2 ] >= n[ ax2 ] )
                continue;
            double db;
            db  = ( ee[ ie( m, i[ 0 ], i[ 1 ], i[ 2 ] ) + ax1 ] * dx[ ax1 ] );
            db -= ( ee[ ie( m, i[ 0 ], i[ 1 ], i[ 2 ] ) + ax2 ] * dx[ ax2 ] );
            ++ i[ ax1 ];
            db += ( ee[ ie( m, i[ 0 ], i[ 1 ], i[ 2 ] ) + ax2 ] * dx[ ax2 ] );
            -- i[ ax1 ];
            ++ i[ ax2 ];
            db -= ( ee[ ie( m, i[ 0 ], i[ 1 ], i[ 2 ] ) + ax1 ] * dx[ ax1 ] );
            -- i[ ax2 ];
            const double sfc = m->sfc0[ b * 3 + a ];
            db *= ( sfc > 0 ? ( -ca->dt / sfc ) : 0. );
            const long k = ib( m, i[ 0 ], i[ 1 ], i[ 2 ] ) + a;
            bt[ k ] = db + ( step == 0 ? bs[ k ]
                           : ( m->c.integrator == 1 ? bt[ k ] : ( bs[ k ] + bt[ k ] ) / 2 ) );
        }
    }
}

/* ------------------------------------------------------------------ */
/* One Heun step (dynamics.h:74-114 integrate, dynamics.cpp:156-161    */
/* step; cycle.cpp:77-115 dt reduction).                                */

int kro_step( kro_mesh * m, int n_steps, double * t, double * dt_bound, double * dt_last )
{
    for( int s = 0; s < n_steps; ++ s )
    {
        double dt_use = 0;
        for( int stage = 0; stage < 2; ++ stage )
        {
            c2p_arg ca = { stage };
            par_blocks( m, c2p_block, & ca );
            if( stage == 0 )
            {
                double d = * dt_bound;
                for( int b = 0; b < m->nblk; ++ b )
                    d = fmin( d, m->dtc[ b ] );
                dt_use = d;
                if( ! isfinite( dt_use ) || dt_use <= 0 )
                    return -1;
            }
            ghost_arg ga = { stage };
            if( m->smr && m->c.mhd )
                mh_act_bnd( m, stage );
            else if( m->smr )
            {   /* keeper.cpp:148-160 act_bnd */
                par_blocks( m, smr_restrict_block, NULL );
                par_blocks( m, bc_block, & ga );
                par_blocks( m, smr_same_block, NULL );
                for( int l = 1; l <= m->tree.max_level; ++ l )
                {
                    prol_arg pa = { l };
                    par_blocks( m, smr_prolong_block, & pa );
                }
            }
            else
            {
                par_blocks( m, ghost_block, & ga );
                par_blocks( m, m->c.mhd ? bc_block_mhd : bc_block, & ga );
            }
            /* Heun: U* = U + dt L(U), U' = (U + U*) / 2 + dt / 2 L(U*).
             * VL2 (van Leer predictor-corrector with CT; Stone & Gardiner 2009,
             * New Astronomy 14, 139): U* = U + dt / 2 L1(U) with donor-cell
             * states, U' = U + dt L(U*) with PLM states.  No counterpart in
             * the reference. */
            const double dt = m->c.integrator == 1 ? dt_use * ( stage == 0 ? ( double ) 0.5f : 1.0 )
                                                   : dt_use * ( stage == 0 ? 1.0 : ( double ) 0.5f );
            for( int axis = 2; axis >= 0; -- axis )
            {
                flux_arg fa = { stage, axis };
                par_blocks( m, flux_block, & fa );
            }
            if( m->smr && m->c.mhd )
            {   /* dynamics.h:80-99: calc_flx (sweeps, then the edge E), act_flx, intg_flx */
                par_blocks( m, emf_block, NULL );
                mh_act_flx( m );
            }
            else if( m->smr )            /* keeper.cpp:162-166 act_flx */
                par_blocks( m, smr_flux_block, NULL );
            upd_arg ua = { stage, dt };
            par_blocks( m, update_block, & ua );
            if( m->c.mhd )
            {
                if( ! m->smr )
                    par_blocks( m, emf_block, NULL );
                ct_arg cta = { stage, dt };
                par_blocks( m, ct_block, & cta );
            }
        }
        * t += dt_use;
        * dt_bound = dt_use * m->c.dt_expand;
        if( dt_last ) * dt_last = dt_use;
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* initial conditions (the pgen side: oracle/pgen/kr_ref_pgen.cpp)       */

int kro_init_problem( kro_mesh * m, const char * name, unsigned long long seed )
{
    const int * n = m->c.n;
    int nglob[ 3 ];
    for( int a = 0; a < 3; ++ a )
        nglob[ a ] = n[ a ] * m->c.nb[ a ];
    const int is_shock = ! strcmp( name, "shock" ), is_turb = ! strcmp( name, "turb" );
    const int is_blast = ! strcmp( name, "blast" );
    const int is_ot = ! strcmp( name, "ot" ) || is_turb || is_blast;   /* the MHD workloads */
    double centre[ 3 ];
    for( int a = 0; a < 3; ++ a )
        centre[ a ] = ( m->c.x_min[ a ] + m->c.x_max[ a ] ) / 2;
    if( ! is_shock && ! is_ot )
        return -1;
    if( is_ot != m->c.mhd )
        return -1;
    kr_turb_t modes;
    if( is_turb )
        kr_turb_modes( & modes, seed );
    for( int b = 0; b < m->nblk; ++ b )
    {
        const int * reg = blk_reg( m, b );
        double * u  = m->u[ 0 ] + ( size_t ) b * m->ncell * m->nw;
        double * bf = is_ot ? m->bf[ 0 ] + ( size_t ) b * m->nbf : NULL;
        if( is_ot )
            for( int i2 = 0; i2 <= n[ 2 ]; ++ i2 )
            for( int i1 = 0; i1 <= n[ 1 ]; ++ i1 )
            for( int i0 = 0; i0 <= n[ 0 ]; ++ i0 )
            {
                double * p = bf + ib( m, i0, i1, i2 );
                p[ 0 ] = is_blast ? kr_blast_b( 0 ) : ( is_turb ? kr_turb_bx( m->c.gamma ) : kr_ot_bx( kro_x_cc( m, b, 1, i1 ) ) );
                p[ 1 ] = is_blast ? kr_blast_b( 1 ) : ( is_turb ? 0.0 : kr_ot_by( kro_x_cc( m, b, 0, i0 ) ) );
                p[ 2 ] = is_blast ? kr_blast_b( 2 ) : ( is_turb ? 0.0 : kr_ot_bz(  ) );
            }
        for( int i2 = 0; i2 < n[ 2 ]; ++ i2 )
        for( int i1 = 0; i1 < n[ 1 ]; ++ i1 )
        for( int i0 = 0; i0 < n[ 0 ]; ++ i0 )
        {
            const int ii[ 3 ] = { i0, i1, i2 };
            int ig[ 3 ];
            for( int a = 0; a < 3; ++ a )
                ig[ a ] = reg[ a ] * n[ a ] + ii[ a ];
            const uint64_t key = kr_cell_key( m->tree.level[ b ], ig, nglob );
            double * c = u + iu( m, i0, i1, i2 );
            if( is_shock )
                kr_shock_cell( c, kro_x_cc( m, b, 0, i0 ), m->c.gamma, seed, key );
            else
            {
                double x[ 3 ], bc[ 3 ];
                for( int a = 0; a < 3; ++ a )
                {
                    int jj[ 3 ] = { i0, i1, i2 };
                    x[ a ] = kro_x_cc( m, b, a, ii[ a ] );
                    const double bl = bf[ ib( m, jj[ 0 ], jj[ 1 ], jj[ 2 ] ) + a ];
                    ++ jj[ a ];
                    bc[ a ] = ( bl + bf[ ib( m, jj[ 0 ], jj[ 1 ], jj[ 2 ] ) + a ] ) / 2;
                }
                if( is_blast )
                    kr_blast_cell( c, x, bc, centre, m->c.gamma );
                else if( is_turb )
                    kr_turb_cell( c, x, bc, m->c.gamma, & modes );
                else
                    kr_ot_cell( c, x, bc, m->c.gamma, seed, key );
            }
        }
    }
    return 0;
}

/* One box of a batch of independent periodic boxes (problems.h kr_box_*): the
 * mesh is the box (the reference runs each box as its own single-block mesh;
 * oracle/pgen/kr_ref_pgen.cpp box_mhd_t). */
int kro_init_box( kro_mesh * m, unsigned long long seed, int box )
{
    const int * n = m->c.n;
    if( ! m->c.mhd || box < 0 )
        return -1;
    int nglob[ 3 ];
    for( int a = 0; a < 3; ++ a )
        nglob[ a ] = n[ a ] * m->c.nb[ a ];
    kr_box_t p;
    kr_box_params( & p, seed, box, m->c.gamma );
    for( int b = 0; b < m->nblk; ++ b )
    {
        const int * reg = blk_reg( m, b );
        double * u  = m->u[ 0 ] + ( size_t ) b * m->ncell * m->nw;
        double * bf = m->bf[ 0 ] + ( size_t ) b * m->nbf;
        for( int i2 = 0; i2 <= n[ 2 ]; ++ i2 )
        for( int i1 = 0; i1 <= n[ 1 ]; ++ i1 )
        for( int i0 = 0; i0 <= n[ 0 ]; ++ i0 )
            for( int a = 0; a < 3; ++ a )
                bf[ ib( m, i0, i1, i2 ) + a ] = p.b[ a ];
        for( int i2 = 0; i2 < n[ 2 ]; ++ i2 )
        for( int i1 = 0; i1 < n[ 1 ]; ++ i1 )
        for( int i0 = 0; i0 < n[ 0 ]; ++ i0 )
        {
            const int ii[ 3 ] = { i0, i1, i2 };
            int ig[ 3 ];
            double x[ 3 ], bc[ 3 ];
            for( int a = 0; a < 3; ++ a )
            {
                int jj[ 3 ] = { i0, i1, i2 };
                ig[ a ] = reg[ a ] * n[ a ] + ii[ a ];
                x[ a ] = kro_x_cc( m, b, a, ii[ a ] );
                const double bl = bf[ ib( m, jj[ 0 ], jj[ 1 ], jj[ 2 ] ) + a ];
                ++ jj[ a ];
                bc[ a ] = ( bl + bf[ ib( m, jj[ 0 ], jj[ 1 ], jj[ 2 ] ) + a ] ) / 2;
            }
            kr_box_cell( u + iu( m, i0, i1, i2 ), x, bc, m->c.gamma, & p,
                         kr_cell_key( m->tree.level[ b ], ig, nglob ) );
        }
    }
    return 0;
}

/* edge length (cells) of box `box` of a batch */
int kro_box_n( unsigned long long seed, int box )
{
    kr_box_t p;
    kr_box_params( & p, seed, box, 5.0 / 3.0 );
    return p.n;
}
