/* Seeded initial conditions for the hydro / MHD step workloads.
 *
 * Header-only, valid C99 and C++, host-side, so that every party that sets up a
 * mesh (the problem generators of this package, the CPU restatement of the
 * step, and the problem generator compiled against the original Kratos
 * sources) builds bit-identical initial states from the same cell coordinates.
 * The noise is a counter-based generator (SplitMix64 of seed and global cell
 * index), so it does not depend on how the mesh is split into blocks.
 *
 * Workloads (coordinates on [0,1)^3, periodic):
 *   shock : rho = 1 | 0.125, p = 1 | 0.1 split at x = 0.5, v = 0,
 *           rho *= 1 + 1e-3 U(-1,1)
 *   ot    : Orszag-Tang-type vortex, rho = 25/(36 pi), p = 5/(12 pi),
 *           v = (-sin 2 pi y, sin 2 pi x, 0) + 1e-3 U(-1,1) per component,
 *           B = (-sin 2 pi y, sin 4 pi x, 0) / sqrt(4 pi) sampled at face
 *           centres (exactly divergence free: B_x has no x dependence, B_y no
 *           y dependence)
 *   turb  : decaying supersonic MHD turbulence (the initial field of a driven
 *           run; no forcing): rho = 1, sound speed 1 (p = 1 / gamma), a
 *           random-phase solenoidal velocity on the 128 integer wavevectors
 *           with 1 <= |k| <= 4 (one of each +-k pair), mode amplitude |k|^-2
 *           (shell spectrum E(k) ~ k^-2), scaled to rms Mach 5, and a uniform
 *           B_x giving plasma beta 2 p / B^2 = 0.1
 *   box   : one of a batch of independent periodic MHD boxes (box = 0, 1, ...):
 *           edge length from {16, 24, 32, 48, 64} cells, rho in [0.5, 2),
 *           p in [0.1, 10), v = A (sin 2 pi y, sin 2 pi z, sin 2 pi x) with
 *           A / c_s in [0.1, 2) plus 1e-3 A U(-1,1) per component, uniform B of
 *           random orientation with beta in [0.05, 10), all drawn uniformly
 *           from (seed, box)
 *   blast : magnetized blast wave, rho = 1, v = 0, p = 100 in the cells whose
 *           centre lies within r < 0.1 of the domain's centre, 0.1 elsewhere,
 *           uniform B = (1, 1, 0) / sqrt(2)
 */
#ifndef KR_PROBLEMS_H
#define KR_PROBLEMS_H

#include <math.h>
#include <stdint.h>

static inline uint64_t kr_splitmix64( uint64_t x )
{
    x += 0x9E3779B97F4A7C15ull;
    x  = ( x ^ ( x >> 30 ) ) * 0xBF58476D1CE4E5B9ull;
    x  = ( x ^ ( x >> 27 ) ) * 0x94D049BB133111EBull;
    return x ^ ( x >> 31 );
}

/* Uniform in [-1, 1): 53 random bits of the hashed (seed, stream, cell) key. */
static inline double kr_uniform_pm1( uint64_t seed, uint64_t stream, uint64_t cell )
{
    const uint64_t h = kr_splitmix64( kr_splitmix64( seed * 0x100000001B3ull + stream ) ^ cell );
    return ( double )( h >> 11 ) * ( 2.0 / 9007199254740992.0 ) - 1.0;
}

/* Global linear cell index at a refinement level (x fastest). */
static inline uint64_t kr_cell_key( int level, const int ig[ 3 ], const int n_glob[ 3 ] )
{
    const uint64_t nx = ( uint64_t ) n_glob[ 0 ] << level;
    const uint64_t ny = ( uint64_t ) n_glob[ 1 ] << level;
    return ( ( uint64_t ) level << 58 )
         ^ ( ( uint64_t ) ig[ 0 ] + nx * ( ( uint64_t ) ig[ 1 ] + ny * ( uint64_t ) ig[ 2 ] ) );
}

#define KR_PI 3.14159265358979323846

/* shock: conserved state of one cell.  u[0] rho, u[1] E, u[2..4] momentum. */
static inline void kr_shock_cell( double * u, double x, double gamma,
                                  uint64_t seed, uint64_t key )
{
    const int left = x < 0.5;
    double rho = left ? 1.0 : 0.125;
    const double pre = left ? 1.0 : 0.1;
    rho *= 1.0 + 1e-3 * kr_uniform_pm1( seed, 0, key );
    u[ 0 ] = rho;
    u[ 1 ] = pre / ( gamma - 1.0 );
    u[ 2 ] = u[ 3 ] = u[ 4 ] = 0.0;
}

/* ot: face fields and the conserved state of one cell. */
static inline double kr_ot_bx( double y_cc ) { return -sin( 2 * KR_PI * y_cc ) / sqrt( 4 * KR_PI ); }
static inline double kr_ot_by( double x_cc ) { return  sin( 4 * KR_PI * x_cc ) / sqrt( 4 * KR_PI ); }
static inline double kr_ot_bz( void )        { return 0.0; }

/* u[0] rho, u[1] E (incl. magnetic energy of the face-averaged field),
 * u[2..4] momentum, u[5..7] cell-centred B.  b_cc: face-averaged B of the cell. */
static inline void kr_ot_cell( double * u, const double x_cc[ 3 ], const double b_cc[ 3 ],
                               double gamma, uint64_t seed, uint64_t key )
{
    const double rho = 25.0 / ( 36.0 * KR_PI );
    const double pre =  5.0 / ( 12.0 * KR_PI );
    double v[ 3 ], ek = 0, em = 0;
    v[ 0 ] = -sin( 2 * KR_PI * x_cc[ 1 ] ) + 1e-3 * kr_uniform_pm1( seed, 0, key );
    v[ 1 ] =  sin( 2 * KR_PI * x_cc[ 0 ] ) + 1e-3 * kr_uniform_pm1( seed, 1, key );
    v[ 2 ] =                                 1e-3 * kr_uniform_pm1( seed, 2, key );
    for( int a = 0; a < 3; ++ a )
    {
        ek += v[ a ] * v[ a ];
        em += b_cc[ a ] * b_cc[ a ];
    }
    u[ 0 ] = rho;
    u[ 1 ] = pre / ( gamma - 1.0 ) + 0.5 * rho * ek + 0.5 * em;
    for( int a = 0; a < 3; ++ a )
    {
        u[ 2 + a ] = rho * v[ a ];
        u[ 5 + a ] = b_cc[ a ];
    }
}

/* turb: the mode table (built once per seed) and the state of one cell. */
#define KR_TURB_MODES 128

typedef struct
{
    double k[ KR_TURB_MODES ][ 3 ];      /* integer wavevector */
    double a[ KR_TURB_MODES ][ 3 ];      /* amplitude vector, perpendicular to k */
    double phase[ KR_TURB_MODES ];
} kr_turb_t;

static inline void kr_turb_modes( kr_turb_t * t, uint64_t seed )
{
    int m = 0;
    double sum_a2 = 0;
    for( int kz = -4; kz <= 4; ++ kz )
    for( int ky = -4; ky <= 4; ++ ky )
    for( int kx = -4; kx <= 4; ++ kx )
    {
        const int k2 = kx * kx + ky * ky + kz * kz;
        if( k2 < 1 || k2 > 16 || ! ( kx > 0 || ( kx == 0 && ( ky > 0 || ( ky == 0 && kz > 0 ) ) ) ) )
            continue;
        const double k[ 3 ] = { ( double ) kx, ( double ) ky, ( double ) kz };
        double r[ 3 ], e[ 3 ], rk = 0, e2 = 0;
        for( int d = 0; d < 3; ++ d )
        {
            r[ d ] = kr_uniform_pm1( seed, 16 + d, ( uint64_t ) m );
            rk += r[ d ] * k[ d ];
        }
        for( int d = 0; d < 3; ++ d )    /* r minus its component along k */
        {
            e[ d ] = r[ d ] - rk / k2 * k[ d ];
            e2 += e[ d ] * e[ d ];
        }
        if( e2 < 1e-6 )
        {   /* r (nearly) parallel to k: use k x (0, 0, 1), or k x (1, 0, 0) */
            const int z = kx == 0 && ky == 0;
            e[ 0 ] = z ? 0.0 : k[ 1 ];
            e[ 1 ] = z ? k[ 2 ] : -k[ 0 ];
            e[ 2 ] = z ? -k[ 1 ] : 0.0;
            e2 = e[ 0 ] * e[ 0 ] + e[ 1 ] * e[ 1 ] + e[ 2 ] * e[ 2 ];
        }
        const double amp = 1.0 / k2;     /* |k|^-2 */
        const double s = amp / sqrt( e2 );
        for( int d = 0; d < 3; ++ d )
        {
            t->k[ m ][ d ] = k[ d ];
            t->a[ m ][ d ] = s * e[ d ];
        }
        t->phase[ m ] = KR_PI * ( kr_uniform_pm1( seed, 19, ( uint64_t ) m ) + 1.0 );
        sum_a2 += amp * amp;
        ++ m;
    }
    /* <|v|^2> over the periodic cell = sum a^2 / 2 (distinct modes are
     * orthogonal, also on a uniform grid of more than 8 points per axis):
     * scale to rms Mach 5 at sound speed 1 */
    const double scale = 5.0 / sqrt( sum_a2 / 2 );
    for( m = 0; m < KR_TURB_MODES; ++ m )
        for( int d = 0; d < 3; ++ d )
            t->a[ m ][ d ] *= scale;
}

static inline double kr_turb_bx( double gamma ) { return sqrt( 2.0 / gamma / 0.1 ); }

/* u[0] rho, u[1] E (incl. magnetic energy of the face-averaged field),
 * u[2..4] momentum, u[5..7] cell-centred B.  b_cc: face-averaged B of the cell. */
static inline void kr_turb_cell( double * u, const double x_cc[ 3 ], const double b_cc[ 3 ],
                                 double gamma, const kr_turb_t * t )
{
    const double rho = 1.0, pre = 1.0 / gamma;
    double v[ 3 ] = { 0, 0, 0 }, ek = 0, em = 0;
    for( int m = 0; m < KR_TURB_MODES; ++ m )
    {
        const double c = cos( 2 * KR_PI * ( t->k[ m ][ 0 ] * x_cc[ 0 ] + t->k[ m ][ 1 ] * x_cc[ 1 ]
                                          + t->k[ m ][ 2 ] * x_cc[ 2 ] ) + t->phase[ m ] );
        for( int d = 0; d < 3; ++ d )
            v[ d ] += t->a[ m ][ d ] * c;
    }
    for( int a = 0; a < 3; ++ a )
    {
        ek += v[ a ] * v[ a ];
        em += b_cc[ a ] * b_cc[ a ];
    }
    u[ 0 ] = rho;
    u[ 1 ] = pre / ( gamma - 1.0 ) + 0.5 * rho * ek + 0.5 * em;
    for( int a = 0; a < 3; ++ a )
    {
        u[ 2 + a ] = rho * v[ a ];
        u[ 5 + a ] = b_cc[ a ];
    }
}

/* box: the parameters of box `box` of a batch, and the state of one of its
 * cells (cell key: the box's own lexicographic cell index at level 0). */
typedef struct
{
    int    n;                            /* cells per axis */
    double rho, pre, amp, beta, b[ 3 ];
    uint64_t seed;                       /* the box's noise seed */
} kr_box_t;

static inline void kr_box_params( kr_box_t * p, uint64_t seed, int box, double gamma )
{
    const uint64_t k = ( uint64_t ) box;
    int s = ( int )( ( kr_uniform_pm1( seed, 32, k ) + 1.0 ) * 2.5 );
    if( s > 4 )
        s = 4;
    p->n    = s == 0 ? 16 : ( s == 1 ? 24 : ( s == 2 ? 32 : ( s == 3 ? 48 : 64 ) ) );
    p->rho  = 0.5  + 0.75  * ( kr_uniform_pm1( seed, 33, k ) + 1.0 );
    p->pre  = 0.1  + 4.95  * ( kr_uniform_pm1( seed, 34, k ) + 1.0 );
    p->beta = 0.05 + 4.975 * ( kr_uniform_pm1( seed, 35, k ) + 1.0 );
    p->amp  = sqrt( gamma * p->pre / p->rho ) * ( 0.1 + 0.95 * ( kr_uniform_pm1( seed, 36, k ) + 1.0 ) );
    const double ct = kr_uniform_pm1( seed, 37, k );              /* cos theta */
    const double st = sqrt( 1.0 - ct * ct );
    const double ph = KR_PI * ( kr_uniform_pm1( seed, 38, k ) + 1.0 );
    const double bm = sqrt( 2.0 * p->pre / p->beta );
    p->b[ 0 ] = bm * st * cos( ph );
    p->b[ 1 ] = bm * st * sin( ph );
    p->b[ 2 ] = bm * ct;
    p->seed = kr_splitmix64( seed ^ ( 0xD1B54A32D192ED03ull * ( k + 1 ) ) );
}

/* u[0] rho, u[1] E (incl. magnetic energy of the face-averaged field),
 * u[2..4] momentum, u[5..7] cell-centred B.  b_cc: face-averaged B of the cell. */
static inline void kr_box_cell( double * u, const double x_cc[ 3 ], const double b_cc[ 3 ],
                                double gamma, const kr_box_t * p, uint64_t key )
{
    double v[ 3 ], ek = 0, em = 0;
    v[ 0 ] = p->amp * ( sin( 2 * KR_PI * x_cc[ 1 ] ) + 1e-3 * kr_uniform_pm1( p->seed, 40, key ) );
    v[ 1 ] = p->amp * ( sin( 2 * KR_PI * x_cc[ 2 ] ) + 1e-3 * kr_uniform_pm1( p->seed, 41, key ) );
    v[ 2 ] = p->amp * ( sin( 2 * KR_PI * x_cc[ 0 ] ) + 1e-3 * kr_uniform_pm1( p->seed, 42, key ) );
    for( int a = 0; a < 3; ++ a )
    {
        ek += v[ a ] * v[ a ];
        em += b_cc[ a ] * b_cc[ a ];
    }
    u[ 0 ] = p->rho;
    u[ 1 ] = p->pre / ( gamma - 1.0 ) + 0.5 * p->rho * ek + 0.5 * em;
    for( int a = 0; a < 3; ++ a )
    {
        u[ 2 + a ] = p->rho * v[ a ];
        u[ 5 + a ] = b_cc[ a ];
    }
}

/* blast: face fields and the conserved state of one cell.  c: the domain's
 * centre.  u[0] rho, u[1] E (incl. magnetic energy of the face-averaged
 * field), u[2..4] momentum, u[5..7] cell-centred B. */
static inline double kr_blast_b( int axis ) { return axis < 2 ? sqrt( 0.5 ) : 0.0; }

static inline double kr_blast_pre( const double x_cc[ 3 ], const double c[ 3 ] )
{
    double r2 = 0;
    for( int a = 0; a < 3; ++ a )
        r2 += ( x_cc[ a ] - c[ a ] ) * ( x_cc[ a ] - c[ a ] );
    return r2 < 0.01 ? 100.0 : 0.1;
}

static inline void kr_blast_cell( double * u, const double x_cc[ 3 ], const double b_cc[ 3 ],
                                  const double c[ 3 ], double gamma )
{
    double em = 0;
    for( int a = 0; a < 3; ++ a )
        em += b_cc[ a ] * b_cc[ a ];
    u[ 0 ] = 1.0;
    u[ 1 ] = kr_blast_pre( x_cc, c ) / ( gamma - 1.0 ) + 0.5 * em;
    for( int a = 0; a < 3; ++ a )
    {
        u[ 2 + a ] = 0.0;
        u[ 5 + a ] = b_cc[ a ];
    }
}

#endif
