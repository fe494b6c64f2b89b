/* Static mesh refinement: the block tree and the face neighbours of its
 * leaves, as Kratos builds them (mesh/meshgen/meshgen.cpp:111-160
 * load_refinement / generate_tree / search_blk_idx, mesh/tree/tree.cpp:139-232
 * map_neighbor / insert / fill_base_level, mesh/geometry/region.h neighbour
 * modes).  C99, header only: shared by the device engine's host code and the
 * CPU restatement (the topology is not arithmetic; both are checked against the
 * reference's own snapshots).
 *
 * A refinement region [refine_region*] (level L, box x_min..x_max) inserts every
 * level-L node whose block contains a point of the box.  Inserting a node
 * refines its parent (creating all 8 children) and inserts the parent's 26
 * neighbours, so adjacent leaves differ by at most one level; afterwards every
 * level-0 node is inserted.  Leaves are the nodes not refined.
 *
 * Leaves are numbered level by level, lexicographically (x fastest) inside a
 * level.  For every leaf and face direction (axis a, side s: 2 a + s) the
 * neighbour is one of
 *   KR_FACE_PHYS   past a non-periodic domain side
 *   KR_FACE_SAME   a leaf of the same level             (nb[0])
 *   KR_FACE_COARSE a leaf one level coarser             (nb[0])
 *   KR_FACE_FINE   four leaves one level finer, ordered by their offsets
 *                  (d1, d2) along axes (a+1)%3, (a+2)%3, d1 outer  (nb[0..3])
 */
#ifndef KR_SMR_TREE_H
#define KR_SMR_TREE_H

#include <stdlib.h>
#include <string.h>

#define KR_TREE_MAX_LEVEL 6
enum { KR_FACE_PHYS = 0, KR_FACE_SAME = 1, KR_FACE_COARSE = 2, KR_FACE_FINE = 3 };

typedef struct
{
    int    level;
    double x_min[ 3 ], x_max[ 3 ];
} kr_tree_region;

typedef struct
{
    int   nb[ 3 ], periodic[ 3 ], max_level;
    unsigned char * node[ KR_TREE_MAX_LEVEL + 1 ];   /* 0 absent, 1 leaf, 2 refined */
    int   nblk;
    int * level;          /* [nblk]        */
    int * reg;            /* [nblk][3]     logical position at its level */
    int * face;           /* [nblk][6]     KR_FACE_*                     */
    int * fnb;            /* [nblk][6][4]  neighbour leaves             */
} kr_tree;

static inline long kr_tree_lim( const kr_tree * t, int l, int a ) { return ( long ) t->nb[ a ] << l; }

static inline long kr_tree_idx( const kr_tree * t, int l, const int * r )
{
    return r[ 0 ] + kr_tree_lim( t, l, 0 ) * ( r[ 1 ] + kr_tree_lim( t, l, 1 ) * ( long ) r[ 2 ] );
}

/* tree.cpp:64-81 is_inside / regularize: wrap periodic axes; 0 if outside */
static inline int kr_tree_regularize( const kr_tree * t, int l, int * r )
{
    for( int a = 0; a < 3; ++ a )
    {
        const long lim = kr_tree_lim( t, l, a );
        if( t->periodic[ a ] )
            r[ a ] = ( int )( ( r[ a ] + lim ) % lim );
        if( r[ a ] < 0 || r[ a ] >= lim )
            return 0;
    }
    return 1;
}

static inline void kr_tree_insert( kr_tree * t, int l, const int * r_in )
{
    int r[ 3 ] = { r_in[ 0 ], r_in[ 1 ], r_in[ 2 ] };
    unsigned char * n = t->node[ l ];
    if( n[ kr_tree_idx( t, l, r ) ] )
        return;
    if( l > 0 )
    {
        int p[ 3 ] = { r[ 0 ] >> 1, r[ 1 ] >> 1, r[ 2 ] >> 1 };
        kr_tree_insert( t, l - 1, p );
        t->node[ l - 1 ][ kr_tree_idx( t, l - 1, p ) ] = 2;
        for( int d2 = 0; d2 < 2; ++ d2 )          /* map_refined: all 8 children */
        for( int d1 = 0; d1 < 2; ++ d1 )
        for( int d0 = 0; d0 < 2; ++ d0 )
        {
            const int c[ 3 ] = { 2 * p[ 0 ] + d0, 2 * p[ 1 ] + d1, 2 * p[ 2 ] + d2 };
            unsigned char * e = & n[ kr_tree_idx( t, l, c ) ];
            if( ! * e ) * e = 1;
        }
        for( int s0 = -1; s0 <= 1; ++ s0 )         /* map_neighbor of the parent */
        for( int s1 = -1; s1 <= 1; ++ s1 )
        for( int s2 = -1; s2 <= 1; ++ s2 )
        {
            if( ! s0 && ! s1 && ! s2 )
                continue;
            int q[ 3 ] = { p[ 0 ] + s0, p[ 1 ] + s1, p[ 2 ] + s2 };
            if( kr_tree_regularize( t, l - 1, q ) )
                kr_tree_insert( t, l - 1, q );
        }
    }
    unsigned char * e = & n[ kr_tree_idx( t, l, r ) ];
    if( ! * e ) * e = 1;
}

/* meshgen.cpp:365-384: the block index (at level l, axis a) whose left edge is
 * the last one below loc (bisection on the logical coordinate) */
static inline int kr_tree_search( const kr_tree * t, double lo, double hi, double loc, int l, int a )
{
    if( loc > hi || loc < lo )
        return -1;
    const int i_tot = ( int ) kr_tree_lim( t, l, a );
    int i_r = i_tot, i_l = 0;
    const double i_ftot = ( double ) i_tot;
    while( i_r - i_l > 1 )
    {
        const int i_m = ( i_l + i_r ) / 2;
        if( lo + i_m / i_ftot * ( hi - lo ) < loc )
            i_l = i_m;
        else
            i_r = i_m;
    }
    return i_l;
}

static inline void kr_tree_free( kr_tree * t )
{
    for( int l = 0; l <= KR_TREE_MAX_LEVEL; ++ l )
        free( t->node[ l ] );
    free( t->level ); free( t->reg ); free( t->face ); free( t->fnb );
    memset( t, 0, sizeof( * t ) );
}

/* Build the tree and the leaves' face neighbours.  Returns 0, or -1 with a
 * message in err (a region outside the domain or deeper than the maximum). */
static inline int kr_tree_build( kr_tree * t, const int nb[ 3 ], const int periodic[ 3 ],
                                 const double x_min[ 3 ], const double x_max[ 3 ],
                                 int n_regions, const kr_tree_region * regions,
                                 char * err, int errlen )
{
    memset( t, 0, sizeof( * t ) );
    int max_level = 0;
    for( int k = 0; k < n_regions; ++ k )
    {
        if( regions[ k ].level < 0 || regions[ k ].level > KR_TREE_MAX_LEVEL - 1 )
        {
            if( err ) strncpy( err, "refinement level out of range", errlen );
            return -1;
        }
        if( regions[ k ].level > max_level ) max_level = regions[ k ].level;
    }
    for( int a = 0; a < 3; ++ a ) { t->nb[ a ] = nb[ a ]; t->periodic[ a ] = periodic[ a ]; }
    t->max_level = max_level;
    for( int l = 0; l <= max_level + 1 && l <= KR_TREE_MAX_LEVEL; ++ l )
        t->node[ l ] = ( unsigned char * ) calloc( ( size_t ) kr_tree_lim( t, l, 0 ) * kr_tree_lim( t, l, 1 )
                                                    * kr_tree_lim( t, l, 2 ), 1 );
    for( int k = 0; k < n_regions; ++ k )
    {
        const kr_tree_region * g = regions + k;
        if( g->level <= 0 )
            continue;
        int i0[ 3 ], i1[ 3 ];
        for( int a = 0; a < 3; ++ a )
        {
            i0[ a ] = kr_tree_search( t, x_min[ a ], x_max[ a ], g->x_min[ a ], g->level, a );
            i1[ a ] = kr_tree_search( t, x_min[ a ], x_max[ a ], g->x_max[ a ], g->level, a );
            if( i0[ a ] < 0 || i1[ a ] < 0 )
            {
                if( err ) strncpy( err, "Incorrect SMR region", errlen );
                kr_tree_free( t );
                return -1;
            }
        }
        int r[ 3 ];
        for( r[ 2 ] = i0[ 2 ]; r[ 2 ] <= i1[ 2 ]; ++ r[ 2 ] )   /* loop(.., .., true): inclusive */
        for( r[ 1 ] = i0[ 1 ]; r[ 1 ] <= i1[ 1 ]; ++ r[ 1 ] )
        for( r[ 0 ] = i0[ 0 ]; r[ 0 ] <= i1[ 0 ]; ++ r[ 0 ] )
            kr_tree_insert( t, g->level, r );
    }
    {   /* fill_base_level */
        int r[ 3 ];
        for( r[ 2 ] = 0; r[ 2 ] < nb[ 2 ]; ++ r[ 2 ] )
        for( r[ 1 ] = 0; r[ 1 ] < nb[ 1 ]; ++ r[ 1 ] )
        for( r[ 0 ] = 0; r[ 0 ] < nb[ 0 ]; ++ r[ 0 ] )
            kr_tree_insert( t, 0, r );
    }
    /* leaves, level by level, lexicographic */
    int n = 0;
    for( int l = 0; l <= max_level; ++ l )
    {
        const long tot = kr_tree_lim( t, l, 0 ) * kr_tree_lim( t, l, 1 ) * kr_tree_lim( t, l, 2 );
        for( long i = 0; i < tot; ++ i )
            n += t->node[ l ][ i ] == 1;
    }
    t->nblk = n;
    t->level = ( int * ) malloc( sizeof( int ) * n );
    t->reg = ( int * ) malloc( sizeof( int ) * n * 3 );
    t->face = ( int * ) malloc( sizeof( int ) * n * 6 );
    t->fnb = ( int * ) malloc( sizeof( int ) * n * 24 );
    /* leaf number per node, for the neighbour lookup */
    int * id[ KR_TREE_MAX_LEVEL + 1 ] = { 0 };
    n = 0;
    for( int l = 0; l <= max_level; ++ l )
    {
        const long tot = kr_tree_lim( t, l, 0 ) * kr_tree_lim( t, l, 1 ) * kr_tree_lim( t, l, 2 );
        id[ l ] = ( int * ) malloc( sizeof( int ) * tot );
        for( long i = 0; i < tot; ++ i )
        {
            id[ l ][ i ] = -1;
            if( t->node[ l ][ i ] != 1 )
                continue;
            id[ l ][ i ] = n;
            t->level[ n ] = l;
            t->reg[ 3 * n + 0 ] = ( int )( i % kr_tree_lim( t, l, 0 ) );
            t->reg[ 3 * n + 1 ] = ( int )( ( i / kr_tree_lim( t, l, 0 ) ) % kr_tree_lim( t, l, 1 ) );
            t->reg[ 3 * n + 2 ] = ( int )( i / ( kr_tree_lim( t, l, 0 ) * kr_tree_lim( t, l, 1 ) ) );
            ++ n;
        }
    }
    for( int b = 0; b < t->nblk; ++ b )
    {
        const int l = t->level[ b ];
        for( int f = 0; f < 6; ++ f )
        {
            const int a = f / 2, s = f & 1;
            int * fn = t->fnb + ( b * 6 + f ) * 4;
            fn[ 0 ] = fn[ 1 ] = fn[ 2 ] = fn[ 3 ] = -1;
            int r[ 3 ] = { t->reg[ 3 * b ], t->reg[ 3 * b + 1 ], t->reg[ 3 * b + 2 ] };
            r[ a ] += s ? 1 : -1;
            if( ! kr_tree_regularize( t, l, r ) )
            {
                t->face[ b * 6 + f ] = KR_FACE_PHYS;
                continue;
            }
            const unsigned char st = t->node[ l ][ kr_tree_idx( t, l, r ) ];
            if( st == 1 )
            {
                t->face[ b * 6 + f ] = KR_FACE_SAME;
                fn[ 0 ] = id[ l ][ kr_tree_idx( t, l, r ) ];
            }
            else if( st == 2 )
            {   /* refined: the four children that touch this face */
                t->face[ b * 6 + f ] = KR_FACE_FINE;
                const int a1 = ( a + 1 ) % 3, a2 = ( a + 2 ) % 3;
                for( int d1 = 0; d1 < 2; ++ d1 )
                for( int d2 = 0; d2 < 2; ++ d2 )
                {
                    int c[ 3 ];
                    c[ a ] = 2 * r[ a ] + ( s ? 0 : 1 );
                    c[ a1 ] = 2 * r[ a1 ] + d1;
                    c[ a2 ] = 2 * r[ a2 ] + d2;
                    fn[ d1 * 2 + d2 ] = id[ l + 1 ][ kr_tree_idx( t, l + 1, c ) ];
                }
            }
            else
            {   /* absent at this level: a coarser leaf holds the position */
                t->face[ b * 6 + f ] = KR_FACE_COARSE;
                int p[ 3 ] = { r[ 0 ] >> 1, r[ 1 ] >> 1, r[ 2 ] >> 1 };
                fn[ 0 ] = l > 0 ? id[ l - 1 ][ kr_tree_idx( t, l - 1, p ) ] : -1;
            }
        }
    }
    for( int l = 0; l <= max_level; ++ l )
        free( id[ l ] );
    return 0;
}

#endif
