// Static refinement, MHD: the ghost exchange across level jumps and the edge-E
// correction; included by kr_core.cu ahead of the context (namespace kr).
//
// The reference enrols one exchange holder per (host block, neighbour) pair,
// faces, edges and vertices alike (mhd/boundary/keeper.h:280-285
// desired_mode), and each holder pushes from its host into its guest: the
// primitives by copy (same level, to_same), volume average (finer host,
// to_coarser) or limited-slope prolongation (coarser host, to_finer), and for
// face holders the tangential face B of the guest's first ghost layer: copy,
// area average of the finer faces, or Toth & Roe's divergence-preserving
// prolongation (mhd/boundary/comm_functions.h:422-780).  After the flux
// sweeps and the edge EMF, a finer host's face holder sets the coarser
// guest's tangential edge E on the refined face to the length average of its
// two finer edges, and an edge holder the E along a refined edge, each
// writing the average back onto its own edges (comm_functions.h:818-954).
//
// Here the holders are built on the host in the reference's order (hosts by
// level, then logical position with x most significant, region.h lex_ord_t;
// each host's neighbours by their direction flags), with the reference's
// launch grid of each (resource_pack / resource_flux / resource_edge, at most
// MH_TH threads per CTA row, the last CTA's second pass).  A phase of the
// exchange (restrictions, prolongations by the coarser host's level) is one
// launch of one thread per work item (holder, item); inside a phase no two
// holders write the same slot (each writes its own guest's band), so the
// order of the items does not matter.  Same-level copies use the push of the
// uniform step instead (k_c2p writes each cell into the neighbours whose ghost
// shell holds it, the CT update the face-B strips): the same copies, written
// while the data is in registers.  The edge-E correction reads what
// earlier holders wrote back, so its holders run in waves: a holder waits for
// every earlier holder that reads or writes one of its edges.
//
// Every written ghost cell also gets its cell E, B x v from the written
// primitives (mhd/integrator/integrator.h:201-213 computes a ghost cell's E
// that way); same-level copies copy the E of the host's cell, which c2p
// computed from the same B and v.

enum { MH_TH = 64, MH_ORD = 2, MH_NGH = 2 };     // [dynamics] bnd_thread_limit (its default); PLM order; ghosts
enum { MH_RESTRICT = 1, MH_PROLONG = 2, MH_FLUX = 3 };

struct mh_t
{
    int host, guest, mode, d_lvl, rhs;
    int ax[ 3 ];
    int os[ 3 ], oc[ 3 ];                // primitives: host / guest offsets
    int obs[ 3 ], obc[ 3 ], obr[ 3 ];    // face B
    int oes[ 3 ], oec[ 3 ];              // edge E
    int nbx, nby, nth;                   // launch grid of the holder's exchange kernel
    int fbx, fby, fth;                   // and of its edge-E correction
    int n1;                              // the exchange grid's extent along ax[ 1 ]
    int dir;                             // the guest's direction ( x + 1 ) + 3 ( y + 1 ) + 9 ( z + 1 )
    int rw[ 2 ], rb[ 2 ];                // restriction / prolongation: the (ax[ 1 ], ax[ 2 ]) extents
                                         // of the primitives' and the face B's rows
};

__device__ __forceinline__ void mh_dispatch( const mh_t & h, int nth, int bx, int by, int tx, int * i )
{   // hydro/boundary/comm_functions.h:160-166 dispatch
    i[ h.ax[ 0 ] ] = 0;
    i[ h.ax[ 1 ] ] = bx * nth + tx;
    i[ h.ax[ 2 ] ] = by;
}

// Accessors with their own bounds check: an index outside the array's box
// (W: ghosts -2..n+1; face B: -2..n+2; edge E: -1..n+1) sets status bit 2 and
// the access goes to a scratch word instead.
__device__ double mh_sink[ 4 ];

template< class R > __device__ __forceinline__
bool mh_in( const args_t< R > & a, int b, const int * i, int lo, int hi_extra )
{
    const int nn[ 3 ] = { a.n0, a.n1, a.n2 };
    bool ok = b >= 0 && b < a.nblk;
    for( int d = 0; d < 3; ++ d )
        ok &= i[ d ] >= lo && i[ d ] <= nn[ d ] + hi_extra;
    if( ! ok )
        atomicOr( & a.s[ 0 ].status, 4 );
    return ok;
}
template< class R > __device__ __forceinline__
R * mh_w( const args_t< R > & a, int b, int c, const int * i )
{
    return mh_in( a, b, i, -2, 1 ) ? a.w + iw( a, b, c, 11, i[ 0 ], i[ 1 ], i[ 2 ] ) : ( R * ) mh_sink;
}
template< class R > __device__ __forceinline__
double * mh_bf( const args_t< R > & a, int step, int b, int c, const int * i )
{
    return mh_in( a, b, i, -2, 2 ) ? a.bf[ step ] + ibf( a, b, c, i[ 0 ], i[ 1 ], i[ 2 ] ) : mh_sink;
}
template< class R > __device__ __forceinline__
R * mh_ee( const args_t< R > & a, int b, int c, const int * i )
{
    return mh_in( a, b, i, -1, 1 ) ? a.ee + ifx( a, b, c, 3, i[ 0 ], i[ 1 ], i[ 2 ] ) : ( R * ) mh_sink;
}

__device__ __forceinline__ double mh_minmod( double x, double y )
{   // utilities/functions.h:164-170
    return ( ( x < 0 ) != ( y < 0 ) ) ? 0. : ( fabs( x ) < fabs( y ) ? x : y );
}

// Cell E of a written ghost cell from its primitives (the words 8..10).
template< class R > __device__ __forceinline__
void mh_cell_e( const args_t< R > & a, int b, const int * i )
{
    R q[ 6 ];
    for( int k = 0; k < 3; ++ k )
    {
        q[ k ] = * mh_w( a, b, MOM + k, i );
        q[ 3 + k ] = * mh_w( a, b, BCC + k, i );
    }
    for( int c = 0; c < 3; ++ c )
    {
        const int c1 = mod3( c + 1 ), c2 = mod3( c + 2 );
        * mh_w( a, b, 8 + c, i ) = q[ 3 + c1 ] * q[ c2 ] - q[ 3 + c2 ] * q[ c1 ];
    }
}

__device__ __forceinline__ bool mh_in_band( int i, int off )
{   // mhd/boundary/comm_functions.h:446-452 in_band_axis
    return off == 0 || ( i - off >= 0 && i - off < MH_ORD );
}

// finer host -> coarser guest (hydro comm_functions.h:329-380 to_coarser
// inside MHD 693-780: NGH-wide bands for edge / vertex holders, the area
// average of the tangential face B for face holders).  One row (c1, c2) of
// the reference's dispatch (ax[ 1 ], ax[ 2 ]) per call; the face-B rows include
// the last CTA's second pass.
template< class R > __device__ __forceinline__
void mh_restrict_w( const args_t< R > & a, const mh_t & h, int c1, int c2 )
{
    const int ax = h.ax[ 0 ], a1 = h.ax[ 1 ], a2 = h.ax[ 2 ];
    int i0[ 3 ], im[ 3 ], ib[ 3 ];
    i0[ ax ] = 0; i0[ a1 ] = c1; i0[ a2 ] = c2;
    for( int d = 0; d < 3; ++ d )
    {
        im[ d ] = h.os[ d ] + 2 * i0[ d ];
        ib[ d ] = i0[ d ] + h.oc[ d ];
    }
    const double dv = a.geo[ h.host ].vol;
    for( int k2 = 0; k2 < MH_ORD; ++ k2 )
    {
        double p[ 8 ], norm = 0;
        for( int c = 0; c < 8; ++ c )
            p[ c ] = 0;
        for( int kk = 0; kk < 2; ++ kk )
        {
            im[ ax ] = 2 * k2 + kk + h.os[ ax ];
            const int s1 = im[ a1 ], s2 = im[ a2 ];
            for( int d1 = 0; d1 < 2; ++ d1 )
            for( int d2 = 0; d2 < 2; ++ d2 )
            {
                im[ a1 ] = s1 + d1;
                im[ a2 ] = s2 + d2;
                for( int c = 0; c < 8; ++ c )
                    p[ c ] += double( * mh_w( a, h.host, c, im ) ) * dv;
                norm += dv;
            }
            im[ a1 ] = s1;
            im[ a2 ] = s2;
        }
        ib[ ax ] = k2 + h.oc[ ax ];
        for( int c = 0; c < 8; ++ c )
            * mh_w( a, h.guest, c, ib ) = R( p[ c ] / norm );
        mh_cell_e( a, h.guest, ib );
    }
}

template< class R > __device__ __forceinline__
void mh_restrict_b( const args_t< R > & a, const mh_t & h, int step, int c1, int c2, const int * n )
{
    const int ax = h.ax[ 0 ], a1 = h.ax[ 1 ], a2 = h.ax[ 2 ];
    const geo_t & g = a.geo[ h.host ];
    int i0[ 3 ], im[ 3 ], ib[ 3 ];
    i0[ ax ] = 0; i0[ a1 ] = c1; i0[ a2 ] = c2;
    for( int d = 0; d < 3; ++ d )
    {
        im[ d ] = 2 * i0[ d ] + h.obs[ d ];
        ib[ d ] = i0[ d ] + h.obc[ d ];
    }
    if( h.obs[ ax ] > 0 )
        -- im[ ax ];
    for( int l = 0; l < 2; ++ l )
    {
        const int c = h.ax[ 1 + l ], cp = h.ax[ 2 - l ];
        if( im[ cp ] >= n[ cp ] )
            continue;
        const double ds = g.sfc[ c ];
        double bsum = 0, s = 0;
        for( int k = 0; k < 2; ++ k )
        {
            bsum += ds * * mh_bf( a, step, h.host, c, im );
            s += ds;
            ++ im[ cp ];
            bsum += ds * * mh_bf( a, step, h.host, c, im );
            s += ds;
            -- im[ cp ];
            ++ im[ ax ];
        }
        im[ ax ] -= 2;
        * mh_bf( a, step, h.guest, c, ib ) = s > 0 ? bsum / s : 0.;
    }
}

// coarser host -> finer guest (MHD comm_functions.h:467-691 to_finer), one
// row (c1, c2) of the reference's dispatch per call: the primitives of one
// coarser cell (rows include the last CTA's second pass), or the face B of
// one coarser cell's fine ghost faces.
template< class R > __device__ __forceinline__
void mh_prolong_w( const args_t< R > & a, const mh_t & h, int c1, int c2 )
{
    const int ax = h.ax[ 0 ], a1 = h.ax[ 1 ], a2 = h.ax[ 2 ];
    int i0[ 3 ], im[ 3 ], ib[ 3 ];
    i0[ ax ] = 0; i0[ a1 ] = c1; i0[ a2 ] = c2;
    for( int d = 0; d < 3; ++ d )
    {
        ib[ d ] = h.oc[ d ] + 2 * i0[ d ];
        im[ d ] = h.os[ d ] + i0[ d ];
    }
    double qc[ 8 ], dq[ 3 ][ 8 ];
    im[ ax ] = h.os[ ax ];
    for( int c = 0; c < 8; ++ c )
        qc[ c ] = double( * mh_w( a, h.host, c, im ) );
    for( int q = 0; q < 3; ++ q )
    {
        const int aq = h.ax[ q ];
        ++ im[ aq ];
        double qr[ 8 ];
        for( int c = 0; c < 8; ++ c )
            qr[ c ] = double( * mh_w( a, h.host, c, im ) );
        im[ aq ] -= 2;
        for( int c = 0; c < 8; ++ c )
            dq[ aq ][ c ] = mh_minmod( qr[ c ] - qc[ c ], qc[ c ] - double( * mh_w( a, h.host, c, im ) ) ) * 0.25f;
        ++ im[ aq ];
    }
    for( int k = 0; k < MH_ORD; ++ k )
    {
        ib[ ax ] = h.oc[ ax ] + k;
        for( int d1 = 0; d1 < 2; ++ d1 )
        for( int d2 = 0; d2 < 2; ++ d2 )
        {
            ib[ a1 ] += d1;
            ib[ a2 ] += d2;
            if( h.mode == 0 || ( mh_in_band( ib[ a1 ], h.oc[ a1 ] ) && mh_in_band( ib[ a2 ], h.oc[ a2 ] ) ) )
            {
                for( int c = 0; c < 8; ++ c )
                    * mh_w( a, h.guest, c, ib ) = R( qc[ c ] + dq[ ax ][ c ] * ( 2 * ( k & 1 ) - 1 )
                                                    + dq[ a1 ][ c ] * ( 2 * d1 - 1 )
                                                    + dq[ a2 ][ c ] * ( 2 * d2 - 1 ) );
                mh_cell_e( a, h.guest, ib );
            }
            ib[ a1 ] -= d1;
            ib[ a2 ] -= d2;
        }
    }
}

template< class R > __device__ __forceinline__
void mh_prolong_b( const args_t< R > & a, const mh_t & h, int step, int c1, int c2, const int * n )
{
    const int ax = h.ax[ 0 ], a1 = h.ax[ 1 ], a2 = h.ax[ 2 ];
    int i0[ 3 ], im[ 3 ], ib[ 3 ];
    i0[ ax ] = 0; i0[ a1 ] = c1; i0[ a2 ] = c2;
    for( int d = 0; d < 3; ++ d )
    {
        ib[ d ] = 2 * i0[ d ] + h.obc[ d ];
        im[ d ] = i0[ d ] + h.obr[ d ];
    }
    if( ib[ a2 ] > n[ a2 ] - 2 || ib[ a1 ] > n[ a1 ] - 2 )
        return;
    ib[ ax ] = h.rhs ? -1 : n[ ax ];
    im[ ax ] = h.rhs ? n[ ax ] - 1 : 0;
    double bb[ 3 ][ 3 ][ 2 ][ 2 ], db2[ 3 ], db3[ 3 ];
    for( int c = 0; c < 3; ++ c )
    {
        const int cp[ 2 ] = { mod3( c + 1 ), mod3( c + 2 ) };
        for( int d = 0; d < 2; ++ d )
        {
            im[ c ] += d;
            const double bc = * mh_bf( a, step, h.host, c, im );
            double db1[ 2 ];
            for( int q = 0; q < 2; ++ q )
            {
                im[ cp[ q ] ] -= 1;
                const double bl = * mh_bf( a, step, h.host, c, im );
                im[ cp[ q ] ] += 2;
                const double br = * mh_bf( a, step, h.host, c, im );
                im[ cp[ q ] ] -= 1;
                db1[ q ] = mh_minmod( br - bc, bc - bl ) / 4;
            }
            bb[ c ][ 2 * d ][ 0 ][ 0 ] = bc - db1[ 0 ] - db1[ 1 ];
            bb[ c ][ 2 * d ][ 0 ][ 1 ] = bc - db1[ 0 ] + db1[ 1 ];
            bb[ c ][ 2 * d ][ 1 ][ 0 ] = bc + db1[ 0 ] - db1[ 1 ];
            bb[ c ][ 2 * d ][ 1 ][ 1 ] = bc + db1[ 0 ] + db1[ 1 ];
            im[ c ] -= d;
        }
    }
    for( int c = 0; c < 3; ++ c )
    {
        const int c1 = mod3( c + 1 ), c2 = mod3( c + 2 );
        db2[ c ] = 0;
        for( int l = 0; l < 2; ++ l )
            for( int q = 0; q < 2; ++ q )   // only the second term is divided by 8, as in the reference
                db2[ c ] += ( 2 * q - 1 ) * ( bb[ c1 ][ 2 ][ l ][ q ] - bb[ c1 ][ 0 ][ l ][ q ] )
                          + ( 2 * l - 1 ) * ( bb[ c2 ][ 2 ][ l ][ q ] - bb[ c2 ][ 0 ][ l ][ q ] ) / 8;
        db3[ c ] = 0;
        for( int k = 0; k < 2; ++ k )
            for( int l = 0; l < 2; ++ l )
                for( int q = 0; q < 2; ++ q )
                    db3[ c ] += ( 2 * k - 1 ) / 16.f * ( 2 * l - 1 ) * ( 2 * q - 1 ) * bb[ c ][ 2 * k ][ l ][ q ];
    }
    for( int c = 0; c < 3; ++ c )
    {
        const int c1 = mod3( c + 1 ), c2 = mod3( c + 2 );
        for( int l = 0; l < 2; ++ l )
            for( int q = 0; q < 2; ++ q )
                bb[ c ][ 1 ][ l ][ q ] = db2[ c ] + ( bb[ c ][ 2 ][ l ][ q ] + bb[ c ][ 0 ][ l ][ q ] ) / 2
                                       + db3[ c1 ] * ( 2 * l - 1 ) + db3[ c2 ] * ( 2 * q - 1 );
    }
    const int l_max = ( ib[ a1 ] == n[ a1 ] - 2 ) + 2;
    const int q_max = ( ib[ a2 ] == n[ a2 ] - 2 ) + 2;
    for( int l = 0; l < l_max; ++ l )
        for( int q = 0; q < q_max; ++ q )
        {
            ib[ a1 ] += l;
            ib[ a2 ] += q;
            if( q < 2 )
                * mh_bf( a, step, h.guest, a1, ib ) = bb[ a1 ][ l ][ q ][ h.rhs ];
            if( l < 2 )
                * mh_bf( a, step, h.guest, a2, ib ) = bb[ a2 ][ q ][ h.rhs ][ l ];
            ib[ a1 ] -= l;
            ib[ a2 ] -= q;
        }
}

// edge-E correction of a finer host's face holder (comm_functions.h:818-884;
// its flux average is k_flux_avg's) or edge holder (918-954)
template< class R > __device__ __forceinline__
void mh_edge_e( const args_t< R > & a, const mh_t & h, int bx, int by, int tx, const int * n )
{
    const int ax = h.ax[ 0 ], a1 = h.ax[ 1 ];
    const geo_t & g = a.geo[ h.host ];
    int i0[ 3 ], im[ 3 ], ib[ 3 ];
    mh_dispatch( h, h.fth, bx, by, tx, i0 );
    if( h.mode == 1 )
    {
        if( i0[ a1 ] >= n[ a1 ] / 2 )
            return;
        for( int d = 0; d < 3; ++ d )
        {
            im[ d ] = h.oes[ d ] + 2 * i0[ d ];
            ib[ d ] = h.oec[ d ] + i0[ d ];
        }
        R * el = mh_ee( a, h.host, a1, im );
        const double dl = g.dx[ a1 ];
        double et = double( * el ) * dl;
        ++ im[ a1 ];
        R * er = mh_ee( a, h.host, a1, im );
        et += double( * er ) * dl;
        const R ea = R( et / ( dl + dl ) );
        * mh_ee( a, h.guest, a1, ib ) = ea;
        * el = ea;
        * er = ea;
        return;
    }
    for( int d = 0; d < 3; ++ d )
    {
        im[ d ] = 2 * i0[ d ] + h.oes[ d ];
        ib[ d ] = i0[ d ] + h.oec[ d ];
    }
    const int jmax = ( bx == h.fbx - 1 ) + 1;
    const int ib_max = n[ a1 ] / 2 + ( h.oec[ a1 ] > 1 );
    for( int j = 0; j < jmax && i0[ a1 ] < ib_max; ++ j )
    {
        im[ a1 ] = 2 * i0[ a1 ] + h.oes[ a1 ];
        for( int q = 0; q < 3; ++ q )
        {
            const int am = h.ax[ mod3( ax + q ) ];
            if( am == ax )
                continue;
            const double dl = g.dx[ am ];
            R * em = mh_ee( a, h.host, am, im );
            const double e_l = double( * em ) * dl;
            ++ im[ am ];
            R * ep = mh_ee( a, h.host, am, im );
            const double e_r = double( * ep ) * dl;
            -- im[ am ];
            const R av = R( ( e_l + e_r ) / ( dl + dl ) );
            * mh_ee( a, h.guest, am, ib ) = av;
            * em = av;
            * ep = av;
        }
        ib[ a1 ] += h.fth;
        i0[ a1 ] += h.fth;
    }
}

// One phase: one thread per work item (holder, item).  For restrictions and
// prolongations an item is one row (ax[ 1 ], ax[ 2 ]) of the reference's
// dispatch, the rows of its CTAs' second passes included; for the edge-E
// correction one (CTA row, CTA, thread) triple of its launch.
template< class R, int KIND >
__global__ void __launch_bounds__( 256 ) k_mh( const args_t< R > a, const mh_t * list, const uint2 * work, int n_work,
                                              int step )
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if( t >= n_work )
        return;
    const uint2 wk = work[ t ];
    const mh_t & h = list[ wk.x ];
    const int n[ 3 ] = { a.n0, a.n1, a.n2 };
    int it = int( wk.y );
    if constexpr( KIND == MH_FLUX )
    {
        const int tx = it % h.fth, bx = ( it / h.fth ) % h.fbx, by = it / ( h.fth * h.fbx );
        mh_edge_e( a, h, bx, by, tx, n );
        return;
    }
    // a row (c1, c2): the primitives' rows first, then the face B's, each
    // with x fastest where x is one of the two dispatch axes
    const bool w = it < h.rw[ 0 ] * h.rw[ 1 ];
    if( ! w )
        it -= h.rw[ 0 ] * h.rw[ 1 ];
    const int * e = w ? h.rw : h.rb;
    const bool x2 = h.ax[ 2 ] == 0;
    const int c1 = x2 ? it / e[ 1 ] : it % e[ 0 ], c2 = x2 ? it % e[ 1 ] : it / e[ 0 ];
    if constexpr( KIND == MH_RESTRICT )
    {
        if( w ) mh_restrict_w( a, h, c1, c2 );
        else    mh_restrict_b( a, h, step, c1, c2, n );
    }
    if constexpr( KIND == MH_PROLONG )
    {
        if( w ) mh_prolong_w( a, h, c1, c2 );
        else    mh_prolong_b( a, h, step, c1, c2, n );
    }
}

////////////////////////////////////////////////////////////
// Host: the holders of a refined MHD mesh

// region.h:110-145 neighbor_t: flags of g (level lg) seen from h (level lh)
static void mh_flags( const int * h, int lh, const int * g, int lg, int * x )
{
    const int d = lg - lh;
    for( int k = 0; k < 3; ++ k )
    {
        const int base = d >= 0 ? h[ k ] * ( 1 << d ) : ( h[ k ] >> -d );
        x[ k ] = g[ k ] - base;
        if( x[ k ] > 0 && d <= 0 )
            x[ k ] *= 2;
    }
}

static int mh_grid_th( int n1 ) { return n1 < MH_TH ? n1 : MH_TH; }

// boundary.cpp:33-60 set_geo (axis, rhs), mhd/boundary/comm_functions.h:58-122
// set_geo (offsets, one rank) and 323-429 resource_pack / resource_flux /
// resource_edge (grids)
static mh_t mh_make( int host, int guest, int d_lvl, const int * x, const int * xr, const int * n )
{
    mh_t h;
    std::memset( & h, 0, sizeof( h ) );
    h.host = host; h.guest = guest; h.d_lvl = d_lvl;
    h.dir = 0;
    for( int k = 2; k >= 0; -- k )           // flags -1 | 0, 1 | 2: below, beside, above
        h.dir = 3 * h.dir + ( x[ k ] < 0 ? 0 : ( x[ k ] > 1 ? 2 : 1 ) );
    h.mode = -1;
    for( int k = 0; k < 3; ++ k )
        h.mode += x[ k ] != 0 && x[ k ] != 1;
    for( int k = 0; k < 3; ++ k )
    {
        h.ax[ k ] = 0;
        const bool out = x[ k ] < 0 || x[ k ] > 1;
        if( ( h.mode != 0 ) != out )
        {
            h.rhs = x[ k ] > 0;
            for( int q = 0; q < 3; ++ q )
                h.ax[ ( h.mode + q ) % 3 ] = ( k + q ) % 3;
            break;
        }
        else if( h.mode == 2 )
            h.ax[ k ] = k;
    }
    const int ax = h.ax[ 0 ], a1 = h.ax[ 1 ], a2 = h.ax[ 2 ];
    const int sh = d_lvl == 0 ? MH_ORD : ( d_lvl > 0 ? MH_ORD >> 1 : MH_ORD << 1 );   // shift(ord, -d_lvl)
    for( int k = 0; k < 3; ++ k )
    {
        const int n2 = n[ k ] / 2, xp = std::max( x[ k ], 0 ), rp = std::max( xr[ k ], 0 );
        h.oes[ k ] = xp * n2; h.oec[ k ] = rp * n2;
        h.obs[ k ] = xp * n2; h.obc[ k ] = rp * n2; h.obr[ k ] = xp * n2;
        h.os[ k ] = xp * n2 - sh * ( x[ k ] > 0 );
        h.oc[ k ] = rp * n2 - MH_ORD * ( x[ k ] > 0 );
    }
    h.obs[ ax ] -= x [ ax ] > 1;
    h.obr[ ax ] -= xr[ ax ] > 1;
    h.obc[ ax ] -= x [ ax ] > 1;
    if( h.mode == 1 )
    {
        h.os[ a1 ] = x [ a1 ] * ( n[ a1 ] / 2 );
        h.oc[ a1 ] = xr[ a1 ] * ( n[ a1 ] / 2 );
    }
    // exchange grid (resource_pack)
    int nc[ 3 ] = { n[ 0 ], n[ 1 ], n[ 2 ] };
    if( d_lvl >= 0 )
    {
        if( h.mode > 0 ) nc[ a2 ] = MH_ORD;
        if( h.mode > 1 ) nc[ a1 ] = MH_ORD;
    }
    for( int k = 0; k < 3; ++ k )
        nc[ k ] /= 1 + ( d_lvl != 0 );
    if( d_lvl < 0 && h.mode > 0 )
    {
        nc[ a2 ] = MH_NGH;
        if( h.mode > 1 ) nc[ a1 ] = MH_NGH;
    }
    h.n1 = nc[ a1 ];
    h.nth = mh_grid_th( nc[ a1 ] );
    h.nbx = ( h.nth - 1 + nc[ a1 ] ) / h.nth;
    h.nby = nc[ a2 ];
    if( h.mode == 0 )
        h.nby += d_lvl > 0 ? MH_NGH / 2 : ( d_lvl < 0 ? xr[ a2 ] > 0 : 1 );
    // restriction / prolongation rows (ax[ 1 ], ax[ 2 ]) that the reference's
    // guards admit: first passes [ 0, nbx nth ), the last CTA's second pass
    // up to ( nbx + 1 ) nth
    const int first = h.nbx * h.nth, second = ( h.nbx + 1 ) * h.nth;
    if( d_lvl < 0 )
    {
        const int lim2 = h.mode > 0 ? MH_NGH : n[ a2 ] / 2;
        const int lim1 = h.mode > 1 ? MH_NGH : n[ a1 ] / 2;
        h.rw[ 0 ] = std::min( lim1, first );
        h.rw[ 1 ] = std::min( lim2, h.nby );
        if( h.mode == 0 )
        {
            h.rb[ 0 ] = std::min( n[ a1 ] / 2 + ( h.obc[ a1 ] > 1 ), second );
            h.rb[ 1 ] = h.nby;
        }
    }
    else if( d_lvl > 0 )
    {
        const int im_max = ( h.mode > 0 && h.oc[ a1 ] != 0 ) ? 1 : ( n[ a1 ] + MH_ORD ) / 2;
        h.rw[ 0 ] = std::min( im_max, second );
        h.rw[ 1 ] = h.nby;
        if( h.mode == 0 )
        {
            h.rb[ 0 ] = first;
            h.rb[ 1 ] = h.nby;
        }
    }
    // edge-E grid: resource_flux (face holders), resource_edge (edge holders)
    if( h.mode == 0 )
    {
        h.fth = mh_grid_th( n[ a1 ] / 2 );
        h.fbx = ( h.fth - 1 + n[ a1 ] / 2 ) / h.fth;
        h.fby = n[ a2 ] / 2 + ( xr[ a2 ] > 0 );
    }
    else
    {
        h.fth = mh_grid_th( n[ a1 ] / 2 );
        h.fbx = ( h.fth - 1 + n[ a1 ] / 2 ) / h.fth;
        h.fby = 1;
    }
    return h;
}

// tree.cpp:176-197 neighbors, for every leaf in the reference's host order
static std::vector< mh_t > mh_holders( const kr_tree & t, const int * n )
{
    // leaf index by (level, position)
    std::vector< std::vector< int > > leaf( t.max_level + 1 );
    for( int l = 0; l <= t.max_level; ++ l )
        leaf[ l ].assign( size_t( kr_tree_lim( & t, l, 0 ) * kr_tree_lim( & t, l, 1 ) * kr_tree_lim( & t, l, 2 ) ), -1 );
    for( int b = 0; b < t.nblk; ++ b )
        leaf[ t.level[ b ] ][ size_t( kr_tree_idx( & t, t.level[ b ], t.reg + 3 * b ) ) ] = b;
    auto leaf_at = [ & ]( int l, const int * r ) -> int
    {
        return l <= t.max_level ? leaf[ l ][ size_t( kr_tree_idx( & t, l, r ) ) ] : -1;
    };
    std::vector< int > order( t.nblk );
    for( int b = 0; b < t.nblk; ++ b )
        order[ b ] = b;
    std::sort( order.begin(  ), order.end(  ), [ & ]( int p, int q )
    {
        if( t.level[ p ] != t.level[ q ] )
            return t.level[ p ] < t.level[ q ];
        for( int k = 0; k < 3; ++ k )
            if( t.reg[ 3 * p + k ] != t.reg[ 3 * q + k ] )
                return t.reg[ 3 * p + k ] < t.reg[ 3 * q + k ];
        return false;
    } );
    std::vector< mh_t > out;
    for( int b : order )
    {
        const int l = t.level[ b ];
        const int * r = t.reg + 3 * b;
        struct nb_t { int x[ 3 ], xr[ 3 ], g, d; };
        std::vector< nb_t > nbs;
        int di[ 3 ];
        for( di[ 0 ] = -1; di[ 0 ] < 3; ++ di[ 0 ] )
        for( di[ 1 ] = -1; di[ 1 ] < 3; ++ di[ 1 ] )
        for( di[ 2 ] = -1; di[ 2 ] < 3; ++ di[ 2 ] )
        {
            if( di[ 0 ] >= 0 && di[ 0 ] <= 1 && di[ 1 ] >= 0 && di[ 1 ] <= 1 && di[ 2 ] >= 0 && di[ 2 ] <= 1 )
                continue;
            int s[ 3 ], s0[ 3 ];
            for( int k = 0; k < 3; ++ k )
                s[ k ] = s0[ k ] = 2 * r[ k ] + di[ k ];
            if( ! kr_tree_regularize( & t, l + 1, s ) )
                continue;
            for( int lt = l + 1; lt >= std::max( l - 1, 0 ); -- lt )
            {
                const int g = leaf_at( lt, s );
                if( g >= 0 )
                {
                    nb_t v;
                    mh_flags( r, l, s0, lt, v.x );
                    mh_flags( s0, lt, r, l, v.xr );
                    v.g = g;
                    v.d = lt - l;
                    bool dup = false;
                    for( const nb_t & o : nbs )
                        dup |= o.x[ 0 ] == v.x[ 0 ] && o.x[ 1 ] == v.x[ 1 ] && o.x[ 2 ] == v.x[ 2 ];
                    if( ! dup )
                        nbs.push_back( v );
                    break;
                }
                for( int k = 0; k < 3; ++ k )   // region.h:61-69 coarsen
                {
                    s [ k ] = ( s [ k ] > 0 ? s [ k ] : s [ k ] - 1 ) / 2;
                    s0[ k ] = ( s0[ k ] > 0 ? s0[ k ] : s0[ k ] - 1 ) / 2;
                }
            }
        }
        std::sort( nbs.begin(  ), nbs.end(  ), []( const nb_t & p, const nb_t & q )
        {
            for( int k = 0; k < 3; ++ k )
                if( p.x[ k ] != q.x[ k ] )
                    return p.x[ k ] < q.x[ k ];
            return false;
        } );
        for( const nb_t & v : nbs )
            out.push_back( mh_make( b, v.g, v.d, v.x, v.xr, n ) );
    }
    return out;
}

// The edges (block, component, index) that a finer host's edge-E correction
// reads or writes, as 64-bit keys (the index arithmetic of mh_edge_e).
static void mh_edge_keys( const mh_t & h, const int * n, std::vector< unsigned long long > & keys )
{
    auto key = [ & ]( int b, int c, const int * i )
    {
        return ( ( ( unsigned long long ) b * 3 + c ) << 33 )
             | ( ( unsigned long long )( i[ 0 ] + 1 ) << 22 ) | ( ( unsigned long long )( i[ 1 ] + 1 ) << 11 )
             | ( unsigned long long )( i[ 2 ] + 1 );
    };
    keys.clear(  );
    const int ax = h.ax[ 0 ], a1 = h.ax[ 1 ];
    for( int by = 0; by < h.fby; ++ by )
    for( int bx = 0; bx < h.fbx; ++ bx )
    for( int tx = 0; tx < h.fth; ++ tx )
    {
        int i0[ 3 ], im[ 3 ], ib[ 3 ];
        i0[ ax ] = 0; i0[ a1 ] = bx * h.fth + tx; i0[ h.ax[ 2 ] ] = by;
        if( h.mode == 1 )
        {
            if( i0[ a1 ] >= n[ a1 ] / 2 )
                continue;
            for( int d = 0; d < 3; ++ d ) { im[ d ] = h.oes[ d ] + 2 * i0[ d ]; ib[ d ] = h.oec[ d ] + i0[ d ]; }
            keys.push_back( key( h.guest, a1, ib ) );
            keys.push_back( key( h.host, a1, im ) );
            ++ im[ a1 ];
            keys.push_back( key( h.host, a1, im ) );
            continue;
        }
        for( int d = 0; d < 3; ++ d ) { im[ d ] = 2 * i0[ d ] + h.oes[ d ]; ib[ d ] = i0[ d ] + h.oec[ d ]; }
        const int jmax = ( bx == h.fbx - 1 ) + 1;
        const int ib_max = n[ a1 ] / 2 + ( h.oec[ a1 ] > 1 );
        for( int j = 0; j < jmax && i0[ a1 ] < ib_max; ++ j )
        {
            im[ a1 ] = 2 * i0[ a1 ] + h.oes[ a1 ];
            for( int q = 0; q < 3; ++ q )
            {
                const int am = h.ax[ ( ax + q ) % 3 ];
                if( am == ax )
                    continue;
                keys.push_back( key( h.guest, am, ib ) );
                keys.push_back( key( h.host, am, im ) );
                ++ im[ am ];
                keys.push_back( key( h.host, am, im ) );
                -- im[ am ];
            }
            ib[ a1 ] += h.fth;
            i0[ a1 ] += h.fth;
        }
    }
}

// The launch lists of a refined MHD mesh: copies, restrictions, the
// prolongations grouped by the coarser host's level, and the edge-E
// correction's waves (a holder runs after every earlier holder that touches
// one of its edges).  Every segment of holders is also flattened into work
// items (holder, item) for one thread each.
struct mh_plan_t
{
    std::vector< mh_t > list;
    std::vector< uint2 > work;
    std::vector< int > same_nbr;         // (block, direction 0..26, neighbour) of same-level holders
    int restrict_[ 2 ] = { 0, 0 };       // work-item range
    std::vector< int > prolong;          // [levels + 1] work offsets
    std::vector< int > waves;            // [waves + 1] work offsets
};

static mh_plan_t mh_plan( const kr_tree & t, const int * n )
{
    const std::vector< mh_t > hs = mh_holders( t, n );
    mh_plan_t p;
    auto add = [ & ]( const mh_t & h, bool flux )
    {
        const unsigned idx = unsigned( p.list.size(  ) );
        p.list.push_back( h );
        const int items = flux ? h.fbx * h.fby * h.fth : h.rw[ 0 ] * h.rw[ 1 ] + h.rb[ 0 ] * h.rb[ 1 ];
        for( int k = 0; k < items; ++ k )
            p.work.push_back( make_uint2( idx, unsigned( k ) ) );
    };
    auto phase = [ & ]( auto pred, bool flux )
    {
        for( const mh_t & h : hs )
            if( pred( h ) )
                add( h, flux );
        return int( p.work.size(  ) );
    };
    // same level: the push of the uniform step (k_c2p, the CT update) through
    // the neighbour table, direction ( x + 1 ) + 3 ( y + 1 ) + 9 ( z + 1 ) with
    // flags 2 taken as +1; its copies are the ones to_same makes
    for( const mh_t & h : hs )
        if( h.d_lvl == 0 )
            p.same_nbr.insert( p.same_nbr.end(  ), { h.host, h.dir, h.guest } );
    p.restrict_[ 0 ] = 0;
    p.restrict_[ 1 ] = phase( []( const mh_t & h ) { return h.d_lvl < 0; }, false );
    p.prolong.push_back( p.restrict_[ 1 ] );
    for( int l = 0; l < t.max_level; ++ l )
        p.prolong.push_back( phase( [ & ]( const mh_t & h ) { return h.d_lvl > 0 && t.level[ h.host ] == l; }, false ) );
    // edge-E waves, in holder order
    std::vector< const mh_t * > fx;
    for( const mh_t & h : hs )
        if( h.d_lvl < 0 && h.mode < 2 )
            fx.push_back( & h );
    std::vector< int > wave( fx.size(  ), 0 );
    std::unordered_map< unsigned long long, int > last;
    std::vector< unsigned long long > keys;
    int n_wave = 0;
    for( size_t q = 0; q < fx.size(  ); ++ q )
    {
        mh_edge_keys( * fx[ q ], n, keys );
        int w = 0;
        for( unsigned long long k : keys )
        {
            auto it = last.find( k );
            if( it != last.end(  ) )
                w = std::max( w, it->second + 1 );
        }
        wave[ q ] = w;
        for( unsigned long long k : keys )
            last[ k ] = w;
        n_wave = std::max( n_wave, w + 1 );
    }
    p.waves.push_back( int( p.work.size(  ) ) );
    for( int w = 0; w < n_wave; ++ w )
    {
        for( size_t q = 0; q < fx.size(  ); ++ q )
            if( wave[ q ] == w )
                add( * fx[ q ], true );
        p.waves.push_back( int( p.work.size(  ) ) );
    }
    return p;
}
