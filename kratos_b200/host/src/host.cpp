// kratos_b200 host layer: parameter files, problem-generator entry, the
// default initial conditions of the dynamics modules, the mesh / time loop on
// top of the B200 engine, and the binary snapshot writer.
#include <array>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <iomanip>
#include <iostream>
#include <map>
#include <set>
#include <stdexcept>

#include "../../../include/kratos_b200.h"
#include "mesh/mesh.h"
#include "modules/dynamics/hydro/hydro.h"
#include "modules/dynamics/mhd/mhd.h"
#include "user/probgen.h"
#include "utilities/mapping/loop.h"

////////////////////////////////////////////////////////////
// Parameter files (input.cpp:70-150 of the reference)

bool input::read_text( std::istream & in )
{
    std::string line, pre;
    while( std::getline( in, line ) )
    {
        const auto hash = line.find( '#' );
        if( hash != std::string::npos )
            line = line.substr( 0, hash );
        line = trim( line );
        if( line.empty(  ) )
            continue;
        if( line[ 0 ] == '[' )
        {
            const auto e = line.find( ']' );
            if( e == std::string::npos )
                throw std::runtime_error( "input: incorrect section line: " + line );
            pre = line.substr( 1, e - 1 );
            prefixes_.insert( pre );
            continue;
        }
        const auto eq = line.find( '=' );
        const std::string k = trim( line.substr( 0, eq ) );
        std::string v = eq == std::string::npos ? "" : line.substr( eq + 1 );
        const auto eq2 = v.find( '=' );              // text after a second '=' is dropped
        if( eq2 != std::string::npos )
            v = v.substr( 0, eq2 );
        items_[ key( pre, k ) ] = trim( v );
    }
    return true;
}

namespace
{
// Binary snapshot: header (binary_io_base.cpp:101-118) + entries.
struct snap_entry { char u_size; std::vector< char > bytes; };

void put_size( std::vector< char > & o, size_t v )
{
    const char * p = reinterpret_cast< const char * >( & v );
    o.insert( o.end(  ), p, p + sizeof( v ) );
}
void put_str( std::vector< char > & o, const std::string & s )
{
    put_size( o, s.size(  ) );
    o.insert( o.end(  ), s.begin(  ), s.end(  ) );
}

// Global block ids in the reference's order: blocks along a Hilbert curve
// (meshgen.cpp:188-243 dist_fractal) drawn by an L-system turtle
// (utilities/l_system/l_system.cpp): the 3-D rule below, 'F' one unit step
// along the turtle's x axis, the other symbols quarter turns composed on the
// right (+ - about z, & ^ about y, > < about x), kept here as integer rotation
// matrices; a refined node is replaced by its children in the order of the same
// curve one level down, placed where that curve's bounding box meets the
// node's children.  lvl[b], reg[3b..3b+2]: each block's level and position.
struct hilbert_walk
{
    const char * rule = "^<XF^<XFX-F^>>XFX&F+>>XFX-F>X->";
    std::map< std::array< int, 4 >, int > leaf;      // (level, x) -> block
    std::set< std::array< int, 4 > > refined;
    std::vector< int > ids;
    std::vector< std::array< int, 3 > > nodes;
    int l_base = 1, lim = 1, next = 0;
    bool dry = false;
    struct turtle { int l; int x[ 3 ]; int m[ 3 ][ 3 ]; };

    static void turn( int m[ 3 ][ 3 ], char c )
    {   // m = m * R, R the quarter turn of c
        const int axis = ( c == '+' || c == '-' ) ? 2 : ( ( c == '&' || c == '^' ) ? 1 : 0 );
        const int sgn = ( c == '+' || c == '&' || c == '>' ) ? 1 : -1;
        const int a1 = ( axis + 1 ) % 3, a2 = ( axis + 2 ) % 3;
        int r[ 3 ][ 3 ] = { { 0, 0, 0 }, { 0, 0, 0 }, { 0, 0, 0 } };
        r[ axis ][ axis ] = 1;
        r[ a2 ][ a1 ] = sgn;
        r[ a1 ][ a2 ] = -sgn;
        int o[ 3 ][ 3 ];
        for( int i = 0; i < 3; ++ i )
            for( int j = 0; j < 3; ++ j )
            {
                o[ i ][ j ] = 0;
                for( int k = 0; k < 3; ++ k )
                    o[ i ][ j ] += m[ i ][ k ] * r[ k ][ j ];
            }
        std::memcpy( m, o, sizeof( o ) );
    }
    bool visit( const turtle & t )
    {   // true: a refined node, walked one level down instead
        const std::array< int, 4 > key = { t.l - l_base, t.x[ 0 ], t.x[ 1 ], t.x[ 2 ] };
        if( refined.count( key ) )
            return true;
        const auto it = leaf.find( key );
        if( it != leaf.end(  ) )
            ids[ it->second ] = next ++;
        return false;
    }
    void step( turtle & t )
    {
        if( t.l >= lim )
            return node( t );
        for( const char * c = rule; * c; ++ c )
            if( * c == 'X' )
            {
                ++ t.l;
                step( t );
                -- t.l;
            }
            else if( * c == 'F' )
                for( int a = 0; a < 3; ++ a )
                    t.x[ a ] += t.m[ a ][ 0 ];
            else
                turn( t.m, * c );
    }
    void node( const turtle & t )
    {
        if( dry || ! visit( t ) )
        {
            nodes.push_back( { t.x[ 0 ], t.x[ 1 ], t.x[ 2 ] } );
            return;
        }
        const size_t start = nodes.size(  );
        dry = true;
        ++ lim;
        turtle m = t;
        m.x[ 0 ] = m.x[ 1 ] = m.x[ 2 ] = 0;
        step( m );
        int dx[ 3 ] = { 0, 0, 0 };
        for( size_t k = start; k < nodes.size(  ); ++ k )
            for( int a = 0; a < 3; ++ a )
                dx[ a ] = std::min( dx[ a ], nodes[ k ][ a ] );
        nodes.resize( start );
        m = t;
        for( int a = 0; a < 3; ++ a )
            m.x[ a ] = 2 * t.x[ a ] - dx[ a ];
        dry = false;
        step( m );
        -- lim;
    }
};

std::vector< int > hilbert_ids( const std::vector< int > & lvl, const std::vector< int > & reg, const int * nb )
{
    hilbert_walk h;
    const size_t nblk = lvl.size(  );
    h.ids.assign( nblk, -1 );
    for( size_t b = 0; b < nblk; ++ b )
    {
        int x[ 3 ] = { reg[ 3 * b ], reg[ 3 * b + 1 ], reg[ 3 * b + 2 ] };
        h.leaf[ { lvl[ b ], x[ 0 ], x[ 1 ], x[ 2 ] } ] = int( b );
        for( int l = lvl[ b ]; l > 0; -- l )
        {   // every ancestor is a refined node (region.h:60-66 coarsen)
            for( int a = 0; a < 3; ++ a )
                x[ a ] = ( x[ a ] > 0 ? x[ a ] : x[ a ] - 1 ) / 2;
            h.refined.insert( { l - 1, x[ 0 ], x[ 1 ], x[ 2 ] } );
        }
    }
    int n_base = std::max( nb[ 0 ], std::max( nb[ 1 ], nb[ 2 ] ) ) - 1, l_base = 0;
    while( n_base >>= 1 )
        ++ l_base;
    h.l_base = h.lim = l_base + 1;
    hilbert_walk::turtle t = { 0, { 0, 0, 0 }, { { 1, 0, 0 }, { 0, 1, 0 }, { 0, 0, 1 } } };
    h.step( t );
    for( int id : h.ids )
        if( id < 0 )
            throw std::runtime_error( "block numbering: a block off the Hilbert walk" );
    return h.ids;
}

// The serialized block tree (mesh/tree/tree.cpp:11-20 write, through
// utilities/data_transfer/serialize.h): the map of nodes -- refined ones
// (mask) and leaves with their ids -- in key order (level, then x0, x1, x2),
// as size_t count and raw (region_logic_t: 3 x int + level; tree_node_t: id_l,
// id_g, rank, mask + padding) pairs, then n_dim, reg_max and the periodic
// flags.  A reference restart reads it (meshgen.cpp:96-104).
snap_entry mesh_tree_blob( const std::vector< mesh::block_t > & blocks, const int * nb,
                           const bool * periodic )
{
    std::map< std::array< int, 4 >, std::array< int, 4 > > nodes;   // key -> id_l, id_g, rank, mask
    for( const auto & b : blocks )
    {
        int x[ 3 ] = { b.reg[ 0 ], b.reg[ 1 ], b.reg[ 2 ] };
        nodes[ { b.reg.level, x[ 0 ], x[ 1 ], x[ 2 ] } ] = { b.id_g, b.id_g, 0, 0 };
        for( int l = b.reg.level; l > 0; -- l )
        {
            for( int a = 0; a < 3; ++ a )
                x[ a ] = ( x[ a ] > 0 ? x[ a ] : x[ a ] - 1 ) / 2;
            nodes[ { l - 1, x[ 0 ], x[ 1 ], x[ 2 ] } ] = { -1, -1, -1, 1 };
        }
    }
    snap_entry e;
    e.u_size = 1;
    put_size( e.bytes, nodes.size(  ) );
    auto put_i = [ & ]( int v )
    {
        const char * p = reinterpret_cast< const char * >( & v );
        e.bytes.insert( e.bytes.end(  ), p, p + 4 );
    };
    for( const auto & kv : nodes )
    {
        put_i( kv.first[ 1 ] ); put_i( kv.first[ 2 ] ); put_i( kv.first[ 3 ] ); put_i( kv.first[ 0 ] );
        put_i( kv.second[ 0 ] ); put_i( kv.second[ 1 ] ); put_i( kv.second[ 2 ] );
        const char tail[ 4 ] = { char( kv.second[ 3 ] ), 0, 0, 0 };
        e.bytes.insert( e.bytes.end(  ), tail, tail + 4 );
    }
    put_i( 3 );
    for( int a = 0; a < 3; ++ a )
        put_i( nb[ a ] );
    for( int a = 0; a < 3; ++ a )
        e.bytes.push_back( char( periodic[ a ] ? 1 : 0 ) );
    return e;
}

// Whole-file snapshot reader: tag -> bytes of its blob.
struct snap_file
{
    std::map< std::string, snap_entry > e;

    bool load( const std::string & file )
    {
        std::ifstream f( file, std::ios::binary );
        if( ! f ) return false;
        std::vector< char > raw( ( std::istreambuf_iterator< char >( f ) ),
                                 std::istreambuf_iterator< char >(  ) );
        if( raw.size(  ) < 17 || ( raw[ 0 ] & 0x7e ) != 8 )
            return false;
        size_t hdr, n, pos = 17;
        std::memcpy( & hdr, & raw[ 1 ], 8 );
        std::memcpy( & n, & raw[ 9 ], 8 );
        for( size_t k = 0; k < n; ++ k )
        {
            size_t kl, size, off;
            std::memcpy( & kl, & raw[ pos ], 8 ); pos += 8;
            const std::string tag( & raw[ pos ], kl ); pos += kl;
            std::memcpy( & size, & raw[ pos ], 8 ); pos += 8;
            snap_entry x;
            x.u_size = raw[ pos ]; pos += 1;
            std::memcpy( & off, & raw[ pos ], 8 ); pos += 8;
            if( hdr + off + size > raw.size(  ) )
                throw std::runtime_error( "snapshot truncated at " + tag );
            x.bytes.assign( raw.begin(  ) + hdr + off, raw.begin(  ) + hdr + off + size );
            e[ tag ] = std::move( x );
        }
        return true;
    }
    const std::vector< char > & at( const std::string & tag ) const
    {
        const auto it = e.find( tag );
        if( it == e.end(  ) )
            throw std::runtime_error( "snapshot: no entry " + tag );
        return it->second.bytes;
    }
    template< class T > void get( const std::string & tag, T * p, size_t n ) const
    {
        const auto & b = at( tag );
        if( b.size(  ) != n * sizeof( T ) )
            throw std::runtime_error( "snapshot: size mismatch at " + tag );
        std::memcpy( p, b.data(  ), b.size(  ) );
    }
    std::map< std::string, std::string > args(  ) const
    {
        std::map< std::string, std::string > items;
        const auto & b = at( "input_args" );
        size_t q = 0, cnt;
        auto size = [ & ](  ) { size_t v; std::memcpy( & v, & b[ q ], 8 ); q += 8; return v; };
        cnt = size(  );
        for( size_t i = 0; i < cnt; ++ i )
        {
            const size_t l1 = size(  );
            std::string a( & b[ q ], l1 ); q += l1;
            const size_t l2 = size(  );
            std::string v( & b[ q ], l2 ); q += l2;
            items[ a ] = v;
        }
        return items;
    }
};
}   // namespace

bool input::read(  )
{
    if( files_.empty(  ) )
        return false;
    const std::string file = files_.back(  );
    std::ifstream in( file, std::ios::binary );
    if( ! in )
    {
        std::cerr << "Unable to open input file: " << file << std::endl;
        return false;
    }
    const int c = in.peek(  );
    if( 32 <= c && c <= 126 )
    {
        std::cout << "Reading input parameters from ascii : " << file << std::endl;
        return read_text( in );
    }
    std::cout << "Reading input parameters from binary: " << file << std::endl;
    snap_file s;
    if( ! s.load( file ) )
        throw std::runtime_error( "input: unreadable snapshot " + file );
    for( const auto & p : s.args(  ) )
    {
        items_[ p.first ] = p.second;
        const auto bar = p.first.find( '|' );
        if( bar != std::string::npos )
            prefixes_.insert( p.first.substr( 0, bar ) );
    }
    set( "file", "binary", file );
    return true;
}

////////////////////////////////////////////////////////////
// Problem-generator entry (src/user/probgen.cpp of the reference)

namespace prob
{
void cmd( int argc, char * argv[  ], input & args )
{
    for( int i = 1; i < argc; ++ i )
    {
        args.set_file( argv[ i ] );
        args.read(  );
    }
}

void __attribute__( ( weak ) ) run( int, char * [  ] )
{
    std::cerr << "Default run function is empty!\n";
}
}   // namespace prob

////////////////////////////////////////////////////////////
// Default initial conditions (hydro.cpp:27-45, mhd.cpp:27-55 of the reference)

namespace dynamics
{
void hydro_t::init_cond( mesh::block::dual_t & d )
{
    auto & b_h = dynamic_cast< hydro::block_data_t & >( d.h(  ) );
    const auto & geo = d.b_w.get(  ).geo;
    for( auto i : utils::loop( geo.n_ceff ) )
    {
        double * u = b_h.hyd.u.at( i );
        u[ 0 ] = rho0;
        u[ 1 ] = pre0 / ( p_eos->gamma - 1 );
        for( int n = 0; n < 3; ++ n )
        {
            u[ 1 ] += std::pow( vel0[ n ], 2 ) * rho0 / 2;
            u[ 2 + n ] = vel0[ n ] * rho0;
        }
    }
}

void mhd_t::init_cond( mesh::block::dual_t & d )
{
    hydro_t::init_cond( d );
    auto & b_h = dynamic_cast< mhd::block_data_t & >( d.h(  ) );
    const auto & geo = d.b_w.get(  ).geo;
    auto n_face = geo.n_ceff;
    for( auto & n_s : n_face.x )
        n_s += ( n_s > 1 );
    for( auto i : utils::loop( n_face ) )
    {
        double * bf = b_h.fld.bf.at( i );
        bool is_cc = true;
        for( int a = 0; a < 3; ++ a )
        {
            bf[ a ] = b0[ a ];
            is_cc &= i[ a ] < geo.n_ceff[ a ];
        }
        if( is_cc )
        {
            double * u = b_h.hyd.u.at( i );
            for( int a = 0; a < 3; ++ a )
                u[ 1 ] += std::pow( b0[ a ], 2 ) / 2;
        }
    }
}
}   // namespace dynamics

////////////////////////////////////////////////////////////
// Mesh and time loop

namespace mesh
{
mesh_t::mesh_t(  ) {}
mesh_t::~mesh_t(  ) { if( ctx_ ) kr_ctx_destroy( ctx_ ); }

static int bc_kind( const std::string & s )
{
    if( s.find( "per" ) != std::string::npos )  return KR_BC_PER;
    if( s.find( "fixd" ) != std::string::npos ) return KR_BC_FIXD;
    if( s.find( "out" ) != std::string::npos )  return KR_BC_OUT;
    if( s.find( "ref" ) != std::string::npos )  return KR_BC_REF;
    if( s.find( "fre" ) != std::string::npos )  return KR_BC_FRE;
    throw std::runtime_error( "Undef bnd " + s );
}

void mesh_t::init( const input & args )
{
    args_ = & args;
    if( mods_.size(  ) != 1 )
        throw std::runtime_error( "mesh_t::init: enrol exactly one dynamics module" );
    auto & mod = * mods_[ 0 ];
    mod.read( args );
    mhd_ = mod.is_mhd(  );
    const auto x_lo = args.get< type::coord2_t >( "mesh", "x_min" );
    const auto x_hi = args.get< type::coord2_t >( "mesh", "x_max" );
    const auto ng = args.get< type::idx_t >( "mesh", "n_cell_global" );
    const auto nbl = args.get< type::idx_t >( "mesh", "n_cell_block", ng );
    for( int a = 0; a < 3; ++ a )
    {
        if( ng[ a ] % nbl[ a ] )
            throw std::runtime_error( "Mesh size indivisible by sub-mesh." );
        n_[ a ] = nbl[ a ];
        nb_[ a ] = ng[ a ] / nbl[ a ];
    }
    // engine configuration
    kr_cfg c;
    kr_cfg_default( & c );
    c.mhd = mhd_;
    c.precision = args.get< int >( "b200", "precision", 2 );
    c.riemann = args.get< int >( "b200", "riemann", 0 );
    {   // [b200] integrator = rk2 (the reference's Heun step) | vl2
        const std::string itg = args.get< std::string >( "b200", "integrator", "rk2" );
        if( itg != "rk2" && itg != "vl2" )
            throw std::runtime_error( "[b200] integrator must be rk2 or vl2, not " + itg );
        c.integrator = itg == "vl2" ? KR_INTEGRATOR_VL2 : KR_INTEGRATOR_RK2;
    }
    for( int a = 0; a < 3; ++ a )
    {
        c.nb[ a ] = nb_[ a ];
        c.n[ a ] = n_[ a ];
        c.x_min[ a ] = x_lo[ a ];
        c.x_max[ a ] = x_hi[ a ];
    }
    c.gamma = mod.p_eos->gamma;
    c.cfl = mod.p_eos->cfl;
    c.rho_floor = mod.p_eos->d_floor;
    c.tmp_floor = mod.p_eos->t_floor;
    c.dt_init = args.get< double >( "cycle", "dt_init", 0.0 );
    c.dt_expand = args.get< double >( "cycle", "dt_expand", 2.0 );
    c.device = args.get< int >( "device", "idx_device", 0 );
    std::vector< std::string > kinds;
    args( "boundary", "kinds", kinds );
    for( int s = 0; s < 6; ++ s )
        c.bc[ s ] = s < int( kinds.size(  ) ) ? bc_kind( kinds[ s ] ) : KR_BC_PER;
    for( int a = 0; a < 3; ++ a )
        periodic_[ a ] = c.bc[ 2 * a ] == KR_BC_PER && c.bc[ 2 * a + 1 ] == KR_BC_PER;
    c.w_fix[ 0 ] = args.get< double >( "init", "rho0", 0 );
    c.w_fix[ 1 ] = args.get< double >( "init", "pre0", 0 );
    const auto v0 = args.get< type::coord2_t >( "init", "vel0", 0 );
    for( int a = 0; a < 3; ++ a ) c.w_fix[ 2 + a ] = v0[ a ];
    const auto b0 = args.get< type::coord2_t >( "init", "b0", 0 );
    for( int a = 0; a < 3; ++ a ) c.b_fix[ a ] = b0[ a ];
    // static refinement: every [refine_region*] section (meshgen.cpp:111-137
    // load_refinement: level, loc / x_min, x_max defaulting to x_min)
    std::vector< kr_region > regions;
    for( const auto & p : args.get_prefixes(  ) )
    {
        if( p.find( "refine_region" ) == std::string::npos )
            continue;
        kr_region r;
        r.level = args.get< int >( p, "level", 0 );
        type::coord2_t lo( 0 ), hi;
        args( p, "loc", lo );
        args( p, "x_min", lo );
        hi = lo;
        args( p, "x_max", hi );
        for( int a = 0; a < 3; ++ a ) { r.x_min[ a ] = lo[ a ]; r.x_max[ a ] = hi[ a ]; }
        regions.push_back( r );
    }
    ctx_ = kr_ctx_create_refined( & c, int( regions.size(  ) ), regions.data(  ) );
    if( ! ctx_ )
        throw std::runtime_error( std::string( "kratos_b200: " ) + kr_last_error( nullptr ) );
    // blocks (the engine's: the tree's leaves, level by level) and their
    // geometry (meshgen.cpp:252-363: loc(i) = ( reg + i / n ) / ( nb << level ))
    const int nblk = kr_block_info( ctx_, nullptr, nullptr );
    std::vector< int > lvl( nblk ), regs( 3 * size_t( nblk ) );
    kr_block_info( ctx_, lvl.data(  ), regs.data(  ) );
    blocks_.assign( nblk, block_t(  ) );
    for( int b = 0; b < nblk; ++ b )
    {
        block_t & blk = blocks_[ b ];
        blk.id_l = b;
        blk.reg.level = lvl[ b ];
        double vol = 1.;
        for( int a = 0; a < 3; ++ a )
        {
            const int reg = regs[ 3 * b + a ];
            blk.reg[ a ] = reg;
            blk.geo.n_ceff[ a ] = n_[ a ];
            const double lim = double( nb_[ a ] << lvl[ b ] );
            const double l0 = x_lo[ a ] + ( reg + 0.0 / n_[ a ] ) / lim * ( x_hi[ a ] - x_lo[ a ] );
            const double l1 = x_lo[ a ] + ( reg + 1.0 / n_[ a ] ) / lim * ( x_hi[ a ] - x_lo[ a ] );
            blk.geo.xf0[ a ] = l0;
            blk.geo.dx0[ a ] = l1 - l0;
        }
        for( int a = 0; a < 3; ++ a )
        {
            double s = 1.;
            s *= blk.geo.dx0[ ( a + 1 ) % 3 ];
            s *= blk.geo.dx0[ ( a + 2 ) % 3 ];
            blk.geo.sfc0[ a ] = s;
            vol *= blk.geo.dx0[ a ];
        }
        blk.geo.vol0 = vol;
    }
    // host block data: initial conditions, or the snapshot of a restart
    std::unique_ptr< snap_file > snap;
    if( args.found( "file", "binary" ) )
    {
        snap.reset( new snap_file );
        if( ! snap->load( args.get< std::string >( "file", "binary" ) ) )
            throw std::runtime_error( "restart: unreadable snapshot" );
    }
    // Global ids as the reference assigns them (its Hilbert-curve order), so
    // that snapshots name their blocks as a reference restart looks them up
    {
        const std::vector< int > ids = hilbert_ids( lvl, regs, nb_ );
        for( int b = 0; b < nblk; ++ b )
            blocks_[ b ].id_g = ids[ b ];
    }
    // Stored blocks are matched by level and logical position (i_logic): the
    // reference numbers blocks along a Hilbert curve (meshgen.cpp:188-243),
    // this layer level by level, lexicographically.
    std::vector< std::string > snap_block( nblk );
    if( snap )
    {
        std::map< std::array< int, 4 >, int > where;
        for( int b = 0; b < nblk; ++ b )
            where[ { lvl[ b ], regs[ 3 * b ], regs[ 3 * b + 1 ], regs[ 3 * b + 2 ] } ] = b;
        const std::string suffix = "|i_logic";
        for( const auto & kv : snap->e )
        {
            const auto & tag = kv.first;
            if( tag.compare( 0, 6, "block_" ) || tag.size(  ) < suffix.size(  ) ||
                tag.compare( tag.size(  ) - suffix.size(  ), suffix.size(  ), suffix ) )
                continue;
            int il[ 3 ], lv = 0;
            const std::string pre = tag.substr( 0, tag.size(  ) - suffix.size(  ) + 1 );
            snap->get( tag, il, 3 );
            snap->get( pre + "level", & lv, 1 );
            const auto it = where.find( { lv, il[ 0 ], il[ 1 ], il[ 2 ] } );
            if( it == where.end(  ) )
                throw std::runtime_error( "restart: the snapshot's blocks are not this mesh's" );
            snap_block[ it->second ] = pre;
        }
        for( const auto & p : snap_block )
            if( p.empty(  ) )
                throw std::runtime_error( "restart: snapshot lacks a block of this mesh" );
    }
    data_.clear(  );
    for( size_t ib = 0; ib < blocks_.size(  ); ++ ib )
    {
        block_t & blk = blocks_[ ib ];
        std::shared_ptr< block::base_data_t > p;
        if( mhd_ )
        {
            auto q = std::make_shared< dynamics::mhd::block_data_t >(  );
            q->hyd.u.init( blk.geo.n_ceff, type::idx_t( 0 ), 8 );
            type::idx_t nf = blk.geo.n_ceff;
            for( auto & x : nf.x ) x += ( x > 1 );
            q->fld.bf.init( nf, type::idx_t( 2 ), 3 );
            p = q;
        }
        else
        {
            auto q = std::make_shared< dynamics::hydro::block_data_t >(  );
            q->hyd.u.init( blk.geo.n_ceff, type::idx_t( 0 ), 5 );
            p = q;
        }
        p->geo = blk.geo;
        if( snap )
        {   // restart: slot 0 of the stored fields (hyd_data.cpp:49-57, fld_data.cpp:87-95)
            const std::string pre = snap_block[ ib ];
            auto & h = dynamic_cast< dynamics::hydro::block_data_t & >( * p );
            snap->get( pre + "hydro_cons_field", h.hyd.u.dat, h.hyd.u.n_ctot );
            if( mhd_ )
            {
                auto & m = dynamic_cast< dynamics::mhd::block_data_t & >( * p );
                snap->get( pre + "field_bf_field", m.fld.bf.dat, m.fld.bf.n_ctot );
            }
        }
        else
        {
            block::dual_t d( blk );
            d.p_h = p;
            mod.init_cond( d );
        }
        data_.push_back( p );
    }
    std::vector< double > u, bf;
    gather( u, bf );
    if( kr_set_state( ctx_, u.data(  ), mhd_ ? bf.data(  ) : nullptr ) )
        throw std::runtime_error( std::string( "kratos_b200: " ) + kr_last_error( ctx_ ) );
    // cycle parameters (cycle.cpp:30-65)
    t_ = args.get< double >( "cycle", "t_0", 0.0 );
    t_lim_ = args.get< double >( "cycle", "t_lim", 3.4028234663852886e38 );
    n_cycle_lim_ = args.get< int >( "cycle", "n_cycle_lim", 0 );
    n_display_ = std::max( 1, args.get< int >( "cycle", "n_display_freq", 1 ) );
    prefix_ = args.get< std::string >( "cycle", "prefix_output", "test" );
    t_output_ = args.get< double >( "cycle", "t_output_next", 0.0 );
    dt_output_ = args.get< double >( "cycle", "dt_output", 1e32 );
    final_output_ = args.get< bool >( "cycle", "final_output", false );
    double dtb = c.dt_init;
    if( snap )
    {   // cycle.cpp:268-276: the stored dt is the unclamped CFL dt
        snap->get( "time", & t_, 1 );
        snap->get( "dt", & dtb, 1 );
        snap->get( "cycle", & i_cycle_, 1 );
        snap->get( "i_out", & i_output_, 1 );
        snap->get( "t_out", & t_output_, 1 );
    }
    if( dtb < FLT_MIN )                              // cycle.cpp:163-164
        dtb = FLT_MAX / 10;
    kr_set_time( ctx_, t_, dtb );
}

void mesh_t::gather( std::vector< double > & u, std::vector< double > & bf )
{
    u.clear(  );
    bf.clear(  );
    for( auto & p : data_ )
    {
        auto & h = dynamic_cast< dynamics::hydro::block_data_t & >( * p );
        u.insert( u.end(  ), h.hyd.u.buf.begin(  ), h.hyd.u.buf.end(  ) );
        if( mhd_ )
        {
            auto & m = dynamic_cast< dynamics::mhd::block_data_t & >( * p );
            bf.insert( bf.end(  ), m.fld.bf.buf.begin(  ), m.fld.bf.buf.end(  ) );
        }
    }
}

void mesh_t::scatter( const std::vector< double > & u, const std::vector< double > & bf )
{
    size_t ou = 0, ob = 0;
    for( auto & p : data_ )
    {
        auto & h = dynamic_cast< dynamics::hydro::block_data_t & >( * p );
        std::copy( u.begin(  ) + ou, u.begin(  ) + ou + h.hyd.u.n_ctot, h.hyd.u.buf.begin(  ) );
        ou += h.hyd.u.n_ctot;
        if( mhd_ )
        {
            auto & m = dynamic_cast< dynamics::mhd::block_data_t & >( * p );
            std::copy( bf.begin(  ) + ob, bf.begin(  ) + ob + m.fld.bf.n_ctot, m.fld.bf.buf.begin(  ) );
            ob += m.fld.bf.n_ctot;
        }
    }
}

std::string mesh_t::file_name(  ) const
{
    std::ostringstream ss;
    ss << prefix_ << "_" << std::setfill( '0' ) << std::setw( 5 ) << i_output_ << ".bin";
    return ss.str(  );
}

void mesh_t::save( const std::string & file )
{
    std::vector< double > u, bf;
    gather( u, bf );
    if( kr_get_state( ctx_, u.data(  ), mhd_ ? bf.data(  ) : nullptr ) )
        throw std::runtime_error( std::string( "kratos_b200: " ) + kr_last_error( ctx_ ) );
    scatter( u, bf );
    double t = 0, dt_last = 0, dt_bound = 0;
    long long n_done = 0;
    kr_get_time( ctx_, & t, & dt_last, & dt_bound, & n_done );
    if( n_done == 0 )                                 // before the first step: the bound
        dt_last = dt_bound;
    std::cout << "Making output at cycle = " << i_cycle_ << ", t = " << t
              << "; file name: " << file << std::endl;
    ++ i_output_;                                     // cycle.cpp:273-282
    std::map< std::string, snap_entry > e;
    auto put = [ & ]( const std::string & k, const void * p, size_t n, int u_size )
    {
        snap_entry x;
        x.u_size = char( u_size );
        x.bytes.assign( ( const char * ) p, ( const char * ) p + n * u_size );
        e[ k ] = x;
    };
    {   // input_args: serialized map< string, string >
        snap_entry x;
        x.u_size = 1;
        put_size( x.bytes, args_->get_item_map(  ).size(  ) );
        for( const auto & kv : args_->get_item_map(  ) )
        {
            put_str( x.bytes, kv.first );
            put_str( x.bytes, kv.second );
        }
        e[ "input_args" ] = x;
    }
    put( "time", & t, 1, 8 );
    put( "dt", & dt_last, 1, 8 );
    put( "cycle", & i_cycle_, 1, 4 );
    put( "i_out", & i_output_, 1, 4 );
    put( "t_out", & t_output_, 1, 8 );
    e[ "mesh_tree" ] = mesh_tree_blob( blocks_, nb_, periodic_ );
    for( size_t b = 0; b < blocks_.size(  ); ++ b )
    {
        const block_t & blk = blocks_[ b ];
        const std::string pre = "block_" + std::to_string( blk.id_g ) + "|";
        put( pre + "i_logic", blk.reg.x, 3, 4 );
        put( pre + "level", & blk.reg.level, 1, 4 );
        put( pre + "xf0", blk.geo.xf0, 3, 8 );
        put( pre + "dx0", blk.geo.dx0, 3, 8 );
        put( pre + "sfc0", blk.geo.sfc0, 3, 8 );
        put( pre + "vol0", & blk.geo.vol0, 1, 8 );
        put( pre + "n_gh", & blk.geo.n_gh, 1, 4 );
        put( pre + "n_ceff", blk.geo.n_ceff.x, 3, 4 );
        const char uni[ 3 ] = { 1, 1, 1 };
        put( pre + "uniform", uni, 3, 1 );
        auto & h = dynamic_cast< dynamics::hydro::block_data_t & >( * data_[ b ] );
        auto dat = [ & ]( const std::string & p, const dat_3d_t< double > & d )
        {
            const int n_step = 2;
            put( pre + p + "n_int", & d.n_int, 1, 4 );
            put( pre + p + "n_step", & n_step, 1, 4 );
            put( pre + p + "n_cell", d.n_cell.x, 3, 4 );
            put( pre + p + "n_gh", d.n_gh.x, 3, 4 );
            put( pre + p + "field", d.dat, d.n_ctot, 8 );
        };
        dat( "hydro_cons_", h.hyd.u );
        if( mhd_ )
            dat( "field_bf_", dynamic_cast< dynamics::mhd::block_data_t & >( * data_[ b ] ).fld.bf );
    }
    std::vector< char > hdr;
    put_size( hdr, e.size(  ) );
    size_t off = 0;
    for( const auto & kv : e )
    {
        put_str( hdr, kv.first );
        put_size( hdr, kv.second.bytes.size(  ) );
        hdr.push_back( kv.second.u_size );
        put_size( hdr, off );
        off += kv.second.bytes.size(  );
    }
    const size_t header_size = 1 + 8 + hdr.size(  );
    std::ofstream f( file, std::ios::binary );
    if( ! f )
        throw std::runtime_error( "Cannot open file " + file );
    const char sst = char( 1 | sizeof( size_t ) );
    f.write( & sst, 1 );
    f.write( reinterpret_cast< const char * >( & header_size ), 8 );
    f.write( hdr.data(  ), hdr.size(  ) );
    for( const auto & kv : e )
        f.write( kv.second.bytes.data(  ), kv.second.bytes.size(  ) );
}

void mesh_t::evolve(  )
{
    const double n_cell_tot = double( blocks_.size(  ) ) * n_[ 0 ] * n_[ 1 ] * n_[ 2 ];
    const int i_cycle_0 = i_cycle_;
    const auto start = std::chrono::steady_clock::now(  );
    auto update_tout = [ & ](  )
    {   // cycle.cpp:228-237
        const double delta_t = t_ - t_output_;
        if( delta_t < 0 ) return false;
        t_output_ += double( size_t( delta_t / dt_output_ ) + 1 ) * dt_output_;
        return true;
    };
    // Time-dependent control (outputs at t_output_next + k dt_output, t_lim)
    // needs t after every step; otherwise the steps up to the next displayed
    // cycle run as one batch of graph launches with a single host sync.
    const bool per_step = dt_output_ < 1e30 || t_lim_ < 3e38;
    // cycle.cpp:168-180: an error inside the loop (here: the device status
    // word, checked after every batch of steps) ends it; with final_output the
    // state reached is written and evolve returns.
    bool to_stop = false;
    try
    {
    for( ;; )
    {
        if( update_tout(  ) )
            save( file_name(  ) );
        if( t_ >= t_lim_ )
            break;
        int stop = i_cycle_;
        if( ! per_step )
        {
            const int next_show = ( i_cycle_ / n_display_ + ( i_cycle_ % n_display_ != 0 ) ) * n_display_;
            stop = std::max( i_cycle_, std::min( next_show, n_cycle_lim_ ) );
        }
        if( kr_step( ctx_, stop - i_cycle_ + 1 ) )
            throw std::runtime_error( std::string( "kratos_b200: " ) + kr_last_error( ctx_ ) );
        i_cycle_ = stop;
        double dt = 0;
        kr_get_time( ctx_, & t_, & dt, nullptr, nullptr );
        if( const int st = kr_status( ctx_ ) )
            throw std::runtime_error( std::string( "kratos_b200: device status " ) + std::to_string( st )
                                      + ( st & 2 ? " (NaN velocity in the state)" : " (non-finite or non-positive dt)" )
                                      + " at cycle " + std::to_string( i_cycle_ ) + "\n" );
        if( i_cycle_ % n_display_ == 0 )
            std::cout << "cycle = " << std::setw( 5 ) << i_cycle_ << std::scientific
                      << std::setprecision( 6 ) << ", t = " << t_ << ", dt = " << dt
                      << std::defaultfloat << std::endl;
        if( i_cycle_ >= n_cycle_lim_ )
            break;
        ++ i_cycle_;
    }
    }
    catch( const std::exception & exc )
    {
        std::cerr << exc.what(  );
        to_stop = true;
    }
    if( to_stop && final_output_ )
    {
        save( file_name(  ) );
        return;
    }
    kr_get_time( ctx_, & t_, nullptr, nullptr, nullptr );
    const double dwt = std::chrono::duration< double >( std::chrono::steady_clock::now(  ) - start ).count(  );
    const double speed = n_cell_tot / dwt * ( i_cycle_ - i_cycle_0 + 1 );
    std::cout << "Duration = " << dwt << " s, Speed = " << speed << " cell/s,\n"
              << "Pace = " << 1 / speed << " s/cell." << std::endl;
    if( final_output_ )
        save( file_name(  ) );
}
}   // namespace mesh
