// Problem generator compiled together with the original Kratos sources (test
// infrastructure, built by oracle/Makefile.ref into oracle/_ref/).
//
// It enrols the reference's own dynamics modules (dynamics::hydro_t with its
// default PLM + HLLC + RK2 policies, dynamics::mhd_t with PLM + HLLD + CT + RK2)
// exactly as a user pgen does (usr_example/bow_shock/usr.cpp:20-40 of the
// reference) and overrides only init_cond, so that the reference integrates the
// same seeded initial states as this package (kratos_b200/csrc/problems.h).
//
// [problem] name = shock | ot | turb | box | blast ; [problem] seed = <int>
#include <iostream>

#include "device/general.h"
#include "mesh/mesh_enroll.h"
#include "utilities/mapping/loop.h"
#include "user/probgen.h"
#include "modules/dynamics/hydro/hydro.h"
#include "modules/dynamics/mhd/mhd.h"

#include "../../kratos_b200/csrc/problems.h"

// Built with -DKR_B200_MODULE (oracle/Makefile.ref, kratos_ref_b200), the same
// problem generator runs the reference's mesh, cycle and outputs with the
// dynamics step of the B200 engine (kratos_b200/reference_binding).
#ifdef KR_B200_MODULE
#include "../../kratos_b200/reference_binding/b200_dynamics.h"
using hydro_base_t = kratos_b200::b200_t< dynamics::hydro_t >;
using mhd_base_t   = kratos_b200::b200_t< dynamics::mhd_t >;
#else
using hydro_base_t = dynamics::hydro_t;
using mhd_base_t   = dynamics::mhd_t;
#endif

namespace
{
int          g_seed = 1;
int          g_nglob[ 3 ] = { 1, 1, 1 };

uint64_t cell_key( const mesh::block_t & b, const type::idx_t & i )
{
    int ig[ 3 ];
    for( int a = 0; a < 3; ++ a )
        ig[ a ] = b.reg[ a ] * b.geo.n_ceff[ a ] + i[ a ];
    return kr_cell_key( b.reg.level, ig, g_nglob );
}
}   // namespace

struct shock_hydro_t : hydro_base_t
{
    // hydro_t::enroll_default enrols the block data and boundary keeper only;
    // the default policy set (PLM + HLLC + RK2) is enrolled here, as a hydro
    // pgen does.
    void enroll_default(  ) override
    {
        dynamics::hydro_t::enroll_default(  );
        if( ! integrate )
            enroll<  >(  );
    }
    void init_cond( mesh::block::dual_t & d ) override
    {
        auto & b_h = dynamic_cast< dynamics::hydro::block_data_t & >( d.h(  ) );
        const auto & blk = d.b_w.get(  );
        const auto & geo = blk.geo;
        for( auto i : utils::loop( geo.n_ceff ) )
        {
            auto * u = b_h.hyd.u.at( i );
            double uu[ 5 ];
            kr_shock_cell( uu, geo.x_cc( 0, i[ 0 ] ), p_eos->gamma,
                                 g_seed, cell_key( blk, i ) );
            for( int n = 0; n < 5; ++ n )
                u[ n ] = uu[ n ];
        }
    }
};

struct ot_mhd_t : mhd_base_t
{
    void init_cond( mesh::block::dual_t & d ) override
    {
        auto & b_h = dynamic_cast< dynamics::mhd::block_data_t & >( d.h(  ) );
        const auto & blk = d.b_w.get(  );
        const auto & geo = blk.geo;
        auto n_face = geo.n_ceff;
        for( auto & n_s : n_face.x )
            n_s += ( n_s > 1 );
        for( auto i : utils::loop( n_face ) )
        {
            auto * bf = b_h.fld.bf.at( i );
            bf[ 0 ] = kr_ot_bx( geo.x_cc( 1, i[ 1 ] ) );
            bf[ 1 ] = kr_ot_by( geo.x_cc( 0, i[ 0 ] ) );
            bf[ 2 ] = kr_ot_bz(  );
        }
        for( auto i : utils::loop( geo.n_ceff ) )
        {
            double x[ 3 ], bc[ 3 ];
            for( int a = 0; a < 3; ++ a )
            {
                x[ a ] = geo.x_cc( a, i[ a ] );
                auto j = i;
                ++ j[ a ];
                bc[ a ] = ( b_h.fld.bf.at( i )[ a ] + b_h.fld.bf.at( j )[ a ] ) / 2;
            }
            double uu[ 8 ];
            kr_ot_cell( uu, x, bc, p_eos->gamma, g_seed, cell_key( blk, i ) );
            auto * u = b_h.hyd.u.at( i );
            for( int n = 0; n < 8; ++ n )
                u[ n ] = uu[ n ];
        }
    }
};

// Decaying supersonic turbulence: uniform B_x, random-phase solenoidal velocity.
struct turb_mhd_t : mhd_base_t
{
    void init_cond( mesh::block::dual_t & d ) override
    {
        auto & b_h = dynamic_cast< dynamics::mhd::block_data_t & >( d.h(  ) );
        const auto & blk = d.b_w.get(  );
        const auto & geo = blk.geo;
        kr_turb_t modes;
        kr_turb_modes( & modes, ( uint64_t ) g_seed );
        auto n_face = geo.n_ceff;
        for( auto & n_s : n_face.x )
            n_s += ( n_s > 1 );
        for( auto i : utils::loop( n_face ) )
        {
            auto * bf = b_h.fld.bf.at( i );
            bf[ 0 ] = kr_turb_bx( p_eos->gamma );
            bf[ 1 ] = bf[ 2 ] = 0;
        }
        for( auto i : utils::loop( geo.n_ceff ) )
        {
            double x[ 3 ], bc[ 3 ];
            for( int a = 0; a < 3; ++ a )
            {
                x[ a ] = geo.x_cc( a, i[ a ] );
                auto j = i;
                ++ j[ a ];
                bc[ a ] = ( b_h.fld.bf.at( i )[ a ] + b_h.fld.bf.at( j )[ a ] ) / 2;
            }
            double uu[ 8 ];
            kr_turb_cell( uu, x, bc, p_eos->gamma, & modes );
            auto * u = b_h.hyd.u.at( i );
            for( int n = 0; n < 8; ++ n )
                u[ n ] = uu[ n ];
        }
    }
};

// Magnetized blast wave: over-pressured sphere at the domain's centre, uniform B.
static double g_centre[ 3 ] = { 0.5, 0.5, 0.5 };

struct blast_mhd_t : mhd_base_t
{
    void init_cond( mesh::block::dual_t & d ) override
    {
        auto & b_h = dynamic_cast< dynamics::mhd::block_data_t & >( d.h(  ) );
        const auto & blk = d.b_w.get(  );
        const auto & geo = blk.geo;
        auto n_face = geo.n_ceff;
        for( auto & n_s : n_face.x )
            n_s += ( n_s > 1 );
        for( auto i : utils::loop( n_face ) )
        {
            auto * bf = b_h.fld.bf.at( i );
            for( int a = 0; a < 3; ++ a )
                bf[ a ] = kr_blast_b( a );
        }
        for( auto i : utils::loop( geo.n_ceff ) )
        {
            double x[ 3 ], bc[ 3 ];
            for( int a = 0; a < 3; ++ a )
            {
                x[ a ] = geo.x_cc( a, i[ a ] );
                auto j = i;
                ++ j[ a ];
                bc[ a ] = ( b_h.fld.bf.at( i )[ a ] + b_h.fld.bf.at( j )[ a ] ) / 2;
            }
            double uu[ 8 ];
            kr_blast_cell( uu, x, bc, g_centre, p_eos->gamma );
            auto * u = b_h.hyd.u.at( i );
            for( int n = 0; n < 8; ++ n )
                u[ n ] = uu[ n ];
        }
    }
};

// One box of a batch of independent periodic boxes ([problem] box = index); the
// mesh is the box: n_cell_global = n_cell_block = its edge length.
static int g_box = 0;

struct box_mhd_t : mhd_base_t
{
    void init_cond( mesh::block::dual_t & d ) override
    {
        auto & b_h = dynamic_cast< dynamics::mhd::block_data_t & >( d.h(  ) );
        const auto & blk = d.b_w.get(  );
        const auto & geo = blk.geo;
        kr_box_t p;
        kr_box_params( & p, ( uint64_t ) g_seed, g_box, p_eos->gamma );
        auto n_face = geo.n_ceff;
        for( auto & n_s : n_face.x )
            n_s += ( n_s > 1 );
        for( auto i : utils::loop( n_face ) )
        {
            auto * bf = b_h.fld.bf.at( i );
            for( int a = 0; a < 3; ++ a )
                bf[ a ] = p.b[ a ];
        }
        for( auto i : utils::loop( geo.n_ceff ) )
        {
            double x[ 3 ], bc[ 3 ];
            for( int a = 0; a < 3; ++ a )
            {
                x[ a ] = geo.x_cc( a, i[ a ] );
                auto j = i;
                ++ j[ a ];
                bc[ a ] = ( b_h.fld.bf.at( i )[ a ] + b_h.fld.bf.at( j )[ a ] ) / 2;
            }
            double uu[ 8 ];
            kr_box_cell( uu, x, bc, p_eos->gamma, & p, cell_key( blk, i ) );
            auto * u = b_h.hyd.u.at( i );
            for( int n = 0; n < 8; ++ n )
                u[ n ] = uu[ n ];
        }
    }
};

namespace prob
{
void run( int argc, char * argv[  ] )
{
    mesh::mesh_t mesh;
    mesh.enroll_device< device_t >(  );
    mesh.enroll_comm< comm::base_t >(  );
    input args;
    args.set_comm( mesh.p_com );
    cmd( argc, argv, args );
    const auto name = args.get< std::string >( "problem", "name" );
    g_seed          = args.get< int >( "problem", "seed", 1 );
    const auto ng   = args.get< type::idx_t >( "mesh", "n_cell_global" );
    for( int a = 0; a < 3; ++ a )
        g_nglob[ a ] = ng[ a ];

    if( name == "shock" )
        mesh.enroll_module< shock_hydro_t >(  );
    else if( name == "ot" )
        mesh.enroll_module< ot_mhd_t >(  );
    else if( name == "turb" )
        mesh.enroll_module< turb_mhd_t >(  );
    else if( name == "blast" )
    {
        const auto x0 = args.get< type::coord2_t >( "mesh", "x_min" );
        const auto x1 = args.get< type::coord2_t >( "mesh", "x_max" );
        for( int a = 0; a < 3; ++ a )
            g_centre[ a ] = ( x0[ a ] + x1[ a ] ) / 2;
        mesh.enroll_module< blast_mhd_t >(  );
    }
    else if( name == "box" )
    {
        g_box = args.get< int >( "problem", "box", 0 );
        mesh.enroll_module< box_mhd_t >(  );
    }
    else
        throw std::runtime_error( "unknown [problem] name " + name );
    mesh.init( args );
    return mesh.evolve(  );
}
};  // namespace prob
