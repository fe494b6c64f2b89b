// The B200 engine bound into the ORIGINAL Kratos tree as a dynamics module.
//
// kratos_b200::b200_t< dynamics::mhd_t > (or < dynamics::hydro_t >) is the
// reference's own module class (src/modules/dynamics/mhd/mhd.h:15-59,
// hydro/hydro.h) with one virtual replaced: step(), which Kratos's cycle calls
// once per time step through mesh_t::step (src/mesh/mesh.cpp:190-197) and
// which the reference implements as two `integrate` stages
// (src/modules/dynamics/dynamics.cpp:37-42, dynamics.h:51-103).  Here a step
// hands the blocks' state to the engine through the C ABI of
// include/kratos_b200.h and takes it back:
//
//   blocks (device copy, slot 0) --copy_d2h--> host arrays, reference layout
//   kr_set_state / kr_set_time (the cycle's t and the dt bound it holds)
//   kr_step( 1 )                 one Heun step on the GPU (captured graph)
//   kr_get_time / kr_get_state   dt taken, new state
//   host arrays --copy_h2d--> blocks; the cycle's dt bookkeeping done as its
//   redc_dt_start / redc_dt_finish (cycle.cpp:77-115) with the engine's dt
//
// so the reference's mesh, cycle, problem generator, outputs and restart work
// unchanged around it.  Everything else of the module (read, block data,
// init_cond, boundary keeper, snapshot I/O) is the reference's.  The engine
// takes a uniform mesh of equal blocks with the reference's [mesh],
// [dynamics], [cycle] and [boundary] keys; [b200] precision / riemann choose
// the engine's mode (defaults: FP64, the reference's solver).
//
// Header-only; compile it into a problem generator built against the Kratos
// sources and link libkrb200.so (oracle/Makefile.ref, target kratos_ref_b200).
#pragma once

#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "mesh/mesh.h"
#include "modules/dynamics/hydro/hydro.h"
#include "modules/dynamics/mhd/mhd.h"

#include "kratos_b200.h"

namespace kratos_b200
{
template< class base_T >
struct b200_t : base_T
{
    static constexpr bool mhd = std::is_base_of_v< dynamics::mhd_t, base_T >;
    using bdt_t = std::conditional_t< mhd, dynamics::mhd::block_data_t, dynamics::hydro::block_data_t >;

    kr_ctx * ctx = nullptr;
    kr_cfg   cfg;
    int      nw = mhd ? 8 : 5;
    std::vector< double > hu, hbf;      // all blocks, lexicographic order

    ~b200_t(  ) { if( ctx ) kr_ctx_destroy( ctx ); }

    static int kind_of( const std::string & k )
    {
        static const std::map< std::string, int > m = {
            { "per", KR_BC_PER }, { "out", KR_BC_OUT }, { "ref", KR_BC_REF },
            { "fre", KR_BC_FRE }, { "fixd", KR_BC_FIXD } };
        const auto it = m.find( k );
        if( it == m.end(  ) )
            throw std::runtime_error( "kratos_b200: unsupported boundary kind " + k );
        return it->second;
    }

    void init( const input & args, mesh::mesh_t & mesh ) override
    {
        base_T::init( args, mesh );        // the reference's blocks, init_cond, keeper
        if( args.get< bool >( "cycle", "t_lim_top_up", false ) )
            throw std::runtime_error( "kratos_b200: [cycle] t_lim_top_up is not supported" );
        kr_cfg_default( & cfg );
        cfg.mhd = mhd;
        cfg.precision = args.get< int >( "b200", "precision", 2 );
        cfg.riemann   = args.get< int >( "b200", "riemann", KR_RIEMANN_DEFAULT );
        cfg.integrator = args.get< std::string >( "b200", "integrator", "rk2" ) == "vl2"
                       ? KR_INTEGRATOR_VL2 : KR_INTEGRATOR_RK2;
        const auto x0 = args.get< type::coord2_t >( "mesh", "x_min" );
        const auto x1 = args.get< type::coord2_t >( "mesh", "x_max" );
        const auto ng = args.get< type::idx_t >( "mesh", "n_cell_global" );
        const auto nc = args.get< type::idx_t >( "mesh", "n_cell_block", ng );
        for( int a = 0; a < 3; ++ a )
        {
            cfg.n[ a ] = nc[ a ];
            cfg.nb[ a ] = ng[ a ] / nc[ a ];
            cfg.x_min[ a ] = x0[ a ];
            cfg.x_max[ a ] = x1[ a ];
        }
        cfg.gamma     = this->p_eos->gamma;
        cfg.cfl       = this->p_eos->cfl;
        cfg.rho_floor = this->p_eos->d_floor;
        cfg.tmp_floor = this->p_eos->t_floor;
        cfg.dt_expand = args.get< double >( "cycle", "dt_expand", 2.0 );
        cfg.device    = args.get< int >( "device", "idx_device", 0 );
        std::vector< std::string > kinds;
        args( "boundary", "kinds", kinds );
        for( int s = 0; s < 6; ++ s )
            cfg.bc[ s ] = kind_of( kinds.at( s ) );
        const auto vel0 = args.get< type::coord2_t >( "init", "vel0", 0 );
        const auto b0   = args.get< type::coord2_t >( "init", "b0", 0 );
        cfg.w_fix[ 0 ] = args.get< double >( "init", "rho0", 0 );
        cfg.w_fix[ 1 ] = args.get< double >( "init", "pre0", 0 );
        for( int a = 0; a < 3; ++ a )
        {
            cfg.w_fix[ 2 + a ] = vel0[ a ];
            cfg.b_fix[ a ] = b0[ a ];
        }
        ctx = kr_ctx_create( & cfg );
        if( ! ctx )
            throw std::runtime_error( std::string( "kratos_b200: " ) + kr_last_error( nullptr ) );
        const size_t nblk = size_t( cfg.nb[ 0 ] ) * cfg.nb[ 1 ] * cfg.nb[ 2 ];
        hu.resize( nblk * cfg.n[ 0 ] * cfg.n[ 1 ] * cfg.n[ 2 ] * nw );
        if( mhd )
            hbf.resize( nblk * size_t( cfg.n[ 0 ] + 5 ) * ( cfg.n[ 1 ] + 5 ) * ( cfg.n[ 2 ] + 5 ) * 3 );
    }

    // lexicographic index of a block of the reference's mesh
    size_t lex( const mesh::block::dual_t & d ) const
    {
        const auto & r = d.b_w.get(  ).reg;
        return size_t( r[ 0 ] + cfg.nb[ 0 ] * ( r[ 1 ] + cfg.nb[ 1 ] * r[ 2 ] ) );
    }

    void step( mesh::mesh_t & mesh ) override
    {
        auto & cyc = * mesh.p_cyc;
        auto & dev = * this->p_dev;
        const size_t ncu = size_t( cfg.n[ 0 ] ) * cfg.n[ 1 ] * cfg.n[ 2 ] * nw;
        const size_t ncb = size_t( cfg.n[ 0 ] + 5 ) * ( cfg.n[ 1 ] + 5 ) * ( cfg.n[ 2 ] + 5 ) * 3;
        for( auto & d : * this )
        {   // slot 0 of the device copy, in the reference's per-block layout
            d.copy_d2h(  );
            auto & b = dynamic_cast< bdt_t & >( d.h(  ) );
            std::memcpy( hu.data(  ) + lex( d ) * ncu, b.hyd.u.dat, ncu * sizeof( double ) );
            if constexpr( mhd )
                std::memcpy( hbf.data(  ) + lex( d ) * ncb, b.fld.bf.dat, ncb * sizeof( double ) );
        }
        // the dt bound this step starts from: the cycle's device dt word
        type::float_t bound = 0;
        dev.cp( & bound, cyc.p_dt, 1 );
        dev.sync_all_streams(  );
        double t = 0, dt = 0;
        if( kr_set_state( ctx, hu.data(  ), mhd ? hbf.data(  ) : nullptr )
            || kr_set_time( ctx, cyc.t, bound )
            || kr_step( ctx, 1 )
            || kr_get_time( ctx, & t, & dt, nullptr, nullptr )
            || kr_get_state( ctx, hu.data(  ), mhd ? hbf.data(  ) : nullptr ) )
            throw std::runtime_error( std::string( "kratos_b200: " ) + kr_last_error( ctx ) );
        if( kr_status( ctx ) )
            throw std::runtime_error( "kratos_b200: device status error (non-finite dt or state)" );
        for( auto & d : * this )
        {
            auto & b = dynamic_cast< bdt_t & >( d.h(  ) );
            std::memcpy( b.hyd.u.dat, hu.data(  ) + lex( d ) * ncu, ncu * sizeof( double ) );
            if constexpr( mhd )
                std::memcpy( b.fld.bf.dat, hbf.data(  ) + lex( d ) * ncb, ncb * sizeof( double ) );
            d.copy_h2d(  );
        }
        // cycle.cpp:77-115: the reduced dt is the one the engine took
        type::float_t taken = type::float_t( dt );
        dev.cp( cyc.p_dt, & taken, 1 );
        dev.sync_all_streams(  );
        cyc.redc_dt_start ( mesh );
        cyc.redc_dt_finish( mesh );
    }
};
}   // namespace kratos_b200
