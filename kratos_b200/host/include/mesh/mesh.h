// The mesh and its time loop (mesh::mesh_t, cycle::base_t of the reference,
// src/mesh/mesh.h:27-122, mesh_enroll.h:154-233, cycle/cycle.cpp:30-250),
// driving the B200 engine through its C ABI (include/kratos_b200.h).
//
// init(): [mesh] x_min x_max n_cell_global n_cell_block, [boundary] kinds,
//   [dynamics] gamma cfl rho_floor tmp_floor, [cycle] dt_init dt_expand
//   n_cycle_lim t_lim prefix_output dt_output t_output_next final_output
//   n_display_freq, [init] rho0 pre0 vel0 b0, [device] idx_device,
//   [b200] precision (2 FP64, 1 mixed) riemann (0 default, 1 HLLE).
//   Blocks are numbered lexicographically; every enrolled dynamics module's
//   init_cond fills its host block data, which is uploaded once.
// evolve(): steps like cycle::base_t::evolve -- n_cycle_lim + 1 steps, stopping
//   early at t >= t_lim -- writes snapshots at t_output_next + k dt_output and
//   at the end if final_output, and prints the reference's Speed line.
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "../comm/comm.h"
#include "../modules/dynamics/dynamics.h"
#include "block/block.h"

struct kr_ctx;

namespace mesh
{
class mesh_t
{
public:
    std::shared_ptr< comm::base_t > p_com;

    mesh_t(  );
    ~mesh_t(  );

    template< class T > void enroll_device(  ) {}
    template< class T > void enroll_comm(  ) { p_com = std::make_shared< T >(  ); }
    template< class T > std::shared_ptr< T > enroll_module(  )
    {
        auto p = std::make_shared< T >(  );
        mods_.push_back( p );
        return p;
    }

    void init( const input & args );
    void evolve(  );
    void save( const std::string & file );

    // blocks in lexicographic order (x fastest)
    std::vector< block_t > & blocks(  ) { return blocks_; }
    kr_ctx * engine(  ) { return ctx_; }

private:
    std::vector< std::shared_ptr< dynamics::base_t > > mods_;
    std::vector< block_t > blocks_;
    std::vector< std::shared_ptr< block::base_data_t > > data_;
    kr_ctx * ctx_ = nullptr;
    const input * args_ = nullptr;
    bool mhd_ = false;
    int nb_[ 3 ] = { 1, 1, 1 }, n_[ 3 ] = { 1, 1, 1 };
    bool periodic_[ 3 ] = { true, true, true };
    // cycle
    double t_ = 0, t_lim_ = 3.4e38, dt_output_ = 1e32, t_output_ = 0;
    int n_cycle_lim_ = 0, i_cycle_ = 0, i_output_ = 0, n_display_ = 1;
    bool final_output_ = false;
    std::string prefix_ = "test";
    std::vector< char > args_blob_;

    void gather( std::vector< double > & u, std::vector< double > & bf );
    void scatter( const std::vector< double > & u, const std::vector< double > & bf );
    std::string file_name(  ) const;
};
}   // namespace mesh
