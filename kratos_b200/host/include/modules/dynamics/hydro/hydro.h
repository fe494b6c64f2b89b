// Hydrodynamics module (dynamics::hydro_t of the reference,
// src/modules/dynamics/hydro/hydro.h:16-58): uniform [init] rho0 / pre0 / vel0
// initial state unless a problem generator overrides init_cond.
#pragma once

#include "../dynamics.h"
#include "types/block_data.h"

namespace dynamics
{
class hydro_t : public base_t
{
protected:
    double rho0 = 0, pre0 = 0;
    type::coord2_t vel0;
public:
    void read( const input & args ) override
    {
        rho0 = args.get< double >( "init", "rho0", 0 );
        pre0 = args.get< double >( "init", "pre0", 0 );
        vel0 = args.get< type::coord2_t >( "init", "vel0", 0 );
        base_t::read( args );
    }
    // hydro_t::enroll_default of the reference enrols data and boundary
    // keeper only; a hydro pgen enrols the policies itself.
    void enroll_default(  ) override {}
    void init_cond( mesh::block::dual_t & d ) override;
};
}   // namespace dynamics
