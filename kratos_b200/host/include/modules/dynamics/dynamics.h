// Dynamics module base (dynamics::base_t of the reference,
// src/modules/dynamics/dynamics.h:30-117).  `enroll<>()` takes the reference's
// policy list (proxy, integrator, EOS, reconstruction, Riemann solver, comm);
// only the defaults exist on the B200 engine (PLM + HLLC / HLLD + Heun RK2,
// adiabatic EOS), so any explicit policy is rejected at compile time.
#pragma once

#include <functional>
#include <memory>
#include "../../mesh/module_base.h"

namespace dynamics
{
namespace eos
{
struct base_t                        // prototypes/eos.h:32-56
{
    double gamma = 1.66667, cfl = 0.3, d_floor = 1e-9, t_floor = 1e-9;
    void read( const input & args )
    {
        gamma   = args.get< double >( "dynamics", "gamma", 1.66667 );
        cfl     = args.get< double >( "dynamics", "cfl", 0.3 );
        d_floor = args.get< double >( "dynamics", "rho_floor", 1e-9 );
        t_floor = args.get< double >( "dynamics", "tmp_floor", 1e-9 );
    }
};
}   // namespace eos

class base_t : public mesh::mod_base_t
{
public:
    std::shared_ptr< eos::base_t > p_eos = std::make_shared< eos::base_t >(  );
    std::function< void( mesh::mesh_t &, const int & ) > integrate;

    void read( const input & args ) override
    {
        p_eos->read( args );
        if( ! integrate )
            enroll_default(  );
    }
    virtual void enroll_default(  ) {}
    virtual bool is_mhd(  ) const { return false; }

    template< class ... policies_T >
    void enroll(  )
    {
        static_assert( sizeof...( policies_T ) == 0,
                       "kratos_b200 runs the default dynamics policies only" );
        integrate = [ ] ( mesh::mesh_t &, const int & ) {};   // the step runs on the B200 engine
    }
};
}   // namespace dynamics
