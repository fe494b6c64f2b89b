// Ideal-MHD module (dynamics::mhd_t of the reference,
// src/modules/dynamics/mhd/mhd.h:15-59): adds the uniform field [init] b0.
#pragma once

#include "../hydro/hydro.h"
#include "types/block_data.h"

namespace dynamics
{
class mhd_t : public hydro_t
{
protected:
    type::coord2_t b0;
public:
    void read( const input & args ) override
    {
        b0 = args.get< type::coord2_t >( "init", "b0", 0 );
        hydro_t::read( args );
    }
    void enroll_default(  ) override
    {
        if( ! integrate )
            enroll<  >(  );
    }
    bool is_mhd(  ) const override { return true; }
    void init_cond( mesh::block::dual_t & d ) override;
};
}   // namespace dynamics
