// Hydro block data (dynamics::hydro::block_data_t of the reference,
// hydro/types/hyd_data.h): conserved state u, n_int = 5 (rho, E, m0..2), no
// ghosts, slot 0 only on the host.
#pragma once

#include "../../../../mesh/block/dual_data.h"
#include "../../../../mesh/types/dat_3d.h"

namespace dynamics::hydro
{
struct hyd_t
{
    mesh::dat_3d_t< double > u;
};
struct block_data_t : mesh::block::base_data_t
{
    hyd_t hyd;
};
}   // namespace dynamics::hydro
