// MHD block data (dynamics::mhd::block_data_t of the reference,
// mhd/types/fld_data.h): u with n_int = 8 (rho, E, m0..2, B_cc0..2) and the
// face field bf on the (n+1)^3 lattice with 2 ghost layers.
#pragma once

#include "../../hydro/types/block_data.h"

namespace dynamics::mhd
{
struct fld_t
{
    mesh::dat_3d_t< double > bf;
};
struct block_data_t : ::dynamics::hydro::block_data_t
{
    fld_t fld;
};
}   // namespace dynamics::mhd
