// Blocks of the uniform mesh (src/mesh/block/block.h, geometry/region.h of the
// reference): logical position `reg` (with its refinement level) and geometry.
#pragma once

#include "../geometry/geometry.h"

namespace mesh
{
struct region_logic_t : public type::idx_t
{
    int level = 0;
};
struct region_t : public region_logic_t {};

struct block_t
{
    int      id_g = 0, id_l = 0, rank = 0;
    geo_t    geo;
    region_t reg;
};
}   // namespace mesh
