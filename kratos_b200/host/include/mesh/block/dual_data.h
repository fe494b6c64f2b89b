// Host view of one block's module data, as a problem generator's init_cond
// receives it (mesh::block::dual_t of the reference, src/mesh/block/dual_data.h:
// h() = host data, b_w = the block).  The device copy lives in the B200 engine.
#pragma once

#include <functional>
#include <memory>
#include "block.h"

namespace mesh::block
{
struct base_data_t
{
    virtual ~base_data_t(  ) {}
    geo_t geo;
};

struct dual_t
{
    std::shared_ptr< base_data_t > p_h;
    std::reference_wrapper< block_t > b_w;
    explicit dual_t( block_t & b ) : b_w( b ) {}
    base_data_t & h(  ) const { return * p_h; }
    const geo_t & geo(  ) const { return b_w.get(  ).geo; }
};
}   // namespace mesh::block
