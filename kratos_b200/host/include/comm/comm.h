// Serial communicator (comm::base_t of the reference, src/comm/comm.h:20-88):
// one rank.  Multi-GPU runs shard blocks across processes through
// kratos_b200's Python/NCCL layer, not through this host layer.
#pragma once

namespace comm
{
struct base_t
{
    virtual ~base_t(  ) {}
    virtual bool is_root(  ) const { return true; }
    virtual int  rank   (  ) const { return 0; }
    virtual int  n_rank (  ) const { return 1; }
};
}   // namespace comm
