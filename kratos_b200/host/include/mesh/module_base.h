// Module base of the mesh (mesh::mod_base_t of the reference,
// src/mesh/module_base/module_base.h:15-97), reduced to what a dynamics module
// needs here: parameters in, initial conditions out.
#pragma once

#include "../io/args/input.h"
#include "block/dual_data.h"

namespace mesh
{
class mesh_t;

class mod_base_t
{
public:
    virtual ~mod_base_t(  ) {}
    virtual void read( const input & ) {}
    virtual void init_cond( block::dual_t & ) {}
};
}   // namespace mesh
