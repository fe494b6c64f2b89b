// mesh_t's enrolment templates (src/mesh/mesh_enroll.h of the reference).
#pragma once

#include "mesh.h"
