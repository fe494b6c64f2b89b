"""Failure detection without a GPU fault: a bad value planted in the HOST
state, uploaded and stepped.

* Through the C ABI: an infinite momentum makes the CFL dt zero (status bit 0,
  non-positive dt); a NaN momentum, which the dt minimum would drop, sets bit 1
  (the floors heal NaN density and pressure, as the reference's do); a clean
  state leaves the word at 0.  The context stays usable.
* Through the C++ host layer (the reference's evolve contract, cycle.cpp:
  168-180): the loop stops at the error, and with final_output the state
  reached is written; the executable exits normally.
"""
import os
import subprocess

import numpy as np
import pytest

from kratos_b200.snapshot import Snapshot

pytestmark = pytest.mark.gpu


def _ot(nb=(2, 1, 1), n=(8, 8, 8)):
    from kratos_b200 import Dynamics
    d = Dynamics(True, nb, n, gamma=5 / 3)
    d.init_problem("ot", 2)
    return d


@pytest.mark.parametrize("bad, bit", [(np.inf, 1), (np.nan, 2)])
def test_planted_value_sets_status(bad, bit):
    d = _ot()
    u, bf = d.get_state()
    assert d.status() == 0
    u[1, 3, 4, 5, 2] = bad                    # one cell's x-momentum
    d.set_state(u, bf)
    d.step(1)
    assert d.status() & bit, d.status()
    # the context stays usable: a clean state steps again (the word is sticky)
    d2 = _ot()
    d2.step(2)
    assert d2.status() == 0


BAD_PGEN = r"""
#include <limits>
#include "device/general.h"
#include "mesh/mesh_enroll.h"
#include "user/probgen.h"
#include "utilities/mapping/loop.h"
#include "modules/dynamics/mhd/mhd.h"

// The [init] medium with one cell's momentum set to NaN in block 0.
struct bad_mhd_t : dynamics::mhd_t
{
    void init_cond( mesh::block::dual_t & d ) override
    {
        dynamics::mhd_t::init_cond( d );
        auto & b_h = dynamic_cast< dynamics::mhd::block_data_t & >( d.h(  ) );
        const auto & blk = d.b_w.get(  );
        if( blk.reg[ 0 ] == 0 && blk.reg[ 1 ] == 0 && blk.reg[ 2 ] == 0 )
            b_h.hyd.u.at( { 2, 3, 4 } )[ 2 ] = std::numeric_limits< double >::quiet_NaN(  );
    }
};

namespace prob
{
void run( int argc, char * argv[  ] )
{
    mesh::mesh_t mesh;
    mesh.enroll_device< device_t >(  );
    mesh.enroll_comm< comm::base_t >(  );
    input args;
    cmd( argc, argv, args );
    mesh.enroll_module< bad_mhd_t >(  );
    mesh.init( args );
    return mesh.evolve(  );
}
}
"""


def test_host_layer_writes_final_output_on_error(tmp_path):
    from kratos_b200.build import build_host
    src = tmp_path / "bad.cpp"
    src.write_text(BAD_PGEN)
    exe = build_host([str(src)], str(tmp_path / "bad.x"))
    par = tmp_path / "bad.par"
    prefix = tmp_path / "snap"
    par.write_text("\n".join([
        "[mesh]", "x_min = 0 0 0", "x_max = 1 1 1", "n_cell_global = 16 8 8", "n_cell_block = 8 8 8",
        "[cycle]", "prefix_output = %s" % prefix, "n_cycle_lim = 9", "final_output = 1",
        "n_display_freq = 1",
        "[dynamics]", "gamma = 1.6666666666666667",
        "[boundary]", "kinds = per per per per per per",
        "[init]", "rho0 = 1.0", "pre0 = 0.6", "vel0 = 0.1 0 0", "b0 = 0.2 0.1 0", ""]))
    r = subprocess.run([exe, str(par)], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "device status 2" in r.stderr and "NaN velocity" in r.stderr, r.stderr
    # the initial output and the final output (the state reached at the error)
    snaps = sorted(p for p in os.listdir(tmp_path) if p.startswith("snap_"))
    assert len(snaps) == 2, snaps
    s = Snapshot.read(str(tmp_path / snaps[-1]))
    assert int(s.array("cycle", "i")[0]) == 0          # stopped after the first batch
    assert "Speed" not in r.stdout
