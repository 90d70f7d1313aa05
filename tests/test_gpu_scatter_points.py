"""Scattering sources point by point against the reference's own
srcfunc_sca (src/scatter.c:643-662), called by tests/golden/make_golden.py
on single points of the sulfate-like layer:

  order1  single scattering (srcfunc_sca_1d + srcfunc_sca_sun), IP=1, three
          points, two of them by day
  order2  the depth-2 source (SCA_MULT=2: 28 pencils of order 1, each with
          its own scattering points and 28 leaf pencils), one point by
          night and one by day, CO2/H2O continua off (the reference's
          continuum 0/0 on zero-length leaf segments otherwise makes it NaN)
  ip2/ip3 the 3-D source (srcfunc_sca_3d: 32,400 pencils) through the
          horizontally varying curtain atmosphere, at noon

The GPU computes the same sources with jsc_srcfunc_sca (secondary pencils as
child batches, source integral and solar term on the device) through the
balanced pressures the reference used; bar 1e-9 relative."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

REL_TOL = 1e-9


@pytest.mark.parametrize("kind", ["order1", "order2", "ip2", "ip3"])
def test_scattering_source_points(workdir, kind):
    from jscat import api, structs as S
    from make_golden_shim import scattering_point_case, tables_digest
    path = os.path.join(GOLDEN, "sca_points_%s.npz" % kind)
    if not os.path.exists(path):
        pytest.skip("fixture %s not generated" % kind)
    g = dict(np.load(path))
    ctlkw, atm, _, _, order = scattering_point_case(workdir, kind)
    assert tables_digest(ctlkw["tblbase"], ctlkw["emitters"], ctlkw["nus"]) == str(g["table_sha256"])
    ctl = S.make_ctl(**ctlkw)
    a = S.make_atm(atm["z"], g["p"], atm["t"], atm["q"], atm["k"], atm.get("lon"), atm.get("lat"))
    aero = S.AeroT.from_buffer_copy(g["aero"].tobytes())
    src = api.srcfunc_sca(ctl, a, aero, g["x"], g["dx"], g["il"], g["time"], scattering=order)
    assert np.all(np.isfinite(g["src"])) and np.all(g["src"] > 0)
    rel = np.abs(src - g["src"]) / np.abs(g["src"])
    assert rel.max() <= REL_TOL, rel
