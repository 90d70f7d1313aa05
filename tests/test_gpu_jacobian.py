"""GPU parity of the batched Jacobian (jsc_kernel, the reference's
kernel() with all n + 1 forward models in one batch).

Golden fixtures (tests/golden/jacobian_limb*.npz) hold the output of the
reference's own kernel() (src/retrievalmodel.c:201-298, compiled from its
sources by oracle/Makefile and run by make_golden.py): the Jacobian, the
state vector after the hydrostatic balance, its quantity and level
indices, and the undisturbed radiances.  Bars: indices exact, state vector
within 1e-12 relative; radiances within 1e-9 relative (as the forward-model
parity tests); each Jacobian entry within 1e-6 of its column's largest
magnitude (an entry is a difference of two radiances that each carry the
1e-9 relative agreement, divided by the perturbation size); columns the
reference returns as exact zeros (pressure disturbances undone by the
hydrostatic balance) exact zeros here too.  A column also equals, bit for
bit, the finite difference of two calls of this library's drop-in formod.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from helpers import max_rel

pytestmark = pytest.mark.gpu

K_TOL = 1e-6
REL_TOL = 1e-9


def _setup(workdir, bt, fov=False):
    from jscat import structs as S
    from make_golden_shim import jacobian_case, tables_digest
    ctlkw, atm, geom, mask = jacobian_case(workdir, bt, fov)
    name = "jacobian_limb_fov" if fov else "jacobian_limb_bt" if bt else "jacobian_limb"
    g = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    assert tables_digest(ctlkw["tblbase"], ctlkw["emitters"], ctlkw["nus"]) == str(g["table_sha256"])
    ctl = S.make_ctl(**ctlkw)
    a = S.make_atm(atm["z"], atm["p"], atm["t"], atm["q"], atm.get("k"))
    obs = S.make_obs(geom["obsz"], geom["obslat"], geom["vpz"], geom["vplat"],
                     geom["obslon"], geom["vplon"], geom["time"])
    rad = S.arr(obs.rad)
    for ir, id_ in zip(*np.nonzero(mask)):
        rad[id_, ir] = np.nan
    return ctl, a, obs, g


@pytest.mark.parametrize("bt,fov", [(False, False), (True, False), (False, True)],
                         ids=["radiance", "brightness", "field-of-view"])
def test_kernel_matches_reference(workdir, bt, fov):
    from jscat import api, structs as S
    ctl, a, obs, g = _setup(workdir, bt, fov)
    k = api.kernel(ctl, a, obs)
    kref = g["k"]
    assert k.shape == kref.shape
    x, iqa, ipa = api.atm2x(ctl, a)
    np.testing.assert_array_equal(iqa, g["iqa"])
    np.testing.assert_array_equal(ipa, g["ipa"])
    assert max_rel(x, g["x0"]) <= 1e-12
    assert max_rel(S.arr(a.p)[:a.np], g["p"]) <= 1e-12
    rad = S.arr(obs.rad)[:ctl.nd, :obs.nr].T
    np.testing.assert_array_equal(np.isnan(rad), np.isnan(g["rad"]))
    ok = np.isfinite(g["rad"])
    assert max_rel(rad[ok], g["rad"][ok]) <= REL_TOL
    zero = np.all(kref == 0, axis=0)
    assert np.all(k[:, zero] == 0)
    scale = np.max(np.abs(kref), axis=0)
    err = np.abs(k - kref) / np.where(scale > 0, scale, 1.0)
    assert float(err.max()) <= K_TOL


def test_kernel_column_is_two_formods(workdir):
    """Column j of the batched Jacobian equals (formod(x + h e_j) -
    formod(x)) / h with this library's drop-in formod, bit for bit: one
    batch of n + 1 profiles computes what n + 1 separate calls compute."""
    from jscat import api, structs as S
    ctl, a, obs, g = _setup(workdir, False)
    k = api.kernel(ctl, a, obs)
    y0 = api.obs2y(ctl, obs)[0]
    x0, iqa, ipa = api.atm2x(ctl, a)
    assert list(iqa[[6, 45, 60, len(x0) - 1]]) == [1, 2, 3, 4]
    for j in (6, 45, 60, len(x0) - 1):  # temperature, CO2, H2O, extinction
        ctl2, a2, obs2, _ = _setup(workdir, False)
        api.formod(ctl2, a2, obs2)         # hydrostatic pressures as in the kernel
        x = api.atm2x(ctl2, a2)[0]
        h = 1.0 if iqa[j] == 1 else (1e-4 if iqa[j] == 4 else max(abs(0.01 * x[j]), 1e-15))
        x[j] += h
        api.x2atm(ctl2, x, a2)
        obs3 = S.ObsT.from_buffer_copy(obs2)
        api.formod(ctl2, a2, obs3)
        y1 = api.obs2y(ctl2, obs3)[0]
        np.testing.assert_array_equal(k[:, j], (y1 - y0) / h)


def test_kernel_aerosol_parameters(workdir):
    """Temperature plus the aerosol layer's number concentration, median
    radius and width (RETNN/RETRR/RETSS) through aerosol extinction: the
    optical properties of every aerosol column are recomputed (Mie on the
    GPU) and the column runs as its own batch; against the reference's
    kernel(), which calls its get_opt_prop inside every formod."""
    from jscat import api, structs as S
    from make_golden_shim import aerosol_jacobian_case, tables_digest
    ctlkw, atm, geom, aerofile = aerosol_jacobian_case(workdir)
    g = dict(np.load(os.path.join(GOLDEN, "jacobian_aerosol.npz")))
    assert tables_digest(ctlkw["tblbase"], ctlkw["emitters"], ctlkw["nus"]) == str(g["table_sha256"])
    ctl = S.make_ctl(**ctlkw)
    a = S.make_atm(atm["z"], atm["p"], atm["t"], atm["q"], atm.get("k"))
    obs = S.make_obs(geom["obsz"], geom["obslat"], geom["vpz"], geom["vplat"],
                     geom["obslon"], geom["vplon"], geom["time"])
    aero = api.read_aero(ctl, aerofile)
    k = api.kernel(ctl, a, obs, aero)
    kref = g["k"]
    assert k.shape == kref.shape
    x, iqa, ipa = api.atm2x(ctl, a, aero)
    np.testing.assert_array_equal(iqa, g["iqa"])
    assert max_rel(x, g["x0"]) <= 1e-12
    rad = S.arr(obs.rad)[:ctl.nd, :obs.nr].T
    assert max_rel(rad, g["rad"]) <= REL_TOL
    scale = np.max(np.abs(kref), axis=0)
    err = np.abs(k - kref) / np.where(scale > 0, scale, 1.0)
    assert float(err.max()) <= K_TOL


def test_kernel_curtain_ip2(workdir):
    """Temperature of every profile of the IP=2 curtain: each column is its
    own GPU forward model through the whole horizontally varying
    atmosphere; against the reference's kernel()."""
    from jscat import api, structs as S
    from make_golden_shim import curtain_jacobian_case, tables_digest
    ctlkw, atm, geom = curtain_jacobian_case(workdir)
    g = dict(np.load(os.path.join(GOLDEN, "jacobian_curtain_ip2.npz")))
    assert tables_digest(ctlkw["tblbase"], ctlkw["emitters"], ctlkw["nus"]) == str(g["table_sha256"])
    ctl = S.make_ctl(**ctlkw)
    a = S.make_atm(atm["z"], atm["p"], atm["t"], atm["q"], atm["k"], atm["lon"], atm["lat"])
    obs = S.make_obs(geom["obsz"], geom["obslat"], geom["vpz"], geom["vplat"],
                     geom["obslon"], geom["vplon"], geom["time"])
    k = api.kernel(ctl, a, obs)
    kref = g["k"]
    assert k.shape == kref.shape
    x, iqa, ipa = api.atm2x(ctl, a)
    np.testing.assert_array_equal(ipa, g["ipa"])
    assert max_rel(x, g["x0"]) <= 1e-12
    assert max_rel(S.arr(obs.rad)[:ctl.nd, :obs.nr].T, g["rad"]) <= REL_TOL
    scale = np.max(np.abs(kref), axis=0)
    err = np.abs(k - kref) / np.where(scale > 0, scale, 1.0)
    assert float(err.max()) <= K_TOL
