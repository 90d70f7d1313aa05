"""Host logic of the batched Jacobian (jsc_kernel): the state and
measurement vectors against the reference's own atm2x / x2atm / obs2y
(src/atmosphere.c:5-97, src/retrievalmodel.c:379-403,1103-1163, compiled
from the reference's sources into oracle/_ref), and the refusals that
happen before any device work.  No GPU needed."""
import ctypes as C

import numpy as np
import pytest

from oracle import refrun

RET = dict(rett_zmin=5.0, rett_zmax=40.0, retq_zmin=[20.0, 5.0], retq_zmax=[30.0, 25.0],
           retk_zmin=[10.0], retk_zmax=[15.0], retp_zmin=30.0, retp_zmax=35.0)

needs_ref = pytest.mark.skipif(not refrun.kernel_available(),
                               reason="reference retrieval library not built (make -C oracle ref)")


def _case():
    from jscat import synth
    rng = np.random.default_rng(7)
    atm = synth.atmosphere(synth.CFG0_EMITTERS, rng)
    ctlkw = dict(emitters=synth.CFG0_EMITTERS, nus=synth.CFG0_NU, tblbase="-", **RET)
    return ctlkw, atm


def _structs(ctlkw, atm):
    from jscat import structs as S
    return S.make_ctl(**ctlkw), S.make_atm(atm["z"], atm["p"], atm["t"], atm["q"], atm.get("k"))


@needs_ref
def test_state_vector_matches_reference():
    from jscat import api, structs as S
    ctlkw, atm = _case()
    rng = np.random.default_rng(8)
    rad = rng.uniform(1e-4, 1e-2, (30, len(ctlkw["nus"])))
    rad[3, 1] = np.nan
    rad[10, :] = np.nan
    ref = refrun.reference_state_vector(ctlkw, atm, rad, scale=1.5, shift=0.25)
    ctl, a = _structs(ctlkw, atm)
    x, iqa, ipa = api.atm2x(ctl, a)
    assert len(x) == len(ref["x0"]) > 0
    np.testing.assert_array_equal(x, ref["x0"])
    np.testing.assert_array_equal(iqa, ref["iqa"])
    np.testing.assert_array_equal(ipa, ref["ipa"])
    # every quantity of the retrieval settings is present
    assert set(iqa) == {0, 1, 2, 3, 4}
    api.x2atm(ctl, x * 1.5 + 0.25, a)
    na, ng, nw = a.np, ctl.ng, ctl.nw
    np.testing.assert_array_equal(S.arr(a.p)[:na], ref["p"])
    np.testing.assert_array_equal(S.arr(a.t)[:na], ref["t"])
    np.testing.assert_array_equal(S.arr(a.q)[:ng, :na], ref["q"])
    np.testing.assert_array_equal(S.arr(a.k)[:nw, :na], ref["k"])
    obs = S.ObsT()
    obs.nr = rad.shape[0]
    S.arr(obs.rad)[:ctl.nd, :obs.nr] = rad.T
    y, ida, ira = api.obs2y(ctl, obs)
    assert len(y) == rad.size - 5
    np.testing.assert_array_equal(y, ref["y"])
    np.testing.assert_array_equal(ida, ref["ida"])
    np.testing.assert_array_equal(ira, ref["ira"])


def test_empty_state_vector():
    from jscat import api
    ctlkw, atm = _case()
    ctlkw = {k: v for k, v in ctlkw.items() if not k.startswith("ret")}
    ctl, a = _structs(ctlkw, atm)
    x, iqa, ipa = api.atm2x(ctl, a)
    assert len(x) == 0


def test_kernel_refusals_before_device_work():
    """A matrix of the wrong width, and aerosol parameters in the state
    vector without aerosol data, are refused on the host."""
    from jscat import api, lib as L, structs as S
    lib = L.load()
    ctlkw, atm = _case()
    ctl, a = _structs(ctlkw, atm)
    obs = S.make_obs([800.0], [0.0], [20.0], [15.0])
    n = len(api.atm2x(ctl, a)[0])
    k = np.zeros((ctl.nd, n + 1))
    kp = k.ctypes.data_as(C.POINTER(C.c_double))
    st = lib.jsc_kernel(C.byref(ctl), C.byref(a), C.byref(obs), C.byref(S.AeroT()), kp,
                        ctl.nd, n + 1, n + 1)
    assert st == 1 and b"state vector" in lib.jsc_last_error_message()
    ctl.retnn = 1
    st = lib.jsc_kernel(C.byref(ctl), C.byref(a), C.byref(obs), None, kp, ctl.nd, n + 1, n + 1)
    assert st == 1 and b"aerosol" in lib.jsc_last_error_message()
