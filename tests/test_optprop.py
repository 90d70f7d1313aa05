"""Host logic of the aerosol/cloud optical properties: jsc_read_aero
against the reference's read_aero (the mode fields of the golden aero_t
fixtures, which the reference's read_aero + get_opt_prop wrote), and
jsc_get_opt_prop on a layer taken from an external optical-property
database (opt_prop_external, host only) against the reference run here.
No GPU needed."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import refrun


def _fixture(name):
    from jscat import structs as S
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    return S.AeroT.from_buffer_copy(d["aero"].tobytes()), list(d["nus"])


CASES = [("aero_sulfate16", "sulfate_layer_files", 1), ("aero_ice8", "ice_layer_files", 1),
         ("aero_layers8", "layered_aero_files", 3)]


@pytest.mark.parametrize("name,files,sca_n", CASES)
def test_read_aero_matches_reference(workdir, name, files, sca_n):
    from jscat import api, structs as S, synth
    ref, nus = _fixture(name)
    aerofile = getattr(synth, files)(os.path.join(workdir, "aero"))
    ctl = S.make_ctl(synth.CFG0_EMITTERS, nus, "-", sca_n=sca_n)
    aero = api.read_aero(ctl, aerofile)
    assert aero.nm == ref.nm == sca_n
    for f in ("top_mod", "bottom_mod", "trans_mod", "nn", "rr", "ss"):
        np.testing.assert_array_equal(S.arr(getattr(aero, f))[:aero.nm],
                                      S.arr(getattr(ref, f))[:ref.nm])
    for im in range(aero.nm):
        assert aero.type[im].value == ref.type[im].value
        assert os.path.basename(aero.filepath[im].value) == os.path.basename(ref.filepath[im].value)


def test_read_aero_refusals(workdir):
    from jscat import api, lib as L, structs as S, synth
    aerofile = synth.layered_aero_files(os.path.join(workdir, "aero"))
    ctl = S.make_ctl(synth.CFG0_EMITTERS, list(synth.CFG2_NU[::2]), "-", sca_n=1)
    with pytest.raises(L.JscError, match="SCA_N=1 but 3"):
        api.read_aero(ctl, aerofile)
    with pytest.raises(L.JscError, match="cannot open"):
        api.read_aero(ctl, os.path.join(workdir, "aero", "missing.tab"))


@pytest.mark.skipif(not refrun.available(), reason="reference library not built")
def test_external_database_matches_reference(workdir):
    """A layer from an external optical-property database: nearest-
    wavenumber records, no Mie series, so the whole get_opt_prop runs on
    the host and must equal the reference's bit for bit."""
    from jscat import api, structs as S, synth
    nus = list(synth.CFG2_NU)
    aerofile = synth.external_aero_files(os.path.join(workdir, "aero"))
    ctlkw = dict(emitters=synth.CFG0_EMITTERS, nus=nus, tblbase="-", sca_n=1, sca_mult=1)
    ref = S.AeroT.from_buffer_copy(refrun.reference_aero(ctlkw, aerofile,
                                                         os.path.dirname(aerofile)))
    ctl = S.make_ctl(**ctlkw)
    aero = api.get_opt_prop(ctl, api.read_aero(ctl, aerofile))
    assert aero.nl == ref.nl == 1
    nd = len(nus)
    for f in ("beta_e", "beta_s", "beta_a"):
        np.testing.assert_array_equal(S.arr(getattr(aero, f))[:1, :nd],
                                      S.arr(getattr(ref, f))[:1, :nd])
    np.testing.assert_array_equal(S.arr(aero.p)[:1, :nd], S.arr(ref.p)[:1, :nd])
    for f in ("top", "bottom", "trans", "nmod"):
        np.testing.assert_array_equal(S.arr(getattr(aero, f))[:1], S.arr(getattr(ref, f))[:1])
