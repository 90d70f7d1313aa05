"""GPU parity of the aerosol/cloud optical properties (jsc_get_opt_prop:
the Bohren-Huffman Mie series on the GPU, the log-normal size integral and
the layer sums on the host) against the reference's own read_aero +
get_opt_prop (golden aero_t fixtures made by make_golden.py: a sulfate-like
layer on 16 channels, an ice-cloud-like layer with size parameters up to
several hundred on 8 channels, and two layers of three modes, two Mie and
one external database).  Bars: layer structure exact; extinction,
scattering, absorption and phase function within 1e-12 relative (the
series runs in FP64 like the reference's and the size integral sums in the
reference's order; only the rounding of the complex arithmetic differs,
measured at 4e-14)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12

CASES = [("aero_sulfate16", "sulfate_layer_files", 1), ("aero_ice8", "ice_layer_files", 1),
         ("aero_layers8", "layered_aero_files", 3)]


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))


@pytest.mark.parametrize("name,files,sca_n", CASES)
def test_opt_prop_matches_reference(workdir, name, files, sca_n):
    from jscat import api, structs as S, synth
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    ref = S.AeroT.from_buffer_copy(d["aero"].tobytes())
    nus = list(d["nus"])
    aerofile = getattr(synth, files)(os.path.join(workdir, "aero"))
    ctl = S.make_ctl(synth.CFG0_EMITTERS, nus, "-", sca_n=sca_n)
    aero = api.get_opt_prop(ctl, api.read_aero(ctl, aerofile))
    nl, nd = ref.nl, len(nus)
    assert aero.nl == nl
    for f in ("nmod", "top", "bottom", "trans"):
        np.testing.assert_array_equal(S.arr(getattr(aero, f))[:nl], S.arr(getattr(ref, f))[:nl])
    for f in ("beta_e", "beta_s", "beta_a"):
        assert _rel(S.arr(getattr(aero, f))[:nl, :nd], S.arr(getattr(ref, f))[:nl, :nd]) <= REL_TOL, f
    assert _rel(S.arr(aero.p)[:nl, :nd], S.arr(ref.p)[:nl, :nd]) <= REL_TOL
