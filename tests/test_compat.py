"""The non-hot helpers of forwardmodel.h that the drop-in library exports
for link compatibility (read_tbl, intpol_tbl, intpol_tbl_eps/_u,
locate_tbl, formod_continua, srcfunc_planck), against the reference's own
functions (oracle/_ref/libjurassic_ref.so) on the same line of sight: a
limb ray of the clear-air case traced by the reference's raytrace.  CPU
only: these helpers work on the caller's host structs."""
import os

import numpy as np
import pytest

from conftest import REPO


@pytest.fixture(scope="module")
def both(workdir):
    from jscat import lib as L, synth
    from oracle import refrun
    if not refrun.available():
        pytest.skip("reference build absent")
    ctlkw, atm, geom = synth.clear_limb_case(workdir)
    los = refrun.reference_los(ctlkw, atm, geom, ir=20)
    ref = refrun.forwardmodel_helpers(ctlkw, los, lib=refrun.REF_LIB)
    mine = refrun.forwardmodel_helpers(ctlkw, los, lib=L.LIB_PATH)
    return ref, mine


def test_read_tbl_matches_reference(both):
    ref, mine = both
    for k in ("np", "nt", "nu", "p", "t", "u00", "eps00"):
        assert np.array_equal(ref[k], mine[k]), k


def test_intpol_tbl_matches_reference(both):
    """EGA transmittances along the ray (path state carried from point to
    point), bit for bit."""
    ref, mine = both
    assert ref["tau_seg"].shape[0] > 100
    assert np.array_equal(ref["tau_seg"], mine["tau_seg"])
    assert np.array_equal(ref["tau_path"], mine["tau_path"])
    assert np.array_equal(ref["lookups"], mine["lookups"])
    assert np.array_equal(ref["locate"], mine["locate"])


def test_continua_and_planck_match_reference(both):
    ref, mine = both
    np.testing.assert_allclose(mine["beta"], ref["beta"], rtol=1e-13, atol=0)
    assert np.array_equal(ref["src"], mine["src"])
