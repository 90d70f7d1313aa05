"""jsc_formod_batch_noalloc (static device scratch, no allocation) against
jsc_formod_batch on the same inputs: two calls in a row must both agree
with the allocating entry point within the parity tolerance, and an input
beyond the scratch must be refused with a clear error before any GPU work.
Collected last so it also runs after every other GPU test in one process."""
import numpy as np
import pytest

from helpers import max_rel

pytestmark = pytest.mark.gpu

REL_TOL = 1e-9


def _cases(workdir):
    from jscat import synth
    from make_golden_shim import mixed_case
    ctlkw, atm, geom = synth.clear_limb_case(workdir)
    yield "clear_limb", ctlkw, synth.batch_from([atm], np.zeros(len(geom["obsz"]), np.int32), geom)
    ctlkw, atms, ray_atm, geom = mixed_case(workdir)
    yield "mixed_batch", ctlkw, synth.batch_from(atms, ray_atm, geom)


def test_noalloc_matches_formod_batch(workdir):
    from jscat import api, structs as S
    for name, ctlkw, inp in _cases(workdir):
        ctl = S.make_ctl(**ctlkw)
        m = api.Model(ctl)
        try:
            ref = api.formod_batch(ctl, inp, model=m)
            for call in range(2):
                out = api.formod_batch_noalloc(ctl, inp, m)
                np.testing.assert_array_equal(out["nlos"], ref["nlos"], err_msg=name)
                assert max_rel(out["rad"], ref["rad"]) <= REL_TOL, (name, call)
                assert max_rel(out["tau"], ref["tau"]) <= REL_TOL, (name, call)
                np.testing.assert_allclose(out["tpz"], ref["tpz"], rtol=1e-12, atol=1e-12)
        finally:
            m.close()


def test_noalloc_more_than_eight_emitters(workdir):
    """Ten emitters take the wide EGA kernel (ng > 8); the no-allocation
    entry point must agree with jsc_formod_batch there too, twice in a row."""
    from jscat import api, structs as S, synth
    emitters = synth.CFG1_EMITTERS + ["F11", "F12"]
    ctlkw, atms, ray_atm, geom = synth.batched_case(
        workdir, n_rays=24, rays_per_atm=12, seed=20261206, emitters=emitters,
        nus=synth.CFG1_NU[::16])
    inp = synth.batch_from(atms, ray_atm, geom)
    ctl = S.make_ctl(**ctlkw)
    assert ctl.ng == 10
    m = api.Model(ctl)
    try:
        ref = api.formod_batch(ctl, inp, model=m)
        for call in range(2):
            out = api.formod_batch_noalloc(ctl, inp, m)
            np.testing.assert_array_equal(out["nlos"], ref["nlos"])
            assert max_rel(out["rad"], ref["rad"]) <= REL_TOL, call
            assert max_rel(out["tau"], ref["tau"]) <= REL_TOL, call
    finally:
        m.close()


def test_noalloc_zero_rays(workdir):
    """A batch without rays returns JSC_OK after the hydrostatic balance
    alone (one kernel), and the scratch serves a full call afterwards."""
    from jscat import api, structs as S, synth
    ctlkw, atm, geom = synth.clear_limb_case(workdir)
    ctl = S.make_ctl(**ctlkw)
    full = synth.batch_from([atm], np.zeros(len(geom["obsz"]), np.int32), geom)
    empty = dict(full)
    for k in ("ray_atm", "time", "obsz", "obslon", "obslat", "vpz", "vplon", "vplat"):
        empty[k] = full[k][:0]
    m = api.Model(ctl)
    try:
        ref = api.formod_batch(ctl, full, model=m)
        before = api.launch_count()
        out = api.formod_batch_noalloc(ctl, empty, m)
        assert api.launch_count() - before == 1
        assert out["rad"].shape == (0, ctl.nd)
        out = api.formod_batch_noalloc(ctl, full, m)
        assert max_rel(out["rad"], ref["rad"]) <= REL_TOL
    finally:
        m.close()


def _tiled(synth, atm, geom, n):
    g = {k: np.resize(np.asarray(v, dtype=np.float64), n) for k, v in geom.items()}
    return synth.batch_from([atm], np.zeros(n, np.int32), g)


def test_noalloc_rejects_input_beyond_scratch(workdir):
    from jscat import api, lib as L, structs as S, synth
    ctlkw, atm, geom = synth.clear_limb_case(workdir)
    ctl = S.make_ctl(**ctlkw)
    small = synth.batch_from([atm], np.zeros(len(geom["obsz"]), np.int32), geom)
    m = api.Model(ctl)
    try:
        ref = api.formod_batch(ctl, small, model=m)
        # 450,000 rays: inputs and outputs alone exceed the 64 MiB scratch,
        # refused on the host before any GPU work.
        with pytest.raises(L.JscError) as e:
            api.formod_batch_noalloc(ctl, _tiled(synth, atm, geom, 450_000), m)
        assert e.value.status == 1 and "before any LOS point" in str(e.value)
        # 6,100 limb rays of ~270 LOS points: more points than the scratch
        # holds, refused after the counting pass, before any LOS record.
        with pytest.raises(L.JscError) as e:
            api.formod_batch_noalloc(ctl, _tiled(synth, atm, geom, 6100), m)
        assert e.value.status == 1 and "LOS points" in str(e.value)
        # The scratch serves the next call as before.
        out = api.formod_batch_noalloc(ctl, small, m)
        assert max_rel(out["rad"], ref["rad"]) <= REL_TOL
    finally:
        m.close()
