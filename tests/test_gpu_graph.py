"""Fixed-capacity batches captured into CUDA graphs: replays with new inputs
in the same pinned arrays give the results of the ordinary batch path bit
for bit (clear air, aerosol extinction)."""
import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _pin(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()


def _shift(geom, dz):
    g = {k: np.array(v, dtype=np.float64) for k, v in geom.items()}
    g["vpz"] = g["vpz"] + dz
    return g


def test_graph_replay_clear_air(workdir):
    import torch
    from jscat import api, structs as S, synth
    ctlkw, atm, geom = synth.clear_limb_case(workdir)
    ctl = S.make_ctl(**ctlkw)
    n = len(geom["obsz"])
    inp0 = synth.batch_from([atm], np.zeros(n, np.int32), geom)
    inp1 = synth.batch_from([atm], np.zeros(n, np.int32), _shift(geom, 0.37))
    m = api.Model(ctl)
    stream = torch.cuda.Stream()
    gb = api.GraphBatch(m, ctl, inp0, stream.cuda_stream, _pin)
    try:
        for inp in (inp0, inp1, inp0):
            ref = api.formod_batch(ctl, inp, model=m)
            gb.launch(inp)
            stream.synchronize()
            gb.status()
            np.testing.assert_array_equal(gb.out["rad"], ref["rad"])
            np.testing.assert_array_equal(gb.out["tau"], ref["tau"])
            np.testing.assert_array_equal(gb.out["nlos"], ref["nlos"])
    finally:
        gb.close()
        m.close()


def test_graph_replay_aerosol_extinction(workdir):
    import torch
    from jscat import api, structs as S, synth
    from make_golden_shim import aerosol_case
    g = dict(np.load(GOLDEN + "/aerosol_ext_beta_a.npz"))
    aero = S.AeroT.from_buffer_copy(g["aero"].tobytes())
    ctlkw, atm, geom, _ = aerosol_case(workdir, 0)
    ctl = S.make_ctl(**ctlkw)
    n = len(geom["obsz"])
    inp0 = synth.batch_from([atm], np.zeros(n, np.int32), geom)
    inp1 = synth.batch_from([atm], np.zeros(n, np.int32), _shift(geom, -0.61))
    m = api.Model(ctl)
    stream = torch.cuda.Stream()
    gb = api.GraphBatch(m, ctl, inp0, stream.cuda_stream, _pin, aero=aero)
    try:
        for inp in (inp0, inp1):
            ref = api.formod_batch(ctl, inp, model=m, aero=aero)
            gb.launch(inp)
            stream.synchronize()
            gb.status()
            np.testing.assert_array_equal(gb.out["rad"], ref["rad"])
            np.testing.assert_array_equal(gb.out["nlos"], ref["nlos"])
    finally:
        gb.close()
        m.close()


def test_graph_replay_single_scattering(workdir):
    """A single-scattering batch (SCA_MULT=1) in fixed-capacity mode: the
    scattering points are counted and listed on the device and the
    secondary and solar pencils run in a fixed number of rounds, so upload
    + run + download replay from a CUDA graph.  Replays with day and night
    inputs give the ordinary batch path's radiances bit for bit, and the
    reference's within the parity bar."""
    import torch
    from jscat import api, structs as S, synth
    from make_golden_shim import aerosol_case
    from helpers import max_rel
    g = dict(np.load(GOLDEN + "/aerosol_sca1_day.npz"))
    aero = S.AeroT.from_buffer_copy(g["aero"].tobytes())
    ctlkw, atm, geom, _ = aerosol_case(workdir, 1)
    ctl = S.make_ctl(**ctlkw)
    n = len(geom["obsz"])
    day = dict(geom, time=np.full(n, 43200.0))
    night = dict(geom, time=np.zeros(n))
    inp_day = synth.batch_from([atm], np.zeros(n, np.int32), day)
    inp_night = synth.batch_from([atm], np.zeros(n, np.int32), night)
    m = api.Model(ctl)
    stream = torch.cuda.Stream()
    gb = api.GraphBatch(m, ctl, inp_day, stream.cuda_stream, _pin, aero=aero)
    try:
        for inp in (inp_day, inp_night, inp_day):
            ref = api.formod_batch(ctl, inp, model=m, aero=aero)
            gb.launch(inp)
            stream.synchronize()
            gb.status()
            np.testing.assert_array_equal(gb.out["nlos"], ref["nlos"])
            np.testing.assert_array_equal(gb.out["rad"], ref["rad"])
            np.testing.assert_array_equal(gb.out["tau"], ref["tau"])
        gb.launch(inp_day)
        stream.synchronize()
        assert max_rel(gb.out["rad"], g["rad"]) <= 1e-9
    finally:
        gb.close()
        m.close()


def test_fixed_scattering_capacity_overflow(workdir):
    """More scattering points than the fixed capacity: the run reports
    JSC_ERR_QUEUE and the device stays usable."""
    from jscat import api, lib as L, structs as S, synth
    from make_golden_shim import aerosol_case
    g = dict(np.load(GOLDEN + "/aerosol_sca1_day.npz"))
    aero = S.AeroT.from_buffer_copy(g["aero"].tobytes())
    ctlkw, atm, geom, _ = aerosol_case(workdir, 1)
    ctl = S.make_ctl(**ctlkw)
    n = len(geom["obsz"])
    inp = synth.batch_from([atm], np.zeros(n, np.int32), geom)
    m = api.Model(ctl)
    b = api.Batch(m, ctl, 1, len(inp["z"]), n)
    try:
        b.set_aero(aero)
        lib = L.load()
        L.check(lib.jsc_batch_set_fixed_points(b.h, 50), "jsc_batch_set_fixed_points")
        L.check(lib.jsc_batch_set_fixed(b.h, 1), "jsc_batch_set_fixed")
        b.upload(inp)
        b.run()
        with pytest.raises(L.JscError) as e:
            b.download()
        assert e.value.status == 7  # JSC_ERR_QUEUE
        out = api.formod_batch(ctl, inp, model=m, aero=aero)
        assert np.all(np.isfinite(out["rad"]))
    finally:
        b.close()
        m.close()


def test_device_wait_watchdog():
    """The multi-block prefix scan's waits are bounded: with a tile that
    never publishes its sum (a flag nothing sets) and a budget of one poll
    its successor gives up with JSC_ERR_WATCHDOG instead of hanging; with
    the default budget and no stall the scan is exact; the device stays
    usable after the give-up."""
    from jscat import api
    assert api.scan_selftest(n=300_000) == 0
    assert api.scan_selftest(n=300_000, budget=1, stall=0) == 8   # JSC_ERR_WATCHDOG
    assert api.scan_selftest(n=300_000, budget=1, stall=37) == 8
    assert api.scan_selftest(n=1) == 0
    assert api.scan_selftest(n=300_000) == 0
