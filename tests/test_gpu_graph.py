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
