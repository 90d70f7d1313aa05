"""Scattering-source surrogate on the GPU: training gradients against the
FP64 numpy restatement (oracle/mlp_ref.py), training on plain-path samples,
radiances with the surrogate against the plain path, envelope fallback and
rejection by the sampled check."""
import numpy as np
import pytest

from conftest import GOLDEN
from helpers import bt_error

pytestmark = pytest.mark.gpu


def test_training_gradients_match_cpu():
    from jscat import api
    from oracle import mlp_ref
    rng = np.random.default_rng(5)
    s = api.Surrogate(nd=6, seed=11)
    try:
        p = s.get_params()
        p = (p + rng.normal(0, 0.05, p.shape)).astype(np.float32)  # nonzero biases too
        s.set_params(p)
        x = rng.normal(0, 1, (200, 8)).astype(np.float32)
        t = rng.normal(0, 1, (200, 6)).astype(np.float32)
        loss, g = s.loss_grad(x, t)
        ref_loss, ref_g = mlp_ref.loss_and_grads(s.layers(p.astype(np.float64)), x, t)
        assert abs(loss - ref_loss) <= 1e-4 * abs(ref_loss)
        flat = np.concatenate([np.concatenate([gw.ravel(), gb]) for gw, gb in ref_g])
        # FP32 kernels against FP64: relative to the largest gradient
        assert np.max(np.abs(g - flat)) <= 2e-4 * np.max(np.abs(flat))
    finally:
        s.close()


def _sca_case(workdir, n_rays, times):
    from jscat import synth, structs as S
    from make_golden_shim import aerosol_case
    g = dict(np.load(GOLDEN + "/aerosol_sca1_day.npz"))
    aero = S.AeroT.from_buffer_copy(g["aero"].tobytes())
    ctlkw, atm, geom, _ = aerosol_case(workdir, 1, n_rays=n_rays)
    geom["time"] = np.resize(np.asarray(times, dtype=np.float64), n_rays)
    return ctlkw, atm, geom, aero


def test_surrogate_trains_and_replaces_plain_source(workdir):
    from jscat import api, synth, structs as S
    # training data: plain sources of limb rays at several times of day
    ctlkw, atm, geom, aero = _sca_case(workdir, 96, np.linspace(0, 86400, 7))
    ctl = S.make_ctl(**ctlkw)
    m = api.Model(ctl)
    inp = synth.batch_from([atm], np.zeros(96, np.int32), geom)
    b = api.Batch(m, ctl, 1, len(inp["z"]), 96)
    sur = api.Surrogate(ctl.nd, seed=3)
    try:
        b.set_aero(aero)
        b.set_nalpha(10)
        b.upload(inp)
        b.run()
        plain = b.download()
        feat, src = b.scatter_samples()
        assert len(feat) > 500 and np.all(src > 0)
        losses = sur.train(feat, src, epochs=60, batch=256, lr=3e-3)
        assert losses[-1] < 0.5 * losses[0]
        # surrogate path, everything inside the envelope, sampled check on
        b.set_surrogate(sur, tol_rel=0.5, check_stride=16)
        b.run()
        out = b.download()
        st = b.surrogate_stats()
        assert st["used"] and st["fallback"] == 0 and st["checked"] > 0
        assert st["max_rel_err"] < 0.5
        assert bt_error(out["rad"], plain["rad"], ctlkw["nus"]) <= 0.05
        # a tolerance the surrogate cannot meet: the batch falls back whole
        b.set_surrogate(sur, tol_rel=1e-9, check_stride=1)
        b.run()
        out2 = b.download()
        st2 = b.surrogate_stats()
        assert not st2["used"]
        np.testing.assert_array_equal(out2["rad"], plain["rad"])
    finally:
        sur.close()
        b.close()
        m.close()


def test_surrogate_envelope_fallback(workdir):
    """Points outside the training envelope (here: every point, the network
    was trained on features of another layer index) take the plain path and
    reproduce it exactly."""
    from jscat import api, synth, structs as S
    ctlkw, atm, geom, aero = _sca_case(workdir, 24, [43200.0])
    ctl = S.make_ctl(**ctlkw)
    m = api.Model(ctl)
    inp = synth.batch_from([atm], np.zeros(24, np.int32), geom)
    b = api.Batch(m, ctl, 1, len(inp["z"]), 24)
    sur = api.Surrogate(ctl.nd, seed=3)
    try:
        b.set_aero(aero)
        b.set_nalpha(10)
        b.upload(inp)
        b.run()
        plain = b.download()
        feat, src = b.scatter_samples()
        feat[:, 6] += 5.0  # train on a shifted layer index: real points fall outside
        sur.train(feat, src, epochs=2, batch=64, lr=1e-3)
        b.set_surrogate(sur, tol_rel=0.5, check_stride=0)
        b.run()
        out = b.download()
        st = b.surrogate_stats()
        assert st["fallback"] == st["points"] > 0
        np.testing.assert_array_equal(out["rad"], plain["rad"])
    finally:
        sur.close()
        b.close()
        m.close()


@pytest.mark.parametrize("nd", [4, 16, 40])
def test_tcgen05_inference_matches_mma_sync(nd):
    """The tcgen05 inference path (TMEM accumulators) and the mma.sync path
    run the same BF16 weights on the same features: their sources agree to
    the FP32 accumulation order."""
    from jscat import api
    rng = np.random.default_rng(9)
    s = api.Surrogate(nd=nd, seed=2)
    try:
        n = 300  # three 128-point tiles, the last one partial
        feat = rng.normal(0, 1, (n, 8)).astype(np.float32)
        src = np.exp(rng.normal(-3, 0.3, (n, nd)))
        s.train(feat, src, epochs=2, batch=64, lr=1e-3)  # sets the standardisation
        s.set_tensor_path(False)
        a = s.predict(feat)
        s.set_tensor_path(True)
        b = s.predict(feat)
        assert np.all(np.isfinite(b))
        assert np.max(np.abs(np.log(b) - np.log(a))) < 2e-3
    finally:
        s.close()


@pytest.mark.parametrize("nd", [4, 16, 40])
def test_tcgen05_inference_matches_fp32_restatement(nd):
    """The tcgen05 inference (BF16 operands, FP32 accumulators in tensor
    memory) against the numpy restatement of the same inference
    (oracle/mlp_ref.infer_bf16: the same BF16-rounded weights, features and
    hidden activations, FP64 sums, exact tanh).  The remaining differences
    are the FP32 accumulation order and the hardware tanh (relative error
    about 2^-11) before each BF16 rounding."""
    from jscat import api
    from oracle import mlp_ref
    rng = np.random.default_rng(13)
    s = api.Surrogate(nd=nd, seed=4)
    try:
        n = 600
        feat = rng.normal(0, 1, (n, 8)).astype(np.float32) * 3 + 10
        src = np.exp(rng.normal(-3, 0.5, (n, nd)))
        s.train(feat, src, epochs=3, batch=128, lr=2e-3)
        s.set_tensor_path(True)
        got = s.predict(feat)
        want = mlp_ref.infer_bf16(s.layers(s.get_params()), feat, *s.scaling())
        assert np.all(np.isfinite(got)) and np.all(got > 0)
        assert np.max(np.abs(np.log(got) - np.log(want))) < 3e-3
    finally:
        s.close()


def test_surrogate_accuracy_held_out(workdir):
    """Out-of-sample accuracy: the network is trained on the plain sources of
    limb rays A and then replaces the plain source on disjoint rays B
    (other tangent heights and times of day), with the benchmark's sampled
    check (api.SURROGATE_CHECK_TOL, every 16th point here): the surrogate
    path is kept and its brightness temperatures stay within 0.05 K of the
    plain path's."""
    from jscat import api, synth, structs as S
    from make_golden_shim import aerosol_case
    g = dict(np.load(GOLDEN + "/aerosol_sca1_day.npz"))
    aero = S.AeroT.from_buffer_copy(g["aero"].tobytes())
    ctlkw, atm, _, _ = aerosol_case(workdir, 1, n_rays=4)
    ctl = S.make_ctl(**ctlkw)
    rng = np.random.default_rng(21)

    def rays(th, times):
        geom = synth.limb_geometry(th)
        geom["time"] = times
        return synth.batch_from([atm], np.zeros(len(th), np.int32), geom)

    na, nb = 480, 96
    train = rays(rng.uniform(8.0, 30.0, na), rng.uniform(0.0, 86400.0, na))
    test = rays(rng.uniform(8.0, 30.0, nb), rng.uniform(0.0, 86400.0, nb))
    m = api.Model(ctl)
    b = api.Batch(m, ctl, 1, len(train["z"]), na)
    sur = api.Surrogate(ctl.nd, seed=3)
    try:
        b.set_aero(aero)
        b.set_nalpha(10)
        b.upload(train)
        b.run()
        feat, src = b.scatter_samples()
        sur.train(feat, src, epochs=200, batch=512, lr=3e-3)
        b.upload(test)
        b.run()
        plain = b.download()
        b.set_surrogate(sur, tol_rel=api.SURROGATE_CHECK_TOL, check_stride=16)
        b.run()
        out = b.download()
        st = b.surrogate_stats()
        assert st["points"] > 1000 and st["checked"] > 50
        assert st["fallback"] <= 0.05 * st["points"]
        assert st["used"], st
        assert bt_error(out["rad"], plain["rad"], ctlkw["nus"]) <= 0.05
    finally:
        sur.close()
        b.close()
        m.close()


def test_order1_surrogate_inside_double_scattering(workdir):
    """Depth-2 scattering through the ice-cloud layer with a surrogate for
    the order-1 sources only (jsc_batch_set_surrogate_depth, depth 1): the
    order-2 sources stay the plain integral over the order-1 pencils, whose
    own scattering points take the network.  Trained on the order-1 points
    of rays A, used on disjoint rays B: every chunk keeps the surrogate,
    and the brightness temperatures stay within 0.05 K of the plain path."""
    from jscat import api, synth, structs as S
    from make_golden_shim import ice_depth2_case
    ctlkw, atm, _, nalpha = ice_depth2_case(workdir)
    g = np.load(GOLDEN + "/ice_sca2_port.npz")
    aero = S.AeroT.from_buffer_copy(g["aero"].tobytes())
    ctl = S.make_ctl(**ctlkw)
    rng = np.random.default_rng(23)

    def rays(n):
        geom = synth.limb_geometry(rng.uniform(6.0, 14.0, n))
        geom["time"] = rng.uniform(0.0, 86400.0, n)
        return synth.batch_from([atm], np.zeros(n, np.int32), geom)

    na, nb = 192, 64
    train, test = rays(na), rays(nb)
    m = api.Model(ctl)
    b = api.Batch(m, ctl, 1, len(train["z"]), na)
    sur = api.Surrogate(ctl.nd, seed=4)
    try:
        b.set_aero(aero)
        for depth, na_ in nalpha.items():
            b.set_nalpha_depth(depth, na_)
        b.upload(train)
        b.run()
        feat, src = b.scatter_samples(depth=1)
        assert len(feat) > 10000 and np.all(np.isfinite(src))
        sur.train(feat, src, epochs=80, batch=4096, lr=3e-3)
        b.upload(test)
        b.run()
        plain = b.download()
        assert np.all(np.isfinite(plain["rad"]))
        b.set_surrogate(sur, tol_rel=api.SURROGATE_CHECK_TOL, check_stride=16, depth=1)
        b.run()
        out = b.download()
        st = b.surrogate_stats(depth=1)
        assert st["points"] > 1000 and st["checked"] > 50, st
        assert st["used"], st
        assert b.surrogate_stats()["points"] > 0 and not b.surrogate_stats()["used"]
        assert bt_error(out["rad"], plain["rad"], ctlkw["nus"]) <= 0.05
        # detached again: the plain path, bit for bit
        b.set_surrogate(None, depth=1)
        b.run()
        assert np.array_equal(b.download()["rad"], plain["rad"])
    finally:
        sur.close()
        b.close()
        m.close()
