"""GPU parity against the reference forward model.

Golden fixtures hold the reference's own FP64 outputs (tests/golden,
made by make_golden.py with the reference compiled from its sources) for
seeded synthetic inputs regenerated here, plus the per-(ray, channel)
checksums of every emissivity-table index the EGA interpolation selected
(from the C restatement, which reproduces the reference bit for bit).
Bars: LOS point counts and table indices exactly equal, brightness
temperature within 0.01 K, radiance/transmittance within 1e-9 relative
(the GPU keeps the reference's FP64/FP32 operation order; only last-bit
differences of the CUDA and glibc transcendental functions remain)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from helpers import bt_error, max_rel

pytestmark = pytest.mark.gpu

BT_TOL_K = 0.01
REL_TOL = 1e-9


def _load(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def _geom(g):
    return {k[5:]: v for k, v in g.items() if k.startswith("geom_")}


def _check_tables(g, ctlkw):
    from make_golden_shim import tables_digest
    assert tables_digest(ctlkw["tblbase"], ctlkw["emitters"], ctlkw["nus"]) == str(g["table_sha256"])


def test_clear_limb_dropin_formod(workdir):
    from jscat import structs as S, synth, api
    g = _load("clear_limb")
    ctlkw, atm, geom = synth.clear_limb_case(workdir)
    _check_tables(g, ctlkw)
    ctl = S.make_ctl(**ctlkw)
    a = S.make_atm(atm["z"], atm["p"], atm["t"], atm["q"], atm["k"])
    obs = S.make_obs(geom["obsz"], geom["obslat"], geom["vpz"], geom["vplat"])
    api.formod(ctl, a, obs)
    nr, nd = obs.nr, ctl.nd
    rad = S.arr(obs.rad)[:nd, :nr].T
    tau = S.arr(obs.tau)[:nd, :nr].T
    assert bt_error(rad, g["rad"], ctlkw["nus"]) <= BT_TOL_K
    assert max_rel(rad, g["rad"]) <= REL_TOL
    assert max_rel(tau, g["tau"]) <= REL_TOL
    np.testing.assert_allclose(S.arr(obs.tpz)[:nr], g["tpz"], rtol=1e-9, atol=1e-9)


def test_clear_limb_fov_formod(workdir):
    """Drop-in formod with a field-of-view shape (formod_fov,
    src/forwardmodel.c:156-220) against the reference run with the same
    shape file."""
    from jscat import structs as S, api
    from make_golden_shim import fov_case
    g = _load("clear_limb_fov")
    ctlkw, atm, geom = fov_case(workdir)
    _check_tables(g, ctlkw)
    ctl = S.make_ctl(**ctlkw)
    a = S.make_atm(atm["z"], atm["p"], atm["t"], atm["q"], atm["k"])
    obs = S.make_obs(geom["obsz"], geom["obslat"], geom["vpz"], geom["vplat"])
    api.formod(ctl, a, obs)
    nr, nd = obs.nr, ctl.nd
    rad = S.arr(obs.rad)[:nd, :nr].T
    tau = S.arr(obs.tau)[:nd, :nr].T
    assert bt_error(rad, g["rad"], ctlkw["nus"]) <= BT_TOL_K
    assert max_rel(rad, g["rad"]) <= REL_TOL
    assert max_rel(tau, g["tau"]) <= REL_TOL


@pytest.mark.parametrize("ip", [2, 3])
def test_curtain_formod(workdir, ip):
    """Drop-in formod through a horizontally varying atmosphere (five
    profiles along the track): IP=2 blends the two nearest profiles, IP=3
    weights every point within CZ/CX (src/atmosphere.c:324-482), in the ray
    tracer's state and refraction lookups; against the reference."""
    from jscat import structs as S, synth, api
    from make_golden_shim import curtain_ctl
    g = _load("curtain_ip%d" % ip)
    ctlkw, atm, geom = synth.curtain_case(workdir)
    _check_tables(g, ctlkw)
    ctl = S.make_ctl(**curtain_ctl(ctlkw, ip))
    a = S.make_atm(atm["z"], atm["p"], atm["t"], atm["q"], atm["k"], atm["lon"], atm["lat"])
    obs = S.make_obs(geom["obsz"], geom["obslat"], geom["vpz"], geom["vplat"])
    api.formod(ctl, a, obs)
    nr, nd = obs.nr, ctl.nd
    rad = S.arr(obs.rad)[:nd, :nr].T
    tau = S.arr(obs.tau)[:nd, :nr].T
    assert bt_error(rad, g["rad"], ctlkw["nus"]) <= BT_TOL_K
    assert max_rel(rad, g["rad"]) <= REL_TOL
    assert max_rel(tau, g["tau"]) <= REL_TOL
    np.testing.assert_allclose(S.arr(obs.tpz)[:nr], g["tpz"], rtol=1e-9, atol=1e-9)
    np.testing.assert_allclose(S.arr(obs.tplat)[:nr], g["tplat"], rtol=1e-9, atol=1e-9)


@pytest.mark.parametrize("ip", [2, 3])
def test_curtain_aerosol_extinction(workdir, ip):
    """IP=2/3 with aerosol extinction (SCA_MULT=0, beta_e): the layer-edge
    points of the refined line of sight take their state from the same
    horizontal interpolation; against the reference."""
    from jscat import structs as S, synth, api
    from make_golden_shim import curtain_ctl
    g = _load("curtain_ip%d_ext" % ip)
    ctlkw, atm, geom = synth.curtain_case(workdir)
    _check_tables(g, ctlkw)
    ctl = S.make_ctl(**curtain_ctl(dict(ctlkw, sca_n=1, sca_mult=0, sca_ext="beta_e"), ip))
    a = S.make_atm(atm["z"], atm["p"], atm["t"], atm["q"], atm["k"], atm["lon"], atm["lat"])
    obs = S.make_obs(geom["obsz"], geom["obslat"], geom["vpz"], geom["vplat"])
    aero = S.AeroT.from_buffer_copy(g["aero"].tobytes())
    api.formod(ctl, a, obs, aero)
    nr, nd = obs.nr, ctl.nd
    rad = S.arr(obs.rad)[:nd, :nr].T
    assert bt_error(rad, g["rad"], ctlkw["nus"]) <= BT_TOL_K
    assert max_rel(rad, g["rad"]) <= REL_TOL
    assert max_rel(S.arr(obs.tau)[:nd, :nr].T, g["tau"]) <= REL_TOL


# EGA kernel families: -1 the default (variant 17, lanes over a tile of
# rays with the transfer step taken in turn by the emitter warps), 6 a
# thread per (ray, channel), 9 a lane per (ray, channel, emitter), 14 lanes
# over a tile of rays with a transfer warp
VARIANTS = [-1, 6, 9, 14]


@pytest.mark.parametrize("variant", VARIANTS)
def test_clear_limb_batch_indices(workdir, variant):
    from jscat import structs as S, synth, api
    g = _load("clear_limb")
    ctlkw, atm, geom = synth.clear_limb_case(workdir)
    ctl = S.make_ctl(**ctlkw)
    out = api.formod_batch(ctl, synth.batch_from([atm], np.zeros(len(geom["obsz"]), np.int32), geom),
                           digest=True, variant=variant)
    np.testing.assert_array_equal(out["nlos"], g["nlos"])
    np.testing.assert_array_equal(out["digest"], g["digest"])
    assert max_rel(out["rad"], g["rad"]) <= REL_TOL


@pytest.mark.parametrize("variant", VARIANTS)
def test_mixed_batch(workdir, variant):
    from jscat import synth, api, structs as S
    from make_golden_shim import mixed_case
    g = _load("mixed_batch")
    ctlkw, atms, ray_atm, geom = mixed_case(workdir)
    _check_tables(g, ctlkw)
    ctl = S.make_ctl(**ctlkw)
    out = api.formod_batch(ctl, synth.batch_from(atms, ray_atm, geom), digest=True, variant=variant)
    np.testing.assert_array_equal(out["nlos"], g["nlos"])
    np.testing.assert_array_equal(out["digest"], g["digest"])
    assert bt_error(out["rad"], g["rad"], ctlkw["nus"]) <= BT_TOL_K
    assert max_rel(out["rad"], g["rad"]) <= REL_TOL
    assert max_rel(out["tau"], g["tau"]) <= REL_TOL
    np.testing.assert_allclose(out["tpz"], g["tpz"], rtol=1e-9, atol=1e-9)


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("ext", ["beta_a", "beta_e"])
def test_aerosol_extinction(workdir, ext, variant):
    """Aerosol layer with extinction only (SCA_MULT=0): layer-edge LOS
    refinement (add_aerosol_layers) and the aerosol RT branch."""
    from jscat import synth, api, structs as S
    from make_golden_shim import aerosol_case
    g = _load("aerosol_ext_" + ext)
    ctlkw, atm, geom, aerofile = aerosol_case(workdir, 0, sca_ext=ext)
    _check_tables(g, ctlkw)
    aero = S.AeroT.from_buffer_copy(g["aero"].tobytes())
    ctl = S.make_ctl(**ctlkw)
    out = api.formod_batch(ctl, synth.batch_from([atm], np.zeros(len(geom["obsz"]), np.int32), geom),
                           digest=True, aero=aero, variant=variant)
    np.testing.assert_array_equal(out["nlos"], g["nlos"])
    np.testing.assert_array_equal(out["digest"], g["digest"])
    assert bt_error(out["rad"], g["rad"], ctlkw["nus"]) <= BT_TOL_K
    assert max_rel(out["rad"], g["rad"]) <= REL_TOL
    assert max_rel(out["tau"], g["tau"]) <= REL_TOL


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("when", ["night", "day"])
def test_aerosol_single_scattering(workdir, when, variant):
    """Single scattering (SCA_MULT=1) on the sulfate-like layer: secondary
    pencils, source integral and, by day, the solar term (srcfunc_sca_1d
    and srcfunc_sca_sun), against the reference's own outputs.  The
    scattering term alone (radiance minus the extinction-only radiance) is
    checked as well, so that an error in the source cannot hide below the
    radiance tolerance."""
    from jscat import synth, api, structs as S
    from make_golden_shim import aerosol_case
    g = _load("aerosol_sca1_" + when)
    ge = _load("aerosol_ext_beta_a")
    ctlkw, atm, geom, aerofile = aerosol_case(workdir, 1)
    geom["time"] = np.full(len(geom["obsz"]), 0.0 if when == "night" else 43200.0)
    _check_tables(g, ctlkw)
    aero = S.AeroT.from_buffer_copy(g["aero"].tobytes())
    ctl = S.make_ctl(**ctlkw)
    out = api.formod_batch(ctl, synth.batch_from([atm], np.zeros(len(geom["obsz"]), np.int32), geom),
                           aero=aero, variant=variant)
    np.testing.assert_array_equal(out["nlos"], g["nlos"])
    assert bt_error(out["rad"], g["rad"], ctlkw["nus"]) <= BT_TOL_K
    assert max_rel(out["rad"], g["rad"]) <= REL_TOL
    assert max_rel(out["tau"], g["tau"]) <= REL_TOL
    d_ref = g["rad"] - ge["rad"]
    d_gpu = out["rad"] - ge["rad"]
    assert np.max(np.abs(d_gpu - d_ref)) <= 1e-6 * np.max(np.abs(d_ref))


def test_dropin_formod_single_scattering(workdir):
    """The drop-in formod() on the reference's structs with an aerosol layer
    and SCA_MULT=1 (daytime: thermal and solar scattering source)."""
    from jscat import structs as S, synth, api
    from make_golden_shim import aerosol_case
    g = _load("aerosol_sca1_day")
    ctlkw, atm, geom, aerofile = aerosol_case(workdir, 1)
    ctl = S.make_ctl(**ctlkw)
    a = S.make_atm(atm["z"], atm["p"], atm["t"], atm["q"], atm["k"])
    n = len(geom["obsz"])
    obs = S.make_obs(geom["obsz"], geom["obslat"], geom["vpz"], geom["vplat"],
                     geom["obslon"], geom["vplon"], np.full(n, 43200.0))
    aero = S.AeroT.from_buffer_copy(g["aero"].tobytes())
    api.formod(ctl, a, obs, aero)
    rad = S.arr(obs.rad)[:ctl.nd, :n].T
    assert bt_error(rad, g["rad"], ctlkw["nus"]) <= BT_TOL_K
    assert max_rel(rad, g["rad"]) <= REL_TOL


def test_double_scattering_matches_reference_nan(workdir):
    """SCA_MULT=2: the reference returns NaN for this limb ray (second-order
    pencils starting on layer-edge points get a zero-length chord and 0/0
    in the continua); the GPU path follows the same arithmetic and returns
    NaN in the same channels, with the same LOS point count."""
    from jscat import synth, api, structs as S
    from make_golden_shim import aerosol_case
    g = _load("aerosol_sca2")
    ga = _load("aerosol_sca1_day")
    nus = [float(v) for v in g["nus"]]
    ctlkw, atm, _, _ = aerosol_case(workdir, 2, n_rays=1, nus=nus)
    geom = _geom(g)
    aero_full = S.AeroT.from_buffer_copy(ga["aero"].tobytes())
    aero = _aero_for(aero_full, ga, nus)
    ctl = S.make_ctl(**ctlkw)
    out = api.formod_batch(ctl, synth.batch_from([atm], np.zeros(1, np.int32), geom), aero=aero)
    np.testing.assert_array_equal(out["nlos"], g["nlos"])
    np.testing.assert_array_equal(np.isnan(out["rad"]), np.isnan(g["rad"]))


def _aero_for(aero, g, nus):
    """The sulfate layer's optical properties on the channels nus (taken from
    the 4-channel fixture's aero_t, whose channels include them)."""
    import ctypes as C
    from jscat import synth
    have = [synth.CFG2_NU[i] for i in (0, 5, 10, 15)]
    idx = [have.index(v) for v in nus]
    from jscat import structs as S
    out = S.AeroT.from_buffer_copy(bytes(aero))
    for il in range(aero.nl):
        for j, i in enumerate(idx):
            out.beta_e[il][j] = aero.beta_e[il][i]
            out.beta_s[il][j] = aero.beta_s[il][i]
            out.beta_a[il][j] = aero.beta_a[il][i]
            for a in range(181):
                out.p[il][j][a] = aero.p[il][i][a]
    return out


# Every launch variant the autotuner can pick: 0-8 a thread per (ray,
# channel), 9-13 a lane per (ray, channel, emitter), 14-20 lanes over a
# tile of rays with a warp per emitter (14-16 with a transfer warp, 17-20
# with the transfer step taken in turn).
ALL_VARIANTS = list(range(21))


@pytest.fixture(scope="module",
                params=["headline_batch", "continuum_bands", "emitters12", "emitters20"])
def shape_case(request, workdir):
    """The benchmark's 64-channel, 8-emitter shape (O2 continuum in its top
    channels), the O2/N2 continuum-band case and two cases with more
    emitters than the benchmark (12: the ray-tile kernels' 16-warp form;
    20: above the ray-tile kernels' 16, the 32-lane groups of the lane
    kernel and the widest thread-per-channel kernel), with one device model
    per case shared by all launch variants."""
    from jscat import api, structs as S, synth
    from make_golden_shim import band_case, emitters_case, headline_case
    name = request.param
    g = _load(name)
    if name.startswith("emitters"):
        ctlkw, atms, ray_atm, geom = emitters_case(workdir, int(name[len("emitters"):]))
    else:
        ctlkw, atms, ray_atm, geom = (headline_case if name == "headline_batch"
                                      else band_case)(workdir)
    _check_tables(g, ctlkw)
    ctl = S.make_ctl(**ctlkw)
    m = api.Model(ctl)
    yield name, g, ctlkw, ctl, synth.batch_from(atms, ray_atm, geom), m
    m.close()


@pytest.mark.parametrize("variant", ALL_VARIANTS)
def test_every_launch_variant(shape_case, variant):
    """Each launch variant on the headline shape, the continuum-band
    channels and the many-emitter cases: LOS point counts and every EGA
    table index (digests) exactly the reference's, radiances within 1e-9
    relative and 0.01 K."""
    from jscat import api
    name, g, ctlkw, ctl, inp, m = shape_case
    out = api.formod_batch(ctl, inp, model=m, digest=True, variant=variant)
    np.testing.assert_array_equal(out["nlos"], g["nlos"], err_msg=name)
    np.testing.assert_array_equal(out["digest"], g["digest"], err_msg=name)
    assert bt_error(out["rad"], g["rad"], ctlkw["nus"]) <= BT_TOL_K
    assert max_rel(out["rad"], g["rad"]) <= REL_TOL
    assert max_rel(out["tau"], g["tau"]) <= REL_TOL
    np.testing.assert_allclose(out["tpz"], g["tpz"], rtol=1e-9, atol=1e-9)


def test_formod_pencil_clear_and_scattering(workdir):
    """The drop-in formod_pencil (one ray on the GPU, atm as given) on rays
    of the clear limb case and of the daytime single-scattering case, after
    the hydrostatic balance formod applies: the reference's radiances."""
    from jscat import structs as S, synth, api
    from make_golden_shim import aerosol_case
    g = _load("clear_limb")
    ctlkw, atm, geom = synth.clear_limb_case(workdir)
    ctl = S.make_ctl(**ctlkw)
    a = S.make_atm(atm["z"], atm["p"], atm["t"], atm["q"], atm["k"])
    obs = S.make_obs(geom["obsz"], geom["obslat"], geom["vpz"], geom["vplat"])
    api.formod(ctl, a, obs)          # hydrostatic balance of a, as formod leaves it
    nd = ctl.nd
    for ir in (0, 17, 60):
        for id_ in range(nd):
            obs.rad[id_][ir] = obs.tau[id_][ir] = -1.0
        api.formod_pencil(ctl, a, obs, scattering=ctl.sca_mult if ctl.sca_n else 0, ir=ir)
        rad = S.arr(obs.rad)[:nd, ir]
        assert max_rel(rad, g["rad"][ir]) <= REL_TOL
        assert max_rel(S.arr(obs.tau)[:nd, ir], g["tau"][ir]) <= REL_TOL
    ga = _load("aerosol_sca1_day")
    ctlkw, atm, geom, _ = aerosol_case(workdir, 1)
    n = len(geom["obsz"])
    ctl = S.make_ctl(**ctlkw)
    a = S.make_atm(atm["z"], atm["p"], atm["t"], atm["q"], atm["k"])
    obs = S.make_obs(geom["obsz"], geom["obslat"], geom["vpz"], geom["vplat"],
                     geom["obslon"], geom["vplon"], np.full(n, 43200.0))
    aero = S.AeroT.from_buffer_copy(ga["aero"].tobytes())
    api.formod(ctl, a, obs, aero)
    for ir in (3, 11):
        api.formod_pencil(ctl, a, obs, aero, scattering=1, ir=ir)
        assert max_rel(S.arr(obs.rad)[:ctl.nd, ir], ga["rad"][ir]) <= REL_TOL


def test_double_scattering_per_depth_pencils(workdir):
    """Depth 2 with per-order pencil counts (20 pencils per point of order 2,
    10 of order 1) through the ice-cloud layer, CO2/H2O continua off: the
    radiances of the C restatement with the same counts
    (tests/golden/ice_sca2_port.npz)."""
    from jscat import api, structs as S, synth
    from make_golden_shim import ice_depth2_case
    g = _load("ice_sca2_port")
    ctlkw, atm, geom, nalpha = ice_depth2_case(workdir)
    _check_tables(g, ctlkw)
    ctl = S.make_ctl(**ctlkw)
    aero = S.AeroT.from_buffer_copy(g["aero"].tobytes())
    m = api.Model(ctl)
    inp = synth.batch_from([atm], np.zeros(len(geom["obsz"]), np.int32), geom)
    b = api.Batch(m, ctl, 1, len(inp["z"]), len(geom["obsz"]))
    try:
        b.set_aero(aero)
        for depth, na in nalpha.items():
            b.set_nalpha_depth(depth, na)
        b.upload(inp)
        b.run()
        out = b.download()
    finally:
        b.close()
        m.close()
    np.testing.assert_array_equal(out["nlos"], g["nlos"])
    assert np.all(np.isfinite(g["rad"]))
    assert bt_error(out["rad"], g["rad"], ctlkw["nus"]) <= BT_TOL_K
    assert max_rel(out["rad"], g["rad"]) <= REL_TOL
