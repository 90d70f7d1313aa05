"""The CPU oracle (oracle/jurassic_oracle.c) pinned against the reference:
bit for bit against the reference's outputs stored in tests/golden, and
against the reference's own example goldens (examples/org) where the
reference tree is present (this container; not on the GPU box)."""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import GOLDEN, REPO

from oracle import refpath  # noqa: E402

REF_EXAMPLES = refpath.reference_path("examples")
PORT = os.path.join(REPO, "oracle", "build", "libjscat_oracle.so")


def _golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


@pytest.fixture(scope="module")
def port():
    if not os.path.exists(PORT):
        import subprocess
        subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle"), "port"], check=True)
    return PORT


def test_port_bit_exact_clear_limb(workdir, port):
    from jscat import synth
    from oracle import refrun
    g = _golden("clear_limb")
    ctlkw, atm, geom = synth.clear_limb_case(workdir)
    r = refrun.run_port(ctlkw, [atm], np.zeros(len(geom["obsz"]), int), geom, los=True)
    assert np.array_equal(r["rad"], g["rad"])
    assert np.array_equal(r["tau"], g["tau"])
    assert np.array_equal(r["tpz"], g["tpz"])
    assert np.array_equal(r["nlos"], g["nlos"])
    assert np.array_equal(r["digest"], g["digest"])


def test_port_bit_exact_mixed_batch(workdir, port):
    from make_golden_shim import mixed_case
    from oracle import refrun
    g = _golden("mixed_batch")
    ctlkw, atms, ray_atm, geom = mixed_case(workdir)
    r = refrun.run_port(ctlkw, atms, ray_atm, geom, los=True)
    for k in ("rad", "tau", "tpz", "tplon", "tplat", "nlos", "digest"):
        assert np.array_equal(r[k], g[k]), k


@pytest.mark.parametrize("name", ["headline_batch", "continuum_bands"])
def test_port_bit_exact_shapes(workdir, port, name):
    """The benchmark's 64-channel, 8-emitter shape (O2 continuum in the top
    channels) and the O2/N2 continuum-band case."""
    from make_golden_shim import band_case, headline_case
    from oracle import refrun
    g = _golden(name)
    ctlkw, atms, ray_atm, geom = (headline_case if name == "headline_batch" else band_case)(workdir)
    r = refrun.run_port(ctlkw, atms, ray_atm, geom, los=True)
    for k in ("rad", "tau", "tpz", "tplon", "tplat", "nlos", "digest"):
        assert np.array_equal(r[k], g[k]), k


def _read_cols(path):
    rows = []
    for ln in open(path):
        ln = ln.strip()
        if ln and not ln.startswith("#"):
            rows.append(ln.split())
    return rows


def _port_lib():
    lib = C.CDLL(PORT)
    from jscat import structs as S
    P = C.POINTER
    lib.oracle_formod.argtypes = [P(S.CtlT), P(S.AtmT), P(S.ObsT), P(S.AeroT)]
    lib.oracle_formod.restype = C.c_int
    lib.oracle_raytrace.argtypes = [P(S.CtlT), P(S.AtmT), P(S.ObsT), C.c_int] + \
        [P(C.c_double)] * 10
    lib.oracle_raytrace.restype = C.c_int
    return lib


def _example_inputs():
    from jscat import structs as S
    ctl = S.make_ctl(["CO2", "H2O", "O3"], [792.0],
                     os.path.join(REF_EXAMPLES, "tab", "boxcar"))
    a = np.array(_read_cols(os.path.join(REF_EXAMPLES, "org", "atm.tab")), dtype=float)
    atm = S.make_atm(a[:, 1], a[:, 4], a[:, 5], a[:, 6:9].T, a[:, 9:10].T, a[:, 2], a[:, 3])
    return ctl, atm


@pytest.mark.skipif(not os.path.isdir(REF_EXAMPLES), reason="reference tree not present")
def test_port_reproduces_example_rad_clear(port):
    """examples/clear.sh: 11 limb rays, CO2/H2O/O3 RFM tables at 792 cm-1;
    the port's output formatted like write_obs (src/misc.c:377-384) equals
    org/rad_clear.tab."""
    from jscat import structs as S
    ctl, atm = _example_inputs()
    o = np.array(_read_cols(os.path.join(REF_EXAMPLES, "org", "obs.tab")), dtype=float)
    obs = S.make_obs(o[:, 1], o[:, 3], o[:, 4], o[:, 6], o[:, 2], o[:, 5], o[:, 0])
    lib = _port_lib()
    assert lib.oracle_formod(C.byref(ctl), C.byref(atm), C.byref(obs), C.byref(S.AeroT())) == 0
    mine = []
    for ir in range(obs.nr):
        vals = [obs.obsz[ir], obs.obslon[ir], obs.obslat[ir], obs.vpz[ir], obs.vplon[ir],
                obs.vplat[ir], obs.tpz[ir], obs.tplon[ir], obs.tplat[ir],
                obs.rad[0][ir], obs.tau[0][ir]]
        mine.append(["%.2f" % obs.time[ir]] + ["%g" % v for v in vals])
    assert mine == _read_cols(os.path.join(REF_EXAMPLES, "org", "rad_clear.tab"))


@pytest.mark.skipif(not os.path.isdir(REF_EXAMPLES), reason="reference tree not present")
def test_port_reproduces_example_los(port):
    """examples/raytrace.sh: one 8 km limb ray; every LOS record formatted
    like raytrace.c (src/raytrace.c:88-103) equals org/los.0."""
    from jscat import structs as S
    ctl, atm = _example_inputs()
    o = np.array(_read_cols(os.path.join(REF_EXAMPLES, "org", "obs_raytrace.tab")), dtype=float)
    obs = S.make_obs(o[:, 1], o[:, 3], o[:, 4], o[:, 6], o[:, 2], o[:, 5], o[:, 0])
    lib = _port_lib()
    n = 10000
    bufs = [np.zeros(n) for _ in range(6)] + [np.zeros(n * 3), np.zeros(n), np.zeros(n * 3)]
    ts = np.zeros(1)
    np_ = lib.oracle_raytrace(C.byref(ctl), C.byref(atm), C.byref(obs), 0,
                              *[b.ctypes.data_as(C.POINTER(C.c_double)) for b in bufs + [ts]])
    z, lon, lat, p, t, ds, q, k, u = bufs
    rows = []
    for i in range(np_):
        vals = [z[i], lon[i], lat[i], p[i], t[i]] + list(q[3 * i:3 * i + 3]) + [k[i]] + \
            list(u[3 * i:3 * i + 3]) + [0.0, 0.0, 0.0, ds[i]]
        rows.append(["%.2f" % 0.0] + ["%g" % v for v in vals])
    assert rows == _read_cols(os.path.join(REF_EXAMPLES, "org", "los.0"))


def _climatology_atm(ctlname, extra, tmpdir):
    """Example atmosphere made by the reference's climatology program
    (built by oracle/Makefile), as the example scripts do."""
    import subprocess
    clim = os.path.join(REPO, "oracle", "_ref", "climatology")
    src = os.path.join(REF_EXAMPLES, ctlname)
    ctl = os.path.join(tmpdir, ctlname)
    txt = open(src, "rb").read().replace(b"../clim", refpath.reference_path("clim").encode())
    open(ctl, "wb").write(txt)
    out = os.path.join(tmpdir, ctlname + ".atm")
    subprocess.run([clim, ctl, "-", out] + extra, check=True, capture_output=True)
    a = np.array(_read_cols(out), dtype=float)
    return {"z": a[:, 1], "lon": a[:, 2], "lat": a[:, 3], "p": a[:, 4], "t": a[:, 5],
            "q": a[:, 6:9].T, "k": a[:, 9:10].T}


@pytest.mark.skipif(not (os.path.isdir(REF_EXAMPLES) and
                         os.path.exists(os.path.join(REPO, "oracle", "_ref", "climatology"))),
                    reason="reference tree or reference build not present")
@pytest.mark.parametrize("name,ctlname,extra,obsf,aerof,kw", [
    ("ext1", "extinction1.ctl", [], "obs.tab", "aero0.tab", dict(sca_n=1, sca_mult=0)),
    ("aero0", "aerosol0.ctl", ["CLIMZONE", "pwin"], "obs_nadir.tab", "aero0.tab",
     dict(sca_n=1, sca_mult=1)),
    ("aero1", "aerosol1.ctl", [], "obs.tab", "aero1.tab", dict(sca_n=6, sca_mult=1)),
])
def test_port_reproduces_example_scattering(port, tmp_path, name, ctlname, extra, obsf, aerof, kw):
    """examples/extinction1.sh, aerosol0.sh (nadir, single scattering) and
    aerosol1.sh (limb, 6 modes in 3 layers, single scattering): the port's
    output equals org/rad_<name>.tab.  The aero_t input comes from the
    reference's own read_aero + get_opt_prop (Mie)."""
    from oracle import refrun
    atm = _climatology_atm(ctlname, extra, str(tmp_path))
    o = np.array(_read_cols(os.path.join(REF_EXAMPLES, "org", obsf)), dtype=float)
    geom = {"time": o[:, 0], "obsz": o[:, 1], "obslon": o[:, 2], "obslat": o[:, 3],
            "vpz": o[:, 4], "vplon": o[:, 5], "vplat": o[:, 6]}
    ctlkw = dict(emitters=["CO2", "H2O", "O3"], nus=[792.0],
                 tblbase=os.path.join(REF_EXAMPLES, "tab", "boxcar"), **kw)
    aero = refrun.reference_aero(ctlkw, aerof, REF_EXAMPLES)
    r = refrun.run_port(ctlkw, [atm], np.zeros(len(o), int), geom, aero=aero)
    mine = []
    for i in range(len(o)):
        vals = [geom["obsz"][i], geom["obslon"][i], geom["obslat"][i], geom["vpz"][i],
                geom["vplon"][i], geom["vplat"][i], r["tpz"][i], r["tplon"][i], r["tplat"][i],
                r["rad"][i, 0], r["tau"][i, 0]]
        mine.append(["%.2f" % geom["time"][i]] + ["%g" % v for v in vals])
    assert mine == _read_cols(os.path.join(REF_EXAMPLES, "org", "rad_%s.tab" % name))
