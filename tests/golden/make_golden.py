"""Generate the golden fixtures of tests/golden/ by running the reference
forward model (oracle/_ref/libjurassic_ref.so, compiled from the
reference's own sources by oracle/Makefile) on the seeded synthetic
workloads of jscat.synth.

    make -C oracle ref && python tests/golden/make_golden.py [headline|emitters|points [kind...]|ice2|jacobian|aero|fov|aerojac|ip|ipjac|ip3d]

Each fixture stores the reference's outputs in full FP64 precision, the
per-(ray, channel) EGA table-index digests of the C restatement (checked
here to reproduce the reference's radiances bit for bit), and a checksum
of the generated table files, so a test can tell a changed input from a
changed result.
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "jurassic-scatter_b200"))
sys.path.insert(0, REPO)

from jscat import synth  # noqa: E402
from oracle import refrun  # noqa: E402


def tables_digest(tblbase, emitters, nus):
    h = hashlib.sha256()
    for nu in nus:
        for g in emitters:
            with open("%s_%.4f_%s.bin" % (tblbase, nu, g), "rb") as f:
                h.update(f.read())
        with open("%s_%.4f.filt" % (tblbase, nu), "rb") as f:
            h.update(f.read())
    return h.hexdigest()


def mixed_case(workdir):
    """8 emitters, 8 channels of the 64-channel grid, 8 profiles x 40 rays
    (limb and nadir interleaved)."""
    nus = synth.CFG1_NU[::8]
    ctlkw, atms, ray_atm, geom = synth.batched_case(
        workdir, n_rays=320, rays_per_atm=40, seed=20261203, nus=nus)
    return ctlkw, atms, ray_atm, geom


def headline_case(workdir):
    """The benchmark's headline shape on a small ray count: 8 emitters, all
    64 channels 700-1400 cm^-1 (the top four take the O2 continuum,
    src/continua.c:1997-2049), the benchmark's own tables, 3 profiles x 50
    rays (limb and nadir interleaved)."""
    return synth.batched_case(workdir, n_rays=150, rays_per_atm=50, seed=20261203)


# Channels in the O2 (1360-1805 cm^-1) and N2 (2120-2605 cm^-1) continuum
# bands (src/continua.c:1935-2049), plus one below both.
BAND_NU = [1250.0, 1370.0, 1500.0, 1700.0, 2150.0, 2300.0, 2450.0, 2590.0]


def band_case(workdir):
    """2 emitters, the BAND_NU channels, 2 profiles x 30 rays (limb and
    nadir interleaved): exercises ctmn2 and ctmo2."""
    return synth.batched_case(workdir, n_rays=60, rays_per_atm=30, seed=20261205,
                              emitters=synth.CFG0_EMITTERS, nus=BAND_NU)


# Emitter sets beyond the benchmark's eight (the reference holds up to
# NGMAX = 25): the first eight names of the benchmark, then generic gases
# with a flat 1 ppbv profile.
def many_emitters(n):
    return synth.CFG1_EMITTERS + ["GAS%02d" % i for i in range(9, n + 1)]


def emitters_case(workdir, n):
    """n emitters (12: the ray-tile kernels' 16-warp form; 20: the 32-lane
    groups and the widest thread-per-channel kernel), 4 channels of the
    64-channel grid, 2 profiles x 20 rays (limb and nadir interleaved)."""
    return synth.batched_case(workdir, n_rays=40, rays_per_atm=20, seed=20261207 + n,
                              emitters=many_emitters(n), nus=synth.CFG1_NU[3::16])


def reference_ctl(ctlkw):
    """Clear-air cases run the reference with SCA_MULT=0.  With the default
    SCA_MULT=1 and no aerosol models the reference reads los->aerofac, which
    it never initialises in clear air (src/lineofsight.c:188 skips
    add_aerosol_layers, src/forwardmodel.c:317 tests it), so a recycled heap
    block can send a ray down the scattering branch and return NaN.  With
    SCA_MULT=0 the same clear-air arithmetic runs deterministically."""
    return dict(ctlkw, sca_mult=0)


def save(name, ctlkw, atms, ray_atm, geom, ref, port):
    assert np.array_equal(port["rad"], ref["rad"]) and np.array_equal(port["tau"], ref["tau"]), \
        "the C restatement must reproduce the reference bit for bit"
    np.savez_compressed(
        os.path.join(HERE, name + ".npz"),
        rad=ref["rad"], tau=ref["tau"], tpz=ref["tpz"], tplon=ref["tplon"],
        tplat=ref["tplat"], nlos=ref["nlos"], digest=port["digest"],
        table_sha256=tables_digest(ctlkw["tblbase"], ctlkw["emitters"], ctlkw["nus"]),
        ray_atm=np.asarray(ray_atm), **{"geom_" + k: v for k, v in geom.items()})


def aerosol_case(workdir, sca_mult, n_rays=24, nus=None, sca_ext="beta_a"):
    """2 emitters, 4 channels of the 16-channel aerosol grid, limb rays with
    tangent heights 8-30 km through the sulfate-like layer; sca_mult 0:
    extinction only, 1: single scattering."""
    nus = [synth.CFG2_NU[i] for i in (0, 5, 10, 15)] if nus is None else nus
    rng = np.random.default_rng(20261204)
    atm = synth.atmosphere(synth.CFG0_EMITTERS, rng)
    geom = synth.limb_geometry(np.linspace(8.0, 30.0, n_rays))
    base = synth.write_tables(workdir, synth.CFG0_EMITTERS, nus, 20261203)
    aerofile = synth.sulfate_layer_files(os.path.join(workdir, "aero"))
    ctlkw = dict(emitters=synth.CFG0_EMITTERS, nus=nus, tblbase=base, hydz=0.0, sca_n=1,
                 sca_mult=sca_mult, sca_ext=sca_ext)
    return ctlkw, atm, geom, aerofile


def save_aero(name, ctlkw, atm, geom, ref, aero_bytes, port=None):
    extra = {}
    if port is not None:
        assert np.array_equal(port["rad"], ref["rad"]), "port must match the reference"
        extra["digest"] = port["digest"]
    np.savez_compressed(
        os.path.join(HERE, name + ".npz"),
        rad=ref["rad"], tau=ref["tau"], tpz=ref["tpz"], nlos=ref["nlos"],
        aero=np.frombuffer(aero_bytes, dtype=np.uint8),
        table_sha256=tables_digest(ctlkw["tblbase"], ctlkw["emitters"], ctlkw["nus"]),
        **{"geom_" + k: v for k, v in geom.items()}, **extra)


def double_scattering_fixture(workdir):
    """SCA_MULT=2 on one limb ray (tangent height 16.37 km, noon) through
    the sulfate layer, 2 channels.  The reference returns NaN here (a
    zero-length chord at a layer-edge point of a second-order pencil, 0/0 in
    formod_continua); the fixture pins that behaviour.  Slow: about 47 min
    of reference CPU time (28 pencils per scattering point, two orders)."""
    nus = [synth.CFG2_NU[i] for i in (0, 10)]
    ctlkw, atm, geom, aerofile = aerosol_case(workdir, 2, n_rays=1, nus=nus)
    geom = synth.limb_geometry(np.array([16.37]))
    geom["time"] = np.full(1, 43200.0)
    aero = refrun.reference_aero(ctlkw, aerofile, os.path.dirname(aerofile))
    ref = refrun.run(ctlkw, [atm], np.zeros(1, int), geom, aero=aero, timeout=7200, los=True)
    np.savez_compressed(os.path.join(HERE, "aerosol_sca2.npz"), rad=ref["rad"], tau=ref["tau"],
                        nlos=ref["nlos"], nus=np.asarray(nus),
                        **{"geom_" + k: v for k, v in geom.items()})


def aero_fixture(workdir, name, layer_files, nus, sca_n=1):
    """aero_t (as bytes) of a layer file on a channel grid, from the
    reference's read_aero + get_opt_prop (Mie), for benchmark inputs and
    the optical-property parity tests."""
    ctlkw = dict(emitters=synth.CFG0_EMITTERS, nus=nus, tblbase="-", sca_n=sca_n, sca_mult=1)
    aerofile = layer_files(os.path.join(workdir, "aero"))
    aero = refrun.reference_aero(ctlkw, aerofile, os.path.dirname(aerofile))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), nus=np.asarray(nus),
                        aero=np.frombuffer(aero, dtype=np.uint8))


# Retrieval settings of the Jacobian fixtures: temperature, both VMRs and
# the window extinction over parts of the profile, and pressure at levels
# whose disturbance the hydrostatic balance of the disturbed forward model
# undoes (zero columns, as in the reference).
JACOBIAN_RET = dict(rett_zmin=5.0, rett_zmax=40.0, retq_zmin=[20.0, 5.0], retq_zmax=[30.0, 25.0],
                    retk_zmin=[10.0], retk_zmax=[15.0], retp_zmin=30.0, retp_zmax=35.0)


def fov_case(workdir):
    """The clear limb case with a 2-km Gaussian field of view."""
    ctlkw, atm, geom = synth.clear_limb_case(workdir)
    shape = synth.write_fov_shape(os.path.join(workdir, "fov_gauss2km.dat"))
    return dict(ctlkw, fov=shape), atm, geom


def jacobian_case(workdir, bt=False, fov=False):
    """The clear limb case with the retrieval settings above (radiances,
    two observations masked and one ray fully masked), or with brightness
    temperatures, temperature only and every fourth ray (bt=True), or with
    the field of view of fov_case and temperature only (fov=True)."""
    ctlkw, atm, geom = synth.clear_limb_case(workdir)
    if fov:
        ctlkw = dict(fov_case(workdir)[0], rett_zmin=5.0, rett_zmax=40.0)
        mask = np.zeros((len(geom["obsz"]), len(ctlkw["nus"])), bool)
        return ctlkw, atm, geom, mask
    if bt:
        ctlkw = dict(ctlkw, write_bbt=1, rett_zmin=10.0, rett_zmax=30.0)
        geom = {k: v[::4] for k, v in geom.items()}
        mask = np.zeros((len(geom["obsz"]), len(ctlkw["nus"])), bool)
    else:
        ctlkw = dict(ctlkw, **JACOBIAN_RET)
        mask = np.zeros((len(geom["obsz"]), len(ctlkw["nus"])), bool)
        mask[3, 1] = mask[40, 2] = True
        mask[10, :] = True
    return ctlkw, atm, geom, mask


def jacobian_fixture(workdir, name, bt, fov=False):
    """Jacobian of the reference's own kernel() (oracle/_ref/libjurassic_ref_ret.so)."""
    ctlkw, atm, geom, mask = jacobian_case(workdir, bt, fov)
    ref = refrun.reference_kernel(reference_ctl(ctlkw), atm, geom, mask=mask)
    np.savez_compressed(
        os.path.join(HERE, name + ".npz"), k=ref["k"], x0=ref["x0"], iqa=ref["iqa"],
        ipa=ref["ipa"], rad=ref["rad"], p=ref["p"], mask=mask,
        table_sha256=tables_digest(ctlkw["tblbase"], ctlkw["emitters"], ctlkw["nus"]),
        **{"geom_" + k: v for k, v in geom.items()})


def aerosol_jacobian_case(workdir):
    """Aerosol extinction (beta_e) through the sulfate-like layer, state
    vector temperature 10-30 km plus the layer's number concentration,
    median radius and width (RETNN/RETRR/RETSS)."""
    ctlkw, atm, geom, aerofile = aerosol_case(workdir, 0, sca_ext="beta_e")
    ctlkw = dict(ctlkw, rett_zmin=10.0, rett_zmax=30.0, retnn=1, retrr=1, retss=1)
    return ctlkw, atm, geom, aerofile


def aerosol_jacobian_fixture(workdir):
    ctlkw, atm, geom, aerofile = aerosol_jacobian_case(workdir)
    ref = refrun.reference_kernel(ctlkw, atm, geom, aerofile=aerofile,
                                  cwd=os.path.dirname(aerofile))
    np.savez_compressed(
        os.path.join(HERE, "jacobian_aerosol.npz"), k=ref["k"], x0=ref["x0"], iqa=ref["iqa"],
        ipa=ref["ipa"], rad=ref["rad"], p=ref["p"],
        table_sha256=tables_digest(ctlkw["tblbase"], ctlkw["emitters"], ctlkw["nus"]),
        **{"geom_" + k: v for k, v in geom.items()})


# IP=3 influence lengths of the curtain fixtures [km]
IP3_CZ, IP3_CX = 3.0, 700.0


# horizontal influence length of the IP=3 scattering-point fixture [km]
IP3_SCA_CX = 20000.0


def curtain_ctl(ctlkw, ip):
    return dict(ctlkw, ip=ip, cz=IP3_CZ, cx=IP3_CX) if ip == 3 else dict(ctlkw, ip=ip)


def curtain_fixtures(workdir):
    """formod through the horizontally varying curtain atmosphere with
    IP=2 (two nearest profiles) and IP=3 (distance-weighted points)."""
    ctlkw, atm, geom = synth.curtain_case(workdir)
    ra = np.zeros(len(geom["obsz"]), int)
    for ip in (2, 3):
        ref = refrun.run(reference_ctl(curtain_ctl(ctlkw, ip)), [atm], ra, geom, los=True)
        np.savez_compressed(
            os.path.join(HERE, "curtain_ip%d.npz" % ip), rad=ref["rad"], tau=ref["tau"],
            tpz=ref["tpz"], tplat=ref["tplat"], nlos=ref["nlos"],
            table_sha256=tables_digest(ctlkw["tblbase"], ctlkw["emitters"], ctlkw["nus"]),
            **{"geom_" + k: v for k, v in geom.items()})
    # with aerosol extinction through the sulfate-like layer
    ctlx = dict(ctlkw, sca_n=1, sca_mult=0, sca_ext="beta_e")
    aerofile = synth.sulfate_layer_files(os.path.join(workdir, "aero"))
    aero = refrun.reference_aero(ctlx, aerofile, os.path.dirname(aerofile))
    for ip in (2, 3):
        ref = refrun.run(curtain_ctl(ctlx, ip), [atm], ra, geom, aero=aero, los=True)
        np.savez_compressed(
            os.path.join(HERE, "curtain_ip%d_ext.npz" % ip), rad=ref["rad"], tau=ref["tau"],
            tpz=ref["tpz"], nlos=ref["nlos"], aero=np.frombuffer(aero, dtype=np.uint8),
            table_sha256=tables_digest(ctlkw["tblbase"], ctlkw["emitters"], ctlkw["nus"]),
            **{"geom_" + k: v for k, v in geom.items()})


def curtain_jacobian_case(workdir):
    """Jacobian through the IP=2 curtain: temperature at 10-30 km of every
    profile, every third limb ray."""
    ctlkw, atm, geom = synth.curtain_case(workdir)
    ctlkw = dict(ctlkw, ip=2, rett_zmin=10.0, rett_zmax=30.0)
    geom = {k: v[::3] for k, v in geom.items()}
    return ctlkw, atm, geom


def curtain_jacobian_fixture(workdir):
    ctlkw, atm, geom = curtain_jacobian_case(workdir)
    ref = refrun.reference_kernel(reference_ctl(ctlkw), atm, geom)
    np.savez_compressed(
        os.path.join(HERE, "jacobian_curtain_ip2.npz"), k=ref["k"], x0=ref["x0"],
        iqa=ref["iqa"], ipa=ref["ipa"], rad=ref["rad"],
        table_sha256=tables_digest(ctlkw["tblbase"], ctlkw["emitters"], ctlkw["nus"]),
        **{"geom_" + k: v for k, v in geom.items()})


def curtain_scattering_case(workdir):
    """Single scattering (SCA_MULT=1, 3-D source) through the curtain with
    the sulfate-like layer (15-20 km): one limb ray with its tangent point
    0.3 km below the layer top at noon (solar term on), two of the four
    channels.  The short chord through the layer keeps the reference's
    32,400 secondary pencils per scattering point within CPU minutes."""
    ctlkw, atm, _ = synth.curtain_case(workdir)
    ctlkw = dict(ctlkw, nus=list(ctlkw["nus"][:2]), sca_n=1, sca_mult=1, ip=2)
    geom = synth.limb_geometry(np.array([19.7]))
    geom["time"] = np.full(1, 43200.0)
    aerofile = synth.sulfate_layer_files(os.path.join(workdir, "aero"))
    return ctlkw, atm, geom, aerofile


def curtain_scattering_fixture(workdir):
    """The reference's formod on curtain_scattering_case: 32,400 secondary
    pencils per scattering point (srcfunc_sca_3d).  Slow: several minutes
    of reference CPU time."""
    ctlkw, atm, geom, aerofile = curtain_scattering_case(workdir)
    aero = refrun.reference_aero(ctlkw, aerofile, os.path.dirname(aerofile))
    ra = np.zeros(1, int)
    ref = refrun.run(ctlkw, [atm], ra, geom, aero=aero, los=True, timeout=14400)
    np.savez_compressed(
        os.path.join(HERE, "curtain_ip2_sca1.npz"), rad=ref["rad"], tau=ref["tau"],
        nlos=ref["nlos"], aero=np.frombuffer(aero, dtype=np.uint8), seconds=ref["seconds"],
        table_sha256=tables_digest(ctlkw["tblbase"], ctlkw["emitters"], ctlkw["nus"]),
        **{"geom_" + k: v for k, v in geom.items()})


def fov_fixtures(workdir):
    """formod and kernel() with the field of view of fov_case."""
    ctlkw, atm, geom = fov_case(workdir)
    ra = np.zeros(len(geom["obsz"]), int)
    ref = refrun.run(reference_ctl(ctlkw), [atm], ra, geom, los=True)
    save_fov = dict(rad=ref["rad"], tau=ref["tau"], tpz=ref["tpz"],
                    table_sha256=tables_digest(ctlkw["tblbase"], ctlkw["emitters"], ctlkw["nus"]),
                    **{"geom_" + k: v for k, v in geom.items()})
    np.savez_compressed(os.path.join(HERE, "clear_limb_fov.npz"), **save_fov)
    jacobian_fixture(workdir, "jacobian_limb_fov", False, fov=True)


def _geo2cart(z, lon, lat):
    r = 6367.421 + z
    la, lo = np.radians(lat), np.radians(lon)
    return [r * np.cos(la) * np.cos(lo), r * np.cos(la) * np.sin(lo), r * np.sin(la)]


def _chord(z, lon, lat, azimuth_deg, dip_deg, length=20.0):
    """Direction of a line of sight through (z, lon, lat): azimuth from
    north towards east, dip below the local horizontal (a chord dx of the
    given length)."""
    la, lo = np.radians(lat), np.radians(lon)
    up = np.array([np.cos(la) * np.cos(lo), np.cos(la) * np.sin(lo), np.sin(la)])
    east = np.array([-np.sin(lo), np.cos(lo), 0.0])
    north = np.cross(up, east)
    a, d = np.radians(azimuth_deg), np.radians(dip_deg)
    v = np.cos(d) * (np.cos(a) * north + np.sin(a) * east) - np.sin(d) * up
    return list(length * v)


# Scattering points inside the sulfate layer (15-20 km): (z, lon, lat,
# azimuth, dip, time [s since 2000-01-01T00:00Z]).
SCA_POINTS_1D = [(17.3, 0.0, 0.0, 0.0, 1.0, 43200.0), (15.8, 10.0, 5.0, 90.0, -2.0, 43200.0),
                 (19.2, -20.0, -10.0, 200.0, 0.5, 0.0)]
SCA_POINTS_3D = [(17.3, 0.0, 1.5, 10.0, 0.8, 43200.0)]


def scattering_point_case(workdir, kind):
    """Per-point scattering sources through the sulfate-like layer, 2 of the
    aerosol channels: 'order1' single scattering at three points (IP=1, two
    by day), 'order2' the depth-2 source (SCA_MULT=2) at one point by night
    and one by day with the CO2/H2O continua off (with them on, leaf pencils
    that start on a layer-edge point get a zero-length segment and the
    reference's continuum 0/0 turns the source into NaN), 'ip2'/'ip3' the
    3-D source (32,400 pencils) at one point of the curtain atmosphere."""
    nus = [synth.CFG2_NU[i] for i in (0, 10)]
    aerofile = synth.sulfate_layer_files(os.path.join(workdir, "aero"))
    if kind in ("ip2", "ip3"):
        ctlkw, atm, _ = synth.curtain_case(workdir)
        base = synth.write_tables(workdir, synth.CFG0_EMITTERS, nus, 20261203)
        ctlkw = curtain_ctl(dict(ctlkw, nus=nus, tblbase=base, sca_n=1, sca_mult=1),
                            int(kind[2]))
        if kind == "ip3":
            # pencils in every direction leave the curtain; with the curtain's
            # 700 km influence length some then see no profile point and the
            # reference stops ("Too many LOS points!")
            ctlkw = dict(ctlkw, cx=IP3_SCA_CX)
        pts, order = SCA_POINTS_3D, 1
    else:
        ctlkw, atm, _, _ = aerosol_case(workdir, 1, nus=nus)
        pts, order = SCA_POINTS_1D, 1
        if kind == "order2":
            ctlkw = dict(ctlkw, sca_mult=2, ctm_co2=0, ctm_h2o=0)
            pts, order = [SCA_POINTS_1D[2], SCA_POINTS_1D[0]], 2
    points = [(_geo2cart(z, lo, la), _chord(z, lo, la, az, dip), 0, t)
              for z, lo, la, az, dip, t in pts]
    return ctlkw, atm, aerofile, points, order


def scattering_point_fixture(workdir, kind):
    ctlkw, atm, aerofile, points, order = scattering_point_case(workdir, kind)
    aero = refrun.reference_aero(ctlkw, aerofile, os.path.dirname(aerofile))
    ref = refrun.reference_srcfunc(ctlkw, atm, S_aero(aero), points, order)
    np.savez_compressed(
        os.path.join(HERE, "sca_points_%s.npz" % kind), src=ref["src"], p=ref["p"],
        seconds=ref["seconds"], x=np.array([p[0] for p in points]),
        dx=np.array([p[1] for p in points]), il=np.array([p[2] for p in points]),
        time=np.array([p[3] for p in points]), order=order,
        aero=np.frombuffer(aero, dtype=np.uint8),
        table_sha256=tables_digest(ctlkw["tblbase"], ctlkw["emitters"], ctlkw["nus"]))


def S_aero(aero_bytes):
    from jscat import structs as S
    return S.AeroT.from_buffer_copy(aero_bytes)


def ice_depth2_case(workdir):
    """Depth-2 scattering through the ice-cloud layer (9-11 km) with the
    per-order pencil counts of the benchmark (20 pencils per point of order
    2, 10 per point of order 1), two of its channels, CO2/H2O continua off,
    two limb rays by day.  The C restatement computes it (its per-order
    pencil count is an option the reference does not have; with 28 pencils
    at every order it reproduces the reference bit for bit)."""
    g = np.load(os.path.join(HERE, "aero_ice8.npz"))
    nus = [float(v) for v in g["nus"][[0, 4]]]
    rng = np.random.default_rng(20261207)
    atm = synth.atmosphere(synth.CFG0_EMITTERS, rng)
    geom = synth.limb_geometry(np.array([10.4, 12.2]))
    geom["time"] = np.array([43200.0, 50000.0])
    base = synth.write_tables(workdir, synth.CFG0_EMITTERS, nus, 20261203)
    ctlkw = dict(emitters=synth.CFG0_EMITTERS, nus=nus, tblbase=base, hydz=0.0, sca_n=1,
                 sca_mult=2, ctm_co2=0, ctm_h2o=0)
    return ctlkw, atm, geom, {2: 20, 1: 10}


def ice_depth2_fixture(workdir):
    from jscat import structs as S
    ctlkw, atm, geom, nalpha = ice_depth2_case(workdir)
    g = np.load(os.path.join(HERE, "aero_ice8.npz"))
    full = S.AeroT.from_buffer_copy(g["aero"].tobytes())
    aero = aero_channels(full, [0, 4])
    ref = refrun.run_port(ctlkw, [atm], np.zeros(2, int), geom, aero=bytes(aero), los=True,
                          nalpha=nalpha, threads=os.cpu_count(), timeout=7200)
    np.savez_compressed(os.path.join(HERE, "ice_sca2_port.npz"), rad=ref["rad"], tau=ref["tau"],
                        nlos=ref["nlos"], aero=np.frombuffer(bytes(aero), dtype=np.uint8),
                        seconds=ref["seconds"],
                        table_sha256=tables_digest(ctlkw["tblbase"], ctlkw["emitters"],
                                                   ctlkw["nus"]),
                        **{"geom_" + k: v for k, v in geom.items()})


def aero_channels(aero, idx):
    """aero_t restricted to the channels idx (in that order)."""
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


def headline_fixtures(workdir):
    """headline_batch (the benchmark's 64-channel, 8-emitter shape) and
    continuum_bands (O2 and N2 continuum channels)."""
    for name, case in (("headline_batch", headline_case), ("continuum_bands", band_case)):
        ctlkw, atms, ray_atm, geom = case(workdir)
        ref = refrun.run(reference_ctl(ctlkw), atms, ray_atm, geom, los=True)
        port = refrun.run_port(ctlkw, atms, ray_atm, geom, los=True)
        save(name, ctlkw, atms, ray_atm, geom, ref, port)


def emitters_fixtures(workdir):
    """emitters12 and emitters20: more emitters than the benchmark's eight."""
    for n in (12, 20):
        ctlkw, atms, ray_atm, geom = emitters_case(workdir, n)
        ref = refrun.run(reference_ctl(ctlkw), atms, ray_atm, geom, los=True)
        port = refrun.run_port(ctlkw, atms, ray_atm, geom, los=True)
        save("emitters%d" % n, ctlkw, atms, ray_atm, geom, ref, port)


def main():
    workdir = os.environ.get("JSC_WORKDIR", "/tmp/jsc")
    if sys.argv[1:] == ["headline"]:
        headline_fixtures(workdir)
        return
    if sys.argv[1:] == ["emitters"]:
        emitters_fixtures(workdir)
        return
    if sys.argv[1:] == ["ice2"]:
        ice_depth2_fixture(workdir)
        return
    if sys.argv[1:2] == ["points"]:
        # per-point scattering sources; slow kinds (order2, ip2, ip3) take
        # CPU minutes each
        for kind in sys.argv[2:] or ["order1", "order2", "ip2", "ip3"]:
            scattering_point_fixture(workdir, kind)
        return
    if sys.argv[1:] == ["jacobian"]:
        jacobian_fixture(workdir, "jacobian_limb", False)
        jacobian_fixture(workdir, "jacobian_limb_bt", True)
        return
    if sys.argv[1:] == ["fov"]:
        fov_fixtures(workdir)
        return
    if sys.argv[1:] == ["aerojac"]:
        aerosol_jacobian_fixture(workdir)
        return
    if sys.argv[1:] == ["ip"]:
        curtain_fixtures(workdir)
        return
    if sys.argv[1:] == ["ipjac"]:
        curtain_jacobian_fixture(workdir)
        return
    if sys.argv[1:] == ["ip3d"]:
        curtain_scattering_fixture(workdir)
        return
    if sys.argv[1:] == ["aero"]:
        aero_fixture(workdir, "aero_layers8", synth.layered_aero_files, list(synth.CFG2_NU[::2]),
                     sca_n=3)
        return
    ctlkw, atm, geom = synth.clear_limb_case(workdir)
    ra = np.zeros(len(geom["obsz"]), int)
    ref = refrun.run(reference_ctl(ctlkw), [atm], ra, geom, los=True)
    port = refrun.run_port(ctlkw, [atm], ra, geom, los=True)
    save("clear_limb", ctlkw, [atm], ra, geom, ref, port)
    ctlkw, atms, ray_atm, geom = mixed_case(workdir)
    ref = refrun.run(reference_ctl(ctlkw), atms, ray_atm, geom, los=True)
    port = refrun.run_port(ctlkw, atms, ray_atm, geom, los=True)
    save("mixed_batch", ctlkw, atms, ray_atm, geom, ref, port)
    headline_fixtures(workdir)
    for ext in ("beta_a", "beta_e"):
        ctlkw, atm, geom, aerofile = aerosol_case(workdir, 0, sca_ext=ext)
        aero = refrun.reference_aero(ctlkw, aerofile, os.path.dirname(aerofile))
        ra = np.zeros(len(geom["obsz"]), int)
        ref = refrun.run(ctlkw, [atm], ra, geom, aero=aero, los=True)
        port = refrun.run_port(ctlkw, [atm], ra, geom, aero=aero, los=True)
        save_aero("aerosol_ext_" + ext, ctlkw, atm, geom, ref, aero, port)
    for name, sec in (("night", 0.0), ("day", 43200.0)):
        ctlkw, atm, geom, aerofile = aerosol_case(workdir, 1)
        geom["time"] = np.full(len(geom["obsz"]), sec)
        aero = refrun.reference_aero(ctlkw, aerofile, os.path.dirname(aerofile))
        ra = np.zeros(len(geom["obsz"]), int)
        ref = refrun.run(ctlkw, [atm], ra, geom, aero=aero, los=True)
        port = refrun.run_port(ctlkw, [atm], ra, geom, aero=aero)
        assert np.max(np.abs(port["rad"] - ref["rad"]) / np.abs(ref["rad"])) < 1e-12
        save_aero("aerosol_sca1_" + name, ctlkw, atm, geom, ref, aero)
    aero_fixture(workdir, "aero_sulfate16", synth.sulfate_layer_files, list(synth.CFG2_NU))
    if os.environ.get("JSC_SLOW_FIXTURES"):
        double_scattering_fixture(workdir)
    aero_fixture(workdir, "aero_ice8", synth.ice_layer_files, list(synth.CFG2_NU[::2]))
    aero_fixture(workdir, "aero_layers8", synth.layered_aero_files, list(synth.CFG2_NU[::2]),
                     sca_n=3)
    jacobian_fixture(workdir, "jacobian_limb", False)
    jacobian_fixture(workdir, "jacobian_limb_bt", True)
    fov_fixtures(workdir)
    aerosol_jacobian_fixture(workdir)
    curtain_fixtures(workdir)
    curtain_jacobian_fixture(workdir)
    if os.environ.get("JSC_SLOW_FIXTURES"):
        curtain_scattering_fixture(workdir)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
