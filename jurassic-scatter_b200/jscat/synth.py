"""Seeded synthetic workloads for the forward model.

No observation dataset is involved: every input is generated here from a
seed, with the shapes and value ranges of the workloads the forward model is
specified on.

* Atmosphere: 0-120 km at 1 km; T piecewise linear (288 K at the surface,
  -6.5 K/km to 11 km, isothermal to 20 km, +1 K/km to 47 km, then
  -2.8 K/km, floored at 150 K); p from a 7 km scale height (the forward
  model rebuilds it hydrostatically with HYDZ=0); CO2 380 ppmv, H2O
  1e-2*exp(-z/2 km) floored at 5 ppmv, other emitters smooth textbook-like
  shapes; VMRs and T perturbed per level from the seed.
* Emissivity tables per (emitter, channel): 40 log-spaced pressures
  (1e-3..1100 hPa) x 30 temperatures (150..350 K) x 300 log-spaced column
  densities (1e10..1e26 molec/cm^2), eps = 1-exp(-k u^0.8) with log10 k a
  seeded smooth function of p and T; each row keeps the prefix on which u
  and eps (as float) strictly increase.  Written in the binary layout the
  reference's tab2bin writes (src/tab2bin.c:49-63).
* Filters: 1 cm^-1 boxcars, like examples/tab/boxcar_792.0000.filt.
* Geometry: limb rays from 800 km with the reference's limb.c construction
  (src/limb.c:67-73) and nadir/off-nadir rays ending on the ground.
"""
import hashlib
import os
import struct
import zlib

import numpy as np

RE = 6367.421
Z_GRID = np.arange(0.0, 121.0, 1.0)

LUT_P = np.logspace(-3.0, np.log10(1100.0), 40)
LUT_T = np.linspace(150.0, 350.0, 30)
LUT_U = np.logspace(10.0, 26.0, 300)


def standard_temperature(z):
    z = np.asarray(z, dtype=np.float64)
    t = np.where(z <= 11, 288.0 - 6.5 * z, 216.5)
    t = np.where((z > 20) & (z <= 47), 216.5 + (z - 20.0), t)
    t = np.where(z > 47, 243.5 - 2.8 * (z - 47.0), t)
    return np.maximum(t, 150.0)


def vmr_profile(name, z):
    z = np.asarray(z, dtype=np.float64)
    n = name.upper()
    if n == "CO2":
        return np.full_like(z, 380e-6)
    if n == "H2O":
        return np.maximum(1e-2 * np.exp(-z / 2.0), 5e-6)
    if n == "O3":
        return 8e-6 * np.exp(-((z - 35.0) / 10.0) ** 2) + 3e-8
    if n == "N2O":
        return 320e-9 * np.where(z < 15, 1.0, np.exp(-(z - 15.0) / 10.0))
    if n == "CH4":
        return 1.8e-6 * np.where(z < 15, 1.0, np.exp(-(z - 15.0) / 20.0))
    if n == "HNO3":
        return 5e-9 * np.exp(-((z - 25.0) / 7.0) ** 2) + 1e-11
    if n == "CO":
        return 100e-9 * np.exp(-z / 10.0) + 10e-9
    if n == "CCL4":
        return 0.1e-9 * np.where(z < 12, 1.0, np.exp(-(z - 12.0) / 4.0))
    return np.full_like(z, 1e-9)


def atmosphere(emitters, rng, t_sigma=0.0, vmr_sigma=0.05, z=Z_GRID):
    """One profile: dict z, lon, lat, p, t, q[ng][nz], k[1][nz]."""
    z = np.asarray(z, dtype=np.float64)
    t = standard_temperature(z)
    if t_sigma > 0:
        noise = rng.standard_normal(len(z))
        # 5-level running mean keeps the profile smooth; rescale to t_sigma
        sm = np.convolve(noise, np.ones(5) / 5.0, mode="same")
        t = t + t_sigma * sm / max(sm.std(), 1e-12)
    q = np.empty((len(emitters), len(z)))
    for i, e in enumerate(emitters):
        q[i] = vmr_profile(e, z) * np.maximum(1.0 + vmr_sigma * rng.standard_normal(len(z)), 0.05)
    p = 1013.25 * np.exp(-z / 7.0)
    return {"z": z, "lon": np.zeros_like(z), "lat": np.zeros_like(z),
            "p": p, "t": t, "q": q, "k": np.zeros((1, len(z)))}


def limb_geometry(tangent_heights, obsz=800.0):
    """Observer/view-point geometry of the reference's limb program."""
    th = np.asarray(tangent_heights, dtype=np.float64)
    obslat = 180.0 / np.pi * np.arccos((RE + th) / (RE + obsz))
    return {"obsz": np.full_like(th, obsz), "obslon": np.zeros_like(th),
            "obslat": obslat, "vpz": th.copy(), "vplon": np.zeros_like(th),
            "vplat": np.zeros_like(th), "time": np.zeros_like(th)}


def nadir_geometry(zenith_deg, obsz=800.0):
    """Rays that reach the ground at (0, 0) under local zenith angle zeta:
    the observer sits at great-circle distance zeta - asin(RE sin zeta /
    (RE + obsz)) from the ground point."""
    zen = np.radians(np.asarray(zenith_deg, dtype=np.float64))
    gam = zen - np.arcsin(RE * np.sin(zen) / (RE + obsz))
    n = len(zen)
    return {"obsz": np.full(n, obsz), "obslon": np.zeros(n),
            "obslat": np.degrees(gam), "vpz": np.zeros(n),
            "vplon": np.zeros(n), "vplat": np.zeros(n), "time": np.zeros(n)}


# ------------------------------------------------------------ tables ----

def _table_rng(seed, gas, nu):
    return np.random.default_rng([seed, zlib.crc32(gas.upper().encode()),
                                  int(round(nu * 1e4))])


def emissivity_table(gas, nu, seed):
    """(p, t, rows) with rows[ip][it] = (u float32[n], eps float32[n])."""
    rng = _table_rng(seed, gas, nu)
    c0 = rng.uniform(-20.5, -16.5)
    c1 = rng.uniform(0.15, 0.5)
    c2 = rng.uniform(-0.5, 0.5)
    c3 = rng.uniform(-0.2, 0.2)
    lp = np.log10(LUT_P)[:, None]
    tt = LUT_T[None, :]
    logk = c0 + c1 * (lp - 2.0) + c2 * (tt - 250.0) / 100.0 + c3 * np.sin(lp + tt / 60.0)
    k = 10.0 ** logk                                   # [np, nt]
    x = k[:, :, None] * LUT_U[None, None, :] ** 0.8    # [np, nt, nu]
    eps = (-np.expm1(-x)).astype(np.float32)
    u32 = LUT_U.astype(np.float32)
    # prefix of strictly increasing float eps (u is strictly increasing)
    inc = np.diff(eps, axis=2) > 0
    bad = ~inc
    first_bad = np.where(bad.any(axis=2), bad.argmax(axis=2), inc.shape[2])
    n = first_bad + 1
    rows = [[(u32[:n[i, j]], eps[i, j, :n[i, j]]) for j in range(len(LUT_T))]
            for i in range(len(LUT_P))]
    return LUT_P, LUT_T, rows


def write_table_bin(path, p, t, rows):
    parts = [struct.pack("<i", len(p)), np.asarray(p, "<f8").tobytes(),
             np.full(len(p), len(t), "<i4").tobytes()]
    for ip in range(len(p)):
        parts.append(np.asarray(t, "<f8").tobytes())
        parts.append(np.array([len(r[0]) for r in rows[ip]], "<i4").tobytes())
        for u, e in rows[ip]:
            parts.append(u.astype("<f4").tobytes())
            parts.append(e.astype("<f4").tobytes())
    with open(path, "wb") as f:
        f.write(b"".join(parts))


def write_filter(path, nu, half_width=0.5, step=0.005, margin=0.1):
    x = np.arange(nu - half_width - margin, nu + half_width + margin + step / 2, step)
    f = (np.abs(x - nu) <= half_width + 1e-9).astype(int)
    with open(path, "w") as fh:
        fh.write("# $1 = wavenumber [cm^-1]\n# $2 = filter function\n\n")
        for a, b in zip(x, f):
            fh.write("%.4f %d\n" % (a, b))


def write_tables(directory, emitters, nus, seed):
    """Write tables and filters once per parameter set; returns TBLBASE."""
    key = hashlib.sha1(repr((sorted(emitters), sorted(float(v) for v in nus), seed, 2)).encode()).hexdigest()[:12]
    d = os.path.join(directory, "lut_" + key)
    base = os.path.join(d, "synth")
    stamp = os.path.join(d, ".complete")
    if os.path.exists(stamp):
        return base
    os.makedirs(d, exist_ok=True)
    for nu in nus:
        write_filter("%s_%.4f.filt" % (base, nu), nu)
        for g in emitters:
            p, t, rows = emissivity_table(g, nu, seed)
            write_table_bin("%s_%.4f_%s.bin" % (base, nu, g), p, t, rows)
    open(stamp, "w").close()
    return base


# ----------------------------------------------------------- workloads --

def batch_from(atms, ray_atm, geom):
    """Batch input dict from a list of profiles and per-ray geometry."""
    nl = [len(a["z"]) for a in atms]
    off = np.concatenate([[0], np.cumsum(nl)]).astype(np.int32)
    cat = lambda k: np.concatenate([a[k] for a in atms])
    q = np.concatenate([a["q"] for a in atms], axis=1)
    k = np.concatenate([a["k"] for a in atms], axis=1)
    inp = {"atm_off": off, "z": cat("z"), "lon": cat("lon"), "lat": cat("lat"),
           "p": cat("p"), "t": cat("t"), "q": np.ascontiguousarray(q),
           "k": np.ascontiguousarray(k),
           "ray_atm": np.asarray(ray_atm, dtype=np.int32)}
    inp.update({k2: np.asarray(v, dtype=np.float64) for k2, v in geom.items()})
    return inp


CFG0_EMITTERS = ["CO2", "H2O"]
CFG0_NU = [792.0, 800.0, 810.0, 832.0]
CFG1_EMITTERS = ["CO2", "H2O", "O3", "N2O", "CH4", "HNO3", "CO", "CCl4"]
CFG1_NU = list(np.linspace(700.0, 1400.0, 64))


def curtain_case(directory, seed=20261203, n_prof=5, dlat=5.0):
    """Clear-air limb case through a horizontally varying atmosphere for
    IP=2/3: n_prof profiles along the meridian (latitudes dlat apart,
    centred on the tangent points), temperature offsets of -4..+4 K and
    H2O scaled by 0.7..1.3 across the track, one atm_t of n_prof x 121
    points ordered profile by profile; 31 limb rays 5-35 km.  Returns
    (ctl kwargs, atmosphere dict with lon/lat per point, geometry)."""
    rng = np.random.default_rng(seed)
    base = atmosphere(CFG0_EMITTERS, rng, t_sigma=0.0, vmr_sigma=0.05)
    lats = dlat * (np.arange(n_prof) - (n_prof - 1) / 2.0)
    nz = len(base["z"])
    z, lon, lat, p, t, q, k = [], [], [], [], [], [], []
    for i, la in enumerate(lats):
        f = i / (n_prof - 1)
        z.append(base["z"])
        lon.append(np.zeros(nz))
        lat.append(np.full(nz, la))
        p.append(base["p"])
        t.append(base["t"] + (8.0 * f - 4.0))
        qq = np.array(base["q"], dtype=float)
        qq[1] = qq[1] * (0.7 + 0.6 * f)
        q.append(qq)
        k.append(np.asarray(base.get("k", np.zeros((1, nz))), dtype=float))
    atm = {"z": np.concatenate(z), "lon": np.concatenate(lon), "lat": np.concatenate(lat),
           "p": np.concatenate(p), "t": np.concatenate(t), "q": np.concatenate(q, axis=1),
           "k": np.concatenate(k, axis=1)}
    geom = limb_geometry(5.0 + 1.0 * np.arange(31))
    tb = write_tables(directory, CFG0_EMITTERS, CFG0_NU, seed)
    ctlkw = dict(emitters=CFG0_EMITTERS, nus=CFG0_NU, tblbase=tb, hydz=0.0)
    return ctlkw, atm, geom


def clear_limb_case(directory, seed=20261203):
    """Clear-air limb case: 2 emitters, 4 channels, 61 rays with tangent
    heights 5-35 km every 0.5 km from 800 km, one profile.  Returns
    (ctl kwargs, profile, geometry)."""
    rng = np.random.default_rng(seed)
    atm = atmosphere(CFG0_EMITTERS, rng, t_sigma=0.0, vmr_sigma=0.05)
    th = 5.0 + 0.5 * np.arange(61)
    geom = limb_geometry(th)
    base = write_tables(directory, CFG0_EMITTERS, CFG0_NU, seed)
    ctlkw = dict(emitters=CFG0_EMITTERS, nus=CFG0_NU, tblbase=base, hydz=0.0)
    return ctlkw, atm, geom


def batched_case(directory, n_rays=100_000, rays_per_atm=50, seed=20261203,
                 emitters=None, nus=None):
    """Batched clear-air case: n_rays rays, half limb (tangent heights
    U[5, 60] km), half nadir/off-nadir (zenith U[0, 60] deg), profiles drawn
    per group of rays_per_atm rays with T sigma 5 K and VMR sigma 20 %."""
    emitters = CFG1_EMITTERS if emitters is None else emitters
    nus = CFG1_NU if nus is None else nus
    rng = np.random.default_rng(seed + 1)
    n_atm = (n_rays + rays_per_atm - 1) // rays_per_atm
    atms = [atmosphere(emitters, rng, t_sigma=5.0, vmr_sigma=0.2) for _ in range(n_atm)]
    n_limb = (n_rays + 1) // 2
    th = rng.uniform(5.0, 60.0, n_limb)
    zen = rng.uniform(0.0, 60.0, n_rays - n_limb)
    gl, gn = limb_geometry(th), nadir_geometry(zen)
    geom = {k: np.concatenate([gl[k], gn[k]]) for k in gl}
    # interleave limb and nadir rays so every profile gets both kinds
    order = np.empty(n_rays, dtype=np.int64)
    order[0::2] = np.arange(n_limb)
    order[1::2] = n_limb + np.arange(n_rays - n_limb)
    geom = {k: v[order] for k, v in geom.items()}
    ray_atm = np.arange(n_rays) // rays_per_atm
    base = write_tables(directory, emitters, nus, seed)
    ctlkw = dict(emitters=emitters, nus=nus, tblbase=base, hydz=0.0)
    return ctlkw, atms, ray_atm, geom


# ------------------------------------------------------------- aerosols --

CFG2_NU = list(np.linspace(780.0, 1250.0, 16))


def sulfate_refractive_index(nu):
    """n = 1.43 + 0.02 sin(nu/50), k = 0.05 + 0.1 exp(-((nu-1050)/40)^2)."""
    nu = np.asarray(nu, dtype=np.float64)
    return 1.43 + 0.02 * np.sin(nu / 50.0), 0.05 + 0.1 * np.exp(-((nu - 1050.0) / 40.0) ** 2)


def ice_refractive_index(nu):
    """n = 1.3 + 0.05 cos(nu/80), k varying smoothly between 0.02 and 0.4."""
    nu = np.asarray(nu, dtype=np.float64)
    return 1.3 + 0.05 * np.cos(nu / 80.0), 0.02 + 0.38 * (0.5 + 0.5 * np.sin((nu - 700.0) / 150.0)) ** 2


def write_refractive_index(path, fn, lo=600.0, hi=1500.0, step=1.0):
    """Refractive-index file: 'nu n k' lines (the Mie input of read_aero)."""
    nu = np.arange(lo, hi + step / 2, step)
    n, k = fn(nu)
    with open(path, "w") as f:
        for a, b, c in zip(nu, n, k):
            f.write("%.4f %.8f %.8f\n" % (a, b, c))


def write_aero_file(path, layers):
    """Aerosol model file: top bottom transition type refractive-index-file
    concentration radius width (one line per mode; MIE unless a layer
    tuple carries the type as an eighth element)."""
    with open(path, "w") as f:
        f.write("# $1 = top [km]\n# $2 = bottom [km]\n# $3 = transition [km]\n"
                "# $4 = type\n# $5 = refractive index file\n# $6 = N [cm-3]\n"
                "# $7 = median radius [um]\n# $8 = width\n\n")
        for lay in layers:
            kind = lay[7] if len(lay) > 7 else "MIE"
            f.write("%g %g %g %s %s %g %g %g\n" % (lay[:3] + (kind,) + lay[3:7]))


def write_fov_shape(path, fwhm=2.0, half_width=2.0, step=0.1):
    """Field-of-view shape file (read_shape's 'dz weight' lines): a
    Gaussian in tangent-height offset dz [km]."""
    dz = np.arange(-half_width, half_width + step / 2, step)
    w = np.exp(-4.0 * np.log(2.0) * (dz / fwhm) ** 2)
    with open(path, "w") as f:
        f.write("# $1 = offset [km]\n# $2 = weight\n")
        for a, b in zip(dz, w):
            f.write("%.4f %.8e\n" % (a, b))
    return path


def write_optical_database(path, nus):
    """External optical-property database (opt_prop_external's format): per
    line nu, extinction and scattering [1/km] and the phase function at
    NTHETA angles (a normalised Henyey-Greenstein shape whose asymmetry
    varies with nu)."""
    th = np.radians(np.arange(181.0))
    with open(path, "w") as f:
        for nu in nus:
            g = 0.3 + 0.4 * (nu - 700.0) / 700.0
            hg = (1 - g * g) / (1 + g * g - 2 * g * np.cos(th)) ** 1.5
            ext = 1e-3 * (1.0 + 0.5 * np.sin(nu / 90.0))
            sca = 0.6 * ext
            f.write("%.4f %.8e %.8e %s\n" % (nu, ext, sca, " ".join("%.8e" % v for v in hg)))


def layered_aero_files(directory):
    """aero.tab with two layers and three modes: a sulfate-like layer at
    15-20 km with two log-normal Mie modes (0.1 um and 0.4 um), and a
    9-11 km layer from an external optical-property database."""
    os.makedirs(directory, exist_ok=True)
    ri = os.path.join(directory, "sulfate_ri.dat")
    write_refractive_index(ri, sulfate_refractive_index)
    db = os.path.join(directory, "optical_db.dat")
    write_optical_database(db, np.arange(700.0, 1401.0, 50.0))
    aero = os.path.join(directory, "aero_layers.tab")
    write_aero_file(aero, [(20.0, 15.0, 0.1, ri, 10.0, 0.1, 1.5),
                           (20.0, 15.0, 0.1, ri, 2.0, 0.4, 1.3),
                           (11.0, 9.0, 0.1, db, 0.0, 0.0, 0.0, "Ext")])
    return aero


def external_aero_files(directory):
    """aero.tab with one layer from the external database only."""
    os.makedirs(directory, exist_ok=True)
    db = os.path.join(directory, "optical_db.dat")
    write_optical_database(db, np.arange(700.0, 1401.0, 50.0))
    aero = os.path.join(directory, "aero_external.tab")
    write_aero_file(aero, [(11.0, 9.0, 0.1, db, 0.0, 0.0, 0.0, "Ext")])
    return aero


def sulfate_layer_files(directory):
    """aero.tab for a sulfate-like layer at 15-20 km (0.1 km transition),
    median radius 0.1 um, width 1.5, 10 cm-3.  (The reference keeps the
    layer-edge altitudes in a 4*NLMAX array, src/lineofsight.c:200, so a
    transition layer may hold at most ~16 samples of TRANSS.)"""
    os.makedirs(directory, exist_ok=True)
    ri = os.path.join(directory, "sulfate_ri.dat")
    write_refractive_index(ri, sulfate_refractive_index)
    aero = os.path.join(directory, "aero_sulfate.tab")
    write_aero_file(aero, [(20.0, 15.0, 0.1, ri, 10.0, 0.1, 1.5)])
    return aero


def ice_layer_files(directory):
    """aero.tab for an ice-cloud-like layer at 9-11 km (0.1 km transition),
    median radius 10 um, width 1.8, 0.1 cm-3."""
    os.makedirs(directory, exist_ok=True)
    ri = os.path.join(directory, "ice_ri.dat")
    write_refractive_index(ri, ice_refractive_index)
    aero = os.path.join(directory, "aero_ice.tab")
    write_aero_file(aero, [(11.0, 9.0, 0.1, ri, 0.1, 10.0, 1.8)])
    return aero
