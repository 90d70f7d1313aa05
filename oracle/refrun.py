"""Run the reference forward model as the oracle.  TEST INFRASTRUCTURE ONLY:
imported by tests/, __graft_entry__.smoke() and bench.py's CPU baseline,
never by the product.

oracle/_ref/libjurassic_ref.so is the reference's own src/*.c compiled by
oracle/Makefile.  The reference keeps its emissivity tables, Planck table
and emitter indices in static variables initialised by the first call
(src/forwardmodel.c:231-292, :747-786; src/continua.c:846,1894), so every
run happens in a fresh spawned process.
"""
import ctypes as C
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
REF_LIB = os.path.join(HERE, "_ref", "libjurassic_ref.so")
sys.path.insert(0, os.path.join(REPO, "jurassic-scatter_b200"))

from jscat import structs as S  # noqa: E402


LosT = S.LosT  # los_t of src/jurassic.h:352-393 (raytrace output)


def available():
    return os.path.exists(REF_LIB)


def _silence():
    fd = os.open(os.devnull, os.O_WRONLY)
    os.dup2(fd, 1)
    os.close(fd)


def _atm_struct(a):
    return S.make_atm(a["z"], a["p"], a["t"], a["q"], a.get("k"),
                      a.get("lon"), a.get("lat"))


def _child(job):
    if job.get("threads"):
        os.environ["OMP_NUM_THREADS"] = str(job["threads"])
    _silence()
    lib = C.CDLL(job.get("lib", REF_LIB))
    P = C.POINTER
    port = job.get("port", False)
    fm = lib.oracle_formod if port else lib.formod
    if port and job.get("nalpha"):
        na = job["nalpha"]
        if isinstance(na, dict):    # {scattering order: pencils}
            for order, n in na.items():
                if lib.oracle_set_nalpha_order(int(order), int(n)):
                    raise RuntimeError("oracle_set_nalpha_order(%r, %r) refused" % (order, n))
        elif lib.oracle_set_nalpha(int(na)):
            raise RuntimeError("oracle_set_nalpha(%r) refused" % na)
    fm.argtypes = [P(S.CtlT), P(S.AtmT), P(S.ObsT), P(S.AeroT)]
    fm.restype = C.c_int if port else None
    if not port:
        lib.raytrace.argtypes = [P(S.CtlT), P(S.AtmT), P(S.ObsT), P(S.AeroT), P(LosT), C.c_int]
        lib.raytrace.restype = None
    ctl = S.make_ctl(**job["ctl"])
    aero = job.get("aero") or S.AeroT()
    atms, ray_atm, geom = job["atms"], np.asarray(job["ray_atm"]), job["geom"]
    nr, nd = len(ray_atm), ctl.nd
    out = {"rad": np.zeros((nr, nd)), "tau": np.zeros((nr, nd)),
           "tpz": np.zeros(nr), "tplon": np.zeros(nr), "tplat": np.zeros(nr)}
    if job.get("los"):
        out["nlos"] = np.zeros(nr, np.int32)
        out["los"] = []
    groups = []
    for ai in np.unique(ray_atm):
        idx = np.nonzero(ray_atm == ai)[0]
        for s in range(0, len(idx), S.NRMAX):
            groups.append((int(ai), idx[s:s + S.NRMAX]))

    def call(ai, idx):
        atm = _atm_struct(atms[ai])
        obs = S.make_obs(geom["obsz"][idx], geom["obslat"][idx],
                         geom["vpz"][idx], geom["vplat"][idx],
                         geom["obslon"][idx], geom["vplon"][idx],
                         geom["time"][idx])
        st = fm(C.byref(ctl), C.byref(atm), C.byref(obs), C.byref(aero))
        if port and st:
            raise RuntimeError("oracle_formod failed with status %d" % st)
        return atm, obs

    if job.get("warmup"):
        call(*groups[0])
    t0 = time.perf_counter()
    for ai, idx in groups:
        atm, obs = call(ai, idx)
        n = len(idx)
        out["rad"][idx] = S.arr(obs.rad)[:nd, :n].T
        out["tau"][idx] = S.arr(obs.tau)[:nd, :n].T
        out["tpz"][idx] = S.arr(obs.tpz)[:n]
        out["tplon"][idx] = S.arr(obs.tplon)[:n]
        out["tplat"][idx] = S.arr(obs.tplat)[:n]
    out["seconds"] = time.perf_counter() - t0
    if job.get("los") and port:
        lib.oracle_diagnostics.argtypes = [P(S.CtlT), P(S.AtmT), P(S.ObsT), P(S.AeroT),
                                           P(C.c_int), P(C.c_uint64)]
        out["digest"] = np.zeros((nr, nd), np.uint64)
        for ai, idx in groups:
            atm = _atm_struct(atms[ai])
            obs = S.make_obs(geom["obsz"][idx], geom["obslat"][idx],
                             geom["vpz"][idx], geom["vplat"][idx],
                             geom["obslon"][idx], geom["vplon"][idx],
                             geom["time"][idx])
            nl = np.zeros(len(idx), np.int32)
            dg = np.zeros((len(idx), nd), np.uint64)
            lib.oracle_diagnostics(C.byref(ctl), C.byref(atm), C.byref(obs), C.byref(aero),
                                   nl.ctypes.data_as(P(C.c_int)),
                                   dg.ctypes.data_as(P(C.c_uint64)))
            out["nlos"][idx] = nl
            out["digest"][idx] = dg
    elif job.get("los"):
        los = LosT()
        for ai, idx in groups:
            atm = _atm_struct(atms[ai])
            # formod applied hydrostatic balance to its copy; do the same
            obs = S.make_obs(geom["obsz"][idx], geom["obslat"][idx],
                             geom["vpz"][idx], geom["vplat"][idx],
                             geom["obslon"][idx], geom["vplon"][idx],
                             geom["time"][idx])
            lib.hydrostatic.argtypes = [P(S.CtlT), P(S.AtmT)]
            lib.hydrostatic(C.byref(ctl), C.byref(atm))
            for j, r in enumerate(idx):
                lib.raytrace(C.byref(ctl), C.byref(atm), C.byref(obs), C.byref(aero),
                             C.byref(los), j)
                out["nlos"][r] = los.np
                if job["los"] == "full":
                    n = los.np
                    ng = ctl.ng
                    out["los"].append({
                        "z": S.arr(los.z)[:n].copy(), "p": S.arr(los.p)[:n].copy(),
                        "t": S.arr(los.t)[:n].copy(), "ds": S.arr(los.ds)[:n].copy(),
                        "u": S.arr(los.u)[:n, :ng].copy(), "tsurf": los.tsurf})
    return out


def _helpers_child(job):
    """The forwardmodel.h helpers of library job["lib"] (the reference
    build, or the library under test) on one line of sight: read_tbl into a
    calloc'd tbl_t, then per LOS point intpol_tbl (path state carried),
    formod_continua and srcfunc_planck at the point's temperature; plus
    intpol_tbl_eps/_u on a few rows and locate_tbl on a float array.  The
    LOS (a los_t as bytes) comes from the reference's raytrace."""
    _silence()
    lib = C.CDLL(job["lib"])
    libc = C.CDLL(None)
    libc.calloc.restype = C.c_void_p
    libc.calloc.argtypes = [C.c_size_t, C.c_size_t]
    P = C.POINTER
    vp = C.c_void_p
    lib.read_tbl.argtypes = [P(S.CtlT), vp]
    lib.intpol_tbl.argtypes = [P(S.CtlT), vp, P(S.LosT), C.c_int, vp, vp]
    lib.formod_continua.argtypes = [P(S.CtlT), P(S.LosT), C.c_int, P(C.c_double)]
    lib.srcfunc_planck.argtypes = [P(S.CtlT), C.c_double, P(C.c_double)]
    for f in (lib.intpol_tbl_eps, lib.intpol_tbl_u):
        f.restype = C.c_double
        f.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double]
    lib.locate_tbl.restype = C.c_int
    lib.locate_tbl.argtypes = [P(C.c_float), C.c_int, C.c_double]
    ctl = S.make_ctl(**job["ctl"])
    los = S.LosT.from_buffer_copy(job["los"])
    ng, nd = ctl.ng, ctl.nd
    tbl = libc.calloc(1, C.sizeof(S.TblT))
    if not tbl:
        raise MemoryError("tbl_t")
    lib.read_tbl(C.byref(ctl), C.c_void_p(tbl))
    T = S.TblT

    def view(field, ctype, shape):
        off = getattr(T, field).offset
        n = int(np.prod(shape))
        return np.ctypeslib.as_array((ctype * n).from_address(tbl + off)).reshape(shape).copy()

    out = {"np": view("np", C.c_int, (S.NGMAX, S.NDMAX))[:ng, :nd],
           "nt": view("nt", C.c_int, (S.NGMAX, S.NDMAX, S.TBLNPMAX))[:ng, :nd],
           "nu": view("nu", C.c_int, (S.NGMAX, S.NDMAX, S.TBLNPMAX, S.TBLNTMAX))[:ng, :nd],
           "p": view("p", C.c_double, (S.NGMAX, S.NDMAX, S.TBLNPMAX))[:ng, :nd],
           "t": view("t", C.c_double, (S.NGMAX, S.NDMAX, S.TBLNPMAX, S.TBLNTMAX))[:ng, :nd]}
    # rows of emitter 0, channel 0 (the u and eps blocks of one table)
    blk = (S.TBLNPMAX, S.TBLNTMAX, S.TBLNUMAX)
    nblk = int(np.prod(blk))
    for f in ("u", "eps"):
        base = tbl + getattr(T, f).offset
        out[f + "00"] = np.ctypeslib.as_array((C.c_float * nblk).from_address(base)).reshape(blk).copy()
    tau_path = ((C.c_double * S.NDMAX) * S.NGMAX)()
    tau_seg = (C.c_double * S.NDMAX)()
    beta = (C.c_double * S.NDMAX)()
    src = (C.c_double * S.NDMAX)()
    seg, ctm, plk = [], [], []
    for ip in range(los.np):
        lib.intpol_tbl(C.byref(ctl), C.c_void_p(tbl), C.byref(los), ip, C.byref(tau_path),
                       C.byref(tau_seg))
        seg.append(np.array(tau_seg[:nd]))
        lib.formod_continua(C.byref(ctl), C.byref(los), ip, beta)
        ctm.append(np.array(beta[:nd]))
        lib.srcfunc_planck(C.byref(ctl), los.t[ip], src)
        plk.append(np.array(src[:nd]))
    out["tau_seg"], out["beta"], out["src"] = np.array(seg), np.array(ctm), np.array(plk)
    out["tau_path"] = np.array([tau_path[g][:nd] for g in range(ng)])
    vals = []
    for (ig, id_, ip, it) in ((0, 0, 10, 5), (1, nd - 1, 30, 20), (0, 1, 39, 29)):
        for x in np.logspace(12, 25, 7):
            vals.append(lib.intpol_tbl_eps(C.c_void_p(tbl), ig, id_, ip, it, float(x)))
        for e in np.linspace(0.0, 0.999, 7):
            vals.append(lib.intpol_tbl_u(C.c_void_p(tbl), ig, id_, ip, it, float(e)))
    out["lookups"] = np.array(vals)
    xs = (C.c_float * 9)(*[0.5, 1.0, 2.0, 2.0, 3.5, 7.0, 7.25, 9.0, 12.0])
    out["locate"] = np.array([lib.locate_tbl(xs, 9, float(x))
                              for x in (-1.0, 0.5, 1.999, 2.0, 2.0000001, 7.1, 11.99, 12.0, 99.0,
                                        float("nan"))])
    return out


def forwardmodel_helpers(ctl_kw, los_bytes, lib=REF_LIB, timeout=600):
    """Outputs of the forwardmodel.h helpers of lib on one line of sight
    (see _helpers_child)."""
    return _spawn({"helpers_job": True, "ctl": ctl_kw, "los": los_bytes, "lib": lib}, timeout)


def reference_los(ctl_kw, atm, geom, ir=0, timeout=600):
    """los_t (as bytes) of ray ir traced by the reference's raytrace through
    atm after its hydrostatic balance."""
    return _spawn({"los_job": True, "ctl": ctl_kw, "atm": atm, "geom": geom, "ir": ir},
                  timeout)


def _los_child(job):
    _silence()
    lib = C.CDLL(REF_LIB)
    P = C.POINTER
    lib.raytrace.argtypes = [P(S.CtlT), P(S.AtmT), P(S.ObsT), P(S.AeroT), P(S.LosT), C.c_int]
    lib.hydrostatic.argtypes = [P(S.CtlT), P(S.AtmT)]
    ctl = S.make_ctl(**job["ctl"])
    atm = _atm_struct(job["atm"])
    g = job["geom"]
    obs = S.make_obs(g["obsz"], g["obslat"], g["vpz"], g["vplat"], g["obslon"], g["vplon"],
                     g["time"])
    lib.hydrostatic(C.byref(ctl), C.byref(atm))
    los = S.LosT()
    aero = S.AeroT()
    lib.raytrace(C.byref(ctl), C.byref(atm), C.byref(obs), C.byref(aero), C.byref(los),
                 job["ir"])
    return bytes(los)


def _srcfunc_child(job):
    """The reference's srcfunc_sca (src/scatter.c:643-662: the thermal
    source of srcfunc_sca_1d or, for IP 2/3, srcfunc_sca_3d, plus
    srcfunc_sca_sun) at single points, with the queue inactive as formod
    leaves it (src/forwardmodel.c:54-55), after the reference's
    hydrostatic balance of the atmosphere.  Returns the sources [n][nd], the
    balanced pressures and the seconds per point."""
    _silence()
    lib = C.CDLL(REF_LIB)
    P = C.POINTER
    V3 = C.c_double * 3
    lib.hydrostatic.argtypes = [P(S.CtlT), P(S.AtmT)]
    lib.srcfunc_sca.argtypes = [P(S.CtlT), P(S.AtmT), P(S.AeroT), C.c_double, P(V3), P(V3),
                                C.c_int, P(C.c_double), C.c_int]
    lib.srcfunc_sca.restype = None
    ctl = S.make_ctl(**job["ctl"])
    ctl.queue.state = -1            # Queue_Inactive (src/workqueue.h:8)
    atm = _atm_struct(job["atm"])
    aero = S.AeroT.from_buffer_copy(job["aero"])
    lib.hydrostatic(C.byref(ctl), C.byref(atm))
    nd = ctl.nd
    src = (C.c_double * S.NDMAX)()
    out, secs = [], []
    for x, dx, il, sec in job["points"]:
        t0 = time.perf_counter()
        lib.srcfunc_sca(C.byref(ctl), C.byref(atm), C.byref(aero), float(sec), V3(*x), V3(*dx),
                        int(il), src, int(job["scattering"]))
        secs.append(time.perf_counter() - t0)
        out.append(np.array(src[:nd]))
    return {"src": np.array(out), "p": S.arr(atm.p)[:atm.np].copy(), "seconds": np.array(secs)}


def reference_srcfunc(ctl_kw, atm, aero, points, scattering, timeout=14400):
    """srcfunc_sca of the reference build at points [(x[3], dx[3], layer,
    time)], scattering order `scattering`; see _srcfunc_child."""
    return _spawn({"srcfunc_job": True, "ctl": ctl_kw, "atm": atm, "aero": bytes(aero),
                   "points": points, "scattering": scattering}, timeout)


REF_RET_LIB = os.path.join(HERE, "_ref", "libjurassic_ref_ret.so")


class GslMatrix(C.Structure):
    """gsl_matrix of the bundled GSL 1.15 (gsl/gsl_matrix_double.h)."""
    _fields_ = [("size1", C.c_size_t), ("size2", C.c_size_t), ("tda", C.c_size_t),
                ("data", C.POINTER(C.c_double)), ("block", C.c_void_p), ("owner", C.c_int)]


class GslVector(C.Structure):
    """gsl_vector of the bundled GSL 1.15 (gsl/gsl_vector_double.h)."""
    _fields_ = [("size", C.c_size_t), ("stride", C.c_size_t),
                ("data", C.POINTER(C.c_double)), ("block", C.c_void_p), ("owner", C.c_int)]


def kernel_available():
    return os.path.exists(REF_RET_LIB)


def _kernel_child(job):
    """The reference's kernel() (src/retrievalmodel.c:201-298) on one
    profile and the rays of geom; obs->rad starts at 0 with NaN where
    job["mask"] is set.  Also returns the state vector (atm2x after the
    call, i.e. with the hydrostatic pressures), its quantity and level
    indices, and the undisturbed radiances kernel() leaves in obs."""
    _silence()
    lib = C.CDLL(REF_RET_LIB)
    P = C.POINTER
    lib.gsl_matrix_alloc.restype = P(GslMatrix)
    lib.gsl_matrix_alloc.argtypes = [C.c_size_t, C.c_size_t]
    lib.gsl_vector_alloc.restype = P(GslVector)
    lib.gsl_vector_alloc.argtypes = [C.c_size_t]
    lib.atm2x.restype = C.c_size_t
    lib.atm2x.argtypes = [P(S.CtlT), P(S.AtmT), P(S.AeroT), C.c_void_p, C.c_void_p, C.c_void_p]
    lib.obs2y.restype = C.c_size_t
    lib.obs2y.argtypes = [P(S.CtlT), P(S.ObsT), C.c_void_p, C.c_void_p, C.c_void_p]
    lib.kernel.restype = None
    lib.kernel.argtypes = [P(S.CtlT), P(S.AtmT), P(S.ObsT), P(S.AeroT), P(GslMatrix)]
    ctl = S.make_ctl(**job["ctl"])
    atm = _atm_struct(job["atm"])
    g = job["geom"]
    obs = S.make_obs(g["obsz"], g["obslat"], g["vpz"], g["vplat"], g["obslon"], g["vplon"],
                     g["time"])
    nr, nd = obs.nr, ctl.nd
    rad = S.arr(obs.rad)
    mask = job.get("mask")
    if mask is not None:
        for ir in range(nr):
            for id_ in range(nd):
                if mask[ir][id_]:
                    rad[id_, ir] = np.nan
    aero = S.AeroT()
    if job.get("aerofile"):
        # the modes only: formod derives the optical properties itself for
        # aerosol retrievals (src/forwardmodel.c:34-36)
        lib.read_aero.argtypes = [C.c_char_p, C.c_char_p, P(S.CtlT), P(S.AeroT)]
        lib.get_opt_prop.argtypes = [P(S.CtlT), P(S.AeroT)]
        os.chdir(job["cwd"])
        lib.read_aero(None, job["aerofile"].encode(), C.byref(ctl), C.byref(aero))
        if not (ctl.retnn or ctl.retrr or ctl.retss):
            lib.get_opt_prop(C.byref(ctl), C.byref(aero))
    m = lib.obs2y(C.byref(ctl), C.byref(obs), None, None, None)
    n = lib.atm2x(C.byref(ctl), C.byref(atm), C.byref(aero), None, None, None)
    k = lib.gsl_matrix_alloc(m, n)
    t0 = time.perf_counter()
    lib.kernel(C.byref(ctl), C.byref(atm), C.byref(obs), C.byref(aero), k)
    seconds = time.perf_counter() - t0
    km = k.contents
    K = np.ctypeslib.as_array(km.data, shape=(m * km.tda,)).reshape(m, km.tda)[:, :n].copy()
    x = lib.gsl_vector_alloc(n)
    iqa = (C.c_int * max(n, 1))()
    ipa = (C.c_int * max(n, 1))()
    lib.atm2x(C.byref(ctl), C.byref(atm), C.byref(aero), x, iqa, ipa)
    xv = x.contents
    x0 = np.array([xv.data[i * xv.stride] for i in range(n)])
    return {"k": K, "x0": x0, "iqa": np.array(iqa[:n]), "ipa": np.array(ipa[:n]),
            "rad": S.arr(obs.rad)[:nd, :nr].T.copy(), "p": S.arr(atm.p)[:atm.np].copy(),
            "seconds": seconds}


def _state_vector_child(job):
    """The reference's atm2x, x2atm and obs2y (src/atmosphere.c:5-97,
    src/retrievalmodel.c:379-403,1103-1163) on one profile: the state
    vector, then x2atm of x * scale + shift, then the measurement vector of
    an obs_t whose radiances are job["rad"] ([nr][nd], NaN = masked)."""
    _silence()
    lib = C.CDLL(REF_RET_LIB)
    P = C.POINTER
    lib.gsl_vector_alloc.restype = P(GslVector)
    lib.gsl_vector_alloc.argtypes = [C.c_size_t]
    lib.atm2x.restype = C.c_size_t
    lib.atm2x.argtypes = [P(S.CtlT), P(S.AtmT), P(S.AeroT), C.c_void_p, C.c_void_p, C.c_void_p]
    lib.x2atm.restype = None
    lib.x2atm.argtypes = [P(S.CtlT), P(GslVector), P(S.AtmT), P(S.AeroT)]
    lib.obs2y.restype = C.c_size_t
    lib.obs2y.argtypes = [P(S.CtlT), P(S.ObsT), C.c_void_p, C.c_void_p, C.c_void_p]
    ctl = S.make_ctl(**job["ctl"])
    atm = _atm_struct(job["atm"])
    aero = S.AeroT()
    n = lib.atm2x(C.byref(ctl), C.byref(atm), C.byref(aero), None, None, None)
    x = lib.gsl_vector_alloc(max(n, 1))
    iqa = (C.c_int * max(n, 1))()
    ipa = (C.c_int * max(n, 1))()
    lib.atm2x(C.byref(ctl), C.byref(atm), C.byref(aero), x, iqa, ipa)
    xv = x.contents
    x0 = np.array([xv.data[i * xv.stride] for i in range(n)])
    for i in range(n):
        xv.data[i * xv.stride] = x0[i] * job["scale"] + job["shift"]
    lib.x2atm(C.byref(ctl), x, C.byref(atm), C.byref(aero))
    na = atm.np
    out = {"x0": x0, "iqa": np.array(iqa[:n]), "ipa": np.array(ipa[:n]),
           "p": S.arr(atm.p)[:na].copy(), "t": S.arr(atm.t)[:na].copy(),
           "q": S.arr(atm.q)[:ctl.ng, :na].copy(), "k": S.arr(atm.k)[:ctl.nw, :na].copy()}
    rad = np.asarray(job["rad"])
    obs = S.ObsT()
    obs.nr = rad.shape[0]
    S.arr(obs.rad)[:ctl.nd, :obs.nr] = rad.T
    m = lib.obs2y(C.byref(ctl), C.byref(obs), None, None, None)
    y = lib.gsl_vector_alloc(max(m, 1))
    ida = (C.c_int * max(m, 1))()
    ira = (C.c_int * max(m, 1))()
    lib.obs2y(C.byref(ctl), C.byref(obs), y, ida, ira)
    yv = y.contents
    out.update(y=np.array([yv.data[i * yv.stride] for i in range(m)]),
               ida=np.array(ida[:m]), ira=np.array(ira[:m]))
    return out


def reference_state_vector(ctl_kw, atm, rad, scale=1.0, shift=0.0, timeout=600):
    """atm2x / x2atm / obs2y of the reference (see _state_vector_child)."""
    return _spawn({"sv_job": True, "ctl": ctl_kw, "atm": atm, "rad": np.asarray(rad),
                   "scale": scale, "shift": shift}, timeout)


def reference_kernel(ctl_kw, atm, geom, mask=None, timeout=3600, aerofile=None, cwd=None):
    """Jacobian of the reference's kernel() for one profile (dict) and the
    rays of geom; mask [n_rays][nd] marks observations set to NaN; aerofile
    (read in cwd) supplies the aerosol/cloud modes."""
    return _spawn({"kernel_job": True, "ctl": ctl_kw, "atm": atm, "geom": geom,
                   "mask": None if mask is None else np.asarray(mask, bool),
                   "aerofile": aerofile, "cwd": cwd}, timeout)


PORT_LIB = os.path.join(HERE, "build", "libjscat_oracle.so")


def port_available():
    return os.path.exists(PORT_LIB)


def _aero_child(job):
    _silence()
    lib = C.CDLL(REF_LIB)
    P = C.POINTER
    lib.read_aero.argtypes = [C.c_char_p, C.c_char_p, P(S.CtlT), P(S.AeroT)]
    lib.get_opt_prop.argtypes = [P(S.CtlT), P(S.AeroT)]
    ctl = S.make_ctl(**job["ctl"])
    aero = S.AeroT()
    os.chdir(job["cwd"])
    lib.read_aero(None, job["aerofile"].encode(), C.byref(ctl), C.byref(aero))
    t0 = time.perf_counter()
    lib.get_opt_prop(C.byref(ctl), C.byref(aero))
    seconds = time.perf_counter() - t0
    if job.get("timed"):
        return {"aero": bytes(aero), "seconds": seconds}
    return bytes(aero)


def reference_aero(ctl_kw, aerofile, cwd, timeout=600, timed=False):
    """aero_t (as bytes) from the reference's read_aero + get_opt_prop
    (Mie optical properties, src/scatter.c:330-508,583-639), run in cwd;
    with timed=True a dict with the bytes and get_opt_prop's seconds."""
    return _spawn({"aero_job": True, "ctl": ctl_kw, "aerofile": aerofile, "cwd": cwd,
                   "timed": timed}, timeout)


def run_port(ctl_kw, atms, ray_atm, geom, aero=None, threads=None, warmup=False, los=False,
             timeout=1800, nalpha=None):
    """Same as run() with the C restatement (oracle/jurassic_oracle.c)
    instead of the reference build; with los=True it also returns the
    per-(ray, channel) EGA index digests.  nalpha: secondary pencils per
    scattering point (the reference's 28 by default)."""
    return run(ctl_kw, atms, ray_atm, geom, aero=aero, threads=threads, warmup=warmup,
               los=los, lib=PORT_LIB, timeout=timeout, port=True, nalpha=nalpha)


def run(ctl_kw, atms, ray_atm, geom, aero=None, threads=None, warmup=False,
        los=False, lib=None, timeout=1800, port=False, nalpha=None):
    """Reference formod over profiles atms (list of dicts) and rays.
    Returns rad/tau [n_rays][nd], tpz/tplon/tplat, seconds (wall time of
    the formod calls after the optional warm-up call), and with los=True
    the LOS point count per ray (los='full' also returns the LOS records)."""
    import pickle
    import subprocess
    import tempfile
    job = {"ctl": ctl_kw, "atms": atms, "ray_atm": np.asarray(ray_atm),
           "geom": geom, "aero": None if aero is None else bytes(aero),
           "threads": threads, "warmup": warmup, "los": los, "port": port,
           "nalpha": nalpha}
    if lib:
        job["lib"] = lib
    return _spawn(job, timeout)


def _spawn(job, timeout):
    import pickle
    import subprocess
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        jf, of = os.path.join(d, "job.pkl"), os.path.join(d, "out.pkl")
        with open(jf, "wb") as f:
            pickle.dump(job, f)
        res = subprocess.run([sys.executable, os.path.abspath(__file__), jf, of],
                             capture_output=True, text=True, timeout=timeout)
        if res.returncode != 0 or not os.path.exists(of):
            raise RuntimeError("reference run failed (%d): %s" %
                               (res.returncode, res.stderr[-2000:]))
        with open(of, "rb") as f:
            return pickle.load(f)


if __name__ == "__main__":
    import pickle
    with open(sys.argv[1], "rb") as f:
        _job = pickle.load(f)
    if _job.get("aero_job"):
        _out = _aero_child(_job)
    elif _job.get("kernel_job"):
        _out = _kernel_child(_job)
    elif _job.get("srcfunc_job"):
        _out = _srcfunc_child(_job)
    elif _job.get("helpers_job"):
        _out = _helpers_child(_job)
    elif _job.get("los_job"):
        _out = _los_child(_job)
    elif _job.get("sv_job"):
        _out = _state_vector_child(_job)
    else:
        if _job.get("aero") is not None:
            _job["aero"] = S.AeroT.from_buffer_copy(_job["aero"])
        _out = _child(_job)
    with open(sys.argv[2], "wb") as f:
        pickle.dump(_out, f)
