"""ctypes mirrors of the forward-model boundary structs.

Same field order, types and dimensions as the reference's src/jurassic.h
(ctl_t :228-348, obs_t :397-438, aero_t :475-535, atm_t :538-570, queue_t
src/workqueue.h:13-25), hence the same memory layout as the C structs of
include/jurassic_b200.h.  Arrays are reachable as numpy views via arr().
"""
import ctypes as C

import numpy as np

LEN = 5000
NWMAX = 5
NDMAX = 130
NGMAX = 25
NLOS = 10000
NPMAX = 1000
NRMAX = 1000
TBLNPMAX = 50
TBLNTMAX = 30
TBLNUMAX = 320
SCAMOD = 30
NLMAX = 10
NTHETA = 181


class QueueItemT(C.Structure):
    _fields_ = [("input", C.c_void_p), ("result", C.c_void_p), ("ir", C.c_int)]


class QueueT(C.Structure):
    _fields_ = [("items", C.POINTER(QueueItemT)), ("capacity", C.c_int),
                ("begin", C.c_int), ("end", C.c_int), ("state", C.c_int)]


class CtlT(C.Structure):
    _fields_ = [
        ("ng", C.c_int),
        ("emitter", (C.c_char * LEN) * NGMAX),
        ("nd", C.c_int),
        ("nw", C.c_int),
        ("nu", C.c_double * NDMAX),
        ("window", C.c_int * NDMAX),
        ("tblbase", C.c_char * LEN),
        ("hydz", C.c_double),
        ("ctm_co2", C.c_int), ("ctm_h2o", C.c_int),
        ("ctm_n2", C.c_int), ("ctm_o2", C.c_int),
        ("sca_n", C.c_int),
        ("sca_mult", C.c_int),
        ("sca_ext", C.c_char * LEN),
        ("ip", C.c_int),
        ("cz", C.c_double), ("cx", C.c_double),
        ("refrac", C.c_int),
        ("rayds", C.c_double), ("raydz", C.c_double), ("transs", C.c_double),
        ("fov", C.c_char * LEN),
        ("retp_zmin", C.c_double), ("retp_zmax", C.c_double),
        ("rett_zmin", C.c_double), ("rett_zmax", C.c_double),
        ("retq_zmin", C.c_double * NGMAX), ("retq_zmax", C.c_double * NGMAX),
        ("retk_zmin", C.c_double * NWMAX), ("retk_zmax", C.c_double * NWMAX),
        ("retnn_zmin", C.c_double), ("retnn_zmax", C.c_double),
        ("retnn", C.c_int), ("retrr", C.c_int), ("retss", C.c_int),
        ("write_bbt", C.c_int),
        ("write_matrix", C.c_int),
        ("queue", QueueT),
    ]


class ObsT(C.Structure):
    _fields_ = [
        ("nr", C.c_int),
        ("time", C.c_double * NRMAX),
        ("obsz", C.c_double * NRMAX), ("obslon", C.c_double * NRMAX),
        ("obslat", C.c_double * NRMAX),
        ("vpz", C.c_double * NRMAX), ("vplon", C.c_double * NRMAX),
        ("vplat", C.c_double * NRMAX),
        ("tpz", C.c_double * NRMAX), ("tplon", C.c_double * NRMAX),
        ("tplat", C.c_double * NRMAX),
        ("tau", (C.c_double * NRMAX) * NDMAX),
        ("rad", (C.c_double * NRMAX) * NDMAX),
    ]


class AeroT(C.Structure):
    _fields_ = [
        ("nm", C.c_int),
        ("top_mod", C.c_double * SCAMOD), ("bottom_mod", C.c_double * SCAMOD),
        ("trans_mod", C.c_double * SCAMOD),
        ("type", (C.c_char * LEN) * SCAMOD),
        ("filepath", (C.c_char * LEN) * SCAMOD),
        ("nn", C.c_double * SCAMOD), ("rr", C.c_double * SCAMOD),
        ("ss", C.c_double * SCAMOD),
        ("nl", C.c_int),
        ("nmod", C.c_int * NLMAX),
        ("top", C.c_double * NLMAX), ("bottom", C.c_double * NLMAX),
        ("trans", C.c_double * NLMAX),
        ("beta_e", (C.c_double * NDMAX) * NLMAX),
        ("beta_s", (C.c_double * NDMAX) * NLMAX),
        ("beta_a", (C.c_double * NDMAX) * NLMAX),
        ("p", ((C.c_double * NTHETA) * NDMAX) * NLMAX),
    ]


class AtmT(C.Structure):
    _fields_ = [
        ("np", C.c_int),
        ("time", C.c_double * NPMAX),
        ("z", C.c_double * NPMAX), ("lon", C.c_double * NPMAX),
        ("lat", C.c_double * NPMAX),
        ("p", C.c_double * NPMAX), ("t", C.c_double * NPMAX),
        ("q", (C.c_double * NPMAX) * NGMAX),
        ("k", (C.c_double * NPMAX) * NWMAX),
        ("init", C.c_int),
    ]


def arr(field):
    """numpy view (no copy) of a ctypes array field."""
    return np.ctypeslib.as_array(field)


def set_str(obj, name, value, index=None):
    """Store a Python string into a fixed char array field (obj.name, or
    obj.name[index] for arrays of strings)."""
    b = value.encode()
    if len(b) >= LEN:
        raise ValueError("string too long for field %s" % name)
    if index is None:
        setattr(obj, name, b)
    else:
        elem = getattr(obj, name)[index]
        C.memset(C.addressof(elem), 0, LEN)
        C.memmove(C.addressof(elem), b, len(b))


class LosT(C.Structure):
    """los_t (src/jurassic.h:352-393): one ray's line of sight."""
    _fields_ = [
        ("np", C.c_int),
        ("z", C.c_double * NLOS), ("lon", C.c_double * NLOS),
        ("lat", C.c_double * NLOS), ("p", C.c_double * NLOS),
        ("t", C.c_double * NLOS),
        ("q", (C.c_double * NGMAX) * NLOS),
        ("k", (C.c_double * NWMAX) * NLOS),
        ("aeroi", C.c_int * NLOS),
        ("aerofac", C.c_double * NLOS),
        ("tsurf", C.c_double),
        ("ds", C.c_double * NLOS),
        ("u", (C.c_double * NGMAX) * NLOS),
    ]


TBLNSMAX = 1201


class TblT(C.Structure):
    """tbl_t (src/jurassic.h:438-471), about 12.5 GB: for layout checks and
    pointer arithmetic only (allocate it with calloc, never as a ctypes
    instance)."""
    _fields_ = [
        ("np", (C.c_int * NDMAX) * NGMAX),
        ("nt", ((C.c_int * TBLNPMAX) * NDMAX) * NGMAX),
        ("nu", (((C.c_int * TBLNTMAX) * TBLNPMAX) * NDMAX) * NGMAX),
        ("p", ((C.c_double * TBLNPMAX) * NDMAX) * NGMAX),
        ("t", (((C.c_double * TBLNTMAX) * TBLNPMAX) * NDMAX) * NGMAX),
        ("u", ((((C.c_float * TBLNUMAX) * TBLNTMAX) * TBLNPMAX) * NDMAX) * NGMAX),
        ("eps", ((((C.c_float * TBLNUMAX) * TBLNTMAX) * TBLNPMAX) * NDMAX) * NGMAX),
        ("st", C.c_double * TBLNSMAX),
        ("sr", (C.c_double * TBLNSMAX) * NDMAX),
    ]


def make_ctl(emitters, nus, tblbase, **kw):
    """ctl_t with the defaults of the reference's read_ctl
    (src/control.c:7-100), then the keyword overrides (lower-case names)."""
    ctl = CtlT()
    ctl.ng = len(emitters)
    for i, e in enumerate(emitters):
        set_str(ctl, "emitter", e, i)
    ctl.nd = len(nus)
    for i, v in enumerate(nus):
        ctl.nu[i] = float(v)
        ctl.window[i] = 0
    ctl.nw = 1
    set_str(ctl, "tblbase", tblbase)
    ctl.hydz = -999.0
    ctl.ctm_co2 = ctl.ctm_h2o = ctl.ctm_n2 = ctl.ctm_o2 = 1
    ctl.sca_n = 0
    ctl.sca_mult = 1
    set_str(ctl, "sca_ext", "beta_a")
    ctl.ip = 1
    ctl.cz = ctl.cx = 0.0
    ctl.refrac = 1
    ctl.rayds = 10.0
    ctl.raydz = 1.0
    ctl.transs = 0.02
    set_str(ctl, "fov", "-")
    for f in ("retp_zmin", "retp_zmax", "rett_zmin", "rett_zmax",
              "retnn_zmin", "retnn_zmax"):
        setattr(ctl, f, -999.0)
    for i in range(NGMAX):
        ctl.retq_zmin[i] = ctl.retq_zmax[i] = -999.0
    for i in range(NWMAX):
        ctl.retk_zmin[i] = ctl.retk_zmax[i] = -999.0
    ctl.retnn = ctl.retrr = ctl.retss = 0
    ctl.write_bbt = 0
    ctl.write_matrix = 0
    ctl.queue.capacity = -1
    for k, v in kw.items():
        if k in ("sca_ext", "fov", "tblbase"):
            set_str(ctl, k, v)
        elif k == "window":
            for i, w in enumerate(v):
                ctl.window[i] = int(w)
        elif k in ("retq_zmin", "retq_zmax", "retk_zmin", "retk_zmax"):
            for i, w in enumerate(v):
                getattr(ctl, k)[i] = float(w)
        else:
            setattr(ctl, k, v)
    return ctl


def make_atm(z, p, t, q, k=None, lon=None, lat=None):
    """atm_t from 1-D arrays; q is [ng][np], k is [nw][np]."""
    atm = AtmT()
    n = len(z)
    if n > NPMAX:
        raise ValueError("too many levels")
    atm.np = n
    arr(atm.z)[:n] = z
    arr(atm.p)[:n] = p
    arr(atm.t)[:n] = t
    arr(atm.lon)[:n] = 0.0 if lon is None else lon
    arr(atm.lat)[:n] = 0.0 if lat is None else lat
    q = np.atleast_2d(q)
    arr(atm.q)[:q.shape[0], :n] = q
    if k is not None:
        k = np.atleast_2d(k)
        arr(atm.k)[:k.shape[0], :n] = k
    return atm


def make_obs(obsz, obslat, vpz, vplat, obslon=None, vplon=None, time=None):
    """obs_t from per-ray geometry arrays (radiances zero, i.e. unmasked)."""
    obs = ObsT()
    n = len(obsz)
    if n > NRMAX:
        raise ValueError("too many rays")
    obs.nr = n
    arr(obs.obsz)[:n] = obsz
    arr(obs.obslat)[:n] = obslat
    arr(obs.vpz)[:n] = vpz
    arr(obs.vplat)[:n] = vplat
    arr(obs.obslon)[:n] = 0.0 if obslon is None else obslon
    arr(obs.vplon)[:n] = 0.0 if vplon is None else vplon
    arr(obs.time)[:n] = 0.0 if time is None else time
    return obs
