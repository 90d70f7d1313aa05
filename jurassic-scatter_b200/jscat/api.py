"""Python host mirror of the forward-model interface.

formod(ctl, atm, obs, aero) calls the drop-in C entry point with the
reference's structs (src/forwardmodel.c:15).  Model/Batch wrap the batch
C-ABI for many atmospheres and rays per launch; arrays are numpy, copies
to and from the device happen inside the C library.
"""
import ctypes as C

import numpy as np

from . import lib as L
from . import structs as S

_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)


def _dptr(a):
    return a.ctypes.data_as(_D) if a is not None else None


def _iptr(a):
    return a.ctypes.data_as(_I) if a is not None else None


def formod(ctl, atm, obs, aero=None, exit_on_error=False):
    """Drop-in forward model on the structs; raises JscError on failure
    (unless exit_on_error, which keeps the reference's exit behaviour)."""
    lib = L.load()
    if aero is None:
        aero = S.AeroT()
    lib.jsc_set_exit_on_error(1 if exit_on_error else 0)
    lib.formod(C.byref(ctl), C.byref(atm), C.byref(obs), C.byref(aero))
    L.check(lib.jsc_last_status(), "formod")


def formod_pencil(ctl, atm, obs, aero=None, scattering=0, ir=0):
    """Drop-in formod_pencil: ray ir of obs through atm as given, on the
    GPU, scattering sources of order `scattering`; raises JscError on
    failure."""
    lib = L.load()
    if aero is None:
        aero = S.AeroT()
    lib.jsc_set_exit_on_error(0)
    lib.formod_pencil(C.byref(ctl), C.byref(atm), C.byref(obs), C.byref(aero),
                      int(scattering), int(ir))
    L.check(lib.jsc_last_status(), "formod_pencil")


def srcfunc_sca(ctl, atm, aero, x, dx, layer, sec, scattering=1):
    """Scattering sources [n][nd] at n points on the GPU (jsc_srcfunc_sca):
    x, dx [n][3] Cartesian position and line-of-sight direction [km],
    layer [n], sec [n]; atm as given (hydrostatically balanced by the
    caller)."""
    x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 3)
    dx = np.ascontiguousarray(dx, dtype=np.float64).reshape(-1, 3)
    n = len(x)
    layer = np.ascontiguousarray(layer, dtype=np.int32)
    sec = np.ascontiguousarray(sec, dtype=np.float64)
    src = np.zeros((n, ctl.nd))
    L.check(L.load().jsc_srcfunc_sca(C.byref(ctl), C.byref(atm), C.byref(aero), n, _dptr(x),
                                     _dptr(dx), _iptr(layer), _dptr(sec), int(scattering),
                                     _dptr(src)), "jsc_srcfunc_sca")
    return src


def read_aero(ctl, filename, dirname=None):
    """aero_t with the modes of an aerosol file (jsc_read_aero)."""
    aero = S.AeroT()
    L.check(L.load().jsc_read_aero(None if dirname is None else dirname.encode(),
                                   filename.encode(), C.byref(ctl), C.byref(aero)),
            "jsc_read_aero")
    return aero


def get_opt_prop(ctl, aero):
    """Layers and optical properties of aero's modes, Mie series on the GPU
    (jsc_get_opt_prop)."""
    L.check(L.load().jsc_get_opt_prop(C.byref(ctl), C.byref(aero)), "jsc_get_opt_prop")
    return aero


def atm2x(ctl, atm, aero=None):
    """State vector, quantity codes and levels (jsc_atm2x)."""
    lib = L.load()
    aero = S.AeroT() if aero is None else aero
    n = lib.jsc_atm2x(C.byref(ctl), C.byref(atm), C.byref(aero), None, None, None)
    x = np.zeros(n)
    iqa = np.zeros(n, np.int32)
    ipa = np.zeros(n, np.int32)
    if n:
        lib.jsc_atm2x(C.byref(ctl), C.byref(atm), C.byref(aero), _dptr(x), _iptr(iqa),
                      _iptr(ipa))
    return x, iqa, ipa


def x2atm(ctl, x, atm, aero=None):
    """Write a state vector back into atm (and aero) (jsc_x2atm)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    L.load().jsc_x2atm(C.byref(ctl), _dptr(x), C.byref(atm),
                       C.byref(S.AeroT() if aero is None else aero))


def obs2y(ctl, obs):
    """Measurement vector and its channel and ray indices (jsc_obs2y)."""
    lib = L.load()
    m = lib.jsc_obs2y(C.byref(ctl), C.byref(obs), None, None, None)
    y = np.zeros(m)
    ida = np.zeros(m, np.int32)
    ira = np.zeros(m, np.int32)
    if m:
        lib.jsc_obs2y(C.byref(ctl), C.byref(obs), _dptr(y), _iptr(ida), _iptr(ira))
    return y, ida, ira


def kernel(ctl, atm, obs, aero=None):
    """Jacobian [m][n] of the measurement vector by finite differences,
    undisturbed and disturbed forward models in one GPU batch (jsc_kernel,
    the reference's kernel()).  Like the reference it also leaves formod's
    results in atm (hydrostatic pressure) and obs (radiances)."""
    lib = L.load()
    aero = S.AeroT() if aero is None else aero
    m = lib.jsc_obs2y(C.byref(ctl), C.byref(obs), None, None, None)
    n = lib.jsc_atm2x(C.byref(ctl), C.byref(atm), C.byref(aero), None, None, None)
    k = np.zeros((m, n))
    L.check(lib.jsc_kernel(C.byref(ctl), C.byref(atm), C.byref(obs), C.byref(aero),
                           _dptr(k) if k.size else None, m, n, n), "jsc_kernel")
    return k


def brightness(rad, nu):
    return L.load().brightness(float(rad), float(nu))


class Model:
    """Device-resident tables, Planck and continuum data for one ctl."""

    def __init__(self, ctl, device=0):
        lib = L.load()
        self.ctl = ctl
        self.h = C.c_void_p()
        L.check(lib.jsc_model_create(C.byref(ctl), int(device), C.byref(self.h)),
                "jsc_model_create")

    @property
    def table_bytes(self):
        return L.load().jsc_model_table_bytes(self.h)

    def close(self):
        if self.h:
            L.load().jsc_model_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Device buffers for up to max_rays rays over max_atm profiles."""

    def __init__(self, model, ctl, max_atm, max_levels, max_rays, max_seg=0):
        lib = L.load()
        self.model = model
        self.ctl = ctl
        self.nd = ctl.nd
        self.h = C.c_void_p()
        L.check(lib.jsc_batch_create(model.h, C.byref(ctl), int(max_atm),
                                     int(max_levels), int(max_rays),
                                     int(max_seg), C.byref(self.h)),
                "jsc_batch_create")
        self._keep = None

    def upload(self, inp, stream=None):
        """inp: dict with atm_off (int32 [n_atm+1]), z/lon/lat/p/t
        ([n_levels]), q ([ng][n_levels]), k ([nw][n_levels]), ray_atm
        (int32 [n_rays]) and time/obsz/obslon/obslat/vpz/vplon/vplat."""
        a = {}
        for k in ("z", "lon", "lat", "p", "t", "time", "obsz", "obslon",
                  "obslat", "vpz", "vplon", "vplat"):
            v = inp.get(k)
            a[k] = None if v is None else np.ascontiguousarray(v, dtype=np.float64)
        for k in ("q", "k"):
            v = inp.get(k)
            a[k] = None if v is None else np.ascontiguousarray(v, dtype=np.float64)
        a["atm_off"] = np.ascontiguousarray(inp["atm_off"], dtype=np.int32)
        a["ray_atm"] = np.ascontiguousarray(inp["ray_atm"], dtype=np.int32)
        bi = L.BatchInput()
        bi.n_atm = len(a["atm_off"]) - 1
        bi.n_levels = len(a["z"])
        bi.atm_off = _iptr(a["atm_off"])
        for k in ("z", "lon", "lat", "p", "t", "q", "k", "time", "obsz",
                  "obslon", "obslat", "vpz", "vplon", "vplat"):
            setattr(bi, k, _dptr(a[k]))
        bi.n_rays = len(a["ray_atm"])
        bi.ray_atm = _iptr(a["ray_atm"])
        self._keep = (a, bi)  # alive until the stream has consumed them
        self.n_rays = bi.n_rays
        L.check(L.load().jsc_batch_upload(self.h, C.byref(bi), stream),
                "jsc_batch_upload")

    def run(self, stream=None):
        L.check(L.load().jsc_batch_run(self.h, stream), "jsc_batch_run")

    def download(self, stream=None, out=None):
        nr, nd = self.n_rays, self.nd
        if out is None:
            out = {"rad": np.empty((nr, nd)), "tau": np.empty((nr, nd)),
                   "tpz": np.empty(nr), "tplon": np.empty(nr),
                   "tplat": np.empty(nr), "nlos": np.empty(nr, np.int32)}
        bo = L.BatchOutput()
        bo.rad = _dptr(out.get("rad"))
        bo.tau = _dptr(out.get("tau"))
        bo.tpz = _dptr(out.get("tpz"))
        bo.tplon = _dptr(out.get("tplon"))
        bo.tplat = _dptr(out.get("tplat"))
        bo.nlos = _iptr(out.get("nlos"))
        L.check(L.load().jsc_batch_download(self.h, C.byref(bo), stream),
                "jsc_batch_download")
        return out

    def set_digest(self, on=True):
        L.check(L.load().jsc_batch_set_digest(self.h, 1 if on else 0), "jsc_batch_set_digest")

    def index_digest(self):
        out = np.empty((self.n_rays, self.nd), np.uint64)
        L.check(L.load().jsc_batch_index_digest(self.h, out.ctypes.data_as(C.POINTER(C.c_uint64))),
                "jsc_batch_index_digest")
        return out

    def autotune(self, stream=None):
        """Pick the fastest EGA kernel launch variant on this batch."""
        L.check(L.load().jsc_batch_autotune(self.h, stream), "jsc_batch_autotune")
        return self.variant()

    def variant(self):
        v, b, mb = C.c_int(), C.c_int(), C.c_int()
        lib = L.load()
        L.check(lib.jsc_batch_variant(self.h, C.byref(v), C.byref(b), C.byref(mb)),
                "jsc_batch_variant")
        ms = [lib.jsc_batch_variant_ms(self.h, i) for i in range(32)]
        while ms and ms[-1] < 0:  # variants past the last one report -1
            ms.pop()
        return {"variant": v.value, "block": b.value, "min_blocks": mb.value,
                "variant_ms": [round(x, 3) for x in ms]}

    def set_aero(self, aero):
        """Aerosol/cloud layers (an AeroT) for runs with ctl.sca_n > 0."""
        L.check(L.load().jsc_batch_set_aero(self.h, C.byref(aero)), "jsc_batch_set_aero")

    def scatter_samples(self, depth=None):
        """Features [n][8] and plain scattering sources [n][nd] of the last
        run's scattering points (depth: those of the batch generation at
        that scattering depth, default this batch's own)."""
        lib = L.load()
        n = C.c_int64()
        if depth is None:
            def call(f, s_, m):
                return lib.jsc_batch_scatter_samples(self.h, f, s_, m, C.byref(n))
        else:
            def call(f, s_, m):
                return lib.jsc_batch_scatter_samples_depth(self.h, int(depth), f, s_, m,
                                                           C.byref(n))
        L.check(call(None, None, 0), "jsc_batch_scatter_samples")
        feat = np.empty((n.value, Surrogate.NF), np.float32)
        src = np.empty((n.value, self.nd))
        if n.value:
            L.check(call(_fptr(feat), _dptr(src), n.value), "jsc_batch_scatter_samples")
        return feat, src

    def set_surrogate(self, sur, tol_rel=0.05, check_stride=64, depth=None):
        """Attach a surrogate (None: none) for this batch's scattering
        points, or for those of another scattering order (depth)."""
        h = sur.h if sur is not None else None
        if depth is None:
            L.check(L.load().jsc_batch_set_surrogate(self.h, h, float(tol_rel), int(check_stride)),
                    "jsc_batch_set_surrogate")
        else:
            L.check(L.load().jsc_batch_set_surrogate_depth(self.h, int(depth), h, float(tol_rel),
                                                           int(check_stride)),
                    "jsc_batch_set_surrogate_depth")

    def surrogate_stats(self, depth=None):
        """Surrogate counts of the last run (depth: those of the batch
        generation at that scattering depth, which adds the mean checked
        deviation)."""
        p, f, c, u = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int()
        e, mean = C.c_double(), C.c_double()
        if depth is None:
            st = L.load().jsc_batch_surrogate_stats(self.h, C.byref(p), C.byref(f), C.byref(c),
                                                    C.byref(e), C.byref(u))
        else:
            st = L.load().jsc_batch_surrogate_stats_depth(self.h, int(depth), C.byref(p),
                                                          C.byref(f), C.byref(c), C.byref(e),
                                                          C.byref(mean), C.byref(u))
        L.check(st, "jsc_batch_surrogate_stats")
        out = {"points": p.value, "fallback": f.value, "checked": c.value,
               "max_rel_err": e.value, "used": bool(u.value)}
        if depth is not None:
            out["mean_rel_err"] = mean.value
        return out

    def set_variant(self, variant):
        """EGA launch variant (-1: default); see jsc_batch_set_variant."""
        L.check(L.load().jsc_batch_set_variant(self.h, int(variant)), "jsc_batch_set_variant")

    def set_nalpha(self, nalpha):
        """Secondary pencils per scattering point (even, 10..28; 28 default)."""
        L.check(L.load().jsc_batch_set_nalpha(self.h, int(nalpha)), "jsc_batch_set_nalpha")

    def set_nalpha_depth(self, depth, nalpha):
        """Pencils per scattering point of one scattering order."""
        L.check(L.load().jsc_batch_set_nalpha_depth(self.h, int(depth), int(nalpha)),
                "jsc_batch_set_nalpha_depth")

    def set_timing(self, on=True):
        L.load().jsc_batch_set_timing(self.h, 1 if on else 0)

    def kernel_ms(self, name):
        return L.load().jsc_batch_kernel_ms(self.h, name.encode())

    def counters(self):
        a, b = C.c_int64(), C.c_int64()
        L.check(L.load().jsc_batch_counters(self.h, C.byref(a), C.byref(b)),
                "jsc_batch_counters")
        return a.value, b.value

    def close(self):
        if self.h:
            L.load().jsc_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def formod_batch(ctl, inp, device=0, model=None, digest=False, aero=None, nalpha=None,
                 timing=False, variant=None):
    """One-shot batch forward model: returns dict of rad/tau/tp*/nlos (and
    the per-(ray, channel) EGA index digests when digest=True).  aero: an
    AeroT with the layers and optical properties when ctl.sca_n > 0;
    nalpha: secondary pencils per scattering point; timing: adds the
    per-stage milliseconds as out["ms"]."""
    own = model is None
    m = Model(ctl, device) if own else model
    nl = len(inp["z"])
    b = Batch(m, ctl, len(inp["atm_off"]) - 1, nl, max(1, len(inp["ray_atm"])))
    try:
        if aero is not None:
            b.set_aero(aero)
        if digest:
            b.set_digest(True)
        if nalpha is not None:
            b.set_nalpha(nalpha)
        if variant is not None:
            b.set_variant(variant)
        if timing:
            b.set_timing(True)
        b.upload(inp)
        b.run()
        out = b.download()
        if timing:
            out["ms"] = {k: b.kernel_ms(k) for k in ("hydrostatic", "raytrace", "scatter",
                                                     "continua", "ega_rt")}
        if digest:
            out["digest"] = b.index_digest()
        return out
    finally:
        b.close()
        if own:
            m.close()


def formod_batch_noalloc(ctl, inp, model, stream=None):
    """jsc_formod_batch_noalloc: the clear-air batch forward model with every
    per-call device buffer taken from the library's static scratch (no device
    allocation).  model: a Model for ctl.  Returns rad/tau/tp*/nlos."""
    a = {k: None if inp.get(k) is None else np.ascontiguousarray(inp[k], dtype=np.float64)
         for k in ("z", "lon", "lat", "p", "t", "q", "k", "time", "obsz", "obslon",
                   "obslat", "vpz", "vplon", "vplat")}
    a["atm_off"] = np.ascontiguousarray(inp["atm_off"], dtype=np.int32)
    a["ray_atm"] = np.ascontiguousarray(inp["ray_atm"], dtype=np.int32)
    bi = L.BatchInput()
    bi.n_atm = len(a["atm_off"]) - 1
    bi.n_levels = len(a["z"])
    bi.n_rays = len(a["ray_atm"])
    bi.atm_off = _iptr(a["atm_off"])
    bi.ray_atm = _iptr(a["ray_atm"])
    for k in ("z", "lon", "lat", "p", "t", "q", "k", "time", "obsz", "obslon",
              "obslat", "vpz", "vplon", "vplat"):
        setattr(bi, k, _dptr(a[k]))
    nr, nd = bi.n_rays, ctl.nd
    out = {"rad": np.empty((nr, nd)), "tau": np.empty((nr, nd)), "tpz": np.empty(nr),
           "tplon": np.empty(nr), "tplat": np.empty(nr), "nlos": np.empty(nr, np.int32)}
    bo = L.BatchOutput()
    bo.rad, bo.tau = _dptr(out["rad"]), _dptr(out["tau"])
    bo.tpz, bo.tplon, bo.tplat = _dptr(out["tpz"]), _dptr(out["tplon"]), _dptr(out["tplat"])
    bo.nlos = _iptr(out["nlos"])
    L.check(L.load().jsc_formod_batch_noalloc(model.h, C.byref(ctl), C.byref(bi),
                                              C.byref(bo), stream),
            "jsc_formod_batch_noalloc")
    return out


class GraphBatch:
    """A fixed-capacity batch whose upload + run + download is captured once
    into a CUDA graph for one input shape (n_atm, n_levels, n_rays).
    run(inp) copies inp into the pinned staging arrays the graph reads,
    replays it and returns the outputs.  pin(a) must return a pinned copy
    of a numpy array (e.g. through torch's pin_memory)."""

    _KEYS = ("z", "lon", "lat", "p", "t", "q", "k", "time", "obsz", "obslon", "obslat",
             "vpz", "vplon", "vplat")

    def __init__(self, model, ctl, inp, stream, pin, max_seg=0, aero=None, variant=-1,
                 nalpha=None, fixed_points=None):
        lib = L.load()
        self.nd = ctl.nd
        self.stream = stream
        n_atm = len(inp["atm_off"]) - 1
        self.batch = Batch(model, ctl, n_atm, len(inp["z"]), len(inp["ray_atm"]), max_seg)
        if aero is not None:
            self.batch.set_aero(aero)
        if variant >= 0:
            self.batch.set_variant(variant)
        if nalpha is not None:
            self.batch.set_nalpha(nalpha)
        if fixed_points is not None:
            L.check(lib.jsc_batch_set_fixed_points(self.batch.h, int(fixed_points)),
                    "jsc_batch_set_fixed_points")
        L.check(lib.jsc_batch_set_fixed(self.batch.h, 1), "jsc_batch_set_fixed")
        self.host = {k: pin(np.ascontiguousarray(inp[k], dtype=np.float64)) for k in self._KEYS}
        self.host["atm_off"] = pin(np.ascontiguousarray(inp["atm_off"], dtype=np.int32))
        self.host["ray_atm"] = pin(np.ascontiguousarray(inp["ray_atm"], dtype=np.int32))
        nr = len(inp["ray_atm"])
        self.out = {"rad": pin(np.zeros((nr, self.nd))), "tau": pin(np.zeros((nr, self.nd))),
                    "tpz": pin(np.zeros(nr)), "tplon": pin(np.zeros(nr)), "tplat": pin(np.zeros(nr)),
                    "nlos": pin(np.zeros(nr, np.int32))}
        bi = L.BatchInput()
        bi.n_atm = n_atm
        bi.n_levels = len(inp["z"])
        bi.n_rays = nr
        bi.atm_off = _iptr(self.host["atm_off"])
        bi.ray_atm = _iptr(self.host["ray_atm"])
        for k in self._KEYS:
            setattr(bi, k, _dptr(self.host[k]))
        bo = L.BatchOutput()
        for k in ("rad", "tau", "tpz", "tplon", "tplat"):
            setattr(bo, k, _dptr(self.out[k]))
        bo.nlos = _iptr(self.out["nlos"])
        self._keep = (bi, bo)
        L.check(lib.jsc_batch_graph_capture(self.batch.h, C.byref(bi), C.byref(bo), stream),
                "jsc_batch_graph_capture")

    def launch(self, inp=None):
        """Copy inp (same shapes) into the staging arrays and replay; the
        caller synchronises the stream before reading self.out."""
        if inp is not None:
            for k in self._KEYS + ("atm_off", "ray_atm"):
                self.host[k][...] = inp[k]
        L.check(L.load().jsc_batch_graph_launch(self.batch.h, self.stream), "jsc_batch_graph_launch")

    def status(self):
        L.check(L.load().jsc_batch_async_status(self.batch.h), "jsc_batch_async_status")

    def close(self):
        self.batch.close()


_F = C.POINTER(C.c_float)


def _fptr(a):
    return a.ctypes.data_as(_F)


# The surrogate's sampled accuracy check, as the benchmark and the tests use
# it: every SURROGATE_CHECK_STRIDE-th point inside the training envelope is
# also computed by the plain path, and an albedo-weighted relative source
# deviation above SURROGATE_CHECK_TOL sends the whole batch down the plain
# path (jsc_batch_set_surrogate).
SURROGATE_CHECK_TOL = 0.01
SURROGATE_CHECK_STRIDE = 256


class Surrogate:
    """Scattering-source surrogate (jsc_surrogate_*): a 4-layer MLP trained
    on the GPU on plain-path samples, BF16 tensor-core inference."""

    NF = 8

    def __init__(self, nd, device=0, seed=1):
        self.nd = nd
        self.h = C.c_void_p()
        L.check(L.load().jsc_surrogate_create(int(nd), int(device), int(seed), C.byref(self.h)),
                "jsc_surrogate_create")

    @property
    def n_params(self):
        return L.load().jsc_surrogate_param_count(self.h)

    def get_params(self):
        out = np.empty(self.n_params, np.float32)
        L.check(L.load().jsc_surrogate_get_params(self.h, _fptr(out)), "jsc_surrogate_get_params")
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        L.check(L.load().jsc_surrogate_set_params(self.h, _fptr(p)), "jsc_surrogate_set_params")

    def layers(self, flat):
        """Split a flat parameter vector into [(W0, b0), ..., (W3, b3)]."""
        shapes = [(128, self.NF), (128, 128), (128, 128), (self.nd, 128)]
        out, o = [], 0
        for r, c in shapes:
            w = flat[o:o + r * c].reshape(r, c)
            o += r * c
            b = flat[o:o + r]
            o += r
            out.append((w, b))
        return out

    def scaling(self):
        """Feature and target standardisation (xm, xs, ym, ys)."""
        xm, xs = np.zeros(self.NF, np.float32), np.zeros(self.NF, np.float32)
        ym, ys = np.zeros(self.nd, np.float32), np.zeros(self.nd, np.float32)
        L.check(L.load().jsc_surrogate_get_scaling(self.h, _fptr(xm), _fptr(xs), _fptr(ym),
                                                   _fptr(ys)), "jsc_surrogate_get_scaling")
        return xm, xs, ym, ys

    def loss_grad(self, x, t):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        loss = C.c_float()
        g = np.empty(self.n_params, np.float32)
        L.check(L.load().jsc_surrogate_loss_grad(self.h, _fptr(x), _fptr(t), len(x),
                                                 C.byref(loss), _fptr(g)),
                "jsc_surrogate_loss_grad")
        return loss.value, g

    def train(self, feat, src, epochs=20, batch=4096, lr=2e-3, seed=7):
        feat = np.ascontiguousarray(feat, dtype=np.float32)
        src = np.ascontiguousarray(src, dtype=np.float64)
        losses = np.zeros(epochs, np.float32)
        L.check(L.load().jsc_surrogate_train(self.h, _fptr(feat), _dptr(src), len(feat), int(epochs),
                                             int(batch), float(lr), int(seed), _fptr(losses)),
                "jsc_surrogate_train")
        return losses

    def set_tensor_path(self, tcgen05):
        """Inference on the tcgen05 path (True) or mma.sync (False)."""
        L.check(L.load().jsc_surrogate_set_tensor_path(self.h, 1 if tcgen05 else 0),
                "jsc_surrogate_set_tensor_path")

    def predict(self, feat):
        feat = np.ascontiguousarray(feat, dtype=np.float32)
        out = np.empty((len(feat), self.nd))
        L.check(L.load().jsc_surrogate_predict(self.h, _fptr(feat), len(feat), _dptr(out)),
                "jsc_surrogate_predict")
        return out

    def close(self):
        if self.h:
            L.load().jsc_surrogate_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def scan_selftest(device=0, n=100_000, budget=0, stall=-1):
    """Status of the device-wait watchdog self-test (jsc_scan_selftest)."""
    return L.load().jsc_scan_selftest(int(device), int(n), int(budget), int(stall))


def launch_count():
    return int(L.load().jsc_launch_count())
