"""The drop-in boundary: struct layouts and exported symbols (CPU only)."""
import ctypes as C
import json
import os
import re
import subprocess
import sys
import tempfile

import pytest

from conftest import GOLDEN, REPO

sys.path.insert(0, GOLDEN)


def _golden_layout():
    with open(os.path.join(GOLDEN, "struct_layout.json")) as f:
        return json.load(f)


def test_header_struct_layout_matches_reference():
    """sizeof/offsetof of every field of include/jurassic_b200.h equal the
    reference's src/jurassic.h (recorded by make_struct_layout.py)."""
    from make_struct_layout import measure
    mine = measure('#include "jurassic_b200.h"', ["-I" + os.path.join(REPO, "include")])
    assert mine == _golden_layout()


def test_ctypes_layout_matches_reference():
    from jscat import structs as S
    ref = _golden_layout()
    classes = {"ctl_t": S.CtlT, "obs_t": S.ObsT, "aero_t": S.AeroT,
               "atm_t": S.AtmT, "queue_t": S.QueueT, "los_t": S.LosT, "tbl_t": S.TblT}
    for cname, cls in classes.items():
        assert C.sizeof(cls) == ref[cname + ".sizeof"], cname
        for f in cls._fields_:
            assert getattr(cls, f[0]).offset == ref["%s.%s" % (cname, f[0])], (cname, f[0])


def _header_functions():
    src = open(os.path.join(REPO, "include", "jurassic_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    src = re.sub(r"^\s*#.*$", "", src, flags=re.M)  # preprocessor lines
    names = re.findall(r"\b(\w+)\s*\([^;{]*\)\s*;", src)
    return sorted(set(n for n in names if n not in ("sizeof",)))


def test_library_exports_every_declared_symbol():
    from jscat import lib as L
    declared = _header_functions()
    assert set(declared) == set(L.EXPORTS), set(declared) ^ set(L.EXPORTS)
    res = subprocess.run(["nm", "-D", "--defined-only", L.LIB_PATH],
                         capture_output=True, text=True, check=True)
    exported = set(ln.split()[-1] for ln in res.stdout.splitlines() if " T " in ln)
    missing = [n for n in declared if n not in exported]
    assert not missing, missing


def test_library_loads_without_gpu():
    from jscat import lib as L
    lib = L.load()
    for n in L.EXPORTS:
        assert hasattr(lib, n)
    assert lib.jsc_status_string(0) == b"ok"


# Values returned by the reference build for the two example invocations
# of docu/modules.tex ("planck 270 960", "brightness 0.0231451 960").
REF_PLANCK_270_960 = 0.06362961283311917
REF_BRIGHTNESS_00231451_960 = 225.57541385238784


def test_known_answers_planck_brightness():
    from jscat import lib as L
    lib = L.load()
    assert lib.planck(270.0, 960.0) == REF_PLANCK_270_960
    assert lib.brightness(0.0231451, 960.0) == REF_BRIGHTNESS_00231451_960
    assert abs(lib.brightness(REF_PLANCK_270_960, 960.0) - 270.0) < 1e-9


def test_drop_in_links_in_place_of_forwardmodel(tmp_path):
    """The reference's own programs formod and kernel (src/formod.c,
    src/kernel.c), compiled from its sources and linked against its objects
    WITHOUT forwardmodel.o plus this library: every symbol they and the
    reference's scatter.o/misc.o need from forwardmodel.o (formod,
    formod_pencil, read_shape, planck, brightness, ...) resolves here.
    Needs the reference tree and the oracle build (make -C oracle ref ret)."""
    sys.path.insert(0, REPO)
    from oracle import refpath
    from jscat import lib as L
    ref = os.path.join(REPO, "oracle", "_ref")
    objs = [os.path.join(ref, "refobj", f + ".o") for f in
            ("atmosphere", "continua", "control", "lineofsight", "misc", "scatter", "workqueue")]
    ret = os.path.join(ref, "retobj")
    if not refpath.available() or not all(os.path.exists(o) for o in objs) or \
            not os.path.isdir(ret):
        pytest.skip("reference tree or oracle objects absent")
    extra = sorted(os.path.join(ret, f) for f in os.listdir(ret) if f.endswith(".o"))
    for prog in ("formod", "kernel"):
        exe = str(tmp_path / prog)
        res = subprocess.run(
            ["gcc", "-O2", "-fopenmp", "-DWORK_QUEUE", "-DHAVE_INLINE", "-w",
             "-I" + os.path.join(ref, "include"), "-o", exe,
             refpath.reference_path("src", prog + ".c")] + objs + extra +
            [os.path.join(ref, "libgslsubset.a"), L.LIB_PATH,
             "-Wl,-rpath," + os.path.dirname(L.LIB_PATH), "-lm"],
            capture_output=True, text=True)
        assert res.returncode == 0, res.stderr[-2000:]
        # the program's formod is the library's
        nm = subprocess.run(["nm", exe], capture_output=True, text=True, check=True).stdout
        assert re.search(r"\bU formod\b", nm) and re.search(r"\bU formod_pencil\b", nm)
        ldd = subprocess.run(["ldd", exe], capture_output=True, text=True, check=True).stdout
        assert "libjurassic_b200.so" in ldd
