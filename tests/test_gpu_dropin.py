"""The drop-in link on the GPU: the reference's own programs formod and
kernel (src/formod.c, src/kernel.c), linked against the reference's
objects without forwardmodel.o plus this library (oracle/Makefile target
`dropin`), run the reference's example cases (examples/clear.sh,
extinction1.sh, aerosol0.sh, inputs made by the reference's climatology,
limb and nadir programs) and must reproduce the reference's outputs
(examples/org) at the precision the files are written with (%g, six
significant digits).  The clear-air Jacobian of the kernel program is
compared with the reference's own kernel program on the same inputs.
Everything the test reads is staged under oracle/_ref/dropin."""
import os
import subprocess

import numpy as np
import pytest

from conftest import REPO

pytestmark = pytest.mark.gpu

DROP = os.path.join(REPO, "oracle", "_ref", "dropin")
EX = os.path.join(DROP, "examples")

# (ctl, observation file, atmosphere, output, expected, extra arguments)
CASES = {
    "clear": ("clear-air.ctl", "obs_clear.tab", "atm_clear.tab", "rad_clear.tab", []),
    "extinction1": ("extinction1.ctl", "obs_ext1.tab", "atm_ext1.tab", "rad_ext1.tab",
                    ["AEROFILE", "aero0.tab"]),
    "aerosol0": ("aerosol0.ctl", "obs_aero0.tab", "atm_aero0.tab", "rad_aero0.tab",
                 ["AEROFILE", "aero0.tab"]),
}


def _staged():
    return os.path.exists(os.path.join(EX, ".staged")) and \
        os.path.exists(os.path.join(DROP, "bin", "formod"))


def _numbers(path):
    rows = []
    for ln in open(path):
        ln = ln.strip()
        if ln and not ln.startswith("#"):
            rows.append(ln.split())
    return rows


def _close_at_print_precision(got, want):
    """Equal as six-significant-digit numbers: within one unit of the last
    printed digit."""
    a, b = float(got), float(want)
    return a == b or abs(a - b) <= 1e-5 * max(abs(a), abs(b))


@pytest.mark.parametrize("case", sorted(CASES))
def test_reference_formod_program_on_examples(case, tmp_path):
    if not _staged():
        pytest.skip("drop-in programs and examples not staged (make -C oracle dropin)")
    ctl, obs, atm, out, extra = CASES[case]
    dst = str(tmp_path / out)
    res = subprocess.run([os.path.join(DROP, "bin", "formod"), ctl, obs, atm, dst] + extra,
                         cwd=EX, capture_output=True, text=True, timeout=600,
                         env=dict(os.environ, JURASSIC_GPU_DEVICE="0"))
    assert res.returncode == 0, (res.stdout[-2000:], res.stderr[-2000:])
    got, want = _numbers(dst), _numbers(os.path.join(EX, "org", out))
    assert len(got) == len(want) and all(len(g) == len(w) for g, w in zip(got, want))
    bad = [(i, j, g, w) for i, (gr, wr) in enumerate(zip(got, want))
           for j, (g, w) in enumerate(zip(gr, wr)) if not _close_at_print_precision(g, w)]
    assert not bad, bad[:10]


def test_reference_kernel_program_clear_air(tmp_path):
    """The kernel program (the reference's kernel(): n + 1 formod calls, each
    on the GPU) against the reference's own kernel program."""
    if not _staged():
        pytest.skip("drop-in programs and examples not staged (make -C oracle dropin)")
    ret = open(os.path.join(EX, "kernel_ret.txt")).read().split()
    dst = str(tmp_path / "kernel.tab")
    res = subprocess.run([os.path.join(DROP, "bin", "kernel"), "clear-air.ctl", "obs_clear.tab",
                          "atm_clear.tab", "-", dst] + ret, cwd=EX, capture_output=True,
                         text=True, timeout=600, env=dict(os.environ, JURASSIC_GPU_DEVICE="0"))
    assert res.returncode == 0, (res.stdout[-2000:], res.stderr[-2000:])
    got, want = _numbers(dst), _numbers(os.path.join(EX, "org", "kernel_clear.tab"))
    assert len(got) == len(want) > 0
    assert [r[:-1] for r in got] == [r[:-1] for r in want]   # same rows and columns
    g = np.array([float(r[-1]) for r in got])
    w = np.array([float(r[-1]) for r in want])
    # finite differences of radiances that agree to ~1e-9, printed with
    # six digits: within two units of the last digit or 1e-6 of the largest
    # entry
    tol = 2e-5 * np.abs(w) + 1e-6 * np.max(np.abs(w))
    assert np.all(np.abs(g - w) <= tol), float(np.max(np.abs(g - w) / np.maximum(tol, 1e-300)))
