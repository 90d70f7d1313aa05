"""Generate the golden fixtures of tests/golden/ by running the reference
forward model (oracle/_ref/libjurassic_ref.so, compiled from the
reference's own sources by oracle/Makefile) on the seeded synthetic
workloads of jscat.synth.

    make -C oracle ref && python tests/golden/make_golden.py

Each fixture stores the reference's outputs in full FP64 precision plus a
checksum of the generated table files, so a test can tell a changed input
from a changed result.
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


def save(name, ctlkw, atms, ray_atm, geom, ref):
    np.savez_compressed(
        os.path.join(HERE, name + ".npz"),
        rad=ref["rad"], tau=ref["tau"], tpz=ref["tpz"], tplon=ref["tplon"],
        tplat=ref["tplat"], nlos=ref["nlos"],
        table_sha256=tables_digest(ctlkw["tblbase"], ctlkw["emitters"], ctlkw["nus"]),
        ray_atm=np.asarray(ray_atm), **{"geom_" + k: v for k, v in geom.items()})


def main():
    workdir = os.environ.get("JSC_WORKDIR", "/tmp/jsc")
    ctlkw, atm, geom = synth.clear_limb_case(workdir)
    ref = refrun.run(ctlkw, [atm], np.zeros(len(geom["obsz"]), int), geom, los=True)
    save("clear_limb", ctlkw, [atm], np.zeros(len(geom["obsz"]), int), geom, ref)
    ctlkw, atms, ray_atm, geom = mixed_case(workdir)
    ref = refrun.run(ctlkw, atms, ray_atm, geom, los=True)
    save("mixed_batch", ctlkw, atms, ray_atm, geom, ref)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
