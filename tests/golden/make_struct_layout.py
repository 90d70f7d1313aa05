"""Record sizeof/offsetof of every field of the reference's boundary structs
(src/jurassic.h, compiled here with gcc) into struct_layout.json.

    python tests/golden/make_struct_layout.py   (needs the reference tree and
                                                 oracle/_ref/include from
                                                 'make -C oracle ref')
"""
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "jurassic-scatter_b200"))

from jscat import structs as S  # noqa: E402

STRUCTS = {"ctl_t": S.CtlT, "obs_t": S.ObsT, "aero_t": S.AeroT, "atm_t": S.AtmT,
           "queue_t": S.QueueT, "los_t": S.LosT, "tbl_t": S.TblT}


def layout_program(header_include):
    lines = ["#include <stdio.h>", "#include <stddef.h>", header_include,
             "int main(void) {", 'printf("{");']
    first = True
    for cname, cls in STRUCTS.items():
        sep = "" if first else ","
        first = False
        lines.append('printf("%s\\"%s.sizeof\\": %%zu", sizeof(%s));' % (sep, cname, cname))
        for f in cls._fields_:
            lines.append('printf(",\\"%s.%s\\": %%zu", offsetof(%s, %s));' % (cname, f[0], cname, f[0]))
    lines += ['printf("}\\n");', "return 0; }"]
    return "\n".join(lines)


def measure(include_line, cflags):
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "l.c"), os.path.join(d, "l")
        open(src, "w").write(layout_program(include_line))
        subprocess.run(["gcc"] + cflags + [src, "-o", exe], check=True)
        return json.loads(subprocess.run([exe], capture_output=True, text=True,
                                         check=True).stdout)


if __name__ == "__main__":
    sys.path.insert(0, REPO)
    from oracle import refpath
    ref = measure('#include "jurassic.h"', ["-I" + refpath.reference_path("src"),
                                           "-I" + os.path.join(REPO, "oracle", "_ref", "include")])
    with open(os.path.join(HERE, "struct_layout.json"), "w") as f:
        json.dump(ref, f, indent=0, sort_keys=True)
    print(len(ref), "entries")
