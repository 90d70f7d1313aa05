"""Generate ckd_tables.h: the continuum coefficient tables of the CKD-type
CO2/H2O self/foreign continua and the N2/O2 collision-induced bands.

These are measured physical coefficient tables.  Parity with the reference
requires the same numbers, so they are extracted from the reference's
src/continua.c (ctmco2 :11/:285/:561, ctmh2o :883/:1216/:1549/:1883,
ctmn2 :1939-1975, ctmo2 :2001-2032) and written as C arrays under this
library's own names.  Run once where the reference tree is available:

    python gen_ckd_tables.py /path/to/reference/src/continua.c > ckd_tables.h
"""
import re
import sys


def function_bodies(src):
    """Map function name -> source text of its body (top-level functions)."""
    out = {}
    for m in re.finditer(r"\n(double|int|void)\s+(\w+)\s*\(", src):
        name = m.group(2)
        start = src.index("{", m.end())
        depth, i = 0, start
        while True:
            if src[i] == "{":
                depth += 1
            elif src[i] == "}":
                depth -= 1
                if depth == 0:
                    break
            i += 1
        out[name] = src[start:i + 1]
    return out


def arrays(body):
    """Static double arrays declared in a function body: name -> list of str."""
    res = {}
    pat = re.compile(r"static\s+double\s+(\w+)\[(\d+)\]\s*=\s*\{(.*?)\};", re.S)
    for m in pat.finditer(body):
        vals = [v.strip() for v in m.group(3).replace("\n", " ").split(",")]
        vals = [v for v in vals if v]
        assert len(vals) == int(m.group(2)), (m.group(1), len(vals))
        res[m.group(1)] = [repr(float(v)) for v in vals]
    return res


def emit(name, vals, out):
    out.append("static const double %s[%d] = {" % (name, len(vals)))
    for i in range(0, len(vals), 6):
        out.append("  " + ", ".join(vals[i:i + 6]) + ",")
    out.append("};")


def main(path):
    src = open(path).read()
    bodies = function_bodies(src)
    co2 = arrays(bodies["ctmco2"])
    h2o = arrays(bodies["ctmh2o"])
    n2 = arrays(bodies["ctmn2"])
    o2 = arrays(bodies["ctmo2"])
    out = ["/* Generated by gen_ckd_tables.py from the reference's continuum",
           " * coefficient tables; do not edit.  Values as printed there. */",
           "#ifndef JSC_CKD_TABLES_H", "#define JSC_CKD_TABLES_H", ""]
    out.append("/* CO2 continuum at 296/260/230 K, 2 cm^-1 grid from 0 cm^-1. */")
    emit("jsc_ckd_co2_t296", co2["co2296"], out)
    emit("jsc_ckd_co2_t260", co2["co2260"], out)
    emit("jsc_ckd_co2_t230", co2["co2230"], out)
    out.append("/* H2O self continuum at 296/260 K and foreign continuum, 10 cm^-1 grid. */")
    emit("jsc_ckd_h2o_t296", h2o["h2o296"], out)
    emit("jsc_ckd_h2o_t260", h2o["h2o260"], out)
    emit("jsc_ckd_h2o_frn", h2o["h2ofrn"], out)
    out.append("/* H2O self-continuum correction, 820-960 cm^-1 in 10 cm^-1 steps. */")
    emit("jsc_ckd_h2o_xfc", h2o["xfcrev"], out)
    out.append("/* N2 collision-induced band: strength, T exponent, wavenumber grid. */")
    emit("jsc_n2_b", n2["ba"], out)
    emit("jsc_n2_beta", n2["betaa"], out)
    emit("jsc_n2_nu", n2["nua"], out)
    out.append("/* O2 collision-induced band: strength, T exponent, wavenumber grid. */")
    emit("jsc_o2_b", o2["ba"], out)
    emit("jsc_o2_beta", o2["betaa"], out)
    emit("jsc_o2_nu", o2["nua"], out)
    out += ["", "#endif", ""]
    sys.stdout.write("\n".join(out))


if __name__ == "__main__":
    main(sys.argv[1])
