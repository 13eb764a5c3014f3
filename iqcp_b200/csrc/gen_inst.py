"""Write the explicit-instantiation translation units of the quartet kernels.

One unit per (kernel kind, quadrature type, bra class, ket class), so that
`make -j` spreads the template-heavy compile over the host cores, plus one
dispatch unit per (kind, bra class) that declares those instantiations extern.
Run from this directory; the Makefile picks the files up by wildcard.
"""
import glob
import os

CLS = [(0, 0), (1, 0), (1, 1), (2, 0), (2, 1), (2, 2)]
NAME = ["ss", "ps", "pp", "ds", "dp", "dd"]
ARGS = {"jk": "JKArgs", "grad": "GradArgs"}
HEAD = "// Generated by gen_inst.py: {what}\n#include \"eri_launch.cuh\"\n\nnamespace iqcp {{\n"
TAIL = "}  // namespace iqcp\n"


def variant(kind, r, bra, ket):
    return "cudaError_t launch_{k}_variant<{r}, {a}, {b}, {c}, {d}>(const {A}&, cudaStream_t)".format(
        k=kind, r=r, a=bra[0], b=bra[1], c=ket[0], d=ket[1], A=ARGS[kind])


def main():
    for f in glob.glob("eri_inst_*.cu"):
        os.remove(f)
    for x, bra in enumerate(CLS):
        kets = CLS[: x + 1]
        for kind in ("jk", "grad"):
            body = "".join("extern template %s;\n" % variant(kind, r, bra, ket)
                           for r in ("double", "float") for ket in kets)
            body += "template cudaError_t launch_{k}_bra<{a}, {b}>(int, const {A}&, cudaStream_t);\n".format(
                k=kind, a=bra[0], b=bra[1], A=ARGS[kind])
            with open("eri_inst_%s_%s.cu" % (kind, NAME[x]), "w") as fh:
                fh.write(HEAD.format(what="%s dispatch for bra class (%s|" % (kind, NAME[x])) + body + TAIL)
            for y, ket in enumerate(kets):
                for r, tag in (("double", "f64"), ("float", "f32")):
                    with open("eri_inst_%s_%s_%s%s.cu" % (kind, tag, NAME[x], NAME[y]), "w") as fh:
                        fh.write(HEAD.format(what="%s %s kernels for (%s|%s)" % (kind, tag, NAME[x], NAME[y])) +
                                 "template %s;\n" % variant(kind, r, bra, ket) + TAIL)
        with open("eri_inst_store_%s.cu" % NAME[x], "w") as fh:
            fh.write(HEAD.format(what="store kernels for bra class (%s|" % NAME[x]) +
                     "template cudaError_t launch_store_bra<%d, %d>(int, const StoreArgs&, cudaStream_t);\n" % bra +
                     TAIL)


if __name__ == "__main__":
    main()
