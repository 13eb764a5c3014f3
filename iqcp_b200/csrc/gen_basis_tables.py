"""Generate ``basis_tables.inc`` from the reference's built-in basis-set tables.

The reference ships its Gaussian basis sets (STO-3G, 3-21G, 6-31G, 6-31G*,
6-31+G*, cc-pVDZ for H..Ar) as Rust literals in
``crates/qc-core/src/basis/builtin.rs``.  Basis-set exponents and contraction
coefficients are published data that must be reproduced bit-exactly for
results parity, so they are extracted mechanically instead of being retyped:
every ``fn NAME() -> Vec<ShellData>`` body is tokenised into shells
(``AngularMomentum::S|P|D`` followed by ``(exponent, coefficient)`` tuples), the
per-basis dispatch (``get_sto3g`` .. ``get_ccpvdz``, builtin.rs:155-3983) is
resolved by element, and 6-31G* for Li..Ne is assembled the way
``get_631gs`` (builtin.rs:1032-1063) assembles it: the 6-31G shells plus one
uncontracted d shell.  Numbers are emitted with their original decimal text so
the C++ compiler rounds them exactly as rustc does.

Usage: python gen_basis_tables.py <path to builtin.rs> <output .inc>
"""
import re
import sys

ELEMENTS = ["h", "he", "li", "be", "b", "c", "n", "o", "f", "ne",
            "na", "mg", "al", "si", "p", "s", "cl", "ar"]
# basis id, canonical name, function-name prefix
BASES = [
    (0, "sto-3g", "sto3g_"),
    (1, "3-21g", "b321g_"),
    (2, "6-31g", "b631g_"),
    (3, "6-31g*", None),          # assembled, see get_631gs
    (4, "6-31+g*", "b631pgs_"),
    (5, "cc-pvdz", "ccpvdz_"),
]
L_OF = {"S": 0, "P": 1, "D": 2}
NUM = r"[-+]?\d+\.?\d*(?:[eE][-+]?\d+)?"


def parse_functions(src):
    funcs = {}
    for m in re.finditer(r"fn (\w+)\(\) -> Vec<ShellData> \{", src):
        name = m.group(1)
        depth, i = 1, m.end()
        while depth:
            c = src[i]
            depth += (c == "{") - (c == "}")
            i += 1
        body = re.sub(r"//[^\n]*", "", src[m.end():i - 1])
        shells = []
        tok = re.compile(r"AngularMomentum::([SPD])|\(\s*(%s)\s*,\s*(%s)\s*\)" % (NUM, NUM))
        for t in tok.finditer(body):
            if t.group(1):
                shells.append([L_OF[t.group(1)], []])
            else:
                shells[-1][1].append((t.group(2), t.group(3)))
        funcs[name] = shells
    return funcs


def d_exponents_631gs(src):
    m = re.search(r"fn get_631gs\(z: u8\).*?let d_exp = match z \{(.*?)\};", src, re.S)
    out = {}
    for z, e in re.findall(r"(\d+)\s*=>\s*(%s)" % NUM, m.group(1)):
        out[int(z)] = e
    return out


def main():
    src_path, out_path = sys.argv[1], sys.argv[2]
    src = open(src_path).read()
    funcs = parse_functions(src)
    dexp = d_exponents_631gs(src)
    records, prims = [], []
    for bid, bname, prefix in BASES:
        for z, sym in enumerate(ELEMENTS, start=1):
            if prefix is not None:
                shells = funcs[prefix + sym]
            elif z <= 2:
                shells = funcs["b631g_" + sym]
            elif z <= 10:
                shells = funcs["b631g_" + sym] + [[2, [(dexp[z], "1.0000000")]]]
            else:
                shells = funcs["b631gs_" + sym]
            for L, pl in shells:
                records.append((bid, z, L, len(pl), len(prims)))
                prims.extend(pl)
    with open(out_path, "w") as f:
        f.write("// Generated by gen_basis_tables.py from the reference's built-in basis tables\n")
        f.write("// (crates/qc-core/src/basis/builtin.rs). Do not edit by hand.\n")
        f.write("static const char* const kBasisNames[%d] = {%s};\n" % (
            len(BASES), ", ".join('"%s"' % b[1] for b in BASES)))
        f.write("static const int kNumShellRecords = %d;\n" % len(records))
        f.write("// {basis id, Z, L, nprim, first primitive}\n")
        f.write("static const int kShellRecords[%d][5] = {\n" % len(records))
        for r in records:
            f.write("  {%d, %d, %d, %d, %d},\n" % r)
        f.write("};\n")
        f.write("// {exponent, contraction coefficient}, raw (unnormalised) as tabulated\n")
        f.write("static const double kPrimitives[%d][2] = {\n" % len(prims))
        for e, c in prims:
            f.write("  {%s, %s},\n" % (e, c))
        f.write("};\n")
    print("wrote %d shell records, %d primitives" % (len(records), len(prims)))


if __name__ == "__main__":
    main()
