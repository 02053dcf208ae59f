"""Generate gauss9_gen.cuh: straight-line no-pivot elimination of the 9x9 canopy system.

The structural nonzero pattern of the turvap matrix (canopy_exchange.py:620-682)
is filled in symbolically for elimination in row order; only updates of
entries that can be nonzero are emitted, and the result equals the dense
elimination bit for bit in IEEE arithmetic (an update that multiplies a
structural zero leaves its target unchanged).  Run: python gen_gauss9.py
"""
import os

PATTERN = {0: [0, 3, 5], 1: [1, 3, 5], 2: [2, 4, 6], 3: [0, 1, 3, 4], 4: [2, 3, 4, 7, 8],
           5: [0, 1, 5, 6], 6: [2, 5, 6, 7, 8], 7: [4, 6, 7], 8: [4, 6, 8]}


def fill():
    nz = {(i, j) for i, js in PATTERN.items() for j in js}
    ops = []
    for p in range(8):
        for i in range(p + 1, 9):
            if (i, p) not in nz:
                continue
            cols = [j for j in range(p + 1, 9) if (p, j) in nz]
            for j in cols:
                nz.add((i, j))
            ops.append((p, i, cols))
    return nz, ops


def main():
    nz, ops = fill()
    out = ["// Generated by gen_gauss9.py -- do not edit.",
           "// No-pivot Gaussian elimination of the 9x9 canopy system on its filled",
           "// nonzero pattern (%d entries), then back substitution." % len(nz),
           "#pragma once", "", "namespace ibis {", "",
           "struct Sys9 {"]
    out.append("    double " + ", ".join(f"a{i}{j}" for i, j in sorted(nz)) + ";")
    out.append("    double " + ", ".join(f"b{i}" for i in range(9)) + ";")
    out.append("};")
    out.append("")
    out.append("__device__ __forceinline__ void sys9_zero(Sys9& s) {")
    out.append("    " + " ".join(f"s.a{i}{j} = 0.0;" for i, j in sorted(nz)))
    out.append("}")
    out.append("")
    out.append("// Each pivot's reciprocal is formed once and reused by the rows below it and by")
    out.append("// the back substitution (one division per unknown instead of one per update).")
    out.append("__device__ __forceinline__ void sys9_solve(Sys9& s, double (&x)[9]) {")
    out.append("    double f;")
    out.append("    double r0, r1, r2, r3, r4, r5, r6, r7, r8;")
    done = set()
    for p, i, cols in ops:
        if p not in done:
            out.append(f"    r{p} = rcp(s.a{p}{p});")
            done.add(p)
        out.append(f"    f = s.a{i}{p} * r{p};")
        for j in cols:
            out.append(f"    s.a{i}{j} = s.a{i}{j} - f * s.a{p}{j};")
        out.append(f"    s.b{i} = s.b{i} - f * s.b{p};")
    for i in range(8, -1, -1):
        terms = [j for j in range(i + 1, 9) if (i, j) in nz]
        expr = None
        for j in terms:
            expr = f"s.a{i}{j} * x[{j}]" if expr is None else f"({expr} + s.a{i}{j} * x[{j}])"
        if i not in done:
            out.append(f"    r{i} = rcp(s.a{i}{i});")
            done.add(i)
        if expr is None:
            out.append(f"    x[{i}] = s.b{i} * r{i};")
        else:
            out.append(f"    x[{i}] = (s.b{i} - {expr}) * r{i};")
    out.append("}")
    out.append("")
    out.append("}  // namespace ibis")
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "gauss9_gen.cuh")
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


if __name__ == "__main__":
    main()
