"""Generate the CUDA lattice headers from ``tensorlbm_b200.lattice``.

Run ``python -m tensorlbm_b200.csrc.gen_tables`` after changing a velocity set
or a moment basis; the build calls it too, so the headers under
``csrc/generated/`` always match the Python tables.

Two headers come out:

* ``lattice_tables.cuh`` - one struct per lattice with Q, the velocity
  components, opposite directions and weights as compile-time constants.
* ``mrt_tables.cuh`` - the MRT collision written out as straight-line code:
  the non-equilibrium moments ``d_k = sum_j M[k][j] * fneq_j`` of every
  relaxed row and the back-projection ``f_i -= sum_k Minv[i][k] * s_k * d_k``.
  Terms are grouped by coefficient so each multiply happens once per distinct
  value; rows with a zero relaxation rate (mass, momentum) are skipped.
"""

from __future__ import annotations

import pathlib
from collections import defaultdict

import numpy as np

from tensorlbm_b200 import lattice as lat

OUT = pathlib.Path(__file__).resolve().parent / "generated"


def _lit(v: float) -> str:
    """C double literal that round-trips exactly."""
    r = repr(float(v))
    if "e" not in r and "." not in r and "inf" not in r and "nan" not in r:
        r += ".0"
    return r


def gen_lattice_tables() -> str:
    lines = [
        "// Generated by tensorlbm_b200/csrc/gen_tables.py - do not edit.",
        "#pragma once",
        "",
    ]
    for L in (lat.D2Q9, lat.D3Q19, lat.D3Q27):
        cx = ", ".join(str(int(v)) for v in L.c[:, 0])
        cy = ", ".join(str(int(v)) for v in L.c[:, 1])
        cz = ", ".join(str(int(v)) for v in L.c[:, 2])
        opp = ", ".join(str(int(v)) for v in L.opp)
        w = ", ".join(_lit(float(v)) for v in L.w)
        lines += [
            f"struct {L.name} {{",
            f"  static constexpr int Q = {L.q};",
            f"  static constexpr int DIM = {L.dim};",
            f"  __host__ __device__ static constexpr int cx(int q) {{ constexpr int t[{L.q}] = {{{cx}}}; return t[q]; }}",
            f"  __host__ __device__ static constexpr int cy(int q) {{ constexpr int t[{L.q}] = {{{cy}}}; return t[q]; }}",
            f"  __host__ __device__ static constexpr int cz(int q) {{ constexpr int t[{L.q}] = {{{cz}}}; return t[q]; }}",
            f"  __host__ __device__ static constexpr int opp(int q) {{ constexpr int t[{L.q}] = {{{opp}}}; return t[q]; }}",
            f"  __host__ __device__ static constexpr double w(int q) {{ constexpr double t[{L.q}] = {{{w}}}; return t[q]; }}",
            "};",
            "",
        ]
    return "\n".join(lines)


# relaxation-rate symbol per MRT row (None = conserved, skipped)
_RATES = {
    9: [None, "s_e", "s_eps", None, "s_q", None, "s_q", "s_nu", "s_nu"],
    19: [None, "s_e", "s_eps", None, "s_q", None, "s_q", None, "s_q",
         "s_nu", "s_nu", "s_nu", "s_nu", "s_nu", "s_pi", "s_pi", "one", "one", "one"],
    27: [None, None, None, None, "s_e", "s_nu", "s_nu", "s_nu", "s_nu", "s_nu"]
    + ["s_q"] * 9 + ["s_eps"] + ["s_pi"] * 7,
}


def _grouped_sum(terms: list[tuple[float, str]]) -> str:
    """sum c_j * x_j with equal coefficients factored: c*(x_a + x_b + ...)."""
    groups: dict[float, list[str]] = defaultdict(list)
    for c, x in terms:
        if c != 0.0:
            groups[c].append(x)
    parts = []
    for c in sorted(groups, key=lambda v: (abs(v), v)):
        xs = groups[c]
        s = xs[0] if len(xs) == 1 else "(" + " + ".join(xs) + ")"
        if c == 1.0:
            parts.append(s)
        elif c == -1.0:
            parts.append(f"-{s}")
        else:
            parts.append(f"T({_lit(c)}) * {s}")
    if not parts:
        return "T(0)"
    expr = parts[0]
    for p in parts[1:]:
        expr += f" - {p[1:]}" if p.startswith("-") else f" + {p}"
    return expr


def _clean(v: float) -> float:
    # entries below 1e-10 are round-off of the float64 Gram-Schmidt / inverse
    # (the exact matrices have a zero there); dropping them changes results far
    # below float32 resolution and saves an FMA each
    return 0.0 if abs(v) <= 1e-10 else float(v)


def gen_mrt(q: int) -> str:
    """Straight-line MRT relaxation using opposite-direction pairs.

    Every basis row is even (M[k][opp q] = M[k][q]) or odd (= -M[k][q]), so an
    even moment only sees s = fn[q] + fn[opp q] and an odd one only
    a = fn[q] - fn[opp q]; the back-projection splits the same way into an even
    part E and an odd part O with f[q] -= E + O and f[opp q] -= E - O.  This is
    the same operator with half the multiply-adds of the dense form."""
    L = lat.LATTICES[q]
    m, minv = lat.mrt_matrices(q)
    rates = _RATES[q]
    name = {9: "d2q9", 19: "d3q19", 27: "d3q27"}[q]
    opp = [int(v) for v in L.opp]
    pairs = [(i, opp[i]) for i in range(1, q) if i < opp[i]]
    rest = [i for i in range(q) if opp[i] == i]
    # rows TensorLBM's D3Q27 Gram-Schmidt replaced by unit vectors (dependent
    # monomials, d3q27.py:614-625) have no parity and stay dense
    parity = {}
    for k in range(q):
        ev = all(abs(m[k, i] - m[k, opp[i]]) < 1e-9 for i in range(q))
        od = all(abs(m[k, i] + m[k, opp[i]]) < 1e-9 for i in range(q))
        parity[k] = "even" if ev else ("odd" if od else "none")
        if parity[k] != "none":
            sgn = 1.0 if ev else -1.0
            for i in range(q):  # the inverse inherits the parity
                assert abs(minv[opp[i], k] - sgn * minv[i, k]) < 1e-9, (q, k, i)
    out = [
        f"// MRT relaxation for {name}: f_i -= sum_k Minv[i][k] * s_k * (M (f - feq))_k, paired form",
        "template <typename T>",
        f"__device__ __forceinline__ void mrt_relax_{name}(T (&f)[{q}], const T (&fn)[{q}], const MrtRates<T>& r) {{",
        "  const T one = T(1);",
    ]
    for a, b in pairs:
        out.append(f"  const T s{a} = fn[{a}] + fn[{b}], a{a} = fn[{a}] - fn[{b}];")
    relaxed = [k for k in range(q) if rates[k] is not None]
    for k in relaxed:
        if parity[k] == "even":
            terms = [(_clean(m[k, i]), f"fn[{i}]") for i in rest] + [(_clean(m[k, a]), f"s{a}") for a, _ in pairs]
        elif parity[k] == "odd":
            terms = [(_clean(m[k, a]), f"a{a}") for a, _ in pairs]
        else:
            terms = [(_clean(m[k, i]), f"fn[{i}]") for i in range(q)]
        rate = "one" if rates[k] == "one" else f"r.{rates[k]}"
        out.append(f"  const T e{k} = {rate} * ({_grouped_sum(terms)});")
    even = [k for k in relaxed if parity[k] == "even"]
    odd = [k for k in relaxed if parity[k] == "odd"]
    dense = [k for k in relaxed if parity[k] == "none"]

    def nsum(i):
        return _grouped_sum([(_clean(minv[i, k]), f"e{k}") for k in dense]) if dense else "T(0)"

    for i in rest:
        terms = [(_clean(minv[i, k]), f"e{k}") for k in even + dense]
        out.append(f"  f[{i}] -= {_grouped_sum(terms)};")
    for a, b in pairs:
        ev = _grouped_sum([(_clean(minv[a, k]), f"e{k}") for k in even])
        od = _grouped_sum([(_clean(minv[a, k]), f"e{k}") for k in odd])
        if dense:
            out.append(f"  {{ const T E = {ev}; const T O = {od}; f[{a}] -= E + O + ({nsum(a)}); "
                       f"f[{b}] -= E - O + ({nsum(b)}); }}")
        else:
            out.append(f"  {{ const T E = {ev}; const T O = {od}; f[{a}] -= E + O; f[{b}] -= E - O; }}")
    out.append("}")
    out.append("")
    return "\n".join(out)


def gen_mrt_header() -> str:
    parts = [
        "// Generated by tensorlbm_b200/csrc/gen_tables.py - do not edit.",
        "#pragma once",
        "",
        "template <typename T> struct MrtRates {",
        "  T s_e, s_eps, s_q, s_nu, s_pi;",
        "};",
        "",
    ]
    for q in (9, 19, 27):
        parts.append(gen_mrt(q))
    return "\n".join(parts)


# cascaded central-moment collision (cascaded_collision.py:59-187): the D3Q19
# monomial basis, its raw-moment matrix and inverse (float64, as the reference
# builds them with numpy) and the 1-D shift groups
CASCADED_D3Q19_DEGREES = [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (2, 0, 0), (0, 2, 0), (0, 0, 2), (1, 1, 0),
                          (1, 0, 1), (0, 1, 1), (2, 1, 0), (2, 0, 1), (1, 2, 0), (0, 2, 1), (1, 0, 2), (0, 1, 2),
                          (2, 2, 0), (2, 0, 2), (0, 2, 2)]


def _shift_groups(degrees):
    """Per axis, the (degree 0, 1, 2) index triples of moments that agree in
    the other two degrees; incomplete triples are not shifted."""
    out = []
    for dim in range(3):
        other = [d for d in range(3) if d != dim]
        bucket = {}
        for idx, deg in enumerate(degrees):
            bucket.setdefault((deg[other[0]], deg[other[1]]), {})[deg[dim]] = idx
        out.append([(m[0], m[1], m[2]) for key, m in sorted(bucket.items()) if all(k in m for k in (0, 1, 2))])
    return out


def gen_cascaded_header() -> str:
    import numpy as np

    c = np.array(lat.LATTICES[19].c, dtype=np.float64)
    deg = CASCADED_D3Q19_DEGREES
    m = np.array([c[:, 0] ** a * c[:, 1] ** b * c[:, 2] ** d for a, b, d in deg])
    minv = np.linalg.inv(m)
    groups = _shift_groups(deg)
    lines = ["// Generated by tensorlbm_b200/csrc/gen_tables.py - do not edit.",
             "#pragma once",
             "",
             "// D3Q19 cascaded central-moment basis (TensorLBM cascaded_collision.py:59-79 order)",
             "struct CascadedD3Q19 {"]
    rows = ", ".join("{" + ", ".join(str(int(v)) for v in r) + "}" for r in m)
    lines.append(f"  __host__ __device__ static constexpr int M(int i, int q) {{ constexpr int t[19][19] = {{{rows}}}; "
                 "return t[i][q]; }")
    rows = ", ".join("{" + ", ".join(_lit(v) for v in r) + "}" for r in minv)
    lines.append(f"  __host__ __device__ static constexpr double Minv(int q, int i) {{ constexpr double t[19][19] = "
                 f"{{{rows}}}; return t[q][i]; }}")
    for axis, g in zip("xyz", groups):
        body = ", ".join("{" + ", ".join(str(v) for v in t) + "}" for t in g)
        lines.append(f"  static constexpr int kGroups{axis.upper()} = {len(g)};")
        lines.append(f"  __host__ __device__ static constexpr int group_{axis}(int k, int j) {{ constexpr int t[{len(g)}][3] "
                     f"= {{{body}}}; return t[k][j]; }}")
    lines += ["};", ""]
    return "\n".join(lines)


def main() -> None:
    OUT.mkdir(parents=True, exist_ok=True)
    for name, text in (("lattice_tables.cuh", gen_lattice_tables()), ("mrt_tables.cuh", gen_mrt_header()),
                       ("cascaded_tables.cuh", gen_cascaded_header())):
        path = OUT / name
        if not path.exists() or path.read_text() != text:
            path.write_text(text)


if __name__ == "__main__":
    main()
