"""Extract the reference's known-answer vectors for the force hot path into reference_kats.json.

ParticleDynamics.jl (Julia + CUDA.jl) cannot run here, so its golden values are
taken from the text of its own test files:

* test/test_force_precision_gpu.jl:7-20 -- two-atom LJ (eps = sigma = 1, rc = 2.5,
  box 10): separations 1 and 2, forces, per-atom energies, summed virial.
* test/test_force_precision_gpu.jl:23-25 -- the ten near-face particle positions
  (L = 149.38015821857212) of the periodic force-precision test.
* test/test_neighbor_reference.jl:1-6 -- neighbor-row known answers.
* test/test_electrostatics.jl:299-309 -- the solver cases (box, C, r_c, alpha,
  mesh, order) and their force / energy tolerances against the Ewald oracle.

Run with REFERENCE_ROOT set to a checkout of the reference (ParticleDynamics.jl v0.7.0):
``REFERENCE_ROOT=<checkout> python tests/golden/make_fixtures.py``.
"""
from __future__ import annotations

import json
import os
import re
from pathlib import Path

HERE = Path(__file__).resolve().parent
if "REFERENCE_ROOT" not in os.environ:
    raise SystemExit("set REFERENCE_ROOT to a checkout of ParticleDynamics.jl v0.7.0")
REF = Path(os.environ["REFERENCE_ROOT"])


def _lines(rel: str) -> list[str]:
    return (REF / rel).read_text().splitlines()


def two_atom_lj() -> list[dict]:
    src = "\n".join(_lines("test/test_force_precision_gpu.jl")[6:20])
    out = []
    for sep, fblock, eblock, wblock in re.findall(
            r"CuArray\(T\[0,(\d+)\]\).*?Array\(r\.F\) == \[([^\]]*)\].*?Array\(r\.energy\) == \[([^\]]*)\]"
            r".*?dims=2\)\)\[:\] == \[([^\]]*)\]", src, re.S):
        frow = fblock.split(";")[0].split()
        out.append(dict(separation=float(sep), F_x=[eval(v) for v in frow],
                        energy=[eval(v) for v in eblock.split(",")],
                        virial_sum=[eval(v) for v in wblock.split(",")],
                        source="test/test_force_precision_gpu.jl:7-20"))
    return out


def face_positions() -> dict:
    lines = _lines("test/test_force_precision_gpu.jl")
    block = " ".join(lines[22:25])
    nums = [list(map(float, r.split())) for r in block.split("=", 1)[1].replace("[", "").replace("]", "").split(";")]
    L = float(re.search(r"L=T\(([0-9.]+)\)", "\n".join(lines[26:27])).group(1))
    return dict(positions=nums, L=L, tol_f32=2e-5, tol_f64=5e-12, cutoff=2.5,
                source="test/test_force_precision_gpu.jl:22-75")


def neighbor_kats() -> list[dict]:
    # the three value cases of test/test_neighbor_reference.jl:2-4 (transcribed structure, values parsed)
    lines = _lines("test/test_neighbor_reference.jl")[1:4]
    out = []
    for ln in lines:
        m = re.search(r"reference_neighbor_rows\((\(.*\)), (\(.*?\)), (.*?)\) == (\[.*\])", ln)
        coords, box, radii, rows = m.groups()
        radii = radii.replace("fill(1.0, 3)", "[1.0, 1.0, 1.0]")
        conv = lambda s: eval(s.replace("zeros(3)", "[0.0,0.0,0.0]").replace("zeros(2)", "[0.0,0.0]")
                              .replace("Int[]", "[]"))
        c = conv(coords)
        out.append(dict(coords=[list(v) for v in (c if isinstance(c, tuple) else (c,))], box=list(conv(box)),
                        radii=conv(radii), rows=[[j for j in r] for r in conv(rows)],
                        source="test/test_neighbor_reference.jl:2-4"))
    return out


def solver_cases() -> list[dict]:
    lines = _lines("test/test_electrostatics.jl")
    txt = "\n".join(lines[298:310])
    C = float(re.search(r"C = ([0-9.]+)", txt).group(1))
    rc = float(re.search(r"rc = ([0-9.]+)", txt).group(1))
    out = []
    for name, kind, mesh, P, ftol, etol in re.findall(
            r'\("([^"]+)", _(spme|p3m)\(C, rc, 0\.9, \(([0-9, ]+)\), (\d+)(?:, :\w+)?\), ([0-9e.-]+), ([0-9e.-]+)\)',
            txt):
        m = re.search(re.escape(name) + r'", _p3m\(C, rc, 0\.9, \([0-9, ]+\), \d+, :(\w+)', txt)
        influence = "spme" if kind == "spme" else m.group(1)
        out.append(dict(name=name, influence=influence, alpha=0.9, mesh=[int(v) for v in mesh.split(",")],
                        order=int(P), ftol=float(ftol), etol=float(etol)))
    box = [float(v) for v in re.search(r"const _ES_L = \(([^)]*)\)", "\n".join(lines)).group(1).split(",")]
    return [dict(C=C, rc=rc, box=box, n=120, cases=out, source="test/test_electrostatics.jl:299-341")]


def esp_kats() -> dict:
    """Prolate shapes of Table 2 (test/test_electrostatics.jl:55-58), the symmetric window value
    (:88-91) and the ESP solver case of the Ewald comparison (:309)."""
    lines = _lines("test/test_electrostatics.jl")
    txt = "\n".join(lines[54:58])
    table = [[float(a), float(b)] for a, b in re.findall(r"\(([0-9e.-]+), ([0-9.]+)\)", txt)]
    rtol = float(re.search(r"rtol=([0-9e.-]+)", txt).group(1))
    win = "\n".join(lines[87:91])
    P, shape = re.search(r"ProlateWindow\((\d+), ([0-9.]+)\)", win).groups()
    u = float(re.search(r"window_stencil\(pst, ([0-9.]+)\)", win).group(1))
    k0 = int(re.search(r"k0 == (\d+)", win).group(1))
    case = "\n".join(lines[308:309])
    eps, mesh, Pm, ftol, etol = re.search(
        r'\("ESP", _esp\(C, rc, ([0-9e.-]+), \(([0-9, ]+)\), (\d+)\), ([0-9e.-]+), ([0-9e.-]+)\)', case).groups()
    return dict(shape_table=table, shape_rtol=rtol, source_table="test/test_electrostatics.jl:55-58",
                window=dict(order=int(P), shape=float(shape), u=float(u), k0=k0, source="test/test_electrostatics.jl:88-91"),
                solver=dict(eps=float(eps), mesh=[int(v) for v in mesh.split(",")], order=int(Pm), ftol=float(ftol),
                            etol=float(etol), source="test/test_electrostatics.jl:309"))


def main():
    data = dict(two_atom_lj=two_atom_lj(), face=face_positions(), neighbor_rows=neighbor_kats(),
                electrostatics=solver_cases()[0], esp=esp_kats(),
                self_energy="-C alpha/sqrt(pi) sum q^2 (test/test_electrostatics.jl:321)",
                background_energy="-C pi (sum q)^2 / (2 alpha^2 V) (test/test_electrostatics.jl:409)")
    (HERE / "reference_kats.json").write_text(json.dumps(data, indent=1) + "\n")
    print("wrote", HERE / "reference_kats.json")


if __name__ == "__main__":
    main()
