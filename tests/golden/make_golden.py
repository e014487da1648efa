"""Extract the reference's own fixtures into tests/golden/reference_fixtures.json.

Sources (gfn1-rs v0.5.1):
* examples/h2.engrad: H2 at R = 1.3983973 bohr, energy and gradient (the only
  stored absolute result in the reference tree);
* examples/{h2,water,ammonia,methane,water48,water100}.xyz: geometries;
* the molecules embedded in tests/nonpbc_smoke.rs:14-50 (H/C/N/O/F/B/P subset),
  read as text;
* the halogen-bond test systems embedded in src/halogen.rs (its unit tests,
  from :788), keyed by their xyz title line;
* the molecules of tests/scf_accelerators.rs:10-20 (water, 2-bromoethanol),
  keyed by their constant's name in lower case.

Run where the reference tree is available:
    python tests/golden/make_golden.py /path/to/gfn1-rs
"""
from __future__ import annotations

import json
import re
import sys
from pathlib import Path


def read_engrad(path: Path) -> dict:
    lines = [l.strip() for l in path.read_text().splitlines()]
    vals = [l for l in lines if l and not l.startswith("#")]
    nat = int(vals[0])
    energy = float(vals[1])
    grad = [float(v) for v in vals[2:2 + 3 * nat]]
    atoms = [v.split() for v in vals[2 + 3 * nat:2 + 4 * nat]]
    return {
        "numbers": [int(a[0]) for a in atoms],
        "positions_bohr": [[float(x) for x in a[1:4]] for a in atoms],
        "energy": energy,
        "gradient": [grad[3 * i:3 * i + 3] for i in range(nat)],
    }


SYMBOLS = {"H": 1, "He": 2, "Li": 3, "Be": 4, "B": 5, "C": 6, "N": 7, "O": 8, "F": 9, "Ne": 10, "P": 15,
           "S": 16, "Cl": 17, "Fe": 26, "Br": 35, "I": 53}


def read_xyz_text(text: str) -> dict:
    lines = text.strip("\n").splitlines()
    nat = int(lines[0].split()[0])
    numbers, pos = [], []
    for l in lines[2:2 + nat]:
        p = l.split()
        numbers.append(SYMBOLS[p[0]])
        pos.append([float(x) for x in p[1:4]])
    return {"numbers": numbers, "positions_angstrom": pos}


def main(root: str) -> None:
    root = Path(root)
    out = {"source": "gfn1-rs v0.5.1 examples/ and tests/nonpbc_smoke.rs", "h2_engrad": read_engrad(root / "examples/h2.engrad")}
    xyz = {}
    for name in ("h2", "water", "ammonia", "methane", "water48", "water100"):
        xyz[name] = read_xyz_text((root / f"examples/{name}.xyz").read_text())
    out["xyz"] = xyz
    smoke = (root / "tests/nonpbc_smoke.rs").read_text()
    mols = {}
    for m in re.finditer(r'name: "([^"]+)",\s*xyz: "([^"]+)",\s*gradient_fd: (true|false)', smoke):
        text = m.group(2).encode().decode("unicode_escape")
        rec = read_xyz_text(text)
        rec["gradient_fd"] = m.group(3) == "true"
        mols[m.group(1)] = rec
    out["nonpbc_smoke"] = mols
    hal = {}
    src = (root / "src/halogen.rs").read_text()
    for m in re.finditer(r'from_xyz_str\(\s*"((?:[^"\\]|\\.)*)"', src, re.S):
        lit = re.sub(r"\\\n\s*", "", m.group(1))  # Rust line continuations
        text = lit.encode().decode("unicode_escape")
        title = text.splitlines()[1].strip()
        if "Lattice=" in title:  # periodic systems are outside the molecular path
            continue
        hal.setdefault(title, read_xyz_text(text))
    out["halogen_tests"] = hal
    acc = {}
    src = (root / "tests/scf_accelerators.rs").read_text()
    for m in re.finditer(r'const (\w+): &str = "((?:[^"\\]|\\.)*)";', src, re.S):
        lit = re.sub(r"\\\n\s*", "", m.group(2))  # Rust line continuations
        acc[m.group(1).lower()] = read_xyz_text(lit.encode().decode("unicode_escape"))
    out["scf_accelerators"] = acc
    dest = Path(__file__).with_name("reference_fixtures.json")
    dest.write_text(json.dumps(out, indent=1) + "\n")


if __name__ == "__main__":
    import os

    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GFN1_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: make_golden.py REFERENCE_ROOT (or set GFN1_REFERENCE_ROOT): a gfn1-rs v0.5.1 checkout")
    main(root)
