"""Generate ``gfn1_tables.txt``: the GFN1-xTB data tables the engine and the CPU
oracle load at run time.

The tables are published data, not code:

* GFN1-xTB parameters (``$globpar``, ``$pairpar``, ``$Z=`` blocks) from the
  grimme-lab/xtb parameter file (LGPL-3.0-or-later), as bundled by gfn1-rs v0.5.1
  in ``third_party/xtb/param_gfn1-xtb.txt``;
* Stewart's STO-nG expansion exponents/coefficients (J. Chem. Phys. 52, 431
  (1970)) as tabulated in gfn1-rs ``src/sto.rs:24-788``;
* the GFN1 reference shell occupations (gfn1-rs ``src/basis.rs:446-531``), the
  xTB atomic radii, mctc covalent radii, Pauling electronegativities and
  relative atomic masses (gfn1-rs ``src/data_tables.rs:14-174``);
* the DFT-D3 reference coordination numbers, C6 table and <r4>/<r2> values from
  simple-dftd3 (LGPL-3.0-or-later), ``third_party/simple-dftd3/src/dftd3/
  {reference.f90,data/r4r2.f90}``.

Run it where the gfn1-rs v0.5.1 source tree is available::

    python gen_tables.py /path/to/gfn1-rs  > gfn1_tables.txt

The output is a line format ``key count v1 ... vcount`` (``#`` starts a comment)
that both the C++ oracle and the engine parse.  Only elements Z = 1..86 are
emitted (the GFN1 parametrisation ends at Rn).
"""
from __future__ import annotations

import re
import sys
from pathlib import Path

MAX_Z = 86


def _floats(text: str) -> list[float]:
    """Numeric tokens of a Rust or Fortran array literal (``_wp`` suffixes and
    Fortran ``d`` exponents allowed)."""
    out = []
    for tok in re.findall(r"[0-9+\-.eEdD]+", text):
        if not any(c.isdigit() for c in tok):
            continue
        out.append(float(tok.replace("d", "e").replace("D", "e")))
    return out


def _rust_array(src: str, name: str) -> list[float]:
    m = re.search(r"const\s+" + re.escape(name) + r"\s*:[^=]*=\s*\[", src)
    if not m:
        raise KeyError(name)
    depth, i = 0, m.end() - 1
    start = i
    while True:
        c = src[i]
        if c == "[":
            depth += 1
        elif c == "]":
            depth -= 1
            if depth == 0:
                break
        i += 1
    body = src[start + 1 : i]
    body = re.sub(r"//[^\n]*", "", body)
    return _floats(body)


def parse_param_file(text: str):
    globpar, pairpar, elems = {}, {}, {}
    section, cur = None, None
    for raw in text.splitlines():
        line = raw.strip()
        if not line or line.startswith("#"):
            continue
        if line.startswith("$info"):
            section = "info"
            continue
        if line.startswith("$globpar"):
            section = "glob"
            continue
        if line.startswith("$pairpar"):
            section = "pair"
            continue
        if line.startswith("$Z="):
            z = int(line[3:].split()[0])
            cur = {"z": z}
            elems[z] = cur
            section = "elem"
            continue
        if line.startswith("$end"):
            section = None
            continue
        if section == "glob":
            k, v = line.split()
            globpar[k.lower()] = float(v)
        elif section == "pair":
            a, b, v = line.split()
            a, b = int(a), int(b)
            pairpar[(min(a, b), max(a, b))] = float(v)
        elif section == "elem":
            if line.startswith("ao="):
                labels = re.findall(r"(\d+)([spdfg])", line[3:].strip())
                cur["ao"] = [(int(n), "spdfg".index(l)) for n, l in labels]
            else:
                k, v = line.split("=", 1)
                cur[k.strip().upper()] = [float(x) for x in v.split()]
    return globpar, pairpar, elems


def parse_d3(ref_text: str, r4r2_text: str):
    clean = "\n".join(l.split("!")[0] for l in ref_text.splitlines())
    max_elem = int(re.search(r"max_elem\s*=\s*(\d+)", clean).group(1))
    max_ref = int(re.search(r"max_ref\s*=\s*(\d+)", clean).group(1))

    def array_after(marker: str, text: str) -> list[float]:
        pos = text.index(":: " + marker)
        open_ = text.index("[", pos)
        depth, i = 0, open_
        while True:
            if text[i] == "[":
                depth += 1
            elif text[i] == "]":
                depth -= 1
                if depth == 0:
                    break
            i += 1
        return _floats(text[open_ + 1 : i])

    nref = [int(round(v)) for v in array_after("number_of_references", clean)]
    cnref = array_after("reference_cn", clean)
    c6 = []
    for m in re.finditer(r"c6ab_view\(\s*\d+\s*:\s*\d+\s*\)\s*=\s*\[", clean):
        open_ = m.end() - 1
        depth, i = 0, open_
        while True:
            if clean[i] == "[":
                depth += 1
            elif clean[i] == "]":
                depth -= 1
                if depth == 0:
                    break
            i += 1
        c6.extend(_floats(clean[open_ + 1 : i]))
    assert len(nref) == max_elem, len(nref)
    assert len(cnref) == max_ref * max_elem, len(cnref)
    assert len(c6) == max_ref * max_ref * max_elem * (max_elem + 1) // 2, len(c6)
    r4c = "\n".join(l.split("!")[0] for l in r4r2_text.splitlines())
    r4r2 = array_after("r4_over_r2", r4c)
    return max_ref, nref, cnref, c6, r4r2


def fmt(v: float) -> str:
    return repr(float(v))


def main(root: str) -> None:
    root = Path(root)
    ptext = (root / "third_party/xtb/param_gfn1-xtb.txt").read_text()
    globpar, pairpar, elems = parse_param_file(ptext)
    sto = (root / "src/sto.rs").read_text()
    basis = (root / "src/basis.rs").read_text()
    tables = (root / "src/data_tables.rs").read_text()
    d3ref = (root / "third_party/simple-dftd3/src/dftd3/reference.f90").read_text()
    d3r4 = (root / "third_party/simple-dftd3/src/dftd3/data/r4r2.f90").read_text()
    max_ref, nref, cnref, c6, r4r2 = parse_d3(d3ref, d3r4)

    out = []
    w = out.append
    w("# GFN1-xTB data tables generated by gen_tables.py from gfn1-rs v0.5.1")
    w("# parameters: grimme-lab/xtb param_gfn1-xtb.txt (LGPL-3.0-or-later)")
    w("# D3 reference: simple-dftd3 reference.f90 / r4r2.f90 (LGPL-3.0-or-later)")
    w("# STO-nG: Stewart, J. Chem. Phys. 52, 431 (1970)")
    w("# format: key count values...")
    for k in sorted(globpar):
        w(f"glob.{k} 1 {fmt(globpar[k])}")
    for (a, b) in sorted(pairpar):
        w(f"pair.{a}.{b} 1 {fmt(pairpar[(a, b)])}")
    for z in range(1, MAX_Z + 1):
        e = elems[z]
        ao = e["ao"]
        w(f"elem.{z}.ao {2 * len(ao)} " + " ".join(f"{n} {l}" for n, l in ao))
        for key in ("LEV", "EXP"):
            vals = e[key]
            assert len(vals) == len(ao)
            w(f"elem.{z}.{key.lower()} {len(vals)} " + " ".join(fmt(v) for v in vals))
        for key, default in (("GAM", None), ("GAM3", 0.0), ("REPA", None), ("REPB", None),
                             ("POLYS", 0.0), ("POLYP", 0.0), ("POLYD", 0.0),
                             ("LPARS", 0.0), ("LPARP", 0.0), ("LPARD", 0.0)):
            v = e.get(key, [default])[0]
            assert v is not None, (z, key)
            w(f"elem.{z}.{key.lower()} 1 {fmt(v)}")
        if "CXB" in e:  # halogen-bond strength, present for Br, I and At only
            w(f"elem.{z}.cxb 1 {fmt(e['CXB'][0])}")
    nf = 15
    for ng in range(1, 7):
        alpha = _rust_array(sto, f"P_ALPHA{ng}")
        coeff = _rust_array(sto, f"P_COEFF{ng}") if ng > 1 else [1.0] * nf
        assert len(alpha) == nf * ng and len(coeff) == nf * ng, (ng, len(alpha), len(coeff))
        w(f"sto.alpha.{ng} {len(alpha)} " + " ".join(fmt(v) for v in alpha))
        w(f"sto.coeff.{ng} {len(coeff)} " + " ".join(fmt(v) for v in coeff))
    for name in ("P_ALPHA6S", "P_COEFF6S", "P_ALPHA6P", "P_COEFF6P"):
        vals = _rust_array(sto, name)
        assert len(vals) == 6
        w(f"sto.{name[2:].lower()} 6 " + " ".join(fmt(v) for v in vals))
    refocc = _rust_array(basis, "GFN1_REFERENCE_OCC")
    assert len(refocc) == 87 * 3
    w(f"refocc {len(refocc)} " + " ".join(fmt(v) for v in refocc))
    for key, name in (("atomic_radius_ang", "XTB_ATOMIC_RADII_ANGSTROM"),
                      ("covrad_ang", "MCTC_COVALENT_RADII_2009_ANGSTROM"),
                      ("pauling_en", "PAULING_EN"),
                      ("atomic_mass_amu", "RELATIVE_ATOMIC_MASSES")):
        vals = _rust_array(tables, name)[: MAX_Z + 1]
        assert len(vals) == MAX_Z + 1
        w(f"{key} {len(vals)} " + " ".join(fmt(v) for v in vals))
    w(f"d3.nref {MAX_Z} " + " ".join(str(n) for n in nref[:MAX_Z]))
    for z in range(1, MAX_Z + 1):
        n = nref[z - 1]
        vals = cnref[(z - 1) * max_ref : (z - 1) * max_ref + n]
        w(f"d3.cnref.{z} {n} " + " ".join(fmt(v) for v in vals))
    w(f"d3.r4r2 {MAX_Z} " + " ".join(fmt(v) for v in r4r2[:MAX_Z]))
    for a in range(1, MAX_Z + 1):
        for b in range(1, a + 1):
            pair = b + a * (a - 1) // 2 - 1
            na, nb = nref[a - 1], nref[b - 1]
            blk = []
            for ia in range(na):
                for ib in range(nb):
                    blk.append(c6[pair * max_ref * max_ref + ib * max_ref + ia])
            w(f"d3.c6.{a}.{b} {len(blk)} " + " ".join(fmt(v) for v in blk))
    sys.stdout.write("\n".join(out) + "\n")


if __name__ == "__main__":
    import os

    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GFN1_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: gen_tables.py REFERENCE_ROOT (or set GFN1_REFERENCE_ROOT): a gfn1-rs v0.5.1 checkout")
    main(root)
