"""Extract golden reference data from the BoSSS sources into small JSON fixtures.

This script is test infrastructure. It runs only where the reference tree is
available (its root is the required ``--ref`` argument); the fixtures it writes
are committed so that the tests never read the reference tree at run time.

What it extracts (all *data*, no code):

* ``ref_basis_2d.json`` -- the orthonormal polynomial table of the square
  reference element, ``Square.cs:194-6481`` (``OrthonormalPolynomials[i]``
  with ``AddCoeff(coef, {ex, ey})``), for total degree <= 5.
* ``ref_basis_3d.json`` -- the same for the cube, ``Cube_polynomials.cs:15-13834``
  (``AddCoeff(coef, {ex, ey, ez})``), total degree <= 5.
* ``ref_gauss_rules.json`` -- the 1D Gauss rules that both reference elements
  use, decoded from the base64/BSON resource ``LineQuadRules_bin.txt``
  (decoder: ``QuadRuleResource.cs:66-77``; tensor construction
  ``Square.cs:110-127`` and ``Cube.cs:155-200``), first 12 rules.
* ``sipg_consistency_p{1,2,3}.json`` -- the reference's stored operator outputs of the
  CNS SIPG consistency test, ``src/L4-application/CNS/Tests/DiffusiveFlux/
  SIPGConsistencyRefSolution_p{1,2,3}.txt`` (one value per DOF, checked there to 1e-11
  by ``SIPGConsistency.cs:87-160``), copied value by value.

Usage::

    python tests/golden/make_golden.py --ref <root of the BoSSS tree>
"""
import argparse
import base64
import json
import os
import re
import struct

FOUNDATION = "src/L2-foundation/BoSSS.Foundation"
SIPG_DIR = "src/L4-application/CNS/Tests/DiffusiveFlux"


def parse_polys(path, dim, max_degree):
    """Parse ``OrthonormalPolynomials[i] = p; p.AddCoeff(c, new int[] {..});`` blocks."""
    polys = {}
    cur = None
    re_idx = re.compile(r"OrthonormalPolynomials\[(\d+)\]\s*=\s*p\s*;")
    re_coef = re.compile(r"p\.AddCoeff\(\s*([-+0-9.eE]+)\s*,\s*new int\[\]\s*\{([^}]*)\}\s*\)")
    with open(path, encoding="utf-8-sig") as f:
        for line in f:
            m = re_idx.search(line)
            if m:
                cur = int(m.group(1))
                polys[cur] = []
                continue
            m = re_coef.search(line)
            if m and cur is not None:
                exps = [int(t) for t in m.group(2).split(",")]
                assert len(exps) == dim, (path, line)
                polys[cur].append([float(m.group(1)), exps])
    out = []
    for i in sorted(polys):
        deg = max(sum(e) for _, e in polys[i])
        if deg > max_degree:
            break
        out.append({"index": i, "terms": polys[i]})
    return out


class _Bson:
    """Minimal BSON reader (double, string, document, array, int32, int64, bool, null)."""

    def __init__(self, data):
        self.d = data

    def doc(self, off):
        (ln,) = struct.unpack_from("<i", self.d, off)
        end = off + ln - 1
        p = off + 4
        res = {}
        while p < end:
            t = self.d[p]
            p += 1
            z = self.d.index(b"\x00", p)
            key = self.d[p:z].decode()
            p = z + 1
            if t == 0x01:
                res[key] = struct.unpack_from("<d", self.d, p)[0]
                p += 8
            elif t == 0x02:
                (sl,) = struct.unpack_from("<i", self.d, p)
                res[key] = self.d[p + 4:p + 4 + sl - 1].decode()
                p += 4 + sl
            elif t in (0x03, 0x04):
                sub = self.doc(p)
                (sl,) = struct.unpack_from("<i", self.d, p)
                if t == 0x04:
                    sub = [sub[k] for k in sorted(sub, key=int)]
                res[key] = sub
                p += sl
            elif t == 0x10:
                res[key] = struct.unpack_from("<i", self.d, p)[0]
                p += 4
            elif t == 0x12:
                res[key] = struct.unpack_from("<q", self.d, p)[0]
                p += 8
            elif t == 0x08:
                res[key] = bool(self.d[p])
                p += 1
            elif t == 0x0A:
                res[key] = None
            else:
                raise ValueError("unsupported BSON type 0x%02x" % t)
        return res


def parse_line_rules(path, count):
    with open(path) as f:
        raw = base64.b64decode(f.read().strip())
    top = _Bson(raw).doc(0)
    rules = []
    for q in top["Quadrules"][:count]:
        nodes = [row[0] for row in q["Item2"]]
        rules.append({"order": q["Item1"], "nodes": nodes, "weights": list(q["Item3"])})
    rules.sort(key=lambda r: r["order"])
    return rules


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="root of the BoSSS source tree")
    args = ap.parse_args()
    here = os.path.dirname(os.path.abspath(__file__))
    base = os.path.join(args.ref, FOUNDATION)

    sq = parse_polys(os.path.join(base, "Square.cs"), 2, 5)
    cu = parse_polys(os.path.join(base, "Cube_polynomials.cs"), 3, 5)
    rules = parse_line_rules(os.path.join(base, "LineQuadRules_bin.txt"), 60)
    rules = [r for r in rules if r["order"] <= 23]

    src = "BoSSS " + FOUNDATION
    with open(os.path.join(here, "ref_basis_2d.json"), "w") as f:
        json.dump({"source": src + "/Square.cs", "polys": sq}, f, indent=0)
    with open(os.path.join(here, "ref_basis_3d.json"), "w") as f:
        json.dump({"source": src + "/Cube_polynomials.cs", "polys": cu}, f, indent=0)
    with open(os.path.join(here, "ref_gauss_rules.json"), "w") as f:
        json.dump({"source": src + "/LineQuadRules_bin.txt", "rules": rules}, f, indent=0)
    print("2d polys:", len(sq), "3d polys:", len(cu), "rules:", [r["order"] for r in rules])

    sipg = os.path.join(args.ref, SIPG_DIR)
    for p in (1, 2, 3):
        name = "SIPGConsistencyRefSolution_p%d.txt" % p
        with open(os.path.join(sipg, name), encoding="utf-8-sig") as f:
            vals = [float(line) for line in f if line.strip()]
        with open(os.path.join(here, "sipg_consistency_p%d.json" % p), "w") as f:
            json.dump({"source": "BoSSS " + SIPG_DIR + "/" + name, "degree": p, "values": vals}, f, indent=0)
        print(name, len(vals), "values")


if __name__ == "__main__":
    main()
