"""Extract the known-answer data of the reference's own unit tests into reference_kats.json.

Run in a checkout that has the SOD2D sources (default path below or $SOD2D_REF); the JSON it
writes is committed so the tests need no reference tree at run time.

  unitt/unitt_CSR_SPMV_scal/unitt_CSR_SPMV_scal.f90:14-52      CSR matrix, vector, sum(u) = 252
  unitt/unitt_3d_jacobian_inverse/unitt_3d_jacobian_inverse.f90:11-38  TET4 elcod/dN, det(He)=0.0625
  unitt/unitt_char_length/unitt_char_length.f90:13-52          2 QUA04 elements, he = (1, 2)
  unitt/unitt_mass_convec/unitt_mass_convec.f90:30-76          2 QUA04 patch + momentum field
"""
from __future__ import annotations

import json
import os
import re
import sys

REF = os.environ.get("SOD2D_REF", "/root/reference")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_kats.json")


def _vals(txt: str):
    out = []
    for tok in txt.replace("\n", " ").split(","):
        tok = tok.strip().lower().replace("d0", "").replace("_rp", "")
        if tok:
            out.append(float(tok))
    return out


def _arr(src: str, name: str):
    """Concatenate the values of every `name(a:b) = (/ ... /)` assignment in order."""
    vals = []
    for m in re.finditer(re.escape(name) + r"\((\d+):(\d+)\)\s*=\s*\(/(.*?)/\)", src, re.S):
        vals.extend(_vals(m.group(3)))
    return vals


def _rows(src: str, name: str):
    """`name(i,:) = (/ ... /)` rows keyed by i."""
    rows = {}
    for m in re.finditer(re.escape(name) + r"\((\d+),:\)\s*=\s*\(/(.*?)/\)", src, re.S):
        rows[int(m.group(1))] = _vals(m.group(2))
    return [rows[k] for k in sorted(rows)]


def main():
    rd = lambda p: open(os.path.join(REF, p)).read()
    kats = {}
    s = rd("unitt/unitt_CSR_SPMV_scal/unitt_CSR_SPMV_scal.f90")
    kats["csr_spmv"] = {
        "source": "unitt/unitt_CSR_SPMV_scal/unitt_CSR_SPMV_scal.f90:14-52",
        "Mc": _arr(s, "Mc"),
        "cdom": [int(v) for v in _arr(s, "cdom")],
        "rdom": [int(v) for v in _arr(s, "rdom")],
        "v": _arr(s, "v"),
        "sum_u": float(re.search(r"sum\(u\)\s*\.gt\.\s*([0-9.]+)d0", s).group(1)),
    }
    s = rd("unitt/unitt_3d_jacobian_inverse/unitt_3d_jacobian_inverse.f90")
    elcod = [[_vals(m.group(2)) for m in re.finditer(r"elcod\((\d),1:4\)\s*=\s*\(/(.*?)/\)", s)]][0]
    dN = [[_vals(m.group(2)) for m in re.finditer(r"dN\((\d),1:4\)\s*=\s*\(/(.*?)/\)", s)]][0]
    kats["jacobian_inverse"] = {
        "source": "unitt/unitt_3d_jacobian_inverse/unitt_3d_jacobian_inverse.f90:11-38",
        "elcod": elcod, "dN": dN,
        "det_He": float(re.search(r"detHe \.gt\. ([0-9.]+)d0", s).group(1)),
        "tol": 1e-10,
    }
    s = rd("unitt/unitt_char_length/unitt_char_length.f90")
    kats["char_length"] = {
        "source": "unitt/unitt_char_length/unitt_char_length.f90:13-52",
        "connec": [[int(v) for v in r] for r in _rows(s, "connec")],
        "coord": _rows(s, "coord"),
        "he": [1.0, 2.0],
    }
    s = rd("unitt/unitt_mass_convec/unitt_mass_convec.f90")
    kats["mass_convec_patch"] = {
        "source": "unitt/unitt_mass_convec/unitt_mass_convec.f90:30-76,157-163",
        "connec": [[int(v) for v in r] for r in _rows(s, "connec")],
        "coord": _rows(s, "coord"),
        "q": _rows(s, "q"),
        "sum_tol": 1e-14,
    }
    with open(OUT, "w") as f:
        json.dump(kats, f, indent=1)
    print(OUT)


if __name__ == "__main__":
    sys.exit(main())
