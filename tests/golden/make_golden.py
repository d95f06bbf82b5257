"""Extract the known-answer data of the reference's own unit tests into reference_kats.json.

Run with the SOD2D source tree as the argument (or in $SOD2D_REF):
    python tests/golden/make_golden.py <path to the SOD2D checkout>
The JSON it writes is committed so the tests need no reference tree at run time.

  unitt/unitt_CSR_SPMV_scal/unitt_CSR_SPMV_scal.f90:14-52      CSR matrix, vector, sum(u) = 252
  unitt/unitt_3d_jacobian_inverse/unitt_3d_jacobian_inverse.f90:11-38  TET4 elcod/dN, det(He)=0.0625
  unitt/unitt_char_length/unitt_char_length.f90:13-52          2 QUA04 elements, he = (1, 2)
  unitt/unitt_mass_convec/unitt_mass_convec.f90:30-76          2 QUA04 patch + momentum field
  unitt/unitt_{mass,mom,ener,generic_scalar}_convec/*.f90, unitt/unitt_mom_diffu/*.f90
      the legacy element-loop tests: their hard-coded patch, fields, the QUA04 2x2-Gauss tables
      they build (Ngp, gpcar = He dN, gpvol = w detJ as in the .f90 set-up) and, where the test
      directory has a companion .m script, the residual that script computes (restated here)
"""
from __future__ import annotations

import json
import os
import re
import sys

REF = ""  # the SOD2D checkout, set by main() from argv[1] or $SOD2D_REF
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


def qua04_tables(connec, coord):
    """QUA04 shape tables at the 2x2 Gauss points and the per-element gpcar/gpvol, as the
    legacy unit tests build them: Je = elcod dN^T, He = inverse by the 2x2 formula,
    gpcar = He dN (rows of He times dN), gpvol = w detJe with w = 1."""
    import numpy as np
    g = 1.0 / np.sqrt(3.0)
    xgp = [(-g, -g), (g, -g), (g, g), (-g, g)]
    X = np.array(coord, float)
    C = np.array(connec, int) - 1
    nelem, nnode, ngaus = C.shape[0], 4, 4
    Ngp = np.zeros((ngaus, nnode))
    gpcar = np.zeros((2, nnode, ngaus, nelem))
    gpvol = np.zeros((1, ngaus, nelem))
    for ig, (s_, t_) in enumerate(xgp):
        N = 0.25 * np.array([(1 - s_) * (1 - t_), (1 + s_) * (1 - t_), (1 + s_) * (1 + t_), (1 - s_) * (1 + t_)])
        dN = 0.25 * np.array([[-1 + t_, 1 - t_, 1 + t_, -1 - t_], [-1 + s_, -1 - s_, 1 + s_, 1 - s_]])
        Ngp[ig] = N
        for e in range(nelem):
            elcod = X[C[e]].T                       # (ndime, nnode)
            Je = elcod @ dN.T
            det = Je[0, 0] * Je[1, 1] - Je[1, 0] * Je[0, 1]
            He = np.array([[Je[1, 1], -Je[0, 1]], [-Je[1, 0], Je[0, 0]]]) / det
            gpcar[:, :, ig, e] = He @ dN
            gpvol[0, ig, e] = det
    return {"Ngp": Ngp.tolist(), "gpcar": gpcar.tolist(), "gpvol": gpvol.tolist()}


def legacy_expected(name, case):
    """The residual of the test's companion .m script: R_a += gpvol N_a div(flux) at each Gauss
    point, flux formed at the nodes (mass/generic: q; momentum: q_i u + p e_i; energy: u (E + p))."""
    import numpy as np
    C = np.array(case["connec"]) - 1
    Ngp, gpcar, gpvol = np.array(case["Ngp"]), np.array(case["gpcar"]), np.array(case["gpvol"])
    npoin = len(case["coord"])
    mom = name == "mom_convec"
    R = np.zeros((npoin, 2)) if mom else np.zeros(npoin)
    for e in range(C.shape[0]):
        ind = C[e]
        for ig in range(Ngp.shape[0]):
            car = gpcar[:, :, ig, e]
            if mom:
                q, u, p = np.array(case["q"])[ind], np.array(case["u"])[ind], np.array(case["pr"])[ind]
                div = np.array([sum(car[j] @ (q[:, i] * u[:, j]) for j in range(2)) + car[i] @ p for i in range(2)])
                R[ind] += gpvol[0, ig, e] * np.outer(Ngp[ig], div)
            else:
                if name == "ener_convec":
                    u = np.array(case["u"])[ind]
                    f = u * (np.array(case["E"])[ind] + np.array(case["pr"])[ind])[:, None]
                else:
                    f = np.array(case["q"])[ind]
                div = car[0] @ f[:, 0] + car[1] @ f[:, 1]
                R[ind] += gpvol[0, ig, e] * Ngp[ig] * div
    return R.tolist()


def main():
    global REF
    REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SOD2D_REF", "")
    if not REF or not os.path.isdir(os.path.join(REF, "unitt")):
        sys.stderr.write("usage: make_golden.py <SOD2D checkout with unitt/> (or set SOD2D_REF)\n")
        return 2
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
    for name in ("mass_convec", "mom_convec", "ener_convec", "generic_scalar_convec", "mom_diffu"):
        path = f"unitt/unitt_{name}/unitt_{name}.f90"
        s = rd(path)
        case = {"source": path, "connec": [[int(v) for v in r] for r in _rows(s, "connec")],
                "coord": _rows(s, "coord"), "sum_tol": 1e-14}
        npoin = len(case["coord"])
        if name in ("mass_convec", "generic_scalar_convec"):
            case["q"] = _rows(s, "q")
        else:
            case["u"] = _rows(s, "u")
        m = re.search(r"q\s*=\s*([0-9.]+)d0\s*\*\s*u", s)
        if m:
            case["q"] = [[float(m.group(1)) * x for x in r] for r in case["u"]]
        for scal in ("pr", "E", "mu_e"):
            m = re.search(r"\b" + scal + r"\s*=\s*([0-9.]+)d0", s)
            if m:
                n = len(case["connec"]) if scal == "mu_e" else npoin
                case[scal] = [float(m.group(1))] * n
        tables = qua04_tables(case["connec"], case["coord"])
        case.update(tables)
        mfile = f"unitt/unitt_{name}/unitt_{name}.m"
        if os.path.exists(os.path.join(REF, mfile)):
            case["R_expected"] = legacy_expected(name, case)
            case["R_expected_source"] = mfile
        kats["legacy_" + name] = case
    with open(OUT, "w") as f:
        json.dump(kats, f, indent=1)
    print(OUT)


if __name__ == "__main__":
    sys.exit(main())
