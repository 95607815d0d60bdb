"""Generates the fixtures of SALMON's bulk-Si testsuites for the end-to-end tests.

Run where the reference tree is present:

    python tests/golden/make_testsuite_golden.py [REFERENCE_ROOT]

Outputs (committed):
  si_rps_ky.npz          the tables of testsuites/pseudo/Si_rps.dat as the KY
                         reader parses them (header, cut-off radii, V_l and u_l
                         rows, file units), so machines without the reference
                         tree can build the physical Si system
  testsuite_si.json      the inputs (&system, &rgrid, &kgrid, &tgrid, &scf,
                         &emfield) and the verification tables of
                         testsuites/001_bulk_gs and testsuites/002_bulk_rt:
                         (file, row, column, reference value, tolerance, label)

The verification scripts are read as text: the `reference['<file>'] = [...]`
tables are taken out with a regular expression and parsed with
a small literal evaluator; nothing from the reference tree is executed.
"""
import ast
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def _literal(node):
    """Numbers, strings, lists and + - * on numbers (the tables write rows as
    `1-1`); anything else is rejected."""
    if isinstance(node, ast.Expression):
        return _literal(node.body)
    if isinstance(node, ast.Constant) and isinstance(node.value, (int, float, str)):
        return node.value
    if isinstance(node, (ast.List, ast.Tuple)):
        return [_literal(e) for e in node.elts]
    if isinstance(node, ast.UnaryOp) and isinstance(node.op, (ast.UAdd, ast.USub)):
        v = _literal(node.operand)
        return v if isinstance(node.op, ast.UAdd) else -v
    if isinstance(node, ast.BinOp) and isinstance(node.op, (ast.Add, ast.Sub, ast.Mult)):
        lhs, rhs = _literal(node.left), _literal(node.right)
        if not all(isinstance(v, (int, float)) for v in (lhs, rhs)):
            raise ValueError("arithmetic on non-numbers")
        return {ast.Add: lhs + rhs, ast.Sub: lhs - rhs, ast.Mult: lhs * rhs}[type(node.op)]
    raise ValueError(f"unexpected expression {ast.dump(node)}")


def parse_verification(path):
    text = open(path).read()
    out = []
    for m in re.finditer(r"reference\['([^']+)'\]\s*=\s*(\[.*?\n\])", text, re.S):
        fname, body = m.group(1), m.group(2)
        # keep only the list rows; the comment lines are not Python literals
        rows = [ln for ln in body.splitlines() if not ln.strip().startswith("#")]
        table = _literal(ast.parse("\n".join(rows), mode="eval"))
        for row_expr in table:
            r, c, val, tol, info = row_expr
            out.append({"file": fname, "row": int(r), "col": int(c), "value": float(val), "tol": float(tol),
                        "label": info})
    return out


def parse_rps(path):
    toks = open(path).read().split()
    mr, step, mlps, rzps = int(toks[0]), float(toks[1]), int(toks[2]), float(toks[3])
    pos = 4
    irpc = int(toks[pos]); pos += 1
    rrc = np.array([float(v) for v in toks[pos:pos + mlps + 1]]); pos += mlps + 1
    vrows = np.array([float(v) for v in toks[pos:pos + (mr + 1) * (mlps + 3)]]).reshape(mr + 1, mlps + 3)
    pos += (mr + 1) * (mlps + 3)
    urows = np.array([float(v) for v in toks[pos:pos + (mr + 1) * (mlps + 2)]]).reshape(mr + 1, mlps + 2)
    return dict(mr=mr, step=step, mlps=mlps, zps=rzps, irpc=irpc, rrc=rrc, vpp=vrows[:, 2:], upp=urows[:, 1:],
                r=vrows[:, 0])


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REF_ROOT")
    if not ref:
        sys.exit("usage: make_testsuite_golden.py <SALMON source tree>  (or set REF_ROOT)")
    ts = os.path.join(ref, "testsuites")
    d = parse_rps(os.path.join(ts, "pseudo", "Si_rps.dat"))
    np.savez_compressed(os.path.join(HERE, "si_rps_ky.npz"), **d)
    gs = parse_verification(os.path.join(ts, "001_bulk_gs", "verification"))
    rt = parse_verification(os.path.join(ts, "002_bulk_rt", "verification"))
    inputs = {
        # testsuites/00{1,2}_*/inputfile, as read: the values both runs share, then the RT ones
        "al": [10.26, 10.26, 10.26], "nstate": 32, "nelec": 32, "natom": 8, "izatom": 14, "lloc_ps": 2,
        "xc": "PZ", "num_rgrid": [8, 8, 8], "num_kgrid": [4, 4, 4], "ncg": 5, "nscf": 100, "threshold": 1e-9,
        "nt": 1200, "dt": 0.10, "propagator": "middlepoint", "ae_shape1": "Acos2", "rlaser_int_wcm2_1": 1e12,
        "pulse_tw1": 110.30592311334672, "omega1": 0.05696144984638035, "epdir_re1": [0.0, 0.0, 1.0],
    }
    for name, key in (("001_bulk_gs", "inputfile"), ("002_bulk_rt", "inputfile")):
        text = open(os.path.join(ts, name, key)).read()
        checks = [("nstate", "32"), ("nelec", "32"), ("natom", "8"), ("num_rgrid", "8, 8, 8"),
                  ("num_kgrid", "4, 4, 4"), ("lloc_ps(1)", "2"), ("xc", "'PZ'"), ("ncg", "5"), ("nscf", "100"),
                  ("threshold", "1.d-9")]
        if name == "002_bulk_rt":
            checks += [("nt", "1200"), ("dt", "0.10"), ("propagator", "'middlepoint'"), ("ae_shape1", "'Acos2'"),
                       ("rlaser_int_wcm2_1", "1d12"), ("pulse_tw1", "110.30592311334672d0"),
                       ("omega1", "0.05696144984638035d0"), ("epdir_re1", "0., 0., 1.")]
        for k, v in checks:
            if not re.search(r"\b" + re.escape(k) + r"\s*=\s*" + re.escape(v), text):
                raise SystemExit(f"{name}/inputfile: expected {k} = {v}")
    with open(os.path.join(HERE, "testsuite_si.json"), "w") as f:
        json.dump({"inputs": inputs, "001_bulk_gs": gs, "002_bulk_rt": rt}, f, indent=1)
    print(f"wrote si_rps_ky.npz ({d['mr'] + 1} rows) and testsuite_si.json ({len(gs)} + {len(rt)} checks)")


if __name__ == "__main__":
    main()
