"""Extract the reference's known-answer vectors into JSON fixtures.

The reference (Fortran) keeps its known answers inside its test programs.
This script reads those programs AS TEXT (it compiles and runs nothing) and
writes the inputs and expected values to small JSON files next to it, so the
tests can pin the oracle without access to the reference tree.

Usage:  python tests/golden/make_golden.py <reference_root>
(the root of a checkout of the reference project; required)

Sources:
  src/test_files/test_augeanstables/test_mattsson_operators.f
      known values of the Mattsson operators (:150-946), inputs
      initialize_nodes_x/_y (:1594-1699), check routine test_operator
      (:1241-1497) with the secondary procedure gradient_av (:1219-1238).
  src/test_files/test_lernaeanhydra/test_dim2d_fluxes.f
      26 DIM face-flux values (:291-367) on a 5x5x4 array.
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
NUM = r"[-+]?(?:\d+\.?\d*|\.\d+)(?:[dDeE][-+]?\d+)?"


def fnum(s):
    return float(s.lower().replace("d", "e"))


def literal_tolerance(s, value):
    """Absolute tolerance implied by a printed literal.

    Literals with 6+ significant digits are rounded/truncated prints of an
    irrational result: allow half a unit of their last printed digit.
    Shorter literals are exact answers: allow 1e-9 relative."""
    m = s.lower().replace("d", "e").lstrip("+-")
    mant = m.split("e")[0]
    digits = mant.replace(".", "").lstrip("0")
    dec = len(mant.split(".")[1]) if "." in mant else 0
    if len(digits) >= 6:
        return 0.5 * 10.0 ** (-dec) + 1e-9 * abs(value)
    return 1e-9 * max(1.0, abs(value))


def parse_init(lines, name):
    """nodes(i,j,1)=v assignments and dx/dy of subroutine `name`."""
    start = next(k for k, l in enumerate(lines) if re.search(r"subroutine\s+%s\b" % name, l))
    out = {"nodes": [], "dx": None, "dy": None}
    for l in lines[start + 1:]:
        if re.search(r"end subroutine", l):
            break
        m = re.match(r"\s*nodes\((\d+),(\d+),1\)\s*=\s*(%s)" % NUM, l)
        if m:
            out["nodes"].append([int(m.group(1)), int(m.group(2)), fnum(m.group(3))])
        m = re.match(r"\s*(dx|dy)\s*=\s*(%s)" % NUM, l)
        if m:
            out[m.group(1)] = fnum(m.group(2))
    return out


def mattsson(ref):
    path = os.path.join(ref, "src/test_files/test_augeanstables/test_mattsson_operators.f")
    lines = open(path).read().splitlines()
    inits = {n: parse_init(lines, n) for n in ("initialize_nodes_x", "initialize_nodes_y")}
    cases = []
    current_init = None
    name = None
    data = {}
    k = 0
    while k < len(lines):
        l = lines[k]
        m = re.search(r"call (initialize_nodes_[xy])\(", l)
        if m:
            current_init = m.group(1)
        m = re.search(r"print '\(''test ([A-Za-z0-9_]+)''\)'", l)
        if m:
            name = m.group(1)
            data = {}
        m = re.match(r"\s*test_data\((\d+)\)\s*=\s*(%s)" % NUM, l)
        if m:
            data[int(m.group(1))] = m.group(2)
        if re.search(r"call test_operator\($", l.rstrip()):
            block = []
            k += 1
            while True:
                block.append(lines[k].strip().lstrip("$").strip())
                if ")" in lines[k] and "test_data" in lines[k] or lines[k].rstrip().endswith(")"):
                    if lines[k].rstrip().endswith(")"):
                        break
                k += 1
            text = " ".join(block)
            toks = [t.strip() for t in text.rstrip(")").split(",")]
            sd_set, gx, gy = toks[0], toks[1], toks[2]
            i1, j1, i2, j2 = (int(t) for t in toks[3:7])
            only_f = "test_only_f=.true." in text
            only_g = "test_only_g=.true." in text
            vals = {}
            for idx, s in sorted(data.items()):
                v = fnum(s)
                vals[idx] = {"value": v, "literal": s, "tol": literal_tolerance(s, v)}
            cases.append({
                "name": name, "set": sd_set, "gradient_x": gx, "gradient_y": gy,
                "i1": i1, "j1": j1, "i2": i2, "j2": j2,
                "test_only_f": only_f, "test_only_g": only_g,
                "init": current_init, "expected": vals,
            })
        k += 1
    return {
        "source": "src/test_files/test_augeanstables/test_mattsson_operators.f",
        "ops": ["f", "dfdx", "dfdy", "d2fdx2", "d2fdy2", "d2fdxdy", "gradient_x",
                "g", "dgdx", "dgdy", "d2gdx2", "d2gdy2", "d2gdxdy", "gradient_y",
                "dfdx_nl(gradient_av)", "dgdy_nl(gradient_av)"],
        "inits": inits, "cases": cases,
    }


def dim2d_fluxes(ref):
    path = os.path.join(ref, "src/test_files/test_lernaeanhydra/test_dim2d_fluxes.f")
    src = open(path).read()
    body = src[src.index("subroutine initialize_data"):]
    arr = body[body.index("reshape((/") + len("reshape((/"):body.index("/),")]
    arr = re.sub(r"\n\s*\$", " ", arr)
    values = [fnum(t) for t in re.findall(NUM, arr)]
    assert len(values) == 100, len(values)
    expected = {}
    for m in re.finditer(r"test_data\((\d+)\)\s*=\s*(%s)" % NUM, body):
        v = fnum(m.group(2))
        expected[int(m.group(1))] = {"value": v, "literal": m.group(2),
                                     "tol": literal_tolerance(m.group(2), v)}
    dx = fnum(re.search(r"\bdx\s*=\s*(%s)" % NUM, body).group(1))
    dy = fnum(re.search(r"\bdy\s*=\s*(%s)" % NUM, body).group(1))
    i = int(re.search(r"\bi\s*=\s*(\d+)", body).group(1))
    j = int(re.search(r"\bj\s*=\s*(\d+)", body).group(1))
    params = {}
    for key in ("viscous_r", "re", "pr", "we", "cv_r"):
        m = re.search(r"\(%s\.eq\.(%s)\)" % (key, NUM), src)
        params[key] = fnum(m.group(1))
    return {
        "source": "src/test_files/test_lernaeanhydra/test_dim2d_fluxes.f",
        "shape": [5, 5, 4], "order": "fortran", "nodes": values,
        "dx": dx, "dy": dy, "i": i, "j": j, "params": params,
        "expected": expected,
    }


def _reshape_blocks(text, ne):
    """All `reshape((/ ... /),(/a,b,c/))` literals of a Fortran text, in order
    (`ne` stands for the number of equations of that test)."""
    out = []
    for m in re.finditer(r"reshape\(\(/(.*?)/\)[\s$]*,[\s$]*\(/([\w,\s]+)/\)\)", text, re.S):
        body = re.sub(r"\n\s*\$", " ", m.group(1))
        if "=" in body:  # implied-do constructors are generated, not literal
            continue
        vals = [fnum(t) for t in re.findall(NUM, body)]
        shape = [ne if s.strip() == "ne" else int(s) for s in m.group(2).split(",")]
        out.append({"values": vals, "shape": shape})
    return out


def hedstrom(ref):
    """test_bc_operators/test_hedstrom_xy.f:54-178."""
    path = os.path.join(ref, "src/test_files/test_bc_operators/test_hedstrom_xy.f")
    src = open(path).read()
    blocks = _reshape_blocks(src, 4)
    nodes_L0, nodes_R0 = blocks[0], blocks[1]
    vecs = re.findall(r"\[([^\]]*)\]", src)
    vecs = [[fnum(t) for t in re.findall(NUM, re.sub(r"\n\s*\$", " ", v))] for v in vecs]
    vecs = [v for v in vecs if len(v) in (4, 5)]
    td_L0, td_R0 = [v for v in vecs if len(v) == 4][:2]
    obc = [v for v in vecs if len(v) == 5]
    dx = fnum(re.search(r"\bdx\s*=\s*(%s)" % NUM, src).group(1))
    return {
        "source": "src/test_files/test_bc_operators/test_hedstrom_xy.f",
        "note": "obc_eigenqties_lin: the 5 far-field eigen-quantities (rho,u,v,P,c) are the "
                "values get_prim_obc_eigenqties must return in the same test",
        "nodes_L0": nodes_L0, "nodes_R0": nodes_R0, "i_L0": 1, "i_R0": 3, "j": 1,
        "dx": dx, "cv_r": 2.5,
        "obc_prim": obc[-1], "obc_prim_input": obc[0] if len(obc) > 1 else None,
        "timedev_L0": td_L0, "timedev_R0": td_R0,
    }


def periodic(ref):
    """test_bc_operators/test_periodic_xy.f:94-190: nodes(i,j,k) =
    (i-1)+8(j-1)+100(k-1) on 8x10x3 and the expected ghost blocks."""
    path = os.path.join(ref, "src/test_files/test_bc_operators/test_periodic_xy.f")
    src = open(path).read()
    body = src[src.index("function test_apply_bc_on_nodes("):]
    body = body[:body.index("end function test_apply_bc_on_nodes")]
    targets = re.findall(r"test_nodes\((\d+):(\d+),(\d+):(\d+),:\)\s*=", body)
    blocks = _reshape_blocks(body, 3)
    assert len(targets) == len(blocks) == 4, (len(targets), len(blocks))
    out = []
    for (i0, i1, j0, j1), b in zip(targets, blocks):
        out.append({"i": [int(i0), int(i1)], "j": [int(j0), int(j1)], "shape": b["shape"],
                    "values": b["values"]})
    return {
        "source": "src/test_files/test_bc_operators/test_periodic_xy.f",
        "nx": 8, "ny": 10, "ne": 3,
        "nodes_formula": "(i-1)+8*(j-1)+100*(k-1), 1-based i,j,k",
        "expected_blocks": out,
    }


def wall(ref):
    """test_bc_operators/test_wall_xy_equilibrium.f: the known answers that
    the test constant set reproduces (capillarity parts of the wall flux at
    face (4,3) of get_nodes_for_flux_test :349-381, and the unit functions
    dwallInternalEnergy_dmd, temperature, dmddx, md_average :978-1060)."""
    path = os.path.join(ref, "src/test_files/test_bc_operators/test_wall_xy_equilibrium.f")
    src = open(path).read()
    body = src[src.index("subroutine get_nodes_for_flux_test"):]
    body = body[:body.index("end subroutine get_nodes_for_flux_test")]
    assign = []
    for m in re.finditer(r"nodes\((\d+):(\d+),(\d+),(\d+)\)\s*=\s*\[([^\]]*)\]", body):
        vals = [fnum(t) for t in re.findall(NUM, m.group(5))]
        assign.append({"i": [int(m.group(1)), int(m.group(2))], "j": int(m.group(3)),
                       "k": int(m.group(4)), "values": vals})
    m = re.search(r"nodes\((\d+),(\d+),(\d+)\)\s*=\s*(%s)" % NUM, body)
    assign.append({"i": [int(m.group(1)), int(m.group(1))], "j": int(m.group(2)),
                   "k": int(m.group(3)), "values": [fnum(m.group(4))]})
    fill = fnum(re.search(r"nodes\(i,j,k\)\s*=\s*(%s)" % NUM, body).group(1))

    def expect(fn_name):
        blk = src[src.index("function test_%s(" % fn_name):]
        blk = blk[:blk.index("end function test_%s" % fn_name)]
        lits = re.findall(r",\s*\$?\s*(%s)d0,\s*\$?\s*detailled" % NUM, blk.replace("\n", " "))
        return fnum(lits[-1] + "d0")

    def call_args(fn_name, callee):
        blk = src[src.index("function test_%s(" % fn_name):]
        blk = blk[:blk.index("end function test_%s" % fn_name)].replace("\n", " ")
        blk = re.sub(r"\s*\$\s*", " ", blk)
        start = re.search(r"[^\w]%s\(" % callee, blk[blk.index("result("):]).end()
        inner = blk[blk.index("result("):][start:]
        depth, out = 1, ""
        for ch in inner:
            depth += ch == "("
            depth -= ch == ")"
            if depth == 0:
                break
            out += ch
        return out

    dE_args = [fnum(t) for t in re.findall(NUM, call_args("dwallInternalEnergy_dmd",
                                                          "dwallInternalEnergy_dmd"))]
    T_args = [fnum(t) for t in re.findall(NUM, call_args("temperature", "temperature"))]
    dm = call_args("dmddx", "dmddx")
    dm_args = [fnum(t) for t in re.findall(NUM, dm)]
    av_args = [fnum(t) for t in re.findall(NUM, call_args("md_average", "md_average"))]
    return {
        "source": "src/test_files/test_bc_operators/test_wall_xy_equilibrium.f",
        "flux_nodes": {"shape": [5, 5, 4], "fill": fill, "assign": assign, "dx": 0.1, "dy": 0.2,
                       "face": [4, 3]},
        "flux_x_capillarity_momentum_x": expect("flux_x_capillarity_momentum_x"),
        "flux_x_capillarity_momentum_y": expect("flux_x_capillarity_momentum_y"),
        "dwallInternalEnergy_dmd": {"args": dE_args, "value": expect("dwallInternalEnergy_dmd")},
        "temperature": {"args": T_args, "value": expect("temperature")},
        "dmddx": {"args": dm_args, "grad_type": "sd_interior_type", "value": expect("dmddx")},
        "md_average": {"args": av_args, "value": expect("md_average")},
    }


def main():
    if len(sys.argv) != 2 or not os.path.isdir(os.path.join(sys.argv[1], "src")):
        sys.exit("usage: python tests/golden/make_golden.py <reference_root>")
    ref = sys.argv[1]
    out = {
        "mattsson_operators.json": mattsson(ref),
        "dim2d_fluxes.json": dim2d_fluxes(ref),
        "hedstrom_xy.json": hedstrom(ref),
        "periodic_xy.json": periodic(ref),
        "wall_xy_equilibrium.json": wall(ref),
    }
    for name, obj in out.items():
        with open(os.path.join(HERE, name), "w") as fh:
            json.dump(obj, fh, indent=1, sort_keys=True)
        print("wrote", name)


if __name__ == "__main__":
    main()
