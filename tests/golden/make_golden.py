"""Generate the golden fixtures in this folder from the reference's own tests.

Run in a container that holds the reference source tree (the fixtures it
writes are committed, so the tests never need the reference at run time):

    python tests/golden/make_golden.py /path/to/lfric_core

The reference is Fortran and cannot be compiled here, so nothing is
executed: the literal inputs and expected answers are read out of the pFUnit
test files (``*.pf``) as text, and where a test builds an input or an answer
with a short loop, that loop is restated below next to its citation.  The
mesh fixtures are read from the reference's UGRID netCDF test meshes.
"""
from __future__ import annotations

import ast
import json
import operator
import re
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
UT = "components/science/unit-test/kernel"

_KIND = re.compile(r"_(r_def|r_double|r_single|r_solver|i_def)\b")


def _eval_num(expr: str) -> float:
    """Evaluate one Fortran numeric literal expression (+ - * / only)."""
    expr = _KIND.sub("", expr.strip())
    expr = re.sub(r"real\((.*?),\s*\w+\)", r"(\1)", expr)
    ops = {ast.Add: operator.add, ast.Sub: operator.sub, ast.Mult: operator.mul,
           ast.Div: operator.truediv, ast.USub: operator.neg, ast.UAdd: operator.pos}

    def ev(node):
        if isinstance(node, ast.Expression):
            return ev(node.body)
        if isinstance(node, ast.Constant):
            return node.value
        if isinstance(node, ast.BinOp):
            return ops[type(node.op)](ev(node.left), ev(node.right))
        if isinstance(node, ast.UnaryOp):
            return ops[type(node.op)](ev(node.operand))
        raise ValueError(f"unsupported literal {expr!r}")

    return ev(ast.parse(expr, mode="eval"))


def _source(path: Path) -> str:
    """The test file with comments removed and continuation lines joined."""
    lines = []
    for line in path.read_text().splitlines():
        if line.lstrip().startswith("!"):
            continue
        lines.append(line.split("!")[0] if "!" in line and "'" not in line else line)
    return re.sub(r"&\s*\n\s*&?", " ", "\n".join(lines))


def array_literal(text: str, lhs_regex: str, occurrence: int = 0) -> list[float]:
    """Values of the array constructor assigned to a left-hand side."""
    pat = re.compile(lhs_regex + r"\s*=\s*(?:reshape\(\s*|real\(\s*)?\(/(.*?)/\)", re.S)
    found = pat.findall(text)
    if len(found) <= occurrence:
        raise KeyError(f"no array literal for {lhs_regex!r}")
    return [_eval_num(v) for v in found[occurrence].split(",")]


def scalar_literal(text: str, lhs_regex: str) -> float:
    m = re.search(lhs_regex + r"\s*=\s*([^\n]+)", text)
    if not m:
        raise KeyError(lhs_regex)
    return _eval_num(m.group(1))


def tol_literal(text: str, occurrence: int = 0) -> float:
    found = re.findall(r"tol\s*=\s*([0-9.eE+\-]+_r_\w+)", text)
    return _eval_num(found[occurrence])


def write(name: str, obj: dict) -> None:
    (HERE / name).write_text(json.dumps(obj, indent=1) + "\n")
    print("wrote", name)


def main(ref: Path) -> None:
    # ---------------------------------------------------------- tri-solve KAT
    p = ref / UT / "solver/sci_tri_solve_kernel_mod_test.pf"
    t = _source(p)
    x = array_literal(t, r"\bx")
    ans = array_literal(t, r"answer")
    write("tri_solve_kat.json", {
        "source": f"{UT}/solver/sci_tri_solve_kernel_mod_test.pf",
        "nlayers": len(x), "x": x, "answer": ans,
        "tri_0": scalar_literal(t, r"\bA0"), "tri_plus": scalar_literal(t, r"\bAP"),
        "tri_minus": scalar_literal(t, r"\bAM"),
        "reference_tol": tol_literal(t), "pinned_rel_tol": 1e-12,
    })

    p = ref / UT / "solver/sci_operator_tri_solve_kernel_mod_test.pf"
    t = _source(p)
    nz = 10
    a0, ap, am = (scalar_literal(t, r"\ba0"), scalar_literal(t, r"\bap"),
                  scalar_literal(t, r"\bam"))
    # The test fills tri(2,2,nz-1) with tri(1,1,k)=tri(2,2,k)=a0/2,
    # tri(1,2,k)=ap, tri(2,1,k)=am (operator_tri_solve_kernel_mod_test.pf:52-57)
    # and passes it where the kernel expects matrix(ncell=nz-1, 2, 2).
    tri = np.zeros((2, 2, nz - 1), order="F")
    tri[0, 0, :] = 0.5 * a0
    tri[1, 1, :] = 0.5 * a0
    tri[0, 1, :] = ap
    tri[1, 0, :] = am
    write("operator_tri_solve_kat.json", {
        "source": f"{UT}/solver/sci_operator_tri_solve_kernel_mod_test.pf",
        "nlayers": nz - 1, "x": array_literal(t, r"\bx"),
        "answer": array_literal(t, r"answer"),
        "a0": a0, "ap": ap, "am": am,
        "tri_as_passed_fortran_order": tri.ravel(order="F").tolist(),
        "reference_tol": tol_literal(t),
    })

    # ------------------------------------------------------- LMA kernels
    def dmat(t: str) -> np.ndarray:
        d = np.zeros((1, 4, 2))
        for r in range(4):
            d[0, r, :] = array_literal(t, rf"d\(1,{r + 1},:\)")
        return d

    for name, fname in [("matrix_vector", "matrix_vector_mod_test.pf"),
                        ("dg_matrix_vector", "dg_matrix_vector_mod_test.pf")]:
        t = _source(ref / UT / "algebra" / fname)
        d = dmat(t)
        x = array_literal(t, r"x\(:\)")
        write(f"{name}_kat.json", {
            "source": f"{UT}/algebra/{fname}",
            "matrix_fortran_order": d.ravel(order="F").tolist(),
            "shape": [1, 4, 2], "x": x, "map1": [1, 2, 3, 4], "map2": [1, 2],
            "answer": (d[0] @ np.array(x)).tolist(),
            "tol_r_double": tol_literal(t, 0), "tol_r_single": tol_literal(t, 1),
        })

    t = _source(ref / UT / "algebra/transpose_matrix_vector_mod_test.pf")
    d = dmat(t)
    x = array_literal(t, r"x\(:\)")
    write("transpose_matrix_vector_kat.json", {
        "source": f"{UT}/algebra/transpose_matrix_vector_mod_test.pf",
        "matrix_fortran_order": d.ravel(order="F").tolist(), "shape": [1, 4, 2],
        "x": x, "map1": [1, 2], "map2": [1, 2, 3, 4],
        "answer": (d[0].T @ np.array(x)).tolist(),
        "tol_r_double": tol_literal(t, 0), "tol_r_single": tol_literal(t, 1),
    })

    t = _source(ref / UT / "algebra/mm_diagonal_kernel_mod_test.pf")
    mm = np.zeros((2, 3, 3))
    for cell in range(2):
        for j in range(3):
            mm[cell, :, j] = array_literal(t, rf"mm\(cell,:,{j + 1}\)")
    write("mm_diagonal_kat.json", {
        "source": f"{UT}/algebra/mm_diagonal_kernel_mod_test.pf",
        "matrix_fortran_order": mm.ravel(order="F").tolist(), "shape": [2, 3, 3],
        "nlayers": 1, "map": [array_literal(t, r"map\(:,1\)"),
                              array_literal(t, r"map\(:,2\)")],
        "undf": 5, "answer": array_literal(t, r"answer"),
    })

    # ------------------------------------------------------- CMA (m3x3 data)
    t = _source(ref / UT / "columnwise_operators/columnwise_op_appinv_kernel_mod_test.pf")
    asserted = dict(re.findall(r"@assertEqual\((ndf|alpha|g_m|bw),\s*(\d+)\)", t))
    write("cma_m3x3_kat.json", {
        "source": [f"{UT}/columnwise_operators/columnwise_op_app_kernel_mod_test.pf",
                   f"{UT}/columnwise_operators/columnwise_op_appinv_kernel_mod_test.pf",
                   "components/science/unit-test/support/get_unit_test_m3x3_cma_data_mod.f90"],
        "space": "Wtheta->Wtheta", "nlayers": 3,
        "asserted": {k: int(v) for k, v in asserted.items()},
        "band_first_row": [0.0, 1.0 / 3.0, 1.0 / 6.0],
        "band_interior": [1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0],
        "band_last_row": [1.0 / 6.0, 1.0 / 3.0, 0.0],
        "tol": tol_literal(t),
    })

    # ------------------------------------------- CMA assembly and algebra
    cw = ref / UT / "columnwise_operators"

    def scalar(text, name):
        m = re.search(rf"\b{name}\s*=\s*([-+0-9.eE_a-z]+)", text)
        return _eval_num(m.group(1))

    asm = _source(cw / "columnwise_op_asm_kernel_mod_test.pf")
    stencil = re.search(r"reshape\(\s*\(/(.*?)/\)", asm).group(1)
    mul = _source(cw / "columnwise_op_mul_kernel_mod_test.pf")
    sadd = _source(cw / "columnwise_op_scaledadd_kernel_mod_test.pf")
    hm = _source(cw / "columnwise_op_asm_diag_hmht_kernel_mod_test.pf")
    m2v = _source(cw / "columnwise_op_asm_m2v_lumped_inv_kernel_mod_test.pf")
    m2v_stencil = re.search(r"reshape\(\s*\(/(.*?)/\)", m2v).group(1)
    write("cma_assembly_kat.json", {
        "source": [f"{UT}/columnwise_operators/columnwise_op_asm_kernel_mod_test.pf",
                   f"{UT}/columnwise_operators/columnwise_op_mul_kernel_mod_test.pf",
                   f"{UT}/columnwise_operators/columnwise_op_scaledadd_kernel_mod_test.pf",
                   f"{UT}/columnwise_operators/columnwise_op_asm_diag_hmht_kernel_mod_test.pf",
                   f"{UT}/columnwise_operators/columnwise_op_asm_m2v_lumped_inv_kernel_mod_test.pf",
                   "components/science/unit-test/support/get_unit_test_m3x3_cma_data_mod.f90"],
        "nlayers": int(scalar(asm, "nlayers")),
        # columnwise_op_asm: Wtheta->Wtheta, every cell's 2x2 stencil (Fortran order)
        "asm_stencil_fortran_order": [_eval_num(v) for v in stencil.split(",")],
        "asm_first_row": [_eval_num("1.0_r_solver/3.0_r_solver"),
                          _eval_num("1.0_r_solver/6.0_r_solver")],
        "asm_interior_row": [_eval_num("1.0_r_solver/6.0_r_solver"),
                             _eval_num("2.0_r_solver/3.0_r_solver"),
                             _eval_num("1.0_r_solver/6.0_r_solver")],
        "asm_last_row": [_eval_num("1.0_r_solver/6.0_r_solver"),
                         _eval_num("1.0_r_solver/3.0_r_solver")],
        # columnwise_op_mul: D (W3 <- Wtheta) bands (+1, -1), D^T bands (-1, +1)
        "mul_D_bands": [1.0, -1.0], "mul_DT_bands": [-1.0, 1.0],
        "mul_nlayers": int(scalar(mul, "nlayers")),
        # columnwise_op_scaledadd: C = mu M + nu DTD, M = I (W3), DTD bands (1, 2, 1)
        "scaledadd_mu": scalar(sadd, "mu"), "scaledadd_nu": scalar(sadd, "nu"),
        "scaledadd_DTD_bands": [1.0, 2.0, 1.0],
        # columnwise_op_asm_diag_hmht: Dh row (rho), diagonal M2h (sigma); answer sum rho^2/sigma
        "hmht_rho": [scalar(hm, rf"rho\({i}\)") for i in range(1, 5)],
        "hmht_sigma": [scalar(hm, rf"sigma\({i}\)") for i in range(1, 5)],
        # columnwise_op_asm_m2v_lumped_inv: W2v 2x2 stencil; ends 3, interior 3/2
        "m2v_stencil_fortran_order": [_eval_num(v) for v in m2v_stencil.split(",")],
        "m2v_end_rows": 3.0, "m2v_interior_rows": 1.5,
        "tol": tol_literal(asm),
    })

    # ------------------------------------------------ W2 intergrid KATs
    im2 = ref / UT / "inter_mesh"

    def int_list(text, lhs):
        m = re.search(lhs + r"\s*=\s*(?:reshape\(\s*)?\(/(.*?)/\)", text, re.S)
        return [int(v) for v in m.group(1).replace("&", " ").split(",")]

    def fields_w2(t, nl, nx, ny, map_f, undf_f, with_b, with_t):
        # the fine-field loop of restrict_w2{,h}_kernel_mod_test.pf: W of the
        # first column, E of the last, N of the first row, S of the last,
        # B (and T on the top layer) everywhere; -100 on faces not read
        f = np.zeros(undf_f)
        for k in range(nl):
            for x in range(1, nx + 1):
                for y in range(1, ny + 1):
                    c = x + nx * (y - 1)
                    m = map_f[c - 1]
                    if x == 1:
                        f[m[0] + k - 1] = y + k
                    elif x == nx:
                        f[m[2] + k - 1] = y + k + 1
                    else:
                        f[m[0] + k - 1] = f[m[2] + k - 1] = -100.0
                    if y == 1:
                        f[m[3] + k - 1] = x + k
                    elif y == ny:
                        f[m[1] + k - 1] = x + k + 1
                    else:
                        f[m[3] + k - 1] = f[m[1] + k - 1] = -100.0
                    if with_b:
                        f[m[4] + k - 1] = y + k
                        if with_t and k == nl - 1:
                            f[m[5] + k - 1] = x + k
        return f

    kat = {}
    for name, ndf, with_b in (("restrict_w2", 6, True), ("restrict_w2h", 4, False)):
        t = _source(im2 / f"{name}_kernel_mod_test.pf")
        nl, nx, ny = int(scalar(t, "nlayers")), int(scalar(t, "ncell_f_per_c_x")), \
            int(scalar(t, "ncell_f_per_c_y"))
        mf = np.array(int_list(t, "map_f")).reshape(nx * ny, ndf)
        mc = int_list(t, "map_c")
        undf_f, undf_c = int(scalar(t, "undf_f")), int(scalar(t, "undf_c"))
        fine = fields_w2(t, nl, nx, ny, mf, undf_f, with_b, with_b)
        ans = np.zeros(undf_c)
        for k in range(nl):   # the test's answer loop
            ans[mc[0] + k - 1] = 6 + 3 * k
            ans[mc[1] + k - 1] = 5 + 2 * k
            ans[mc[2] + k - 1] = 9 + 3 * k
            ans[mc[3] + k - 1] = 3 + 2 * k
            if with_b:
                ans[mc[4] + k - 1] = 12 + 6 * k
                if k == nl - 1:
                    ans[mc[5] + k - 1] = 9 + 6 * k
        kat[name] = dict(nlayers=nl, nx=nx, ny=ny, ndf=ndf, map_f=mf.tolist(), map_c=mc,
                         face_selector=2, fine=fine.tolist(), answer=ans.tolist())
    t = _source(im2 / "restrict_w2v_kernel_mod_test.pf")
    nl, nx, ny = 3, int(scalar(t, "ncell_f_per_c_x")), int(scalar(t, "ncell_f_per_c_y"))
    mf = np.array(int_list(t, "map_f")).reshape(nx * ny, 2)
    mc = int_list(t, "map_c")
    fine = np.zeros(nx * ny * (nl + 1))
    for k in range(nl):
        for x in range(1, nx + 1):
            for y in range(1, ny + 1):
                c = x + nx * (y - 1)
                fine[mf[c - 1][0] + k - 1] = y + k
                if k == nl - 1:
                    fine[mf[c - 1][1] + k - 1] = x + k
    ans = np.zeros(nl + 1)
    for k in range(nl):
        ans[mc[0] + k - 1] = 12 + 6 * k
        if k == nl - 1:
            ans[mc[1] + k - 1] = 9 + 6 * k
    kat["restrict_w2v"] = dict(nlayers=nl, nx=nx, ny=ny, ndf=2, map_f=mf.tolist(), map_c=mc,
                               fine=fine.tolist(), answer=ans.tolist())
    for name in ("prolong_w2", "weights_prolong_w2"):
        t = _source(im2 / f"{name}_kernel_mod_test.pf")
        nl, nx, ny = 3, int(scalar(t, "ncell_f_per_c_x")), int(scalar(t, "ncell_f_per_c_y"))
        mf = np.array(int_list(t, "map_f")).reshape(nx * ny, 6)
        mc = int_list(t, "map_c")
        undf_f, undf_c = int(scalar(t, "undf_f")), int(scalar(t, "undf_c"))
        coarse = np.zeros(undf_c)
        w = np.zeros(undf_f)
        ans = np.zeros(undf_f)
        for k in range(nl):   # the tests' coarse field, weights and answers
            coarse[mc[0] + k - 1] = 6 + 3 * k
            coarse[mc[1] + k - 1] = 5 + 2 * k
            coarse[mc[2] + k - 1] = 9 + 3 * k
            coarse[mc[3] + k - 1] = 3 + 2 * k
            coarse[mc[4] + k - 1] = 12 + 6 * k
            if k == nl - 1:
                coarse[mc[5] + k - 1] = 9 + 6 * k
            for x in range(1, nx + 1):
                for y in range(1, ny + 1):
                    m = mf[x + nx * (y - 1) - 1]
                    P = name == "prolong_w2"
                    if x == 1:
                        ans[m[0] + k - 1] = (2 + k) if P else 1.0 / ny
                        w[m[0] + k - 1] = 1.0 / ny
                        ans[m[2] + k - 1] = (2.5 + k) if P else 0.5
                        w[m[2] + k - 1] = 0.5
                    elif x == nx:
                        ans[m[2] + k - 1] = (3 + k) if P else 1.0 / ny
                        w[m[2] + k - 1] = 1.0 / ny
                    if y == 1:
                        ans[m[3] + k - 1] = (1.5 + k) if P else 1.0 / nx
                        w[m[3] + k - 1] = 1.0 / nx
                    elif y == ny:
                        ans[m[1] + k - 1] = (2.5 + k) if P else 1.0 / nx
                        w[m[1] + k - 1] = 1.0 / nx
                    else:
                        ans[m[1] + k - 1] = (13.0 / 6.0 + k) if P else 1.0 / 3.0
                        ans[m[3] + k - 1] = (11.0 / 6.0 + k) if P else 2.0 / 3.0
                        w[m[3] + k - 1] = 2.0 / 3.0
                        w[m[1] + k - 1] = 1.0 / 3.0
                    ans[m[4] + k - 1] = (2 + k) if P else 1.0 / (nx * ny)
                    w[m[4] + k - 1] = 1.0 / (nx * ny)
                    if k == nl - 1:
                        ans[m[5] + k - 1] = 3.5 if P else 1.0 / (nx * ny)
                        w[m[5] + k - 1] = 1.0 / (nx * ny)
        kat[name] = dict(nlayers=nl, nx=nx, ny=ny, ndf=6, map_f=mf.tolist(), map_c=mc,
                         coarse=coarse.tolist(), weights=w.tolist(), answer=ans.tolist())
    t = _source(im2 / "restrict_w2_kernel_mod_test.pf")
    write("w2_intergrid_kat.json", {
        "source": [f"{UT}/inter_mesh/{n}_kernel_mod_test.pf" for n in
                   ("restrict_w2", "restrict_w2h", "restrict_w2v", "prolong_w2",
                    "weights_prolong_w2")],
        "tol": tol_literal(t), **kat})

    # ------------------------------------------------------- intergrid KATs
    im = ref / UT / "inter_mesh"
    kats = {}
    t = _source(im / "restrict_scalar_unweighted_kernel_mod_test.pf")
    kats["restrict_scalar_unweighted"] = {"nlayers": 3, "fine": 1.0, "coarse": [1.0] * 3}
    t = _source(im / "prolong_scalar_unweighted_kernel_mod_test.pf")
    kats["prolong_scalar_unweighted"] = {"nlayers": 3, "coarse": 2.5, "fine": [2.5] * 3}
    t = _source(im / "restrict_mass_w3_kernel_mod_test.pf")
    kats["restrict_mass_w3"] = {"nlayers": 3, "fine": 1.0, "coarse": [4.0] * 3}
    t = _source(im / "restrict_scalar_weighted_kernel_mod_test.pf")
    kats["restrict_scalar_weighted"] = {
        "nlayers": 1, "fine": array_literal(t, r"fine_field\(:\)"),
        "weights": array_literal(t, r"weights\(:\)"), "coarse": [0.5]}
    t = _source(im / "prolong_scalar_weighted_kernel_mod_test.pf")
    kats["prolong_scalar_weighted"] = {
        "nlayers": 1, "coarse": 0.5, "weights": array_literal(t, r"weights\(:\)"),
        "fine": [_eval_num(v) for v in re.findall(
            r"@assertEqual\(\s*fine_field\(\d\),\s*([0-9.]+_r_def)", t)]}
    # cell_map(x, y) = x + (y-1)*ny and map_f(1,c) = 1 + (c-1)*nlayers for the
    # scalar tests (restrict_scalar_unweighted_kernel_mod_test.pf:61-68).
    kats["scalar_layout"] = {"cell_map_rule": "x + (y-1)*2", "map_fine_rule": "1 + (c-1)*nlayers"}

    t = _source(im / "restrict_w0_kernel_mod_test.pf")
    map_fine = np.array(array_literal(t, r"map_fine"), dtype=int).reshape(6, 8)  # [cell][df]
    map_coarse = [int(v) for v in array_literal(t, r"map_coarse")]
    nl, nx, ny = 3, 3, 2
    cell_map = np.zeros((nx, ny), dtype=int)             # cell_map(x, y)
    for y in range(1, ny + 1):
        for x in range(1, nx + 1):
            cell_map[x - 1, y - 1] = x + (2 - y) * nx      # restrict_w0_kernel_mod_test.pf
    SWB, SEB, NEB, NWB = 1, 2, 3, 4
    fine = 0.5 * np.arange(1, 49, dtype=float)            # fine_field(df) = 0.5*df
    for k in range(nl + 1):
        fine[map_fine[0, SWB - 1] + k - 1] = 1.0 + k
        fine[map_fine[2, SEB - 1] + k - 1] = 0.0 + k
        fine[map_fine[5, NEB - 1] + k - 1] = 6.0 + k
        fine[map_fine[3, NWB - 1] + k - 1] = 2.0 + k
    kats["restrict_w0"] = {
        "source": f"{UT}/inter_mesh/restrict_w0_kernel_mod_test.pf",
        "nlayers": nl, "nx": nx, "ny": ny, "cell_map_xy": cell_map.tolist(),
        "map_fine": map_fine.tolist(), "map_coarse": map_coarse,
        "fine": fine.tolist(), "coarse": array_literal(t, r"answer\(:\)"),
        "tol": tol_literal(t)}

    t = _source(im / "prolong_w0_kernel_mod_test.pf")
    coarse = array_literal(t, r"coarse_field\(:\)")
    ans = np.zeros(48)
    # The answer loop of prolong_w0_kernel_mod_test.pf: value + k on the
    # listed fine dofs, zero elsewhere.
    rows = re.findall(r"answer\(map_fine\((\w+),(\d)\)\+k\)\s*=\s*(-?[0-9.]+_r_def)", t)
    named = {"SWB": 1, "SEB": 2, "NEB": 3, "NWB": 4}
    for corner, cell, val in rows:
        for k in range(nl + 1):
            ans[map_fine[int(cell) - 1, named[corner] - 1] + k - 1] = _eval_num(val) + k
    kats["prolong_w0"] = {
        "source": f"{UT}/inter_mesh/prolong_w0_kernel_mod_test.pf",
        "nlayers": nl, "nx": nx, "ny": ny, "cell_map_xy": cell_map.tolist(),
        "map_fine": map_fine.tolist(), "map_coarse": map_coarse,
        "coarse": coarse, "fine": ans.tolist(), "tol": tol_literal(t)}
    write("intergrid_kat.json", kats)

    # ------------------------------------------------------- meshes
    from scipy.io import netcdf_file
    f = netcdf_file(str(ref / "infrastructure/unit-test/data/mesh_C32_MG.nc"), "r", mmap=False)
    mesh = {"source": "infrastructure/unit-test/data/mesh_C32_MG.nc", "meshes": {}, "maps": {}}
    for m in ("C4", "C8"):
        fn = f.variables[m + "_face_nodes"][:] - 1
        nxv = f.variables[m + "_node_x"][:]
        nyv = f.variables[m + "_node_y"][:]
        mesh["meshes"][m] = {
            "face_links_WSEN": (f.variables[m + "_face_links"][:] - 1).tolist(),
            "corner_lon_SW_SE_NE_NW": np.round(nxv[fn], 12).tolist(),
            "corner_lat_SW_SE_NE_NW": np.round(nyv[fn], 12).tolist(),
            "face_lon": np.round(f.variables[m + "_face_x"][:], 12).tolist(),
            "face_lat": np.round(f.variables[m + "_face_y"][:], 12).tolist(),
        }
    for a, b in (("C4", "C8"), ("C8", "C16")):
        mesh["maps"][f"{a}_{b}"] = (f.variables[f"{a}_{b}_map"][:] - 1).tolist()
    write("mesh_mg_kat.json", mesh)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the reference checkout>")
    main(Path(sys.argv[1]))
