"""The C++ host layer (deco_b200/host/deco.hpp) through its driver, deco_cpr_gpu,
on parameter files in the reference's format and on its binary CSR files."""
import json
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import cpr_json, sol_json

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "deco_b200", "deco_cpr_gpu")


def write_params(tmp_path, io, prec, sol, hardware="GPU"):
    text = "{\n  // reference-style parameter file (comments are stripped)\n" + \
        '  "IO": ' + json.dumps(io) + ',\n  "sol": ' + json.dumps(sol) + ',\n  "prec": ' + json.dumps(prec) + \
        ',\n  "parallel": {"hardware": "' + hardware + '", "np": "1", "nranks": "1"}\n}\n'
    p = tmp_path / "param.json"
    p.write_text(text)
    return str(p)


def run(param, *extra):
    out = subprocess.run([DRIVER, param, *extra], capture_output=True, text=True, timeout=600)
    m = re.search(r"iteration count =\s+(\d+)", out.stdout)
    r = re.search(r"residual = ([0-9.e+-]+)", out.stdout)
    return out.returncode, (int(m.group(1)) if m else None), (float(r.group(1)) if r else None), out


@pytest.mark.gpu
def test_driver_synthetic_matches_oracle(tmp_path):
    from deco_b200 import gen
    from oracle import port
    prec = cpr_json(2)
    sol = sol_json()
    param = write_params(tmp_path, {"format": "synthetic", "preset": "1", "seed": "1234"}, prec, sol)
    rc, it, res, out = run(param)
    assert rc == 0, out.stderr
    s = gen.generate(gen.preset(1, 1234))
    ref_it = port.Cpr(prec, s.r, s.c, s.v, s.b).solve(sol)["iter"]
    assert abs(it - ref_it) <= max(1, 0.1 * ref_it) and res < 1e-8
    assert "Global precond" in out.stdout and "Local  precond" in out.stdout


@pytest.mark.gpu
def test_driver_reads_reference_binary_files(tmp_path):
    """IO/cpp_read.hpp:331-442 layout: int n, m, nz; r; c; v  and  int n; b."""
    from deco_b200 import gen
    s = gen.grid(10, 8, 5, bs=3, seed=4)
    fa, fb = tmp_path / "A.bin", tmp_path / "b.bin"
    with open(fa, "wb") as f:
        np.array([s.n, s.n, s.nnz], np.int32).tofile(f)
        s.r.tofile(f); s.c.tofile(f); s.v.tofile(f)
    with open(fb, "wb") as f:
        np.array([s.n], np.int32).tofile(f)
        s.b.tofile(f)
    io = {"file_A": str(fa), "file_b": str(fb), "format": "bin", "wfile_x": str(tmp_path / "x.bin")}
    param = write_params(tmp_path, io, cpr_json(3), sol_json("lgmres"))
    rc, it, res, out = run(param)
    assert rc == 0, out.stderr
    assert it > 0 and res < 1e-8
    x = np.fromfile(tmp_path / "x.bin", dtype=np.float64, offset=4)
    assert x.shape == (s.n,) and np.all(np.isfinite(x))
    rc32, it32, res32, out32 = run(param, "--precision", "32")
    assert rc32 == 0 and res32 < 1e-8, out32.stderr


@pytest.mark.gpu
def test_driver_rejects_cpu_only_preconditioners(tmp_path):
    prec = cpr_json(2)
    prec["prec_loc"] = {"type": "hypre_AMG", "tol_rel": "1e-4"}
    param = write_params(tmp_path, {"format": "synthetic", "preset": "1"}, prec, sol_json())
    rc, it, res, out = run(param)
    assert rc == 3 and "hypre" in out.stderr


@pytest.mark.gpu
def test_driver_adjoint_section(tmp_path):
    """The optional "adjoint" object: A^T lambda = dL/dx for L = sum_k w_k p(cell_k),
    with CPR on A^T, against the oracle's adjoint of the same seeded observations."""
    from deco_b200 import gen
    from oracle import adjoint
    prec, sol = cpr_json(2), sol_json(reltol=1e-10)
    io = {"format": "synthetic", "preset": "1", "seed": "1234"}
    text = json.dumps({"IO": io, "sol": sol, "prec": prec, "parallel": {"hardware": "GPU"},
                       "adjoint": {"observations": "12", "seed": "5",
                                   "wfile_lambda": str(tmp_path / "lambda.bin")}})
    param = tmp_path / "param.json"
    param.write_text(text)
    rc, it, res, out = run(str(param))
    assert rc == 0, out.stderr + out.stdout
    assert re.search(r"adjoint iteration count =\s+\d+", out.stdout)
    s = gen.generate(gen.preset(1, 1234))
    ncell = s.n // 2
    u = gen.uniform(5, 77, 24)
    g = np.zeros(s.n)
    for k in range(12):
        g[min(ncell - 1, int(u[2 * k] * ncell)) * 2] += u[2 * k + 1]
    raw = np.fromfile(tmp_path / "lambda.bin", dtype=np.uint8)
    assert int(np.frombuffer(raw[:4].tobytes(), np.int32)[0]) == s.n
    lam = np.frombuffer(raw[4:].tobytes(), np.float64)
    lam_ref = adjoint.adjoint(prec, sol, s.r, s.c, s.v, g, "port")["x"]
    assert np.linalg.norm(lam - lam_ref) / np.linalg.norm(lam_ref) < 1e-7


@pytest.mark.gpu
def test_driver_block_reorder(tmp_path):
    """prec.row_order / col_order "21" (adapter/csr2coo.cpp:18-86): a system stored
    saturation-first is reordered pressure-first by the driver and solves like the
    pressure-first original."""
    from deco_b200 import gen
    from oracle import port
    s = gen.grid(10, 8, 5, bs=2, seed=4)
    rows = np.repeat(np.arange(s.n), np.diff(s.r))
    swap = lambda i: i - i % 2 + (1 - i % 2)
    # scrambled copy: row i of it is original row swap(i), columns swapped within cells
    perm_rows = swap(np.arange(s.n))
    r2 = np.zeros(s.n + 1, np.int32)
    np.cumsum(np.diff(s.r)[perm_rows], out=r2[1:])
    c2, v2 = np.empty_like(s.c), np.empty_like(s.v)
    for i in range(s.n):
        a, e = s.r[perm_rows[i]], s.r[perm_rows[i] + 1]
        cc, vv = swap(s.c[a:e]), s.v[a:e]
        o = np.argsort(cc, kind="stable")
        c2[r2[i]:r2[i + 1]], v2[r2[i]:r2[i + 1]] = cc[o], vv[o]
    b2 = s.b[perm_rows]
    fa, fb = tmp_path / "A.bin", tmp_path / "b.bin"
    with open(fa, "wb") as f:
        np.array([s.n, s.n, s.nnz], np.int32).tofile(f)
        r2.tofile(f); c2.astype(np.int32).tofile(f); v2.tofile(f)
    with open(fb, "wb") as f:
        np.array([s.n], np.int32).tofile(f)
        b2.tofile(f)
    prec = dict(cpr_json(2), row_order="21", col_order="21")
    sol = sol_json()
    io = {"file_A": str(fa), "file_b": str(fb), "format": "bin", "wfile_x": str(tmp_path / "x.bin")}
    rc, it, res, out = run(write_params(tmp_path, io, prec, sol))
    assert rc == 0, out.stderr
    ref_it = port.Cpr(cpr_json(2), s.r, s.c, s.v, s.b).solve(sol)["iter"]
    assert abs(it - ref_it) <= max(1, 0.1 * ref_it) and res < 1e-8
    del rows


@pytest.mark.gpu
def test_driver_norne_parameters_restart_100(tmp_path):
    """The shipped Norne parameter file's settings (param_norne.json): bs 3 with the
    unknowns stored in 2-1-3 order (row_order / col_order "213"), quasiimpes_GE + DRS
    (e_dd 0.2) + CPD, global FSAI with tol_rel 0.2, rgmres with restart 100, itmax 100
    and reltol 1e-6, changed only in prec_loc (FSAI instead of hypre AMG, which stays on
    the CPU build) and IO (binary files of a seeded 40x40x20 three-phase system with 1 %
    fault connections instead of the Git-LFS sample).  Its one cycle runs past 64 basis
    columns; the iteration count is within 10% of the reference build's on the
    pressure-first system."""
    from deco_b200 import gen
    from oracle import ref
    p = gen.preset(2, 1234)
    p.nx, p.ny, p.nz = 40, 40, 20
    s = gen.generate(p)
    bs = 3
    # stored order: position q of every cell holds original unknown perm[q] (2-1-3 order),
    # which row_order / col_order "213" undo (adapter/csr2coo.cpp:18-86)
    perm = np.array([1, 0, 2])
    sw = lambda i: i - i % bs + perm[i % bs]
    rows_st = sw(np.arange(s.n))
    r2 = np.zeros(s.n + 1, np.int64)
    np.cumsum(np.diff(s.r)[rows_st], out=r2[1:])
    c2, v2 = np.empty_like(s.c), np.empty_like(s.v)
    inv = np.argsort(perm)
    swc = lambda i: i - i % bs + inv[i % bs]
    for i in range(s.n):
        a, e = s.r[rows_st[i]], s.r[rows_st[i] + 1]
        cc, vv = swc(s.c[a:e]), s.v[a:e]
        o = np.argsort(cc, kind="stable")
        c2[r2[i]:r2[i + 1]], v2[r2[i]:r2[i + 1]] = cc[o], vv[o]
    fa, fb = tmp_path / "A.bin", tmp_path / "b.bin"
    with open(fa, "wb") as f:
        np.array([s.n, s.n, s.nnz], np.int32).tofile(f)
        r2.astype(np.int32).tofile(f); c2.astype(np.int32).tofile(f); v2.tofile(f)
    with open(fb, "wb") as f:
        np.array([s.n], np.int32).tofile(f)
        s.b[rows_st].tofile(f)
    prec = {"type": "CPR", "verbosity": "0", "row_order": "213", "col_order": "213", "block_size": "3",
            "pressure_id": "0", "seq": "3", "weights": "quasiimpes_GE", "use_drs": "1",
            "drs": {"e_dd": "0.2", "e_ps": "0.0"}, "CPD": "1", "tol_zero": "0.0",
            "prec_glo": {"type": "FSAI", "input_file": "optional", "tol_rel": "0.2", "tol_abs": "1e-16",
                         "verbosity": "0", "power": "1", "block_size": "1"},
            "prec_loc": {"type": "FSAI", "tol_rel": "1e-4", "tol_abs": "1e-16", "power": "1", "block_size": "1"}}
    sol = {"type": "rgmres", "input_file": "optional", "reltol": "1e-6", "restart": "100", "itmax": "100",
           "verbosity": "1"}
    io = {"file_A": str(fa), "file_b": str(fb), "header": "1", "format": "bin", "write": "0",
          "wfile_x": str(tmp_path / "x.bin")}
    rc, it, res, out = run(write_params(tmp_path, io, prec, sol))
    assert rc == 0, out.stderr
    ref_prec = {k: v for k, v in prec.items() if k not in ("row_order", "col_order")}
    R = ref.Cpr({"prec": ref_prec}, s.r, s.c, s.v, s.b)
    rres = R.solve(dict(sol, verbosity="0"))
    assert rres["iter"] > 64 and rres["flag"] == 0
    assert abs(it - rres["iter"]) <= max(1, 0.1 * rres["iter"]), (it, rres["iter"])
    assert res < 1e-6
    # x is written in the reordered (pressure-first) order, that of the reference's system
    x = np.fromfile(tmp_path / "x.bin", dtype=np.float64, offset=4)
    assert np.linalg.norm(x - rres["x"]) / np.linalg.norm(rres["x"]) < 1e-4
