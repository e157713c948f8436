"""The C ABI library: loads without a GPU, exports every symbol include/deco_b200.h
declares, and the Python binding declares exactly those symbols."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions(name):
    text = open(os.path.join(ROOT, "include", name)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(deco_\w+)\s*\(", text)) - {"deco_cpr_params", "deco_sol_params"})


@pytest.fixture(scope="module")
def gpu_lib():
    from deco_b200 import build
    build.build_gpu()
    from deco_b200 import _lib
    return _lib


def test_library_exports_every_declared_symbol(gpu_lib):
    L = C.CDLL(gpu_lib.LIB_PATH)
    names = header_functions("deco_b200.h")
    assert len(names) > 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_binding_covers_the_header(gpu_lib):
    assert sorted(gpu_lib.SIGNATURES) == header_functions("deco_b200.h")


def test_generator_library_exports(gpu_lib):
    from deco_b200 import gen
    L = gen.lib()
    for n in header_functions("deco_gen.h"):
        assert hasattr(L, n), n


def test_version_and_error_string(gpu_lib):
    L = gpu_lib.lib()
    assert L.deco_version().decode().startswith("deco_b200")
    assert isinstance(L.deco_last_error(), bytes)
    assert L.deco_launch_count() >= 0


def test_no_device_is_an_error_status_not_a_crash(gpu_lib):
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    L = gpu_lib.lib()
    h = C.c_void_p()
    rc = L.deco_ctx_create(0, None, C.byref(h))
    assert rc != 0
    assert L.deco_last_error().decode()
    import deco_b200
    with pytest.raises(deco_b200.DecoError):
        deco_b200.Context(0)


def test_null_arguments_are_rejected(gpu_lib):
    L = gpu_lib.lib()
    assert L.deco_csr_info(None, None, None, None) == -1
    assert L.deco_fsai_info(None, None, None, None) == -1
    assert L.deco_cpr_timings(None, None) == -1
    assert L.deco_ctx_sync(None) == -1
    assert L.deco_csr_set_subwarp(None, 3) == -1
    assert "NULL" in L.deco_last_error().decode() or L.deco_last_error()


def test_params_mapping_follows_reference_keys():
    import deco_b200 as d
    text = """{
      // comment lines and /* blocks */ are stripped first (IO/ptree.hpp:27-84)
      "sol": {"type": "lgmres", "reltol": "1e-6", "restart": "30", "itmax": "100", "verbosity": "1"},
      "prec": {"block_size": "3", "pressure_id": "0", "seq": "3", "weights": "quasiimpes_GE",
               "use_drs": "1", "drs": {"e_dd": "0.2", "e_ps": "0.0"}, "CPD": "1", "tol_zero": "0.0",
               /* global */ "prec_glo": {"type": "FSAI", "tol_rel": "0.2", "tol_abs": "1e-16", "power": "1"},
               "prec_loc": {"type": "FSAI", "tol_rel": "1e-4", "tol_abs": "1e-16", "power": "2"}}
    }"""
    p = d.load_params(text)
    cp = d.cpr_params(p["prec"], 32)
    assert (cp.block_size, cp.seq, cp.weights, cp.use_drs, cp.cpd, cp.loc_power, cp.precision) == (3, 3, 2, 1, 1, 2, 32)
    assert cp.glo_tol_rel == 0.2 and cp.loc_tol_rel == 1e-4
    sp = d.sol_params(p["sol"])
    assert (sp.type, sp.restart, sp.itmax, sp.verbosity) == (1, 30, 100, 1) and sp.reltol == 1e-6
    with pytest.raises(d.DecoError):
        d.sol_params({"type": "pcg", "reltol": "1", "restart": "1", "itmax": "1"})


def test_handles_hold_no_reference_cycles():
    """Borrowed views (the pressure matrix, the FSAI factors) point at their owner,
    never the other way, so dropping a CPR frees it by reference counting alone."""
    import inspect
    import deco_b200
    src = inspect.getsource(deco_b200.CPR.__init__)
    assert "self.Ap" not in src and "_owner = self" not in src
