"""deco_fsai_apply_static: the FSAI apply for callers that may not allocate device
memory while they run (their own pool owns the device after start-up, or their
time loop must not allocate).  Its intermediate vector is a fixed device array
inside the library instead of per-handle storage, so its result must equal the
allocating entry point's, call after call, and factors larger than that array
must be refused with a clear error.  Collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

STATIC_ROWS = 1 << 20


def _ptr(t):
    return C.c_void_p(t.data_ptr())


@pytest.fixture(scope="module")
def d():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import deco_b200
    deco_b200.default_context()
    return deco_b200


@pytest.mark.parametrize("precision", [64, 32])
def test_static_scratch_apply_matches_the_allocating_apply(d, precision):
    from deco_b200 import _lib, gen
    L = _lib.lib()
    s = gen.generate(gen.preset(1))
    A = d.CSR.from_system(s)
    F = d.FSAI({"tol_rel": 0.0, "tol_abs": 1e-16, "power": 1}, A, precision=precision)
    rng = np.random.default_rng(17)
    for _ in range(2):  # two calls in a row share (and overwrite) the library's array
        x = torch.from_numpy(rng.standard_normal(s.n)).cuda()
        want = F.apply(x)
        got = torch.full_like(x, float("nan"))
        before = L.deco_alloc_count()
        rc = L.deco_fsai_apply_static(d.default_context().h, F.h, _ptr(x), _ptr(got))
        assert rc == 0, L.deco_last_error().decode()
        assert L.deco_alloc_count() == before, "the static apply asked the library's allocator for memory"
        torch.cuda.synchronize()
        err = ((got - want).norm() / want.norm()).item()
        assert err < 1e-12, err


@pytest.mark.parametrize("precision", [64, 32])
def test_static_scratch_apply_without_padded_copies(d, precision):
    """With the slot-padded copies switched off (DECO_PADDED=0 at context creation)
    the static apply takes the CSR kernel at the heuristic width, while the
    allocating apply may take the cell-block kernel: the same products summed in
    another order, equal to rounding (1e-12 float64; 1e-6 for the float32 factor,
    whose float32 partial sums differ by a few float32 roundings)."""
    import os
    from deco_b200 import _lib, gen
    L = _lib.lib()
    os.environ["DECO_PADDED"] = "0"
    try:
        ctx = d.Context(0)
    finally:
        os.environ.pop("DECO_PADDED", None)
    s = gen.generate(gen.preset(1))
    A = d.CSR.from_system(s, ctx)
    F = d.FSAI({"tol_rel": 0.0, "tol_abs": 1e-16, "power": 1}, A, precision=precision)
    assert F.padded == (0, 0)
    rng = np.random.default_rng(23)
    for _ in range(2):
        x = torch.from_numpy(rng.standard_normal(s.n)).cuda()
        want = F.apply(x)
        got = torch.full_like(x, float("nan"))
        before = L.deco_alloc_count()
        rc = L.deco_fsai_apply_static(ctx.h, F.h, _ptr(x), _ptr(got))
        assert rc == 0, L.deco_last_error().decode()
        assert L.deco_alloc_count() == before
        ctx.sync()
        err = ((got - want).norm() / want.norm()).item()
        assert err < (1e-12 if precision == 64 else 1e-6), err


def test_static_scratch_apply_refuses_too_many_rows(d):
    from deco_b200 import _lib, gen
    L = _lib.lib()
    s = gen.grid(128, 128, 33, bs=2, seed=3)  # 1,081,344 rows > 2^20
    assert s.n > STATIC_ROWS
    A = d.CSR.from_system(s)
    F = d.FSAI({"tol_rel": 0.0, "tol_abs": 0.0, "power": 1}, A)
    x = torch.zeros(s.n, dtype=torch.float64, device="cuda")
    y = torch.zeros_like(x)
    rc = L.deco_fsai_apply_static(d.default_context().h, F.h, _ptr(x), _ptr(y))
    assert rc == -1
    assert "static scratch" in L.deco_last_error().decode()
