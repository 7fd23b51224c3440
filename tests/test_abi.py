"""The C-ABI library loads, exports every entry point of include/mgpcg_b200.h
and validates plans on the host (no GPU needed)."""
import ctypes

import pytest

import mg_lib


def test_library_exports_every_header_symbol():
    lib = mg_lib.load()
    names = mg_lib.header_entry_points()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert lib.mg_version() >= 10000


def _desc(dim=3, res=(64, 64, 64), levels=4, storage=0):
    d = mg_lib.PlanDesc()
    d.dim = dim
    for k in range(3):
        d.res[k] = res[k] if k < len(res) else 1
    d.levels = levels
    d.pre_post = 2
    d.bottom = 50
    d.storage = storage
    return d


def _create(d):
    lib = mg_lib.load()
    p = ctypes.c_void_p()
    rc = lib.mg_plan_create(ctypes.byref(d), ctypes.byref(p))
    return rc, p


@pytest.mark.parametrize("dim,res,levels", [(2, (128, 128), 4), (3, (64, 64, 64), 5), (2, (96, 64), 4)])
def test_plan_layout(dim, res, levels):
    lib = mg_lib.load()
    rc, p = _create(_desc(dim, res, levels))
    assert rc == 0
    try:
        ws = lib.mg_plan_workspace_bytes(p)
        spans = []
        for f in range(9):
            for l in range(levels):
                ncomp = dim if f == mg_lib.FIELD_AX else 1
                for c in range(ncomp):
                    off, nb = ctypes.c_int64(), ctypes.c_int64()
                    r = lib.mg_plan_field(p, f, l, c, ctypes.byref(off), ctypes.byref(nb))
                    if f in (mg_lib.FIELD_B, mg_lib.FIELD_X, mg_lib.FIELD_P, mg_lib.FIELD_AP) and l > 0:
                        assert r == mg_lib.MG_E_BADARG
                        continue
                    assert r == 0
                    assert off.value % 16 == 0 and 0 <= off.value and off.value + nb.value <= ws
                    cells = 1
                    for v in res:
                        cells *= v >> l
                    esz = {mg_lib.FIELD_TYPE: 1}.get(f, 4)
                    assert nb.value == cells * esz
                    spans.append((off.value, off.value + nb.value))
        spans.sort()
        for a, b in zip(spans, spans[1:]):
            assert a[1] <= b[0], "fields overlap"
    finally:
        lib.mg_plan_destroy(p)


@pytest.mark.parametrize("kw", [dict(dim=4), dict(levels=0), dict(levels=13), dict(res=(100, 64, 64), levels=4),
                                dict(storage=7)])
def test_plan_rejects_bad_descriptions(kw):
    args = dict(dim=3, res=(64, 64, 64), levels=4, storage=0)
    args.update(kw)
    rc, p = _create(_desc(**args))
    assert rc == mg_lib.MG_E_BADARG
    assert "bad argument" in mg_lib.last_error()


def test_unbound_plan_is_refused():
    lib = mg_lib.load()
    rc, p = _create(_desc())
    assert rc == 0
    try:
        assert lib.mg_initialize(p, None) == mg_lib.MG_E_UNBOUND
        assert lib.mg_v_cycle(p, None) == mg_lib.MG_E_UNBOUND
        assert lib.mg_plan_bind(p, ctypes.c_void_p(1234)) == mg_lib.MG_E_BADARG  # misaligned
    finally:
        lib.mg_plan_destroy(p)


def test_launch_shape_choices_need_a_prepared_plan():
    """mg_plan_split / mg_plan_grid / mg_plan_steps read 0 (no streamed levels)
    and refuse to force a choice before prepare, and refuse null pointers."""
    lib = mg_lib.load()
    rc, p = _create(_desc())
    assert rc == 0
    try:
        bits = ctypes.c_uint32(0)
        streamed = ctypes.c_int32(-1)
        assert lib.mg_plan_split(p, 0, ctypes.byref(bits), ctypes.byref(streamed)) == 0
        assert (bits.value, streamed.value) == (0, 0)
        for fn in (lib.mg_plan_grid, lib.mg_plan_steps):
            bits.value = 0
            assert fn(p, 0, ctypes.byref(bits)) == 0 and bits.value == 0
            bits.value = 1
            assert fn(p, 1, ctypes.byref(bits)) == mg_lib.MG_E_BADARG
            assert "no fused V-cycle" in mg_lib.last_error()
            assert fn(p, 0, None) == mg_lib.MG_E_BADARG
            assert fn(None, 0, ctypes.byref(bits)) == mg_lib.MG_E_BADARG
        bits.value = 1
        assert lib.mg_plan_split(p, 1, ctypes.byref(bits), None) == mg_lib.MG_E_BADARG
    finally:
        lib.mg_plan_destroy(p)


def test_static_reduce_refuses_bad_arguments_before_any_cuda_call():
    """mg_reduce_static checks its pointers, its cell count and its scratch
    limit on the host, before it touches a device."""
    lib = mg_lib.load()
    p = ctypes.c_void_p(256)  # never dereferenced: every call below is refused first
    assert lib.mg_reduce_static(None, p, p, 16, p, None) == mg_lib.MG_E_BADARG
    assert "null pointer" in mg_lib.last_error()
    assert lib.mg_reduce_static(p, None, p, 16, p, None) == mg_lib.MG_E_BADARG
    assert lib.mg_reduce_static(p, p, None, 16, p, None) == mg_lib.MG_E_BADARG
    assert lib.mg_reduce_static(p, p, p, 16, None, None) == mg_lib.MG_E_BADARG
    assert lib.mg_reduce_static(p, p, p, -1, p, None) == mg_lib.MG_E_BADARG
    assert "negative cell count" in mg_lib.last_error()
    assert lib.mg_reduce_static(p, p, p, 33_554_433, p, None) == mg_lib.MG_E_TOO_BIG
    assert "static scratch limit" in mg_lib.last_error()


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    """Without the built library the product path raises; nothing falls back
    to a CPU or PyTorch implementation."""
    import mg_lib
    monkeypatch.setattr(mg_lib, "_lib", None)
    monkeypatch.setattr(mg_lib, "LIB_PATH", str(tmp_path / "libmgpcg_b200.so"))
    with pytest.raises(ImportError, match="no fallback"):
        mg_lib.load()
    from mgpcg import MGPCGPoissonSolver
    with pytest.raises(ImportError, match="no fallback"):
        MGPCGPoissonSolver(2, (64, 64), 3, 2, 50)
