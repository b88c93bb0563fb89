"""CPU checks of the C ABI boundary and of host-side logic (no GPU calls)."""

import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "pfb200.h")


def _declared():
    hdr = open(HEADER).read()
    return set(re.findall(r"^(?:int|const char \*)\s*(pfb_\w+)\(", hdr, re.M))


def test_library_loads_and_exports_every_declared_symbol():
    from pyfourier_b200 import _lib

    L = _lib.load()
    declared = _declared()
    assert declared == set(_lib.EXPORTS)
    for name in declared:
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (pfb_\w+)", out))
    assert declared <= exported
    assert L.pfb_version().startswith(b"pyfourier_b200")


def test_status_mapping_without_gpu():
    """Argument validation happens before any CUDA call and maps to ValueError."""
    from pyfourier_b200 import _lib

    L = _lib.load()
    out = ctypes.c_void_p()
    st = L.pfb_plan_create(None, 4, 1, None, 1, None, None, None, None, None, None, 0, None,
                           ctypes.byref(out))
    assert st == _lib.PFB_ERR_INVALID
    assert b"ndim" in L.pfb_last_error()
    with pytest.raises(ValueError):
        _lib.check(st)
    st = L.pfb_gram_create(2, None, None, 4, 1, 1, None, 0, None, ctypes.byref(out))
    assert st == _lib.PFB_ERR_INVALID
    # NULL handles are rejected, destroy(NULL) is a no-op
    assert L.pfb_plan_destroy(None) == 0
    assert L.pfb_gram_destroy(None) == 0
    info = _lib.PlanInfoT()
    assert L.pfb_plan_info(None, ctypes.byref(info)) == _lib.PFB_ERR_INVALID
    assert L.pfb_plan_check(None, None) == _lib.PFB_ERR_INVALID


def test_apply_struct_layout_matches_header(tmp_path):
    """The ctypes mirrors have the size and field offsets the C compiler gives the
    header's structs."""
    import shutil

    from pyfourier_b200 import _lib

    # int64 + 2*int32 + 4 pointers + 2*int32 = 8 + 8 + 32 + 8 = 56 bytes on LP64
    assert ctypes.sizeof(_lib.ApplyT) == 56
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    lines = []
    for cname, mirror in (("pfb_apply_t", _lib.ApplyT), ("pfb_plan_info_t", _lib.PlanInfoT)):
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in mirror._fields_:
            lines.append(f'printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    src = tmp_path / "layout.c"
    src.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "pfb200.h"\nint main(void) {\n'
                   + "\n".join(lines) + "\nreturn 0;\n}\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.join(root, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l}
    for cname, mirror in (("pfb_apply_t", _lib.ApplyT), ("pfb_plan_info_t", _lib.PlanInfoT)):
        assert got[(cname, "size")] == ctypes.sizeof(mirror), cname
        for f, _ in mirror._fields_:
            assert got[(cname, f)] == getattr(mirror, f).offset, (cname, f)


def test_host_parameter_math_matches_oracle():
    from oracle import nufft_oracle as orc
    from pyfourier_b200 import _plan

    for w, o in [((4, 4), (2.0, 2.0)), ((4, 4, 4), (1.25,) * 3), ((6, 3), (1.25, 1.5))]:
        np.testing.assert_array_equal(_plan.beta_f32(w, o), orc.beta_f32(w, o))
    for n, o in [((128, 128), (2.0, 2.0)), ((200, 200, 200), (1.25,) * 3), ((192, 220), (1.25, 1.1))]:
        assert _plan.oversamp_shape(n, o) == orc.oversamp_shape(n, o)


def test_frames_from_coord_shapes():
    from pyfourier_b200._plan import _frames_from_coord

    flat, offs, ro, ds = _frames_from_coord(np.zeros((3, 5, 7, 2), np.float32))
    assert flat.shape == (105, 2) and list(offs) == [0, 35, 70, 105] and ro == 7 and ds == (5, 7)
    flat, offs, ro, ds = _frames_from_coord(np.zeros((7, 3), np.float32))
    assert flat.shape == (7, 3) and list(offs) == [0, 7] and ds == (7,)
    flat, offs, ro, ds = _frames_from_coord([np.zeros((2, 8, 2), np.float32), np.zeros((5, 8, 2), np.float32)])
    assert flat.shape == (56, 2) and list(offs) == [0, 16, 56] and ro == 8 and ds is None


def test_b0_basis_fp64_matches_oracle():
    from oracle import nufft_oracle as orc
    from pyfourier_b200._b0 import mri_exp_approx

    rng = np.random.default_rng(0)
    zmap = 100 * rng.standard_normal((16, 16))
    t = 5e-3 * np.arange(64) / 64
    b1, c1 = mri_exp_approx(zmap, t, 6, 40)
    b2, c2 = orc.mri_exp_approx(zmap, t, 6, 40)
    np.testing.assert_allclose(b1, b2, rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(c1, c2, rtol=1e-12)


@pytest.mark.parametrize("kind", ["planes", "basis", "field_map", "line_mask"])
def test_dense_gram_kernel_matches_oracle(kind):
    """The Cartesian Gram kernel built on the host (torch on CPU) equals the
    oracle's restatement of src/pyfourier/_gram/_plan.py."""
    import torch

    from oracle import nufft_oracle as orc
    from pyfourier_b200._cgram import _dense_kernel

    rng = np.random.default_rng(1)
    N = (16, 20)
    m = (rng.random((4, *N)) < 0.3).astype(np.float32)
    B = np.linalg.qr(rng.standard_normal((4, 3)) + 1j * rng.standard_normal((4, 3)))[0].astype(np.complex64)
    kw = {}
    if kind == "basis":
        kw = dict(basis=B)
    elif kind == "line_mask":
        m, kw = m[0, :, 0], dict(basis=B[:1])  # (ny,) -> (1, ny, 1), broadcast along x
    elif kind == "field_map":
        yy, xx = np.mgrid[:N[0], :N[1]] / N[0] - 0.5
        kw = dict(zmap=100 * np.exp(-((xx - 0.1) ** 2 + yy ** 2) / 0.05) - 50,
                  T=1e-4 * np.broadcast_to(np.arange(N[1]), N), L=6)
    o = orc.plan_gram(m, N, **kw)
    v, zs, lowrank = _dense_kernel(torch.as_tensor(m), N, kw.get("basis"), kw.get("zmap"), kw.get("T"),
                                   kw.get("L", 6), (40, 40))
    assert lowrank == o.islowrank and tuple(v.shape) == o.value.shape
    np.testing.assert_allclose(v.numpy(), o.value, rtol=0, atol=1e-6 * np.abs(o.value).max())
    if kind == "field_map":
        np.testing.assert_allclose(zs.numpy(), o.zmap_s_kernel, rtol=0, atol=1e-6)
    else:
        assert zs is None


@pytest.mark.parametrize("ndim", [2, 3])
def test_grog_tables_and_offsets_match_oracle(ndim):
    """GROG host math (torch on CPU): operators, fractional-power table and offset
    lookup equal the oracle's restatement of src/pyfourier/_preinterp/_grog.py."""
    import torch

    from oracle import nufft_oracle as orc
    from pyfourier_b200 import _preinterp as P
    from tests.test_oracle import shift_invariant_kspace

    rng = np.random.default_rng(2)
    _, cal = shift_invariant_kspace(rng, 5, ndim)
    cal = cal + 0.05 * (rng.standard_normal(cal.shape) + 1j * rng.standard_normal(cal.shape))
    if ndim == 2:
        cal = np.stack([cal, 0.5 * cal[:, ::-1]], 1)  # two calibration slices
    cal = cal / np.linalg.norm(cal)
    ops_o = orc.grog_operators(cal, ndim, 0.01)
    ops_p = P._operators(torch.as_tensor(cal), ndim, 0.01)
    for a, b in zip(ops_p, ops_o):
        np.testing.assert_allclose(a.numpy(), b, rtol=0, atol=1e-10 * np.abs(b).max())
    t_o = orc.grog_table(ops_o, 11)
    t_p = P._table(ops_p, 11).numpy()
    assert t_p.shape == t_o.shape
    np.testing.assert_allclose(t_p, t_o, rtol=0, atol=1e-9 * np.abs(t_o).max())
    coord = ((rng.random((3, 50, ndim)) - 0.5) * 20).astype(np.float32)
    coord[0, :4] = np.array([0.5, -0.5, 1.5, 2.5], np.float32)[:, None]  # ties round half to even
    i_o, l_o = orc.grog_lut(coord, 11)
    i_p, l_p = P._lut(torch.as_tensor(coord), 11)
    np.testing.assert_array_equal(i_p.numpy(), i_o)
    np.testing.assert_array_equal(l_p.numpy(), l_o)
    assert l_o.min() >= 0 and l_o.max() < 11 ** ndim
