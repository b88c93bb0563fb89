"""Generate golden vectors from the reference's own Numba CPU kernels.

Run where the pyfourier reference source tree is available, naming its
``src`` directory (the one holding the ``pyfourier`` package):

    PYFOURIER_REF_SRC=<reference checkout>/src python tests/golden/make_golden.py

The reference package cannot be imported as shipped on a GPU-less host
(``detect_gpu_backend`` leaves ``gpu_backend`` unbound, and
``importlib.metadata.version`` needs an installed distribution).  The shim
below therefore loads only the kernel modules by file path, under stub parent
packages whose ``_utils`` exposes ``detect_gpu_backend() -> (False, None)``.
Nothing in the reference tree is modified.

Kernels exercised (paths inside the pyfourier project):
  _subroutines/_grid/_plan.py: _kaiser_bessel_kernel, _get_kernel_scaling,
      _prepare_interpolator_nb
  _subroutines/_grid/_noncart2cart/_{1,2,3}D[_subspace].py: _grid_nb
  _subroutines/_grid/_cart2noncart/_{1,2,3}D[_subspace].py: _degrid_nb
  _subroutines/_mask/_dense2sparse/_{2,3}D[_subspace].py: _mask_nb
  _subroutines/_mask/_sparse2dense/_{2,3}D[_subspace].py: _zerofill_nb

The inputs are seeded; coordinates are scaled onto the oversampled grid with
the float32 arithmetic of _subroutines/_traj.py:57-65 before the table build,
exactly as oracle/nufft_oracle.py does.  Output: tests/golden/kernels.npz.
"""

import importlib.util
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SRC = os.environ.get("PYFOURIER_REF_SRC", "")
os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/pyfourier_golden_numba_cache")


def _stub_package(name, path=None):
    mod = types.ModuleType(name)
    mod.__path__ = [path] if path else []
    sys.modules[name] = mod
    return mod


def load_reference_kernels():
    if not REF_SRC or not os.path.isdir(os.path.join(REF_SRC, "pyfourier")):
        raise SystemExit("set PYFOURIER_REF_SRC to the reference's src directory (holding the pyfourier package)")
    root = os.path.join(REF_SRC, "pyfourier")
    _stub_package("pyfourier", root)
    sub = _stub_package("pyfourier._subroutines", os.path.join(root, "_subroutines"))
    utils = types.ModuleType("pyfourier._subroutines._utils")
    utils.detect_gpu_backend = lambda: (False, None)
    sys.modules["pyfourier._subroutines._utils"] = utils
    sub._utils = utils
    _stub_package("pyfourier._subroutines._grid", os.path.join(root, "_subroutines", "_grid"))
    for d in ("_noncart2cart", "_cart2noncart"):
        _stub_package(
            "pyfourier._subroutines._grid." + d, os.path.join(root, "_subroutines", "_grid", d)
        )
    _stub_package("pyfourier._subroutines._mask", os.path.join(root, "_subroutines", "_mask"))
    for d in ("_dense2sparse", "_sparse2dense"):
        _stub_package(
            "pyfourier._subroutines._mask." + d, os.path.join(root, "_subroutines", "_mask", d)
        )

    def load(modname, relpath):
        spec = importlib.util.spec_from_file_location(modname, os.path.join(root, relpath))
        mod = importlib.util.module_from_spec(spec)
        sys.modules[modname] = mod
        spec.loader.exec_module(mod)
        return mod

    k = {"plan": load("pyfourier._subroutines._grid._plan", "_subroutines/_grid/_plan.py")}
    for d in (1, 2, 3):
        for sfx in ("", "_subspace"):
            k[f"grid{d}{sfx}"] = load(
                f"pyfourier._subroutines._grid._noncart2cart._{d}D{sfx}",
                f"_subroutines/_grid/_noncart2cart/_{d}D{sfx}.py",
            )._grid["cpu"][True]
            k[f"degrid{d}{sfx}"] = load(
                f"pyfourier._subroutines._grid._cart2noncart._{d}D{sfx}",
                f"_subroutines/_grid/_cart2noncart/_{d}D{sfx}.py",
            )._degrid["cpu"]
    for d in (2, 3):
        for sfx in ("", "_subspace"):
            k[f"mask{d}{sfx}"] = load(
                f"pyfourier._subroutines._mask._dense2sparse._{d}D{sfx}",
                f"_subroutines/_mask/_dense2sparse/_{d}D{sfx}.py",
            )._mask["cpu"]
            k[f"zerofill{d}{sfx}"] = load(
                f"pyfourier._subroutines._mask._sparse2dense._{d}D{sfx}",
                f"_subroutines/_mask/_sparse2dense/_{d}D{sfx}.py",
            )._zerofill["cpu"][True]
    return k


def scale_coord_f32(coord, shape, oversamp):
    """Float32 restatement of _subroutines/_traj.py:57-65 (axes in (x, y, z) order)."""
    out = np.array(coord, dtype=np.float32, copy=True)
    for i in range(coord.shape[-1]):
        n_os = np.ceil(np.float32(oversamp[i]) * np.float32(shape[i]))
        s = np.float32(n_os / np.float32(shape[i]))
        shift = np.float32(n_os // 2)
        out[..., i] = out[..., i] * s
        out[..., i] = out[..., i] + shift
    return out


def beta_f32(width, oversamp):
    """_nufft/_plan.py:128 with int16 width and float32 oversampling."""
    w = np.asarray(width, dtype=np.int16)
    o = np.asarray(oversamp, dtype=np.float32)
    return (np.pi * (((w / o) * (o - 0.5)) ** 2 - 0.8) ** 0.5).astype(np.float32)


def build_tables(k, c_os, os_shape_zyx, width_zyx, beta_zyx):
    """Interpolator tables exactly as _grid/_plan.py:14-91 lays them out (z, y, x)."""
    nframes, npts, ndim = c_os.shape
    flat = c_os.reshape(nframes * npts, ndim)
    idx, val = [], []
    for ax_xyz in range(ndim):
        ax_zyx = ndim - 1 - ax_xyz
        w = int(width_zyx[ax_zyx])
        v = np.zeros((nframes * npts, w), np.float32)
        i = np.zeros((nframes * npts, w), np.int32)
        k["plan"]._prepare_interpolator_nb(
            v, i, np.ascontiguousarray(flat[:, ax_xyz]), w, float(beta_zyx[ax_zyx]),
            int(os_shape_zyx[ax_zyx]),
        )
        idx.append(i.reshape(nframes, npts, w))
        val.append(v.reshape(nframes, npts, w))
    return tuple(idx[::-1]), tuple(val[::-1])


def main():
    k = load_reference_kernels()
    rng = np.random.default_rng(20240607)
    out = {}

    # 1. KB kernel samples and kernel scaling
    xs = np.concatenate([np.linspace(-1.05, 1.05, 211), [-1.0, 1.0, 0.0, 0.999999, -0.5]])
    betas = np.array([2.34, 4.5, 6.9966590477, 8.9961522936, 13.9], np.float64)
    kb = np.array([[k["plan"]._kaiser_bessel_kernel(float(x), float(b)) for x in xs] for b in betas])
    out["kb_x"], out["kb_beta"], out["kb_val"] = xs, betas, kb
    scal_cases = [((4, 4), (2.0, 2.0)), ((4, 4, 4), (1.25,) * 3), ((4, 4), (1.25, 1.25)),
                  ((6, 6), (1.25, 1.25)), ((3, 5), (1.5, 2.0)), ((2,), (2.0,)), ((8, 7, 6), (1.25, 1.5, 2.0))]
    sc_w, sc_b, sc_v = [], [], []
    for w, o in scal_cases:
        b = beta_f32(w, o)
        s = k["plan"]._get_kernel_scaling(list(b.astype(np.float64)), list(w))
        sc_w.append(list(w) + [0] * (3 - len(w)))
        sc_b.append(list(b.astype(np.float64)) + [0.0] * (3 - len(w)))
        sc_v.append(float(s))
    out["scal_width"], out["scal_beta"], out["scal_value"] = (
        np.array(sc_w, np.int32), np.array(sc_b), np.array(sc_v))

    # 2. Tables for edge-case coordinates, several widths
    N = 32
    edge = np.array([-16.0, -15.5, -8.25, -1e-7, 0.0, 1e-7, 0.5, 3.0, 7.75, 15.5, 15.999, 16.0,
                     -17.3, 21.0, 9.0001, -0.4999], np.float32)
    for w in (2, 3, 4, 5, 6, 7, 8):
        for osf in (1.25, 2.0):
            b = beta_f32((w,), (osf,))
            c_os = scale_coord_f32(edge[None, :, None], (N,), (osf,))
            n_os = int(np.ceil(np.float32(osf) * np.float32(N)))
            idx, val = build_tables(k, c_os, (n_os,), (w,), b)
            tag = f"tab_w{w}_os{osf}"
            out[tag + "_index"], out[tag + "_value"] = idx[0], val[0]
    out["tab_coord"], out["tab_N"] = edge, np.int32(N)

    # 3. Spread / interp on seeded small problems, 1D / 2D / 3D, plain and subspace
    cases = {
        1: dict(N=(40,), osf=(2.0,), w=(4,), F=2, B=3, M=97, K=2),
        2: dict(N=(24, 32), osf=(1.25, 2.0), w=(4, 4), F=3, B=2, M=211, K=3),
        3: dict(N=(12, 10, 14), osf=(1.25, 1.25, 1.5), w=(4, 3, 5), F=2, B=2, M=157, K=2),
    }
    for d, c in cases.items():
        N_zyx = np.array(c["N"])
        N_xyz = N_zyx[::-1]
        osf_zyx = np.array(c["osf"], np.float32)
        w_zyx = np.array(c["w"], np.int16)
        beta_zyx = beta_f32(w_zyx, osf_zyx)
        os_zyx = np.ceil(osf_zyx * N_zyx.astype(np.float32)).astype(np.int64)
        F, B, M, K = c["F"], c["B"], c["M"], c["K"]
        coord = (rng.random((F, M, d), dtype=np.float32) - 0.5) * N_xyz.astype(np.float32)
        coord[0, :3] = -N_xyz.astype(np.float32) / 2  # exact lower edge
        c_os = scale_coord_f32(coord, N_xyz, osf_zyx[::-1])
        idx, val = build_tables(k, c_os, os_zyx, w_zyx, beta_zyx)
        nc = (rng.standard_normal((F, B, M)) + 1j * rng.standard_normal((F, B, M))).astype(np.complex64)
        cart = np.zeros((F, B, *os_zyx), np.complex64)
        k[f"grid{d}"](cart, nc, val, idx)
        grid_in = (rng.standard_normal((F, B, *os_zyx)) + 1j * rng.standard_normal((F, B, *os_zyx))).astype(np.complex64)
        deg = np.zeros((F, B, M), np.complex64)
        k[f"degrid{d}"](deg, grid_in, val, idx)
        basis = (rng.standard_normal((F, K)) + 1j * rng.standard_normal((F, K))).astype(np.complex64)
        cart_s = np.zeros((K, B, *os_zyx), np.complex64)
        k[f"grid{d}_subspace"](cart_s, nc, val, idx, np.ascontiguousarray(basis.conj().T))
        grid_in_s = (rng.standard_normal((K, B, *os_zyx)) + 1j * rng.standard_normal((K, B, *os_zyx))).astype(np.complex64)
        deg_s = np.zeros((F, B, M), np.complex64)
        k[f"degrid{d}_subspace"](deg_s, grid_in_s, val, idx, basis)
        p = f"k{d}d_"
        out.update({
            p + "N": N_zyx.astype(np.int32), p + "osf": osf_zyx, p + "width": w_zyx.astype(np.int32),
            p + "beta": beta_zyx, p + "os": os_zyx.astype(np.int32), p + "coord": coord,
            p + "noncart": nc, p + "spread": cart, p + "grid_in": grid_in, p + "interp": deg,
            p + "basis": basis, p + "spread_sub": cart_s, p + "grid_in_sub": grid_in_s,
            p + "interp_sub": deg_s,
        })
        for a in range(d):
            out[p + f"index{a}"], out[p + f"value{a}"] = idx[a], val[a]

    # 4. Cartesian masking kernels (sparse FFT gather / scatter-add), 2D and 3D, plain
    # and subspace; a separate seeded generator keeps the arrays above unchanged
    mrng = np.random.default_rng(20240608)
    for d, (N_zyx, F, B, npts, K) in {2: ((12, 16), 3, 2, 40, 2), 3: ((6, 8, 10), 2, 2, 50, 3)}.items():
        idx = np.stack([mrng.integers(0, n, (F, npts)) for n in N_zyx], -1).astype(np.int32)  # (F, npts, d) z, y, x
        idx[0, :6] = idx[0, 6]  # repeated points: the scatter adds them
        index = tuple(np.ascontiguousarray(idx[..., a]) for a in range(d))
        dense = (mrng.standard_normal((F, B, *N_zyx)) + 1j * mrng.standard_normal((F, B, *N_zyx))).astype(np.complex64)
        sparse = np.zeros((F, B, npts), np.complex64)
        k[f"mask{d}"](sparse, dense, index)
        ksp = (mrng.standard_normal((F, B, npts)) + 1j * mrng.standard_normal((F, B, npts))).astype(np.complex64)
        fill = np.zeros((F, B, *N_zyx), np.complex64)
        k[f"zerofill{d}"](fill, ksp, index)
        basis = (mrng.standard_normal((F, K)) + 1j * mrng.standard_normal((F, K))).astype(np.complex64)
        dense_s = (mrng.standard_normal((K, B, *N_zyx)) + 1j * mrng.standard_normal((K, B, *N_zyx))).astype(np.complex64)
        sparse_s = np.zeros((F, B, npts), np.complex64)
        k[f"mask{d}_subspace"](sparse_s, dense_s, index, basis)  # basis_adjoint (F, K)
        fill_s = np.zeros((K, B, *N_zyx), np.complex64)
        k[f"zerofill{d}_subspace"](fill_s, ksp, index, np.ascontiguousarray(basis.conj().T))  # basis (K, F)
        p = f"m{d}d_"
        out.update({p + "shape": np.array(N_zyx, np.int32), p + "index": idx, p + "dense": dense,
                    p + "sparse": sparse, p + "ksp": ksp, p + "fill": fill, p + "basis": basis,
                    p + "dense_sub": dense_s, p + "sparse_sub": sparse_s, p + "fill_sub": fill_s})

    path = os.path.join(HERE, "kernels.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes,", len(out), "arrays")


if __name__ == "__main__":
    main()
