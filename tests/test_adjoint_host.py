"""CPU checks of the hand-written discrete adjoint (awflcloud_b200/csrc/awfl_adj.h,
awfl_adj_split.h), compiled for the host with g++:

* each reverse-mode building block (WENO, one cell's reconstruction + ADER + time
  averages, the Riemann flux) against fourth-order finite differences of its forward;
* the adjoint of a whole directional split (halo mapping, wall/periodic edges, sim2d)
  against central finite differences of the oracle's split (the C restatement of the
  reference, oracle/awfl_oracle.c): <lam, dS(v)> == <S^T lam, v>.
"""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

from awflcloud_b200 import capi
from oracle.pyoracle import Oracle

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(ROOT, "awflcloud_b200", "csrc")
CUDA_INC = "/usr/local/cuda/include"

pytestmark = pytest.mark.skipif(shutil.which("g++") is None or not os.path.isdir(CUDA_INC),
                                reason="needs g++ and the CUDA headers")


def _tables_flat(ord_):
    t = capi.Context(16, 12, 8, ord_=ord_, device=-1).tables()
    return np.concatenate([t["weno_recon"], t["coefs_to_gll"], t["sten_to_gll"], t["deriv"], t["idl"],
                           t["sigma"], t["gll_wts_ngll"]]).astype(np.float64)


def _compile(tmp, src, out, shared):
    cmd = ["g++", "-O2", "-std=c++17", "-I" + CSRC, "-I" + CUDA_INC, src, "-o", out]
    if shared:
        cmd[1:1] = ["-shared", "-fPIC"]
    subprocess.run(cmd, check=True, cwd=tmp)
    return out


def test_reverse_building_blocks_match_finite_differences(tmp_path):
    exe = _compile(tmp_path, os.path.join(HERE, "adj_host_check.cpp"), str(tmp_path / "adj_check"), False)
    paths = []
    for o in (5, 9):
        p = str(tmp_path / ("tables%d.bin" % o))
        _tables_flat(o).astype("<f8").tofile(p)
        paths.append(p)
    r = subprocess.run([exe] + paths, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = [l.split() for l in r.stdout.splitlines() if l and not l.startswith("FAIL")]
    assert len(lines) == 3 + 2 * (2 + 10)
    assert all(float(e) < 1e-6 for _, e in lines), r.stdout


@pytest.fixture(scope="module")
def split_lib(tmp_path_factory):
    tmp = tmp_path_factory.mktemp("adjsplit")
    so = _compile(tmp, os.path.join(HERE, "adj_split_host.cpp"), str(tmp / "libadjsplit.so"), True)
    L = ctypes.CDLL(so)
    D, I, P = ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_double)
    for f in (L.adj_split_host, L.fwd_split_host):
        f.restype = I
        f.argtypes = [I, I, P] + [I] * 7 + [D, D] + [P] * 7
    return L


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _state_with_winds(O, seed):
    """Rising-bubble state plus a smooth wind field, so that no face sits on the upwind
    switch (the flux is not differentiable where the normal velocity changes sign)."""
    st = O.new_state()
    O.init_state(st)
    O.set_bubble(st, 1, 10000., 10000., 2000., 2000., 2000., 2000., 3.0, 1.0)
    O.add_theta_noise(st, seed, 0.01)
    hs = O.hs
    bg = O.background()
    nz, ny, nx = O.nz, O.ny, O.nx
    rho = st[0, hs:hs + nz, hs:hs + ny, hs:hs + nx] + bg["hyDensCells"][hs:hs + nz, None, None]
    z = ((np.arange(nz) + 0.5) / nz)[:, None, None]
    y = ((np.arange(ny) + 0.5) / ny)[None, :, None]
    x = ((np.arange(nx) + 0.5) / nx)[None, None, :]
    ph = 0.1 * seed
    # every component varies along every direction: on exactly uniform data the smoothness
    # indicators vanish and the WENO weights turn on a scale (tv^2 ~ 1e-20) far below any
    # usable finite-difference step
    st[1, hs:hs + nz, hs:hs + ny, hs:hs + nx] = rho * (6.0 + np.sin(2 * np.pi * (x + 0.3))
                                                       + 0.8 * np.sin(2 * np.pi * (y + 0.1 + ph)) + 0.5 * np.cos(np.pi * z))
    st[2, hs:hs + nz, hs:hs + ny, hs:hs + nx] = rho * (-4.0 + np.cos(2 * np.pi * (x - ph))
                                                       + 0.7 * np.sin(2 * np.pi * (y + 0.2)) + 0.3 * np.cos(np.pi * z))
    st[3, hs:hs + nz, hs:hs + ny, hs:hs + nx] = rho * np.sin(np.pi * z) * (3.0 + 0.5 * np.sin(2 * np.pi * (x + y))
                                                                           + 0.3 * np.cos(2 * np.pi * (x - 0.2)))
    return st


def _interior_random(O, rng, scale):
    a = np.zeros(O.state_shape)
    hs = O.hs
    for v in range(5):
        a[v, hs:hs + O.nz, hs:hs + O.ny, hs:hs + O.nx] = scale[v] * rng.standard_normal((O.nz, O.ny, O.nx))
    return a


CASES = [
    # ord, (nx, ny, nz), bc, dirs, weno
    (5, (10, 8, 7), (0, 0, 1), (0, 1, 2), True),
    (5, (7, 6, 5), (1, 1, 0), (0, 1, 2), True),   # wall x/y, periodic z
    (5, (9, 1, 6), (0, 0, 1), (0, 2), True),      # sim2d (ny = 1): y split skipped
    (5, (8, 6, 6), (0, 0, 1), (0, 1, 2), False),  # linear reconstruction
    (9, (12, 10, 9), (0, 0, 1), (0, 1, 2), True),
    (9, (10, 9, 8), (1, 1, 0), (0, 1, 2), True),
]


def _setup(ord_, n, bc, weno):
    nx, ny, nz = n
    xlen, ylen, zlen = 20000.0, 20000.0 if ny > 1 else 20000.0 / 64, 10000.0
    O = Oracle(nx, ny, nz, xlen, ylen, zlen, bc=bc, weno_scalars=weno, weno_winds=weno, ord_=ord_)
    H = capi.Context(nx, ny, nz, xlen, ylen, zlen, bc=bc, weno_scalars=weno, weno_winds=weno, ord_=ord_, device=-1)
    bg = H.background()
    bgp = [_p(bg[k]) for k in ("hyDensCells", "hyDensThetaCells", "hyDensGLL", "hyDensThetaGLL", "hyPressureGLL")]
    st = _state_with_winds(O, 7 + ord_)
    dt = O.compute_dt(st, 0.8 if ord_ == 5 else 0.4)
    return O, _tables_flat(ord_), bgp, st, dt, {0: xlen / nx, 1: ylen / ny, 2: zlen / nz}


@pytest.mark.parametrize("ord_,n,bc,dirs,weno", CASES)
def test_adjoint_forward_recomputation_matches_oracle(split_lib, ord_, n, bc, dirs, weno):
    """The linearisation point: the adjoint's forward functions give the oracle's
    tendencies to rounding (they use reciprocals and contracted multiply-adds)."""
    O, tabs, bgp, st, dt, dx = _setup(ord_, n, bc, weno)
    nx, ny, nz = n
    for d in dirs:
        t_ref = np.zeros(O.tend_shape)
        O.compute_tendencies_dir(st.copy(), t_ref, dt, d)
        t = np.zeros(O.tend_shape)
        assert split_lib.fwd_split_host(ord_, d, _p(tabs), nx, ny, nz, bc[d], int(weno), int(weno), int(ny == 1),
                                        dx[d], dt, *bgp, _p(st), _p(t)) == 0
        for v in range(5):
            scale = np.abs(t_ref[v]).max()
            assert np.abs(t[v] - t_ref[v]).max() <= 1e-10 * max(scale, 1e-300), (d, v)


@pytest.mark.parametrize("ord_,n,bc,dirs,weno", CASES)
def test_split_adjoint_matches_oracle_finite_differences(split_lib, ord_, n, bc, dirs, weno):
    O, tabs, bgp, st, dt, dx = _setup(ord_, n, bc, weno)
    nx, ny, nz = n
    rng = np.random.default_rng(123)
    scale = [1e-3, 1.0, 1.0, 1.0, 0.3]
    hs = O.hs
    for d in dirs:
        lam = _interior_random(O, rng, [1.0] * 5)
        lam_t = lam[:, hs:hs + nz, hs:hs + ny, hs:hs + nx]

        def T(s):  # dt * tendency of the split (the identity part of the split is exact)
            s = s.copy()
            t = np.zeros(O.tend_shape)
            O.compute_tendencies_dir(s, t, dt, d)
            return dt * t

        out = lam.copy()
        rc = split_lib.adj_split_host(ord_, d, _p(tabs), nx, ny, nz, bc[d], int(weno), int(weno), int(ny == 1),
                                      dx[d], dt, *bgp, _p(st), _p(out))
        assert rc == 0
        # One variable at a time, perturbed by ~1e-7 (density 3e-8) in absolute terms. At a
        # wall the halo repeats the edge cell, so a low-order WENO stencil there is exactly
        # uniform: its smoothness indicator tv is zero and the weight idl/(tv^2 + 1e-20)
        # changes by ~delta^4/1e-20 under a perturbation delta, so a finite difference sees
        # the exact (zero) derivative only for delta well below 1e-5; below ~1e-7 rounding
        # of the pressure terms (~1e5) takes over. Hence the 1e-6 bound.
        for var, h in ((0, 3e-5), (1, 1e-7), (2, 1e-7), (3, 1e-7), (4, 1e-6)):
            v = np.zeros(O.state_shape)
            v[var] = _interior_random(O, rng, scale)[var]
            fd = (8 * (T(st + h * v) - T(st - h * v)) - (T(st + 2 * h * v) - T(st - 2 * h * v))) / (12 * h)
            lhs = float(np.sum(lam_t * fd))
            rhs = float(np.sum((out - lam) * v))
            ref = float(np.sum(np.abs(lam_t * fd)))
            assert abs(lhs - rhs) <= 1e-6 * ref, (d, var, lhs, rhs, ref)
        # halo entries of the adjoint are not touched
        mask = np.ones(O.state_shape, bool)
        mask[:, hs:hs + nz, hs:hs + ny, hs:hs + nx] = False
        assert np.all(out[mask] == lam[mask])
