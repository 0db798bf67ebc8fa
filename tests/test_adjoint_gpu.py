"""Differentiation form on the GPU: the tangent-linear step (awfl_step_tlm) and the
hand-written discrete adjoint (awfl_step_adjoint, with recomputation from checkpoints).

Bars: the tangent-linear derivative and the adjoint gradient agree with FP64 central
finite differences (eps = 1e-6) to <= 1e-6 relative on 32x32x16 over 20 steps (16
seeded directions for the gradient of J = 1/2 sum (rho*theta_final - target)^2); the
adjoint is the transpose of the tangent-linear model (dot-product test).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from awflcloud_b200 import capi  # noqa: E402
from awflcloud_b200.adjoint import euler_steps  # noqa: E402

N = (32, 32, 16)
STEPS = 20


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def interior(c, a):
    h = c.hs
    return a[..., h:h + c.nz, h:h + c.ny, h:h + c.nx]


def base_state(c, seed=3, noise_sigma=0.0):
    """Rising bubble + uniform theta noise + a smooth wind field (no face on the upwind
    switch); optionally N(0, noise_sigma) theta noise on top (the gradient target)."""
    s = c.new_state()
    c.init_state(s, kind=capi.INIT_BUBBLE, noise_amp=0.01, noise_seed=seed)
    bg = c.background()
    h = c.hs
    dens = torch.tensor(bg["hyDensCells"][h:h + c.nz], dtype=torch.float64, device=s.device)[:, None, None]
    rho = interior(c, s[0]) + dens
    z = ((torch.arange(c.nz, dtype=torch.float64, device=s.device) + 0.5) / c.nz)[:, None, None]
    y = ((torch.arange(c.ny, dtype=torch.float64, device=s.device) + 0.5) / c.ny)[None, :, None]
    x = ((torch.arange(c.nx, dtype=torch.float64, device=s.device) + 0.5) / c.nx)[None, None, :]
    pi = np.pi
    # the normal velocity vanishes toward a wall (and keeps one sign inside)
    fx = torch.sin(pi * x) if c.cfg.bc_x == 1 else 1.0
    fy = torch.sin(pi * y) if c.cfg.bc_y == 1 else 1.0
    fz = torch.sin(pi * z) if c.cfg.bc_z == 1 else 1.0
    interior(c, s[1])[:] = rho * fx * (6.0 + torch.sin(2 * pi * (x + 0.3)) + 0.8 * torch.sin(2 * pi * (y + 0.1))
                                       + 0.5 * torch.cos(pi * z))
    interior(c, s[2])[:] = rho * fy * (-4.0 + torch.cos(2 * pi * x) + 0.7 * torch.sin(2 * pi * (y + 0.2))
                                       + 0.3 * torch.cos(pi * z))
    interior(c, s[3])[:] = rho * fz * (3.0 + 0.5 * torch.sin(2 * pi * (x + y)) + 0.3 * torch.cos(2 * pi * (x - 0.2)))
    if noise_sigma > 0:
        g = torch.Generator().manual_seed(seed + 1000)
        n = torch.randn((c.nz, c.ny, c.nx), generator=g, dtype=torch.float64).to(s.device) * noise_sigma
        interior(c, s[4])[:] += dens * n
    return s


def unit_direction(c, gen):
    """A seeded random direction on the interior, unit 2-norm, zero in the halos."""
    v = torch.zeros(c.state_shape, dtype=torch.float64)
    h = c.hs
    v[:, h:h + c.nz, h:h + c.ny, h:h + c.nx] = torch.randn((5, c.nz, c.ny, c.nx), generator=gen, dtype=torch.float64)
    v /= torch.linalg.vector_norm(v)
    return v.cuda()


def run(c, s, steps, dt, ds=1):
    s = s.clone()
    c.dimswitch = ds
    for _ in range(steps):
        c.step(s, dt)
    return s


def test_tlm_value_plane_is_the_fp64_step():
    c1, c2 = capi.Context(*N), capi.Context(*N)
    s = base_state(c1)
    dt = c1.cfl(s, 0.8)
    st = torch.cat([s.clone(), torch.zeros_like(s)])
    g = torch.Generator().manual_seed(1)
    st[5:] = unit_direction(c1, g)
    for _ in range(3):
        c1.step(s, dt)
        c2.step_tlm(st, dt)
    torch.cuda.synchronize()
    assert torch.equal(interior(c1, st[:5]), interior(c1, s))


@pytest.mark.parametrize("bc", [("periodic", "periodic", "wall"), ("wall", "wall", "wall")])
def test_tlm_matches_central_finite_differences(bc):
    c = capi.Context(*N, bc=bc)
    s0 = base_state(c)
    dt = c.cfl(s0, 0.8)
    g = torch.Generator().manual_seed(11)
    eps = 1e-6
    for _ in range(4):
        v = unit_direction(c, g)
        st = torch.cat([s0.clone(), v.clone()])
        c.dimswitch = 1
        for _ in range(STEPS):
            c.step_tlm(st, dt)
        jv = interior(c, st[5:])
        fd = (interior(c, run(c, s0 + eps * v, STEPS, dt)) - interior(c, run(c, s0 - eps * v, STEPS, dt))) / (2 * eps)
        err = (torch.linalg.vector_norm(jv - fd) / torch.linalg.vector_norm(fd)).item()
        assert err <= 1e-6, err


@pytest.mark.parametrize("ord_,bc", [(5, ("periodic", "periodic", "wall")), (5, ("wall", "wall", "wall")),
                                     (9, ("periodic", "periodic", "wall")), (9, ("wall", "periodic", "wall"))])
def test_adjoint_is_the_transpose_of_the_tlm(ord_, bc):
    """<lam, M v> == <M^T lam, v> for the 20-step map M."""
    c = capi.Context(*N, bc=bc, ord_=ord_)
    s0 = base_state(c)
    dt = c.cfl(s0, 0.8 if ord_ == 5 else 0.4)
    g = torch.Generator().manual_seed(5)
    v = unit_direction(c, g)
    lam = unit_direction(c, g)
    st = torch.cat([s0.clone(), v.clone()])
    c.dimswitch = 1
    for _ in range(STEPS):
        c.step_tlm(st, dt)
    lhs = torch.sum(lam * st[5:]).item()
    c.dimswitch = 1
    lam_in = lam.clone()
    c.step_adjoint(s0, lam_in, STEPS, dt)
    rhs = torch.sum(lam_in * v).item()
    assert c.dimswitch == 1
    scale = (torch.sum(torch.abs(lam_in * v))).item()
    assert abs(lhs - rhs) <= 1e-11 * scale, (lhs, rhs, scale)


@pytest.mark.parametrize("m", [1, 3, 7])
def test_two_level_window_equals_one_level(m):
    """Sub-windows of m steps (one plain forward pass keeping every m-th state, then each
    sub-window recorded and reversed) give exactly the one-level adjoint of the 20-step
    window -- odd m included, whose sub-windows start with the other dimSwitch -- on a
    smaller tape."""
    c = capi.Context(*N)
    s0 = base_state(c)
    dt = c.cfl(s0, 0.8)
    g = torch.Generator().manual_seed(13)
    lam = unit_direction(c, g)
    a = lam.clone()
    c.dimswitch = 1
    c.step_adjoint(s0, a, 20, dt)
    one_level = c.adjoint_tape_bytes(20)
    c.set_adjoint_subwindow(m)
    b = lam.clone()
    c.dimswitch = 1
    c.step_adjoint(s0, b, 20, dt)
    torch.cuda.synchronize()
    assert c.dimswitch == 1
    assert torch.equal(a, b)
    assert c.adjoint_tape_bytes(20) < one_level / 2
    c.set_adjoint_subwindow(0)


def test_adjoint_segments_equal_one_window():
    """Two 10-step windows (the second from the recomputed checkpoint) give exactly the
    adjoint of one 20-step window."""
    c = capi.Context(*N)
    s0 = base_state(c)
    dt = c.cfl(s0, 0.8)
    g = torch.Generator().manual_seed(9)
    lam = unit_direction(c, g)
    a = lam.clone()
    c.dimswitch = 1
    c.step_adjoint(s0, a, 20, dt)
    s10 = run(c, s0, 10, dt)  # dimswitch after 10 steps is back to 1
    b = lam.clone()
    c.dimswitch = 1
    c.step_adjoint(s10, b, 10, dt)
    c.dimswitch = 1
    c.step_adjoint(s0, b, 10, dt)
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    # halos of the adjoint are zero
    mask = torch.ones_like(a, dtype=torch.bool)
    interior(c, mask)[:] = False
    assert torch.count_nonzero(a[mask]).item() == 0


def test_gradient_matches_central_finite_differences():
    """J = 1/2 sum (rho*theta_final - target)^2 over the interior, target = the FP64 run of
    the bubble with N(0, 0.1 K) theta noise; gradient through the autograd wrapper over
    awfl_step_adjoint (checkpoint every 10 steps) against FP64 central differences,
    eps = 1e-6, 16 seeded unit directions.

    This test meets 2e-6 (measured 1.6e-6), not the north star's 1e-6, and the shortfall is
    the FP64 finite difference's own error, not the adjoint's: the difference's rounding
    part grows as 1/eps (1.1e-5 at eps = 1e-7; the fluxes carry the full ~1e5 Pa
    pressure, so every step leaves ~1e-13 of rounding noise in the state) and its
    truncation part as eps^2 (9.7e-5 at eps = 1e-5); directions scaled to the state's own
    magnitudes do no better (1.1e-6 at best). The 1e-6 bar is met against the same
    differences taken in extended precision (test_gradient_matches_extended_precision_
    finite_differences: ~1e-8), and the adjoint agrees with the FP64 tangent-linear model
    to ~1e-12 (test_adjoint_is_the_transpose_of_the_tlm)."""
    c = capi.Context(*N)
    s0 = base_state(c)
    dt = c.cfl(s0, 0.8)
    target = interior(c, run(c, base_state(c, noise_sigma=0.1), STEPS, dt)[4])

    def J(s):
        return 0.5 * torch.sum((interior(c, run(c, s, STEPS, dt)[4]) - target) ** 2).item()

    x = s0.clone().requires_grad_(True)
    c.dimswitch = 1
    sN = euler_steps(x, c, STEPS, dt, ckpt_every=10)
    loss = 0.5 * torch.sum((interior(c, sN[4]) - target) ** 2)
    loss.backward()
    grad = x.grad
    assert abs(loss.item() - J(s0)) <= 1e-12 * loss.item()
    g = torch.Generator().manual_seed(20261203)
    eps = 1e-6
    gv, fd = [], []
    for _ in range(16):
        v = unit_direction(c, g)
        gv.append(torch.sum(grad * v).item())
        fd.append((J(s0 + eps * v) - J(s0 - eps * v)) / (2 * eps))
    gv, fd = np.array(gv), np.array(fd)
    err = np.linalg.norm(gv - fd) / np.linalg.norm(fd)
    assert err <= 2e-6, (err, gv, fd)


def test_gradient_matches_extended_precision_finite_differences():
    """The same gradient against central differences of the same J evaluated by the
    oracle's restatement in x87 long double (oracle/liboracle_o5_ld.so, 11 more bits):
    with the FD's rounding error out of the way, the fourth-order difference at eps = 1e-6
    and the second-order one at eps = 1e-7 both agree with the adjoint to ~1e-8 (the
    second-order difference at eps = 1e-6 carries ~1e-6 of truncation error)."""
    from oracle.pyoracle import OracleLD
    c = capi.Context(*N)
    s0 = base_state(c)
    dt = c.cfl(s0, 0.8)
    target = interior(c, run(c, base_state(c, noise_sigma=0.1), STEPS, dt)[4])
    x = s0.clone().requires_grad_(True)
    c.dimswitch = 1
    sN = euler_steps(x, c, STEPS, dt, ckpt_every=10)
    (0.5 * torch.sum((interior(c, sN[4]) - target) ** 2)).backward()
    grad = x.grad
    O = OracleLD(*N)
    tgt = target.cpu().numpy().astype(np.longdouble)
    base = s0.cpu().numpy().astype(np.longdouble)
    h = c.hs

    def J(s):
        s = s.copy()
        O.dimswitch = 1
        for _ in range(STEPS):
            O.time_step(s, dt)
        d = s[4, h:h + c.nz, h:h + c.ny, h:h + c.nx] - tgt
        return 0.5 * np.sum(d * d)

    g = torch.Generator().manual_seed(20261203)
    gv, fd4, fd2 = [], [], []
    for _ in range(16):
        v = unit_direction(c, g)
        gv.append(torch.sum(grad * v).item())
        vl = v.cpu().numpy().astype(np.longdouble)
        e = np.longdouble(1e-6)
        fd4.append(float((8 * (J(base + e * vl) - J(base - e * vl)) - (J(base + 2 * e * vl) - J(base - 2 * e * vl)))
                         / (12 * e)))
        e = np.longdouble(1e-7)
        fd2.append(float((J(base + e * vl) - J(base - e * vl)) / (2 * e)))
    gv, fd4, fd2 = np.array(gv), np.array(fd4), np.array(fd2)
    err4 = np.linalg.norm(gv - fd4) / np.linalg.norm(fd4)
    err2 = np.linalg.norm(gv - fd2) / np.linalg.norm(fd2)
    assert err4 <= 1e-7 and err2 <= 1e-7, (err4, err2)


def test_adjoint_rejects_bad_arguments():
    c = capi.Context(*N)
    s = c.new_state()
    lam = c.new_state()
    with pytest.raises(capi.AwflError):
        c.step_adjoint(s, lam, -1, 1.0)
    with pytest.raises(capi.AwflError):
        c.step_adjoint(s, lam, 2, float("nan"))
    with pytest.raises(capi.AwflError):
        c.step_adjoint(s, s, 2, 1.0)
    c32 = capi.Context(*N, precision=capi.FP32)  # the adjoint is an FP64 form
    rc = c32.L.awfl_step_adjoint(c32.h, capi._ptr(c32.new_state()), capi._ptr(c32.new_state()), 1, 1.0, None)
    assert rc == -1  # AWFL_ERR_ARG
