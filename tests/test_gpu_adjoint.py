"""GPU checks of the discrete adjoint of the fused step (hcl_adjoint_*).

Gresho vortex (2-D, periodic, gamma=5/3, HLLC, van Leer), dt recorded from a
CFL run and held fixed.  Objective J = 0.5 ||rho^N - rho_target||^2 over the
interior, rho_target from a run whose initial density carries a seeded 1 %
multiplicative perturbation.  The gradient with respect to every initial
conserved value is checked against central finite differences of the FP64
forward along seeded random directions, and the FP32-mixed sweep against the
FP64 one."""
import numpy as np
import pytest

from heraclespp_b200 import Domain, setups
from oracle import Oracle

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

KW = dict(gamma=5.0 / 3.0, limiter="VanLeer", riemann="HLLC", bc=["Periodic"] * 4)


def smooth_background(grid, prim, amp=0.02, seed=11):
    """Adds smooth seeded Fourier modes to rho and P.  The plain Gresho vortex
    is exactly uniform for r > 0.4; there every limited slope sits on the
    limiter's kink (phi(R, L) is homogeneous of degree one at R = L = 0), so a
    central difference sees a directional derivative that no branch-following
    derivative has.  The modulation removes the flat region."""
    rng = np.random.default_rng(seed)
    s3, (X, Y, Z), _ = grid.interior()
    rho, u, P = (a.copy() for a in prim)
    for _ in range(3):
        kx, ky = rng.integers(1, 3, size=2)
        ph = rng.uniform(0, 2 * np.pi, size=2)
        m = np.sin(2 * np.pi * kx * X + ph[0]) * np.sin(2 * np.pi * ky * Y + ph[1])
        rho[s3] = rho[s3] * (1 + amp * m)
        P[s3] = P[s3] * (1 + amp * np.roll(m, 3, axis=-1))
    return rho, u, P


def problem(n, nsteps, precision="fp64", smooth=True):
    o = Oracle(2, [n, n], **KW)
    grid = setups.Grid.from_domain(o)
    prim = setups.gresho_vortex(grid)
    if smooth:
        prim = smooth_background(grid, prim)
    rho, rhou, E, _ = o.init_from_prim(*prim)
    U0 = np.concatenate([rho[None], rhou, E[None]])  # (4, 1, n+4, n+4)
    d = Domain(2, [n, n], precision=precision, **KW)
    d.set_state(rho, rhou, E)
    r = d.run(cfl=0.4, nsteps=nsteps)
    dts = d.dt_log()[:nsteps]
    assert r.iter == nsteps
    # target: seeded 1 % perturbation of the initial density
    rng = np.random.default_rng(2025)
    prim_t = [a.copy() for a in prim]
    prim_t[0] = prim_t[0] * (1 + 0.01 * rng.uniform(-1, 1, prim_t[0].shape))
    rt, mt, Et, _ = o.init_from_prim(*prim_t)
    d.set_state(rt, mt, Et)
    d.run(nsteps=nsteps, dts=dts)
    target = d.get_state()[0].copy()
    return o, d, U0, dts, target


def J_of(d, o, U, dts, target, ng=2):
    U = U.copy()
    o.boundaries(U[0], U[1:3], U[3])
    d.set_state(U[0], U[1:3], U[3])
    d.run(nsteps=len(dts), dts=dts)
    r = d.get_state()[0]
    diff = (r - target)[0, ng:-ng, ng:-ng]
    return 0.5 * float(np.sum(diff * diff))


def adjoint_grad(d, U0, dts, target, precision, k, ng=2):
    d.set_state(U0[0], U0[1:3], U0[3])
    d.adjoint_forward(len(dts), dts=dts, precision=precision, checkpoint_every=k)
    rN = d.get_state()[0]
    lam = np.zeros_like(U0)
    lam[0, 0, ng:-ng, ng:-ng] = (rN - target)[0, ng:-ng, ng:-ng]
    return d.adjoint_backward(lam)


@pytest.mark.parametrize("n,nsteps,k,ndir", [(32, 24, 8, 12), (512, 400, 32, 64)])
def test_adjoint_matches_finite_differences(n, nsteps, k, ndir):
    o, d, U0, dts, target = problem(n, nsteps)
    g = adjoint_grad(d, U0, dts, target, "fp64", k)
    ng = 2
    assert np.all(g[:, :, :ng, :] == 0) and np.all(g[:, :, :, :ng] == 0)
    rng = np.random.default_rng(64)
    errs = []
    for _ in range(ndir):
        v = np.zeros_like(U0)
        v[:, :, ng:-ng, ng:-ng] = rng.uniform(-1, 1, (4, 1, n, n)) * np.abs(U0[:, :, ng:-ng, ng:-ng])
        eps = 1e-7
        jp = J_of(d, o, U0 + eps * v, dts, target)
        jm = J_of(d, o, U0 - eps * v, dts, target)
        fd = (jp - jm) / (2 * eps)
        ad = float(np.sum(g * v))
        errs.append(abs(fd - ad) / max(abs(fd), 1e-300))
    errs = np.array(errs)
    print(f"n={n} steps={nsteps}: FD rel err median {np.median(errs):.2e} max {errs.max():.2e}")
    # smooth flow: the directions agree to 1e-5 except any that straddle a
    # limiter / wave-speed switch (the map is only piecewise smooth)
    assert np.median(errs) < 1e-6, errs
    assert np.mean(errs < 1e-5) >= 0.9, errs


def test_mixed_adjoint_close_to_fp64():
    o, d, U0, dts, target = problem(64, 40)
    g64 = adjoint_grad(d, U0, dts, target, "fp64", 16)
    g32 = adjoint_grad(d, U0, dts, target, "fp32_mixed", 16)
    rel = np.linalg.norm(g32 - g64) / np.linalg.norm(g64)
    assert rel < 1e-4, rel


def test_autograd_wrapper_gives_the_adjoint():
    from autograd_step import FusedSteps

    o, d, U0, dts, target = problem(32, 16)
    ng = 2
    U0t = torch.tensor(U0, device="cuda", requires_grad=True)
    tt = torch.tensor(target, device="cuda")
    UN = FusedSteps.apply(U0t, d, len(dts), dts, "fp64", 4)
    J = 0.5 * ((UN[0, 0, ng:-ng, ng:-ng] - tt[0, ng:-ng, ng:-ng]) ** 2).sum()
    J.backward()
    g_direct = adjoint_grad(d, U0, dts, target, "fp64", 4)
    # FP64 atomics accumulate in a different order on every call
    np.testing.assert_allclose(U0t.grad.cpu().numpy(), g_direct, rtol=1e-10, atol=1e-14 * np.abs(g_direct).max())
