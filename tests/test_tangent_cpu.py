"""CPU checks of the tangent-linear restatement (tests/tangent_step.py), which
the GPU dot-product test of the adjoint relies on:
  * its forward equals the oracle's main loop bit for bit over fixed dts;
  * its J v equals central differences of the oracle's main loop;
  * <J v, lambda> equals <v, J^T lambda> of the loop-based reference adjoint
    of one step (the per-cell reverse functions of adjoint_cell.cuh)."""
import numpy as np
import pytest

from adjoint_reference import NG, Ref, build_cell_lib, smooth_state
from oracle import Oracle

torch = pytest.importorskip("torch")
from tangent_step import TangentStep  # noqa: E402

CASES = [("VanLeer", "HLLC"), ("Minmod", "HLL"), ("VanLeer", "HLL"), ("Minmod", "HLLC")]


def state(o, seed):
    """Seeded periodic primitives with a shear layer on the oracle's grid.
    Every variable carries seeded noise: without it the symmetric sines give
    neighbouring cells equal values, whose zero differences sit on the
    limiter's kink, where central differences and every branch-following
    derivative disagree."""
    g = o.grid()
    X, Y = np.meshgrid(g["x0c"], g["x1c"])
    rng = np.random.default_rng(seed)
    rho = (1 + 0.3 * (np.abs(Y - 0.5) < 0.25) + 0.1 * np.sin(2 * np.pi * X) * np.cos(2 * np.pi * Y)
           + 0.02 * rng.uniform(-1, 1, X.shape))
    ux = 0.4 * np.tanh((0.25 - np.abs(Y - 0.5)) * 20) + 0.02 * rng.uniform(-1, 1, X.shape)
    uy = 0.05 * np.sin(4 * np.pi * X) + 0.02 * rng.uniform(-1, 1, X.shape)
    P = 2.5 + 0.1 * np.cos(2 * np.pi * (X + Y)) + 0.02 * rng.uniform(-1, 1, X.shape)
    u = np.stack([ux, uy])[:, None]
    return o.init_from_prim(rho[None], u, P[None])


def interior(a, ng=NG):
    return a[..., 0, ng:-ng, ng:-ng]


def setup(lim, rs, n=(32, 16), seed=3, steps=8):
    kw = dict(gamma=5.0 / 3.0, limiter=lim, riemann=rs, bc=["Periodic"] * 4)
    o = Oracle(2, list(n), **kw)
    rho, rhou, E, _ = state(o, seed)
    o.boundaries(rho, rhou, E)
    probe = [a.copy() for a in (rho, rhou, E)]
    *_, dts = o.run(*probe, max_iter=steps, record_dts=True)
    ts = TangentStep.from_grid(o.grid(), 5.0 / 3.0, lim, rs)
    U0 = np.concatenate([interior(rho)[None], interior(rhou), interior(E)[None]])
    return o, (rho, rhou, E), ts, U0, dts


def oracle_final(o, cons, dts):
    rho, rhou, E = (a.copy() for a in cons)
    o.run(rho, rhou, E, dts=dts, max_iter=len(dts))
    return np.concatenate([interior(rho)[None], interior(rhou), interior(E)[None]])


@pytest.mark.parametrize("lim,rs", CASES)
def test_forward_matches_oracle_bitwise(lim, rs):
    o, cons, ts, U0, dts = setup(lim, rs)
    ref = oracle_final(o, cons, dts)
    out = ts.run(torch.from_numpy(U0), dts).numpy()
    assert np.array_equal(out, ref), np.abs(out - ref).max()


@pytest.mark.parametrize("lim,rs", CASES[:2])
def test_jvp_matches_oracle_central_differences(lim, rs):
    o, cons, ts, U0, dts = setup(lim, rs, steps=5)
    rng = np.random.default_rng(7)
    V = rng.uniform(-1, 1, U0.shape) * np.abs(U0)
    _, JV = ts.jvp(torch.from_numpy(U0), torch.from_numpy(V), dts)
    JV = JV.numpy()
    lam = rng.normal(size=U0.shape)
    eps = 1e-7

    def shifted(sign):
        c = [a.copy() for a in cons]
        c[0][0, NG:-NG, NG:-NG] += sign * eps * V[0]
        c[1][:, 0, NG:-NG, NG:-NG] += sign * eps * V[1:3]
        c[2][0, NG:-NG, NG:-NG] += sign * eps * V[3]
        o.boundaries(*c)
        return oracle_final(o, c, dts)

    fd = float(np.sum(lam * (shifted(1) - shifted(-1)))) / (2 * eps)
    tl = float(np.sum(lam * JV))
    assert tl == pytest.approx(fd, rel=1e-6)


@pytest.fixture(scope="module")
def cell_lib(tmp_path_factory):
    return build_cell_lib(tmp_path_factory.mktemp("tangent") / "libadjcheck.so")


@pytest.mark.parametrize("lim,solver,rs", [(1, 1, "HLLC"), (2, 0, "HLL"), (1, 0, "HLL"), (2, 1, "HLLC")])
def test_dot_product_against_loop_adjoint(cell_lib, lim, solver, rs):
    """<J v, lambda> (tangent restatement) = <v, J^T lambda> (loop-based
    reference adjoint) for one step on a smooth periodic 8 x 8 state."""
    n = 8
    U = smooth_state(n, seed=lim + 2 * solver)
    dt, dx = 0.02, (1.0 / n, 1.0 / n)
    ref = Ref(cell_lib, gamma=1.4, lim=lim, solver=solver)
    rng = np.random.default_rng(11)
    lam = np.zeros_like(U)
    lam[:, NG:NG + n, NG:NG + n] = rng.normal(size=(4, n, n))
    g = ref.step_adjoint(U, lam, dt, dx)
    ts = TangentStep(1.4, dx[0], dx[1], dx[0] * dx[1], (dx[1], dx[0]), ("VanLeer", "Minmod")[lim - 1], rs)
    Ui = torch.from_numpy(np.ascontiguousarray(U[:, NG:NG + n, NG:NG + n]))
    for _ in range(3):
        v = rng.uniform(-1, 1, (4, n, n))
        _, JV = ts.jvp(Ui, torch.from_numpy(v), [dt])
        tl = float(np.sum(lam[:, NG:NG + n, NG:NG + n] * JV.numpy()))
        ad = float(np.sum(g[:, NG:NG + n, NG:NG + n] * v))
        assert ad == pytest.approx(tl, rel=1e-11, abs=1e-13)


@pytest.mark.parametrize("steps", [15, 23, 30])
def test_dot_product_on_plain_gresho(cell_lib, steps):
    """One step from the plain Gresho vortex (64^2) after some oracle steps,
    where flat and solid-body regions leave slope differences at rounding
    level: the loop reference adjoint takes its primitives with the forward's
    rounding and each limiter's branch from the forward's test on the
    differences divided by the spacing (after 15 and 23 steps a raw product
    underflows to 0 where that one is a positive subnormal), as the FP64
    sweep does, so <J v, lambda> = <v, J^T lambda> to rounding."""
    from heraclespp_b200 import setups

    n, g = 64, 5.0 / 3.0
    o = Oracle(2, [n, n], gamma=g, limiter="VanLeer", riemann="HLLC", bc=["Periodic"] * 4)
    rho, rhou, E, _ = o.init_from_prim(*setups.gresho_vortex(setups.Grid.from_domain(o)))
    o.run(rho, rhou, E, max_iter=steps)
    *_, dts = o.run(*[a.copy() for a in (rho, rhou, E)], max_iter=1, record_dts=True)
    dt = float(dts[0])
    U = np.concatenate([rho[None], rhou, E[None]])[:, 0]
    ref = Ref(cell_lib, gamma=g, lim=1, solver=1)
    rng = np.random.default_rng(steps)
    lam = np.zeros_like(U)
    lam[:, NG:-NG, NG:-NG] = rng.normal(size=(4, n, n))
    grad = ref.step_adjoint(U, lam, dt, (1.0 / n, 1.0 / n))
    ts = TangentStep.from_grid(o.grid(), g, "VanLeer", "HLLC")
    Ui = torch.from_numpy(np.ascontiguousarray(U[:, NG:-NG, NG:-NG]))
    for _ in range(3):
        v = rng.uniform(-1, 1, (4, n, n))
        _, JV = ts.jvp(Ui, torch.from_numpy(v), [dt])
        tl = float(np.sum(lam[:, NG:-NG, NG:-NG] * JV.numpy()))
        ad = float(np.sum(grad[:, NG:-NG, NG:-NG] * v))
        assert ad == pytest.approx(tl, rel=1e-12)
