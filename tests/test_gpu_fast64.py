"""Fast FP64 (precision "fp64_fast", HCL_FP64_FAST): the FP64 fused step with
FMA contraction and the perfect gas without the temperature round trip, held
to 1e-12 relative L1 per variable against the FP64 oracle on the case matrix
(1-D to 3-D, Cartesian and spherical, every boundary kind, uniform, point-mass
and internal-mass gravity, every limiter and Riemann solver).  The same dt
sequence is fed to both, and the kernel's own CFL reduction is compared with
the oracle's dts to the same bound."""
import numpy as np
import pytest

from cases import CASES, make_pair

pytestmark = pytest.mark.gpu

BOUND = 1e-12
STEPS = 30


def rel_l1_scaled(a, b, scale):
    return float(np.sum(np.abs(a - b)) / scale)


def check_fields(got, ref):
    rho_d, m_d, E_d = got
    rho, rhou, E = ref
    s_rho = float(np.sum(np.abs(rho)))
    assert rel_l1_scaled(rho_d, rho, s_rho) < BOUND
    assert rel_l1_scaled(E_d, E, float(np.sum(np.abs(E)))) < BOUND
    for k in range(rhou.shape[0]):
        # momenta that stay near zero are measured on the density's scale
        scale = max(float(np.sum(np.abs(rhou[k]))), 1e-3 * s_rho)
        assert rel_l1_scaled(m_d[k], rhou[k], scale) < BOUND, k


@pytest.mark.parametrize("name", [n for n in CASES])
def test_fast64_within_1e12_of_oracle(name):
    o, d, (rho0, u0, P0) = make_pair(name, "fp64_fast")
    rho, rhou, E, fx = o.init_from_prim(rho0, u0, P0)
    _, it, st, dts = o.run(rho, rhou, E, fx, cfl=0.4, max_iter=STEPS, record_dts=True)
    assert st == 0 and it == STEPS
    d.set_state_from_prim(rho0, u0, P0)
    d.run(nsteps=STEPS, dts=dts)
    check_fields(d.get_state(), (rho, rhou, E))
    # the in-pass CFL reduction of the same run: the dts it would take
    d2 = make_pair(name, "fp64_fast")[1]
    d2.set_state_from_prim(rho0, u0, P0)
    r = d2.run(cfl=0.4, max_iter=STEPS)
    assert r.iter == STEPS
    own = d2.dt_log()[:STEPS]
    assert float(np.max(np.abs(own - dts) / dts)) < BOUND
    d.close()
    d2.close()


def test_fast64_refuses_radgas():
    import heraclespp_b200 as hb

    with pytest.raises(hb.HclError):
        hb.Domain(1, [64], precision="fp64_fast", eos="RadGas", bc=["NullGradient"] * 2)


def test_fast64_adjoint_recomputes_with_its_own_step():
    """The checkpointed gradient of a fast-FP64 handle (its checkpoints and
    recomputed segments come from the fast step; FP64 reverse sweep) against
    the plain FP64 handle's, same dts, on a Gresho vortex with smooth seeded
    modes (no flat region, where limited slopes sit on the limiter's kink and
    a rounding-level difference picks another branch)."""
    import torch

    from heraclespp_b200 import Domain, setups
    from test_gpu_adjoint import smooth_background

    kw = dict(gamma=5.0 / 3.0, limiter="VanLeer", riemann="HLLC", bc=["Periodic"] * 4)
    grads = []
    dts = None
    for prec in ("fp64", "fp64_fast"):
        d = Domain(2, [48, 48], precision=prec, **kw)
        grid = setups.Grid.from_domain(d)
        prim = smooth_background(grid, setups.gresho_vortex(grid))
        d.set_state_from_prim(*prim)
        if dts is None:
            d.run(cfl=0.4, nsteps=12)
            dts = d.dt_log()[:12]
            d.set_state_from_prim(*prim)
        d.adjoint_forward(12, dts=dts, checkpoint_every=4, precision="fp64")
        lam = torch.zeros((4,) + d.shape3, dtype=torch.float64, device="cuda")
        lam[0] = 1.0
        g = torch.zeros_like(lam)
        d.adjoint_backward(lam, g, device=True)
        grads.append(g.cpu().numpy())
        d.close()
    a, b = grads
    assert float(np.abs(a - b).sum() / np.abs(a).sum()) < 1e-8
