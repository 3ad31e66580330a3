"""The batched ensemble (hcl_ensemble_*): uneven 2-D four-quadrant problems
stepped by one persistent cooperative launch must reproduce, problem by
problem, the single-problem warp-strip kernel (same strip code, same CFL
reduction: bitwise), keep each problem's clock and dt log, hand the handles
back in a state hcl_run continues from, and give the same adjoint as the
single-problem adjoint."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# ragged sides: not multiples of the 28 output lanes of a strip or of its rows
SIDES = [(40, 56), (64, 64), (100, 37), (130, 200), (9, 9), (256, 90)]
KW = dict(gamma=1.4, limiter="Minmod", riemann="HLLC", bc=["NullGradient"] * 4)


def configs(sides=SIDES):
    return [dict(nx=list(s), **KW) for s in sides]


def initial(dom, p):
    from heraclespp_b200 import setups

    return setups.four_quadrant(setups.Grid.from_domain(dom), seed=100 + p)


def single(p, nx, strip_rows):
    from heraclespp_b200 import Domain

    d = Domain(2, nx, precision="fp32_mixed", **KW)
    d.set_schedule({32: 3, 64: 4, 128: 5}[strip_rows])
    d.set_state_from_prim(*initial(d, p))
    return d


def make_ensemble(sides=SIDES):
    from heraclespp_b200 import Ensemble

    ens = Ensemble(configs(sides))
    for p, d in enumerate(ens.domains):
        d.set_state_from_prim(*initial(d, p))
    return ens


@pytest.mark.parametrize("strip_rows,use_graph,nw", [(64, False, 4), (32, True, 4), (128, True, 4), (64, True, 16),
                                                     (32, False, 16)])
def test_ensemble_matches_single_problem_kernel(strip_rows, use_graph, nw):
    n = 24
    ens = make_ensemble()
    r = ens.run(n, strip_rows=strip_rows, use_graph=use_graph, warps_per_cta=nw)
    assert r.status == 0 and r.strip_rows == strip_rows and r.launches == 1 and r.warps_per_cta == nw
    assert r.graph == (1 if use_graph else 0)
    assert r.cells == sum(a * b for a, b in SIDES)
    for p, (nx, d_e) in enumerate(zip(SIDES, ens.domains)):
        d = single(p, list(nx), strip_rows)
        d.run(nsteps=n)
        for a, b in zip(d_e.get_state(), d.get_state()):
            assert np.array_equal(a, b), f"problem {p}"
        assert np.array_equal(d_e.dt_log(), d.dt_log())
    ens.close()


def test_ensemble_autotune_and_continue_with_run():
    """Autotuned schedule; 10 ensemble steps then 14 hcl_run steps on each
    handle equal 24 single-problem steps."""
    ens = make_ensemble()
    r = ens.run(10)
    assert r.strip_rows in (32, 64, 128) and r.blocks_per_sm >= 1 and r.grid >= r.blocks_per_sm
    assert r.warps_per_cta in (4, 16)
    for p, (nx, d_e) in enumerate(zip(SIDES, ens.domains)):
        res = d_e.run(nsteps=14)
        assert res.iter == 24
        d = single(p, list(nx), r.strip_rows)
        res1 = d.run(nsteps=24)
        assert res.t == res1.t
        for a, b in zip(d_e.get_state(), d.get_state()):
            assert np.array_equal(a, b), f"problem {p}"
    # and a second ensemble run resumes from where the handles stand
    r2 = ens.run(6, strip_rows=r.strip_rows)
    assert r2.status == 0
    assert all(d.dt_log().size == 30 for d in ens.domains)
    ens.close()


def test_ensemble_rejects_bad_configs():
    from heraclespp_b200 import Ensemble, HclError

    with pytest.raises(HclError):
        Ensemble([dict(nx=[32, 32], **KW), dict(nx=[32, 32], **{**KW, "riemann": "HLL"})])
    with pytest.raises(HclError):
        Ensemble([dict(nx=[32, 32], **KW), dict(nx=[32, 32], precision="fp64", **KW)])
    ens = make_ensemble(SIDES[:2])
    with pytest.raises(HclError):
        ens.run(4, strip_rows=48)
    with pytest.raises(HclError):
        ens.run(4, warps_per_cta=8)
    ens.close()


def total_energy_lam(d):
    """lam_final of J = sum_p sum_cells E_p dV (rho, rhou, E planes; zero ghosts)."""
    import torch

    ng = 2
    lam = torch.zeros((d.ndim + 2,) + d.shape3, dtype=torch.float64, device="cuda")
    g = d.grid()
    lam[d.ndim + 1, :, ng:-ng, ng:-ng] = torch.from_numpy(g["dv"][:, ng:-ng, ng:-ng]).cuda()
    return lam


@pytest.mark.parametrize("precision", ["fp64", "fp32_mixed"])
def test_ensemble_adjoint_matches_single_adjoint(precision):
    import torch

    n, k = 30, 8
    ens = make_ensemble()
    r = ens.run(n, strip_rows=64, checkpoint_every=k, adjoint_precision=precision)
    assert r.launches == (n + k - 1) // k
    lams = [total_energy_lam(d) for d in ens.domains]
    grads = [torch.empty_like(x) for x in lams]
    torch.cuda.synchronize()  # the sweeps run on the handles' own streams
    ens.adjoint(lams, grads)
    torch.cuda.synchronize()
    for p, (nx, d_e) in enumerate(zip(SIDES, ens.domains)):
        d = single(p, list(nx), 64)
        dts = d.adjoint_forward(n, cfl=0.4, checkpoint_every=k, precision=precision)
        assert np.array_equal(dts, d_e.dt_log()[:n])
        g1 = torch.empty_like(lams[p])
        d.adjoint_backward(lams[p], g1, device=True)
        torch.cuda.synchronize()
        # same forward trajectory and sweep; atomics reorder the sums (FP32
        # shared-memory accumulators in the mixed sweep)
        scale = float(torch.max(torch.abs(g1)))
        tol = 1e-12 if precision == "fp64" else 1e-4
        assert float(torch.max(torch.abs(grads[p] - g1))) <= tol * scale, f"problem {p}"
        # the objective is not trivial: outflow boundaries let energy leave
        E_grad = grads[p][3, 0, 2:-2, 2:-2]
        dv = lams[p][3, 0, 2:-2, 2:-2]
        assert torch.any(E_grad != dv)
    ens.close()
