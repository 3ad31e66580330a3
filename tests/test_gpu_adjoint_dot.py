"""Dot-product test of the discrete adjoint on the GPU: the library's gradient
g = J^T lambda (hcl_adjoint_forward/backward, FP64 sweep, checkpointed) against
tangent-linear products J v formed by forward-mode differentiation of a torch
FP64 restatement of the step (tests/tangent_step.py) on the same device:
<g, v> = <lambda, J v> must hold to rounding for every direction v.

Unlike central differences, the two sides differentiate the same branches
(limiter zero unless R*L > 0 as the forward forms it, wave-speed and
star-side selections), so the test holds on the plain Gresho vortex too, whose
flat and solid-body regions sit on the limiter's kink with slope differences
at rounding level, and at the full 512^2 x 400-step size of the adjoint
workload with checkpoints every 32 steps."""
import numpy as np
import pytest

from test_gpu_adjoint import problem

torch = pytest.importorskip("torch")
from tangent_step import TangentStep  # noqa: E402

pytestmark = pytest.mark.gpu

NG = 2

# (n, steps, checkpoint, smooth background, directions)
DOT_CASES = [(64, 40, 16, False, 6), (64, 40, 16, True, 6), (512, 400, 32, False, 6), (512, 400, 32, True, 4)]


def interior(a):
    return np.ascontiguousarray(a[:, 0, NG:-NG, NG:-NG])


@pytest.mark.parametrize("n,nsteps,k,smooth,ndir", DOT_CASES)
def test_adjoint_dot_product(n, nsteps, k, smooth, ndir):
    o, d, U0, dts, target = problem(n, nsteps, smooth=smooth)
    d.set_state(U0[0], U0[1:3], U0[3])
    d.adjoint_forward(len(dts), dts=dts, precision="fp64", checkpoint_every=k)
    rN = d.get_state()[0].copy()
    resid = (rN - target)[0, NG:-NG, NG:-NG]
    lam = np.zeros_like(U0)
    lam[0, 0, NG:-NG, NG:-NG] = resid
    g = d.adjoint_backward(lam)

    dev = torch.device("cuda:0")
    ts = TangentStep.from_grid(o.grid(), 5.0 / 3.0, "VanLeer", "HLLC")
    U = torch.from_numpy(interior(U0)).to(dev)

    # the restated forward follows the library's FP64 trajectory
    UN = ts.run(U, dts)[0].cpu().numpy()
    ref = rN[0, NG:-NG, NG:-NG]
    fwd_rel = float(np.abs(UN - ref).max() / np.abs(ref).max())
    print(f"n={n} steps={nsteps} smooth={smooth}: torch forward vs library max rel {fwd_rel:.2e} "
          f"({'bitwise' if np.array_equal(UN, ref) else 'not bitwise'})")
    assert fwd_rel < 1e-12

    rng = np.random.default_rng(99)
    errs = []
    res_t = torch.from_numpy(resid).to(dev)
    for _ in range(ndir):
        v = rng.uniform(-1, 1, (4, n, n)) * np.abs(interior(U0))
        _, JV = ts.jvp(U, torch.from_numpy(v).to(dev), dts)
        tl = float(torch.sum(res_t * JV[0]).item())
        ad = float(np.sum(interior(g) * v))
        errs.append(abs(ad - tl) / abs(tl))
    errs = np.array(errs)
    print(f"  <g, v> vs <lambda, J v>: rel err median {np.median(errs):.2e} max {errs.max():.2e}")
    assert np.median(errs) < 1e-12 and np.max(errs) < 1e-10, errs
