"""CPU check of the adjoint assembly: the loop-based reference of one step and
its adjoint (tests/adjoint_reference.py) against central finite differences
on a small smooth periodic 2-D state."""
import numpy as np
import pytest

from adjoint_reference import NG, Ref, build_cell_lib, smooth_state


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    return build_cell_lib(tmp_path_factory.mktemp("adjstep") / "libadjcheck.so")


@pytest.mark.parametrize("lim,solver", [(1, 1), (2, 0), (3, 1)])
def test_one_step_adjoint_matches_fd(lib, lim, solver):
    n = 6
    ref = Ref(lib, lim=lim, solver=solver)
    U = smooth_state(n, seed=lim)
    dt, dx = 0.02, (1.0 / n, 1.0 / n)
    rng = np.random.default_rng(5)
    lam = np.zeros_like(U)
    lam[:, NG:NG + n, NG:NG + n] = rng.normal(size=(4, n, n))
    g = ref.step_adjoint(U, lam, dt, dx)

    def J(Ux):
        Ux = Ux.copy()
        Ref.fill_periodic(Ux)
        out = ref.step(Ux, dt, dx)
        return float(np.sum(lam[:, NG:NG + n, NG:NG + n] * out[:, NG:NG + n, NG:NG + n]))

    for _ in range(4):
        v = np.zeros_like(U)
        v[:, NG:NG + n, NG:NG + n] = rng.uniform(-1, 1, (4, n, n))
        eps = 1e-6
        fd = (J(U + eps * v) - J(U - eps * v)) / (2 * eps)
        ad = float(np.sum(g * v))
        assert ad == pytest.approx(fd, rel=1e-6, abs=1e-9)
