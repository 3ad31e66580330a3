"""hcl_hydro_reconstruction_noalloc (fixed device scratch, no allocation in
the call) against hcl_hydro_reconstruction (the handle's own scratch), through
the C ABI: identical face states on two calls in a row, and a clear error for
grids whose scratch does not fit the fixed array.  Collected last so that it
also runs after every other test of the session."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

vp, i, d = C.c_void_p, C.c_int, C.c_double


def noalloc_lib():
    from heraclespp_b200 import lib

    L = lib()
    L.hcl_hydro_reconstruction_noalloc.argtypes = [vp, i, d] + [vp] * 9
    L.hcl_hydro_reconstruction_noalloc.restype = i
    return L


def inputs(torch, dom, nfx, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    N = int(np.prod(dom.n))
    nd = dom.ndim

    def u(lo, hi, n):
        return lo + (hi - lo) * torch.rand(n, generator=g, device="cuda", dtype=torch.float64)

    rho = u(0.5, 1.5, N)
    vel = u(-0.5, 0.5, N * nd)
    P = u(0.5, 1.5, N)
    fx = u(0.0, 1.0, N * max(nfx, 1))
    return rho, vel, P, fx


def outputs(torch, dom, nfx):
    N = int(np.prod(dom.n))
    nd = dom.ndim
    z = lambda n: torch.full((n,), float("nan"), device="cuda", dtype=torch.float64)  # noqa: E731
    return z(N * 2 * nd), z(N * 2 * nd * nd), z(N * 2 * nd), z(N * 2 * nd * max(nfx, 1))


@pytest.mark.parametrize("ndim,nx,nfx", [(1, [200], 0), (2, [64, 48], 0), (3, [20, 12, 16], 1)])
def test_noalloc_matches_handle_scratch_twice(ndim, nx, nfx):
    import torch

    from heraclespp_b200 import Domain
    from heraclespp_b200._native import check

    L = noalloc_lib()
    dom = Domain(ndim, nx, nfx=nfx, gamma=1.4, limiter="VanLeer", riemann="HLLC", g=(0.1, -0.2, 0.05))
    p = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    fxp = lambda t: p(t) if nfx else None  # noqa: E731
    ng_eff, dt = 1, 2e-3
    for call, seed in enumerate((1, 2)):
        rho, vel, P, fx = inputs(torch, dom, nfx, seed)
        ref = outputs(torch, dom, nfx)
        got = outputs(torch, dom, nfx)
        torch.cuda.synchronize()
        check(L.hcl_hydro_reconstruction(dom.h, ng_eff, dt, p(rho), p(vel), p(P), fxp(fx), p(ref[0]), p(ref[1]),
                                         p(ref[2]), fxp(ref[3]), None, None, None))
        check(L.hcl_hydro_reconstruction_noalloc(dom.h, ng_eff, dt, p(rho), p(vel), p(P), fxp(fx), p(got[0]),
                                                 p(got[1]), p(got[2]), fxp(got[3]), None))
        torch.cuda.synchronize()
        for a, b in zip(got, ref):
            # entries outside the reconstructed range stay NaN in both
            np.testing.assert_array_equal(a.cpu().numpy(), b.cpu().numpy(), err_msg=f"call {call}")
        assert torch.isfinite(ref[0]).any()
    dom.close()


def test_noalloc_rejects_grids_beyond_the_fixed_scratch():
    import torch

    from heraclespp_b200 import Domain, HclError
    from heraclespp_b200._native import check

    L = noalloc_lib()
    dom = Domain(2, [600, 600], gamma=1.4)  # (600 + 4)^2 cells x 12 doubles > 2^22
    x = torch.zeros(1, device="cuda", dtype=torch.float64)
    p = C.c_void_p(x.data_ptr())
    rc = L.hcl_hydro_reconstruction_noalloc(dom.h, 1, 1e-3, p, p, p, None, p, p, p, None, None)
    assert rc != 0
    with pytest.raises(HclError, match="fixed buffer"):
        check(rc)
    dom.close()
