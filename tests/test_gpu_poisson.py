"""GPU parity of the Poisson (inverse Laplacian) FMM, through the C ABI,
against the reference's own solve (tests/golden/make_golden_poisson.py), and
the sh43 known answer on a grid with exact Clenshaw-Curtis weights.

Tolerances: <= 1e-12 relative against the reference; the known answer within
the discretisation error of the log kernel's quadrature (the same sum taken
directly is 2.6e-2 from f/20 at levels 5)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

CASES = ("poisson_L4.npz", "poisson_L3_d2.npz")


def rel(a, b):
    a = a.detach().cpu().numpy() if hasattr(a, "detach") else np.asarray(a)
    return float(np.abs(a - b).max() / np.abs(b).max())


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def ctx_for(sb, levels, degree, theta):
    return sb.Context(sb.config_default(levels=levels, interp_degree=degree, fmm_theta=theta, kernel_eps=1e-4,
                                        omega=2 * np.pi, dt=1.0))


@pytest.mark.parametrize("name", CASES)
def test_poisson_fmm_matches_reference(sb, name):
    gd = dict(np.load(os.path.join(GOLDEN, name)))
    ctx = ctx_for(sb, int(gd["levels"]), int(gd["degree"]), float(gd["theta"]))
    soln = torch.zeros_like(cuda(gd["pots"]))
    ctx.poisson_fmm(cuda(gd["area"]), cuda(gd["pots"]), soln)
    assert rel(soln, gd["soln"]) <= 1e-12, rel(soln, gd["soln"])
    tgt = cuda(gd["rand_target_in"])
    ctx.poisson_fmm_interactions(cuda(gd["rand_source"]), tgt)
    assert rel(tgt, gd["rand_target_out"]) <= 1e-12
    # downward pass alone on the reference's proxy targets
    t = cuda(gd["proxy_target"])
    s = torch.zeros_like(soln)
    pt = torch.zeros_like(t)
    ctx.poisson_fmm_interactions(cuda(gd["proxy_source"]), pt)
    ctx.downward_pass(pt, s)
    assert rel(s, gd["soln"]) <= 1e-12 and rel(pt, gd["proxy_target"]) <= 1e-12


def test_poisson_fmm_known_answer(sb):
    g = sb.build_grid(5, 3, exact_cc=True)
    f = 1.770130769779931 * g.x * (g.x * g.x - 3.0 * g.y * g.y) * g.z
    ctx = ctx_for(sb, 5, 3, 0.7)
    soln = torch.zeros_like(cuda(f))
    ctx.poisson_fmm(cuda(g.area), cuda(f), soln)
    err = rel(soln, f / 20)
    print("Poisson FMM vs f/20 at levels 5: %.2e" % err)
    assert err <= 5e-2
