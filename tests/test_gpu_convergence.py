"""Convergence of the device solver on the smooth isentropic MHD vortex (GPU).

The vortex convergence study is one of the workloads this path serves: the vortex of the problems
module advected with velocity (1, 1) on [-10, 10]^2, periodic, against its exact solution
(problems.vortex_exact).  Here to t = 0.5 on two meshes, with the mean absolute nodal error over
the momentum and field components:

  * OEDG off (LDF and the positivity limiter on, neither active on this smooth flow): order
    >= p + 0.6 for p = 1, 2, 3 on 32^2 -> 64^2 (the oracle gives 1.8, 2.9, 4.1);
  * OEDG on: order >= p + 0.6 for p = 1, 2 on 64^2 -> 128^2 (the oracle gives 2.1, 3.9).  At p = 3
    these meshes are still pre-asymptotic for the damping (the oracle gives 1.1 on 32^2 -> 64^2),
    so p = 3 with OEDG is not asserted here.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

T = 0.5


def _error(pkg, n, p, oedg):
    prob = pkg.problems.make("vortex")
    with pkg.DGSolver.for_problem(prob, n, n, p) as g:
        st = g.solve_execute(prob.initial_state(n, n, p), T, prob.cfl, oedg, 1, 0)
        u = g.download_state(0)[:, :, :, 1:-1, 1:-1]
    assert st["flags"] == 0 and abs(st["t"] - T) <= 1e-14 * T
    ex = pkg.problems.vortex_exact(n, n, p, st["t"])
    return np.abs(u - ex)[[1, 2, 4, 5]].mean()


@pytest.mark.parametrize("p,oedg,meshes", [(1, 0, (32, 64)), (2, 0, (32, 64)), (3, 0, (32, 64)),
                                           (1, 1, (64, 128)), (2, 1, (64, 128))])
def test_vortex_converges_at_the_design_order(pkg, p, oedg, meshes):
    coarse, fine = (_error(pkg, n, p, oedg) for n in meshes)
    order = np.log2(coarse / fine)
    assert order >= p + 0.6, (p, oedg, coarse, fine, order)
