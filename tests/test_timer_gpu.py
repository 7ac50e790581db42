"""tbs_resid_timer: the device-clock record of the sweeps' residual
launches counts every one of them, graph-launched solves included, and its
average is bracketed by CUDA events around the same kernel launched
eagerly: at most the events' time plus 5 % (the record runs from the
earliest CTA start to the last CTA's finish, the events also hold the
launch's own start-up) and at least half of it."""
import pytest

from triblocksolve_b200 import ALGO_FP64, Jacobian, Mesh, Solver

pytestmark = pytest.mark.gpu


def test_timer_counts_graph_launches_and_agrees_with_events():
    mesh = Mesh.structured(600, 640)
    jac = Jacobian.generate(mesh, 9.0, 3)
    s = Solver(0)
    try:
        s.set_mesh(mesh)
        s.set_jacobian(jac)
        s.factor(ALGO_FP64)
        s.solve(1e-10, 200)                       # builds the graph
        s.resid_timer(reset=True)
        total = 0
        for _ in range(3):
            n, _h = s.solve(1e-10, 200)
            total += n
        us, launches = s.resid_timer(reset=True)
        assert launches == total                  # one residual launch per sweep
        assert us > 0.0
        s.profile(True)
        s.profile_reset()
        for _ in range(3):
            s.solve(1e-10, 200)
        prof = s.profile_read()
        s.profile(False)
        n_ev, ms_ev = prof["fast_resid"]
        ev_us = 1e3 * ms_ev / n_ev
        assert 0.5 * ev_us <= us / launches <= 1.05 * ev_us, (us / launches, ev_us)
        us2, n2 = s.resid_timer()                 # the eager launches are recorded too
        assert n2 == n_ev and us2 > 0.0
    finally:
        s.close()
