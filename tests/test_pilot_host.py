"""Host-side logic of the learned pilot's training (no GPU): the collapse
detector that restarts a run whose network went dead."""
from isp_mw_b200 import pilot


def _hist(first, last, n=2000):
    return [(i, first if i < 50 else last) for i in range(n)]


def test_converged_run_is_not_collapsed():
    assert not pilot.collapsed(_hist(1.5e-2, 4e-4))


def test_dead_network_is_collapsed():
    # a dead network passes the noisy plane through: the loss stays at the
    # noisy-vs-basic error it started from
    assert pilot.collapsed(_hist(1.5e-2, 1.2e-2))


def test_short_runs_are_never_flagged_as_collapsed():
    assert not pilot.collapsed(_hist(1.5e-2, 1.5e-2, n=100))
