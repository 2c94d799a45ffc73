"""CPU tests of the seeded workload generators."""
import numpy as np

from hawkes_b200 import workloads


def test_uniform_is_seeded_sorted_and_in_range():
    a_loc, a_t = workloads.uniform(1000, seed=0)
    b_loc, b_t = workloads.uniform(1000, seed=0)
    assert np.array_equal(a_loc, b_loc) and np.array_equal(a_t, b_t)
    assert a_loc.shape == (1000, 2)
    assert np.all(np.diff(a_t) >= 0)
    assert a_loc.min() >= 0 and a_loc.max() < 20 and a_t.min() >= 0 and a_t.max() < 8760


def test_proposals_are_lognormal_around_base():
    p = workloads.proposals(256, seed=2)
    assert p.shape == (256, 6)
    z = np.log(p / workloads.BASE_PARAMS)
    assert abs(z.std() - 0.3) < 0.02


def test_uneven_sizes_are_log_uniform_in_range():
    sets = workloads.uneven(64, seed=3)
    sizes = np.array([len(t) for _, t, _ in sets])
    assert len(sets) == 64 and sizes.min() >= 1000 and sizes.max() <= 100000
    for loc, t, p in sets[:3]:
        assert loc.shape == (len(t), 2) and p.shape == (6,)


def test_clustered_branching_process_small():
    loc, t = workloads.clustered(N=20000, background=12000)
    assert loc.shape == (20000, 2)
    assert np.all(np.diff(t) >= 0) and t.max() < 8760
    # offspring add about as many events again as the background (mean 0.5 per
    # event, recursively), so the horizon is cut well before 8760 h
    assert t.max() < 8760
