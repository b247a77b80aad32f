"""Host logic of the Schedule and Observer (share/src/bi/state/Schedule.hpp,
share/src/bi/simulator/Observer.hpp): grouping of sparse observations by
time, the merged grid, and the validation of times."""
import numpy as np
import pytest

from libbi_b200.schedule import Observer, Schedule


def test_observer_groups_sparse_observations_by_time():
    obs = Observer([0.1, 0.05, 0.1, 0.05, 0.2], [3, 7, 1, 2, 0], [1.0, 2.0, 3.0, 4.0, 5.0])
    assert list(obs.times) == [0.05, 0.1, 0.2]
    idx, val = obs.get(0)
    assert list(idx) == [2, 7] and list(val) == [4.0, 2.0]
    idx, val = obs.get(1)
    assert list(idx) == [1, 3] and list(val) == [3.0, 1.0]
    with pytest.raises(ValueError):
        Observer([0.1, 0.1], [2, 2], [1.0, 1.0])
    with pytest.raises(ValueError):
        Observer([0.1], [1, 2], [1.0])


def test_schedule_merges_the_delta_grid_observations_and_outputs():
    obs = Observer([0.15, 0.05], [0, 1], [1.0, 2.0])
    s = Schedule(0.0, 0.05, obs, output_times=[0.1, 0.25])
    times = [e.time for e in s.elements]
    np.testing.assert_allclose(times, [0.0, 0.05, 0.1, 0.15, 0.2, 0.25])
    assert [e.observed for e in s.elements] == [False, True, False, True, False, False]
    assert [e.index_obs for e in s.elements] == [-1, 0, -1, 1, -1, -1]
    assert [e.output for e in s.elements] == [False, False, True, False, False, True]
    with pytest.raises(ValueError):
        Schedule(0.0, 0.05, Observer([0.07], [0], [1.0]))
    with pytest.raises(ValueError):
        Schedule(0.0, 0.05, Observer([0.0], [0], [1.0]))
    assert len(Schedule(1.0, 1.0, None, t_end=4.0)) == 4
