"""Schedule and Observer: the time grid of a filter run and the observations
at its times (share/src/bi/state/Schedule.hpp:107-315,
share/src/bi/state/ScheduleElement.hpp:17-238,
share/src/bi/simulator/Observer.hpp:97-126), driving the C ABI's steps.

Observations come in LibBi's sparse layout: three equal-length arrays of
observation times, observed component indices and values (the time,
coordinate and value variables of an observation file).  The schedule is
the grid of multiples of the transition's delta from t0, merged with the
observation and output times; every observation time must lie on that grid
(the transition block draws its noise once per delta).  Running a schedule
is Filter::filter with BootstrapPF::step per element: an observed element
is bpf_step_sparse with that time's components, an unobserved one a predict
only (bpf_step_sparse with none)."""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional

import numpy as np


class Observer:
    """Observations grouped by time: Observer::update / getMask."""

    def __init__(self, times, coords, values):
        t = np.asarray(times, dtype=np.float64).reshape(-1)
        c = np.asarray(coords, dtype=np.int64).reshape(-1)
        v = np.asarray(values, dtype=np.float64).reshape(-1)
        if not (t.size == c.size == v.size):
            raise ValueError("times, coords and values must have equal length")
        if (c < 0).any():
            raise ValueError("component indices must be non-negative")
        order = np.lexsort((c, t))
        t, c, v = t[order], c[order], v[order]
        self.times = np.unique(t)
        self._groups = []
        for tt in self.times:
            sel = t == tt
            cc = c[sel]
            if np.unique(cc).size != cc.size:
                raise ValueError(f"component observed twice at time {tt}")
            self._groups.append((cc.astype(np.int32), v[sel]))

    def __len__(self):
        return self.times.size

    def get(self, k: int):
        """(component indices, values) of the k-th observation time (its Mask)."""
        return self._groups[k]


@dataclass
class ScheduleElement:
    time: float
    observed: bool
    index_obs: int      # observation index when observed, else -1
    output: bool


class Schedule:
    """The ordered, de-duplicated grid of a run: t0, the multiples of delta up
    to the last time, observation times and output times."""

    def __init__(self, t0: float, delta: float, observer: Optional[Observer] = None, output_times=(),
                 t_end: Optional[float] = None, tol: float = 1e-9):
        if not delta > 0:
            raise ValueError("delta must be positive")
        obs_t = observer.times if observer is not None else np.zeros(0)
        out_t = np.asarray(output_times, dtype=np.float64).reshape(-1)
        last = max([t0] + list(obs_t) + list(out_t) + ([t_end] if t_end is not None else []))
        nsteps = int(round((last - t0) / delta))
        if t0 + nsteps * delta < last - tol * max(1.0, abs(last)):
            nsteps += 1
        grid = t0 + delta * np.arange(nsteps + 1)

        def on_grid(t):
            k = int(round((t - t0) / delta))
            return 0 <= k <= nsteps and abs(grid[k] - t) <= tol * max(1.0, abs(t)), k

        obs_at = {}
        for i, t in enumerate(obs_t):
            ok, k = on_grid(t)
            if not ok or k == 0:
                raise ValueError(f"observation time {t} is not a multiple of delta after t0")
            obs_at[k] = i
        out_at = set()
        for t in out_t:
            ok, k = on_grid(t)
            if not ok:
                raise ValueError(f"output time {t} is not on the schedule's grid")
            out_at.add(k)
        self.elements: List[ScheduleElement] = [
            ScheduleElement(float(grid[k]), k in obs_at, obs_at.get(k, -1), k in out_at) for k in range(nsteps + 1)
        ]
        self.observer = observer

    def __len__(self):
        return len(self.elements)

    def run(self, pf):
        """Filter::filter over the schedule with a BootstrapPF (or its
        subclass): returns dict(loglik, log_increments, ess, resampled) with
        one entry per observed element."""
        pf.init()
        inc, ess, res = [], [], []
        ll = 0.0
        for prev, el in zip(self.elements[:-1], self.elements[1:]):
            if el.observed:
                idx, vals = self.observer.get(el.index_obs)
                r = pf.step_sparse(prev.time, el.time, vals, idx)
                inc.append(r.log_increment)
                ess.append(r.ess)
                res.append(r.resampled)
                ll = r.log_likelihood
            else:
                pf.step_sparse(prev.time, el.time, [], [])
        return dict(loglik=ll, log_increments=np.array(inc), ess=np.array(ess), resampled=np.array(res))
