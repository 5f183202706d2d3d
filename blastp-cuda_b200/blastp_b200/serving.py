"""Open-loop request driver for the serving loop: Poisson arrivals of
synthetic queries (log-normal lengths), submitted on schedule from one
thread, then collected.  Latency is the server's own arrival-to-completion
time of each request."""
from __future__ import annotations

import time

import numpy as np


def poisson_arrivals(rng: np.random.Generator, rate_per_s: float, n: int) -> np.ndarray:
    """Arrival times (s, from 0) of n requests at a Poisson rate."""
    if n == 0:
        return np.zeros(0)
    gaps = rng.exponential(1.0 / rate_per_s, size=n)
    return np.cumsum(gaps) - gaps[0]


def percentile(values, p: float) -> float:
    """Nearest-rank percentile (the same rule as the server's statistics)."""
    v = np.sort(np.asarray(values, dtype=np.float64))
    if len(v) == 0:
        return 0.0
    i = int(min(len(v) - 1, max(0, np.ceil(p / 100.0 * len(v)) - 1)))
    return float(v[i])


def drive(server, queries, arrivals, keep_results: bool = True, release: bool = True, digests=None,
          digest_first: int = 0):
    """Submits queries[i] at arrivals[i] (seconds after the call), waits for
    all, and returns (results or None, latencies in ms, submit lateness in ms).
    With a list as `digests`, the result digests of the first `digest_first`
    requests are appended to it (taken after every request was submitted, so
    they do not delay submissions)."""
    t0 = time.perf_counter()
    tickets, late = [], []
    for q, at in zip(queries, arrivals):
        d = at - (time.perf_counter() - t0)
        if d > 0:
            time.sleep(d)
        late.append(max(0.0, (time.perf_counter() - t0 - at) * 1e3))
        tickets.append(server.submit(q))
    results, lat = [], []
    for i, t in enumerate(tickets):
        server.wait(t)
        if digests is not None and i < digest_first:
            digests.append(server.digest(t))
        if keep_results:
            r, ms = server.result(t)
            results.append(r)
        else:
            ms = server.latency(t)
        lat.append(ms)
        if release:
            server.release(t)
    return (results if keep_results else None), np.array(lat), np.array(late)
