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
    With `release`, every request is collected (result or latency, digest)
    and released as soon as it finishes, also between submissions, the way a
    serving client frees what it has read: results held by the server count
    against its device-memory budget.  With a list as `digests`, the result
    digests of the first `digest_first` requests are appended to it, in
    request order; those requests are held until every request has been
    submitted (a digest runs on the device and could wait for SMs the
    running search holds, which would delay submissions)."""
    n = len(queries)
    results = [None] * n
    lat = np.zeros(n)
    got = {}
    tickets, late, open_ = [], [], []

    def collect(i):
        t = tickets[i]
        if digests is not None and i < digest_first:
            got[i] = server.digest(t)
        if keep_results:
            results[i], lat[i] = server.result(t)
        else:
            lat[i] = server.latency(t)
        if release:
            server.release(t)

    def poll():
        still = []
        for i in open_:
            if (digests is None or i >= digest_first) and server.state(tickets[i]) >= 3:   # done or failed
                collect(i)
            else:
                still.append(i)
        open_[:] = still

    t0 = time.perf_counter()
    for i, (q, at) in enumerate(zip(queries, arrivals)):
        while True:
            d = at - (time.perf_counter() - t0)
            if d <= 0:
                break
            if release and open_:
                poll()
                d = at - (time.perf_counter() - t0)
            if d > 0:
                time.sleep(min(d, 0.001) if release and open_ else d)
        late.append(max(0.0, (time.perf_counter() - t0 - at) * 1e3))
        tickets.append(server.submit(q))
        open_.append(i)
    for i in open_:
        server.wait(tickets[i])
        collect(i)
    if digests is not None:
        digests.extend(got[i] for i in range(min(digest_first, n)))
    return (results if keep_results else None), lat, np.array(late)
