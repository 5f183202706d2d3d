"""CPU checks of the serving driver's arrival process and percentile rule."""
import numpy as np

from blastp_b200 import serving


def test_poisson_arrivals_rate_and_order():
    rng = np.random.default_rng(0)
    a = serving.poisson_arrivals(rng, 1000.0, 20000)
    assert a[0] == 0.0 and np.all(np.diff(a) >= 0)
    assert abs(np.mean(np.diff(a)) - 1e-3) < 5e-5
    assert len(serving.poisson_arrivals(rng, 5.0, 0)) == 0


def test_percentile_nearest_rank():
    v = list(range(1, 101))
    assert serving.percentile(v, 50) == 50
    assert serving.percentile(v, 99) == 99
    assert serving.percentile([7.0], 99) == 7.0
    assert serving.percentile([], 50) == 0.0


class FakeServer:
    """The server calls the driver makes, with each request finishing a
    fixed time after its submission (on the host clock)."""

    def __init__(self, service_s):
        import time
        self.clock = time.perf_counter
        self.service = list(service_s)
        self.submitted, self.released = {}, {}

    def submit(self, q):
        t = len(self.submitted)
        self.submitted[t] = (self.clock(), q)
        return t

    def _done_at(self, t):
        return self.submitted[t][0] + self.service[t]

    def state(self, t):
        return 3 if self.clock() >= self._done_at(t) else 2

    def wait(self, t):
        import time
        d = self._done_at(t) - self.clock()
        if d > 0:
            time.sleep(d)

    def latency(self, t):
        assert self.state(t) == 3
        return 1e3 * self.service[t]

    def result(self, t):
        return ("result", self.submitted[t][1]), self.latency(t)

    def digest(self, t):
        assert t not in self.released
        return (t, 0)

    def release(self, t):
        assert t not in self.released and self.state(t) == 3
        self.released[t] = self.clock()


def test_drive_releases_requests_as_they_finish():
    # request 0 runs 0.3 s; requests 1-3 (submitted 0.05 s apart) 0.01 s each:
    # they are read and released while request 0 still runs, before the last
    # submission; results, latencies and digests come back in request order
    # (a request whose digest is wanted is held until all are submitted)
    srv = FakeServer([0.3, 0.01, 0.01, 0.01])
    digests = []
    res, lat, late = serving.drive(srv, ["a", "b", "c", "d"], [0.0, 0.05, 0.1, 0.15], digests=digests,
                                   digest_first=1)
    assert [r[1] for r in res] == ["a", "b", "c", "d"]
    assert list(lat) == [300.0, 10.0, 10.0, 10.0]
    assert digests == [(0, 0)]
    assert set(srv.released) == {0, 1, 2, 3}
    t_last_submit = srv.submitted[3][0]
    assert srv.released[1] < t_last_submit and srv.released[2] < t_last_submit
    assert srv.released[1] < srv._done_at(0)
    assert max(late) < 20.0


def test_drive_without_release_keeps_everything():
    srv = FakeServer([0.02, 0.01])
    res, lat, _ = serving.drive(srv, ["a", "b"], [0.0, 0.03], keep_results=False, release=False)
    assert res is None and list(lat) == [20.0, 10.0] and srv.released == {}


def test_drive_holds_digested_requests_until_all_are_submitted():
    srv = FakeServer([0.01, 0.01, 0.01])
    digests = []
    serving.drive(srv, ["a", "b", "c"], [0.0, 0.05, 0.1], keep_results=False, digests=digests, digest_first=2)
    assert digests == [(0, 0), (1, 0)]
    assert srv.released[0] > srv.submitted[2][0] and srv.released[1] > srv.submitted[2][0]
