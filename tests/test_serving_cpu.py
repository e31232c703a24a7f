"""The serving scheduler (he_dft_2024_b200/serving.py) on the CPU with a fake context: grid choice,
seeded request stream, HBM-budget admission, continuous batching and context reuse.  The device
parity of served trajectories is in test_gpu_serving.py."""
import numpy as np
import pytest

from he_dft_2024_b200 import serving as S


def test_grid_choice():
    for n4 in (300, 1000, 3000, 10000):
        n, h = S.grid_for(n4)
        R = 2.22 * n4 ** (1.0 / 3.0)
        assert n * h / 2 >= R + S.MARGIN
        smaller = [g for g in S.GRIDS if g < n]
        assert all(g * S.H_MAX / 2 < R + S.MARGIN for g in smaller)
        assert S.H_MIN <= h <= S.H_MAX and h in S.H_STEPS
        # the finest served spacing whose box still holds the droplet
        assert all(n * f / 2 < R + S.MARGIN for f in S.H_STEPS if f < h)
    # a droplet whose box fits 128^3 at 0.6 A gets 0.6 A there (N = 1000: R + 15 = 37.2 A)
    assert S.grid_for(1000) == (128, 0.6)


def test_request_stream_is_seeded():
    a = S.make_requests(count=20, seed=7)
    b = S.make_requests(count=20, seed=7)
    assert [(r.arrival_s, r.n4, r.speed_ms) for r in a] == [(r.arrival_s, r.n4, r.speed_ms) for r in b]
    assert all(300 <= r.n4 <= 10000 and 100 <= r.speed_ms <= 500 for r in a)
    assert all(x.arrival_s < y.arrival_s for x, y in zip(a, a[1:]))


class FakeCtx:
    """Records the call surface the scheduler drives; each context holds 1 GB."""
    made = 0

    def __init__(self, w):
        FakeCtx.made += 1
        self.w = w
        self.device_bytes = 1e9
        self.calls = []
        self.steps = 0

    def _shape(self, name):
        return (1, 3)

    def set_impurities(self, w):
        self.calls.append("set_impurities")
        self.steps = 0

    def upload(self, name, a):
        self.calls.append("upload:" + name)

    def download(self, name):
        return np.zeros((1, 3))

    def potenimp(self): self.calls.append("potenimp")
    def poten(self): self.calls.append("poten")
    def forceimp(self, want=False): self.calls.append("forceimp")
    def set_accel(self): self.calls.append("set_accel")

    def steprk(self, dt):
        self.steps += 1
        self.calls.append("steprk")

    def steppc(self, dt, errors=False):
        self.steps += 1
        self.calls.append("steppc")

    def synchronize(self): pass
    def energy(self): return {"etot": float(self.steps)}
    def close(self): pass


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        self.t += 0.01  # every clock read advances 10 ms
        return self.t

    def sleep(self, s):
        self.t += s


def reqs(k, steps=6, n=32, spacing=0.05):
    out = []
    for i in range(k):
        r = S.Request(rid=i, arrival_s=i * spacing, n4=200, speed_ms=200.0, steps=steps)
        r.n, r.h = n, 0.7
        out.append(r)
    return out


def test_every_request_completes_with_its_step_count():
    FakeCtx.made = 0
    clk = FakeClock()
    srv = S.Server(FakeCtx, hbm_budget_gb=100, clock=clk, sleep=clk.sleep)
    rs = reqs(5, steps=7)
    rep = srv.run(rs, dt_for=lambda r: 1e-5)
    assert rep["requests"] == 5
    for r in rs:
        assert r.final["energy"]["etot"] == 7
        assert len(r.step_ms) == 7
        assert r.arrival_s <= r.admitted_s <= r.done_s
    assert rep["step_ms_p50"] > 0 and rep["trajectory_s_p99"] >= rep["trajectory_s_p50"]


def test_budget_limits_concurrency_and_contexts_are_reused():
    FakeCtx.made = 0
    clk = FakeClock()
    srv = S.Server(FakeCtx, hbm_budget_gb=2.0, clock=clk, sleep=clk.sleep)
    rs = reqs(6, steps=4, spacing=0.0)
    srv.run(rs, dt_for=lambda r: 1e-5)
    assert srv.peak_active <= 2
    assert FakeCtx.made == 2          # two contexts serve all six trajectories
    # continuous batching: the third request starts when one of the first two finishes
    first_done = min(rs[0].done_s, rs[1].done_s)
    assert rs[2].admitted_s >= first_done


def test_driver_sequence_per_trajectory():
    FakeCtx.made = 0
    clk = FakeClock()
    made = []

    def mk(w):
        c = FakeCtx(w)
        made.append(c)
        return c

    srv = S.Server(mk, hbm_budget_gb=100, clock=clk, sleep=clk.sleep)
    srv.run(reqs(1, steps=5), dt_for=lambda r: 1e-5)
    calls = [c for c in made[0].calls if c in ("steprk", "steppc")]
    assert calls == ["steprk"] * 3 + ["steppc"] * 2   # DFT4He3d.f90:677-684
    assert made[0].calls.index("set_impurities") < made[0].calls.index("steprk")


def test_max_active_caps_concurrency():
    FakeCtx.made = 0
    clk = FakeClock()
    srv = S.Server(FakeCtx, hbm_budget_gb=100, clock=clk, sleep=clk.sleep, max_active=2)
    rs = reqs(5, steps=3, spacing=0.0)
    srv.run(rs, dt_for=lambda r: 1e-5)
    assert srv.peak_active == 2
    assert all(r.final is not None for r in rs)


def test_device_step_timer_gets_one_interval_per_trajectory_and_tick():
    class Timer:
        def __init__(self):
            self.open, self.n = [], 0

        def start(self, ctx):
            self.open.append(ctx)

        def stop(self, ctx):
            assert self.open[-1] is ctx

        def intervals(self):
            out = [1.5] * len(self.open)
            self.open = []
            return out

    FakeCtx.made = 0
    clk = FakeClock()
    srv = S.Server(FakeCtx, hbm_budget_gb=100, clock=clk, sleep=clk.sleep, step_timer=Timer())
    rs = reqs(3, steps=5, spacing=0.0)
    rep = srv.run(rs, dt_for=lambda r: 1e-5)
    for r in rs:
        assert r.device_step_ms == [1.5] * 5
    assert rep["device_step_ms_p50"] == 1.5 and rep["device_step_ms_p99"] == 1.5
