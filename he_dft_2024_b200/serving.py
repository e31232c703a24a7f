"""Serving loop: many independent droplet trajectories on one GPU with continuous batching.

The reference runs one trajectory per process (Dynamics_TDDFT/DFT4He3d.f90).  A service that takes
trajectory requests as they arrive needs, around the same call surface, a scheduler that

* picks each request's grid: the smallest n in GRIDS with n*h/2 >= R + MARGIN for some h in
  [H_MIN, H_MAX], R = 2.22 N^(1/3) (readen.f90:98), and then the finest spacing of H_STEPS
  (0.5, 0.6, 0.7 A) at which that box still holds the droplet; requests on the same (n, h) share
  k-space kernels, weights and absorber tables, and a retired trajectory's context serves the
  next request on that grid;
* admits requests while their device footprint fits an HBM budget (footprints are measured from
  the contexts themselves, he_device_bytes), queueing the rest in arrival order;
* advances every admitted trajectory by one driver iteration per tick (3 RK-Gill starts, then
  Hamming PMC, DFT4He3d.f90:677-697), trajectories grouped by grid so that the grid's contexts
  are issued back to back; each context has its own CUDA stream, so small grids overlap;
* retires finished trajectories at tick boundaries and admits waiting ones in their place
  (continuous batching), reusing the retired trajectory's context when the grid matches.

A context is reset for a new trajectory by uploading its initial state and zeroing the
integrator history (q, pc, psiold, hpsiold and the impurity rings), so a served trajectory is
bit-identical to the same request run alone in a fresh context (tested).

Device work goes through Context (the C-ABI); the scheduler itself is plain Python and takes any
object with Context's methods, which the CPU tests exploit.
"""
import math
import time
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional

import numpy as np

from . import config as C
from . import driver as D

GRIDS = (64, 96, 128, 160, 192, 256)
H_MIN, H_MAX = 0.5, 0.7
H_STEPS = (0.5, 0.6, 0.7)  # spacings served (requests on one (n, h) share contexts)
MARGIN = 15.0


def grid_for(n4: int):
    """(n, h) for a droplet of n4 atoms: the smallest admissible n whose box at h = H_MAX covers
    R + MARGIN, then the finest spacing of H_STEPS at which that box still covers it."""
    R = 2.22 * n4 ** (1.0 / 3.0)
    need = R + MARGIN
    for n in GRIDS:
        if n * H_MAX / 2.0 >= need:
            return n, next(h for h in H_STEPS if n * h / 2.0 >= need)
    raise ValueError(f"droplet of {n4} atoms does not fit the largest grid")


@dataclass
class Request:
    rid: int
    arrival_s: float
    n4: int
    speed_ms: float
    steps: int
    n: int = 0
    h: float = 0.0
    # filled by the server
    admitted_s: Optional[float] = None
    done_s: Optional[float] = None
    step_ms: List[float] = field(default_factory=list)       # tick times (the step as seen)
    device_step_ms: List[float] = field(default_factory=list)  # this trajectory's own step
    final: Optional[dict] = None

    def workload(self) -> C.Workload:
        """The request's workload: 4He_N Woods-Saxon droplet (not relaxed), one 85 u classical
        Morse impurity starting R + 8 A out on z, moving inward at speed_ms, dt = 0.1 fs."""
        xm = self.n * self.h / 2.0
        R = 2.22 * self.n4 ** (1.0 / 3.0)
        return C.replace(C.tddft_1000(n=self.n), name=f"serve-{self.rid}", xmax=xm, ymax=xm, zmax=xm,
                         n4=self.n4, rimp0=((0.0, 0.0, R + 8.0),),
                         vimp0_aps=((0.0, 0.0, -self.speed_ms / 100.0),), steps=self.steps)


def make_requests(count=128, rate_hz=20.0, n_min=300, n_max=10000, steps=1000, seed=1234,
                  speed=(100.0, 500.0)):
    """Seeded request stream: Poisson arrivals at rate_hz, N log-uniform in [n_min, n_max],
    impurity speed uniform in `speed` (m/s)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(count):
        t += rng.exponential(1.0 / rate_hz)
        n4 = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
        r = Request(rid=i, arrival_s=t, n4=n4, speed_ms=float(rng.uniform(*speed)), steps=steps)
        r.n, r.h = grid_for(n4)
        out.append(r)
    return out


HISTORY_FIELDS = ("q", "pc", "psiold1", "psiold2", "psiold3", "hpsiold1", "hpsiold2")
IMP_HISTORY = ("rimpold", "vimpold", "aimpold", "pcr", "pcv", "qr", "qv")


def start_trajectory(ctx, w: C.Workload):
    """Put a (fresh or reused) context at the start of w's trajectory: impurity set-up, zeroed
    integrator history, initial psi/den, then the driver's set-up calls."""
    ctx.set_impurities(w)
    z = np.zeros((w.nx, w.ny, w.nz), dtype=np.complex128)
    for f in HISTORY_FIELDS:
        ctx.upload(f, z)
    for f in IMP_HISTORY:
        ctx.upload(f, np.zeros(ctx._shape(f)))
    den = C.woods_saxon(w)
    D.dynamics_setup(ctx, D.initial_wavefunction(w, den), w.n_imp)


class _Active:
    def __init__(self, req, ctx, key):
        self.req, self.ctx, self.key = req, ctx, key
        self.it = 1


class Server:
    """Continuous-batching scheduler over per-grid context pools.

    make_context(workload) -> context (its device_bytes is the footprint charged against the
    budget; idle pooled contexts count too, and other grids' idle contexts are closed when they
    block an admission).  clock() returns seconds since the start of the run (wall time by
    default; tests pass a fake)."""

    def __init__(self, make_context: Callable, hbm_budget_gb=120.0, clock: Callable = None,
                 sleep: Callable = None, max_active: Optional[int] = None, step_timer=None):
        self.make_context = make_context
        # optional device timer: start(ctx) / stop(ctx) around each trajectory's iteration,
        # intervals() (after the tick's synchronisation) each one's device time in that order
        self.step_timer = step_timer
        self.budget = hbm_budget_gb * 1e9
        # cap on concurrently advancing trajectories: every active trajectory shares each tick,
        # so fewer active ones finish sooner (latency) at about the same aggregate throughput
        self.max_active = max_active
        self.pool: Dict[tuple, list] = {}
        self.bytes_of: Dict[tuple, int] = {}
        self.in_use = 0
        self.clock = clock
        self.sleep = sleep or time.sleep
        self.ticks = 0
        self.peak_bytes = 0
        self.peak_active = 0

    def _key(self, r):
        return (r.n, round(r.h, 12))

    def _acquire(self, r):
        key = self._key(r)
        pool = self.pool.setdefault(key, [])
        if pool:
            ctx = pool.pop()
        else:
            known = self.bytes_of.get(key)
            if known is not None and self.in_use + self._pooled_bytes() + known > self.budget:
                return None
            ctx = self.make_context(r.workload())
            self.bytes_of[key] = int(ctx.device_bytes)
        self.in_use += self.bytes_of[key]
        return ctx

    def _release(self, a):
        self.in_use -= self.bytes_of[a.key]
        self.pool.setdefault(a.key, []).append(a.ctx)

    def _pooled_bytes(self):
        return sum(self.bytes_of[k] * len(v) for k, v in self.pool.items())

    def run(self, requests: List[Request], dt_for=None):
        reqs = sorted(requests, key=lambda r: r.arrival_s)
        t0 = time.perf_counter()
        clock = self.clock or (lambda: time.perf_counter() - t0)
        waiting: List[Request] = []
        active: List[_Active] = []
        nxt = 0
        done = 0
        while done < len(reqs):
            now = clock()
            while nxt < len(reqs) and reqs[nxt].arrival_s <= now:
                waiting.append(reqs[nxt])
                nxt += 1
            # admission in arrival order while the HBM budget allows (pooled contexts of other
            # grids are freed first when they block an admission)
            still = []
            for r in waiting:
                if self.max_active is not None and len(active) >= self.max_active:
                    still.append(r)
                    continue
                ctx = self._acquire(r)
                if ctx is None and self._pooled_bytes() > 0:
                    self._drop_pool(keep=self._key(r))
                    ctx = self._acquire(r)
                if ctx is None:
                    still.append(r)
                    continue
                start_trajectory(ctx, r.workload())
                r.admitted_s = clock()
                active.append(_Active(r, ctx, self._key(r)))
            waiting = still
            if not active:
                if nxt < len(reqs):
                    self.sleep(max(0.0, reqs[nxt].arrival_s - clock()))
                    continue
                raise RuntimeError("requests cannot be admitted within the HBM budget")
            # one driver iteration for every active trajectory, grouped by grid
            active.sort(key=lambda a: a.key)
            ts = clock()
            for a in active:
                w_dt = a.req.workload().deltat if dt_for is None else dt_for(a.req)
                if self.step_timer:
                    self.step_timer.start(a.ctx)
                D.dynamics_iteration(a.ctx, a.it, w_dt, 1)
                if self.step_timer:
                    self.step_timer.stop(a.ctx)
            for a in active:
                a.ctx.synchronize()
            te = clock()
            if self.step_timer:
                for a, ms in zip(active, self.step_timer.intervals()):
                    a.req.device_step_ms.append(ms)
            self.ticks += 1
            self.peak_active = max(self.peak_active, len(active))
            self.peak_bytes = max(self.peak_bytes, self.in_use + self._pooled_bytes())
            keep = []
            for a in active:
                a.req.step_ms.append((te - ts) * 1e3)
                a.it += 1
                if a.it > a.req.steps:
                    a.req.done_s = te
                    a.req.final = {"rimp": a.ctx.download("rimp"), "energy": a.ctx.energy()}
                    self._release(a)
                    done += 1
                else:
                    keep.append(a)
            active = keep
        return self.report(reqs, clock())

    def _drop_pool(self, keep):
        for k in list(self.pool):
            if k == keep:
                continue
            for ctx in self.pool.pop(k):
                if hasattr(ctx, "close"):
                    ctx.close()

    def report(self, reqs, wall_s):
        steps = np.concatenate([np.asarray(r.step_ms) for r in reqs]) if reqs else np.zeros(1)
        dev = np.concatenate([np.asarray(r.device_step_ms) for r in reqs]) if reqs else np.zeros(0)
        lat = np.asarray([r.done_s - r.arrival_s for r in reqs])
        pts = float(sum(r.n ** 3 * r.steps for r in reqs))
        return {
            "requests": len(reqs),
            "ticks": self.ticks,
            "wall_s": wall_s,
            "grid_pt_steps_per_s": pts / wall_s if wall_s > 0 else None,
            "step_ms_p50": float(np.percentile(steps, 50)),
            "step_ms_p99": float(np.percentile(steps, 99)),
            "device_step_ms_p50": float(np.percentile(dev, 50)) if dev.size else None,
            "device_step_ms_p99": float(np.percentile(dev, 99)) if dev.size else None,
            "trajectory_s_p50": float(np.percentile(lat, 50)),
            "trajectory_s_p99": float(np.percentile(lat, 99)),
            "peak_active": self.peak_active,
            "peak_device_gb": self.peak_bytes / 1e9,
            "grids": {f"{n}^3": sum(1 for r in reqs if r.n == n) for n in sorted({r.n for r in reqs})},
        }
