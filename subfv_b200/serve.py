"""Serving: a request loop over the batched explicit Euler and Lagrangian engines.

No counterpart in the reference (one solve per process run). A request is a solve
(mesh, initial state, end time): a Gresho vortex (explicit Euler, the multi-point
second-order scheme of subfvns) or a 2-D Sedov blast (Lagrangian hydro of
subfvlagrange) on a jittered triangle or quadrilateral mesh. Requests arrive on a seeded
Poisson stream; host threads build their meshes (topology, upload, geometry) as they
arrive; the loop admits built requests while their device bytes fit the HBM budget,
keeps every admitted state resident, advances all in-flight solves of a kind in shared
launches (the two kinds on their own streams, so their work overlaps on the device),
and returns each result as its solve reaches its end time. Each result is bit-identical
to the same request solved alone (tests/test_serve_gpu.py).
"""
from __future__ import annotations

import math
import time
from collections import deque
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from . import meshgen
from .lagrange import LagBatch, LagrangeState, init_sol_sedov
from .mesh import Mesh
from .ns import NsBatch, NsConfig, NsState, init_gresho

# Gresho: multi_point, second order (method 4), bc_style 2, CFL 0.4, peak Mach 0.1
GRESHO_CFG = dict(scheme=1, second_order=True, method=4, bc_style=2, boundary_2d=True, cfl=0.4)
GRESHO_MACH = 0.1
# the time 200 iterations of the 64 x 64 Gresho case reach (its nominal end time)
GRESHO_T_NOMINAL = 0.027
SEDOV_E = 0.244816
SEDOV_CFL = 0.5
SEDOV_T_NOMINAL = 1.0
# Result.status bit of a solve the server stopped because its time step collapsed
# (an average step below STALL_REL x its end time over a whole chunk)
SERVE_STALLED = 1 << 8
STALL_REL = 1e-10


@dataclass
class Request:
    rid: int
    kind: str        # "gresho" or "sedov"
    tri: bool        # triangles (prism slab) or quadrilaterals (hex slab)
    n: int           # squares per side
    seed: int
    arrival: float   # seconds after the start of the stream
    t_end: float

    @property
    def n_cells(self) -> int:
        return self.n * self.n * (2 if self.tri else 1)


def make_requests(n_requests: int, rate: float, seed: int = 0, cells_min: int = 4096, cells_max: int = 1 << 20,
                  time_scale: float = 1.0) -> list[Request]:
    """A seeded Poisson stream: exponential gaps of mean 1/rate seconds, Gresho or Sedov
    with equal odds, a cell count log-uniform in [cells_min, cells_max], an end time
    uniform in [0.1, 1] x the case's nominal end time x time_scale. Gresho meshes are
    triangles or quadrilaterals with equal odds; Sedov meshes are triangles, as in the
    Sedov case: on jittered quadrilaterals the classic Lagrangian scheme lets the corner
    subcell next to the blast shrink towards zero volume near t = 0.013, and the CFL
    bound of compute_dt (proportional to that volume) then shrinks the step
    geometrically, so the solve never reaches its end time (the CPU restatement does
    the same)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n_requests):
        t += rng.exponential(1.0 / rate)
        kind = "gresho" if rng.random() < 0.5 else "sedov"
        tri = bool(rng.random() < 0.5) or kind == "sedov"
        cells = math.exp(rng.uniform(math.log(cells_min), math.log(cells_max)))
        n = max(4, int(round(math.sqrt(cells / (2 if tri else 1)))))
        nominal = GRESHO_T_NOMINAL if kind == "gresho" else SEDOV_T_NOMINAL
        out.append(Request(i, kind, tri, n, int(rng.integers(1 << 30)), t, rng.uniform(0.1, 1.0) * nominal * time_scale))
    return out


def build(req: Request):
    """The request's device mesh and host initial state (and mass for Sedov)."""
    if req.kind == "gresho":
        lo, hi, jit = -0.5, 0.5, 0.1
    else:
        lo, hi, jit = 0.0, 1.2, 0.05
    gen = meshgen.prism_slab if req.tri else meshgen.hex_slab
    raw = gen(req.n, req.n, lo, hi, lo, hi, -0.5, 0.5, jitter=jit, seed=req.seed)
    m = Mesh.from_raw(raw)
    if req.kind == "gresho":
        sol = init_gresho(m, GRESHO_MACH)
        mass = None
    else:
        t = m.topo
        mask = meshgen.sedov_origin_mask(t.array("elem_vert_off"), t.array("elem_vert"), t.coords())
        sol = init_sol_sedov(m, e_total=SEDOV_E, mask=mask)
        mass = m.geometry("elem_volume") / sol[:, 0]
    m.topo.close()
    m.topo = None
    return m, sol, mass


@dataclass
class Result:
    rid: int
    kind: str
    n_cells: int
    steps: int
    t: float
    status: int
    arrival: float
    admitted: float
    done: float
    sol: np.ndarray = field(repr=False)

    @property
    def latency(self) -> float:
        return self.done - self.arrival


class Server:
    """The request loop. budget_bytes bounds the device bytes (meshes plus states) of
    the admitted requests; precision 0 is plain FP64, 1 the mixed path."""

    def __init__(self, budget_bytes: int = int(150e9), capacity: int = 1024, precision: int = 0, chunk: int = 8,
                 build_threads: int = 8, keep_solutions: bool = True):
        self.budget = int(budget_bytes)
        self.chunk = int(chunk)
        self.keep = keep_solutions
        self.ns = NsBatch(NsConfig(**GRESHO_CFG, precision=precision), capacity, self.budget)
        self.lag = LagBatch(capacity, self.budget, precision=precision)
        self.pool = ThreadPoolExecutor(max(1, build_threads))
        self.live = {}  # (kind, slot) -> (request, admitted time, n_cells)

    def used_bytes(self) -> int:
        return self.ns.size()[1] + self.lag.size()[1]

    def _admit(self, req, mesh, sol, mass, now):
        batch = self.ns if req.kind == "gresho" else self.lag
        need = batch.state_bytes(mesh) + mesh.device_bytes
        if need > self.budget:
            raise ValueError(f"request {req.rid} needs {need} device bytes, more than the whole budget")
        if self.used_bytes() + need > self.budget:
            return False
        n_cells = mesh.n_elems
        if req.kind == "gresho":
            k = self.ns.add(mesh, sol, req.t_end, take_mesh=True)
        else:
            k = self.lag.add(mesh, sol, req.t_end, cfl=SEDOV_CFL, mass=mass, take_mesh=True)
        if k is None:
            return False
        self.live[(req.kind, k)] = (req, now, n_cells)
        return True

    def run(self, requests: list[Request], clock=time.perf_counter, progress=None, progress_every: float = 1.0):
        """Serve the stream in real time; returns the results in completion order and the
        makespan (seconds from the first arrival to the last result). progress, if given,
        is called about every progress_every seconds with a dict of counts and, per
        in-flight solve, its kind, cells, time, end time and steps."""
        t0 = clock()
        last_report = 0.0
        arrivals = deque(sorted(requests, key=lambda r: r.arrival))
        building = deque()   # (request, future) in arrival order
        ready = deque()      # (request, mesh, sol, mass) built, waiting for memory
        results = []
        pending = {"gresho": 0, "sedov": 0}  # snapshots queued and not yet taken
        seen = {}  # in-flight solve -> (t, steps) at its previous check
        while arrivals or building or ready or self.live:
            now = clock() - t0
            if progress is not None and now - last_report >= progress_every:
                last_report = now
                inflight = []
                for (k, slot), (req, _, n_cells) in self.live.items():
                    t, steps, _, st = (self.ns if k == "gresho" else self.lag).info(slot)
                    inflight.append((k, n_cells, t, req.t_end, steps, st))
                progress({"time_s": now, "arrivals_left": len(arrivals), "building": len(building),
                          "ready": len(ready), "done": len(results), "inflight": inflight})
            while arrivals and arrivals[0].arrival <= now:
                r = arrivals.popleft()
                building.append((r, self.pool.submit(build, r)))
            while building and building[0][1].done():
                r, fut = building.popleft()
                ready.append((r,) + fut.result())
            while ready:
                r, m, s, ms = ready[0]
                if not self._admit(r, m, s, ms, clock() - t0):
                    break
                ready.popleft()
            if not self.live and not any(pending.values()):
                # nothing on the device: wait for the next build or arrival
                if building:
                    building[0][1].result()
                elif arrivals and not ready:
                    time.sleep(max(0.0, arrivals[0].arrival - (clock() - t0)))
                continue
            # one chunk stays queued behind the one being read back, so the device never
            # waits for the host: advance, then take the older snapshot
            for k in ("gresho", "sedov"):
                b = self.ns if k == "gresho" else self.lag
                keys = [key for key in self.live if key[0] == k]
                if not keys and not pending[k]:
                    continue
                if keys:
                    b.advance(self.chunk)
                    pending[k] += 1
                if pending[k] < 2 and keys:
                    continue
                b.poll(wait=True)
                pending[k] -= 1
                for key in keys:
                    t, steps, done, st = b.info(key[1])
                    if not (done or st):
                        # a time step collapsed to nothing: stop the solve, report it
                        t_prev, s_prev = seen.get(key, (t, steps))
                        seen[key] = (t, steps)
                        req = self.live[key][0]
                        if steps - s_prev >= self.chunk and t - t_prev < STALL_REL * req.t_end * (steps - s_prev):
                            st = SERVE_STALLED
                        else:
                            continue
                    seen.pop(key, None)
                    req, adm, n_cells = self.live.pop(key)
                    sol = b.sol(key[1], n_cells) if self.keep else np.empty((0, 5))
                    b.remove(key[1])
                    results.append(Result(req.rid, req.kind, n_cells, steps, t, st, req.arrival, adm,
                                          clock() - t0, sol))
        makespan = (clock() - t0) - (requests[0].arrival if requests else 0.0)
        return results, makespan

    def close(self):
        self.pool.shutdown(wait=True)
        self.ns.close()
        self.lag.close()


def solve_alone(req: Request, precision: int = 0, chunk: int = 256):
    """The same request solved by itself on the solo path; returns (steps, t, status, sol)."""
    m, sol, mass = build(req)
    if req.kind == "gresho":
        s = NsState(m, NsConfig(**GRESHO_CFG, precision=precision, tmax=req.t_end), sol)
        steps = t = st = 0
        while True:
            st, steps_new, t = s.advance(chunk)
            if st or steps_new < steps + chunk:
                steps = steps_new
                break
            steps = steps_new
        return steps, t, st, s.sol()
    s = LagrangeState(m, sol, mass, cfl=SEDOV_CFL, t_max=req.t_end, precision=precision)
    steps = t = st = 0
    while True:
        st, steps_new, t = s.advance(chunk)
        if st or steps_new < steps + chunk:
            steps = steps_new
            break
        steps = steps_new
    out = np.empty((m.n_elems, 5))
    from . import _lib
    _lib.check(_lib.load().subfv_lag_get_sol(s._h, _lib.pd(out)), "subfv_lag_get_sol")
    return steps, t, st, out


def latency_stats(results: list[Result]) -> dict:
    """Latency percentiles over the solves that reached their end time."""
    lat = np.array([r.latency for r in results if r.status == 0])
    if lat.size == 0:
        return {}
    return {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "max_s": float(lat.max())}
