"""Serving loop over libtdda's request engine (include/tdda.h, tdda_server_*).

`DDAServer` owns one GPU's request loop: `submit` queues a solve and returns a
ticket at once, `wait` returns its polarisation P and internal field E.  The
engine admits requests against an HBM budget, keeps the FFT'd interaction
tensor of each (grid, d, lambda, nback, period, method) resident, merges
queued requests that share a tensor into one multi-right-hand-side solve, and
overlaps the batches of its workers on the device (continuous batching).

`synthetic_stream` makes the mixed-size request stream with Poisson arrivals
and `run_stream` replays it against a server in real time, returning latency
percentiles and throughput.
"""
from __future__ import annotations

import ctypes
import math
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib

PREC = {"complex128": 0, "c128": 0, "mixed": 1}


@dataclass
class Request:
    """One structure under one plane wave; each polarisation is a right-hand side."""
    shape: tuple                       # (nx, ny, nz), dipole i = x + nx*(y + ny*z)
    rho: np.ndarray                    # nx*ny*nz densities in [0, 1]
    lam: float = 542.0
    d: float = 25.0
    nback: float = 1.0
    E0: float = 1.0
    material: tuple = (1.0 + 0j, 3.5 + 0.01j)
    n_K: tuple = (0.0, 0.0, 1.0)
    polarisations: tuple = ((1.0, 0.0, 0.0),)
    MAXm: int = 0
    MAXn: int = 0
    Lm: float = 0.0
    Ln: float = 0.0
    method: str = "FCD"
    precision: str = "mixed"
    tol: float = 1e-8
    max_iter: int = 100000
    arrival_s: float = 0.0             # used by run_stream
    tag: object = None


@dataclass
class Result:
    P: np.ndarray                      # [npol, 3N] complex128, dipole order
    E: np.ndarray                      # [npol, 3N] E_int = al P / ((2 + eps) / 3)
    info: list
    batch_rhs: int
    batch_requests: int
    cache_hit: bool
    worker: int
    queue_ms: float
    build_ms: float
    solve_ms: float
    total_ms: float
    tag: object = None


def incidence(theta_deg: float):
    """Propagation direction at polar angle theta (azimuth 0) and the two
    polarisations perpendicular to it: p-like in the x-z plane and s-like (y)."""
    t = math.radians(theta_deg)
    nK = (math.sin(t), 0.0, math.cos(t))
    p = (math.cos(t), 0.0, -math.sin(t))
    return nK, (p, (0.0, 1.0, 0.0))


class DDAServer:
    def __init__(self, hbm_budget_bytes=120 * 10**9, workers=8, max_rhs=8, use_graphs=True, graph_steps=4,
                 sici=None):
        from . import sici_tables

        self._lib = _lib.load()
        si, ci = sici if sici is not None else sici_tables()
        self._si = np.ascontiguousarray(si, dtype=np.float64)
        self._ci = np.ascontiguousarray(ci, dtype=np.float64)
        cfg = _lib.ServerConfig(int(hbm_budget_bytes), int(workers), int(max_rhs), 1 if use_graphs else 0,
                                int(graph_steps))
        h = ctypes.c_void_p()
        dp = ctypes.POINTER(ctypes.c_double)
        _lib.check(self._lib.tdda_server_create(ctypes.byref(cfg), self._si.ctypes.data_as(dp),
                                                self._ci.ctypes.data_as(dp), self._si.size, ctypes.byref(h)))
        self._h = h
        self._pending = {}   # ticket -> (request, output arrays, ctypes struct)
        self._mu = threading.Lock()

    def submit(self, req: Request) -> int:
        nx, ny, nz = (int(v) for v in req.shape)
        n = nx * ny * nz
        rho = np.ascontiguousarray(np.asarray(req.rho, dtype=np.float64).ravel())
        if rho.size != n:
            raise ValueError(f"rho has {rho.size} values, the grid {req.shape} has {n}")
        npol = len(req.polarisations)
        P = np.zeros((npol, 3 * n), dtype=np.complex128)
        E = np.zeros((npol, 3 * n), dtype=np.complex128)
        r = _lib.Request()
        r.num_x, r.num_y, r.num_z = nx, ny, nz
        r.d, r.lam, r.nback, r.E0 = float(req.d), float(req.lam), float(req.nback), float(req.E0)
        m = [complex(v) for v in req.material]
        r.material[:] = [m[0].real, m[0].imag, m[1].real, m[1].imag]
        r.MAXm, r.MAXn, r.Lm, r.Ln = int(req.MAXm), int(req.MAXn), float(req.Lm), float(req.Ln)
        r.method = {"FCD": 0, "LDR": 1}[req.method]
        r.n_K[:] = [float(v) for v in req.n_K]
        r.npol = npol
        for q, e in enumerate(req.polarisations):
            r.n_E0[q][:] = [float(v) for v in e]
        dp = ctypes.POINTER(ctypes.c_double)
        r.rho = rho.ctypes.data_as(dp)
        r.precision = PREC[req.precision]
        r.tol, r.max_iter = float(req.tol), int(req.max_iter)
        r.P_out = P.ctypes.data_as(dp)
        r.E_out = E.ctypes.data_as(dp)
        t = ctypes.c_int64()
        _lib.check(self._lib.tdda_server_submit(self._h, ctypes.byref(r), ctypes.byref(t)))
        with self._mu:
            self._pending[t.value] = (req, P, E)
        return t.value

    def wait(self, ticket: int, timeout: float = -1.0) -> Result:
        res = _lib.RequestResult()
        _lib.check(self._lib.tdda_server_wait(self._h, int(ticket), float(timeout), ctypes.byref(res)))
        with self._mu:
            req, P, E = self._pending.pop(ticket)
        _lib.check(res.status)
        npol = len(req.polarisations)
        return Result(P=P, E=E, info=[res.info[q].as_dict() for q in range(npol)], batch_rhs=res.batch_rhs,
                      batch_requests=res.batch_requests, cache_hit=bool(res.cache_hit), worker=res.worker,
                      queue_ms=res.queue_ms, build_ms=res.build_ms, solve_ms=res.solve_ms,
                      total_ms=res.total_ms, tag=req.tag)

    def solve(self, req: Request) -> Result:
        return self.wait(self.submit(req))

    def reserve(self, shape, precision="mixed"):
        """Allocate every worker's workspace for this grid now (before any
        submit), so that the first requests of the grid do not wait for it."""
        nx, ny, nz = (int(v) for v in shape)
        _lib.check(self._lib.tdda_server_reserve(self._h, nx, ny, nz, PREC[precision]))

    def stats(self) -> dict:
        s = _lib.ServerStats()
        _lib.check(self._lib.tdda_server_get_stats(self._h, ctypes.byref(s)))
        return s.as_dict()

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.tdda_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


SERVE_SHAPES = ((32, 32, 8), (48, 48, 12), (64, 64, 16), (96, 96, 16))


def synthetic_stream(n=512, rate=200.0, seed=7, shapes=SERVE_SHAPES, lam_range=(450.0, 700.0),
                     theta_max_deg=30.0, precision="mixed", tol=1e-8, d=25.0, material=(1.0 + 0j, 3.5 + 0.01j)):
    """n requests with Poisson arrivals at `rate` per second: grid uniform over
    `shapes`, wavelength ~ U[lam_range] nm, polar angle ~ U[0, theta_max] (azimuth
    0), two polarisations each (p-like and y), densities ~ U[0, 1]."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        shape = shapes[rng.integers(len(shapes))]
        lam = float(rng.uniform(*lam_range))
        theta = float(rng.uniform(0.0, theta_max_deg))
        nK, pols = incidence(theta)
        rho = rng.random(int(np.prod(shape)))
        out.append(Request(shape=tuple(shape), rho=rho, lam=lam, d=d, material=material, n_K=nK,
                           polarisations=pols, precision=precision, tol=tol, arrival_s=t, tag=i))
    return out


@dataclass
class StreamReport:
    results: list = field(default_factory=list)
    requests: list = field(default_factory=list)
    wall_s: float = 0.0
    latency_ms: np.ndarray = None

    def summary(self):
        lat = self.latency_ms
        nrhs = sum(len(r.info) for r in self.results)
        conv = sum(1 for r in self.results for i in r.info if i["status"] == "converged")
        return {
            "requests": len(self.results), "rhs": nrhs, "converged_rhs": conv,
            "wall_s": self.wall_s,
            "requests_per_s": len(self.results) / self.wall_s if self.wall_s > 0 else float("nan"),
            "solves_per_s": nrhs / self.wall_s if self.wall_s > 0 else float("nan"),
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "max_true_error": max(i["true_error"] for r in self.results for i in r.info),
        }

    def per_shape(self):
        """Per grid: requests, mean batch size (right-hand sides), batches,
        device-side solve time of a batch (median), the GPU seconds the grid's
        batches took in total (each batch counted once), and the mean inner
        iterations per right-hand side."""
        out = {}
        shapes = [tuple(q.shape) for q in self.requests]
        for shape in sorted(set(shapes)):
            rs = [r for r, sh in zip(self.results, shapes) if sh == shape]
            key = "x".join(str(v) for v in shape)
            out[key] = {
                "requests": len(rs),
                "batches": sum(1.0 / r.batch_requests for r in rs),
                "mean_batch_rhs": float(np.mean([r.batch_rhs for r in rs])),
                "median_batch_solve_ms": float(np.median([r.solve_ms for r in rs])),
                "solve_s_total": sum(r.solve_ms / r.batch_requests for r in rs) / 1e3,
                "mean_inner_iterations": float(np.mean([i["inner_iterations"] for r in rs for i in r.info])),
            }
        return out


def run_stream(server: DDAServer, requests, realtime=True) -> StreamReport:
    """Submit each request at its arrival time (relative to the start) from one
    thread while another collects results; latency = result ready - submit."""
    tickets = [None] * len(requests)
    ready = [threading.Event() for _ in requests]
    results = [None] * len(requests)
    errors = []
    t0 = time.perf_counter()

    def submitter():
        try:
            for i, r in enumerate(requests):
                if realtime:
                    dt = r.arrival_s - (time.perf_counter() - t0)
                    if dt > 0:
                        time.sleep(dt)
                tickets[i] = server.submit(r)
                ready[i].set()
        except Exception as e:  # surfaced below
            errors.append(e)
            for ev in ready:
                ev.set()

    th = threading.Thread(target=submitter)
    th.start()
    for i in range(len(requests)):
        ready[i].wait()
        if errors:
            break
        results[i] = server.wait(tickets[i])
    th.join()
    if errors:
        raise errors[0]
    rep = StreamReport(results=results, requests=list(requests), wall_s=time.perf_counter() - t0)
    rep.latency_ms = np.array([r.total_ms for r in results])
    return rep
