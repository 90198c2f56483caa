"""Benchmark: DDA solves/s (+ p50/p99 latency), mixed precision vs plain
complex128, at a 1e-8 relative residual, on a 128x128x32 dipole
structure, periodic 128d in x and y.

Workload (one "step" = the solves of both polarisations):
  128 x 128 x 32 dipoles (524,288), d = 25 nm, lambda = 542 nm, vacuum
  background, eps_mat = 3.5 + 0.01i, FCD Green tensor, periodic with period
  128 d in x and y and the lattice sums over |m|,|n| <= 50 (the reference's
  damping exp(-(0.01 K r)^4) on every image).  Design: seeded binary 0/1 field
  -> radius-2d cone filter -> tanh projection (beta 8, eta 0.5), one density
  per dipole.  Plane wave along +z; x- and y-polarised right-hand sides (2 RHS
  per step), zero initial guess, solved concurrently, each by its own model on
  its own CUDA stream from its own host thread.
  value = mixed-precision solves/s: complex128 iterative refinement on the
          TRUE residual ||E - A P|| / ||E|| <= 1e-8 around inner solves of
          deflated restarted GMRES on the Jacobi-scaled complex64 operator
          (FP64 Gram-Schmidt sums and projected problems);
  plain = the same solver with complex128 inner solves.
  The reference's own BiCGSTAB does not reach 1e-8 on this structure (it
  fills its periodic cell); the line records where it stalls.
Inputs live in HBM before the timed region; the working set (> 2 GB) exceeds
the 126 MB L2, so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun each rank runs an independent replica (the solves shard by
request; no collective on the data path) and rank 0 prints one JSON line.

Secondary records in the line: the isolated 128x128x32 structure (the
previous workload, BiCGSTAB), the 16x16x8 isolated workload on the GPU (the reference arm's
workload, for the algorithm-matched ratio), the 64x64x16 workload (periodic
64d, complex128), the differentiation step (96x96x24 periodic 96d:
forward solve + adjoint gradient through the autograd path), the lattice-sum
kernel, the cuFFT restatement of the reference's A.x, and "serving": the
request loop of dda_model.serving on 512 requests with seeded Poisson
arrivals at 200 req/s, grids drawn from {32x32x8, 48x48x12, 64x64x16,
96x96x16}, lambda ~ U[450, 700] nm, polar angle ~ U[0, 30] deg, x- and
y-like polarisations (2 RHS each), rho ~ U[0, 1], mixed precision to a 1e-8
true residual under a 120 GB admission budget, plus the same mix at 30 req/s
("serving.below_capacity").  --no-serving skips both.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "topo-dda_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

MAX_ITER = 400000  # inner operator applications per solve; the benchmark solves converge well below this
# solver of the periodic workloads: GMRES on the scaled operator times a polynomial of
# `degree`, cycles of `restart` steps keeping `deflate` harmonic Ritz vectors
SOLVER = dict(degree=1, restart=40, deflate=10)
# basis vectors a Gram-Schmidt pass reads on average in a GMRES-DR(40, 10)
# cycle (11 to 40 after a deflated restart)
GS_NV = 25
_T0 = time.perf_counter()


def log(msg):
    print(f"[bench {time.perf_counter() - _T0:7.1f}s] {msg}", file=sys.stderr, flush=True)


METRIC = "DDA solves/sec + p50/p99 latency, mixed vs plain c128, same B200 @1e-8 resid"
WORKLOAD = dict(nx=128, ny=128, nz=32, d=25.0, lam=542.0, eps=3.5 + 0.01j, period=128, M=50,
                seed=2024, filter_radius=2.0, beta=8.0, eta=0.5, tol=1e-8)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="tdda", choices=["tdda", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving-loop stream")
    ap.add_argument("--small", action="store_true", help="32x32x8, M=5 (quick check, not a bench line)")
    ap.add_argument("--profile-solve", type=int, default=0, metavar="K",
                    help="profile case: K mixed-precision solves of the x-polarised RHS, then exit "
                         "(prints the library's launch count before each, for ncu -s)")
    ap.add_argument("--profile-matvec", type=int, default=0, metavar="K",
                    help="only build the benchmark model and apply the operator K times per precision "
                         "(the case the kernel profiles capture); prints per-pass times")
    ap.add_argument("--profile-gs", type=int, default=0, metavar="K",
                    help="time K projection and K update passes of the Gram-Schmidt kernels against "
                         "GS_NV complex64 basis vectors of the benchmark grid, then exit (profiling case)")
    ap.add_argument("--profile-gmres", type=int, default=0, metavar="K",
                    help="profile case of the GMRES-DR kernels: one mixed-precision solve of the x-polarised "
                         "RHS of the benchmark structure, capped at K inner operator applications; prints the "
                         "solve record")
    return ap.parse_args()


def run_profile_gmres(k, sici):
    """One GMRES-DR solve of the benchmark structure cut off after k inner
    operator applications (the case the Gram-Schmidt kernel profiles capture:
    1.57 M complex64 unknowns per basis vector, a basis of up to 61 vectors)."""
    import torch

    from dda_model import DDAModel

    w = workload()
    m = DDAModel(**model_kwargs(w, sici), precision="mixed")
    m.setDensities(design(w))
    m.setSolver("pgmres", **SOLVER)
    B = torch.from_numpy(np.stack([incident(w, 0)])).cuda()
    X = torch.zeros_like(B)
    s = torch.cuda.current_stream()
    torch.cuda.synchronize()
    t = time.perf_counter()
    info = m.solve_batch_device(B.data_ptr(), X.data_ptr(), 1, True, k, w["tol"], s.cuda_stream)[0]
    torch.cuda.synchronize()
    dt = time.perf_counter() - t
    print(json.dumps(dict(grid=[w["nx"], w["ny"], w["nz"]], M=w["M"], seconds=dt,
                          ms_per_step=1e3 * dt / max(1, info["iterations"]), **info)))
    return 0


def workload(small=False):
    w = dict(WORKLOAD)
    if small:
        w.update(nx=32, ny=32, nz=8, period=32, M=5)
    return w


def design(w):
    from dda_model import filters

    b = filters.binary_design(w["nx"], w["ny"], w["nz"], w["seed"])
    rho = filters.tanh_projection(filters.cone_filter(b, w["filter_radius"]), w["beta"], w["eta"])
    return filters.dipole_order(np.clip(rho, 0.0, 1.0))


def model_kwargs(w, sici):
    from dda_model import _generate_geometry

    nx, ny, nz = w["nx"], w["ny"], w["nz"]
    N = nx * ny * nz
    si, ci = sici
    return dict(
        betaMin=0.0, betaMax=50.0, ita=0.5, betaType="piecewise", filterIterations=[100],
        filterRadii=[2.0], useFilter=False, symmetryType="None", symmetryAxis=[0.0, 0.0],
        isPeriodic=True, objectiveName="IntegratedE",
        objPara=[2.0, 0, nx - 1.0, 0, ny - 1.0, 0, nz - 1.0, 0.95, 50.0],
        geometry=_generate_geometry(nx, ny, nz), inputDielectrics=np.zeros(3 * N),
        num_x=nx, num_y=ny, num_z=nz, num_total=N, n_K=[0, 0, 1], E0=1.0, n_E0=[1, 0, 0],
        lam=w["lam"], material=[1.0 + 0j, w["eps"]], nback=1.0, MAXm=w["M"], MAXn=w["M"],
        Lm=w["period"], Ln=w["period"], matrixAMethodName="FCD", d=w["d"],
        sineIntegralValues=si, cosineIntegralValues=ci, integralDelta=0.1, verbose=False)


def incident(w, pol):
    """Plane wave along +z, polarisation `pol`, in dipole order (complex[3N])."""
    from dda_model import _generate_geometry

    g = _generate_geometry(w["nx"], w["ny"], w["nz"]).reshape(-1, 3)
    K = 2 * math.pi / w["lam"]
    ph = K * w["d"] * g[:, 2]
    e = np.cos(ph) + 1j * np.sin(ph)
    E = np.zeros((len(g), 3), dtype=np.complex128)
    E[:, pol] = e
    return E.ravel()


class ClockSampler:
    """nvidia-smi clocks / throttle reasons every 200 ms while running."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,utilization.gpu")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._proc = None

    def __enter__(self):
        try:
            self._proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self._proc = None
        return self

    def _read(self):
        for line in self._proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self._proc is not None:
            time.sleep(0.25)
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self._proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if len(r) > 4 + i and r[4 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "samples": len(self.rows), "reasons": reasons}

    def gpu_busy(self):
        """Mean of nvidia-smi's utilization.gpu (percent of time a kernel ran)."""
        u = [float(r[8]) for r in self.rows if len(r) > 8 and r[8].replace(".", "").isdigit()]
        return statistics.mean(u) / 100.0 if u else None


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_record(name="matvec_c64_traffic.txt"):
    """DRAM bytes per launch from a committed ncu summary under profiles/
    ('key: value' lines): the fused complex64 matvec, or the Gram-Schmidt
    projection kernel."""
    path = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(path):
        return None
    rec = {}
    with open(path) as f:
        for line in f:
            if line.startswith("#") or ":" not in line:
                continue
            k, v = line.split(":", 1)
            rec[k.strip()] = float(v)
    return rec


def dist_setup():
    from dda_model.replicas import env_rank

    return env_rank()


# ----------------------------------------------------------------------------
# CPU reference arm: the oracle port (the reference has no CPU A.x, and its
# own build needs Eigen and cuFFT) timed on the host cores
# ----------------------------------------------------------------------------
# the 16x16x8 workload: dipoles isolated, rho ~ U[0, 1] per dipole, complex128,
# the reference's BiCGSTAB from a zero guess to 1e-8
SMALL16 = dict(WORKLOAD, nx=16, ny=16, nz=8, period=16, M=0, seed=7)


def small16_design():
    return np.random.default_rng(SMALL16["seed"]).random(SMALL16["nx"] * SMALL16["ny"] * SMALL16["nz"])


class CpuPort:
    """The reference's algorithm on the host cores: the complex128 oracle
    (scipy.fft with every core, the reference's 2n-1 padding) and its BiCGSTAB
    (unscaled, zero guess, stopping on the recursive residual).  With
    images=False the lattice sum is taken without periodic images (for timing
    operator applications only: the FFT convolution's cost does not depend on
    the tensor values)."""

    def __init__(self, w, rho, pol=0, images=True):
        from oracle import dda_oracle as O

        self.O = O
        si, ci = O.sici_tables()
        kw = model_kwargs(w, (si, ci))
        if not images:
            kw["MAXm"] = kw["MAXn"] = 0
        kw["n_E0"] = [1, 0, 0] if pol == 0 else [0, 1, 0]
        kw["inputDielectrics"] = np.repeat(rho, 3)
        self.m = O.OracleModel(**kw)
        self.m.set_densities(rho)
        self.cores = os.cpu_count() or 1

    def solve(self, tol, max_iter=100000):
        """Seconds and info of one full solve."""
        m = self.m
        t0 = time.perf_counter()
        info = self.O.bicgstab(m.aproduct_with_alb, m.E, np.zeros(3 * m.N, complex), max_iter, tol)[1]
        return time.perf_counter() - t0, info

    def per_apply(self, k):
        """Seconds per operator application, over k applications."""
        m = self.m
        x = m.E.copy()
        t0 = time.perf_counter()
        for _ in range(k):
            x = m.aproduct_with_alb(x)
            x /= np.linalg.norm(x)
        return (time.perf_counter() - t0) / k


def run_reference(args):
    """The reference arm: the reference's algorithm on the host cores.  Its
    headline is measured full solves at 16x16x8 (isolated, where the CPU
    finishes them in about a second); on the 128x128x32 periodic workload the
    reference's BiCGSTAB does not reach 1e-8 at all (the GPU arm's line
    records its residual), so that workload gets a measured seconds-per-
    operator sample instead."""
    world, rank, local = dist_setup()
    if rank != 0:
        return 0
    rho0 = small16_design()
    ports = [CpuPort(SMALL16, rho0, pol) for pol in (0, 1)]
    cores = ports[0].cores
    steps, infos = [], []
    for k in range(args.warmup + max(args.steps, 5)):
        t = 0.0
        for p in ports:
            dt, info = p.solve(SMALL16["tol"])
            t += dt
            infos.append(info)
        if k >= args.warmup:
            steps.append(t)
    med = statistics.median(steps)
    sps = 2.0 / med
    # the 64x64x16 and 128x128x32 grids: seconds per complex128 operator application (the unit of
    # work of every solver here), measured on the full grid
    g64 = dict(WORKLOAD, nx=64, ny=64, nz=16, period=64, M=50)
    p1 = CpuPort(g64, np.random.default_rng(1).random(64 * 64 * 16), images=False)
    s1 = [p1.per_apply(4) for _ in range(3)]
    w2 = workload(args.small)
    p2 = CpuPort(w2, design(w2), images=False)
    s2 = [p2.per_apply(1) for _ in range(3)]
    line = {
        "impl": "reference", "metric": METRIC, "value": sps, "unit": "solves/s", "n_gpus": args.gpus,
        "steps": len(steps), "warmup": args.warmup, "ms_per_step": med * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
        "data": "synthetic",
        "config": {"workload": "16x16x8 dipoles, isolated, d=25nm, lambda=542nm, eps 3.5+0.01i, FCD, "
                               "rho ~ U[0,1] per dipole, x+y polarised (2 RHS/step), the reference's BiCGSTAB "
                               "(unscaled complex128, zero guess) to a 1e-8 recursive residual",
                   "grid": [16, 16, 8], "dipoles": 2048, "rhs_per_step": 2, "tol": SMALL16["tol"],
                   "why_not_the_gpu_workload": "the reference's BiCGSTAB does not reach 1e-8 on the 128x128x32 "
                                               "periodic workload (see the GPU arm's reference_algorithm_gpu)"},
        "samples_s_per_step": steps,
        "spread": {"min": min(steps), "median": med, "max": max(steps)},
        "iterations": sorted({i.iterations for i in infos}),
        "converged": all(i.converged for i in infos),
        "cpu_baseline": {"value": sps, "unit": "solves/s", "cores": cores, "kind": "port",
                         "sample": f"full solves at 16x16x8, both polarisations, {len(steps)} timed steps after "
                                   f"{args.warmup} warm-up; oracle port (scipy.fft, {cores} workers)"},
        "operator_apply_s": {
            "grid_64x64x16": {"median": statistics.median(s1), "samples": s1},
            "grid_128x128x32": {"median": statistics.median(s2), "samples": s2},
            "note": "complex128 A.x + (1/alpha) x of the oracle port on the full grid (reference padding 2n-1)"},
        "e2e": {"value": sps, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def cpu_lattice_rate(w, npts=200, seed=3):
    """Image evaluations per second of the oracle's restatement of the
    reference's constructor loop (src/AProductCore.cpp:63-244: every padded
    offset sums every image (m, n), |m|,|n| <= M, damped; single thread, as the
    reference's constructor), timed on npts random offsets of the grid."""
    import ctypes

    from oracle import dda_oracle as O

    lib = O._load_lib()
    si, ci = O.sici_tables()
    rng = np.random.default_rng(seed)
    d = w["d"]
    off = np.stack([rng.integers(-(w[a] - 1), w[a], npts) for a in ("nx", "ny", "nz")], axis=1).astype(np.float64) * d
    off = np.ascontiguousarray(off)
    out = np.zeros(12 * npts)
    K = 2 * math.pi / w["lam"]
    dp = ctypes.POINTER(ctypes.c_double)
    t0 = time.perf_counter()
    lib.oracle_lattice_points(0, npts, off.ctypes.data_as(dp), w["M"], w["M"], w["period"] * d, w["period"] * d, K, d,
                              si.ctypes.data_as(dp), ci.ctypes.data_as(dp), len(si), 0.1, out.ctypes.data_as(dp))
    dt = time.perf_counter() - t0
    return npts * (2 * w["M"] + 1) ** 2 / dt, dt


def lattice_record(m, w, cpu_rate=None):
    """The lattice-sum kernel of one model: device time, and the work the
    reference's constructor does for the same tensor ((2nx-1)(2ny-1)(2nz-1)
    offsets x (2M+1)^2 images) per second of it."""
    nfft = (2 * w["nx"] - 1) * (2 * w["ny"] - 1) * (2 * w["nz"] - 1)
    evals = nfft * (2 * w["M"] + 1) ** 2
    ms = m.info["lattice_ms"]
    rec = {"lattice_ms": ms, "tensor_fft_ms": m.info["tensor_fft_ms"], "reference_image_evaluations": evals,
           "reference_equivalent_evals_per_s": evals / (ms * 1e-3),
           "note": "the kernel evaluates the non-negative octant (parity gives the rest) and skips images whose "
                   "damping exp(-(0.01 K r)^4) is exactly 0; FP64-issue-bound, not graded against HBM"}
    if cpu_rate is not None:
        rec["cpu_port_evals_per_s_1_thread"] = cpu_rate
        rec["cpu_port_constructor_estimate_s"] = evals / cpu_rate
        rec["speedup_vs_cpu_constructor"] = (evals / cpu_rate) / (ms * 1e-3)
    return rec


def config_block(w, ngpu):
    per = f"periodic {w['period']}d, |m|,|n|<={w['M']}" if w["M"] > 0 else "isolated (no periodic images)"
    return {"workload": f"{w['nx']}x{w['ny']}x{w['nz']} dipoles, {per}, d=25nm, lambda=542nm, eps 3.5+0.01i, "
                        f"FCD, filtered+tanh-projected binary design, x+y polarised (2 RHS/step), tol 1e-8",
            "grid": [w["nx"], w["ny"], w["nz"]], "dipoles": w["nx"] * w["ny"] * w["nz"], "rhs_per_step": 2,
            "schedule": "the 2 polarisations solved concurrently, one model and CUDA stream each",
            "design": "seeded binary field -> radius-2d cone filter -> tanh projection (beta 8, eta 0.5)",
            "rhs_per_solve": 1,
            "tol": w["tol"], "parallelism": f"replicas x{ngpu}",
            "l2": "working set > 126 MB L2 (no flush needed)"}


def run_cufft_restatement(w, sici, iters=20):
    """The reference's A.x, restated with cuFFT (torch.fft) and labelled as a
    restatement: AProductCore::Aproduct (src/AProductCore.cpp:461-515) with the
    element-wise kernels of src/Kernel.cu:44-125 -- zero padding to the
    reference's (2 nx - 1) x (2 ny - 1) x (2 nz - 1) grid, the six tensor
    components FFT'd once (cufftExecZ2Z, :262-279), per product three forward
    FFTs of the scattered vector components, the symmetric 3x3 multiply, three
    inverse FFTs, the crop and the division by NFFT, complex128.  Timed on the
    device alone and with the host round trip of the reference's Aproduct
    (host vector in, host vector out), and compared with this library's
    operator (same lattice sums) for correctness."""
    import torch

    from dda_model import DDAModel

    dev = torch.device("cuda")
    nx, ny, nz = w["nx"], w["ny"], w["nz"]
    m = DDAModel(**model_kwargs(w, sici), precision="mixed")
    m.setDensities(design(w))
    P = (2 * nx - 1, 2 * ny - 1, 2 * nz - 1)
    G = torch.empty(P + (6,), dtype=torch.complex128, device=dev)
    m.lattice_offsets_device((-(nx - 1), -(ny - 1), -(nz - 1)), P, G.data_ptr(),
                             torch.cuda.current_stream().cuda_stream)
    # offset o sits at index o mod P, as in the reference's AHos
    G = torch.roll(G, shifts=(-(nx - 1), -(ny - 1), -(nz - 1)), dims=(0, 1, 2))
    Ah = torch.fft.fftn(G.permute(3, 0, 1, 2).contiguous(), dim=(1, 2, 3))
    del G
    A00, A01, A02, A11, A12, A22 = Ah
    N = nx * ny * nz
    idx = torch.arange(N, device=dev)
    gx, gy, gz = idx % nx, (idx // nx) % ny, idx // (nx * ny)   # dipole order, x fastest

    def aproduct(b):  # b: [N, 3] complex128 on the device
        grid = torch.zeros((3,) + P, dtype=torch.complex128, device=dev)
        grid[:, gx, gy, gz] = b.T
        bh = torch.fft.fftn(grid, dim=(1, 2, 3))
        c = torch.stack((A00 * bh[0] + A01 * bh[1] + A02 * bh[2], A01 * bh[0] + A11 * bh[1] + A12 * bh[2],
                         A02 * bh[0] + A12 * bh[1] + A22 * bh[2]))
        y = torch.fft.ifftn(c, dim=(1, 2, 3))    # includes the 1/NFFT of src/AProductCore.cpp:510
        return y[:, gx, gy, gz].T.contiguous()

    rng = np.random.default_rng(5)
    xh = (rng.standard_normal(3 * N) + 1j * rng.standard_normal(3 * N)).astype(np.complex128)
    x = torch.from_numpy(xh.reshape(N, 3)).to(dev)
    ref = aproduct(x).reshape(-1).cpu().numpy()
    ours = m.matvec(xh, with_al=False)
    rel = float(np.linalg.norm(ref - ours) / np.linalg.norm(ours))
    for _ in range(3):
        aproduct(x)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(iters):
        aproduct(x)
    e1.record()
    e1.synchronize()
    dev_ms = e0.elapsed_time(e1) / iters
    xp = torch.from_numpy(xh.reshape(N, 3)).pin_memory()
    yp = torch.empty_like(xp).pin_memory()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(iters):
        yp.copy_(aproduct(xp.to(dev, non_blocking=True)), non_blocking=True)
    torch.cuda.synchronize()
    host_ms = (time.perf_counter() - t0) / iters * 1e3
    ms128, _ = m.profile_matvec("complex128", nrhs=1, iters=20)
    ms64, _ = m.profile_matvec("mixed", nrhs=1, iters=20)
    out = {"what": "restatement of the reference's Aproduct call sequence with cuFFT via torch.fft (the "
                   "reference's own build needs Eigen and is not buildable here)",
           "fft_grid": list(P), "matvec_device_ms": dev_ms, "matvec_with_host_copies_ms": host_ms,
           "this_library_c128_ms": ms128, "this_library_c64_ms": ms64,
           "speedup_c128_device": dev_ms / ms128, "speedup_c64_device": dev_ms / ms64,
           "rel_diff_vs_this_library": rel}
    del Ah, A00, A01, A02, A11, A12, A22
    torch.cuda.empty_cache()
    return out


def run_serving(rank=0, world=1, device=None):
    """The serving workload (see the module docstring) through dda_model.serving.
    With several ranks each serves the requests routed to it by tensor key
    (replicas; arrival times unchanged), and the throughput is all ranks'
    requests over the slowest rank's wall time."""
    from dda_model.replicas import max_over_ranks, shard, sum_over_ranks
    from dda_model.serving import DDAServer, run_stream, synthetic_stream

    from dda_model.serving import SERVE_SHAPES

    reqs = shard(synthetic_stream(n=512, rate=200.0, seed=7), rank, world)
    with DDAServer(hbm_budget_bytes=120 * 10**9, workers=4, max_rhs=8, use_graphs=True) as srv:
        for shape in SERVE_SHAPES:   # workspaces allocated before the stream starts
            srv.reserve(shape)
        with ClockSampler(torch_index(device)) as clk:
            rep = run_stream(srv, reqs)
        st = srv.stats()
    s = rep.summary()
    log(f"serving (rank {rank}/{world}, {len(reqs)} requests): {s}")
    wall = max_over_ranks(s["wall_s"], device)
    nreq = sum_over_ranks(s["requests"], device)
    s["requests_per_s"] = nreq / wall
    s["solves_per_s"] = 2 * nreq / wall
    s["wall_s"] = wall
    return {"workload": "512 requests, Poisson 200 req/s, grids 32x32x8/48x48x12/64x64x16/96x96x16, "
                        "lambda U[450,700] nm, angle U[0,30] deg, 2 RHS each, mixed precision, tol 1e-8, "
                        "120 GB budget, 4 workers, up to 8 RHS per batch",
            "requests_per_s": s["requests_per_s"], "solves_per_s": s["solves_per_s"],
            "p50_ms": s["p50_ms"], "p99_ms": s["p99_ms"], "mean_ms": s["mean_ms"], "wall_s": s["wall_s"],
            "converged_rhs": s["converged_rhs"], "rhs": s["rhs"], "max_true_error": s["max_true_error"],
            "batches": st["batches"], "merged_requests": st["merged_requests"],
            "peak_bytes": st["peak_bytes"], "latency": "submit to result, wall clock, includes queueing",
            "gpu_busy": clk.gpu_busy(), "per_grid": rep.per_shape(),
            "below_capacity": run_serving_light(rank, world, device)}


def torch_index(device):
    import torch

    return torch.device(device).index if device is not None else torch.cuda.current_device()


def run_serving_light(rank=0, world=1, device=None, n=256, rate=30.0):
    """The same request mix at an arrival rate the server keeps up with, so
    that p50/p99 show service time rather than queueing."""
    from dda_model.replicas import max_over_ranks, shard
    from dda_model.serving import DDAServer, run_stream, synthetic_stream

    from dda_model.serving import SERVE_SHAPES

    reqs = shard(synthetic_stream(n=n, rate=rate, seed=9), rank, world)
    with DDAServer(hbm_budget_bytes=120 * 10**9, workers=4, max_rhs=8, use_graphs=True) as srv:
        for shape in SERVE_SHAPES:
            srv.reserve(shape)
        rep = run_stream(srv, reqs)
    s = rep.summary()
    return {"requests": n, "arrival_rate_per_s": rate, "p50_ms": s["p50_ms"], "p99_ms": s["p99_ms"],
            "mean_ms": s["mean_ms"], "wall_s": max_over_ranks(s["wall_s"], device),
            "converged_rhs": s["converged_rhs"], "max_true_error": s["max_true_error"]}


# ----------------------------------------------------------------------------
# GPU arm
# ----------------------------------------------------------------------------
def both(fn):
    """fn(k) for the two polarisations on two host threads (the library
    releases the GIL inside its calls); re-raises the first error."""
    errs = []

    def run(k):
        try:
            fn(k)
        except BaseException as e:  # noqa: BLE001
            errs.append(e)

    th = [threading.Thread(target=run, args=(k,)) for k in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    if errs:
        raise errs[0]


class PolPair:
    """The two polarisations of one structure: a model each (their
    polarisabilities differ only through n_E0), each on its own CUDA stream."""

    def __init__(self, w, sici, rho, precision="mixed", solver=None, device="cuda"):
        import torch

        from dda_model import DDAModel

        kw = model_kwargs(w, sici)
        self.models = [DDAModel(**dict(kw, n_E0=e), precision=precision) for e in ([1, 0, 0], [0, 1, 0])]
        for m in self.models:
            m.setDensities(rho)
            if solver is None:
                m.setPreconditioner("jacobi")
            else:
                m.setSolver("pgmres", **solver)
        self.B = torch.from_numpy(np.stack([incident(w, 0), incident(w, 1)])).to(device)
        self.X = torch.zeros_like(self.B)
        self.side = (torch.cuda.Stream(), torch.cuda.Stream())
        self.tol = w["tol"]

    def step(self, prec, max_iter=MAX_ITER):
        import torch

        stream = torch.cuda.current_stream()
        for m in self.models:
            m.setPrecision(prec)
        out = [None, None]

        def solve(k):
            out[k] = self.models[k].solve_batch_device(self.B[k].data_ptr(), self.X[k].data_ptr(), 1, True, max_iter,
                                                       self.tol, self.side[k].cuda_stream)

        for sd in self.side:
            sd.wait_stream(stream)
        both(solve)
        for sd in self.side:
            stream.wait_stream(sd)
        return out[0] + out[1]

    def timed(self, prec, k, max_iter=MAX_ITER):
        import torch

        stream = torch.cuda.current_stream()
        times, infos = [], None
        for _ in range(k):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            infos = self.step(prec, max_iter)
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
            log(f"{prec}: {times[-1]:.1f} ms " + ", ".join(
                f"{i['status']} it={i['iterations']} mv={i['inner_iterations']} err={i['true_error']:.2e}"
                for i in infos))
        return times, infos


def summary(ts, infos):
    q = np.percentile
    return {"solves_per_s": 2 * len(ts) / (sum(ts) / 1e3), "ms_per_step": statistics.mean(ts),
            "p50_ms": float(q(ts, 50)), "p99_ms": float(q(ts, 99)),
            "status": [i["status"] for i in infos], "true_residual": [i["true_error"] for i in infos],
            "operator_applications": [i["inner_iterations"] for i in infos],
            "gmres_steps": [i["iterations"] for i in infos], "refinements": [i["refinements"] for i in infos]}


def run_isolated16_gpu(sici):
    """The 16x16x8 isolated workload (the reference arm's) on the GPU: the reference's
    algorithm (unscaled complex128 BiCGSTAB from zero to a 1e-8 recursive
    residual) and the mixed-precision refinement, both polarisations."""
    rho = small16_design()
    out = {}
    for name, prec, solver in (("reference_algorithm", "complex128", "none"), ("mixed", "mixed", "jacobi")):
        pair = PolPair(SMALL16, sici, rho, precision="mixed")
        for m in pair.models:
            m.setPreconditioner(solver)
        pair.timed(prec, 2, 100000)
        ts, infos = pair.timed(prec, 5, 100000)
        out[name] = {"solves_per_s": 2 * len(ts) / (sum(ts) / 1e3), "ms_per_step": statistics.mean(ts),
                     "iterations": [i["iterations"] for i in infos], "status": [i["status"] for i in infos]}
    return out


def run_isolated(sici, steps=2):
    """The isolated 128x128x32 structure (no periodic images), mixed-precision
    BiCGSTAB refinement: the previous headline workload, for continuity."""
    w = dict(WORKLOAD, M=0)
    pair = PolPair(w, sici, design(w))
    pair.timed("mixed", 1)
    ts, infos = pair.timed("mixed", steps)
    return dict(summary(ts, infos), workload="128x128x32 isolated, mixed BiCGSTAB refinement")


def run_periodic64(sici):
    """The 64x64x16 workload: periodic 64d, |m|,|n| <= 50, rho ~ U[0,1] per
    dipole, complex128 throughout: the operator, a complex128 solve to 1e-8
    with the periodic solver, and the lattice sums."""
    from dda_model import DDAModel

    w = dict(WORKLOAD, nx=64, ny=64, nz=16, period=64, M=50)
    m = DDAModel(**model_kwargs(w, sici), precision="mixed")
    m.setDensities(np.random.default_rng(w["seed"]).random(m.N))
    ms, passes = m.profile_matvec("complex128", nrhs=1, iters=50)
    m.setSolver("pgmres", **SOLVER)
    out = {"workload": "64x64x16 dipoles, periodic 64d, |m|,|n|<=50, rho ~ U[0,1] per dipole",
           "matvec_c128_us": ms * 1e3, "matvec_pass_us": [p * 1e3 for p in passes],
           "matvec_gbs_algorithmic": 1648.0 * m.N / (ms * 1e-3) / 1e9, "lattice": lattice_record(m, w)}
    for prec in ("complex128", "mixed"):
        m.setPrecision(prec)
        t0 = time.perf_counter()
        m.solveElectricField(None, MAX_ITER, 1e-8)
        out[f"solve_{prec}_s"] = time.perf_counter() - t0
        out[f"solve_{prec}"] = m.last_solve
    return out


def run_gradient(sici):
    """The differentiation step: 96x96x24 dipoles, periodic 96d,
    |m|,|n| <= 50, raw rho ~ U[0,1] -> radius-2 cone filter -> tanh (beta 8,
    eta 0.5) -> densities, objective mean |E|^2 over an 8x8x1 patch 3 cells
    above the top face; forward solve + adjoint gradient through
    dda_model.autograd (densities and gradient stay on the GPU), mixed
    precision to a 1e-10 true residual."""
    import torch

    from dda_model import DDAModel
    from dda_model.autograd import design_objective

    nx, ny, nz = 96, 96, 24
    w = dict(WORKLOAD, nx=nx, ny=ny, nz=nz, period=96, M=50)
    m = DDAModel(**model_kwargs(w, sici), precision="mixed")
    m.setSolver("pgmres", **SOLVER)
    c0x, c0y = nx // 2 - 4, ny // 2 - 4
    m.setObservationPoints(np.array([[x, y, nz - 1 + 3] for x in range(c0x, c0x + 8) for y in range(c0y, c0y + 8)]))
    raw = torch.tensor(np.random.default_rng(44).random((nx, ny, nz)), device="cuda", requires_grad=True)
    times = []
    for k in range(2):
        raw.grad = None
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        J = design_objective(raw, m, radius=2.0, beta=8.0, eta=0.5, kind="patch", max_iter=MAX_ITER, tol=1e-10)
        t1 = time.perf_counter()
        J.backward()
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        times.append((t1 - t0, t2 - t1))
    fwd = statistics.median(t[0] for t in times)
    bwd = statistics.median(t[1] for t in times)
    return {"workload": "96x96x24 periodic 96d, |m|,|n|<=50, filter+tanh, patch objective, mixed to 1e-10",
            "forward_s": fwd, "adjoint_s": bwd, "gradients_per_s": 1.0 / (fwd + bwd),
            "forward": m.last_solve, "adjoint": m.last_adjoint, "objective": float(J),
            "path": "raw design (CUDA tensor) -> design kernels -> device densities -> solve -> objective; "
                    "backward: adjoint solve -> device gradient -> design adjoint kernels"}


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import torch

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
        pg = dist
    import dda_model
    from dda_model import DDAModel

    w = workload(args.small)
    sici = dda_model.sici_tables()
    if args.profile_gmres > 0:
        return run_profile_gmres(args.profile_gmres, sici)
    rho = design(w)
    t0 = time.perf_counter()
    pair = PolPair(w, sici, rho, solver=SOLVER, device=f"cuda:{local}")
    setup_s = time.perf_counter() - t0
    m = pair.models[0]
    log(f"models built in {setup_s:.2f} s (lattice {m.info['lattice_ms']:.1f} ms, tensor FFT "
        f"{m.info['tensor_fft_ms']:.1f} ms)")
    if args.profile_gs > 0:
        ms = m.profile_gram_schmidt("mixed", GS_NV, args.profile_gs)
        print(json.dumps({"nv": GS_NV, "ms_projection": ms[0], "ms_update": ms[1]}))
        return 0
    if args.profile_matvec > 0:
        for prec in ("mixed", "complex128"):
            ms, passes = m.profile_matvec(prec, nrhs=1, iters=args.profile_matvec)
            print(json.dumps({"precision": prec, "ms_matvec": ms, "ms_pass": passes}))
        return 0
    if args.profile_solve > 0:
        P0 = np.zeros(3 * m.N, dtype=np.complex128)
        m.setPrecision("mixed")
        for k in range(args.profile_solve):
            n0 = DDAModel.kernel_launches()
            m.solveElectricField(P0, MAX_ITER, w["tol"])
            print(json.dumps({"solve": k, "launches_before": n0, "launches_after": DDAModel.kernel_launches(),
                              "info": m.last_solve}), flush=True)
        return 0
    N = m.N
    stream = torch.cuda.current_stream()

    for _ in range(args.warmup):
        pair.step("mixed")
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    launches0 = DDAModel.kernel_launches()
    with ClockSampler(local) as clk:
        t_mixed, info_mixed = pair.timed("mixed", args.steps)
    launches = DDAModel.kernel_launches() - launches0
    torch.cuda.synchronize()
    # plain complex128: the same solver with complex128 inner solves (one
    # warm-up and one timed step: each takes ~2-3x the mixed one)
    pair.step("complex128")
    plain_steps = 1
    t_plain, info_plain = pair.timed("complex128", plain_steps)
    torch.cuda.synchronize()

    from dda_model.replicas import max_over_ranks

    def agg(ts):
        # device-timed region of every rank; the job's time is the slowest rank's
        return max_over_ranks(sum(ts), f"cuda:{local}")

    tot_mixed = agg(t_mixed)
    tot_plain = agg(t_plain)
    value = 2 * args.steps * world / (tot_mixed / 1e3)
    plain = 2 * plain_steps * world / (tot_plain / 1e3)

    # roofline of the dominant kernel: the complex64 fused matvec (3 passes)
    ms64, pass64 = m.profile_matvec("mixed", nrhs=1, iters=20)
    ms128, pass128 = m.profile_matvec("complex128", nrhs=1, iters=10)
    # the largest single kernel of the solve: the Gram-Schmidt projection pass
    gs_proj, gs_upd = m.profile_gram_schmidt("mixed", GS_NV, 20)
    gs_bytes = (GS_NV + 1) * 3.0 * N * 8
    gs_upd_bytes = (GS_NV + 2) * 3.0 * N * 8
    trg = traffic_record("k_multidot_bulk_gs_traffic.txt") or {}
    peak, peak_kind = peaks()
    b64 = 824.0 * N
    b128 = 1648.0 * N
    achieved = b64 / (ms64 * 1e-3) / 1e9
    tr = traffic_record()
    mv_mixed = statistics.mean(i["inner_iterations"] for i in info_mixed)

    # end to end through the public API with host buffers (mixed): per step,
    # each polarisation's model gets the densities from the host, solves and
    # returns its field to the host, the two on two host threads
    for mm in pair.models:
        mm.setPrecision("mixed")
    P0 = np.zeros(3 * N, dtype=np.complex128)
    rho_host = np.ascontiguousarray(rho)
    fields = [None, None]

    def public(k):
        pair.models[k].setDensities(rho_host)
        pair.models[k].solveElectricField(P0, MAX_ITER, w["tol"])
        fields[k] = pair.models[k].getElectricField()

    # (the models and their kernels are warm from the steps above)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    te = []
    e2e_steps = 1
    for _ in range(e2e_steps):
        t1 = time.perf_counter()
        both(public)
        te.append(time.perf_counter() - t1)
    e2e_tot = max_over_ranks(sum(te), f"cuda:{local}")
    e2e = 2 * e2e_steps * world / e2e_tot
    E = np.concatenate(fields)
    assert np.all(np.isfinite(E))

    # the reference's own algorithm (unscaled complex128 BiCGSTAB, stopping on
    # the recursive residual) on this workload, with a bounded iteration budget
    ref_model = DDAModel(**model_kwargs(w, sici), precision="complex128")
    ref_model.setDensities(rho)
    Bx = pair.B[0:1].contiguous()
    Xx = torch.zeros_like(Bx)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    budget = 3000
    e0.record(stream)
    ref_info = ref_model.solve_batch_device(Bx.data_ptr(), Xx.data_ptr(), 1, True, budget, w["tol"],
                                            stream.cuda_stream)[0]
    e1.record(stream)
    e1.synchronize()
    ref_alg = {"iterations": ref_info["iterations"], "status": ref_info["status"],
               "recursive_residual": ref_info["error"], "ms": e0.elapsed_time(e1), "iteration_budget": budget,
               "iterations_per_s": ref_info["iterations"] / (e0.elapsed_time(e1) / 1e3)}
    log(f"reference algorithm on GPU: {ref_alg}")
    del ref_model

    extra = {}
    if not args.small:
        for name, fn in (("isolated_128x128x32", lambda: run_isolated(sici)), ("isolated_16x16x8_gpu", lambda: run_isolated16_gpu(sici)),
                         ("periodic_64x64x16", lambda: run_periodic64(sici)), ("gradient_96x96x24", lambda: run_gradient(sici)),
                         ("reference_cufft_restatement", lambda: run_cufft_restatement(dict(w, M=0), sici))):
            extra[name] = fn()
            log(f"{name}: {json.dumps(extra[name])[:400]}")
            torch.cuda.empty_cache()
    serving = None
    if not args.no_serving and not args.small:
        serving = run_serving(rank, world, f"cuda:{local}" if world > 1 else None)

    cpu = None
    lat_cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        port = CpuPort(w, rho, images=False)
        s_apply = statistics.median([port.per_apply(1) for _ in range(3)])
        mv_plain = statistics.mean(i["inner_iterations"] for i in info_plain)
        cores = port.cores
        cpu = {"value": 1.0 / (s_apply * mv_plain), "unit": "solves/s", "cores": cores, "kind": "port",
               "extrapolated": True,
               "sample": f"3 complex128 operator applications of the oracle port (scipy.fft, {cores} workers, the "
                         f"reference's 2n-1 padding) on the full 128x128x32 grid, {s_apply:.3f} s each, times the "
                         f"{mv_plain:.0f} operator applications the complex128 solve of this solver takes on the GPU "
                         f"(the reference's own BiCGSTAB does not converge here; a measured full CPU solve is the "
                         f"reference arm's 16x16x8 line)"}
        lat_cpu = cpu_lattice_rate(w, npts=300)[0]

    if rank == 0:
        q = np.percentile
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": statistics.mean(t_mixed), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c64 matvec, f64 sums, c128 refinement",
            "data": "synthetic", "config": config_block(w, world),
            "p50_ms": float(q(t_mixed, 50)), "p99_ms": float(q(t_mixed, 99)),
            "solver": dict(SOLVER, name="deflated restarted GMRES in complex128 refinement"),
            "mixed": summary(t_mixed, info_mixed),
            "plain_c128": dict(summary(t_plain, info_plain), value=plain, unit="solves/s", warmup=1,
                               steps=plain_steps),
            "mixed_over_plain": value / plain,
            "reference_algorithm_gpu": ref_alg,
            "roofline_gram_schmidt": {"bound": "hbm", "achieved": gs_bytes / (gs_proj * 1e-3) / 1e9, "peak": peak,
                         "unit": "GB/s", "frac": gs_bytes / (gs_proj * 1e-3) / 1e9 / peak, "peak_kind": peak_kind,
                         "traffic": trg.get("bytes_per_launch"),
                         "traffic_source": "profiles/k_multidot_bulk_gs_traffic.txt (ncu dram bytes, nv = 25)",
                         "kernel": f"k_multidot_bulk<float2> (GMRES projections V^H w and ||w||^2 against "
                                   f"{GS_NV} basis vectors, + block sums), 22% of the solve's device time "
                                   f"(profiles/launches_gmres_solve_128x128x32.md)",
                         "algorithmic_bytes": gs_bytes, "ms": gs_proj,
                         "update": {"kernel": "k_gs_update_scale<float2>", "ms": gs_upd,
                                    "achieved": gs_upd_bytes / (gs_upd * 1e-3) / 1e9,
                                    "frac": gs_upd_bytes / (gs_upd * 1e-3) / 1e9 / peak}},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": (tr or {}).get("bytes_per_launch_cold"),
                         "traffic_warm": (tr or {}).get("bytes_per_launch_warm"),
                         "dram_frac": ((tr or {}).get("bytes_per_launch_cold") or 0) / (ms64 * 1e-3) / 1e9 / peak,
                         "traffic_source": "profiles/matvec_c64_traffic.txt (ncu dram bytes, 3 passes, 1 RHS)",
                         "kernel": "fused complex64 matvec (3 passes), 1 RHS: 48% of the solve's device time, its "
                                   "pass 2 (k_xconv_reg, 24%) the largest single kernel "
                                   "(profiles/launches_gmres_solve_128x128x32.md)",
                         "algorithmic_bytes": b64, "ms": ms64, "pass_ms": pass64,
                         "c128": {"ms": ms128, "achieved": b128 / (ms128 * 1e-3) / 1e9,
                                  "frac": b128 / (ms128 * 1e-3) / 1e9 / peak, "pass_ms": pass128},
                         "share_of_solve": mv_mixed * ms64 / (statistics.mean(t_mixed) / 2)},
            "matvecs_per_s": 1e3 / ms64,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e, "unit": "solves/s", "h2d_bytes_per_step": 2 * 8 * N,
                    "d2h_bytes_per_step": 2 * 16 * 3 * N, "steps": e2e_steps,
                    "path": "per polarisation: setDensities + solveElectricField + getElectricField "
                            "(host numpy buffers), the two polarisations' models on two host threads"},
            "clocks": clk.summary(),
            "gpu_launches": int(launches),
            "setup_s": setup_s,
            "lattice_128x128x32": lattice_record(m, w, lat_cpu),
            **extra,
            "serving": serving,
        }
        print(json.dumps(line))
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
