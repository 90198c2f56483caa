"""ORACLE — test infrastructure only.

This module is the CPU checker for the CUDA implementation.  Only the tests,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import it;
the product (``dda_model`` and ``libtdda``) never does.

It restates, in numpy complex128 (plus the plain-C lattice sums in
``oracle/lattice.c``), the algorithm of Topo-DDA's forward and adjoint solve:

==========================================  ======================================
oracle function                             reference (path within Topo-DDA)
==========================================  ======================================
``sici_tables``                             python_bindings/dda_model/__init__.py:205-210
``generate_geometry``                       python_bindings/dda_model/__init__.py:8-20
``lattice_tensor`` (C)                      src/AProductCore.cpp:12-298,335-459; src/SiCi.cpp:12-44
``rescale_material``                        src/AProductCore.cpp:25-33
``get_alpha``                               src/Tools.cpp:353-366
``parameter_map``                           src/DDAModel.cpp:163-247 (FCurrentinsert :37-64)
``OracleModel.al`` (material interp.)       src/DDAModel.cpp:319-328,1122-1151
``incident_field``                          src/DDAModel.cpp:312-316,1113-1120
``OracleModel.aproduct``                    src/AProductCore.cpp:461-515, src/Kernel.cu:44-125
``OracleModel.aproduct_with_alb``           src/DDAModel.cpp:1194-1203
``bicgstab``                                src/DDAModel.cpp:899-1009
``OracleModel.solve_electric_field``        src/DDAModel.cpp:874-885,1153-1192
``OracleModel.calculate_objective``         src/ObjDDAModel.cpp:103-218 (IntegratedE)
``OracleModel.calculate_gradients``         src/DDAModel.cpp:398-578
``OracleModel.dense_operator``              (dense 3N x 3N form of the same operator)
``beta_schedule``                           src/FilterOption.cpp:23-45, src/Tools.cpp:473-516
``smooth_density`` / ``smooth_density_d``   src/FilterOption.cpp:48-62, src/DDAModel.cpp:340-352
``LegacyFilter`` (weights)                  src/DDAModel.cpp:66-77,580-712
``LegacyFilter.update``                     src/DDAModel.cpp:774-838 (filter branch)
``LegacyFilter.gradients``                  src/DDAModel.cpp:354-396
==========================================  ======================================

Parity pins: ``tests/test_oracle_golden.py`` checks this oracle against the
reference's only known-answer test (objective 11.005338768207627 at rel 1e-4
on the 22x22x10 fixture, python_tests/test_DDAModelWrapper.py:32-40) and
against the fixture geometry ordering (:42-48), plus a dense direct solve.
"""
from __future__ import annotations

import ctypes
import itertools
import math
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle_lattice.so")
_lib = None


def _load_lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(
            os.path.join(_HERE, "lattice.c")
        ):
            subprocess.run(["make", "-s", "-C", _HERE], check=True)
        lib = ctypes.CDLL(_LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        lib.oracle_lattice.argtypes = [
            ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
            ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
            dp, dp, ctypes.c_long, ctypes.c_double, ctypes.c_int, ctypes.c_int, dp,
        ]
        lib.oracle_lattice.restype = ctypes.c_int
        lib.oracle_green_image.argtypes = [
            ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
            ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
            dp, dp, ctypes.c_long, ctypes.c_double, dp,
        ]
        lib.oracle_green.argtypes = [
            ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
            ctypes.c_double, dp, dp, ctypes.c_long, ctypes.c_double, dp,
        ]
        lib.oracle_get_si.argtypes = [dp, ctypes.c_long, ctypes.c_double, ctypes.c_double]
        lib.oracle_get_si.restype = ctypes.c_double
        lib.oracle_get_ci.argtypes = [dp, ctypes.c_long, ctypes.c_double, ctypes.c_double]
        lib.oracle_get_ci.restype = ctypes.c_double
        lib.oracle_guard_hits.restype = ctypes.c_long
        lib.oracle_lattice_points.argtypes = [
            ctypes.c_int, ctypes.c_long, dp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
            ctypes.c_double, ctypes.c_double, dp, dp, ctypes.c_long, ctypes.c_double, dp,
        ]
        _lib = lib
    return _lib


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


# ----------------------------------------------------------------------------
# inputs
# ----------------------------------------------------------------------------

def sici_tables(delta: float = 0.1, n: int = 1_000_000):
    """Sine/cosine-integral tables exactly as DDAModelWrapper builds them
    (python_bindings/dda_model/__init__.py:205-210): n-1 samples of
    np.linspace(delta, delta*n, n-1), which the C++ side looks up as if they sat
    at (k+1)*delta (src/SiCi.cpp:12-44)."""
    from scipy.special import sici

    pos = np.linspace(delta, delta * n, n - 1)
    si, ci = sici(pos)
    return np.ascontiguousarray(si, dtype=np.float64), np.ascontiguousarray(ci, dtype=np.float64)


def generate_geometry(nx: int, ny: int, nz: int) -> np.ndarray:
    """x-fastest integer coordinates, flattened [x0,y0,z0,x1,...]
    (python_bindings/dda_model/__init__.py:8-20)."""
    mesh = itertools.product(range(nz), range(ny), range(nx))
    g = np.array(list(mesh))[:, ::-1]
    return g.flatten().astype(np.int64)


def rescale_material(material, nback: float) -> np.ndarray:
    """material / nback^2, then +0.01 to any entry with |m| < 1.01
    (src/AProductCore.cpp:25-33)."""
    m = np.asarray(material, dtype=np.complex128) / (nback * nback)
    m = np.where(np.abs(m) < 1.01, m + 0.01, m)
    return m


def get_alpha(lam, K, d, diel, n_E0, n_K):
    """Lattice-dispersion-relation polarisability (src/Tools.cpp:353-366)."""
    b1, b2, b3 = -1.891531, 0.1648469, -1.7700004
    diel = np.asarray(diel, dtype=np.complex128)
    a1 = (3 * d**3 / (4 * math.pi)) * (diel - 1.0) / (diel + 2.0)
    res = 0.0 + (2.0 / 3.0) * (K * d) ** 3 * 1j
    S = (n_E0[0] * n_K[0]) ** 2 + (n_E0[1] * n_K[1]) ** 2 + (n_E0[2] * n_K[2]) ** 2
    res = 1.0 + (a1 / d**3) * ((b1 + diel * b2 + diel * b3 * S) * (K * d) ** 2 - res)
    return a1 / res


def interp_material(rho, material):
    """dielectric_old -> diel by linear interpolation between the two materials
    (src/DDAModel.cpp:319-326)."""
    rho = np.asarray(rho, dtype=np.float64)
    lf = np.floor(rho).astype(np.int64)
    ln = np.where(lf >= 1, lf, lf + 1)
    if np.any(lf < 0) or np.any(ln > len(material) - 1):
        raise ValueError("density outside [0, 1]")
    m = np.asarray(material)
    return m[lf] + (rho - lf) * (m[ln] - m[lf])


def parameter_map(geometry: np.ndarray, Nz: int, symmetry: str, symaxis):
    """geometryPara / Paratogeometry / NFpara (src/DDAModel.cpp:163-225)."""
    if symmetry == "None":
        dividesym = 1
    elif symmetry == "4fold":
        dividesym = 4
    else:
        raise RuntimeError("Unknown internal error")  # `throw 1` (src/DDAModel.cpp:170-173)
    N = len(geometry) // 3
    nf = int(round(len(geometry) // 3 // Nz // dividesym))
    cur: dict = {}
    pos = 0
    gp = np.zeros(N, dtype=np.int64)
    for i in range(N):
        xy = (int(geometry[3 * i]), int(geometry[3 * i + 1]))
        if xy not in cur:
            if symmetry == "None":
                cur[xy] = pos
                pos += 1
            else:
                s1 = (int(round(2 * symaxis[0] - xy[0])), xy[1])
                s2 = (int(round(2 * symaxis[0] - xy[0])), int(round(2 * symaxis[1] - xy[1])))
                s3 = (xy[0], int(round(2 * symaxis[1] - xy[1])))
                if s1 in cur:
                    cur[xy] = cur[s1]
                elif s2 in cur:
                    cur[xy] = cur[s2]
                elif s3 in cur:
                    cur[xy] = cur[s3]
                else:
                    cur[xy] = pos
                    pos += 1
        gp[i] = cur[xy]
    p2g = [[] for _ in range(nf)]
    for i in range(N):
        if gp[i] >= nf:
            raise RuntimeError("parameter index beyond NFpara")
        p2g[gp[i]].append(i)
    return gp, p2g, nf


def incident_field(geometry, K, d, E0, n_E0, n_K):
    """E_c = E0 n_E0,c exp(i K d (n_K . idx)) (src/DDAModel.cpp:312-316)."""
    g = np.asarray(geometry, dtype=np.float64).reshape(-1, 3)
    ph = K * d * (n_K[0] * g[:, 0] + n_K[1] * g[:, 1] + n_K[2] * g[:, 2])
    e = np.cos(ph) + 1j * np.sin(ph)
    E = np.empty(3 * len(g), dtype=np.complex128)
    for c in range(3):
        E[c::3] = E0 * n_E0[c] * e
    return E


def lattice_tensor(Nx, Ny, Nz, d, K, Lm, Ln, MAXm, MAXn, method, si, ci, delta, full=False,
                   nthreads=None):
    """Padded interaction tensor in the reference AHos layout, returned as a
    complex array of shape (2Nx-1, 2Ny-1, 2Nz-1, 6) (components xx,xy,xz,yy,yz,zz).
    Lm, Ln are lengths (nm).  See oracle/lattice.c."""
    lib = _load_lib()
    NxF, NyF, NzF = 2 * Nx - 1, 2 * Ny - 1, 2 * Nz - 1
    out = np.zeros(12 * NxF * NyF * NzF, dtype=np.float64)
    si = np.ascontiguousarray(si, dtype=np.float64)
    ci = np.ascontiguousarray(ci, dtype=np.float64)
    meth = {"FCD": 0, "LDR": 1}[method]
    if nthreads is None:
        nthreads = os.cpu_count() or 1
    lib.oracle_lattice(Nx, Ny, Nz, d, K, Lm, Ln, MAXm, MAXn, meth, _dptr(si), _dptr(ci), len(si),
                       delta, 1 if full else 0, nthreads, _dptr(out))
    return out.view(np.complex128).reshape(NxF, NyF, NzF, 6)


def green_image(method, x, y, z, m, n, Lm, Ln, K, d, si, ci, delta):
    """One damped image term A_dic_generator(x,y,z,m,n) as a 3x3 complex matrix."""
    lib = _load_lib()
    out = np.zeros(12)
    lib.oracle_green_image({"FCD": 0, "LDR": 1}[method], x, y, z, m, n, Lm, Ln, K, d,
                           _dptr(si), _dptr(ci), len(si), delta, _dptr(out))
    return _sym33(out.view(np.complex128))


def green(method, x, y, z, K, d, si, ci, delta):
    """Undamped single term A_dic_generator(x,y,z) as a 3x3 complex matrix."""
    lib = _load_lib()
    out = np.zeros(12)
    lib.oracle_green({"FCD": 0, "LDR": 1}[method], x, y, z, K, d, _dptr(si), _dptr(ci), len(si),
                     delta, _dptr(out))
    return _sym33(out.view(np.complex128))


def _sym33(c6):
    xx, xy, xz, yy, yz, zz = c6
    return np.array([[xx, xy, xz], [xy, yy, yz], [xz, yz, zz]], dtype=np.complex128)


# ----------------------------------------------------------------------------
# solver
# ----------------------------------------------------------------------------

@dataclass
class SolveInfo:
    iterations: int
    error: float
    converged: bool
    breakdown: bool


def bicgstab(matvec, E, P0, max_iter, tol):
    """BiCGSTAB exactly as DDAModel::bicgstab (src/DDAModel.cpp:899-1009):
    one full step before the loop, Eigen conjugate-first dots, stop on the
    recursive residual ||r||/||E|| <= tol, breakdown guard r0.rl == 0.
    Returns (P, SolveInfo); iterations counts loop passes (it+1)."""
    dot = np.vdot
    P = np.array(P0, dtype=np.complex128, copy=True)
    Enorm = np.linalg.norm(E)
    r = E - matvec(P)
    r0 = r.copy()
    p = r.copy()
    Ap0 = matvec(p)
    alpha = dot(r0, r) / dot(r0, Ap0)
    t = r - alpha * Ap0
    At0 = matvec(t)
    zeta = dot(At0, t) / dot(At0, At0)
    u = zeta * Ap0
    z = zeta * r - alpha * u
    P = P + alpha * p + z
    rl = r
    r = t - zeta * At0
    for it in range(max_iter):
        r0dotrl = dot(r0, rl)
        if r0dotrl.real == 0 and r0dotrl.imag == 0:
            return P, SolveInfo(it + 1, float(np.linalg.norm(r) / Enorm), False, True)
        beta = (alpha / zeta) * dot(r0, r) / dot(r0, rl)
        p = r + beta * (p - u)
        Ap = matvec(p)
        alpha = dot(r0, r) / dot(r0, Ap)
        t = r - alpha * Ap
        At = matvec(t)
        zeta = dot(At, t) / dot(At, At)
        u = zeta * Ap
        z = zeta * r - alpha * u
        P = P + alpha * p + z
        rl = r
        r = t - zeta * At
        err = np.linalg.norm(r) / Enorm
        if err <= tol:
            return P, SolveInfo(it + 1, float(err), True, False)
    return P, SolveInfo(max_iter, float(np.linalg.norm(r) / Enorm), False, False)


class OracleModel:
    """CPU restatement of DDAModel for the forward/adjoint path, constructed
    from the same 35 arguments as the pybind11 constructor
    (python_bindings/PythonBindings.cpp:19-59).  The filter arguments are
    accepted and ignored (the reference's own filter is disabled on every
    Python path, python_bindings/dda_model/__init__.py:128)."""

    def __init__(self, betaMin, betaMax, ita, betaType, filterIterations, filterRadii, useFilter,
                 symmetryType, symmetryAxis, isPeriodic, objectiveName, objPara, geometry,
                 inputDielectrics, num_x, num_y, num_z, num_total, n_K, E0, n_E0, lam, material,
                 nback, MAXm, MAXn, Lm, Ln, matrixAMethodName, d, sineIntegralValues,
                 cosineIntegralValues, integralDelta, verbose=False, lattice=None,
                 lattice_full=False):
        g = np.asarray(geometry, dtype=np.int64).copy()
        self.geometry = g
        self.Nx, self.Ny, self.Nz, self.N = int(num_x), int(num_y), int(num_z), int(num_total)
        if len(g) != 3 * self.N:
            raise RuntimeError("geometry size != 3 * num_total")
        self.d = float(d)
        self.lam = float(lam)
        self.nback = float(nback)
        self.K = 2.0 * math.pi / (self.lam / self.nback)
        self.material = rescale_material(material, self.nback)
        self.n_K = np.asarray(n_K, dtype=np.float64)
        self.n_E0 = np.asarray(n_E0, dtype=np.float64)
        self.E0 = float(E0)
        self.objPara = list(objPara)
        self.powNum = int(round(self.objPara[0]))
        diel_in = np.asarray(inputDielectrics, dtype=np.float64)
        if len(diel_in) != len(g):
            raise RuntimeError("Unknown internal error")
        self.geometryPara, self.p2g, self.NFpara = parameter_map(g, self.Nz, symmetryType,
                                                                 symmetryAxis)
        inputmap = {}
        for i in range(len(g) // 3):
            inputmap[(g[3 * i], g[3 * i + 1], g[3 * i + 2])] = diel_in[3 * i]
        self.parameters = np.array(
            [inputmap[tuple(g[3 * self.p2g[i][0]:3 * self.p2g[i][0] + 3])] for i in range(self.NFpara)],
            dtype=np.float64)
        self.MAXm, self.MAXn = int(MAXm), int(MAXn)
        self.Lm, self.Ln = float(Lm) * self.d, float(Ln) * self.d
        self.method = matrixAMethodName
        self.si = np.asarray(sineIntegralValues, dtype=np.float64)
        self.ci = np.asarray(cosineIntegralValues, dtype=np.float64)
        self.delta = float(integralDelta)
        if lattice is None:
            lattice = lattice_tensor(self.Nx, self.Ny, self.Nz, self.d, self.K, self.Lm, self.Ln,
                                     self.MAXm, self.MAXn, self.method, self.si, self.ci,
                                     self.delta, full=lattice_full)
        self.A = lattice
        self.NF = lattice.shape[:3]
        import scipy.fft as sfft

        self._fft = sfft
        self.Ahat = [sfft.fftn(lattice[..., l], workers=-1) for l in range(6)]
        self.E_inc = incident_field(g, self.K, self.d, self.E0, self.n_E0, self.n_K)
        self.E = self.E_inc.copy()
        self.P = np.zeros(3 * self.N, dtype=np.complex128)
        self.EResult = np.zeros(3 * self.N, dtype=np.complex128)
        self.E_int = 0.0
        self._update_dielectric()
        self.last_info = None

    # --- material / polarisability ------------------------------------------------
    def _update_dielectric(self):
        rho = self.parameters[self.geometryPara]
        self.dielectric_old = np.repeat(rho, 3)
        self.diel = interp_material(self.dielectric_old, self.material)
        self.al = 1.0 / get_alpha(self.lam, self.K, self.d, self.diel, self.n_E0, self.n_K)

    def al_of_rho(self, rho):
        diel = interp_material(rho, self.material)
        return 1.0 / get_alpha(self.lam, self.K, self.d, diel, self.n_E0, self.n_K)

    def setParameters(self, values):
        v = np.asarray(values, dtype=np.float64)
        if len(v) != self.NFpara:
            raise RuntimeError("Unknown internal error")
        self.parameters = v.copy()
        self._update_dielectric()

    def getParameters(self):
        return self.parameters.copy()

    def getDielectrics(self):
        return self.dielectric_old.copy()

    def getElectricField(self):
        return self.EResult.copy()

    # --- operator -----------------------------------------------------------------
    def aproduct(self, b):
        """Interaction part A.b by zero-padded FFT convolution
        (src/AProductCore.cpp:461-515)."""
        sfft = self._fft
        g = self.geometry.reshape(-1, 3)
        grid = np.zeros((3,) + tuple(self.NF), dtype=np.complex128)
        for c in range(3):
            grid[c][g[:, 0], g[:, 1], g[:, 2]] = b[c::3]
        bh = [sfft.fftn(grid[c], workers=-1) for c in range(3)]
        A00, A01, A02, A11, A12, A22 = self.Ahat
        cx = A00 * bh[0] + A01 * bh[1] + A02 * bh[2]
        cy = A01 * bh[0] + A11 * bh[1] + A12 * bh[2]
        cz = A02 * bh[0] + A12 * bh[1] + A22 * bh[2]
        out = np.empty(3 * self.N, dtype=np.complex128)
        for c, cc in enumerate((cx, cy, cz)):
            y = sfft.ifftn(cc, workers=-1)
            out[c::3] = y[g[:, 0], g[:, 1], g[:, 2]]
        return out

    def aproduct_with_alb(self, b):
        """A.b + (1/alpha) o b (src/DDAModel.cpp:1194-1203)."""
        return self.aproduct(b) + self.al * b

    def dense_operator(self):
        """The same operator as an explicit 3N x 3N matrix (small N only)."""
        g = self.geometry.reshape(-1, 3)
        NxF, NyF, NzF = self.NF
        N = self.N
        M = np.zeros((3 * N, 3 * N), dtype=np.complex128)
        comp = [[0, 1, 2], [1, 3, 4], [2, 4, 5]]
        for i in range(N):
            off = (g[i][None, :] - g)  # r_i - r_j
            ix = off[:, 0] % NxF
            iy = off[:, 1] % NyF
            iz = off[:, 2] % NzF
            blk = self.A[ix, iy, iz]  # (N, 6)
            for a in range(3):
                for b in range(3):
                    M[3 * i + a, b::3] = blk[:, comp[a][b]]
        M[np.arange(3 * N), np.arange(3 * N)] += self.al
        return M

    # --- forward ------------------------------------------------------------------
    def solveElectricField(self, originPolarization, BGS_MAX_ITER, BGS_MAX_ERROR):
        """src/DDAModel.cpp:874-885: P0 -> BiCGSTAB -> E_int = al P / ((2+eps)/3)."""
        P0 = np.asarray(originPolarization, dtype=np.complex128)
        self.P, self.last_info = bicgstab(self.aproduct_with_alb, self.E, P0, int(BGS_MAX_ITER),
                                          float(BGS_MAX_ERROR))
        self.EResult = self.al * self.P / ((2.0 + self.diel) / 3.0)
        return self.last_info

    def _contrib(self, al, P):
        return np.abs(al * P) ** self.powNum

    def calculateObjective(self):
        """IntegratedE: log sum_i sum_c |al_ic P_ic|^pow over every dipole
        (src/ObjDDAModel.cpp:130-157,205-212; the chained comparison at :135 is
        always true)."""
        self.E_int = float(np.sum(self._contrib(self.al, self.P)))
        return math.log(self.E_int)

    # --- adjoint ------------------------------------------------------------------
    def devx_and_adevxp(self, eps, origin):
        """One-sided finite differences in each free parameter
        (src/DDAModel.cpp:471-536)."""
        devx = np.zeros(self.NFpara)
        change = np.zeros(self.N, dtype=np.complex128)
        E_int = self.E_int
        P3 = self.P.reshape(-1, 3)
        al3 = self.al.reshape(-1, 3)
        for i in range(self.NFpara):
            p0 = self.parameters[i]
            sign = -1.0 if p0 >= eps else 1.0
            ptmp = p0 + sign * eps
            idx = np.asarray(self.p2g[i])
            al_new = self.al_of_rho(np.full(len(idx), ptmp))
            old = np.sum(self._contrib(al3[idx], P3[idx]), axis=1)
            new = np.sum(self._contrib(al_new[:, None], P3[idx]), axis=1)
            E_mod = E_int
            for k in range(len(idx)):
                E_mod = E_mod - old[k] + new[k]
            change[idx] = (al_new - al3[idx, 0]) / (sign * eps)
            devx[i] = (math.log(E_mod) - origin) / (sign * eps)
        adevxp = np.repeat(change, 3) * self.P
        return devx, adevxp

    def devp(self, eps, origin):
        """dJ/dx - i dJ/dy by one-sided differences in Re and Im of each P_i
        (src/DDAModel.cpp:538-578)."""
        P = self.P
        al = self.al
        base = self._contrib(al, P).reshape(-1, 3).sum(axis=1)
        res = np.zeros(len(P), dtype=np.complex128)
        E_int = self.E_int
        for i in range(len(P)):
            pos = i // 3
            Pd = P[3 * pos:3 * pos + 3].copy()
            Pd[i % 3] += eps
            c_re = np.sum(self._contrib(al[3 * pos:3 * pos + 3], Pd))
            Pd = P[3 * pos:3 * pos + 3].copy()
            Pd[i % 3] += 1j * eps
            c_im = np.sum(self._contrib(al[3 * pos:3 * pos + 3], Pd))
            res[i] = (math.log(E_int - base[pos] + c_re) - origin) / eps
            res[i] += (math.log(E_int - base[pos] + c_im) - origin) / (1j * eps)
        return res

    def calculateGradients(self, epsilon_partial, originalObjValue, MAX_ITERATION, MAX_ERROR):
        """src/DDAModel.cpp:398-469: FD partials, adjoint solve with the same
        (complex-symmetric) operator, grad = devx - Re(sum lambda * Adevxp).
        As in the reference, the model's P holds the adjoint solution afterwards."""
        devx, adevxp = self.devx_and_adevxp(epsilon_partial, originalObjValue)
        dp = self.devp(epsilon_partial, originalObjValue)
        lam, info = bicgstab(self.aproduct_with_alb, dp, np.zeros_like(dp), int(MAX_ITERATION),
                             float(MAX_ERROR))
        self.adjoint_info = info
        self.P = lam
        prod = (lam * adevxp).reshape(-1, 3).sum(axis=1)
        mult = np.zeros(self.NFpara, dtype=np.complex128)
        np.add.at(mult, self.geometryPara, prod)
        return devx - mult.real

    # --- observation patch (extension objective; no reference counterpart) ------
    def observation_matrix(self, obs):
        """Gobs[3 nobs, 3N]: the damped periodic lattice sum G(r_o - r_j) between
        every observation grid point r_o and every dipole r_j (component blocks
        xx,xy,xz / yx,yy,yz / zx,zy,zz)."""
        lib = _load_lib()
        g = self.geometry.reshape(-1, 3)
        obs = np.asarray(obs).reshape(-1, 3)
        comp = [[0, 1, 2], [1, 3, 4], [2, 4, 5]]
        G = np.zeros((3 * len(obs), 3 * self.N), dtype=np.complex128)
        for k, o in enumerate(obs):
            off = np.ascontiguousarray(((o[None, :] - g) * self.d).astype(np.float64))
            out = np.zeros(12 * len(g))
            lib.oracle_lattice_points({"FCD": 0, "LDR": 1}[self.method], len(g), _dptr(off), self.MAXm,
                                      self.MAXn, self.Lm, self.Ln, self.K, self.d, _dptr(self.si),
                                      _dptr(self.ci), len(self.si), self.delta, _dptr(out))
            T = out.view(np.complex128).reshape(-1, 6)
            for a in range(3):
                for b in range(3):
                    G[3 * k + a, b::3] = T[:, comp[a][b]]
        return G

    def observation_field(self, obs):
        """E_obs = E_inc(r_o) - sum_j G(r_o - r_j) P_j at grid points obs[nobs, 3]."""
        obs = np.asarray(obs).reshape(-1, 3)
        ph = self.K * self.d * (obs.astype(np.float64) @ self.n_K)
        Einc = self.E0 * self.n_E0[None, :] * np.exp(1j * ph)[:, None]
        return Einc - (self.observation_matrix(obs) @ self.P).reshape(-1, 3)

    def patch_objective(self, obs):
        E = self.observation_field(obs)
        return float(np.sum(np.abs(E) ** 2) / len(E))

    # --- per-dipole densities (extension of setParameters) ----------------------
    def set_densities(self, rho):
        """Free per-dipole densities (no symmetry map): rho[N] -> diel, 1/alpha."""
        rho = np.asarray(rho, dtype=np.float64)
        if rho.shape != (self.N,):
            raise RuntimeError("densities must have num_total entries")
        self.dielectric_old = np.repeat(rho, 3)
        self.diel = interp_material(self.dielectric_old, self.material)
        self.al = 1.0 / get_alpha(self.lam, self.K, self.d, self.diel, self.n_E0, self.n_K)

    def density_gradient(self, kind="integrated", obs=None):
        """Exact dJ/drho_j by a dense direct forward and adjoint solve (small N).

        (A + diag al) P = E with a complex-symmetric matrix, so for
        J(P, al): dJ/drho_j = Re(sum_c [dJ/dal_jc - lambda_jc P_jc] dal_j/drho_j)
        with (A + diag al) lambda = v, v = dJ/dP (holomorphic part)."""
        M = self.dense_operator()
        P = np.linalg.solve(M, self.E)
        self.P = P
        if kind == "integrated":
            q = self.powNum
            z = self.al * P
            S = float(np.sum(np.abs(z) ** q))
            w = q * np.abs(z) ** (q - 2) * np.conj(z)  # d|z|^q = Re(w dz)
            v = w * self.al / S
            explicit = w * P / S
        elif kind == "patch":
            G = self.observation_matrix(obs)
            nobs = G.shape[0] // 3
            ph = self.K * self.d * (np.asarray(obs).reshape(-1, 3).astype(np.float64) @ self.n_K)
            Einc = (self.E0 * self.n_E0[None, :] * np.exp(1j * ph)[:, None]).ravel()
            E = Einc - G @ P
            v = -(2.0 / nobs) * (G.T @ np.conj(E))
            explicit = np.zeros(3 * self.N, dtype=np.complex128)
        else:
            raise ValueError(kind)
        lam = np.linalg.solve(M, v)  # M^T = M
        per = (explicit - lam * P).reshape(-1, 3).sum(axis=1)
        return (per * self.dal_drho()).real

    # --- analytic derivative (used to check the analytic adjoint) ---------------
    def dal_drho(self):
        """d(1/alpha)/d rho per dipole, in closed form from get_alpha."""
        b2, b3 = 0.1648469, -1.7700004
        S = (self.n_E0[0] * self.n_K[0]) ** 2 + (self.n_E0[1] * self.n_K[1]) ** 2 + (
            self.n_E0[2] * self.n_K[2]) ** 2
        eps = self.diel[0::3]
        c = 3 * self.d**3 / (4 * math.pi)
        dal_deps = -3.0 / (c * (eps - 1.0) ** 2) + (b2 + b3 * S) * self.K**2 / self.d
        rho = self.dielectric_old[0::3]
        deps_drho = np.where(np.floor(rho) >= 1, self.material[1] - self.material[0],
                             self.material[1] - self.material[0])
        return dal_deps * deps_drho


def reference_fixture(data_dir):
    """The 22x22x10 fixture of python_tests/test_DDAModel.py:8-104 as constructor
    arguments (with the wrapper's SiCi tables)."""
    gc = np.loadtxt(os.path.join(data_dir, "geometry.txt"), dtype=np.int64)
    nx, ny, nz, nt = (int(v) for v in gc[:4])
    diel = np.loadtxt(os.path.join(data_dir, "dielectrics.txt"))
    si, ci = sici_tables()
    mats = [1.01 + 0j, 5.96282 + 3.80423e-7j]
    return dict(
        betaMin=0.0, betaMax=50.0, ita=0.5, betaType="piecewise", filterIterations=[100],
        filterRadii=[2.0], useFilter=False, symmetryType="4fold", symmetryAxis=[10.5, 10.5],
        isPeriodic=True, objectiveName="IntegratedE",
        objPara=[2.0, 0.0, 21.0, 0.0, 21.0, 0.0, 9.0, 0.95, 50.0], geometry=gc[4:],
        inputDielectrics=diel, num_x=nx, num_y=ny, num_z=nz, num_total=nt, n_K=[0, 0, 1],
        E0=1.0, n_E0=[1, 0, 0], lam=542.0, material=mats, nback=math.sqrt(1.01), MAXm=50,
        MAXn=50, Lm=22, Ln=22, matrixAMethodName="FCD", d=15.0, sineIntegralValues=si,
        cosineIntegralValues=ci, integralDelta=0.1, verbose=False)


# ----------------------------------------------------------------------------
# the reference's legacy design filter (in-plane cone filter + exponential
# projection), reachable in the reference only from C++ (DDAModel::UpdateStr,
# gradients_filtered)
# ----------------------------------------------------------------------------

def beta_schedule(beta_type, it, max_it, beta_min, beta_max):
    """FilterOption::update_beta (src/FilterOption.cpp:23-45) with exp_update,
    piecewise_update and linear_update (src/Tools.cpp:473-516)."""
    x, xm = float(it), float(max_it)
    if beta_type == "exp":
        if x <= 300:
            return beta_min + (beta_max - beta_min) * (math.pow(100.0, x / xm) - 1) / (100 - 1)
        return 0.5
    if beta_type == "piecewise":
        if x <= 0.5 * xm:
            return beta_min
        if 0.5 * xm < x <= 0.7 * xm:
            return beta_min + (beta_max - beta_min) / 5
        if 0.7 * xm < x <= 0.8 * xm:
            return beta_min + (beta_max - beta_min) / 2.5
        return beta_max
    if beta_type == "linear":
        return beta_min + (beta_max - beta_min) * x / xm
    raise RuntimeError("Unknown internal error")  # `throw 1` (src/FilterOption.cpp:41-44)


def smooth_density(x, beta, ita):
    """FilterOption::SmoothDensity (src/FilterOption.cpp:48-62)."""
    if 0.0 <= x <= ita:
        return ita * (math.exp(-beta * (1 - x / ita)) - (1 - x / ita) * math.exp(-beta))
    if ita < x <= 1.0:
        return (1 - ita) * (1 - math.exp(-beta * (x - ita) / (1 - ita)) + (x - ita) / (1 - ita) * math.exp(-beta)) + ita
    raise RuntimeError("Unknown internal error")


def smooth_density_d(x, beta, ita):
    """PtoFderivative (src/DDAModel.cpp:340-352), as the reference writes it."""
    if 0.0 <= x <= ita:
        return beta * math.exp(-beta * (1 - x / ita)) + math.exp(-beta)
    if ita < x <= 1.0:
        return beta * math.exp(-beta * (x - ita) / (1 - ita)) + math.exp(-beta)
    raise RuntimeError("Unknown internal error")


class LegacyFilter:
    """The in-plane cone filter of DDAModel::assignFreeWeightsForFilter
    (src/DDAModel.cpp:580-712): for every free parameter i (at the first
    dipole of its list, (xo, yo, zo)) and every parameter j, one weight
    rfilter - dist per dipole of j in the plane z = zo within the circle
    dist^2 <= rfilter^2 - 0.01 (circlerange / calweight, :66-77), with the
    eight in-plane periodic images (+-Lm, +-Ln grid units) when periodic, in
    the reference's order (own cell, (0,-1), (-1,-1), (-1,0), (-1,1), (0,1),
    (1,1), (1,0), (1,-1)).  Quadratic in the number of parameters, as the
    reference is: small cases only."""

    def __init__(self, geometry, p2g, nfpara, rfilter, periodic, Lm, Ln, beta_min, beta_max, ita, beta_type,
                 parameters):
        g = np.asarray(geometry).reshape(-1, 3)
        Lm, Ln = int(Lm), int(Ln)
        shifts = [(0, 0)] + ([(0, -Ln), (-Lm, -Ln), (-Lm, 0), (-Lm, Ln), (0, Ln), (Lm, Ln), (Lm, 0), (Lm, -Ln)]
                             if periodic else [])
        r2 = rfilter * rfilter - 0.01
        self.weights = []
        for i in range(nfpara):
            xo, yo, zo = (int(v) for v in g[p2g[i][0]])
            lst = []
            for j in range(nfpara):
                for pos in p2g[j]:
                    xr, yr, zr = (int(v) for v in g[pos])
                    if zr != zo:
                        continue
                    for sx, sy in shifts:
                        x, y = xr + sx, yr + sy
                        d2 = float(x - xo) * float(x - xo) + float(y - yo) * float(y - yo)
                        if d2 <= r2:
                            lst.append((rfilter - math.sqrt(d2), j))
            self.weights.append(lst)
        self.nfpara = nfpara
        self.beta_min, self.beta_max, self.ita, self.beta_type = beta_min, beta_max, ita, beta_type
        self.beta = beta_min
        self.origin = np.array(parameters, dtype=np.float64)
        self.filtered = np.array(parameters, dtype=np.float64)

    def update(self, step, it, max_it):
        """DDAModel::UpdateStr, filter branch (src/DDAModel.cpp:785-817): the
        raw parameters take the step (clamped to [0, 1]), are filtered and
        projected; returns the new (physical) parameters."""
        self.beta = beta_schedule(self.beta_type, it, max_it, self.beta_min, self.beta_max)
        self.origin = np.clip(self.origin + np.asarray(step, dtype=np.float64), 0.0, 1.0)
        phys = np.zeros(self.nfpara)
        for i in range(self.nfpara):
            num = 0.0
            den = 0.0
            for w, j in self.weights[i]:
                num += w * self.origin[j]
                den += w
            self.filtered[i] = num / den
            phys[i] = smooth_density(self.filtered[i], self.beta, self.ita)
        return phys

    def gradients(self, grad, it, max_it):
        """DDAModel::gradients_filtered (src/DDAModel.cpp:354-396): each
        parameter's gradient times the sum of its normalised weights over the
        filters it enters, times the projection derivative at its filtered
        value."""
        self.beta = beta_schedule(self.beta_type, it, max_it, self.beta_min, self.beta_max)
        res = np.zeros(self.nfpara)
        for i in range(self.nfpara):
            sw = 0.0
            for w, j in self.weights[i]:
                sw += w
            for w, j in self.weights[i]:
                res[j] += w / sw
        for i in range(self.nfpara):
            res[i] = res[i] * smooth_density_d(self.filtered[i], self.beta, self.ita) * grad[i]
        return res
