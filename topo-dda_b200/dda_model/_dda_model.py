"""`DDAModel`: the reference's pybind11 class, re-exposed over the C ABI.

Same constructor argument names and order as
python_bindings/PythonBindings.cpp:19-59 and the same seven methods
(:61-69).  Inputs are copied into the model; outputs are fresh numpy arrays,
as pybind11 returned copies of the Eigen vectors.  Invalid input raises
RuntimeError (the reference's `throw 1` surfaced as RuntimeError too).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

_PRECISIONS = {"complex128": 0, "c128": 0, "mixed": 1}


def _f64(a, n=None, name="array"):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel())
    if n is not None and a.size != n:
        raise RuntimeError(f"{name} must have {n} entries, got {a.size}")
    return a


def _c128(a, n=None, name="array"):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.complex128).ravel())
    if n is not None and a.size != n:
        raise RuntimeError(f"{name} must have {n} entries, got {a.size}")
    return a


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class DDAModel:
    """Discrete-dipole model of one structure at one wavelength.

    Positional/keyword arguments follow the reference constructor exactly;
    ``precision`` ("complex128" or "mixed") is an extra keyword-only option.
    """

    def __init__(self, betaMin, betaMax, ita, betaType, filterIterations, filterRadii, useFilter,
                 symmetryType, symmetryAxis, isPeriodic, objectiveName, objPara, geometry,
                 inputDielectrics, num_x, num_y, num_z, num_total, n_K, E0, n_E0, lam, material,
                 nback, MAXm, MAXn, Lm, Ln, matrixAMethodName, d, sineIntegralValues,
                 cosineIntegralValues, integralDelta, verbose, *, precision="complex128"):
        lib = _lib.load()
        self._handle = None
        N = int(num_total)
        geo = np.ascontiguousarray(np.asarray(geometry).ravel().astype(np.int32))
        if geo.size != 3 * N:
            raise RuntimeError("geometry must hold 3*num_total integers")
        diel = _f64(inputDielectrics, 3 * N, "inputDielectrics")
        obj = _f64(objPara)
        mat = np.asarray(material, dtype=np.complex128).ravel()
        if mat.size != 2:
            raise RuntimeError("material must hold two complex permittivities")
        si = _f64(sineIntegralValues)
        ci = _f64(cosineIntegralValues)
        if si.size != ci.size:
            raise RuntimeError("sine and cosine integral tables differ in length")
        if precision not in _PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(_PRECISIONS)}")
        p = _lib.Params()
        p.beta_min, p.beta_max, p.ita = float(betaMin), float(betaMax), float(ita)
        p.beta_type = str(betaType).encode()
        p.use_filter = 1 if useFilter else 0
        p.symmetry_type = str(symmetryType).encode()
        ax = list(symmetryAxis) + [0.0, 0.0]
        p.symmetry_axis[0], p.symmetry_axis[1] = float(ax[0]), float(ax[1])
        p.is_periodic = 1 if isPeriodic else 0
        p.objective_name = str(objectiveName).encode()
        p.obj_para = _dp(obj)
        p.n_obj_para = obj.size
        p.num_x, p.num_y, p.num_z, p.num_total = int(num_x), int(num_y), int(num_z), N
        for c in range(3):
            p.n_K[c] = float(n_K[c])
            p.n_E0[c] = float(n_E0[c])
        p.E0 = float(E0)
        p.lam = float(lam)
        p.material[0], p.material[1] = mat[0].real, mat[0].imag
        p.material[2], p.material[3] = mat[1].real, mat[1].imag
        p.nback = float(nback)
        p.MAXm, p.MAXn = int(MAXm), int(MAXn)
        p.Lm, p.Ln = float(Lm), float(Ln)
        p.matrix_method = str(matrixAMethodName).encode()
        p.d = float(d)
        p.integral_delta = float(integralDelta)
        p.verbose = 1 if verbose else 0
        p.precision = _PRECISIONS[precision]
        fit = np.ascontiguousarray(np.asarray(filterIterations, dtype=np.int32).ravel())
        frad = _f64(filterRadii)
        if fit.size != frad.size:
            raise RuntimeError("filterIterations and filterRadii differ in length")
        p.filter_iterations = fit.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        p.filter_radii = _dp(frad)
        p.n_filters = int(frad.size)
        h = ctypes.c_void_p()
        _lib.check(lib.tdda_model_create(ctypes.byref(p), geo.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                         _dp(diel), _dp(si), _dp(ci), si.size, ctypes.byref(h)))
        self._handle = h
        self._lib = lib
        info = _lib.ModelInfo()
        _lib.check(lib.tdda_model_get_info(h, ctypes.byref(info)))
        self._info = info
        self.N = N
        self.NFpara = info.NFpara
        self.last_solve = None

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            self._lib.tdda_model_destroy(h)
            self._handle = None

    # --- the reference's seven methods -----------------------------------------
    def solveElectricField(self, originPolarization, BGS_MAX_ITER, BGS_MAX_ERROR):
        """src/DDAModel.cpp:874-885 (originPolarization=None: zero initial guess)."""
        if originPolarization is None:
            ptr = None
        else:
            p0 = _c128(originPolarization, 3 * self.N, "originPolarization")
            ptr = _dp(p0.view(np.float64))
        info = _lib.SolveInfo()
        _lib.check(self._lib.tdda_solve_electric_field(self._handle, ptr, int(BGS_MAX_ITER), float(BGS_MAX_ERROR),
                                                       ctypes.byref(info)))
        self.last_solve = info.as_dict()
        return None

    def solveElectricFieldWarm(self, BGS_MAX_ITER, BGS_MAX_ERROR):
        """solveElectricField starting from the model's current polarisation
        (already on the device: no host copy of the initial guess)."""
        info = _lib.SolveInfo()
        _lib.check(self._lib.tdda_solve_electric_field_warm(self._handle, int(BGS_MAX_ITER), float(BGS_MAX_ERROR),
                                                            ctypes.byref(info)))
        self.last_solve = info.as_dict()

    def paramsToDensitiesDevice(self, params_ptr, rho_ptr, stream=None):
        """rho[i] = params[parameterMap()[i]] on device arrays (NFpara -> N doubles)."""
        _lib.check(self._lib.tdda_params_to_densities_device(self._handle, params_ptr, rho_ptr, stream))

    def densitiesToParamsDevice(self, grad_ptr, out_ptr, stream=None):
        """Per-parameter sums of a per-dipole gradient on device arrays (N -> NFpara)."""
        _lib.check(self._lib.tdda_densities_to_params_device(self._handle, grad_ptr, out_ptr, stream))

    def calculateObjective(self):
        """src/DDAModel.cpp:870-872 (IntegratedE)."""
        out = ctypes.c_double()
        _lib.check(self._lib.tdda_calculate_objective(self._handle, ctypes.byref(out)))
        return out.value

    def calculateGradients(self, epsilon_partial, originalObjValue, MAX_ITERATION, MAX_ERROR):
        """src/DDAModel.cpp:398-469."""
        g = np.zeros(self.NFpara)
        _lib.check(self._lib.tdda_calculate_gradients(self._handle, float(epsilon_partial),
                                                      float(originalObjValue), int(MAX_ITERATION),
                                                      float(MAX_ERROR), _dp(g), g.size))
        return g

    def setParameters(self, values):
        """src/DDAModel.cpp:747-772."""
        v = _f64(values, self.NFpara, "parameters")
        _lib.check(self._lib.tdda_set_parameters(self._handle, _dp(v), v.size))

    def getParameters(self):
        g = np.zeros(self.NFpara)
        _lib.check(self._lib.tdda_get_parameters(self._handle, _dp(g), g.size))
        return g

    def lattice_offsets_device(self, lo, nb, out_ptr, stream=None):
        """Lattice sums at the offsets lo + [0, nb) into the device array out_ptr
        (complex128 [nb0][nb1][nb2][6]); measurement support."""
        lo_a = (ctypes.c_int32 * 3)(*[int(v) for v in lo])
        nb_a = (ctypes.c_int32 * 3)(*[int(v) for v in nb])
        _lib.check(self._lib.tdda_lattice_offsets_device(self._handle, lo_a, nb_a, out_ptr, stream))

    def parameterMap(self):
        """Free parameter of every dipole (src/DDAModel.cpp:163-247), int32[N]."""
        out = np.zeros(self.N, dtype=np.int32)
        _lib.check(self._lib.tdda_get_parameter_map(self._handle, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                                    out.size))
        return out

    def getDielectrics(self):
        g = np.zeros(3 * self.N)
        _lib.check(self._lib.tdda_get_dielectrics(self._handle, _dp(g), g.size))
        return g

    def getElectricField(self):
        g = np.zeros(3 * self.N, dtype=np.complex128)
        _lib.check(self._lib.tdda_get_electric_field(self._handle, _dp(g.view(np.float64)), g.size))
        return g

    # --- additions ---------------------------------------------------------------
    def getPolarization(self):
        g = np.zeros(3 * self.N, dtype=np.complex128)
        _lib.check(self._lib.tdda_get_polarization(self._handle, _dp(g.view(np.float64)), g.size))
        return g

    def matvec(self, x, with_al=True, precision="complex128"):
        """A.x (+ (1/alpha) o x): AProductCore::Aproduct / DDAModel::Aproductwithalb.
        precision="complex64" applies the single-precision operator of a mixed model."""
        xx = _c128(x, 3 * self.N, "x")
        y = np.zeros_like(xx)
        fn = self._lib.tdda_matvec_c64 if precision == "complex64" else self._lib.tdda_matvec
        _lib.check(fn(self._handle, _dp(xx.view(np.float64)), _dp(y.view(np.float64)), 1 if with_al else 0))
        return y

    def solve_batch_device(self, B_ptr, X_ptr, nrhs, x0_zero=True, max_iter=100000, tol=1e-8,
                           stream=None):
        """Batched solve on device buffers (complex128 [nrhs][3N]); returns per-RHS info dicts."""
        infos = (_lib.SolveInfo * int(nrhs))()
        _lib.check(self._lib.tdda_solve_batch_device(self._handle, B_ptr, X_ptr, int(nrhs),
                                                     1 if x0_zero else 0, int(max_iter), float(tol),
                                                     stream, infos))
        return [infos[k].as_dict() for k in range(int(nrhs))]

    def matvec_device(self, x_ptr, y_ptr, nrhs=1, with_al=True, stream=None):
        _lib.check(self._lib.tdda_matvec_device(self._handle, x_ptr, y_ptr, int(nrhs),
                                                1 if with_al else 0, stream))

    def setDensities(self, rho):
        """Per-dipole densities (3-D design; extension of setParameters)."""
        v = _f64(rho, self.N, "densities")
        _lib.check(self._lib.tdda_set_densities(self._handle, _dp(v), v.size))

    def setDensitiesDevice(self, rho_ptr, stream=None):
        """Per-dipole densities from a device array (double[N], dipole order),
        ordered after `stream`."""
        _lib.check(self._lib.tdda_set_densities_device(self._handle, rho_ptr, stream))

    def gradientDensitiesDevice(self, grad_ptr, max_iter=100000, tol=1e-10, stream=None):
        """gradientDensities into a device array (double[N], dipole order), ready on `stream`."""
        info = _lib.SolveInfo()
        _lib.check(self._lib.tdda_gradient_densities_device(self._handle, int(max_iter), float(tol), grad_ptr,
                                                            stream, ctypes.byref(info)))
        self.last_adjoint = info.as_dict()

    def patchGradientDevice(self, grad_ptr, max_iter=100000, tol=1e-10, stream=None):
        """patchGradient into a device array (double[N], dipole order), ready on `stream`."""
        info = _lib.SolveInfo()
        _lib.check(self._lib.tdda_patch_gradient_device(self._handle, int(max_iter), float(tol), grad_ptr,
                                                        stream, ctypes.byref(info)))
        self.last_adjoint = info.as_dict()

    def gradientDensities(self, max_iter=100000, tol=1e-10):
        """Exact adjoint gradient of the objective w.r.t. every dipole density
        (uses the polarisation of the last solve)."""
        g = np.zeros(self.N)
        info = _lib.SolveInfo()
        _lib.check(self._lib.tdda_gradient_densities(self._handle, int(max_iter), float(tol), _dp(g), g.size,
                                                     ctypes.byref(info)))
        self.last_adjoint = info.as_dict()
        return g

    def setObservationPoints(self, xyz):
        """Observation points (grid units, shape [nobs, 3]) for the patch objective."""
        a = np.ascontiguousarray(np.asarray(xyz).reshape(-1, 3).astype(np.int32))
        _lib.check(self._lib.tdda_set_observation_points(self._handle, a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                                          a.shape[0]))
        self.nobs = a.shape[0]

    def observationField(self):
        e = np.zeros(3 * self.nobs, dtype=np.complex128)
        _lib.check(self._lib.tdda_observation_field(self._handle, _dp(e.view(np.float64)), e.size))
        return e

    def patchObjective(self):
        """mean over observation points of |E|^2 (uses the last solve)."""
        out = ctypes.c_double()
        _lib.check(self._lib.tdda_patch_objective(self._handle, ctypes.byref(out)))
        return out.value

    def patchGradient(self, max_iter=100000, tol=1e-10):
        """Exact adjoint gradient of patchObjective w.r.t. every dipole density."""
        g = np.zeros(self.N)
        info = _lib.SolveInfo()
        _lib.check(self._lib.tdda_patch_gradient(self._handle, int(max_iter), float(tol), _dp(g), g.size,
                                                 ctypes.byref(info)))
        self.last_adjoint = info.as_dict()
        return g

    def profile_matvec(self, precision="complex128", nrhs=1, iters=20):
        """Device time of one operator application (ms) and of each of its 3 passes."""
        tot = ctypes.c_double()
        passes = (ctypes.c_double * 3)()
        _lib.check(self._lib.tdda_profile_matvec(self._handle, 0 if precision in ("complex128", "c128") else 1,
                                                 int(nrhs), int(iters), ctypes.byref(tot), passes))
        return tot.value, [passes[0], passes[1], passes[2]]

    def profile_gram_schmidt(self, precision="mixed", nv=25, iters=20):
        """Device time (ms) of one GMRES projection pass and of one update pass
        against nv basis vectors of this model's size (scratch basis)."""
        ms = (ctypes.c_double * 2)()
        _lib.check(self._lib.tdda_profile_gram_schmidt(self._handle, 0 if precision in ("complex128", "c128") else 1,
                                                       int(nv), int(iters), ms))
        return ms[0], ms[1]

    def setPrecision(self, precision):
        """Switch later solves between "complex128" and "mixed" (mixed models only)."""
        _lib.check(self._lib.tdda_set_precision(self._handle, _PRECISIONS[precision]))

    def matvec_device_noalloc(self, x_ptr, y_ptr, with_al=True, stream=None):
        """A.x (+ (1/alpha) o x) on device buffers without any device allocation:
        for callers that cannot have memory allocated during the call (fixed
        memory budgets, latency-bound host threads).  Works in a fixed 32 MiB
        scratch area of the library; larger grids raise.  Calls that overlap on
        the GPU share that scratch and must be serialised by the caller."""
        _lib.check(self._lib.tdda_matvec_device_noalloc(self._handle, x_ptr, y_ptr, 1 if with_al else 0, stream))

    def setPreconditioner(self, kind):
        """"none" (the reference's plain BiCGSTAB) or "jacobi" (diagonally scaled
        solves inside a complex128 refinement on the true residual)."""
        k = {"none": 0, "jacobi": 1}[kind]
        _lib.check(self._lib.tdda_set_preconditioner(self._handle, k))

    def setTimeLimit(self, seconds):
        """Device-side time limit of later BiCGSTAB solves (0: none): running
        right-hand sides end with status "timeout"."""
        _lib.check(self._lib.tdda_set_time_limit(self._handle, float(seconds)))

    # --- the reference's legacy filter (models created with useFilter=True) ---
    def updateStructure(self, step, current_it, max_it):
        """DDAModel::UpdateStr (src/DDAModel.cpp:774-838) + the polarisability
        update: raw parameters += step (clamped), in-plane cone filter,
        exponential projection at the scheduled beta."""
        v = _f64(step, self.NFpara, "step")
        _lib.check(self._lib.tdda_filter_update(self._handle, _dp(v), v.size, int(current_it), int(max_it)))

    def filterGradients(self, gradients, current_it, max_it):
        """DDAModel::gradients_filtered (src/DDAModel.cpp:354-396)."""
        g = _f64(gradients, self.NFpara, "gradients")
        out = np.zeros(self.NFpara)
        _lib.check(self._lib.tdda_filter_gradients(self._handle, _dp(g), g.size, int(current_it), int(max_it),
                                                   _dp(out)))
        return out

    def filterState(self):
        """(raw parameters, filtered parameters, beta) of the legacy filter."""
        raw = np.zeros(self.NFpara)
        filt = np.zeros(self.NFpara)
        beta = ctypes.c_double()
        _lib.check(self._lib.tdda_filter_state(self._handle, _dp(raw), _dp(filt), raw.size, ctypes.byref(beta)))
        return raw, filt, beta.value

    def setSolver(self, kind, degree=24, restart=40, deflate=0):
        """"bicgstab" (the reference's solver) or "pgmres": restarted GMRES on the
        Jacobi-scaled operator times a polynomial of `degree` in it, cycles of
        `restart` steps keeping `deflate` harmonic Ritz vectors across restarts,
        inside complex128 refinement (for structures that fill their periodic
        cell, where BiCGSTAB stalls).  "gmres-dr-recycle": "pgmres" whose inner
        solve of each refinement step after the first starts from the deflation
        space the previous inner solve ended with."""
        k = {"bicgstab": 0, "pgmres": 1, "gmres-dr-recycle": 2}[kind]
        _lib.check(self._lib.tdda_set_solver(self._handle, k, int(degree), int(restart), int(deflate)))

    @staticmethod
    def kernel_launches():
        return int(_lib.load().tdda_kernel_launches())

    @property
    def info(self):
        i = self._info
        return {"N": i.N, "NFpara": i.NFpara, "grid": (i.nx, i.ny, i.nz), "fft": (i.Lx, i.Ly, i.Lz),
                "K": i.K, "material": [complex(i.material[0], i.material[1]),
                                       complex(i.material[2], i.material[3])],
                "lattice_ms": i.lattice_ms, "tensor_fft_ms": i.tensor_fft_ms}
