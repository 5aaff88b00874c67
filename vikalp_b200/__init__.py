"""ctypes bindings of the B200 PDHG library (include/vikalp_b200.h).

The solver itself is ``libvikalp_b200.so`` (hand-written sm_100a CUDA behind a
C ABI); this module only marshals numpy arrays across that ABI. There is no
CPU fallback: every call goes to the CUDA library, and importing this module
fails loudly when the library has not been built (``python -m vikalp_b200.build``).
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libvikalp_b200.so")

VK_OK = 0
VK_ERR_INVALID = -1
VK_ERR_UNSUPPORTED = -2
VK_ERR_CUDA = -3
VK_ERR_INTERNAL = -4

ALGO_REFERENCE = 0
ALGO_HALPERN = 1
PREC_FP64 = 0
PREC_MIXED = 1
SPMV_FAST = 0
SPMV_SEQUENTIAL = 1

STATUS = {0: "NotSolved", 1: "Optimal", 2: "LocallyOptimal", 3: "Feasible", 4: "Infeasible",
          5: "Unbounded", 6: "IterationLimit", 7: "NodeLimit", 8: "TimeLimit",
          9: "NumericalFailure", 10: "UnsupportedModel", 11: "InvalidModel"}

_i64p = C.POINTER(C.c_int64)
_f64p = C.POINTER(C.c_double)


FAST_VARIANTS = 18  # kernel variants of the sparse pass (vk_spmat_set_variant)


class VkError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code
        self.msg = msg


class Csr(C.Structure):
    _fields_ = [("rows", C.c_int64), ("cols", C.c_int64), ("row_offsets", _i64p),
                ("col_indices", _i64p), ("values", _f64p)]


class Problem(C.Structure):
    _fields_ = [("A", Csr), ("Q", Csr), ("c", _f64p), ("objective_offset", C.c_double),
                ("var_lower", _f64p), ("var_upper", _f64p), ("row_lower", _f64p), ("row_upper", _f64p)]


class Options(C.Structure):
    _fields_ = [("iteration_limit", C.c_int64), ("time_limit_seconds", C.c_double),
                ("primal_tolerance", C.c_double), ("dual_tolerance", C.c_double),
                ("continuous_method", C.c_int32), ("algorithm", C.c_int32), ("precision", C.c_int32),
                ("spmv_order", C.c_int32), ("check_every", C.c_int32), ("relative_tolerance", C.c_double),
                ("device", C.c_int32), ("verbose", C.c_int32)]


class Result(C.Structure):
    _fields_ = [("x", _f64p), ("y", _f64p), ("row_lower_dual", _f64p), ("row_upper_dual", _f64p),
                ("var_lower_dual", _f64p), ("var_upper_dual", _f64p), ("status", C.c_int32),
                ("iterations", C.c_int64), ("restarts", C.c_int64), ("objective", C.c_double),
                ("primal_residual", C.c_double), ("stationarity_residual", C.c_double),
                ("complementarity_residual", C.c_double), ("rel_primal", C.c_double),
                ("rel_dual", C.c_double), ("rel_gap", C.c_double), ("last_metric", C.c_double),
                ("solve_seconds", C.c_double), ("iterate_seconds", C.c_double),
                ("fp32_iterations", C.c_int64), ("kernel_launches", C.c_int64), ("message", C.c_char * 256)]


class PassProfile(C.Structure):
    _fields_ = [("count", C.c_int32), ("name", (C.c_char * 48) * 8), ("ms_per_launch", C.c_double * 8),
                ("launches", C.c_int64 * 8), ("bytes_per_launch", C.c_double * 8)]


class AdjointOptions(C.Structure):
    _fields_ = [("active_tolerance", C.c_double), ("solve_tolerance", C.c_double), ("iteration_limit", C.c_int64),
                ("device", C.c_int32)]


class AdjointInfo(C.Structure):
    _fields_ = [("rows_active", C.c_int64), ("cols_free", C.c_int64), ("iterations", C.c_int64),
                ("status", C.c_int32), ("residual", C.c_double), ("normal_residual", C.c_double)]


# Every symbol include/vikalp_b200.h declares, with its ctypes signature.
_SIGNATURES = {
    "vk_default_options": (None, [C.POINTER(Options)]),
    "vk_last_error": (C.c_char_p, []),
    "vk_version": (C.c_char_p, []),
    "vk_pdhg_create": (C.c_int, [C.POINTER(Problem), C.POINTER(Options), C.POINTER(C.c_void_p)]),
    "vk_pdhg_solve": (C.c_int, [C.c_void_p, _f64p, _f64p, _f64p, C.POINTER(Result)]),
    "vk_pdhg_set_options": (C.c_int, [C.c_void_p, C.POINTER(Options)]),
    "vk_pdhg_destroy": (None, [C.c_void_p]),
    "vk_pdhg_profile": (C.c_int, [C.c_void_p, C.c_int64, C.POINTER(PassProfile)]),
    "vk_csr_transpose": (C.c_int, [C.POINTER(Csr), _i64p, _i64p, _f64p, _i64p]),
    "vk_spmv": (C.c_int, [C.POINTER(Csr), C.c_double, _f64p, C.c_double, _f64p, C.c_int, C.c_int]),
    "vk_spmat_create": (C.c_int, [C.POINTER(Csr), C.c_int32, C.POINTER(C.c_void_p)]),
    "vk_spmat_apply_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "vk_spmat_bytes": (C.c_int64, [C.c_void_p, C.c_int]),
    "vk_spmat_variant": (C.c_int, [C.c_void_p, C.c_int]),
    "vk_spmat_set_variant": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "vk_spmat_destroy": (None, [C.c_void_p]),
    "vk_spmat_set_values": (C.c_int, [C.c_void_p, _f64p, C.c_int64]),
    "vk_spmat_multiply": (C.c_int, [C.c_void_p, C.c_double, C.c_void_p, C.c_double, C.c_void_p, C.c_int, C.c_int]),
    "vk_device_select": (C.c_int, [C.c_int32]),
    "vk_device_synchronize": (C.c_int, []),
    "vk_dvec_create": (C.c_int, [C.c_int64, C.POINTER(C.c_void_p)]),
    "vk_dvec_destroy": (None, [C.c_void_p]),
    "vk_dvec_size": (C.c_int64, [C.c_void_p]),
    "vk_dvec_upload": (C.c_int, [C.c_void_p, _f64p, C.c_int64]),
    "vk_dvec_download": (C.c_int, [C.c_void_p, _f64p, C.c_int64]),
    "vk_dvec_fill": (C.c_int, [C.c_void_p, C.c_double]),
    "vk_dvec_copy": (C.c_int, [C.c_void_p, C.c_void_p]),
    "vk_dvec_axpby": (C.c_int, [C.c_double, C.c_void_p, C.c_double, C.c_void_p]),
    "vk_dvec_dot": (C.c_int, [C.c_void_p, C.c_void_p, _f64p]),
    "vk_dvec_norm_inf": (C.c_int, [C.c_void_p, _f64p]),
    "vk_dvec_project_box": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "vk_vec_dot_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]),
    "vk_vec_norm_inf_device": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]),
    "vk_vec_dot_device_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]),
    "vk_batch_solve": (C.c_int, [C.POINTER(Problem), C.c_int32, C.POINTER(Options), C.POINTER(Result)]),
    "vk_batch_solve_shared": (C.c_int, [C.POINTER(Problem), C.c_int32, _f64p, _f64p, _f64p, C.POINTER(Options),
                                        C.POINTER(Result)]),
    "vk_default_adjoint_options": (None, [C.POINTER(AdjointOptions)]),
    "vk_lp_adjoint": (C.c_int, [C.POINTER(Problem), C.c_int32, _f64p, _f64p, _f64p, C.c_double,
                                C.POINTER(AdjointOptions), _f64p, _f64p, _f64p, C.POINTER(AdjointInfo)]),
    "vk_diag_bounded_wait": (C.c_int, [C.c_int32]),
    "vk_batch_solve_together": (C.c_int, [C.POINTER(Problem), C.c_int32, _f64p, _f64p, _f64p, C.POINTER(Problem),
                                          C.c_int32, C.POINTER(Options), C.POINTER(Result), C.POINTER(Result)]),
}

# include/vikalp_mps.h: the MPS ingest path, exported by the C++ host layer (libvikalp.so).
HOST_LIB_PATH = os.path.join(HERE, "libvikalp.so")
_MPS_SIGNATURES = {
    "vk_mps_read": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "vk_mps_problem": (C.c_int, [C.c_void_p, C.POINTER(Problem), C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                 C.POINTER(C.c_int64)]),
    "vk_mps_name": (C.c_char_p, [C.c_void_p]),
    "vk_mps_binary_count": (C.c_int32, [C.c_void_p]),
    "vk_mps_error_count": (C.c_int32, [C.c_void_p]),
    "vk_mps_error": (C.c_char_p, [C.c_void_p, C.c_int32, C.POINTER(C.c_int64)]),
    "vk_mps_free": (None, [C.c_void_p]),
}

_lib = None
_host = None


def host_lib():
    """Loads libvikalp.so, the C++ host layer (raises if it has not been built)."""
    global _host
    if _host is None:
        lib()  # the CUDA library it links against
        if not os.path.exists(HOST_LIB_PATH):
            raise ImportError(f"{HOST_LIB_PATH} is missing: build it with `python -m vikalp_b200.build`")
        L = C.CDLL(HOST_LIB_PATH)
        for name, (res, args) in _MPS_SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _host = L
    return _host


class MpsModel:
    """A model read from an MPS file by vikalp::MpsReader (vk_mps_read): the
    arrays of a synthetic.Instance-like object, plus the reader's errors."""

    def __init__(self, path: str):
        L = host_lib()
        h = C.c_void_p()
        rc = L.vk_mps_read(os.fsencode(path), C.byref(h))
        if rc == VK_ERR_INTERNAL or not h:
            raise VkError(rc, "MPS reader failed")
        try:
            self.ok = rc == VK_OK
            self.errors = []
            for i in range(L.vk_mps_error_count(h)):
                ln = C.c_int64()
                msg = L.vk_mps_error(h, i, C.byref(ln)).decode()
                self.errors.append((int(ln.value), msg))
            self.name = L.vk_mps_name(h).decode()
            self.binaries = int(L.vk_mps_binary_count(h))
            p = Problem()
            m, n, nnz = C.c_int64(), C.c_int64(), C.c_int64()
            L.vk_mps_problem(h, C.byref(p), C.byref(m), C.byref(n), C.byref(nnz))
            self.m, self.n = int(m.value), int(n.value)
            k = int(nnz.value)
            cp = lambda ptr, cnt, dt: np.ctypeslib.as_array(ptr, shape=(cnt,)).astype(dt, copy=True) if cnt > 0 else np.zeros(0, dt)  # noqa: E731
            self.row_offsets = cp(p.A.row_offsets, self.m + 1, np.int64)
            self.col_idx = cp(p.A.col_indices, k, np.int64)
            self.values = cp(p.A.values, k, np.float64)
            self.c = cp(p.c, self.n, np.float64)
            self.var_lower = cp(p.var_lower, self.n, np.float64)
            self.var_upper = cp(p.var_upper, self.n, np.float64)
            self.row_lower = cp(p.row_lower, self.m, np.float64)
            self.row_upper = cp(p.row_upper, self.m, np.float64)
            self.objective_offset = float(p.objective_offset)
            self.q_row_offsets = self.q_col_idx = self.q_values = None
        finally:
            L.vk_mps_free(h)

    @property
    def nnz(self):
        return int(self.col_idx.shape[0])

    @property
    def q_nnz(self):
        return 0


def read_mps(path: str) -> MpsModel:
    return MpsModel(path)


def lib():
    """Loads libvikalp_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m vikalp_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    return lib().vk_last_error().decode()


def _check(rc: int):
    if rc != VK_OK:
        raise VkError(rc, last_error())


def _p(a, typ=_f64p):
    return None if a is None else a.ctypes.data_as(typ)


class _Keep(list):
    def f(self, a):
        if a is None:
            return None
        a = np.ascontiguousarray(a, dtype=np.float64)
        self.append(a)
        return _p(a)

    def i(self, a):
        if a is None:
            return None
        a = np.ascontiguousarray(a, dtype=np.int64)
        self.append(a)
        return _p(a, _i64p)


def _csr(keep: _Keep, rows, cols, ro, ci, v) -> Csr:
    return Csr(rows, cols, keep.i(ro), keep.i(ci), keep.f(v))


def options(**kw) -> Options:
    o = Options()
    lib().vk_default_options(C.byref(o))
    names = {"algorithm": {"reference": ALGO_REFERENCE, "halpern": ALGO_HALPERN},
             "precision": {"fp64": PREC_FP64, "mixed": PREC_MIXED},
             "spmv_order": {"fast": SPMV_FAST, "sequential": SPMV_SEQUENTIAL}}
    for k, v in kw.items():
        if k in names and isinstance(v, str):
            v = names[k][v]
        setattr(o, k, v)
    return o


def problem_struct(inst, keep: _Keep) -> Problem:
    """A vk_problem pointing into the arrays of a ``synthetic.Instance``-like object."""
    p = Problem()
    p.A = _csr(keep, inst.m, inst.n, inst.row_offsets, inst.col_idx, inst.values)
    if getattr(inst, "q_col_idx", None) is not None and inst.q_nnz > 0:
        p.Q = _csr(keep, inst.n, inst.n, inst.q_row_offsets, inst.q_col_idx, inst.q_values)
    else:
        p.Q = Csr(0, 0, keep.i(np.zeros(1, np.int64)), None, None)
    p.c = keep.f(inst.c)
    p.objective_offset = float(getattr(inst, "objective_offset", 0.0))
    p.var_lower, p.var_upper = keep.f(inst.var_lower), keep.f(inst.var_upper)
    p.row_lower, p.row_upper = keep.f(inst.row_lower), keep.f(inst.row_upper)
    return p


class Pdhg:
    """A model resident on the GPU (vk_pdhg_create) that can be solved repeatedly."""

    def __init__(self, inst, **opts):
        self._keep = _Keep()
        self.m, self.n = inst.m, inst.n
        self.opts = options(**opts)
        prob = problem_struct(inst, self._keep)
        h = C.c_void_p()
        _check(lib().vk_pdhg_create(C.byref(prob), C.byref(self.opts), C.byref(h)))
        self._h = h
        self._keep.clear()

    def set_options(self, **limits):
        """Per-solve limits / tolerances (vk_pdhg_set_options)."""
        o = Options()
        C.pointer(o)[0] = self.opts
        for k, v in limits.items():
            setattr(o, k, v)
        _check(lib().vk_pdhg_set_options(self._h, C.byref(o)))
        self.opts = o

    def solve(self, warm=None, lower=None, upper=None, duals: bool = True, **limits) -> dict:
        if limits:
            self.set_options(**limits)
        keep = _Keep()
        m, n = self.m, self.n
        out = {"x": np.zeros(n), "y": np.zeros(m)}
        if duals:
            out.update(row_lower_dual=np.zeros(m), row_upper_dual=np.zeros(m),
                       var_lower_dual=np.zeros(n), var_upper_dual=np.zeros(n))
        r = Result()
        for k, a in out.items():
            setattr(r, k, _p(a))
        _check(lib().vk_pdhg_solve(self._h, keep.f(warm), keep.f(lower), keep.f(upper), C.byref(r)))
        out.update(status=STATUS.get(r.status, str(r.status)), iterations=r.iterations, restarts=r.restarts,
                   objective=r.objective, primal_residual=r.primal_residual,
                   stationarity_residual=r.stationarity_residual,
                   complementarity_residual=r.complementarity_residual, rel_primal=r.rel_primal,
                   rel_dual=r.rel_dual, rel_gap=r.rel_gap, last_metric=r.last_metric,
                   solve_seconds=r.solve_seconds, iterate_seconds=r.iterate_seconds,
                   fp32_iterations=r.fp32_iterations, kernel_launches=r.kernel_launches,
                   message=r.message.decode())
        return out

    def profile(self, iterations: int) -> list[dict]:
        """Per-kernel-kind device times of `iterations` eager iterations (vk_pdhg_profile)."""
        pp = PassProfile()
        _check(lib().vk_pdhg_profile(self._h, int(iterations), C.byref(pp)))
        return [{"name": pp.name[q].value.decode(), "ms": pp.ms_per_launch[q], "launches": pp.launches[q],
                 "bytes": pp.bytes_per_launch[q]} for q in range(pp.count)]

    def close(self):
        if getattr(self, "_h", None):
            lib().vk_pdhg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def solve(inst, warm=None, lower=None, upper=None, **opts) -> dict:
    """Create + solve + destroy: the one-shot C-ABI route."""
    with Pdhg(inst, **opts) as h:
        return h.solve(warm, lower, upper)


def _batch_outputs(results, sizes, duals):
    """Host arrays for each batch member (x, y, and the split duals when asked)."""
    outs = []
    for (m, n), r in zip(sizes, results):
        o = {"x": np.zeros(n), "y": np.zeros(m)}
        if duals:
            o.update(row_lower_dual=np.zeros(m), row_upper_dual=np.zeros(m), var_lower_dual=np.zeros(n),
                     var_upper_dual=np.zeros(n))
        for k, a in o.items():
            setattr(r, k, _p(a))
        outs.append(o)
    return outs


def _batch_fields(out, r):
    out.update(status=STATUS.get(r.status, str(r.status)), iterations=r.iterations, restarts=r.restarts,
               objective=r.objective, rel_primal=r.rel_primal, rel_dual=r.rel_dual, rel_gap=r.rel_gap,
               last_metric=r.last_metric, solve_seconds=r.solve_seconds, iterate_seconds=r.iterate_seconds,
               fp32_iterations=r.fp32_iterations, kernel_launches=r.kernel_launches, message=r.message.decode(),
               primal_residual=r.primal_residual, stationarity_residual=r.stationarity_residual,
               complementarity_residual=r.complementarity_residual)


def batch_solve(instances, duals: bool = False, **opts) -> list[dict]:
    """Independent LPs in one batch (vk_batch_solve); one result dict per
    instance. duals=True also asks for the split duals and the reference's
    residuals of every member."""
    opts.setdefault("algorithm", "halpern")
    keep = _Keep()
    probs = (Problem * len(instances))(*[problem_struct(inst, keep) for inst in instances])
    results = (Result * len(instances))()
    outs = _batch_outputs(results, [(i.m, i.n) for i in instances], duals)
    o = options(**opts)
    _check(lib().vk_batch_solve(probs, len(instances), C.byref(o), results))
    for out, r in zip(outs, results):
        _batch_fields(out, r)
    return outs


def batch_solve_shared(inst, count, lower=None, upper=None, warm=None, duals: bool = False, **opts) -> list[dict]:
    """Relaxations of one LP differing in variable bounds (vk_batch_solve_shared).

    lower / upper / warm: None or arrays of shape (count, n). duals=True also
    asks for the split duals and the reference's residuals of every node."""
    opts.setdefault("algorithm", "halpern")
    keep = _Keep()
    p = problem_struct(inst, keep)
    arr = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(count, inst.n)  # noqa: E731
    lower, upper, warm = arr(lower), arr(upper), arr(warm)
    results = (Result * count)()
    outs = _batch_outputs(results, [(inst.m, inst.n)] * count, duals)
    o = options(**opts)
    _check(lib().vk_batch_solve_shared(C.byref(p), count, keep.f(lower), keep.f(upper), keep.f(warm), C.byref(o),
                                       results))
    for out, r in zip(outs, results):
        _batch_fields(out, r)
    return outs


def batch_solve_together(inst, count, instances, lower=None, upper=None, warm=None, duals: bool = False,
                         **opts) -> tuple[list[dict], list[dict]]:
    """A node batch of `inst` (as batch_solve_shared) and the independent LPs
    `instances` (as batch_solve) with both device loops in flight at once
    (vk_batch_solve_together). Returns (node results, instance results)."""
    opts.setdefault("algorithm", "halpern")
    keep = _Keep()
    p = problem_struct(inst, keep)
    arr = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(count, inst.n)  # noqa: E731
    lower, upper, warm = arr(lower), arr(upper), arr(warm)
    probs = (Problem * len(instances))(*[problem_struct(i, keep) for i in instances])
    nres = (Result * count)()
    ires = (Result * len(instances))()
    nouts = _batch_outputs(nres, [(inst.m, inst.n)] * count, duals)
    iouts = _batch_outputs(ires, [(i.m, i.n) for i in instances], duals)
    o = options(**opts)
    _check(lib().vk_batch_solve_together(C.byref(p), count, keep.f(lower), keep.f(upper), keep.f(warm), probs,
                                         len(instances), C.byref(o), nres, ires))
    for out, r in zip(nouts, nres):
        _batch_fields(out, r)
    for out, r in zip(iouts, ires):
        _batch_fields(out, r)
    return nouts, iouts


def lp_adjoint(instances, xs, ys, grads, dL_dobj=0.0, **opts) -> list[dict]:
    """Active-set adjoint of solved LPs (vk_lp_adjoint): per instance the
    gradients {"c", "b", "A"} of L = grad'x* + dL_dobj * c'x* and the solve info."""
    keep = _Keep()
    probs = (Problem * len(instances))(*[problem_struct(inst, keep) for inst in instances])
    cat = lambda arrs: np.ascontiguousarray(np.concatenate([np.asarray(a, np.float64) for a in arrs]))  # noqa: E731
    x, y, g = cat(xs), cat(ys) if sum(i.m for i in instances) else np.zeros(1), cat(grads)
    o = AdjointOptions()
    lib().vk_default_adjoint_options(C.byref(o))
    for k, v in opts.items():
        setattr(o, k, v)
    dc, db = np.zeros(x.size), np.zeros(max(1, sum(i.m for i in instances)))
    nnz = [int(np.asarray(i.row_offsets)[i.m]) for i in instances]
    da = np.zeros(max(1, sum(nnz)))
    info = (AdjointInfo * len(instances))()
    _check(lib().vk_lp_adjoint(probs, len(instances), _p(x), _p(y), _p(g), float(dL_dobj), C.byref(o), _p(dc),
                               _p(db), _p(da), info))
    out, jn, im, kz = [], 0, 0, 0
    for inst, f, nz in zip(instances, info, nnz):
        out.append({"c": dc[jn:jn + inst.n].copy(), "b": db[im:im + inst.m].copy(), "A": da[kz:kz + nz].copy(),
                    "rows_active": f.rows_active, "cols_free": f.cols_free, "iterations": f.iterations,
                    "status": STATUS.get(f.status, str(f.status)), "residual": f.residual,
                    "normal_residual": f.normal_residual})
        jn, im, kz = jn + inst.n, im + inst.m, kz + nz
    return out


def spmv(ro, ci, v, rows, cols, x, y=None, alpha=1.0, beta=0.0, transpose=False, order="fast"):
    keep = _Keep()
    a = _csr(keep, rows, cols, ro, ci, v)
    x = np.ascontiguousarray(x, dtype=np.float64)
    ylen = cols if transpose else rows
    y = np.zeros(ylen) if y is None else np.array(y, dtype=np.float64, copy=True)
    _check(lib().vk_spmv(C.byref(a), alpha, _p(x), beta, _p(y), int(transpose),
                         SPMV_SEQUENTIAL if order == "sequential" else SPMV_FAST))
    return y


def csr_transpose(ro, ci, v, rows, cols):
    keep = _Keep()
    a = _csr(keep, rows, cols, ro, ci, v)
    nnz = int(np.asarray(ro)[rows]) if rows >= 0 else 0
    tro = np.zeros(cols + 1, np.int64)
    tci = np.zeros(max(nnz, 1), np.int64)
    tv = np.zeros(max(nnz, 1))
    perm = np.zeros(max(nnz, 1), np.int64)
    _check(lib().vk_csr_transpose(C.byref(a), _p(tro, _i64p), _p(tci, _i64p), _p(tv), _p(perm, _i64p)))
    return tro, tci[:nnz], tv[:nnz], perm[:nnz]


class SpMat:
    """A sparse operator resident on the GPU; apply() works on device pointers."""

    def __init__(self, ro, ci, v, rows, cols, precision="fp64"):
        keep = _Keep()
        a = _csr(keep, rows, cols, ro, ci, v)
        h = C.c_void_p()
        _check(lib().vk_spmat_create(C.byref(a), PREC_MIXED if precision == "mixed" else PREC_FP64, C.byref(h)))
        self._h = h
        self.rows, self.cols = rows, cols

    def apply(self, x_ptr: int, y_ptr: int, transpose: bool = False, stream: int = 0):
        _check(lib().vk_spmat_apply_device(self._h, C.c_void_p(x_ptr), C.c_void_p(y_ptr), int(transpose),
                                           C.c_void_p(stream)))

    def bytes(self, transpose: bool = False) -> int:
        return int(lib().vk_spmat_bytes(self._h, int(transpose)))

    def variant(self, transpose: bool = False) -> int:
        return int(lib().vk_spmat_variant(self._h, int(transpose)))

    def set_variant(self, variant: int, transpose: bool = False):
        _check(lib().vk_spmat_set_variant(self._h, int(transpose), int(variant)))

    def close(self):
        if getattr(self, "_h", None):
            lib().vk_spmat_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
