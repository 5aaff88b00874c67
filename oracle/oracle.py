"""ctypes bindings for the CPU checkers -- TEST / BASELINE INFRASTRUCTURE ONLY.

``Oracle``    wraps ``oracle/liboracle.so`` (the C restatement in pdhg_oracle.c).
``Reference`` wraps ``oracle/_ref/libvkref.so`` (the reference's own CPU sources,
              built by oracle/Makefile where the reference tree is present; the
              built library travels with the repository snapshot).
``ReferenceCuda`` wraps ``oracle/_ref/libvkref_cuda.so``: the same sources with
              the reference's CUDA backend (cuda/cuda_ops.cu, cuSPARSE) built
              for sm_100a, for the GPU-to-GPU comparison in bench.py.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's baseline legs (the
reference's CPU code, and its CUDA backend as a comparison figure) use these;
the CUDA library never does.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libvkref.so")
REF_CUDA_SO = os.path.join(HERE, "_ref", "libvkref_cuda.so")

_i64p = C.POINTER(C.c_int64)
_f64p = C.POINTER(C.c_double)

STATUS = {0: "NotSolved", 1: "Optimal", 2: "LocallyOptimal", 3: "Feasible", 4: "Infeasible",
          5: "Unbounded", 6: "IterationLimit", 7: "NodeLimit", 8: "TimeLimit",
          9: "NumericalFailure", 10: "UnsupportedModel", 11: "InvalidModel"}


def _p(a, typ=_f64p):
    return None if a is None else a.ctypes.data_as(typ)


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def _i64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.int64)


class _Problem(C.Structure):
    _fields_ = [("m", C.c_int64), ("n", C.c_int64), ("ro", _i64p), ("ci", _i64p), ("v", _f64p),
                ("q_nnz", C.c_int64), ("qro", _i64p), ("qci", _i64p), ("qv", _f64p),
                ("c", _f64p), ("rl", _f64p), ("ru", _f64p), ("objective_offset", C.c_double)]


class _RefProblem(C.Structure):
    _fields_ = _Problem._fields_ + [("l", _f64p), ("u", _f64p)]


class _Options(C.Structure):
    _fields_ = [("iteration_limit", C.c_int64), ("time_limit_seconds", C.c_double),
                ("primal_tolerance", C.c_double), ("dual_tolerance", C.c_double)]


class _RefOptions(C.Structure):
    _fields_ = _Options._fields_ + [("backend", C.c_int32), ("method", C.c_int32)]


class _Result(C.Structure):
    _fields_ = [("x", _f64p), ("y", _f64p), ("row_lower_dual", _f64p), ("row_upper_dual", _f64p),
                ("var_lower_dual", _f64p), ("var_upper_dual", _f64p), ("scaled_x", _f64p),
                ("scaled_y", _f64p), ("status", C.c_int), ("iterations", C.c_int64),
                ("restarts", C.c_int64), ("objective", C.c_double), ("primal_residual", C.c_double),
                ("stationarity_residual", C.c_double), ("complementarity_residual", C.c_double),
                ("last_metric", C.c_double), ("tau", C.c_double), ("solve_seconds", C.c_double)]


class _RefResult(C.Structure):
    _fields_ = [("x", _f64p), ("row_lower_dual", _f64p), ("row_upper_dual", _f64p),
                ("var_lower_dual", _f64p), ("var_upper_dual", _f64p), ("status", C.c_int32),
                ("iterations", C.c_int64), ("objective", C.c_double), ("primal_residual", C.c_double),
                ("stationarity_residual", C.c_double), ("complementarity_residual", C.c_double),
                ("dual_bound", C.c_double), ("solve_seconds", C.c_double),
                ("solver", C.c_char * 32), ("backend", C.c_char * 32), ("message", C.c_char * 256)]


class _Kkt(C.Structure):
    _fields_ = [("primal_residual", C.c_double), ("dual_residual", C.c_double), ("gap", C.c_double),
                ("primal_objective", C.c_double), ("dual_objective", C.c_double),
                ("rel_primal", C.c_double), ("rel_dual", C.c_double), ("rel_gap", C.c_double)]


class _Keep:
    """Holds the numpy arrays a ctypes struct points into."""

    def __init__(self):
        self.refs = []

    def f(self, a):
        a = _f64(a)
        self.refs.append(a)
        return _p(a)

    def i(self, a):
        a = _i64(a)
        self.refs.append(a)
        return _p(a, _i64p)


def _fill_problem(st, inst, keep: _Keep):
    st.m, st.n = inst.m, inst.n
    st.ro, st.ci, st.v = keep.i(inst.row_offsets), keep.i(inst.col_idx), keep.f(inst.values)
    if inst.q_nnz > 0:
        st.q_nnz = inst.q_nnz
        st.qro, st.qci, st.qv = keep.i(inst.q_row_offsets), keep.i(inst.q_col_idx), keep.f(inst.q_values)
    else:
        st.q_nnz = 0
    st.c, st.rl, st.ru = keep.f(inst.c), keep.f(inst.row_lower), keep.f(inst.row_upper)
    st.objective_offset = float(inst.objective_offset)


class Oracle:
    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
        lib = C.CDLL(path)
        lib.or_pdhg_solve.restype = C.c_int
        lib.or_pdhg_solve.argtypes = [C.POINTER(_Problem), C.POINTER(_Options), _f64p, _f64p, _f64p,
                                      C.POINTER(_Result)]
        lib.or_rel_kkt.argtypes = [C.POINTER(_Problem), _f64p, _f64p, _f64p, _f64p, C.POINTER(_Kkt)]
        lib.or_spmv.argtypes = [C.c_int64, _i64p, _i64p, _f64p, C.c_double, _f64p, C.c_double, _f64p]
        lib.or_spmv_t.argtypes = [C.c_int64, C.c_int64, _i64p, _i64p, _f64p, C.c_double, _f64p,
                                  C.c_double, _f64p]
        lib.or_csr_transpose.argtypes = [C.c_int64, C.c_int64, _i64p, _i64p, _f64p, _i64p, _i64p,
                                         _f64p, _i64p]
        lib.or_operator_bound.restype = C.c_double
        lib.or_operator_bound.argtypes = [C.c_int64, C.c_int64, _i64p, _i64p, _f64p]
        self.lib = lib

    def spmv(self, ro, ci, v, x, alpha=1.0, beta=0.0, y=None):
        ro, ci, v, x = _i64(ro), _i64(ci), _f64(v), _f64(x)
        m = ro.shape[0] - 1
        y = np.zeros(m) if y is None else _f64(y).copy()
        self.lib.or_spmv(m, _p(ro, _i64p), _p(ci, _i64p), _p(v), alpha, _p(x), beta, _p(y))
        return y

    def spmv_t(self, ro, ci, v, n, x, alpha=1.0, beta=0.0, y=None):
        ro, ci, v, x = _i64(ro), _i64(ci), _f64(v), _f64(x)
        m = ro.shape[0] - 1
        y = np.zeros(n) if y is None else _f64(y).copy()
        self.lib.or_spmv_t(m, n, _p(ro, _i64p), _p(ci, _i64p), _p(v), alpha, _p(x), beta, _p(y))
        return y

    def transpose(self, ro, ci, v, n):
        ro, ci, v = _i64(ro), _i64(ci), _f64(v)
        m = ro.shape[0] - 1
        nnz = int(ro[-1])
        tro = np.zeros(n + 1, np.int64)
        trow = np.zeros(max(nnz, 1), np.int64)
        tv = np.zeros(max(nnz, 1))
        perm = np.zeros(max(nnz, 1), np.int64)
        self.lib.or_csr_transpose(m, n, _p(ro, _i64p), _p(ci, _i64p), _p(v), _p(tro, _i64p),
                                  _p(trow, _i64p), _p(tv), _p(perm, _i64p))
        return tro, trow[:nnz], tv[:nnz], perm[:nnz]

    def operator_bound(self, ro, ci, v, n):
        ro, ci, v = _i64(ro), _i64(ci), _f64(v)
        return self.lib.or_operator_bound(ro.shape[0] - 1, n, _p(ro, _i64p), _p(ci, _i64p), _p(v))

    def pdhg_solve(self, inst, iteration_limit=100000, primal_tolerance=1e-7, dual_tolerance=1e-7,
                   time_limit_seconds=float("inf"), warm=None, lower=None, upper=None):
        keep = _Keep()
        prob = _Problem()
        _fill_problem(prob, inst, keep)
        opt = _Options(iteration_limit, time_limit_seconds, primal_tolerance, dual_tolerance)
        lo = _f64(inst.var_lower if lower is None else lower)
        hi = _f64(inst.var_upper if upper is None else upper)
        m, n = inst.m, inst.n
        out = {k: np.zeros(m) for k in ("y", "row_lower_dual", "row_upper_dual", "scaled_y")}
        out.update({k: np.zeros(n) for k in ("x", "var_lower_dual", "var_upper_dual", "scaled_x")})
        res = _Result()
        for k, a in out.items():
            setattr(res, k, _p(a))
        rc = self.lib.or_pdhg_solve(C.byref(prob), C.byref(opt), _p(_f64(warm)), _p(lo), _p(hi), C.byref(res))
        if rc != 0:
            return {"status": "InvalidModel"}
        out.update(status=STATUS[res.status], iterations=res.iterations, restarts=res.restarts,
                   objective=res.objective, primal_residual=res.primal_residual,
                   stationarity_residual=res.stationarity_residual,
                   complementarity_residual=res.complementarity_residual, last_metric=res.last_metric,
                   tau=res.tau, solve_seconds=res.solve_seconds)
        return out

    def rel_kkt(self, inst, x, y, lower=None, upper=None):
        keep = _Keep()
        prob = _Problem()
        _fill_problem(prob, inst, keep)
        lo = _f64(inst.var_lower if lower is None else lower)
        hi = _f64(inst.var_upper if upper is None else upper)
        k = _Kkt()
        self.lib.or_rel_kkt(C.byref(prob), _p(lo), _p(hi), _p(_f64(x)), _p(_f64(y)), C.byref(k))
        return {f: getattr(k, f) for f, _ in _Kkt._fields_}


class Reference:
    """The reference's own CPU implementation (compiled from its sources)."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: build it with `make -C oracle ref REF=<reference tree>`")
        lib = C.CDLL(path)
        lib.vkref_solve_continuous.restype = C.c_int
        lib.vkref_solve_continuous.argtypes = [C.POINTER(_RefProblem), C.POINTER(_RefOptions), _f64p,
                                               _f64p, _f64p, C.c_int, C.POINTER(_RefResult)]
        lib.vkref_solve.restype = C.c_int
        lib.vkref_solve.argtypes = [C.POINTER(_RefProblem), C.POINTER(_RefOptions), C.POINTER(_RefResult)]
        lib.vkref_multiply.restype = C.c_int
        lib.vkref_multiply.argtypes = [C.c_int64, C.c_int64, _i64p, _i64p, _f64p, C.c_double, _f64p,
                                       C.c_int64, C.c_double, _f64p, C.c_int64, C.c_int, C.c_char_p, C.c_int]
        lib.vkref_mps_read.restype = C.c_void_p
        lib.vkref_mps_read.argtypes = [C.c_char_p]
        lib.vkref_mps_ok.argtypes = [C.c_void_p]
        lib.vkref_mps_sizes.argtypes = [C.c_void_p, _i64p, _i64p, _i64p]
        lib.vkref_mps_sizes.restype = None
        lib.vkref_mps_arrays.argtypes = [C.c_void_p, _i64p, _i64p, _f64p, _f64p, _f64p, _f64p, _f64p, _f64p,
                                         C.POINTER(C.c_int32)]
        lib.vkref_mps_arrays.restype = None
        lib.vkref_mps_name.restype = C.c_char_p
        lib.vkref_mps_name.argtypes = [C.c_void_p]
        lib.vkref_mps_error_count.argtypes = [C.c_void_p]
        lib.vkref_mps_error.restype = C.c_char_p
        lib.vkref_mps_error.argtypes = [C.c_void_p, C.c_int, _i64p]
        lib.vkref_mps_free.argtypes = [C.c_void_p]
        lib.vkref_mps_free.restype = None
        lib.vkref_pdhg_replay.restype = C.c_double
        lib.vkref_pdhg_replay.argtypes = [C.POINTER(_RefProblem), C.c_double, C.c_int64, _f64p, _f64p]
        self.lib = lib

    def read_mps(self, path):
        """vikalp::MpsReader::read on `path`: ok flag, errors [(line, message)],
        and the model's arrays (MpsReader.cpp:10-559)."""
        h = self.lib.vkref_mps_read(path.encode())
        try:
            errors = []
            for i in range(self.lib.vkref_mps_error_count(h)):
                ln = C.c_int64()
                msg = self.lib.vkref_mps_error(h, i, C.byref(ln)).decode()
                errors.append((int(ln.value), msg))
            out = {"ok": bool(self.lib.vkref_mps_ok(h)), "errors": errors,
                   "name": self.lib.vkref_mps_name(h).decode()}
            m, n, nnz = C.c_int64(), C.c_int64(), C.c_int64()
            self.lib.vkref_mps_sizes(h, C.byref(m), C.byref(n), C.byref(nnz))
            m, n, nnz = m.value, n.value, nnz.value
            ro = np.zeros(m + 1, np.int64)
            ci = np.zeros(nnz, np.int64)
            arr = {k: np.zeros(n) for k in ("c", "var_lower", "var_upper")}
            arr.update(values=np.zeros(nnz), row_lower=np.zeros(m), row_upper=np.zeros(m))
            types = np.zeros(n, np.int32)
            if len(out["errors"]) == 0 or out["ok"]:
                self.lib.vkref_mps_arrays(h, _p(ro, _i64p), _p(ci, _i64p), _p(arr["values"]), _p(arr["c"]),
                                          _p(arr["var_lower"]), _p(arr["var_upper"]), _p(arr["row_lower"]),
                                          _p(arr["row_upper"]), types.ctypes.data_as(C.POINTER(C.c_int32)))
            out.update(m=m, n=n, row_offsets=ro, col_idx=ci, types=types, **arr)
            return out
        finally:
            self.lib.vkref_mps_free(h)

    def _prob(self, inst, keep, lower=None, upper=None):
        st = _RefProblem()
        _fill_problem(st, inst, keep)
        st.l = keep.f(inst.var_lower if lower is None else lower)
        st.u = keep.f(inst.var_upper if upper is None else upper)
        return st

    def _solve(self, fn, inst, opts, extra):
        keep = _Keep()
        prob = self._prob(inst, keep)
        o = _RefOptions(opts.get("iteration_limit", 100000), opts.get("time_limit_seconds", float("inf")),
                        opts.get("primal_tolerance", 1e-7), opts.get("dual_tolerance", 1e-7),
                        opts.get("backend", 0), opts.get("method", 0))
        m, n = inst.m, inst.n
        out = {k: np.zeros(m) for k in ("row_lower_dual", "row_upper_dual")}
        out.update({k: np.zeros(n) for k in ("x", "var_lower_dual", "var_upper_dual")})
        res = _RefResult()
        for k, a in out.items():
            setattr(res, k, _p(a))
        rc = fn(C.byref(prob), C.byref(o), *extra(keep), C.byref(res))
        out.update(rc=rc, status=STATUS.get(res.status, str(res.status)), iterations=res.iterations,
                   objective=res.objective, primal_residual=res.primal_residual,
                   stationarity_residual=res.stationarity_residual,
                   complementarity_residual=res.complementarity_residual, dual_bound=res.dual_bound,
                   solve_seconds=res.solve_seconds, solver=res.solver.decode(),
                   backend=res.backend.decode(), message=res.message.decode())
        out["y"] = out["row_upper_dual"] - out["row_lower_dual"]
        return out

    def solve_continuous(self, inst, qp=False, warm=None, lower=None, upper=None, **opts):
        def extra(keep):
            return (keep.f(warm) if warm is not None else None,
                    keep.f(lower) if lower is not None else None,
                    keep.f(upper) if upper is not None else None, int(qp))
        return self._solve(self.lib.vkref_solve_continuous, inst, opts, extra)

    def solve(self, inst, **opts):
        return self._solve(self.lib.vkref_solve, inst, opts, lambda keep: ())

    def multiply(self, ro, ci, v, n, x, y, alpha=1.0, beta=0.0, transpose=False):
        ro, ci, v, x = _i64(ro), _i64(ci), _f64(v), _f64(x)
        y = _f64(y).copy()
        err = C.create_string_buffer(256)
        rc = self.lib.vkref_multiply(ro.shape[0] - 1, n, _p(ro, _i64p), _p(ci, _i64p), _p(v), alpha, _p(x),
                                     x.shape[0], beta, _p(y), y.shape[0], int(transpose), err, 256)
        if rc != 0:
            raise ValueError(err.value.decode())
        return y

    def pdhg_replay(self, inst, step, iterations):
        keep = _Keep()
        prob = self._prob(inst, keep)
        x = np.zeros(inst.n)
        y = np.zeros(inst.m)
        secs = self.lib.vkref_pdhg_replay(C.byref(prob), step, iterations, _p(x), _p(y))
        return secs, x, y


class ReferenceCuda(Reference):
    """The reference built with its CUDA backend (cuda/cuda_ops.cu: cuSPARSE
    SpMV, SIMT vector kernels, host-finished reductions) for sm_100a -- the
    GPU-to-GPU comparison. Needs a GPU."""

    def __init__(self, path: str = REF_CUDA_SO):
        super().__init__(path)
        self.lib.vkref_pdhg_replay_cuda.restype = C.c_double
        self.lib.vkref_pdhg_replay_cuda.argtypes = [C.POINTER(_RefProblem), C.c_double, C.c_int64, _f64p, _f64p]

    def pdhg_replay_cuda(self, inst, step, iterations):
        """Seconds for `iterations` iterations of the pdhg.cpp:92-130 call
        sequence on the reference's CUDA backend, and the final x, y."""
        keep = _Keep()
        prob = self._prob(inst, keep)
        x = np.zeros(inst.n)
        y = np.zeros(inst.m)
        secs = self.lib.vkref_pdhg_replay_cuda(C.byref(prob), step, iterations, _p(x), _p(y))
        if secs < 0:
            raise RuntimeError("the reference's CUDA backend threw")
        return secs, x, y
