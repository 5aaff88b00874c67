"""The C-ABI library itself, without a GPU: it loads, exports every entry point
include/*.h declares, mirrors SolverOptions' defaults, and rejects invalid
models with the reference's statuses and messages before touching the device
(Model.cpp:118-199, continuous_common.hpp:36-126, pdhg.cpp:274-291,
pdqp.cpp:313-327)."""

import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

import vikalp_b200 as vk

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions(header="vikalp_b200.h"):
    names = set()
    for h in [os.path.join(ROOT, "include", header)]:
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(vk_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return names


def test_exports_every_declared_symbol():
    names = declared_functions()
    assert {"vk_pdhg_create", "vk_pdhg_solve", "vk_pdhg_destroy", "vk_spmv", "vk_csr_transpose"} <= names
    L = C.CDLL(vk.LIB_PATH)
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing
    # and the Python binding knows every one of them
    assert names <= set(vk._SIGNATURES), names - set(vk._SIGNATURES)
    # the MPS entry points live in the C++ host layer
    mps = declared_functions("vikalp_mps.h")
    assert {"vk_mps_read", "vk_mps_problem", "vk_mps_free"} <= mps
    H = C.CDLL(vk.HOST_LIB_PATH)
    assert not [n for n in sorted(mps) if not hasattr(H, n)]
    assert mps <= set(vk._MPS_SIGNATURES), mps - set(vk._MPS_SIGNATURES)
    # every header under include/ is one of the two
    assert sorted(os.path.basename(h) for h in glob.glob(os.path.join(ROOT, "include", "*.h"))) == \
        ["vikalp_b200.h", "vikalp_mps.h"]


def test_defaults_mirror_solver_options():
    o = vk.options()
    # SolverOptions.hpp:16-27
    assert o.iteration_limit == 100000
    assert np.isinf(o.time_limit_seconds)
    assert o.primal_tolerance == 1e-7 and o.dual_tolerance == 1e-7
    assert o.continuous_method == 0
    assert o.algorithm == vk.ALGO_REFERENCE and o.precision == vk.PREC_FP64
    assert vk.lib().vk_version().startswith(b"vikalp_b200")


class M:
    """Minimal model (1 variable, no rows) in Instance form."""

    def __init__(self, **kw):
        self.m, self.n = 0, 1
        self.row_offsets = np.zeros(1, np.int64)
        self.col_idx = np.zeros(0, np.int64)
        self.values = np.zeros(0)
        self.c = np.array([-1.0])
        self.var_lower, self.var_upper = np.array([0.0]), np.array([10.0])
        self.row_lower = self.row_upper = np.zeros(0)
        self.objective_offset = 0.0
        self.q_row_offsets = self.q_col_idx = self.q_values = None
        self.__dict__.update(kw)

    @property
    def q_nnz(self):
        return 0 if self.q_col_idx is None else len(self.q_col_idx)


def create_error(model, **opts):
    with pytest.raises(vk.VkError) as e:
        vk.Pdhg(model, **opts)
    return e.value.code, e.value.msg


def test_invalid_variable_bounds():
    # test_pdhg.cpp:193-196: lower 3 > upper 2
    code, msg = create_error(M(var_lower=np.array([3.0]), var_upper=np.array([2.0])))
    assert code == vk.VK_ERR_INVALID
    assert msg == "variable bounds contains an invalid bound at index 0"


def test_negative_iteration_limit():
    # test_pdhg.cpp:212-216
    code, msg = create_error(M(), iteration_limit=-1)
    assert code == vk.VK_ERR_INVALID and msg == "solver limits and tolerances must be non-negative"


def test_nonfinite_objective():
    code, msg = create_error(M(c=np.array([np.nan])))
    assert code == vk.VK_ERR_INVALID and msg == "objective coefficients must be finite"


def test_no_variables():
    code, msg = create_error(M(n=0, c=np.zeros(0), var_lower=np.zeros(0), var_upper=np.zeros(0)))
    assert code == vk.VK_ERR_INVALID and msg == "LP requires at least one variable"


def test_malformed_csr():
    # unordered columns in a row (Model.cpp:46-49)
    m = M(m=1, n=2, row_offsets=np.array([0, 2]), col_idx=np.array([1, 0]), values=np.array([1.0, 1.0]),
          c=np.zeros(2), var_lower=np.zeros(2), var_upper=np.ones(2), row_lower=np.array([0.0]),
          row_upper=np.array([1.0]))
    code, msg = create_error(m)
    assert code == vk.VK_ERR_INVALID and msg == "constraint matrix columns must be strictly ordered per row"
    m.col_idx = np.array([0, 5])
    assert create_error(m)[1] == "constraint matrix contains an out-of-range column"
    m.col_idx = np.array([0, 1])
    m.values = np.array([1.0, np.inf])
    assert create_error(m)[1] == "constraint matrix coefficients must be finite"


def test_malformed_csr_large_first_error_wins():
    # patterns of more than 2^20 rows are checked on several host threads; the
    # message is still the one of the first failing row in order
    rows = 3 << 20
    ro = np.arange(rows + 1, dtype=np.int64) * 2
    ci = np.tile(np.array([0, 1], np.int64), rows)
    m = M(m=rows, n=3, row_offsets=ro, col_idx=ci.copy(), values=np.ones(2 * rows), c=np.zeros(3),
          var_lower=np.zeros(3), var_upper=np.ones(3), row_lower=np.zeros(rows), row_upper=np.ones(rows))
    m.col_idx[2 * (rows - 10)] = 7                   # out of range, late
    m.col_idx[2 * (rows // 2) + 1] = 0              # unordered, earlier
    assert create_error(m)[1] == "constraint matrix columns must be strictly ordered per row"
    m.col_idx[2 * 1000] = -1                        # out of range, earliest
    assert create_error(m)[1] == "constraint matrix contains an out-of-range column"
    m.col_idx = ci.copy()
    m.values[2 * rows - 1] = np.nan                 # the last coefficient
    assert create_error(m)[1] == "constraint matrix coefficients must be finite"
    m.values[2 * rows - 1] = 1.0
    m.row_offsets = ro.copy()
    m.row_offsets[rows - 5] = 2 * rows + 4          # beyond nnz: rows - 6 and rows - 5 fail
    assert create_error(m)[1] == "constraint matrix row_offsets must be ordered and in range"


def test_row_bounds_invalid():
    m = M(m=1, row_offsets=np.array([0, 1]), col_idx=np.array([0]), values=np.array([1.0]),
          row_lower=np.array([2.0]), row_upper=np.array([1.0]))
    assert create_error(m)[1] == "constraint bounds contains an invalid bound at index 0"


def test_nonconvex_qp_is_unsupported():
    # test_pdhg.cpp:161-164
    m = M(c=np.array([-10.0]), q_row_offsets=np.array([0, 1]), q_col_idx=np.array([0]), q_values=np.array([-2.0]))
    code, msg = create_error(m)
    assert code == vk.VK_ERR_UNSUPPORTED and msg == "QP objective matrix is not positive semidefinite"


def test_asymmetric_q():
    m = M(n=2, c=np.zeros(2), var_lower=np.zeros(2), var_upper=np.ones(2),
          q_row_offsets=np.array([0, 2, 3]), q_col_idx=np.array([0, 1, 1]), q_values=np.array([1.0, 0.5, 1.0]))
    assert create_error(m)[1] == "quadratic objective must be stored symmetrically"


def test_unsupported_method():
    code, msg = create_error(M(), continuous_method=2)
    assert code == vk.VK_ERR_UNSUPPORTED and msg == "requested continuous method is not implemented for LP"


def test_large_psd_gate_rejects_indefinite():
    # n above the dense threshold: the Lanczos gate must still reject an
    # indefinite Q (and accept a PSD one, which then fails only at device setup).
    n = 2000
    ro = np.arange(n + 1, dtype=np.int64)
    ci = np.arange(n, dtype=np.int64)
    d = np.ones(n)
    d[1234] = -0.5
    m = M(n=n, c=np.zeros(n), var_lower=-np.ones(n), var_upper=np.ones(n), q_row_offsets=ro, q_col_idx=ci,
          q_values=d)
    code, msg = create_error(m)
    assert code == vk.VK_ERR_UNSUPPORTED and msg == "QP objective matrix is not positive semidefinite"


def batch_error(models, **opts):
    with pytest.raises(vk.VkError) as e:
        vk.batch_solve(models, **opts)
    return e.value.code, e.value.msg


def test_batch_names_the_invalid_member():
    code, msg = batch_error([M(), M(var_lower=np.array([3.0]), var_upper=np.array([2.0]))])
    assert code == vk.VK_ERR_INVALID
    assert msg == "instance 1: variable bounds contains an invalid bound at index 0"


def test_batch_first_invalid_member_in_order():
    # batches of 8 or more members are checked over host threads; the member
    # reported is still the first invalid one in order
    bad_bounds = dict(var_lower=np.array([3.0]), var_upper=np.array([2.0]))
    models = [M() for _ in range(40)]
    models[29] = M(c=np.array([np.inf]))
    models[17] = M(**bad_bounds)
    models[35] = M(**bad_bounds)
    code, msg = batch_error(models)
    assert code == vk.VK_ERR_INVALID
    assert msg == "instance 17: variable bounds contains an invalid bound at index 0"
    models[4] = M(c=np.array([np.nan]))
    assert batch_error(models)[1] == "instance 4: objective coefficients must be finite"


def test_batch_requires_halpern_and_lp():
    code, _ = batch_error([M()], algorithm="reference")
    assert code == vk.VK_ERR_UNSUPPORTED
    q = M(q_row_offsets=np.array([0, 1], np.int64), q_col_idx=np.array([0], np.int64), q_values=np.array([1.0]))
    code, msg = batch_error([M(), q])
    assert code == vk.VK_ERR_UNSUPPORTED and msg.startswith("instance 1")
    assert vk.lib().vk_batch_solve(None, 0, None, None) == vk.VK_ERR_INVALID


def test_shared_batch_validates_the_model():
    with pytest.raises(vk.VkError) as e:
        vk.batch_solve_shared(M(var_lower=np.array([3.0]), var_upper=np.array([2.0])), 4)
    assert e.value.code == vk.VK_ERR_INVALID
    assert e.value.msg == "variable bounds contains an invalid bound at index 0"
    with pytest.raises(vk.VkError) as e:
        vk.batch_solve_shared(M(), 4, algorithm="reference")
    assert e.value.code == vk.VK_ERR_UNSUPPORTED
    assert vk.lib().vk_batch_solve_shared(None, 1, None, None, None, None, None) == vk.VK_ERR_INVALID


def test_adjoint_validates_before_the_device():
    lp = M(m=1, row_offsets=np.array([0, 1], np.int64), col_idx=np.array([0], np.int64), values=np.array([1.0]),
           row_lower=np.array([-np.inf]), row_upper=np.array([4.0]))
    with pytest.raises(vk.VkError) as e:
        vk.lp_adjoint([lp], [np.array([np.nan])], [np.zeros(1)], [np.ones(1)])
    assert e.value.code == vk.VK_ERR_INVALID and e.value.msg == "x and dL_dx must be finite"
    q = M(q_row_offsets=np.array([0, 1], np.int64), q_col_idx=np.array([0], np.int64), q_values=np.array([1.0]))
    with pytest.raises(vk.VkError) as e:
        vk.lp_adjoint([q], [np.zeros(1)], [np.zeros(0)], [np.ones(1)])
    assert e.value.code == vk.VK_ERR_UNSUPPORTED
    with pytest.raises(vk.VkError) as e:
        vk.lp_adjoint([lp], [np.zeros(1)], [np.zeros(1)], [np.ones(1)], solve_tolerance=0.0)
    assert e.value.code == vk.VK_ERR_INVALID


def test_device_vector_argument_errors_without_a_gpu():
    # checked before any CUDA call: a negative size and null handles
    L = vk.lib()
    out = C.c_void_p()
    assert L.vk_dvec_create(-1, C.byref(out)) == vk.VK_ERR_INVALID
    assert "non-negative" in vk.last_error()
    assert L.vk_dvec_size(None) == -1
    r = C.c_double()
    assert L.vk_dvec_dot(None, None, C.byref(r)) == vk.VK_ERR_INVALID
    assert L.vk_dvec_axpby(1.0, None, 1.0, None) == vk.VK_ERR_INVALID
    assert L.vk_spmat_multiply(None, 1.0, None, 0.0, None, 0, 0) == vk.VK_ERR_INVALID
    assert L.vk_spmat_set_values(None, None, 0) == vk.VK_ERR_INVALID
