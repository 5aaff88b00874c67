import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "reference_golden.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA library")


class GoldenModel:
    """A model stored in the golden fixture, in synthetic.Instance form."""

    def __init__(self, d, prefix):
        g = lambda k: d[f"{prefix}__model_{k}"]  # noqa: E731
        self.m, self.n = int(g("m")), int(g("n"))
        self.row_offsets, self.col_idx, self.values = g("ro"), g("ci"), g("v")
        self.c, self.var_lower, self.var_upper = g("c"), g("vl"), g("vu")
        self.row_lower, self.row_upper = g("rl"), g("ru")
        self.objective_offset = 0.0
        key = f"{prefix}__model_qro"
        if key in d:
            self.q_row_offsets, self.q_col_idx, self.q_values = g("qro"), g("qci"), g("qv")
        else:
            self.q_row_offsets = self.q_col_idx = self.q_values = None

    @property
    def nnz(self):
        return int(self.col_idx.shape[0])

    @property
    def q_nnz(self):
        return 0 if self.q_col_idx is None else int(self.q_col_idx.shape[0])


class GoldenCase:
    def __init__(self, d, name):
        p = f"pdhg_{name}"
        self.name = name
        self.model = GoldenModel(d, p)
        self.opts = {k.split("__opt_")[1]: d[k].item() for k in d.files if k.startswith(p + "__opt_")}
        self.extra = {k.split("__extra_")[1]: d[k] for k in d.files if k.startswith(p + "__extra_")}
        self.out = {k.split("__out_")[1]: d[k] for k in d.files if k.startswith(p + "__out_")}
        self.out["status"] = str(self.out["status"])


@pytest.fixture(scope="session")
def golden():
    return np.load(GOLDEN)


@pytest.fixture(scope="session")
def golden_cases(golden):
    return {str(n): GoldenCase(golden, str(n)) for n in golden["pdhg_cases"]}


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


def same_bits(a, b) -> bool:
    """Elementwise == (so -0.0 == +0.0), NaN positions equal."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if a.shape != b.shape:
        return False
    return bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))
