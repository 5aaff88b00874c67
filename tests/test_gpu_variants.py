"""Whole solves on every kernel variant of the sparse pass.

The setup autotuner picks one variant per matrix (and, for the reference
scheme, per fused pass) and only for matrices of 200k+ nonzeros, so the
regular tests reach few of them. Here each variant is pinned with
VIKALP_B200_VARIANT (which also pins it on small matrices) and a subprocess
runs the solver tests whose epilogues cover every hook of the pass: the
reference scheme's fused passes, the Halpern passes with KKT partial sums,
the independent-LP batch (per-tile sums, skipped tiles) and the adjoint
(masked per-tile passes)."""

import os
import subprocess
import sys

import pytest

import vikalp_b200 as vk

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SELECTED = [
    "tests/test_gpu_reference.py::test_fast_order_against_oracle_through_policy_iterations",
    "tests/test_gpu_reference.py::test_fast_order_close",
    "tests/test_gpu_halpern.py::test_iterates_match_restatement",
    "tests/test_gpu_halpern.py::test_solves_to_relative_kkt",
    "tests/test_gpu_halpern.py::test_qp_iterates_match_restatement",
    "tests/test_gpu_batch.py::test_batch_follows_each_single_trajectory",
    "tests/test_gpu_batch.py::test_batch_degenerate_members",
    "tests/test_gpu_batch.py::test_batch_limits",
    "tests/test_gpu_adjoint.py::test_lsqr_matches_oracle_at_the_same_point",
]


@pytest.mark.parametrize("variant", range(vk.FAST_VARIANTS))
def test_solves_on_pinned_variant(variant):
    env = dict(os.environ, VIKALP_B200_VARIANT=str(variant))
    r = subprocess.run([sys.executable, "-m", "pytest", "-x", "-q", "-m", "gpu", "-p", "no:cacheprovider", *SELECTED],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, f"variant {variant}:\n{r.stdout[-4000:]}\n{r.stderr[-2000:]}"
