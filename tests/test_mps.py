"""The MPS ingest path: vikalp::MpsReader (vikalp_b200/host/mps.cpp) against
the reference's own reader (src/io/MpsReader.cpp, compiled into
oracle/_ref/libvkref.so) on generated files -- the same model (arrays, names,
variable types) and the same errors (line, message) -- and, on the GPU, a file
solved through the C ABI equal to the model it was written from."""

import os

import numpy as np
import pytest

import vikalp_b200 as vk
from vikalp_b200 import synthetic

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def reference():
    from oracle.oracle import Reference
    try:
        return Reference()
    except FileNotFoundError as e:  # pragma: no cover - the reference build is part of build()
        pytest.skip(str(e))


def fmt(v):
    return repr(float(v))


def write_mps(path, inst, name="GEN", two_per_line=True, bound_kinds=None, rng=None):
    """Writes `inst` as free-form MPS: E rows for [r, r], L rows for [-inf, u],
    G rows for [l, inf]; bounds LO / UP (or FX / FR / BV from bound_kinds)."""
    rows = []
    for i in range(inst.m):
        lo, hi = inst.row_lower[i], inst.row_upper[i]
        rows.append("E" if lo == hi else ("L" if np.isinf(lo) else "G"))
    lines = [f"NAME {name}", "ROWS", " N COST"] + [f" {t} R{i}" for i, t in enumerate(rows)]
    lines.append("COLUMNS")
    csc = [[] for _ in range(inst.n)]
    for i in range(inst.m):
        for k in range(inst.row_offsets[i], inst.row_offsets[i + 1]):
            csc[inst.col_idx[k]].append((f"R{i}", inst.values[k]))
    for j in range(inst.n):
        ents = [("COST", inst.c[j])] + csc[j] if inst.c[j] != 0.0 else csc[j]
        if not ents:
            ents = [("COST", 0.0)]
        k = 0
        while k < len(ents):
            if two_per_line and k + 1 < len(ents):
                lines.append(f" X{j} {ents[k][0]} {fmt(ents[k][1])} {ents[k + 1][0]} {fmt(ents[k + 1][1])}")
                k += 2
            else:
                lines.append(f" X{j} {ents[k][0]} {fmt(ents[k][1])}")
                k += 1
    lines.append("RHS")
    rhs = [(f"R{i}", inst.row_upper[i] if rows[i] != "G" else inst.row_lower[i]) for i in range(inst.m)]
    for k in range(0, len(rhs), 2):
        pair = rhs[k:k + 2]
        # (a set named RHS would read as the section keyword, in both readers)
        lines.append(" RHS1 " + " ".join(f"{r} {fmt(v)}" for r, v in pair))
    lines.append("BOUNDS")
    for j in range(inst.n):
        kind = (bound_kinds or {}).get(j)
        if kind == "FX":
            lines.append(f" FX BND X{j} {fmt(inst.var_lower[j])}")
        elif kind in ("FR", "BV"):
            lines.append(f" {kind} BND X{j}")
        else:
            lines.append(f" LO BND X{j} {fmt(inst.var_lower[j])}")
            lines.append(f" UP BND X{j} {fmt(inst.var_upper[j])}")
    lines.append("ENDATA")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def same_model(ours, ref):
    assert ours.ok == ref["ok"]
    assert ours.errors == ref["errors"]
    if not ref["ok"] and ref["errors"]:
        return
    assert ours.name == ref["name"]
    assert (ours.m, ours.n) == (ref["m"], ref["n"])
    assert np.array_equal(ours.row_offsets, ref["row_offsets"])
    assert np.array_equal(ours.col_idx, ref["col_idx"])
    for k in ("values", "c", "var_lower", "var_upper", "row_lower", "row_upper"):
        assert np.array_equal(getattr(ours, k), ref[k]), k
    assert ours.binaries == int((ref["types"] == 2).sum())


@pytest.mark.parametrize("seed,two", [(1, True), (2, False), (3, True)])
def test_generated_lp_matches_reference(tmp_path, reference, seed, two):
    inst = synthetic.lp_uniform(40, 90, 3, seed=seed)
    rng = np.random.default_rng(seed)
    kinds = {int(j): k for j, k in zip(rng.choice(90, 12, replace=False), ["FX", "FR", "BV"] * 4)}
    inst.var_lower = inst.var_lower.copy()
    inst.var_upper = inst.var_upper.copy()
    for j, k in kinds.items():
        if k == "FX":
            inst.var_lower[j] = inst.var_upper[j] = 2.5
    path = str(tmp_path / f"gen{seed}.mps")
    write_mps(path, inst, name=f"GEN{seed}", two_per_line=two, bound_kinds=kinds)
    ours, ref = vk.read_mps(path), reference.read_mps(path)
    same_model(ours, ref)
    assert ours.ok


CASES = {
    "duplicates_last_wins": "NAME D\nROWS\n N OBJ\n L R1\nCOLUMNS\n X R1 1.0 X R1 2.0\n X OBJ 3 X OBJ -1\n"
                            " Y R1 4\nRHS\n RHS R1 5 R1 6\nBOUNDS\n UP B X 4\n UP B X 7\nENDATA\n",
    "no_objective_row": "NAME N\nROWS\n G R1\nCOLUMNS\n X R1 1\nRHS\n RHS R1 2\nENDATA\n",
    "rhs_for_objective_and_unknown_rows_ignored": "NAME R\nROWS\n N OBJ\n E R1\nCOLUMNS\n X R1 1 OBJ 1\nRHS\n"
                                                 " B OBJ 9 ZZ 3\n B R1 2\nENDATA\n",
    # a line whose first token is a section keyword is that section's header,
    # so an RHS set named RHS loses its entries (the reference's rule, kept)
    "rhs_set_named_rhs": "NAME Q\nROWS\n N OBJ\n E R1\nCOLUMNS\n X R1 1\nRHS\n RHS R1 2\nENDATA\n",
    "tabs_and_extra_tokens": "NAME\tTAB  extra\nROWS\n\tN\tOBJ\n  L   R1   junk\nCOLUMNS\n X\tR1\t1.5\tOBJ\t2 trailing\n"
                             "RHS\n RHS R1 1e1\nBOUNDS\n FR B X\nENDATA\n",
    "missing_sections": "ROWS\n N OBJ\nCOLUMNS\n X OBJ 1\n",
    "unsupported_row_type": "NAME U\nROWS\n N OBJ\n X R1\n L R2\nCOLUMNS\n X R2 1\nRHS\nENDATA\n",
    "missing_row_name": "NAME M\nROWS\n N OBJ\n L\nCOLUMNS\n X OBJ 1\nRHS\nENDATA\n",
    "invalid_columns_entry": "NAME C\nROWS\n N OBJ\n L R1\nCOLUMNS\n X R1\n Y R1 notanumber\n Z R1 1\nRHS\nENDATA\n",
    "invalid_rhs_entry": "NAME H\nROWS\n N OBJ\n L R1\nCOLUMNS\n X R1 1\nRHS\n RHS R1\nENDATA\n",
    "bounds_errors": "NAME B\nROWS\n N OBJ\n L R1\nCOLUMNS\n X R1 1\nRHS\n RHS R1 1\nBOUNDS\n MI B X\n UP B X\n"
                     " UP B\n LO B Q 1\nENDATA\n",
    "unknown_row_in_columns": "NAME K\nROWS\n N OBJ\n L R1\nCOLUMNS\n X R9 1\n X R1 1\n Y R8 2\nRHS\nENDATA\n",
    "unknown_variable_in_bounds": "NAME V\nROWS\n N OBJ\n L R1\nCOLUMNS\n X R1 1\nRHS\nBOUNDS\n UP B Q 1\n"
                                  " LO B W 2\nENDATA\n",
    "blank_looking_line_in_rows": "NAME W\nROWS\n N OBJ\n   \n L R1\nCOLUMNS\n X R1 1\nRHS\nENDATA\n",
    "number_with_trailing_text": "NAME T\nROWS\n N OBJ\n L R1\nCOLUMNS\n X R1 1.5abc 2\nRHS\n RHS R1 3\nENDATA\n",
    "fails_model_checks": "NAME F\nROWS\n N OBJ\n L R1\nCOLUMNS\n X R1 1\nRHS\n RHS R1 1\nBOUNDS\n LO B X 5\n"
                          " UP B X 1\nENDATA\n",
    "empty_file": "",
    "stops_at_endata": "NAME S\nROWS\n N OBJ\n L R1\nCOLUMNS\n X R1 1\nRHS\nENDATA\nGARBAGE LINE\n",
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_edge_cases_match_reference(tmp_path, reference, name):
    path = str(tmp_path / f"{name}.mps")
    with open(path, "w") as f:
        f.write(CASES[name])
    same_model(vk.read_mps(path), reference.read_mps(path))


def test_missing_file(reference, tmp_path):
    path = str(tmp_path / "nope.mps")
    ours, ref = vk.read_mps(path), reference.read_mps(path)
    assert not ours.ok and ours.errors == ref["errors"] == [(0, f"unable to open MPS file: {path}")]


@pytest.mark.gpu
def test_mps_file_solves_like_its_model(tmp_path):
    # the ingest path feeds the solver: a file written from an LP solves, in
    # the reference scheme's sequential order, bit for bit like the LP itself
    inst = synthetic.lp_uniform(120, 300, 4, seed=11)
    path = str(tmp_path / "lp.mps")
    write_mps(path, inst)
    model = vk.read_mps(path)
    assert model.ok
    opts = dict(algorithm="reference", spmv_order="sequential", iteration_limit=400, primal_tolerance=0.0,
                dual_tolerance=0.0)
    a, b = vk.solve(model, **opts), vk.solve(inst, **opts)
    assert np.array_equal(a["x"], b["x"]) and np.array_equal(a["y"], b["y"])
    h = vk.solve(model, algorithm="halpern", relative_tolerance=1e-6)
    assert h["status"] == "Optimal"
