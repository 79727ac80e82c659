"""The design record and the L-BFGS search, on the host.

The keys and record lines are checked against the reference's own ``Design.key`` and
``Record.append`` (``tests/golden/record_*``, made by ``tests/golden/make_golden.py``), so a
record written by either code resumes in the other.
"""

from __future__ import annotations

import json
import math
import shutil

import numpy as np
import pytest

from beamtracer_b200.optimization import Design, Evaluation, Parameter, Record, lbfgs_search
from tests.golden import host_cases as hc
from tests.gpu_util import GOLDEN


def _design(name: str) -> tuple[Design, list]:
    parameters, points = hc.RECORD_DESIGNS[name]
    return Design(tuple(Parameter(*p) for p in parameters)), points


@pytest.mark.parametrize("name", sorted(hc.RECORD_DESIGNS))
def test_keys_are_the_reference_keys(name):
    design, points = _design(name)
    want = json.loads((GOLDEN / "record_keys.json").read_text())[name]
    assert [design.key(x) for x in points] == want


def _same(a, b) -> bool:
    if isinstance(a, float) and isinstance(b, float) and math.isnan(a) and math.isnan(b):
        return True
    if isinstance(a, dict) and isinstance(b, dict):
        return a.keys() == b.keys() and all(_same(a[k], b[k]) for k in a)
    return a == b


def test_record_lines_are_the_reference_lines(tmp_path):
    design, points = _design(hc.RECORD_CASE)
    record = Record(design, tmp_path / "mine.jsonl")
    record.append([Evaluation(**e) for e in hc.record_evaluations(design.names, points)])
    mine = [json.loads(x) for x in (tmp_path / "mine.jsonl").read_text().splitlines()]
    reference = [json.loads(x) for x in (GOLDEN / "record_reference.jsonl").read_text().splitlines()]
    assert len(mine) == len(reference) == 3
    for a, b in zip(mine, reference, strict=True):
        assert _same(a, b)


def test_a_reference_record_resumes(tmp_path):
    design, points = _design(hc.RECORD_CASE)
    path = tmp_path / "record.jsonl"
    shutil.copy(GOLDEN / "record_reference.jsonl", path)
    record = Record(design, path)
    assert len(record) == 3
    first = record.get(design.key(points[0]))
    assert first is not None and first.feasible and first.objectives["rms_angle"] == 1e-3
    assert not record.get(design.key(points[1])).ok
    assert math.isnan(record.get(design.key(points[2])).diagnostics["current"])
    with pytest.raises(ValueError, match="parameters"):
        Record(Design((Parameter("other", 0.0, 1.0),)), path)


def test_lbfgs_finds_a_bounded_minimum_and_resumes(tmp_path):
    """A quadratic with its minimum inside the box in one parameter and beyond the bound in
    the other: L-BFGS-B finds both; a second search from the record computes nothing."""
    design = Design((Parameter("a", 0.0, 10.0), Parameter("b", -1.0, 1.0)))
    calls = []

    def evaluate(values):
        a, b = values["a"], values["b"]
        calls.append((a, b))
        f = (a - 3.0) ** 2 + 4.0 * (b - 2.0) ** 2
        return Evaluation({"f": f}, diagnostics={"gradient": {"a": 2 * (a - 3.0),
                                                              "b": 8.0 * (b - 2.0)}})  # fmt: skip

    path = tmp_path / "search.jsonl"
    first = lbfgs_search(design, evaluate, {"a": 8.0, "b": 0.0}, objective="f",
                         record=Record(design, path), max_evaluations=40)  # fmt: skip
    assert first.best.parameters["a"] == pytest.approx(3.0, abs=1e-6)
    assert first.best.parameters["b"] == pytest.approx(1.0, abs=1e-9)
    assert first.computed == len(calls) > 1
    lines = path.read_text().splitlines()
    assert len(lines) == first.computed
    assert all("gradient" in json.loads(x)["diagnostics"] for x in lines)
    again = lbfgs_search(design, evaluate, {"a": 8.0, "b": 0.0}, objective="f",
                         record=Record(design, path), max_evaluations=40)  # fmt: skip
    assert again.computed == 0
    assert again.best.parameters == first.best.parameters


def test_failed_evaluations_rank_last():
    good = Evaluation({"f": 5.0}, constraints={"g": -1.0})
    infeasible = Evaluation({"f": 1.0}, constraints={"g": 0.5})
    failed = Evaluation({"f": np.nan}, converged=False, failure="boom")
    ranked = sorted([failed, infeasible, good], key=lambda e: e.rank("f"))
    assert ranked == [good, infeasible, failed]
