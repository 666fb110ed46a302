"""The product's plan compiler (C++, libtdfs_b200.so) against the reference's
own PatternPreprocessor, and its error behaviour.  Host-only: no GPU."""
import json
import os

import pytest

from tests.test_cpu_oracle import _plans, same_plan


def test_product_plans_match_reference(T):
    for r in _plans():
        same_plan(r["plan"], T.PatternPreprocessor(text=r["text"], labeled=r["labeled"]).dump())


def test_multiplicity_exposed(T):
    rec = next(r for r in _plans() if r["name"] == "ref/7.g" and not r["labeled"])
    assert T.PatternPreprocessor(text=rec["text"]).PatternMultiplicity == 120


@pytest.mark.parametrize("text,code", [
    ("v 0 1\nv 1 1\nv 2 1\ne 0 1 1\n", 3),                    # no earlier neighbour
    ("v 0 1\nv 1 1\nv 2 1\ne 0 1 1\ne 1 1 1\n", 3),           # self-loop
    ("v 0 1\nv 1 1\nv 2 1\ne 0 1 1\ne 1 9 1\n", 3),           # endpoint out of range
    ("v 0 1\nv 1 1\nv 2 1\ne 0 1 1\nx 1 2 1\n", 2),           # malformed line
    ("".join(f"v {i} 1\n" for i in range(8)) + "e 0 1 1\n", 3),  # > 7 vertices
])
def test_pattern_errors(T, text, code):
    with pytest.raises(T.TdfsError) as e:
        T.PatternPreprocessor(text=text)
    assert e.value.code == code


def test_missing_pattern_file(T, tmp_path):
    with pytest.raises(T.TdfsError) as e:
        T.PatternPreprocessor(str(tmp_path / "nope.g"))
    assert e.value.code == 1


def test_blank_lines_tolerated(T):
    a = T.PatternPreprocessor(text="# c\nv 0 1\nv 1 1\nv 2 1\ne 0 1 1\ne 1 2 1\ne 0 2 1\n\n\n").dump()
    b = T.PatternPreprocessor(text="# c\nv 0 1\nv 1 1\nv 2 1\ne 0 1 1\ne 1 2 1\ne 0 2 1").dump()
    assert a == b
