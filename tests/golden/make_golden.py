"""Regenerate tests/golden/oracle_golden.json from the CPU oracle.

Run from the repository root: ``python tests/golden/make_golden.py``.
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))
from conftest import load_package  # noqa: E402
import oracle  # noqa: E402  (conftest put oracle/ on sys.path)
from golden_cases import compute_cases  # noqa: E402

pkg = load_package()
table = pkg.helm_table.ensure_table()
oracle.build()
data = compute_cases(oracle, pkg, table)
with open(os.path.join(HERE, "oracle_golden.json"), "w") as fp:
    json.dump(data, fp, indent=1)
print("wrote", len(data), "cases; table sha256", pkg.helm_table.sha256(table))
