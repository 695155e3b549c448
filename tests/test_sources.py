"""Source hygiene of the Python layer: no module defines a top-level function or class twice (a
later definition silently replaces the earlier one)."""
import ast
from collections import Counter
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
FILES = sorted((ROOT / "three-mesh-bvh_b200").glob("*.py")) + [ROOT / "bench.py", ROOT / "__graft_entry__.py"]


@pytest.mark.parametrize("path", FILES, ids=[p.name for p in FILES])
def test_no_duplicate_top_level_definitions(path):
    tree = ast.parse(path.read_text())
    names = Counter(n.name for n in tree.body if isinstance(n, (ast.FunctionDef, ast.AsyncFunctionDef, ast.ClassDef)))
    assert not [k for k, v in names.items() if v > 1], path
