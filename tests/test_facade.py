"""The Alien back-end facade binary (tests/cpp/facade, built against the
reference's own back-end interface headers) loads and reports its traits
without a GPU: AlgebraTraits<BackEnd::tag::b200>::name() is "b200" and the
solver has no parallel support (one GPU)."""
import json
import subprocess
from pathlib import Path

import pytest

BIN = Path(__file__).resolve().parent / "cpp" / "_build" / "facade"


@pytest.mark.skipif(not BIN.exists(), reason="tests/cpp/_build/facade not built (reference sources absent)")
def test_facade_traits_without_gpu():
    out = subprocess.run([str(BIN), "traits"], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stderr
    assert json.loads(out.stdout.strip()) == {"name": "b200", "parallel": 0}
