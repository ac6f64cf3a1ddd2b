"""The Python binding's constants against the C headers' #defines: every
AB2_* value in include/*.h has its counterpart in alien_b200/abi.py with the
same number (no device needed)."""
import re
from pathlib import Path

from alien_b200 import abi

ROOT = Path(__file__).resolve().parents[1]
DEFINE = re.compile(r"^#define (AB2_[A-Z0-9_]+)\s+\(?(-?\d+)\)?", re.M)


def header_defines() -> dict[str, int]:
    out = {}
    for h in sorted((ROOT / "include").glob("*.h")):
        for name, value in DEFINE.findall(h.read_text()):
            out[name] = int(value)
    return out


def binding_value(name: str):
    """The abi.py value standing for the header constant `name`."""
    if name == "AB2_OK" or name.startswith("AB2_ERR_"):
        return getattr(abi, name)
    short = name[len("AB2_"):]
    for prefix in ("FMT_", "SPMV_"):
        if short.startswith(prefix):
            return getattr(abi, short)
    if short == "COMM_ID_BYTES":
        return abi.COMM_ID_BYTES
    tables = {"SOLVER_": abi.SOLVER, "PC_": abi.PRECOND, "ILU_": abi.ILU_SCHEDULE, "FCG_FALLBACK_": abi.FCG_FALLBACK,
              "MIXED_JACOBI_": abi.MIXED_JACOBI, "GNN_LAYER_": abi.GNN_LAYER}
    for prefix, table in tables.items():
        if short.startswith(prefix):
            return table[short[len(prefix):].lower()]
    if short.startswith("BREAKDOWN_"):
        word = short[len("BREAKDOWN_"):].lower()
        return next(k for k, v in abi.BREAKDOWN.items() if v == (None if word == "none" else word))
    raise KeyError(name)


def test_every_header_constant_has_its_binding_value():
    defs = header_defines()
    assert {"AB2_OK", "AB2_SPMV_CSR_VECTOR", "AB2_PC_NEUMANN", "AB2_ERR_TIMEOUT"} <= defs.keys()
    mismatched = {n: (v, binding_value(n)) for n, v in defs.items() if binding_value(n) != v}
    assert not mismatched


def test_binding_tables_hold_nothing_the_headers_lack():
    defs = header_defines()
    assert sorted(set(abi.PRECOND.values())) == sorted(v for n, v in defs.items() if n.startswith("AB2_PC_"))
    assert sorted(set(abi.ILU_SCHEDULE.values())) == sorted(v for n, v in defs.items() if n.startswith("AB2_ILU_"))
    assert sorted(set(abi.SOLVER.values())) == sorted(v for n, v in defs.items() if n.startswith("AB2_SOLVER_"))
    spmv = sorted(v for n, v in defs.items() if n.startswith("AB2_SPMV_"))
    assert spmv == sorted(getattr(abi, n) for n in dir(abi) if n.startswith("SPMV_"))
