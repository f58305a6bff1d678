"""The C ABI: header prototypes, exported symbols, no-GPU failure mode (CPU)."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

from lfric_core_b200 import _lib

ROOT = Path(__file__).resolve().parent.parent


def test_header_parses_every_entry_point():
    protos = _lib.parse_header()
    declared = set(re.findall(r"\b(lfg_\w+)\s*\(", re.sub(r"/\*.*?\*/", "", _lib.HEADER.read_text(), flags=re.S)))
    assert declared == set(protos)
    assert len(protos) >= 60


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    for name in _lib.parse_header():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True,
                         text=True, check=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T lfg_" in l}
    assert exported == set(_lib.parse_header())


def test_version_and_null_handles():
    lib = _lib.load()
    assert b"sm_100a" in lib.lfg_version()
    assert lib.lfg_last_error(None) == b"null context"
    assert lib.lfg_ctx_synchronize(None) == 3          # LFG_ERR_ARG
    assert lib.lfg_field_import(None, None, 8) == 3
    assert lib.lfg_solver_apply(None, None, None, None, None) == 3


def test_python_constants_match_the_header():
    """The Python front end's kinds, statuses and solver methods carry the
    header's values (the Fortran binding reads the same header)."""
    from lfric_core_b200 import api
    text = _lib.HEADER.read_text()
    defs = {m.group(1): int(m.group(2))
            for m in re.finditer(r"#define\s+(LFG_\w+)\s+(\d+)\b", text)}
    assert (api.R_SINGLE, api.R_DOUBLE) == (defs["LFG_R_SINGLE"], defs["LFG_R_DOUBLE"])
    assert (api.OK, api.NOT_CONVERGED, api.NAN_STATUS) == (
        defs["LFG_OK"], defs["LFG_NOT_CONVERGED"], defs["LFG_NAN"])
    solvers = {k[len("LFG_SOLVER_"):].lower(): v for k, v in defs.items()
               if k.startswith("LFG_SOLVER_")}
    assert solvers == api.SOLVERS
