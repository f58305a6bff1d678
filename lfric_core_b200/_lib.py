"""ctypes binding of the C ABI in include/lfg.h (liblfg.so, built in-tree).

The prototypes are read from the header itself, so the binding cannot drift
from the ABI.  Loading fails loudly when the shared library is missing or no
CUDA device is present: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
HEADER = ROOT / "include" / "lfg.h"
LIB_PATH = PKG / "liblfg.so"


class lfg_solver_cfg(C.Structure):
    _fields_ = [("method", C.c_int), ("gcrk", C.c_int), ("r_tol", C.c_double),
                ("a_tol", C.c_double), ("max_iter", C.c_int),
                ("monitor_convergence", C.c_int), ("fail_on_non_converged", C.c_int),
                ("rho_relax", C.c_double), ("lmin", C.c_double), ("lmax", C.c_double)]


class lfg_batch_cfg(C.Structure):
    _fields_ = [("tol", C.c_double), ("inner_tol", C.c_double), ("max_outer", C.c_int),
                ("max_inner", C.c_int), ("tile_cols", C.c_int), ("blocks_per_sm", C.c_int),
                ("use_graph", C.c_int), ("spin_limit", C.c_longlong)]


def _ctype(tok: str):
    t = " ".join(tok.replace("const ", "").split())
    table = {
        "int": C.c_int, "long long": C.c_longlong, "double": C.c_double, "void*": C.c_void_p, "void *": C.c_void_p,
        "int*": C.POINTER(C.c_int), "double*": C.POINTER(C.c_double),
        "uint64_t*": C.POINTER(C.c_uint64), "int64_t*": C.POINTER(C.c_int64),
        "char*": C.c_char_p,
        "void**": C.POINTER(C.c_void_p),
        "lfg_solver_cfg*": C.POINTER(lfg_solver_cfg),
        "lfg_batch_cfg*": C.POINTER(lfg_batch_cfg),
    }
    t = t.replace(" *", "*")
    if t in table:
        return table[t]
    if re.fullmatch(r"lfg_\w+\*", t):      # out-handle or handle array
        return C.POINTER(C.c_void_p)
    if re.fullmatch(r"lfg_\w+", t):        # opaque handle
        return C.c_void_p
    raise TypeError(f"unmapped C type {tok!r}")


def parse_header(text: str | None = None) -> dict:
    """{name: (restype, [argtypes])} for every function the header declares."""
    text = HEADER.read_text() if text is None else text
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    text = re.sub(r"//[^\n]*", " ", text)
    protos = {}
    for m in re.finditer(r"(int|const char\s*\*)\s+(lfg_\w+)\s*\(([^)]*)\)\s*;", text):
        ret, name, args = m.group(1), m.group(2), m.group(3).strip()
        argtypes = []
        if args and args != "void":
            for a in args.split(","):
                a = a.strip()
                mm = re.match(r"(.*?)(\w+)$", a)
                argtypes.append(_ctype(mm.group(1).strip()))
        restype = C.c_int if ret == "int" else C.c_char_p
        protos[name] = (restype, argtypes)
    return protos


_lib = None


def load() -> C.CDLL:
    """Load liblfg.so and attach the header's prototypes (raises if absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with "
                          "`python -c 'import __graft_entry__ as g; g.build()'` "
                          "or `make -C lfric_core_b200/csrc`")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in parse_header().items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib
