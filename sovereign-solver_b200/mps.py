"""MPS reader: ``sov::read_mps_string`` / ``sov::read_mps`` (include/sovereign/io.hpp:14-66).

The parsing runs in the engine library (``pdhg_read_mps``, csrc/mps_reader.cpp),
host threads over the text; this module copies the model into a ``Problem``
plus what the reference's ``ReadResult`` carries besides (names, integrality,
warnings). A malformed model raises ``MpsError`` with the reference's message.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional, Union

import numpy as np

from . import pdhg as _pdhg
from .problem import Problem


class MpsError(ValueError):
    """``sov::Error`` thrown by the reference reader: the same text."""


class _MpsOptions(C.Structure):
    _fields_ = [("negative_upper_bound", C.c_int), ("keep_free_rows", C.c_int),
                ("threads", C.c_int)]


class _ModelInfo(C.Structure):
    _fields_ = [("m", C.c_int32), ("n", C.c_int32), ("nnz", C.c_int64), ("obj_const", C.c_double),
                ("maximize", C.c_int), ("warnings", C.c_int32), ("fixed_format", C.c_int)]


@dataclass
class MpsModel:
    """``sov::ReadResult``: the problem and what the file said besides."""
    problem: Problem
    name: str = ""
    objective_name: str = ""
    row_names: list = field(default_factory=list)
    col_names: list = field(default_factory=list)
    is_integer: np.ndarray = field(default_factory=lambda: np.zeros(0, dtype=bool))
    warnings: list = field(default_factory=list)  # (line, section, message)
    fixed_format: bool = False


_declared = False


def _lib() -> C.CDLL:
    global _declared
    L = _pdhg.lib()
    if not _declared:
        vp, cp, dp = C.c_void_p, C.c_char_p, C.POINTER(C.POINTER(C.c_double))
        L.pdhg_read_mps.argtypes = [cp, C.c_size_t, cp, C.POINTER(_MpsOptions),
                                    C.POINTER(vp), cp, C.c_size_t]
        L.pdhg_read_mps_file.argtypes = [cp, C.POINTER(_MpsOptions), C.POINTER(vp), cp, C.c_size_t]
        L.pdhg_model_free.argtypes = [vp]
        L.pdhg_model_get_info.argtypes = [vp, C.POINTER(_ModelInfo)]
        ip = C.POINTER(C.POINTER(C.c_int32))
        L.pdhg_model_arrays.argtypes = [vp, ip, ip, dp, dp, dp, dp, dp, dp,
                                        C.POINTER(C.POINTER(C.c_uint8))]  # CSR, c, bounds, kinds
        for f in ("pdhg_model_name", "pdhg_model_objective_name"):
            getattr(L, f).argtypes = [vp]
            getattr(L, f).restype = cp
        for f in ("pdhg_model_row_name", "pdhg_model_col_name"):
            getattr(L, f).argtypes = [vp, C.c_int32]
            getattr(L, f).restype = cp
        L.pdhg_model_warning.argtypes = [vp, C.c_int32, C.POINTER(C.c_int64), C.POINTER(cp),
                                         C.POINTER(cp)]
        L.pdhg_model_name_table.argtypes = [vp, C.c_int, C.POINTER(C.c_void_p),
                                            C.POINTER(C.POINTER(C.c_int64))]
        _declared = True
    return L


def _options(negative_upper_bound: str, keep_free_rows: bool, threads: int) -> _MpsOptions:
    rules = {"minus_infinity": 0, "keep_lower_at_zero": 1}
    if negative_upper_bound not in rules:
        raise ValueError(f"negative_upper_bound must be one of {sorted(rules)}")
    return _MpsOptions(rules[negative_upper_bound], int(bool(keep_free_rows)), int(threads))


def _names(L, h, columns: bool, count: int) -> list:
    if count == 0:
        return []
    chars, off = C.c_void_p(), C.POINTER(C.c_int64)()
    L.pdhg_model_name_table(h, int(columns), C.byref(chars), C.byref(off))
    raw = C.string_at(chars, off[count])
    names = raw[:-1].split(b"\0")
    if len(names) != count:  # a name with a NUL byte in it: cut by the offsets
        names = [raw[off[k]:off[k + 1] - 1] for k in range(count)]
    return [x.decode(errors="surrogateescape") for x in names]


def _collect(L, h) -> MpsModel:
    info = _ModelInfo()
    L.pdhg_model_get_info(h, C.byref(info))
    m, n, nnz = info.m, info.n, info.nnz
    ptrs = [C.POINTER(C.c_int32)(), C.POINTER(C.c_int32)()] + \
        [C.POINTER(C.c_double)() for _ in range(6)] + [C.POINTER(C.c_uint8)()]
    L.pdhg_model_arrays(h, *[C.byref(p) for p in ptrs])

    def arr(p, k, dtype):
        if k == 0:
            return np.zeros(0, dtype=dtype)
        return np.ctypeslib.as_array(p, shape=(k,)).astype(dtype, copy=True)

    prob = Problem(m=m, n=n, row_ptr=arr(ptrs[0], m + 1, np.int32), col_idx=arr(ptrs[1], nnz, np.int32),
                   val=arr(ptrs[2], nnz, np.float64), c=arr(ptrs[3], n, np.float64),
                   col_lo=arr(ptrs[4], n, np.float64), col_hi=arr(ptrs[5], n, np.float64),
                   row_lo=arr(ptrs[6], m, np.float64), row_hi=arr(ptrs[7], m, np.float64),
                   obj_const=info.obj_const, maximize=bool(info.maximize),
                   name=L.pdhg_model_name(h).decode())
    warnings = []
    for k in range(info.warnings):
        line, sec, msg = C.c_int64(), C.c_char_p(), C.c_char_p()
        L.pdhg_model_warning(h, k, C.byref(line), C.byref(sec), C.byref(msg))
        warnings.append((line.value, sec.value.decode(), msg.value.decode()))
    return MpsModel(problem=prob, name=prob.name,
                    objective_name=L.pdhg_model_objective_name(h).decode(),
                    row_names=_names(L, h, False, m), col_names=_names(L, h, True, n),
                    is_integer=arr(ptrs[8], n, np.uint8).astype(bool), warnings=warnings,
                    fixed_format=bool(info.fixed_format))


def _finish(L, rc: int, h: C.c_void_p, err) -> MpsModel:
    if rc != 0:
        raise MpsError(err.value.decode(errors="replace"))
    try:
        return _collect(L, h)
    finally:
        L.pdhg_model_free(h)


def read_mps(text: Union[str, bytes], origin: Optional[str] = None, *,
             negative_upper_bound: str = "minus_infinity", keep_free_rows: bool = True,
             threads: int = 0) -> MpsModel:
    """``read_mps_string(text, MpsOptions, origin)`` (io.hpp:57-58)."""
    L = _lib()
    data = text.encode() if isinstance(text, str) else bytes(text)
    o = _options(negative_upper_bound, keep_free_rows, threads)
    h, err = C.c_void_p(), C.create_string_buffer(4096)
    rc = L.pdhg_read_mps(data, len(data), origin.encode() if origin is not None else None,
                         C.byref(o), C.byref(h), err, len(err))
    return _finish(L, rc, h, err)


def read_mps_file(path: str, *, negative_upper_bound: str = "minus_infinity",
                  keep_free_rows: bool = True, threads: int = 0) -> MpsModel:
    """``read_mps(path, MpsOptions)`` (io.hpp:55-56)."""
    L = _lib()
    o = _options(negative_upper_bound, keep_free_rows, threads)
    h, err = C.c_void_p(), C.create_string_buffer(4096)
    rc = L.pdhg_read_mps_file(str(path).encode(), C.byref(o), C.byref(h), err, len(err))
    return _finish(L, rc, h, err)


def write_mps(p: Problem, name: str = "") -> str:
    """``p`` as free MPS text that ``read_mps`` (and the reference's reader)
    turns back into ``p``: rows ``R<i>``, columns ``C<j>``, objective ``OBJ``,
    numbers in their shortest round-trip spelling. A row with two different
    finite ends becomes an E row at its lower end with the range hi - lo,
    which reproduces hi up to that one subtraction's rounding."""
    rp, ci, va = p.row_ptr, p.col_idx, p.val
    m, n = p.m, p.n
    out = [f"NAME {name or p.name or 'MODEL'}"]
    if p.maximize:
        out.append("OBJSENSE MAX")
    out += ["ROWS", " N OBJ"]
    lo, hi = p.row_lo, p.row_hi
    kind = []
    for i in range(m):
        a, b = lo[i], hi[i]
        if a == b:
            k = "E"
        elif np.isinf(a) and np.isinf(b):
            k = "N"
        elif np.isinf(a):
            k = "L"
        elif np.isinf(b):
            k = "G"
        else:
            k = "R"  # E row + range
        kind.append(k)
        out.append(f" {'E' if k == 'R' else k} R{i}")
    out.append("COLUMNS")
    # column-major order of the entries (a stable counting sort by column)
    rows = np.repeat(np.arange(m, dtype=np.int64), np.diff(rp))
    order = np.argsort(ci, kind="stable")
    cs, rs, vs = ci[order], rows[order], va[order]
    starts = np.searchsorted(cs, np.arange(n + 1))
    c = p.c
    for j in range(n):
        if c[j] != 0.0:
            out.append(f"    C{j} OBJ {float(c[j])!r}")
        for k in range(starts[j], starts[j + 1]):
            out.append(f"    C{j} R{rs[k]} {float(vs[k])!r}")
        if c[j] == 0.0 and starts[j] == starts[j + 1]:
            out.append(f"    C{j} OBJ 0")
    out.append("RHS")
    if p.obj_const != 0.0:
        out.append(f"    RHS OBJ {float(-p.obj_const)!r}")
    for i, k in enumerate(kind):
        v = {"E": lo[i], "R": lo[i], "L": hi[i], "G": lo[i]}.get(k)
        if v is not None and v != 0.0:
            out.append(f"    RHS R{i} {float(v)!r}")
    if "R" in kind:
        out.append("RANGES")
        for i, k in enumerate(kind):
            if k == "R":
                out.append(f"    RNG R{i} {float(hi[i] - lo[i])!r}")
    out.append("BOUNDS")
    cl, ch = p.col_lo, p.col_hi
    for j in range(n):
        a, b = cl[j], ch[j]
        if a == 0.0 and np.isposinf(b):
            continue
        if a == b:
            out.append(f" FX BND C{j} {float(a)!r}")
            continue
        if np.isneginf(a):
            out.append(f" {'FR' if np.isposinf(b) else 'MI'} BND C{j}")
        elif a != 0.0:
            out.append(f" LO BND C{j} {float(a)!r}")
        if not np.isposinf(b):
            out.append(f" UP BND C{j} {float(b)!r}")
    out.append("ENDATA")
    return "\n".join(out) + "\n"
