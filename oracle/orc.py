"""ctypes face of the checkers -- TEST INFRASTRUCTURE ONLY.

Loads ``oracle/liborc_pdhg.so`` (the C restatement, pdhg_oracle.c) and, when
present, ``oracle/_ref/libsovref.so`` (the reference PDHG path compiled from the
reference sources by oracle/Makefile). Only the tests, ``__graft_entry__.smoke``
and ``bench.py``'s CPU-baseline leg import this module; the engine never does.

Every entry takes any object with the ``Problem`` attributes (m, n, row_ptr,
col_idx, val, c, col_lo, col_hi, row_lo, row_hi, obj_const, maximize).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORC_SO = os.path.join(HERE, "liborc_pdhg.so")
REF_SO = os.path.join(HERE, "_ref", "libsovref.so")

STATUS = ["optimal", "iteration_limit", "time_limit", "numerical_failure", "not_solved",
          "cancelled"]

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
CHECKPOINT_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_longlong, _dp, _dp, C.c_double)


class OrcProblem(C.Structure):
    _fields_ = [("m", C.c_int32), ("n", C.c_int32), ("nnz", C.c_int64),
                ("row_ptr", _ip), ("col_idx", _ip), ("val", _dp), ("c", _dp),
                ("obj_const", C.c_double), ("maximize", C.c_int),
                ("col_lo", _dp), ("col_hi", _dp), ("row_lo", _dp), ("row_hi", _dp)]


class OrcOptions(C.Structure):
    _fields_ = [("tolerance", C.c_double), ("max_iterations", C.c_longlong),
                ("time_limit_seconds", C.c_double), ("restart_check_period", C.c_longlong),
                ("restart_sufficient_decrease", C.c_double), ("step_size_safety", C.c_double),
                ("power_iterations", C.c_int), ("verbose", C.c_int),
                ("ruiz_iterations", C.c_int), ("ruiz_tolerance", C.c_double),
                ("pock_chambolle_alpha", C.c_double), ("apply_ruiz", C.c_int),
                ("apply_pock_chambolle", C.c_int), ("termination_rule", C.c_int),
                ("trace_iters", C.c_int), ("trace_x", _dp), ("trace_y", _dp),
                ("checkpoint", CHECKPOINT_FN), ("checkpoint_user", C.c_void_p),
                ("cancel_flag", C.POINTER(C.c_int)), ("iter_times", _dp),
                ("iter_times_cap", C.c_longlong), ("restart_rule", C.c_int),
                ("primal_weight_update", C.c_int), ("halpern", C.c_int),
                ("x0", _dp), ("y0", _dp), ("primal_weight0", C.c_double)]


class OrcInfo(C.Structure):
    _fields_ = [("status", C.c_int), ("objective", C.c_double),
                ("primal_infeasibility", C.c_double), ("dual_infeasibility", C.c_double),
                ("duality_gap", C.c_double), ("iterations", C.c_longlong),
                ("restarts", C.c_longlong), ("seconds", C.c_double),
                ("operator_norm_estimate", C.c_double), ("has_point", C.c_int),
                ("message", C.c_char * 256), ("relative_kkt", C.c_double),
                ("primal_weight", C.c_double)]


@dataclass
class Result:
    status: str
    objective: float
    primal: np.ndarray | None
    dual: np.ndarray | None
    reduced_costs: np.ndarray | None
    primal_infeasibility: float
    dual_infeasibility: float
    duality_gap: float
    iterations: int
    restarts: int
    seconds: float
    operator_norm_estimate: float
    message: str
    trace_x: np.ndarray | None = None
    trace_y: np.ndarray | None = None
    checkpoints: list = field(default_factory=list)
    loop_seconds: float = 0.0
    loop_iterations: int = 0
    relative_kkt: float = 0.0
    primal_weight: float = 1.0


_libs: dict = {}


def _lib(path: str) -> C.CDLL:
    if path not in _libs:
        if not os.path.exists(path):
            raise FileNotFoundError(f"checker library not built: {path} (run make -C oracle)")
        lib = C.CDLL(path)
        _libs[path] = lib
    return _libs[path]


def orc_lib() -> C.CDLL:
    lib = _lib(ORC_SO)
    lib.orc_pdhg_solve.argtypes = [C.POINTER(OrcProblem), C.POINTER(OrcOptions),
                                   C.POINTER(OrcInfo), _dp, _dp, _dp]
    lib.orc_default_options.argtypes = [C.POINTER(OrcOptions)]
    lib.orc_scaling.argtypes = [C.c_int32, C.c_int32, _ip, _ip, _dp, C.POINTER(OrcOptions),
                                _dp, _dp]
    lib.orc_spmv.argtypes = [C.c_int32, _ip, _ip, _dp, C.c_double, _dp, C.c_double, _dp]
    lib.orc_spmv_transpose.argtypes = [C.c_int32, C.c_int32, _ip, _ip, _dp, C.c_double, _dp,
                                       C.c_double, _dp]
    lib.orc_project_box.argtypes = [C.c_int32, _dp, _dp, _dp]
    lib.orc_pairwise_dot.argtypes = [_dp, _dp, C.c_int64]
    lib.orc_pairwise_dot.restype = C.c_double
    lib.orc_operator_norm.argtypes = [C.c_int32, C.c_int32, _ip, _ip, _dp, C.c_int]
    lib.orc_operator_norm.restype = C.c_double
    return lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib() -> C.CDLL:
    lib = _lib(REF_SO)
    lib.ref_pdhg_solve.argtypes = [C.POINTER(OrcProblem), C.POINTER(OrcOptions),
                                   C.POINTER(OrcInfo), _dp, _dp, _dp, _dp]
    lib.ref_scaling.argtypes = [C.c_int32, C.c_int32, C.c_int64, _ip, _ip, _dp,
                                C.POINTER(OrcOptions), _dp, _dp]
    lib.ref_backend_spmv.argtypes = [C.c_int, C.c_int32, C.c_int32, C.c_int64, _ip, _ip, _dp,
                                     C.c_double, _dp, C.c_double, _dp]
    lib.ref_read_model_string.argtypes = [C.c_char_p, C.c_int]
    lib.ref_read_model_string.restype = C.c_void_p
    lib.ref_model_shape.argtypes = [C.c_void_p, _ip, _ip, C.POINTER(C.c_int64),
                                    C.POINTER(C.c_int), _dp]
    lib.ref_model_arrays.argtypes = [C.c_void_p, _ip, _ip, _dp, _dp, _dp, _dp, _dp, _dp]
    lib.ref_model_free.argtypes = [C.c_void_p]
    lib.ref_certifies.argtypes = [C.POINTER(OrcProblem), _dp, C.c_double, _dp]
    return lib


def _d(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _i(a: np.ndarray):
    return a.ctypes.data_as(_ip)


def _problem(p, keep: list) -> OrcProblem:
    arrs = {}
    for f in ("row_ptr", "col_idx"):
        arrs[f] = np.ascontiguousarray(getattr(p, f), dtype=np.int32)
    for f in ("val", "c", "col_lo", "col_hi", "row_lo", "row_hi"):
        a = np.ascontiguousarray(getattr(p, f), dtype=np.float64)
        arrs[f] = a if a.size else np.zeros(1)
    if arrs["col_idx"].size == 0:
        arrs["col_idx"] = np.zeros(1, dtype=np.int32)
    keep.append(arrs)
    return OrcProblem(int(p.m), int(p.n), int(np.asarray(p.row_ptr)[-1]), _i(arrs["row_ptr"]),
                      _i(arrs["col_idx"]), _d(arrs["val"]), _d(arrs["c"]), float(p.obj_const),
                      int(bool(p.maximize)), _d(arrs["col_lo"]), _d(arrs["col_hi"]),
                      _d(arrs["row_lo"]), _d(arrs["row_hi"]))


def make_options(**kw) -> OrcOptions:
    o = OrcOptions()
    orc_lib().orc_default_options(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise KeyError(k)
        setattr(o, k, v)
    return o


def _solve(which: str, p, trace_iters: int = 0, checkpoints: bool = False,
           cancel: bool = False, iter_times: np.ndarray | None = None, **kw) -> Result:
    keep: list = []
    prob = _problem(p, keep)
    starts = {k: kw.pop(k) for k in ("x0", "y0") if k in kw}
    o = make_options(**kw)
    for k, v in starts.items():  # warm start arrays (original units), kept alive
        if v is not None:
            a = np.ascontiguousarray(v, dtype=np.float64)
            keep.append(a)
            setattr(o, k, _d(a))
    if iter_times is not None:
        o.iter_times = _d(iter_times)
        o.iter_times_cap = int(iter_times.size)
    tx = ty = None
    if trace_iters > 0:
        tx = np.zeros((trace_iters, max(p.n, 1)))
        ty = np.zeros((trace_iters, max(p.m, 1)))
        o.trace_iters = trace_iters
        o.trace_x = _d(tx)
        o.trace_y = _d(ty)
    cps: list = []
    if checkpoints:
        def cb(_user, it, xp, yp, res):
            x = np.ctypeslib.as_array(xp, shape=(p.n,)).copy() if p.n else np.zeros(0)
            y = np.ctypeslib.as_array(yp, shape=(p.m,)).copy() if p.m else np.zeros(0)
            cps.append((int(it), x, y, float(res)))
        cfn = CHECKPOINT_FN(cb)
        keep.append(cfn)
        o.checkpoint = cfn
    flag = C.c_int(1 if cancel else 0)
    if cancel:
        o.cancel_flag = C.pointer(flag)
    info = OrcInfo()
    x = np.zeros(max(p.n, 1))
    y = np.zeros(max(p.m, 1))
    rc = np.zeros(max(p.n, 1))
    loop = np.zeros(2)
    if which == "oracle":
        orc_lib().orc_pdhg_solve(C.byref(prob), C.byref(o), C.byref(info), _d(x), _d(y), _d(rc))
    else:
        rcode = ref_lib().ref_pdhg_solve(C.byref(prob), C.byref(o), C.byref(info), _d(x), _d(y),
                                         _d(rc), _d(loop))
        if rcode != 0:
            raise RuntimeError(info.message.decode())
    hp = bool(info.has_point)
    return Result(
        status=STATUS[info.status], objective=info.objective,
        primal=x[: p.n].copy() if hp else None, dual=y[: p.m].copy() if hp else None,
        reduced_costs=rc[: p.n].copy() if hp else None,
        primal_infeasibility=info.primal_infeasibility,
        dual_infeasibility=info.dual_infeasibility, duality_gap=info.duality_gap,
        iterations=info.iterations, restarts=info.restarts, seconds=info.seconds,
        operator_norm_estimate=info.operator_norm_estimate, message=info.message.decode(),
        trace_x=None if tx is None else tx[:, : p.n], trace_y=None if ty is None else ty[:, : p.m],
        checkpoints=cps, loop_seconds=float(loop[0]), loop_iterations=int(loop[1]),
        relative_kkt=float(info.relative_kkt), primal_weight=float(info.primal_weight))


def oracle_solve(p, **kw) -> Result:
    """The C restatement of ``Pdhg::solve`` (src/l1/pdhg.cpp:218-502)."""
    return _solve("oracle", p, **kw)


def reference_solve(p, **kw) -> Result:
    """The reference's own ``sov::Pdhg::solve`` on its Host backend."""
    return _solve("reference", p, **kw)


def oracle_scaling(p, **kw):
    rs = np.zeros(max(p.m, 1))
    cs = np.zeros(max(p.n, 1))
    keep: list = []
    prob = _problem(p, keep)
    o = make_options(**kw)
    orc_lib().orc_scaling(prob.m, prob.n, prob.row_ptr, prob.col_idx, prob.val, C.byref(o),
                          _d(rs), _d(cs))
    return rs[: p.m], cs[: p.n]


def reference_scaling(p, **kw):
    rs = np.zeros(max(p.m, 1))
    cs = np.zeros(max(p.n, 1))
    keep: list = []
    prob = _problem(p, keep)
    o = make_options(**kw)
    if ref_lib().ref_scaling(prob.m, prob.n, prob.nnz, prob.row_ptr, prob.col_idx, prob.val,
                             C.byref(o), _d(rs), _d(cs)) != 0:
        raise RuntimeError("reference scaling failed")
    return rs[: p.m], cs[: p.n]


def oracle_spmv(p, alpha, x, beta, y, transpose=False):
    keep: list = []
    prob = _problem(p, keep)
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.array(y, dtype=np.float64)
    if transpose:
        orc_lib().orc_spmv_transpose(prob.m, prob.n, prob.row_ptr, prob.col_idx, prob.val,
                                     alpha, _d(x), beta, _d(y))
    else:
        orc_lib().orc_spmv(prob.m, prob.row_ptr, prob.col_idx, prob.val, alpha, _d(x), beta,
                           _d(y))
    return y


def reference_spmv(p, alpha, x, beta, y, transpose=False):
    keep: list = []
    prob = _problem(p, keep)
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.array(y, dtype=np.float64)
    if ref_lib().ref_backend_spmv(int(transpose), prob.m, prob.n, prob.nnz, prob.row_ptr,
                                  prob.col_idx, prob.val, alpha, _d(x), beta, _d(y)) != 0:
        raise RuntimeError("reference spmv failed")
    return y


def oracle_operator_norm(p, iterations=30) -> float:
    keep: list = []
    prob = _problem(p, keep)
    return orc_lib().orc_operator_norm(prob.m, prob.n, prob.row_ptr, prob.col_idx, prob.val,
                                       iterations)


def reference_read_model(text: str, is_mps: bool = False) -> dict:
    """read_lp_string / read_mps_string (include/sovereign/io.hpp:57-64) -> CSR arrays."""
    lib = ref_lib()
    h = lib.ref_read_model_string(text.encode(), int(is_mps))
    if not h:
        raise ValueError("reference reader rejected the model")
    m, n, nnz, mx, oc = C.c_int32(), C.c_int32(), C.c_int64(), C.c_int(), C.c_double()
    lib.ref_model_shape(h, C.byref(m), C.byref(n), C.byref(nnz), C.byref(mx), C.byref(oc))
    rp = np.zeros(m.value + 1, dtype=np.int32)
    ci = np.zeros(max(nnz.value, 1), dtype=np.int32)
    va = np.zeros(max(nnz.value, 1))
    c = np.zeros(max(n.value, 1))
    cl = np.zeros(max(n.value, 1))
    ch = np.zeros(max(n.value, 1))
    rl = np.zeros(max(m.value, 1))
    rh = np.zeros(max(m.value, 1))
    lib.ref_model_arrays(h, _i(rp), _i(ci), _d(va), _d(c), _d(cl), _d(ch), _d(rl), _d(rh))
    lib.ref_model_free(h)
    k, nn, mm = nnz.value, n.value, m.value
    return {"m": mm, "n": nn, "row_ptr": rp, "col_idx": ci[:k], "val": va[:k], "c": c[:nn],
            "col_lo": cl[:nn], "col_hi": ch[:nn], "row_lo": rl[:mm], "row_hi": rh[:mm],
            "obj_const": oc.value, "maximize": bool(mx.value)}


def _certifies(which: str, p, y, slack: float = 1e-6):
    keep: list = []
    prob = _problem(p, keep)
    yv = np.ascontiguousarray(np.asarray(y, dtype=np.float64))
    ranges = np.zeros(4)
    if which == "oracle":
        lib = orc_lib()
        lib.orc_certifies.argtypes = [C.POINTER(OrcProblem), _dp, C.c_double, _dp]
        ok = lib.orc_certifies(C.byref(prob), _d(yv), slack, _d(ranges))
    else:
        ok = ref_lib().ref_certifies(C.byref(prob), _d(yv), slack, _d(ranges))
        if ok < 0:
            raise RuntimeError("ref_certifies raised")
    return bool(ok), ranges


def oracle_certifies(p, y, slack: float = 1e-6):
    """FarkasCertificate{y}.certifies_infeasibility(p, slack) restated
    (src/l1/duals.cpp:16-79): (certified, [row lo, row hi, col lo, col hi])."""
    return _certifies("oracle", p, y, slack)


def reference_certifies(p, y, slack: float = 1e-6):
    """The reference's own FarkasCertificate checker (compiled duals.cpp)."""
    return _certifies("reference", p, y, slack)


def ray_certifies(p, d, eps: float = 1e-6):
    """The engine's ray test for dual infeasibility, restated in numpy. It has
    no reference counterpart: the reference's PDHG never reports an outcome
    other than those of sov::PdhgStatus (pdhg.hpp:74-81), and its simplex
    reports Unbounded (simplex.hpp:42) without a ray. d, scaled to max |d_j| = 1,
    certifies when c^T d < 0 in the minimize sense and d and A d leave the
    recession cones of the column and row bounds (a finite lower end allows no
    decrease, a finite upper end no increase) by at most eps and eps |c^T d|.
    Returns (certified, c^T d, violation), both for the scaled d."""
    d = np.asarray(d, dtype=np.float64)
    big = np.max(np.abs(d)) if d.size else 0.0
    if not np.isfinite(big) or big == 0.0:
        return False, float("nan"), float("nan")
    d = d / big
    rp = np.asarray(p.row_ptr, dtype=np.int64)
    ci = np.asarray(p.col_idx, dtype=np.int64)
    val = np.asarray(p.val, dtype=np.float64)
    rows = np.repeat(np.arange(p.m), np.diff(rp))
    ad = np.zeros(p.m)
    np.add.at(ad, rows, val * d[ci])
    sign = -1.0 if p.maximize else 1.0
    obj = float(sign * np.dot(np.asarray(p.c, dtype=np.float64), d))

    def cone(v, lo, hi):
        lo = np.asarray(lo, dtype=np.float64)
        hi = np.asarray(hi, dtype=np.float64)
        down = np.where((v < 0) & np.isfinite(lo), -v, 0.0)
        up = np.where((v > 0) & np.isfinite(hi), v, 0.0)
        return float(max(down.max(initial=0.0), up.max(initial=0.0)))

    viol = max(cone(d, p.col_lo, p.col_hi), cone(ad, p.row_lo, p.row_hi))
    ok = obj < 0.0 and viol <= eps and viol <= eps * -obj
    return ok, obj, viol


def reference_read_mps(text, origin: str = "<string>", keep_lower_at_zero: bool = False,
                       keep_free_rows: bool = True) -> dict:
    """The reference's own read_mps_string(text, MpsOptions, origin)
    (src/io/mps_reader.cpp:506-533) -> the model's arrays, names, integrality
    and warnings; {"error": message} when it throws."""
    lib = ref_lib()
    if not getattr(lib, "_mps_declared", False):
        vp = C.c_void_p
        lib.ref_read_mps.argtypes = [C.c_char_p, C.c_size_t, C.c_char_p, C.c_int, C.c_int,
                                     C.c_char_p, C.c_size_t]
        lib.ref_read_mps.restype = vp
        lib.ref_model_kinds.argtypes = [vp, C.POINTER(C.c_uint8)]
        for f in ("ref_model_name", "ref_model_objective_name"):
            getattr(lib, f).argtypes = [vp]
            getattr(lib, f).restype = C.c_char_p
        for f in ("ref_model_row_name", "ref_model_col_name"):
            getattr(lib, f).argtypes = [vp, C.c_int32]
            getattr(lib, f).restype = C.c_char_p
        lib.ref_model_n_warnings.argtypes = [vp]
        lib.ref_model_n_warnings.restype = C.c_int32
        lib.ref_model_warning.argtypes = [vp, C.c_int32, C.POINTER(C.c_int64),
                                          C.POINTER(C.c_char_p), C.POINTER(C.c_char_p)]
        lib._mps_declared = True
    data = text.encode() if isinstance(text, str) else bytes(text)
    err = C.create_string_buffer(4096)
    h = lib.ref_read_mps(data, len(data), origin.encode(), int(keep_lower_at_zero),
                         int(keep_free_rows), err, len(err))
    if not h:
        return {"error": err.value.decode(errors="replace")}
    try:
        m, n, nnz, mx, oc = C.c_int32(), C.c_int32(), C.c_int64(), C.c_int(), C.c_double()
        lib.ref_model_shape(h, C.byref(m), C.byref(n), C.byref(nnz), C.byref(mx), C.byref(oc))
        M, N, K = m.value, n.value, nnz.value
        rp = np.zeros(M + 1, dtype=np.int32)
        ci = np.zeros(max(K, 1), dtype=np.int32)
        va = np.zeros(max(K, 1))
        c, cl, ch = np.zeros(max(N, 1)), np.zeros(max(N, 1)), np.zeros(max(N, 1))
        rl, rh = np.zeros(max(M, 1)), np.zeros(max(M, 1))
        lib.ref_model_arrays(h, _i(rp), _i(ci), _d(va), _d(c), _d(cl), _d(ch), _d(rl), _d(rh))
        kinds = np.zeros(max(N, 1), dtype=np.uint8)
        lib.ref_model_kinds(h, kinds.ctypes.data_as(C.POINTER(C.c_uint8)))
        warnings = []
        for k in range(lib.ref_model_n_warnings(h)):
            line, sec, msg = C.c_int64(), C.c_char_p(), C.c_char_p()
            lib.ref_model_warning(h, k, C.byref(line), C.byref(sec), C.byref(msg))
            warnings.append((line.value, sec.value.decode(), msg.value.decode()))
        return {"m": M, "n": N, "row_ptr": rp, "col_idx": ci[:K], "val": va[:K], "c": c[:N],
                "col_lo": cl[:N], "col_hi": ch[:N], "row_lo": rl[:M], "row_hi": rh[:M],
                "obj_const": oc.value, "maximize": bool(mx.value),
                "is_integer": kinds[:N].astype(bool),
                "name": lib.ref_model_name(h).decode(),
                "objective_name": lib.ref_model_objective_name(h).decode(),
                "row_names": [lib.ref_model_row_name(h, i).decode() for i in range(M)],
                "col_names": [lib.ref_model_col_name(h, j).decode() for j in range(N)],
                "warnings": warnings}
    finally:
        lib.ref_model_free(h)
