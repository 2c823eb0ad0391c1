"""Python face of libpdhg_b200.so, mirroring the reference's PDHG interface.

``Pdhg(PdhgOptions(...)).solve(problem)`` -> ``PdhgResult``, with the field
names, defaults and status strings of ``sov::Pdhg`` / ``sov::PdhgOptions`` /
``sov::PdhgResult`` (include/sovereign/pdhg.hpp:74-172). Solver outcomes come
back in ``status`` + ``message`` and are never raised (pdhg.cpp:223-237,
347-371); errors of the engine itself (no GPU, CUDA failure, bad arguments)
raise ``PdhgError``, the analogue of ``sov::Error`` (status.hpp:53-63).

There is no CPU fallback: importing works anywhere, but every solve needs the
compiled library and a CUDA device, and fails loudly without them.
"""
from __future__ import annotations

import concurrent.futures
import ctypes as C
import os
from dataclasses import dataclass, field, fields
from typing import Callable, Optional

import numpy as np

from .problem import Problem

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libpdhg_b200.so")

STATUS = ["optimal", "iteration_limit", "time_limit", "numerical_failure", "not_solved",
          "cancelled", "primal_infeasible", "dual_infeasible"]
PREC = {"fp64_exact": 0, "mixed": 1, "fp64": 2}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
CHECKPOINT_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_longlong, _dp, _dp, C.c_double)


class _Options(C.Structure):
    _fields_ = [("tolerance", C.c_double), ("max_iterations", C.c_longlong),
                ("time_limit_seconds", C.c_double), ("restart_check_period", C.c_longlong),
                ("restart_sufficient_decrease", C.c_double), ("step_size_safety", C.c_double),
                ("power_iterations", C.c_int), ("verbose", C.c_int),
                ("ruiz_iterations", C.c_int), ("ruiz_tolerance", C.c_double),
                ("pock_chambolle_alpha", C.c_double), ("apply_ruiz", C.c_int),
                ("apply_pock_chambolle", C.c_int), ("precision", C.c_int),
                ("termination_rule", C.c_int), ("polish_iterations", C.c_longlong),
                ("restart_rule", C.c_int), ("primal_weight_update", C.c_int),
                ("x0", _dp), ("y0", _dp), ("checkpoint", CHECKPOINT_FN),
                ("checkpoint_user", C.c_void_p), ("cancel_flag", C.POINTER(C.c_int)),
                ("trace_iters", C.c_int), ("trace_x", _dp), ("trace_y", _dp),
                ("autotune", C.c_int), ("infeasibility_detection", C.c_int),
                ("halpern", C.c_int)]


class _Info(C.Structure):
    _fields_ = [("status", C.c_int), ("objective", C.c_double),
                ("primal_infeasibility", C.c_double), ("dual_infeasibility", C.c_double),
                ("duality_gap", C.c_double), ("iterations", C.c_longlong),
                ("restarts", C.c_longlong), ("seconds", C.c_double),
                ("operator_norm_estimate", C.c_double), ("has_point", C.c_int),
                ("message", C.c_char * 256), ("relative_kkt", C.c_double),
                ("fp64_iterations", C.c_longlong), ("kernel_launches", C.c_longlong),
                ("device_seconds", C.c_double)]


class _KStats(C.Structure):
    _fields_ = [("count", C.c_int), ("name", (C.c_char * 32) * 8), ("avg_ms", C.c_double * 8),
                ("bytes", C.c_double * 8), ("launches", C.c_int * 8)]


class PdhgError(RuntimeError):
    """An engine error (sov::Error analogue): code is a pdhg_error value."""

    def __init__(self, code: int, what: str):
        super().__init__(f"{what}: {error_string(code)}")
        self.code = code


_lib: Optional[C.CDLL] = None


def lib() -> C.CDLL:
    """The loaded engine library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise PdhgError(1, f"engine library missing: {LIB_PATH} (run __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        L.pdhg_abi_version.restype = C.c_int
        L.pdhg_default_options.argtypes = [C.POINTER(_Options)]
        L.pdhg_status_string.restype = C.c_char_p
        L.pdhg_error_string.restype = C.c_char_p
        L.pdhg_create.argtypes = [C.c_int, C.POINTER(C.c_void_p)]
        L.pdhg_destroy.argtypes = [C.c_void_p]
        L.pdhg_last_error.argtypes = [C.c_void_p]
        L.pdhg_last_error.restype = C.c_char_p
        L.pdhg_stream.argtypes = [C.c_void_p]
        L.pdhg_stream.restype = C.c_void_p
        L.pdhg_load_problem.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int64, _ip, _ip,
                                        _dp, _dp, C.c_double, C.c_int, _dp, _dp, _dp, _dp]
        L.pdhg_solve.argtypes = [C.c_void_p, C.POINTER(_Options), C.POINTER(_Info), _dp, _dp,
                                 _dp]
        L.pdhg_profile_kernels.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int,
                                           C.POINTER(_KStats)]
        L.pdhg_csr_spmv.argtypes = [C.c_int, C.c_int, C.c_int32, C.c_int32, C.c_int64, _ip, _ip,
                                    _dp, C.c_double, _dp, C.c_double, _dp]
        L.pdhg_project_box.argtypes = [C.c_int, C.c_int32, _dp, _dp, _dp]
        L.pdhg_scaling.argtypes = [C.c_int32, C.c_int32, C.c_int64, _ip, _ip, _dp,
                                   C.POINTER(_Options), _dp, _dp]
        L.pdhg_get_scaling.argtypes = [C.c_void_p, _dp, _dp]
        L.pdhg_get_tuning.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int)]
        L.pdhg_get_batch_tuning.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int)]
        L.pdhg_load_batch.argtypes = [C.c_void_p, C.c_int32, _ip, _ip, C.c_int64, _ip, _ip, _dp,
                                      _dp, _dp, C.POINTER(C.c_int), _dp, _dp, _dp, _dp]
        L.pdhg_solve_batch.argtypes = [C.c_void_p, C.POINTER(_Options), C.POINTER(_Info), _dp,
                                       _dp, _dp]
        L.pdhg_batch_start_kkt.argtypes = [C.c_void_p, _dp, _dp, _dp]
        _lib = L
    return _lib


def error_string(code: int) -> str:
    try:
        return lib().pdhg_error_string(code).decode()
    except Exception:  # library missing
        return f"error {code}"


def _check(code: int, what: str, ctx=None) -> None:
    if code != 0:
        detail = ""
        if ctx is not None:
            detail = lib().pdhg_last_error(ctx).decode()
        raise PdhgError(code, f"{what} ({detail})" if detail else what)


TERMINATION_RULES = {"absolute": 0, "relative_kkt": 1, "relative_kkt_l2": 2}
RESTART_RULES = {"reference": 0, "adaptive": 1, "adaptive_l2": 2}


@dataclass
class PdhgOptions:
    """``sov::PdhgOptions`` (pdhg.hpp:85-134) + ``ScalingOptions`` + engine extensions."""
    tolerance: float = 1e-4
    max_iterations: int = 1_000_000
    time_limit_seconds: float = 0.0
    restart_check_period: int = 40
    restart_sufficient_decrease: float = 0.5
    step_size_safety: float = 0.9
    power_iterations: int = 30
    verbose: bool = False
    ruiz_iterations: int = 8
    ruiz_tolerance: float = 1e-2
    pock_chambolle_alpha: float = 1.0
    apply_ruiz: bool = True
    apply_pock_chambolle: bool = True
    # extensions (defaults = reference behaviour)
    precision: str = "fp64_exact"
    # "absolute" (the reference's rule), "relative_kkt" (max-norm relative KKT on
    # the reference's residual terms) or "relative_kkt_l2" (PDLP's relative KKT
    # error: l2 norms, sign violations of the duals, relative gap)
    termination_rule: str = "absolute"
    polish_iterations: int = -1
    # "reference", "adaptive" (adaptive restarts on the scaled max-norm KKT
    # residual) or "adaptive_l2" (the same rule on the relative_kkt_l2 measure;
    # needs termination_rule "relative_kkt_l2")
    restart_rule: str = "reference"
    primal_weight_update: bool = False
    checkpoint: Optional[Callable[[int, np.ndarray, np.ndarray, float], None]] = None
    trace_iters: int = 0
    autotune: bool = True
    # engine extension (MIXED / FP64): stop with status "primal_infeasible" and a
    # certificate (PdhgResult.farkas) when the change of y between two checks
    # proves that no x meets the bounds, or with status "dual_infeasible" and a
    # ray (PdhgResult.ray) when the change of x between two checks is a
    # direction of unbounded descent
    infeasibility_detection: bool = False
    # engine extension (MIXED / FP64, with termination_rule "relative_kkt_l2" and
    # restart_rule "adaptive_l2"): the reflected restarted Halpern iteration
    # instead of the averaged PDHG; candidates and the reported point are the
    # PDHG step's output T(z)
    halpern: bool = False


@dataclass
class PdhgResult:
    """``sov::PdhgResult`` (pdhg.hpp:136-153) + engine extensions."""
    status: str = "not_solved"
    objective: float = 0.0
    primal: np.ndarray = field(default_factory=lambda: np.zeros(0))
    dual: np.ndarray = field(default_factory=lambda: np.zeros(0))
    reduced_costs: np.ndarray = field(default_factory=lambda: np.zeros(0))
    primal_infeasibility: float = 0.0
    dual_infeasibility: float = 0.0
    duality_gap: float = 0.0
    iterations: int = 0
    restarts: int = 0
    seconds: float = 0.0
    operator_norm_estimate: float = 0.0
    message: str = ""
    relative_kkt: float = 0.0
    fp64_iterations: int = 0
    kernel_launches: int = 0
    device_seconds: float = 0.0
    trace_x: Optional[np.ndarray] = None
    trace_y: Optional[np.ndarray] = None
    # status "primal_infeasible": the certificate's row multipliers
    # (sov::FarkasCertificate::row_multipliers, duals.hpp:47-70), max |y_i| = 1
    farkas: Optional[np.ndarray] = None
    # status "dual_infeasible": the ray d in x, max |d_j| = 1, along which the
    # objective falls without leaving the bounds (unbounded if feasible)
    ray: Optional[np.ndarray] = None


class CancellationToken:
    """``sov::CancellationToken`` (cancellation.hpp:23-30): a flag the engine polls."""

    def __init__(self) -> None:
        self._flag = C.c_int(0)

    def cancel(self) -> None:
        self._flag.value = 1

    def is_cancelled(self) -> bool:
        return bool(self._flag.value)


def _d(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _i(a: np.ndarray):
    return a.ctypes.data_as(_ip)


def _c_options(opt: PdhgOptions) -> _Options:
    o = _Options()
    lib().pdhg_default_options(C.byref(o))
    for f in fields(PdhgOptions):
        name = f.name
        val = getattr(opt, name)
        if name == "precision":
            o.precision = PREC[val]
        elif name == "termination_rule":
            o.termination_rule = TERMINATION_RULES[val] if isinstance(val, str) else int(val)
        elif name == "restart_rule":
            o.restart_rule = RESTART_RULES[val] if isinstance(val, str) else int(val)
        elif name in ("checkpoint", "trace_iters"):
            continue
        else:
            setattr(o, name, type(getattr(o, name))(val))
    return o


def _c_start(o: _Options, keep: list, cancel, x0, y0) -> None:
    """Cancellation flag and warm start into the C options (arrays kept alive in keep)."""
    if cancel is not None:
        o.cancel_flag = C.pointer(cancel._flag)
    if x0 is not None:
        x0a = np.ascontiguousarray(x0, dtype=np.float64)
        keep.append(x0a)
        o.x0 = _d(x0a)
    if y0 is not None:
        y0a = np.ascontiguousarray(y0, dtype=np.float64)
        keep.append(y0a)
        o.y0 = _d(y0a)


def _result(info: _Info, x: np.ndarray, y: np.ndarray, rc: np.ndarray,
            want_point: bool = True) -> PdhgResult:
    """The result of one solve; x, y, rc are the arrays the engine wrote (views
    into the call's own buffers, handed over without a copy). Without
    want_point nothing was written and the point fields stay empty."""
    hp = bool(info.has_point) and want_point
    farkas = want_point and STATUS[info.status] == "primal_infeasible"
    ray = want_point and STATUS[info.status] == "dual_infeasible"
    return PdhgResult(
        farkas=y if farkas else None, ray=x if ray else None,
        status=STATUS[info.status], objective=info.objective,
        primal=x if hp else np.zeros(0), dual=y if hp else np.zeros(0),
        reduced_costs=rc if hp else np.zeros(0),
        primal_infeasibility=info.primal_infeasibility,
        dual_infeasibility=info.dual_infeasibility, duality_gap=info.duality_gap,
        iterations=info.iterations, restarts=info.restarts, seconds=info.seconds,
        operator_norm_estimate=info.operator_norm_estimate,
        message=info.message.decode(), relative_kkt=info.relative_kkt,
        fp64_iterations=info.fp64_iterations, kernel_launches=info.kernel_launches,
        device_seconds=info.device_seconds)


def stack_batch(problems: list[Problem]) -> dict:
    """The block-diagonal stacking pdhg_load_batch takes: instance k's rows and
    columns follow instance k-1's; column indices become global. The output
    arrays are allocated once and filled instance by instance."""
    ms = np.array([p.m for p in problems], dtype=np.int64)
    ns = np.array([p.n for p in problems], dtype=np.int64)
    nnzs = np.array([p.nnz for p in problems], dtype=np.int64)
    row_off64 = np.concatenate([[0], np.cumsum(ms)])
    col_off64 = np.concatenate([[0], np.cumsum(ns)])
    nz_off = np.concatenate([[0], np.cumsum(nnzs)])
    if row_off64[-1] > np.iinfo(np.int32).max or col_off64[-1] > np.iinfo(np.int32).max or \
            nz_off[-1] > np.iinfo(np.int32).max:
        raise ValueError("the stacked batch does not fit int32 indices")
    m, n, nnz = int(row_off64[-1]), int(col_off64[-1]), int(nz_off[-1])
    row_ptr = np.empty(m + 1, dtype=np.int32)
    col_idx = np.empty(nnz, dtype=np.int32)
    vec = {name: np.empty(size, dtype=np.float64) for name, size in
           (("val", nnz), ("c", n), ("col_lo", n), ("col_hi", n), ("row_lo", m), ("row_hi", m))}
    def fill(ks: range) -> None:
        for k in ks:
            p = problems[k]
            r0, r1 = int(row_off64[k]), int(row_off64[k + 1])
            c0, c1 = int(col_off64[k]), int(col_off64[k + 1])
            z0, z1 = int(nz_off[k]), int(nz_off[k + 1])
            np.add(p.row_ptr[:-1], z0, out=row_ptr[r0:r1], casting="unsafe")
            np.add(p.col_idx, c0, out=col_idx[z0:z1], casting="unsafe")
            vec["val"][z0:z1] = p.val
            vec["c"][c0:c1] = p.c
            vec["col_lo"][c0:c1] = p.col_lo
            vec["col_hi"][c0:c1] = p.col_hi
            vec["row_lo"][r0:r1] = p.row_lo
            vec["row_hi"][r0:r1] = p.row_hi

    # the copies are memory-bound and numpy releases the GIL for them: the
    # instances are filled by a few threads in contiguous runs
    workers = max(1, min(16, os.cpu_count() or 1, len(problems) // 64))
    if workers == 1:
        fill(range(len(problems)))
    else:
        bounds = np.searchsorted(nz_off, np.linspace(0, nnz, workers + 1)).tolist()
        bounds[0], bounds[-1] = 0, len(problems)
        with concurrent.futures.ThreadPoolExecutor(workers) as pool:
            list(pool.map(fill, [range(bounds[i], bounds[i + 1]) for i in range(workers)]))
    row_ptr[m] = nnz
    return {"row_off": row_off64.astype(np.int32), "col_off": col_off64.astype(np.int32),
            "nnz": nnz, "row_ptr": row_ptr, "col_idx": col_idx, **vec,
            "obj_const": np.array([float(p.obj_const) for p in problems], dtype=np.float64),
            "maximize": np.array([int(bool(p.maximize)) for p in problems], dtype=np.intc)}


class Engine:
    """One engine context on one device (the analogue of one ``sov::Backend``)."""

    def __init__(self, device: int = 0) -> None:
        h = C.c_void_p()
        _check(lib().pdhg_create(device, C.byref(h)), "pdhg_create")
        self._h = h
        self.device = device
        self.problem: Optional[Problem] = None

    def stream_handle(self) -> int:
        """The cudaStream_t (as an int) the engine launches every kernel on."""
        return int(lib().pdhg_stream(self._h) or 0)

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().pdhg_destroy(self._h)
            self._h = None

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self) -> "Engine":
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    def load(self, p: Problem) -> None:
        keep = [p.row_ptr, p.col_idx, p.val, p.c, p.col_lo, p.col_hi, p.row_lo, p.row_hi]
        arrs = [np.ascontiguousarray(a) for a in keep]
        rp, ci, va, c, cl, ch, rl, rh = arrs
        if ci.size == 0:
            ci = np.zeros(1, np.int32)
            va = np.zeros(1)
        nz = lambda a: a if a.size else np.zeros(1)  # noqa: E731
        _check(lib().pdhg_load_problem(self._h, p.m, p.n, p.nnz, _i(rp), _i(ci), _d(va),
                                       _d(nz(c)), float(p.obj_const), int(bool(p.maximize)),
                                       _d(nz(cl)), _d(nz(ch)), _d(nz(rl)), _d(nz(rh))),
               "pdhg_load_problem", self._h)
        self.problem = p

    def solve(self, opt: PdhgOptions | None = None, cancel: CancellationToken | None = None,
              x0: np.ndarray | None = None, y0: np.ndarray | None = None,
              want_point: bool = True) -> PdhgResult:
        """``sov::Pdhg::solve`` (pdhg.cpp:218-502) on the loaded problem. With
        ``want_point`` False the engine downloads no point: ``primal``,
        ``dual``, ``reduced_costs``, ``farkas`` and ``ray`` stay empty and
        only the scalar fields are filled (the form timed loops use)."""
        if self.problem is None:
            raise PdhgError(3, "Engine.solve: no problem loaded")
        p = self.problem
        opt = opt or PdhgOptions()
        o = _c_options(opt)
        keep: list = []
        if opt.checkpoint is not None:
            user_cb = opt.checkpoint

            def cb(_u, it, xp, yp, res):
                xv = np.ctypeslib.as_array(xp, shape=(p.n,)).copy() if p.n else np.zeros(0)
                yv = np.ctypeslib.as_array(yp, shape=(p.m,)).copy() if p.m else np.zeros(0)
                user_cb(int(it), xv, yv, float(res))
            cfn = CHECKPOINT_FN(cb)
            keep.append(cfn)
            o.checkpoint = cfn
        _c_start(o, keep, cancel, x0, y0)
        tx = ty = None
        if opt.trace_iters > 0:
            tx = np.zeros((opt.trace_iters, max(p.n, 1)))
            ty = np.zeros((opt.trace_iters, max(p.m, 1)))
            o.trace_iters = opt.trace_iters
            o.trace_x = _d(tx)
            o.trace_y = _d(ty)
        info = _Info()
        # without want_point the engine writes no point: no host buffers of n
        k_n, k_m = (max(p.n, 1), max(p.m, 1)) if want_point else (1, 1)
        x, y, rc = np.zeros(k_n), np.zeros(k_m), np.zeros(k_n)
        null = C.cast(None, _dp)
        _check(lib().pdhg_solve(self._h, C.byref(o), C.byref(info),
                                _d(x) if want_point else null, _d(y) if want_point else null,
                                _d(rc) if want_point else null), "pdhg_solve", self._h)
        r = _result(info, x[: p.n], y[: p.m], rc[: p.n], want_point)
        if tx is not None:
            r.trace_x = tx[:, : p.n]
            r.trace_y = ty[:, : p.m]
        return r

    def load_batch(self, problems: list[Problem]) -> None:
        """Loads LPs to be solved together by ``solve_batch`` (pdhg_load_batch)."""
        b = stack_batch(problems)
        self._batch = (b, [(p.m, p.n) for p in problems])
        ci = b["col_idx"] if b["col_idx"].size else np.zeros(1, np.int32)
        va = b["val"] if b["val"].size else np.zeros(1)
        nz = lambda a: a if a.size else np.zeros(1)  # noqa: E731
        _check(lib().pdhg_load_batch(
            self._h, len(problems), _i(b["row_off"]), _i(b["col_off"]), b["nnz"],
            _i(b["row_ptr"]), _i(ci), _d(va), _d(nz(b["c"])), _d(b["obj_const"]),
            b["maximize"].ctypes.data_as(C.POINTER(C.c_int)), _d(nz(b["col_lo"])),
            _d(nz(b["col_hi"])), _d(nz(b["row_lo"])), _d(nz(b["row_hi"]))),
            "pdhg_load_batch", self._h)

    def solve_batch(self, opt: PdhgOptions | None = None,
                    cancel: CancellationToken | None = None,
                    x0: list[np.ndarray] | None = None, y0: list[np.ndarray] | None = None,
                    want_point: bool = True) -> list[PdhgResult]:
        """One ``PdhgResult`` per loaded instance (pdhg_solve_batch). Precision
        ``mixed`` (the default here) or ``fp64``; x0 / y0 are per-instance lists."""
        if getattr(self, "_batch", None) is None:
            raise PdhgError(3, "Engine.solve_batch: no batch loaded")
        b, shapes = self._batch
        opt = opt or PdhgOptions(precision="mixed")
        o = _c_options(opt)
        o.trace_iters = opt.trace_iters  # the engine rejects traces in a batch
        keep: list = []
        _c_start(o, keep, cancel, None if x0 is None else np.concatenate(x0),
                 None if y0 is None else np.concatenate(y0))
        count = len(shapes)
        infos = (_Info * count)()
        m, n = int(b["row_off"][-1]), int(b["col_off"][-1])
        k_n, k_m = (max(n, 1), max(m, 1)) if want_point else (1, 1)
        x, y, rc = np.zeros(k_n), np.zeros(k_m), np.zeros(k_n)
        null = C.cast(None, _dp)
        _check(lib().pdhg_solve_batch(self._h, C.byref(o), infos,
                                      _d(x) if want_point else null,
                                      _d(y) if want_point else null,
                                      _d(rc) if want_point else null),
               "pdhg_solve_batch", self._h)
        out = []
        for k in range(count):
            r0, r1 = int(b["row_off"][k]), int(b["row_off"][k + 1])
            c0, c1 = int(b["col_off"][k]), int(b["col_off"][k + 1])
            out.append(_result(infos[k], x[c0:c1], y[r0:r1], rc[c0:c1], want_point))
        return out

    def start_kkt(self, x0: list[np.ndarray] | None = None,
                  y0: list[np.ndarray] | None = None) -> np.ndarray:
        """Relative KKT residual of candidate starts for the loaded batch
        (pdhg_batch_start_kkt); None = the cold start."""
        if getattr(self, "_batch", None) is None:
            raise PdhgError(3, "Engine.start_kkt: no batch loaded")
        b, shapes = self._batch
        out = np.zeros(len(shapes))
        keep = []
        xs = ys = C.cast(None, _dp)
        if x0 is not None:
            xa = np.ascontiguousarray(np.concatenate(x0), dtype=np.float64)
            keep.append(xa)
            xs = _d(xa)
        if y0 is not None:
            ya = np.ascontiguousarray(np.concatenate(y0), dtype=np.float64)
            keep.append(ya)
            ys = _d(ya)
        _check(lib().pdhg_batch_start_kkt(self._h, xs, ys, _d(out)), "pdhg_batch_start_kkt",
               self._h)
        return out

    def scaling(self) -> tuple[np.ndarray, np.ndarray]:
        """Row / column factors the engine computed on the device for the loaded LP."""
        p = self.problem
        rs = np.zeros(max(p.m, 1))
        cs = np.zeros(max(p.n, 1))
        _check(lib().pdhg_get_scaling(self._h, _d(rs), _d(cs)), "pdhg_get_scaling", self._h)
        return rs[: p.m], cs[: p.n]

    def tuning(self, precision: str = "mixed") -> dict:
        """The iteration-kernel shapes in use for the loaded LP (pdhg_get_tuning)."""
        out = (C.c_int * 5)()
        _check(lib().pdhg_get_tuning(self._h, PREC[precision], out), "pdhg_get_tuning", self._h)
        return {"primal_lanes": out[0], "primal_long_mode": out[1], "dual_lanes": out[2],
                "dual_long_mode": out[3], "timed": bool(out[4])}

    def batch_tuning(self, precision: str = "mixed") -> dict:
        """Lanes per row of the batched passes for the loaded batch (pdhg_get_batch_tuning)."""
        out = (C.c_int * 3)()
        _check(lib().pdhg_get_batch_tuning(self._h, PREC[precision], out),
               "pdhg_get_batch_tuning", self._h)
        return {"primal_lanes": out[0], "dual_lanes": out[1], "timed": bool(out[2])}

    def profile_kernels(self, precision: str = "mixed", warmup: int = 3,
                        iterations: int = 20) -> list[dict]:
        ks = _KStats()
        _check(lib().pdhg_profile_kernels(self._h, PREC[precision], warmup, iterations,
                                          C.byref(ks)), "pdhg_profile_kernels", self._h)
        return [{"name": ks.name[i].value.decode(), "avg_ms": ks.avg_ms[i],
                 "bytes": ks.bytes[i], "launches": ks.launches[i]} for i in range(ks.count)]


class Pdhg:
    """``sov::Pdhg`` (pdhg.hpp:155-172): ``Pdhg(options).solve(problem)``."""

    def __init__(self, options: PdhgOptions | None = None, device: int = 0) -> None:
        self._options = options or PdhgOptions()
        self._device = device

    def options(self) -> PdhgOptions:
        return self._options

    def solve(self, problem: Problem, cancel: CancellationToken | None = None,
              engine: Engine | None = None, **kw) -> PdhgResult:
        if engine is None:
            with Engine(self._device) as e:
                e.load(problem)
                return e.solve(self._options, cancel=cancel, **kw)
        if engine.problem is not problem:
            engine.load(problem)
        return engine.solve(self._options, cancel=cancel, **kw)


def csr_spmv(p: Problem, alpha: float, x, beta: float, y, transpose: bool = False,
             device: int = 0) -> np.ndarray:
    """``Backend::spmv`` / ``spmv_transpose`` (backend.hpp:120-126) on the engine's kernels."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.array(y, dtype=np.float64)
    ci = p.col_idx if p.nnz else np.zeros(1, np.int32)
    va = p.val if p.nnz else np.zeros(1)
    _check(lib().pdhg_csr_spmv(device, int(transpose), p.m, p.n, p.nnz, _i(p.row_ptr), _i(ci),
                               _d(va), float(alpha), _d(x if x.size else np.zeros(1)),
                               float(beta), _d(y if y.size else np.zeros(1))), "pdhg_csr_spmv")
    return y


def project_box(lo, hi, x, device: int = 0) -> np.ndarray:
    """``Backend::project_box`` (backend.hpp:131): None = unbounded side."""
    x = np.array(x, dtype=np.float64)
    lo_a = None if lo is None else np.ascontiguousarray(lo, dtype=np.float64)
    hi_a = None if hi is None else np.ascontiguousarray(hi, dtype=np.float64)
    null = C.cast(None, _dp)
    _check(lib().pdhg_project_box(device, x.size, null if lo_a is None else _d(lo_a),
                                  null if hi_a is None else _d(hi_a), _d(x)),
           "pdhg_project_box")
    return x


def scaling(p: Problem, opt: PdhgOptions | None = None) -> tuple[np.ndarray, np.ndarray]:
    """``Scaling::equilibrate(CsrMatrix)`` (scaling.cpp:19-104) as the engine computes it."""
    opt = opt or PdhgOptions()
    o = _Options()
    lib().pdhg_default_options(C.byref(o))
    for name in ("ruiz_iterations", "ruiz_tolerance", "pock_chambolle_alpha", "apply_ruiz",
                 "apply_pock_chambolle"):
        setattr(o, name, type(getattr(o, name))(getattr(opt, name)))
    rs = np.zeros(max(p.m, 1))
    cs = np.zeros(max(p.n, 1))
    ci = p.col_idx if p.nnz else np.zeros(1, np.int32)
    va = p.val if p.nnz else np.zeros(1)
    _check(lib().pdhg_scaling(p.m, p.n, p.nnz, _i(p.row_ptr), _i(ci), _d(va), C.byref(o),
                              _d(rs), _d(cs)), "pdhg_scaling")
    return rs[: p.m], cs[: p.n]
