"""ctypes binding of the C ABI in include/b200bssn.h (libb200bssn.so).

This is the Python-side mirror of the reference's per-block entry point
``bssnrhs(uzipVarsRHS, uZipVars, offset, ptmin, ptmax, sz, bflag)``
(bssn/include/rhs.h:33-36) and of its block loop ``bssnRHS``
(bssn/src/rhs.cpp:7-70).  There is no fallback: if the CUDA library is missing or
no sm_100 device is present, every call raises.
"""
from __future__ import annotations

import ctypes
import os
from typing import Sequence

import numpy as np

from .workloads import Block

NUM_VARS = 24
_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "lib", "libb200bssn.so")

FP64 = 0
MIXED = 1
GHOSTS_PRESERVE = 0
GHOSTS_ZERO = 1

STATUS = {
    0: "ok", -1: "invalid argument", -2: "block interior below 7 points", -3: "CUDA runtime error",
    -4: "device out of memory", -5: "no usable sm_100 device", -6: "non-finite right-hand side",
    -7: "bounded device wait timed out", -8: "request exceeds a fixed size limit",
}


class B200BssnError(RuntimeError):
    def __init__(self, code: int, what: str, detail: str = ""):
        self.code = code
        msg = f"{what}: {STATUS.get(code, code)}"
        if detail:
            msg += f" ({detail})"
        super().__init__(msg)


class Params(ctypes.Structure):
    """``b200bssn_params``: the bssn:: globals bssnrhs reads
    (bssn/src/parameters.cpp:99-109) plus precision and ghost policy."""

    _fields_ = [
        ("lambda_", ctypes.c_uint32 * 4),
        ("lambda_f", ctypes.c_double * 2),
        ("eta_const", ctypes.c_double),
        ("eta_r0", ctypes.c_double),
        ("eta_damping_exp", ctypes.c_double),
        ("ko_sigma", ctypes.c_double),
        ("precision", ctypes.c_uint32),
        ("ghost_policy", ctypes.c_uint32),
    ]

    @classmethod
    def make(cls, lambda_=(1, 1, 1, 1), lambda_f=(1.0, 0.0), eta_const=2.0, eta_r0=50.0,
             eta_damping_exp=1.0, ko_sigma=0.01, precision=FP64, ghost_policy=GHOSTS_PRESERVE):
        p = cls()
        for i in range(4):
            p.lambda_[i] = int(lambda_[i])
        p.lambda_f[0], p.lambda_f[1] = float(lambda_f[0]), float(lambda_f[1])
        p.eta_const = eta_const
        p.eta_r0 = eta_r0
        p.eta_damping_exp = eta_damping_exp
        p.ko_sigma = ko_sigma
        p.precision = precision
        p.ghost_policy = ghost_policy
        return p


class BlockC(ctypes.Structure):
    """``b200bssn_block`` (bssn/src/rhs.cpp:43-60 derives these from an ot::Block)."""

    _fields_ = [
        ("offset", ctypes.c_uint64),
        ("sz", ctypes.c_uint32 * 3),
        ("bflag", ctypes.c_uint32),
        ("pmin", ctypes.c_double * 3),
        ("pmax", ctypes.c_double * 3),
    ]


class PlanOptions(ctypes.Structure):
    """``b200bssn_plan_options`` (0 = default)."""

    _fields_ = [
        ("chunk_points", ctypes.c_uint64),
        ("slab_depth", ctypes.c_uint32),
        ("deriv_ctas_per_sm", ctypes.c_uint32),
        ("block_slab_depth", ctypes.POINTER(ctypes.c_uint32)),
        ("advective", ctypes.c_uint32),
        ("single_pass", ctypes.c_uint32),
        ("ring_slots", ctypes.c_uint32),
        ("tile_y", ctypes.c_uint32),
        ("deriv_regs", ctypes.c_uint32),
        ("points_per_thread", ctypes.c_uint32),
    ]


_lib = None

# (name, restype, argtypes) of every symbol declared in include/b200bssn.h
_P = ctypes.c_void_p
SIGNATURES = [
    ("b200bssn_default_params", None, [ctypes.POINTER(Params)]),
    ("b200bssn_create", ctypes.c_int, [ctypes.POINTER(_P), ctypes.c_int]),
    ("b200bssn_destroy", ctypes.c_int, [_P]),
    ("b200bssn_stream", _P, [_P]),
    ("b200bssn_last_error", ctypes.c_char_p, [_P]),
    ("b200bssn_status_string", ctypes.c_char_p, [ctypes.c_int]),
    ("b200bssn_rhs", ctypes.c_int, [_P, _P, _P, ctypes.c_uint32, ctypes.POINTER(ctypes.c_double),
                                    ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_uint32),
                                    ctypes.c_uint32, ctypes.POINTER(Params)]),
    ("b200bssn_plan_create", ctypes.c_int, [_P, ctypes.POINTER(BlockC), ctypes.c_uint32,
                                            ctypes.c_uint32, ctypes.c_uint64, ctypes.POINTER(_P)]),
    ("b200bssn_plan_create_ex", ctypes.c_int, [_P, ctypes.POINTER(BlockC), ctypes.c_uint32,
                                               ctypes.c_uint32, ctypes.POINTER(PlanOptions),
                                               ctypes.POINTER(_P)]),
    ("b200bssn_plan_destroy", ctypes.c_int, [_P]),
    ("b200bssn_plan_points", ctypes.c_uint64, [_P]),
    ("b200bssn_plan_launches", ctypes.c_uint32, [_P]),
    ("b200bssn_plan_single_pass", ctypes.c_uint32, [_P]),
    ("b200bssn_plan_status", ctypes.c_int, [_P]),
    ("b200bssn_rhs_plan_device", ctypes.c_int, [_P, _P, _P, ctypes.POINTER(Params), _P]),
    ("b200bssn_rhs_plan_host", ctypes.c_int, [_P, _P, _P, ctypes.c_uint64, ctypes.POINTER(Params)]),
    ("b200bssn_plan_profile", ctypes.c_int, [_P, _P, _P, ctypes.POINTER(Params),
                                             ctypes.POINTER(ctypes.c_double),
                                             ctypes.POINTER(ctypes.c_double)]),
    ("b200bssn_physical_constraints", ctypes.c_int,
     [_P, _P, _P, ctypes.c_uint32, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
      ctypes.POINTER(ctypes.c_uint32), ctypes.c_uint32, ctypes.c_uint32]),
    ("b200bssn_constraints_plan_device", ctypes.c_int, [_P, _P, _P, _P, _P]),
    ("b200bssn_check_finite", ctypes.c_int, [_P, _P, ctypes.c_uint32,
                                             ctypes.POINTER(ctypes.c_uint64), _P]),
    ("b200bssn_rk4_create", ctypes.c_int, [_P, ctypes.POINTER(_P)]),
    ("b200bssn_rk4_destroy", ctypes.c_int, [_P]),
    ("b200bssn_rk4_init", ctypes.c_int, [_P, _P, _P]),
    ("b200bssn_rk4_stage_state", ctypes.c_int, [_P, ctypes.c_uint32, _P]),
    ("b200bssn_rk4_stage", ctypes.c_int, [_P, ctypes.c_uint32, _P, ctypes.c_double,
                                          ctypes.POINTER(Params), _P]),
    ("b200bssn_rk4_step", ctypes.c_int, [_P, _P, ctypes.c_double, ctypes.POINTER(Params), _P]),
    ("b200bssn_rk4_graph_capture", ctypes.c_int, [_P, _P, ctypes.c_double, ctypes.POINTER(Params),
                                                  ctypes.c_uint32]),
    ("b200bssn_rk4_graph_launch", ctypes.c_int, [_P, _P]),
    ("b200bssn_rk4_graph_steps", ctypes.c_uint32, [_P]),
    ("b200bssn_rhs_noalloc", ctypes.c_int, [_P, _P, ctypes.POINTER(BlockC), ctypes.POINTER(Params), _P]),
    ("b200bssn_debug_block_scratch", ctypes.c_int, [_P, _P, ctypes.c_uint64]),
    ("b200bssn_fma_peak", ctypes.c_int, [ctypes.c_int, ctypes.c_uint32, ctypes.POINTER(ctypes.c_double)]),
]


def load(path: str = LIB_PATH):
    """Load libb200bssn.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(
            f"{path} is missing: build it with `python -m sympygr_b200.build` (no CPU fallback)")
    lib = ctypes.CDLL(path)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _check(rc: int, what: str, ctx=None):
    if rc != 0:
        detail = ""
        if ctx is not None and ctx.handle:
            detail = (load().b200bssn_last_error(ctx.handle) or b"").decode()
        raise B200BssnError(rc, what, detail)


def _ptr_table(arrays: Sequence, n: int = NUM_VARS) -> ctypes.Array:
    """n (default 24) raw pointers from numpy arrays or torch tensors (data pointer only)."""
    if len(arrays) != n:
        raise ValueError(f"need {n} arrays")
    ptrs = []
    for a in arrays:
        if isinstance(a, np.ndarray):
            if a.dtype != np.float64 or not a.flags.c_contiguous:
                raise ValueError("variable arrays must be contiguous float64")
            ptrs.append(a.ctypes.data)
        elif isinstance(a, int):
            ptrs.append(a)
        else:  # torch tensor
            if str(a.dtype) != "torch.float64" or not a.is_contiguous():
                raise ValueError("variable tensors must be contiguous float64")
            ptrs.append(a.data_ptr())
    return (ctypes.c_void_p * n)(*ptrs)


class _TorchOrder:
    """Orders a library call on `stream` with torch's work on the tensors passed.

    torch fills and reads its tensors on its current stream, and the library's
    streams (the context stream included, created non-blocking) do not synchronise
    with it: without this, an evaluation can start before torch has finished writing
    its inputs (or zeroing its outputs, overwriting results written meanwhile), and
    torch can read results before the evaluation wrote them.  Entering makes `stream`
    wait for everything torch has queued on the tensors' device so far; leaving makes
    torch's current stream wait for the call.  Calls given only numpy arrays or raw
    pointers are left as they are."""

    def __init__(self, stream: int, *groups):
        self.stream, self.t = stream, None
        for g in groups:
            for a in (g if g is not None else ()):
                if not isinstance(a, (np.ndarray, int)) and getattr(a, "is_cuda", False):
                    self.t = a
                    break
            if self.t is not None:
                break

    def __enter__(self):
        if self.t is not None:
            import torch

            ev = torch.cuda.Event()
            ev.record(torch.cuda.current_stream(self.t.device))
            torch.cuda.ExternalStream(self.stream, device=self.t.device).wait_event(ev)
        return self

    def __exit__(self, exc_type, exc, tb):
        if self.t is not None and exc_type is None:
            import torch

            ev = torch.cuda.Event()
            ev.record(torch.cuda.ExternalStream(self.stream, device=self.t.device))
            torch.cuda.current_stream(self.t.device).wait_event(ev)
        return False


NOALLOC_MAX_POINTS = 32768
NUM_CONSTRAINTS = 4  # ham, mom0, mom1, mom2


def block_struct(b: Block) -> BlockC:
    c = BlockC()
    c.offset = b.offset
    for a in range(3):
        c.sz[a] = b.sz[a]
        c.pmin[a] = b.pmin[a]
        c.pmax[a] = b.pmax[a]
    c.bflag = b.bflag
    return c


def rhs_noalloc(rhs, u, block: Block, params: Params, stream: int = 0):
    """One block on device arrays through the allocation-free entry point
    (b200bssn_rhs_noalloc); asynchronous on `stream` on the current device."""
    blk = block_struct(block)
    _check(load().b200bssn_rhs_noalloc(_ptr_table(rhs), _ptr_table(u), ctypes.byref(blk),
                                       ctypes.byref(params), ctypes.c_void_p(stream or None)),
           "b200bssn_rhs_noalloc")


def fma_peak_tflops(device: int, precision: int) -> float:
    """Measured FMA throughput (TFLOP/s) of the device's FP64 or FP32 pipe."""
    t = ctypes.c_double()
    _check(load().b200bssn_fma_peak(device, precision, ctypes.byref(t)), "b200bssn_fma_peak")
    return t.value


class Context:
    """``b200bssn_ctx``: a device, its stream and per-context buffers."""

    def __init__(self, device: int = 0):
        lib = load()
        h = ctypes.c_void_p()
        _check(lib.b200bssn_create(ctypes.byref(h), device), "b200bssn_create")
        self.handle = h
        self.device = device

    @property
    def stream(self) -> int:
        return load().b200bssn_stream(self.handle) or 0

    def close(self):
        if self.handle:
            load().b200bssn_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def bssnrhs(self, rhs, u, offset: int, pmin, pmax, sz, bflag: int, params: Params):
        """Drop-in for the reference's ``bssnrhs`` on HOST arrays (24 float64
        arrays each for rhs and u).  Writes the interior of the block in `rhs`."""
        lib = load()
        pm = (ctypes.c_double * 3)(*pmin)
        px = (ctypes.c_double * 3)(*pmax)
        s = (ctypes.c_uint32 * 3)(*sz)
        _check(lib.b200bssn_rhs(self.handle, _ptr_table(rhs), _ptr_table(u), int(offset), pm, px,
                                s, int(bflag), ctypes.byref(params)), "b200bssn_rhs", self)

    def physical_constraints(self, con, u, offset: int, pmin, pmax, sz, bflag: int,
                             precision: int = FP64):
        """Drop-in for the reference's ``physical_constraints`` on HOST arrays: `con`
        is 4 float64 arrays (ham, mom0, mom1, mom2) written at the block's interior."""
        lib = load()
        pm = (ctypes.c_double * 3)(*pmin)
        px = (ctypes.c_double * 3)(*pmax)
        s = (ctypes.c_uint32 * 3)(*sz)
        _check(lib.b200bssn_physical_constraints(self.handle, _ptr_table(con, NUM_CONSTRAINTS),
                                                 _ptr_table(u), int(offset), pm, px, s, int(bflag),
                                                 int(precision)),
               "b200bssn_physical_constraints", self)

    def debug_block_scratch(self, npts: int) -> np.ndarray:
        """Derivative slots [162, npts] of the last single-block call."""
        out = np.zeros((162, npts))
        _check(load().b200bssn_debug_block_scratch(self.handle, out.ctypes.data_as(ctypes.c_void_p),
                                                   npts), "b200bssn_debug_block_scratch", self)
        return out


class Plan:
    """``b200bssn_plan``: descriptors and scratch for a fixed block list."""

    def __init__(self, ctx: Context, blocks: Sequence[Block], precision: int = FP64,
                 chunk_points: int = 0, slab_depth: int = 0, deriv_ctas_per_sm: int = 0,
                 block_slab_depth: Sequence[int] | None = None, advective: bool = False,
                 single_pass: bool = False, ring_slots: int = 0, tile_y: int = 0, deriv_regs: int = 0,
                 points_per_thread: int = 0):
        lib = load()
        arr = (BlockC * len(blocks))()
        for i, b in enumerate(blocks):
            arr[i].offset = b.offset
            for a in range(3):
                arr[i].sz[a] = b.sz[a]
                arr[i].pmin[a] = b.pmin[a]
                arr[i].pmax[a] = b.pmax[a]
            arr[i].bflag = b.bflag
        h = ctypes.c_void_p()
        opts = PlanOptions(chunk_points, slab_depth, deriv_ctas_per_sm)
        opts.advective = 1 if advective else 0
        opts.single_pass = 1 if single_pass else 0
        opts.ring_slots = int(ring_slots)
        opts.tile_y = int(tile_y)
        opts.deriv_regs = int(deriv_regs)
        opts.points_per_thread = int(points_per_thread)
        if block_slab_depth is not None:
            if len(block_slab_depth) != len(blocks):
                raise ValueError("block_slab_depth needs one entry per block")
            depths = (ctypes.c_uint32 * len(blocks))(*[int(d) for d in block_slab_depth])
            opts.block_slab_depth = depths
        _check(lib.b200bssn_plan_create_ex(ctx.handle, arr, len(blocks), precision,
                                           ctypes.byref(opts), ctypes.byref(h)),
               "b200bssn_plan_create_ex", ctx)
        self.ctx = ctx
        self.handle = h
        self.precision = precision
        self.nblocks = len(blocks)

    @property
    def points(self) -> int:
        return int(load().b200bssn_plan_points(self.handle))

    @property
    def launches(self) -> int:
        return int(load().b200bssn_plan_launches(self.handle))

    @property
    def single_pass(self) -> bool:
        """True when the right-hand side runs as the one-pass kernel."""
        return bool(load().b200bssn_plan_single_pass(self.handle))

    def status(self):
        """Synchronise and raise if a bounded device wait of the last evaluation ran out."""
        _check(load().b200bssn_plan_status(self.handle), "b200bssn_plan_status", self.ctx)

    def rhs_device(self, rhs, u, params: Params, stream: int = 0):
        """Batched RHS on device arrays (torch CUDA tensors or raw pointers);
        asynchronous on `stream` (0: the context stream), ordered after torch's work
        on the tensors passed and before torch's later work (_TorchOrder)."""
        with _TorchOrder(stream or self.ctx.stream, rhs, u):
            _check(load().b200bssn_rhs_plan_device(self.handle, _ptr_table(rhs), _ptr_table(u),
                                                   ctypes.byref(params), ctypes.c_void_p(stream or None)),
                   "b200bssn_rhs_plan_device", self.ctx)

    def constraints_device(self, u, con=None, block_norms=None, stream: int = 0):
        """Constraints of every block on device arrays: `con` (4 device arrays or
        None) receives ham, mom0..2 at interior points; `block_norms` (None or a
        contiguous float64 device tensor of nblocks*8) receives per block the sums of
        squares and maxima of |ham|, |mom0..2|.  Asynchronous on `stream`."""
        cp = _ptr_table(con, NUM_CONSTRAINTS) if con is not None else None
        npt = None
        if block_norms is not None:
            if block_norms.numel() < 8 * self.nblocks or str(block_norms.dtype) != "torch.float64":
                raise ValueError("block_norms must hold nblocks*8 float64")
            npt = block_norms.data_ptr()
        with _TorchOrder(stream or self.ctx.stream, u, con, [block_norms] if block_norms is not None else None):
            _check(load().b200bssn_constraints_plan_device(self.handle, cp, _ptr_table(u),
                                                           ctypes.c_void_p(npt),
                                                           ctypes.c_void_p(stream or None)),
                   "b200bssn_constraints_plan_device", self.ctx)

    def check_finite(self, arrays, stream: int = 0):
        """NaN/Inf guard over the interior points of the plan's blocks in the given
        device arrays (1..24).  Returns None if all finite, else the smallest
        offending element index."""
        n = len(arrays)
        bad = ctypes.c_uint64()
        with _TorchOrder(stream or self.ctx.stream, arrays):
            rc = load().b200bssn_check_finite(self.handle, _ptr_table(arrays, n), n, ctypes.byref(bad),
                                              ctypes.c_void_p(stream or None))
        if rc == -6:
            return int(bad.value)
        _check(rc, "b200bssn_check_finite", self.ctx)
        return None

    def profile(self, rhs, u, params: Params):
        """One evaluation with per-launch events: (derivative ms, algebra ms)."""
        d, a = ctypes.c_double(), ctypes.c_double()
        with _TorchOrder(self.ctx.stream, rhs, u):
            _check(load().b200bssn_plan_profile(self.handle, _ptr_table(rhs), _ptr_table(u),
                                                ctypes.byref(params), ctypes.byref(d), ctypes.byref(a)),
                   "b200bssn_plan_profile", self.ctx)
        return d.value, a.value

    def rhs_host(self, rhs, u, n_elems: int, params: Params):
        """Batched RHS on host arrays (H2D, evaluate, D2H; blocks until done)."""
        _check(load().b200bssn_rhs_plan_host(self.handle, _ptr_table(rhs), _ptr_table(u),
                                             int(n_elems), ctypes.byref(params)),
               "b200bssn_rhs_plan_host", self.ctx)

    def close(self):
        if self.handle:
            load().b200bssn_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RK4:
    """``b200bssn_rk4``: classic RK4 over a plan's blocks, stage update fused into the
    algebra kernel.  `u` is the list of 24 device arrays the state lives in; the
    object keeps pointers to them for graph capture, so keep them alive."""

    def __init__(self, plan: Plan):
        lib = load()
        h = ctypes.c_void_p()
        _check(lib.b200bssn_rk4_create(plan.handle, ctypes.byref(h)), "b200bssn_rk4_create", plan.ctx)
        self.plan = plan
        self.handle = h

    def init(self, u, stream: int = 0):
        """Copy the state (ghosts included) into both stage states."""
        with _TorchOrder(stream or self.plan.ctx.stream, u):
            _check(load().b200bssn_rk4_init(self.handle, _ptr_table(u), ctypes.c_void_p(stream or None)),
                   "b200bssn_rk4_init", self.plan.ctx)

    def stage_state(self, stage: int):
        """Device pointers (24 ints; 0 for stage 0) of the state stage `stage` reads."""
        out = (ctypes.c_void_p * NUM_VARS)()
        _check(load().b200bssn_rk4_stage_state(self.handle, stage, out), "b200bssn_rk4_stage_state",
               self.plan.ctx)
        return [int(p or 0) for p in out]

    def stage(self, stage: int, u, dt: float, params: Params, stream: int = 0):
        with _TorchOrder(stream or self.plan.ctx.stream, u):
            _check(load().b200bssn_rk4_stage(self.handle, stage, _ptr_table(u), float(dt),
                                             ctypes.byref(params), ctypes.c_void_p(stream or None)),
                   "b200bssn_rk4_stage", self.plan.ctx)

    def step(self, u, dt: float, params: Params, stream: int = 0):
        with _TorchOrder(stream or self.plan.ctx.stream, u):
            _check(load().b200bssn_rk4_step(self.handle, _ptr_table(u), float(dt), ctypes.byref(params),
                                            ctypes.c_void_p(stream or None)),
                   "b200bssn_rk4_step", self.plan.ctx)

    def capture(self, u, dt: float, params: Params, steps: int = 1):
        """Capture `steps` full steps into a CUDA graph (replay with ``launch``)."""
        self._graph_arrays = list(u)
        _check(load().b200bssn_rk4_graph_capture(self.handle, _ptr_table(u), float(dt),
                                                 ctypes.byref(params), int(steps)),
               "b200bssn_rk4_graph_capture", self.plan.ctx)

    def launch(self, stream: int = 0):
        with _TorchOrder(stream or self.plan.ctx.stream, getattr(self, "_graph_arrays", None)):
            _check(load().b200bssn_rk4_graph_launch(self.handle, ctypes.c_void_p(stream or None)),
                   "b200bssn_rk4_graph_launch", self.plan.ctx)

    @property
    def graph_steps(self) -> int:
        return int(load().b200bssn_rk4_graph_steps(self.handle))

    def close(self):
        if self.handle:
            load().b200bssn_rk4_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
