"""TEST INFRASTRUCTURE ONLY -- Python access to the oracle and the reference build.

* ``oracle_rhs`` / ``oracle_slots`` call the C restatement (oracle/bssn_oracle.c,
  built to oracle/_build/libbssn_oracle.so).
* ``ref_rhs`` / ``ref_blocks_omp`` call the reference's own CPU bssnrhs compiled
  from its sources (oracle/_ref/libbssn_ref_{parity,fast}.so, see oracle/Makefile).
* ``fake_initial_data`` restates the reference's analytic test data
  (bssn/src/grUtils.cpp:15-58) in numpy.

Only tests/, the smoke check and bench.py's CPU-baseline leg import this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "_build", "libbssn_oracle.so")
REF_PARITY = os.path.join(HERE, "_ref", "libbssn_ref_parity.so")
REF_FAST = os.path.join(HERE, "_ref", "libbssn_ref_fast.so")        # -march=x86-64-v3
REF_FAST_V4 = os.path.join(HERE, "_ref", "libbssn_ref_fast_v4.so")  # -march=x86-64-v4
NUM_VARS = 24
NUM_DERIVS = 138
NUM_SLOTS = 162

_libs = {}


class OracleParams(ctypes.Structure):
    _fields_ = [
        ("lambda_", ctypes.c_uint * 4),
        ("lambda_f", ctypes.c_double * 2),
        ("eta_const", ctypes.c_double),
        ("eta_r0", ctypes.c_double),
        ("eta_damping_exp", ctypes.c_double),
        ("ko_sigma", ctypes.c_double),
    ]


def params(lambda_=(1, 1, 1, 1), lambda_f=(1.0, 0.0), eta_const=2.0, eta_r0=50.0,
           eta_damping_exp=1.0, ko_sigma=0.01):
    p = OracleParams()
    for i in range(4):
        p.lambda_[i] = lambda_[i]
    p.lambda_f[0], p.lambda_f[1] = lambda_f
    p.eta_const, p.eta_r0, p.eta_damping_exp, p.ko_sigma = eta_const, eta_r0, eta_damping_exp, ko_sigma
    return p


def reference_checkout() -> str | None:
    """The reference checkout: $SYMPYGR_REFERENCE, else a ``reference`` folder beside
    this repository; None when neither holds bssn/src."""
    cands = [os.environ.get("SYMPYGR_REFERENCE"),
             os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")]
    for c in cands:
        if c and os.path.isdir(os.path.join(c, "bssn", "src")):
            return os.path.abspath(c)
    return None


def build(with_reference: bool | None = None):
    """make -C oracle (the reference flavours only where the reference checkout exists)."""
    targets = ["oracle"]
    ref = reference_checkout()
    if with_reference is None:
        with_reference = ref is not None
    if with_reference:
        targets.append("ref")
    extra = [f"SYMPYGR_REFERENCE={ref}"] if ref else []
    subprocess.run(["make", "-s", "-C", HERE, *extra, *targets], check=True)


def _load(path):
    if path not in _libs:
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        _libs[path] = ctypes.CDLL(path)
    return _libs[path]


def oracle_lib():
    if not os.path.exists(ORACLE_LIB):
        build(with_reference=False)
    return _load(ORACLE_LIB)


def _cpu_has_avx512() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    fl = set(line.split(":", 1)[1].split())
                    return {"avx512f", "avx512dq", "avx512cd", "avx512bw", "avx512vl"} <= fl
    except OSError:
        pass
    return False


def fast_flavour_path() -> str:
    """The timing build for this CPU: x86-64-v4 (AVX-512) where the CPU has it and the
    build exists, else x86-64-v3 -- the closest stand-in for -march=native available
    on a host without the reference sources."""
    if _cpu_has_avx512() and os.path.exists(REF_FAST_V4):
        return REF_FAST_V4
    return REF_FAST


def have_reference(flavour="parity") -> bool:
    return os.path.exists(REF_PARITY if flavour == "parity" else fast_flavour_path())


def _ptrs(arr2d, offset=0):
    return (ctypes.c_void_p * arr2d.shape[0])(*[arr2d[v].ctypes.data + 8 * offset
                                                for v in range(arr2d.shape[0])])


def _dbl3(x):
    return (ctypes.c_double * 3)(*[float(t) for t in x])


def _uint3(x):
    return (ctypes.c_uint * 3)(*[int(t) for t in x])


def oracle_rhs(u, blk, prm=None, rhs=None):
    """C restatement of bssnrhs on one block; u is [24, >= offset+npad] float64."""
    lib = oracle_lib()
    u = np.ascontiguousarray(u, dtype=np.float64)
    if rhs is None:
        rhs = np.zeros_like(u)
    prm = prm or params()
    lib.bssn_oracle_rhs(_ptrs(rhs), _ptrs(u), ctypes.c_uint(blk.offset), _dbl3(blk.pmin),
                        _dbl3(blk.pmax), _uint3(blk.sz), ctypes.c_uint(blk.bflag), ctypes.byref(prm))
    return rhs


def oracle_slots(u, blk):
    """The 162 derivative slots at interior points, shape (162, npts)."""
    lib = oracle_lib()
    u = np.ascontiguousarray(u, dtype=np.float64)
    npts = blk.ninterior
    out = np.zeros((NUM_SLOTS, npts))
    lib.bssn_oracle_derivative_slots(out.ctypes.data_as(ctypes.c_void_p), _ptrs(u),
                                     ctypes.c_uint(blk.offset), _dbl3(blk.pmin), _dbl3(blk.pmax),
                                     _uint3(blk.sz), ctypes.c_uint(blk.bflag))
    return out


def oracle_rhs_adv(u, blk, prm=None, rhs=None):
    """The oracle's RHS in the opt-in upwind mode (advective derivatives from the
    4th-order upwind stencils)."""
    lib = oracle_lib()
    u = np.ascontiguousarray(u, dtype=np.float64)
    if rhs is None:
        rhs = np.zeros_like(u)
    prm = prm or params()
    lib.bssn_oracle_rhs_adv(_ptrs(rhs), _ptrs(u), ctypes.c_uint(blk.offset), _dbl3(blk.pmin),
                            _dbl3(blk.pmax), _uint3(blk.sz), ctypes.c_uint(blk.bflag), ctypes.byref(prm))
    return rhs


def _adv_call(fn, axis, f, h, sz, beta, bflag):
    f = np.ascontiguousarray(f, dtype=np.float64)
    beta = np.ascontiguousarray(beta, dtype=np.float64)
    out = np.zeros_like(f)
    args = (out.ctypes.data_as(ctypes.c_void_p), f.ctypes.data_as(ctypes.c_void_p), ctypes.c_double(h),
            _uint3(sz), beta.ctypes.data_as(ctypes.c_void_p), ctypes.c_uint(bflag))
    if fn is None:
        return out, args
    fn(*args) if axis is None else fn(ctypes.c_int(axis), *args)
    return out


def oracle_deriv42adv(axis, f, h, sz, beta, bflag):
    """The oracle's upwind derivative of one padded block array along `axis`."""
    lib = oracle_lib()
    fn = [lib.bssn_oracle_deriv42adv_x, lib.bssn_oracle_deriv42adv_y, lib.bssn_oracle_deriv42adv_z][axis]
    return _adv_call(fn, None, f, h, sz, beta, bflag)


def ref_deriv42adv(axis, f, h, sz, beta, bflag, flavour="parity"):
    """The reference's own deriv42adv_{x,y,z} (bssn/src/derivs.cpp:495-900)."""
    return _adv_call(_ref(flavour).ref_deriv42adv, axis, f, h, sz, beta, bflag)


def oracle_constraints(u, blk, con=None):
    """C restatement of the Hamiltonian and momentum constraints on one block:
    con[0..3] = ham, mom0, mom1, mom2 at the interior points (others untouched)."""
    lib = oracle_lib()
    u = np.ascontiguousarray(u, dtype=np.float64)
    if con is None:
        con = np.zeros((4, u.shape[1]))
    lib.bssn_oracle_block_constraints(_ptrs(con), _ptrs(u), ctypes.c_uint(blk.offset),
                                      _dbl3(blk.pmin), _dbl3(blk.pmax), _uint3(blk.sz),
                                      ctypes.c_uint(blk.bflag))
    return con


def interior_elements(blocks, n_elems):
    """Boolean mask over element indices: True at every block's interior points."""
    m = np.zeros(n_elems, dtype=bool)
    for b in blocks:
        nx, ny, nz = b.sz
        idx = np.arange(b.npad).reshape(nz, ny, nx)[3:-3, 3:-3, 3:-3].ravel()
        m[b.offset + idx] = True
    return m


class OracleRK4:
    """Classic RK4 over a block list with the oracle's right-hand side: the time
    stepping the device integrator implements (stage states seeded from the state
    at ``init`` and updated at interior points only; the state's ghost points are
    never written).  u is [24, n_elems] float64 and is advanced in place."""

    def __init__(self, blocks, n_elems, prm=None, advective=False):
        self.blocks = list(blocks)
        self.prm = prm or params()
        self.rhs_fn = oracle_rhs_adv if advective else oracle_rhs
        self.mask = interior_elements(self.blocks, n_elems)
        self.sa = self.sb = None

    def init(self, u):
        self.sa = u.copy()
        self.sb = u.copy()

    def _rhs(self, state):
        r = np.zeros_like(state)
        for b in self.blocks:
            self.rhs_fn(state, b, self.prm, rhs=r)
        return r[:, self.mask]

    def step(self, u, dt):
        m = self.mask
        un = u[:, m]
        k = self._rhs(u)
        acc = (dt / 6.0) * k
        self.sa[:, m] = un + (dt * 0.5) * k
        k = self._rhs(self.sa)
        acc += (dt / 3.0) * k
        self.sb[:, m] = un + (dt * 0.5) * k
        k = self._rhs(self.sb)
        acc += (dt / 3.0) * k
        self.sa[:, m] = un + dt * k
        k = self._rhs(self.sa)
        u[:, m] = un + acc + (dt / 6.0) * k


def _ref(flavour):
    lib = _load(REF_PARITY if flavour == "parity" else fast_flavour_path())
    lib.ref_bssnrhs_blocks_omp.restype = ctypes.c_double
    return lib


def ref_set_params(lib, prm):
    lam = (ctypes.c_uint * 4)(*prm.lambda_)
    lf = (ctypes.c_double * 2)(*prm.lambda_f)
    lib.ref_set_params(lam, lf, ctypes.c_double(prm.eta_const), ctypes.c_double(prm.eta_r0),
                       ctypes.c_double(prm.eta_damping_exp), ctypes.c_double(prm.ko_sigma))


def ref_rhs(u, blk, prm=None, rhs=None, flavour="parity"):
    """The reference's own bssnrhs (compiled from its sources) on one block."""
    lib = _ref(flavour)
    prm = prm or params()
    ref_set_params(lib, prm)
    u = np.ascontiguousarray(u, dtype=np.float64)
    if rhs is None:
        rhs = np.zeros_like(u)
    lib.ref_bssnrhs(_ptrs(rhs), _ptrs(u), ctypes.c_uint(blk.offset), _dbl3(blk.pmin),
                    _dbl3(blk.pmax), _uint3(blk.sz), ctypes.c_uint(blk.bflag))
    return rhs


def ref_rhs_sep(u, blk, prm=None, rhs=None, flavour="parity"):
    """The reference's staged bssnrhs_sep (bssn/src/rhs.cpp:392) on one block."""
    lib = _ref(flavour)
    prm = prm or params()
    ref_set_params(lib, prm)
    u = np.ascontiguousarray(u, dtype=np.float64)
    if rhs is None:
        rhs = np.zeros_like(u)
    lib.ref_bssnrhs_sep(_ptrs(rhs), _ptrs(u), ctypes.c_uint(blk.offset), _dbl3(blk.pmin),
                        _dbl3(blk.pmax), _uint3(blk.sz), ctypes.c_uint(blk.bflag))
    return rhs


def ref_constraints(u, blk, flavour="parity"):
    """The reference's own physical_constraints (bssn/CodeGen/physcon.cpp:12) on one
    block: rows ham, mom0, mom1, mom2, psi4_real, psi4_img. The reference uses hx in
    all three directions, so compare on blocks with equal spacings only."""
    lib = _ref(flavour)
    u = np.ascontiguousarray(u, dtype=np.float64)
    con = np.zeros((6, u.shape[1]))
    lib.ref_physical_constraints(_ptrs(con), _ptrs(u), ctypes.c_uint(blk.offset), _dbl3(blk.pmin),
                                 _dbl3(blk.pmax), _uint3(blk.sz), ctypes.c_uint(blk.bflag))
    return con


def ref_blocks_omp(u, rhs, blocks, prm=None, nthreads=0, flavour="fast"):
    """Reference bssnrhs over a block list in an OpenMP parallel-for; returns seconds."""
    lib = _ref(flavour)
    prm = prm or params()
    ref_set_params(lib, prm)
    n = len(blocks)
    offs = (ctypes.c_uint * n)(*[b.offset for b in blocks])
    pmins = (ctypes.c_double * (3 * n))(*[c for b in blocks for c in b.pmin])
    pmaxs = (ctypes.c_double * (3 * n))(*[c for b in blocks for c in b.pmax])
    szs = (ctypes.c_uint * (3 * n))(*[c for b in blocks for c in b.sz])
    bfl = (ctypes.c_uint * n)(*[b.bflag for b in blocks])
    return lib.ref_bssnrhs_blocks_omp(_ptrs(rhs), _ptrs(u), ctypes.c_int(n), offs, pmins, pmaxs,
                                      szs, bfl, ctypes.c_int(nthreads))


def ref_max_threads(flavour="fast") -> int:
    return int(_ref(flavour).ref_max_threads())


def fake_initial_data(x, y, z):
    """numpy restatement of bssn::fake_initial_data (bssn/src/grUtils.cpp:15-58);
    returns [24, ...] in VAR order."""
    pi = np.arccos(-1.0)
    f1 = 31.0 / 17.0
    f2 = 37.0 / 11.0
    u = np.zeros((NUM_VARS,) + np.shape(x))
    e4 = np.exp(-4.0 * np.cos(x) * np.sin(y))
    u[0] = 1.0 - 0.25 * np.sin(f1 * x)
    u[6] = 4.0 / 17.0 * np.sin(x) * np.cos(z)
    u[7] = pi / 5.0 * np.cos(y) * np.sin(z + x)
    u[8] = 4.0 / 17.0 * np.sin(f2 * x) * np.sin(z)
    u[9] = 31.0 * x * np.cos(f1 * z + y)
    u[10] = 7.0 * y * np.sin(f1 * x + y) + 3.0 * np.cos(z)
    u[11] = 5.0 * z * np.cos(f1 * x + y) + 7.0 * np.sin(z + y + x) + 1.0
    u[3] = 5.0 * np.cos(x) / (10.0 * np.sin(x + z) + 26.0 - 1.0 * np.cos(x * z) * np.cos(x))
    u[4] = -5.0 * np.sin(y) / (25.0 + 10.0 * np.cos(y + z) + np.cos(y) * np.cos(y * z))
    u[5] = -5.0 * np.sin(z) / (25.0 + 10.0 * np.cos(y + x) + np.cos(y * x) * np.cos(z))
    u[1] = 1.0 + e4
    u[12] = 1.00 + 0.2 * np.sin(x + z) * np.cos(y)
    u[15] = 1.00 + 0.2 * np.cos(y) * np.cos(z + x)
    u[17] = 1.00 / (u[12] + u[15])
    u[13] = 0.7 * np.cos(x * x + y * y)
    u[14] = 0.3 * np.sin(z) * np.cos(x)
    u[16] = -0.5 * np.sin(x * x) * np.cos(y) * np.cos(z)
    kk = (5.0 * e4 / (5.0 + np.sin(x)) * np.cos(x) + 5.0 * e4 / (5.0 + np.cos(y)) * np.cos(y))
    u[2] = kk + 0.4 * (25.0 + 5.0 * np.cos(y) + 5.0 * np.sin(x) + np.sin(x) * np.cos(y)) * e4 * np.cos(z)
    inner = kk + 0.04 * (25.0 + 5.0 * np.cos(y) + 5.0 * np.sin(x) + np.sin(x) * np.cos(y)) * e4 * np.cos(z)
    ie4 = np.exp(4.0 * np.cos(x) * np.sin(y))
    u[18] = e4 * (np.cos(x) - 0.3333333333 * ie4 * (1.0 + 0.2 * np.sin(x)) * inner)
    u[19] = 1.0 + x * z / (0.1 + x * x + y * y + z * z)
    u[20] = 1.3 - x * y / (3.0 + x * x + 2.0 * y * y + z * z) * (x * x + z * z)
    u[21] = e4 * (np.cos(y) - 0.33333333330 * np.exp(4 * np.cos(x) * np.sin(y)) * (1 + 0.2 * np.cos(y)) * inner)
    u[22] = -1.0 + y * z / (1.0 + 3.0 * x * x + y * y + z * z)
    u[23] = e4 * (np.cos(z) - 0.3333333333 * np.exp(4 * np.cos(x) * np.sin(y)) / (1 + 0.2 * np.sin(x))
                  / (1 + 0.2 * np.cos(y)) * inner)
    return u


def fake_block(n, pmin, h, bflag=0):
    """One padded n^3 block filled with fake_initial_data; returns (u [24,n^3], Block)."""
    from sympygr_b200.workloads import Block, coords

    blk = Block(0, (n, n, n), bflag, tuple(pmin), tuple(pmin[a] + (n - 1) * h for a in range(3)))
    x, y, z = coords(blk)
    u = fake_initial_data(x, y, z).reshape(NUM_VARS, -1)
    return np.ascontiguousarray(u), blk


def interior(arr, blk):
    """[24, interior points] view of the block's interior values (x fastest)."""
    n0, n1, n2 = blk.sz
    a = arr[:, blk.offset:blk.offset + blk.npad].reshape(arr.shape[0], n2, n1, n0)
    return a[:, 3:-3, 3:-3, 3:-3].reshape(arr.shape[0], -1)


def rel_errors(got, ref):
    """Per variable: max|g-r| / max|r| and the RMS analogue."""
    got = np.asarray(got)
    ref = np.asarray(ref)
    d = got - ref
    scale = np.maximum(np.abs(ref).max(axis=1), 1e-300)
    rms_scale = np.maximum(np.sqrt((ref ** 2).mean(axis=1)), 1e-300)
    return np.abs(d).max(axis=1) / scale, np.sqrt((d ** 2).mean(axis=1)) / rms_scale


def batch_rel_errors(pairs, floor=1e-3):
    """MIXED-path norms over several blocks: `pairs` is a list of (got, ref) arrays of
    shape [nv, points] (one per block).  Returns (over_batch, per_block):

    * over_batch[v] = max over blocks of max|g - r| / max over blocks of max|r| -- the
      norm the benchmark reports for a whole batch;
    * per_block[k][v] = max|g - r| / max|r| on block k, where a variable whose largest
      |r| on that block is below `floor` times the block's largest |r| over all
      variables is measured against that fraction of the block scale instead: such a
      right-hand side vanishes there but for the Kreiss-Oliger term of a field at rest,
      a sixth difference made of FP64 rounding noise in both precisions.
    """
    nv = pairs[0][1].shape[0]
    dmax, rmax, per_block = np.zeros(nv), np.zeros(nv), []
    for got, ref in pairs:
        d = np.abs(np.asarray(got) - np.asarray(ref)).max(axis=1)
        r = np.abs(np.asarray(ref)).max(axis=1)
        dmax, rmax = np.maximum(dmax, d), np.maximum(rmax, r)
        scale = np.maximum(r, floor * r.max())
        per_block.append(d / np.maximum(scale, 1e-300))
    return dmax / np.maximum(rmax, 1e-300), per_block

