"""CPU checks of the C ABI boundary: the library loads, exports every function
declared in include/b200bssn.h, its structs have the C layout the ctypes mirror
assumes, host-only entry points work, and without a usable GPU the entry points
fail with an error code (no silent CPU fallback).  The C++ shim exports the
reference's mangled bssnrhs and needs exactly the bssn:: globals the reference
defines."""
import ctypes
import os
import re
import subprocess

import pytest

from sympygr_b200 import build, capi

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "b200bssn.h")


@pytest.fixture(scope="module")
def lib():
    build.build()
    return capi.load()


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char \*|uint64_t|uint32_t|void \*)\s*\*?\s*"
                                 r"(b200bssn_\w+)\s*\(", text, flags=re.M)))


def test_every_declared_function_is_exported(lib):
    names = declared_functions()
    assert len(names) >= 15
    out = subprocess.run(["nm", "-D", "--defined-only", capi.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r" T (b200bssn_\w+)", out))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    # and the ctypes mirror binds every one of them
    bound = {s[0] for s in capi.SIGNATURES}
    assert set(names) == bound, set(names) ^ bound


def test_struct_layouts_match_c(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "b200bssn.h"\n'
                   'int main(void){printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(b200bssn_params),'
                   ' offsetof(b200bssn_params, precision), sizeof(b200bssn_block),'
                   ' offsetof(b200bssn_block, pmin), sizeof(b200bssn_plan_options),'
                   ' offsetof(b200bssn_plan_options, deriv_ctas_per_sm),'
                   ' offsetof(b200bssn_plan_options, block_slab_depth),'
                   ' offsetof(b200bssn_plan_options, advective),'
                   ' offsetof(b200bssn_plan_options, single_pass),'
                   ' offsetof(b200bssn_plan_options, ring_slots),'
                   ' offsetof(b200bssn_plan_options, tile_y),'
                   ' offsetof(b200bssn_plan_options, deriv_regs),'
                   ' offsetof(b200bssn_plan_options, points_per_thread)); return 0;}\n')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(REPO, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True,
                                          check=True).stdout.split()]
    want = [ctypes.sizeof(capi.Params), capi.Params.precision.offset, ctypes.sizeof(capi.BlockC),
            capi.BlockC.pmin.offset, ctypes.sizeof(capi.PlanOptions),
            capi.PlanOptions.deriv_ctas_per_sm.offset, capi.PlanOptions.block_slab_depth.offset,
            capi.PlanOptions.advective.offset, capi.PlanOptions.single_pass.offset,
            capi.PlanOptions.ring_slots.offset, capi.PlanOptions.tile_y.offset,
            capi.PlanOptions.deriv_regs.offset, capi.PlanOptions.points_per_thread.offset]
    assert got == want


def test_default_params_are_the_reference_defaults(lib):
    p = capi.Params()
    lib.b200bssn_default_params(ctypes.byref(p))
    # bssn/src/parameters.cpp:99-109
    assert list(p.lambda_) == [1, 1, 1, 1]
    assert list(p.lambda_f) == [1.0, 0.0]
    assert (p.eta_const, p.eta_r0, p.eta_damping_exp, p.ko_sigma) == (2.0, 50.0, 1.0, 0.01)
    assert lib.b200bssn_status_string(-8) == b"request exceeds a fixed size limit"


def test_fails_loudly_without_a_gpu(lib):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    assert lib.b200bssn_create(ctypes.byref(h), 0) == -5  # B200BSSN_ERR_NO_DEVICE
    with pytest.raises(capi.B200BssnError):
        capi.Context(0)
    # the allocation-free entry point validates arguments before touching a device
    blk = capi.BlockC()
    assert lib.b200bssn_rhs_noalloc(None, None, ctypes.byref(blk), None, None) == -1


def test_shim_exports_the_reference_symbol():
    shim = build.build_shim()
    out = subprocess.run(["nm", "-D", shim], capture_output=True, text=True, check=True).stdout
    defined = set(re.findall(r" T (\S+)", out))
    undefined = set(re.findall(r" U (_ZN4bssn\S+)", out))
    # void bssnrhs(double**, const double**, const unsigned&, const double*, const double*,
    #              const unsigned*, const unsigned&)   (bssn/include/rhs.h:33-36)
    assert "_Z7bssnrhsPPdPPKdRKjS2_S2_PS4_S5_" in defined
    # void physical_constraints(double**, const double**, const unsigned&, const double*,
    #                           const double*, const unsigned*, const unsigned&)
    #                                                  (bssn/CodeGen/physcon.cpp:12-15)
    assert "_Z20physical_constraintsPPdPPKdRKjS2_S2_PS4_S5_" in defined
    assert "_Z11bssnrhs_sepPPdPPKdRKjS2_S2_PS4_S5_" in defined  # bssn/include/rhs.h:39
    assert undefined == {"_ZN4bssn11BSSN_LAMBDAE", "_ZN4bssn13BSSN_LAMBDA_FE", "_ZN4bssn9ETA_CONSTE",
                         "_ZN4bssn6ETA_R0E", "_ZN4bssn15ETA_DAMPING_EXPE", "_ZN4bssn13KO_DISS_SIGMAE"}
    from oracle import pyoracle as po

    if po.have_reference("parity"):  # same mangled entry point and globals as the reference build
        ref = subprocess.run(["nm", "-D", po.REF_PARITY], capture_output=True, text=True,
                             check=True).stdout
        assert "_Z7bssnrhsPPdPPKdRKjS2_S2_PS4_S5_" in ref
        assert "_Z20physical_constraintsPPdPPKdRKjS2_S2_PS4_S5_" in ref
        assert "_Z11bssnrhs_sepPPdPPKdRKjS2_S2_PS4_S5_" in ref
        assert undefined <= set(re.findall(r" [DB] (_ZN4bssn\S+)", ref))
