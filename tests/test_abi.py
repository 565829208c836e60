"""The C-ABI library loads and exports every symbol include/negf_b200.h
declares (no GPU needed, no compute calls)."""
import ctypes
import os
import re

import pytest

from libnegf_b200 import native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "negf_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(negf_b200_\w+)\s*\(", src)))


def test_header_and_binding_agree():
    assert declared_symbols() == sorted(native.EXPORTED)


def test_library_exports_every_declared_symbol():
    L = native.load()
    for name in declared_symbols():
        assert hasattr(L, name), name


def test_version_and_defaults():
    assert "sm_100a" in native.version()
    o = native.Options()
    native.load().negf_b200_default_options(ctypes.byref(o))
    assert o.sgf_tol == 1e-9 and o.sgf_max_iter == 300 and o.scba_tol == 1e-7 and o.eps_drop == 0.0
    assert o.scba_mix == 1.0 and o.scba_rule == 0


def test_no_gpu_is_an_error_not_a_fallback():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(native.NegfError) as ei:
        native.Context(0)
    assert ei.value.code == native.NO_GPU


def test_bad_arguments_are_rejected_without_gpu():
    L = native.load()
    assert L.negf_b200_ctx_create(0, None) == native.BAD_ARG
    assert L.negf_b200_zinv_batched(1, -1, None, None, None, None, None) == native.BAD_ARG
    assert L.negf_b200_decimation_batched(1, 4, None, None, None, None, None, -1.0, 10, None, None) == native.BAD_ARG


def test_fortran_binding_covers_the_header():
    """fortran/negf_b200_bind.F90 (uncompiled on this image) binds every
    function the header declares, under the header's names, and nothing else
    of this library; its derived types list the C structs' fields in order."""
    src = open(os.path.join(ROOT, "fortran", "negf_b200_bind.F90")).read()
    bound = set(re.findall(r"bind\(C,\s*name='(negf_b200_\w+)'\)", src))
    assert bound == set(declared_symbols())
    hdr = re.sub(r"/\*.*?\*/", "", open(os.path.join(ROOT, "include", "negf_b200.h")).read(), flags=re.S)
    for cname, ftype in (("negf_b200_device", "negf_b200_device"), ("negf_b200_options", "negf_b200_options")):
        body = re.search(r"typedef struct %s \{(.*?)\}" % cname, hdr, flags=re.S).group(1)
        cfields = re.findall(r"(\w+)\s*;", body)
        fbody = re.search(r"type, bind\(C\) :: %s(.*?)end type" % ftype, src, flags=re.S).group(1)
        ffields = []
        for line in fbody.splitlines():
            if "::" in line:
                ffields += [f.strip() for f in line.split("::")[1].split(",")]
        assert ffields == cfields, (cname, ffields, cfields)


def test_fortran_backend_exports_the_seam_names():
    """fortran/iterative_b200.F90 exports the public names of libNEGF's GPU
    RGF backend (src/iterative_gpu.F90:44-50) and the decimation seam."""
    src = open(os.path.join(ROOT, "fortran", "iterative_b200.F90")).read()
    public = set(re.findall(r"public :: (\w+)", src))
    assert {"calculate_gsmr_blocks", "calculate_Gr_tridiag_blocks", "calculate_Gn_tridiag_blocks",
            "calculate_single_transmission_2_contacts", "calculate_single_transmission_N_contacts",
            "check_convergence_trid", "check_convergence_vec", "decimation_b200"} <= public
    for name in public:
        assert re.search(r"subroutine %s\(" % name, src), name
