"""The C-ABI libraries load and export every symbol their headers declare.

CPU only: loads the libraries, calls nothing that needs a GPU.
"""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    src = open(os.path.join(ROOT, header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(\w+)\s*\([^;{]*\)\s*;", src, flags=re.M)
    return sorted(set(n for n in names if n.startswith(("cgx_", "orc_"))))


def test_cgx_exports_every_declared_symbol(built):
    from nextgen_b200 import _lib, cgx
    names = declared("include/cgx.h")
    assert len(names) >= 25
    L = ctypes.CDLL(_lib.path("libcgx.so"))
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(cgx.EXPORTS) <= set(names)


def test_cgx_exports_every_operator_build_symbol(built):
    from nextgen_b200 import _lib
    names = declared("include/cgx_ops.h")
    assert names == ["cgx_operators_build", "cgx_operators_free"]
    L = ctypes.CDLL(_lib.path("libcgx.so"))
    assert all(hasattr(L, n) for n in names)


def test_operator_build_checks_arguments_before_the_device(built):
    """Invalid descriptors fail on the host with CGX_E_ARG (no GPU needed)."""
    from nextgen_b200 import meshgen
    L = meshgen._ops_lib()
    out = ctypes.POINTER(meshgen.MeshgenOut)()
    assert L.cgx_operators_build(None, 1.0 / 3.0, 0.45, 0, ctypes.byref(out), None) == -1
    d = meshgen.CompactDesc()  # ncv = 0, no arrays
    assert L.cgx_operators_build(ctypes.byref(d), 1.0 / 3.0, 0.45, 0, ctypes.byref(out), None) == -1
    assert b"invalid argument" in L.cgx_last_error()
    m = meshgen.PeriodicBoxMesh(6, jitter=0.1)
    d = meshgen.compact_desc(m)
    assert L.cgx_operators_build(ctypes.byref(d), 1.0 / 3.0, 0.45, 0, None, None) == -1
    d.L[1] = 0.0
    assert L.cgx_operators_build(ctypes.byref(d), 1.0 / 3.0, 0.45, 0, ctypes.byref(out), None) == -1
    assert not out


def test_meshgen_exports_every_declared_symbol(built):
    from nextgen_b200 import _lib
    names = declared("include/cgx_meshgen.h")
    L = ctypes.CDLL(_lib.path("libcgx_meshgen.so"))
    assert names and all(hasattr(L, n) for n in names)


def test_meshgen_exports_every_mles_symbol(built):
    from nextgen_b200 import _lib
    names = declared("include/cgx_mles.h")
    assert names == ["cgx_mles_free", "cgx_mles_last_error", "cgx_mles_read", "cgx_sles_read", "cgx_sles_write"]
    L = ctypes.CDLL(_lib.path("libcgx_meshgen.so"))
    assert all(hasattr(L, n) for n in names)


def test_oracle_exports_every_declared_symbol(built):
    names = declared("oracle/oracle.h")
    L = ctypes.CDLL(os.path.join(ROOT, "oracle", "liboracle.so"))
    assert names and all(hasattr(L, n) for n in names)


def test_params_default_are_the_reference_defaults(built):
    from nextgen_b200 import cgx
    p = cgx.Params()
    cgx.lib().cgx_params_default(ctypes.byref(p))
    # IdealGasSolver.hpp:147-155, IdealGasSolverSgs.cpp:209-213, IdealGasSolver.cpp:202-203,904
    assert p.gamma == 1.4 and p.mu_power_law == 0.75 and p.Pr_lam == 0.7
    assert p.vreman_coeff == 0.07 and p.a_sgs_coeff == 0.05 and p.a_sgs_coeff2 == 0.0015
    assert p.lambda_dil_coeff == 0.0 and p.Pr_t == 0.9
    assert p.coeff_p == 0.5 and p.coeff_h == 0.1 and p.gr_nrm == 0.03
    q = cgx.Params()
    for f, _ in cgx.Params._fields_:
        if f != "dt_data":
            assert getattr(q, f) == getattr(p, f), f


def test_libcgx_is_sm100a_only(built):
    """The CUDA library carries sm_100a code and nothing else."""
    import subprocess
    from nextgen_b200 import _lib
    out = subprocess.run(["cuobjdump", "--list-elf", _lib.path("libcgx.so")],
                         stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True).stdout
    arches = set(re.findall(r"sm_(\d+a?)", out))
    assert arches == {"100a"}, out


def test_product_never_imports_the_oracle():
    pkg = os.path.join(ROOT, "nextgen_b200")
    for dp, _, fs in os.walk(pkg):
        for f in fs:
            if f.endswith((".py", ".cu", ".cuh", ".cpp", ".h")):
                txt = open(os.path.join(dp, f)).read()
                assert "import oracle" not in txt and "from oracle" not in txt, f
                assert "liboracle" not in txt and "libref" not in txt, f


def test_gpu_paths_fail_loudly_without_a_gpu(built):
    """No CPU fallback: without a CUDA device the mesh upload and the operator
    build return CGX_E_CUDA (-3) instead of computing anything on the host."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from nextgen_b200 import cgx, meshgen
    m = meshgen.PeriodicBoxMesh(6, jitter=0.1)
    with pytest.raises(cgx.CgxError) as e:
        meshgen.DeviceOperatorMesh(m)
    assert e.value.code == -3
    with pytest.raises(cgx.CgxError) as e:
        cgx.Mesh(m, device=0)
    assert e.value.code == -3
