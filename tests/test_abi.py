"""CPU tests of the drop-in boundary: the C-ABI libraries load and export every declared symbol."""
import ctypes as C
import os
import re

from tests.conftest import ROOT


def _declared(header):
    src = open(header).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return set(re.findall(r"^\s*(?:const\s+char\s*\*|int|void|double)\s+(\w+)\s*\(", src, re.M))


def test_library_exports_every_header_symbol():
    from glmmhdturb_b200 import _lib
    names = _declared(os.path.join(ROOT, "include", "glmmhd_b200.h"))
    assert len(names) == 49
    L = C.CDLL(_lib.LIB_PATH)
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing
    assert names == set(_lib.EXPORTS)


def test_legacy_bridge_symbols_match_marchbridge():
    # MarchBridge.jl:34-42 dlsyms march_nv, march_nx, march_set_dtdx, march_run_dev, march_set_glm;
    # set_gamma (:58) march_set_gamma; build_ct.sh / spike_ctm.cu: ct_run, ct_regs, ct_shmem.
    from glmmhdturb_b200 import _lib
    L = C.CDLL(_lib.LIB_PATH)
    for n in ("march_nv", "march_nx", "march_set_dtdx", "march_run_dev", "march_set_glm", "march_set_gamma",
              "march_nsp", "ct_run", "ct_regs", "ct_shmem"):
        assert hasattr(L, n), n
    L.march_nv.restype = C.c_int
    assert L.march_nv() == 9   # no CUDA call


def test_version_string_without_gpu():
    import glmmhdturb_b200 as G
    assert "sm_100a" in G.version()


def test_oracle_exports_header_symbols():
    from oracle import oracle as O
    names = _declared(os.path.join(ROOT, "oracle", "gmt_oracle.h"))
    L = C.CDLL(O.LIB_PATH)
    assert names and all(hasattr(L, n) for n in names)


def test_struct_layouts():
    from glmmhdturb_b200 import _lib
    # gmt_params: 15 int32 + 13 double + int32 + uint32 = 60 + 4 pad... checked against offsets
    assert C.sizeof(_lib.GmtStepArgs) == 40
    assert C.sizeof(_lib.GmtDiag) == 72
    assert _lib.GmtParams.boxlen.offset == 60 + 4 and C.sizeof(_lib.GmtParams) == 64 + 13 * 8 + 8


def test_host_argument_errors_need_no_gpu():
    from glmmhdturb_b200 import turb
    import pytest
    with pytest.raises(ValueError):
        turb.step_plm(None, None, None, turb.Params(N=16), 1e-3, 0.0, tb=6)
    with pytest.raises(ValueError):
        turb.step_tiled(None, None, None, turb.Params(N=18), 1e-3, 0.0)
    ch, fac = turb.glm_parameters(turb.Params(N=64), 1e-3)
    assert abs(ch - 0.7 / 64 / 1e-3 / 3 * 0.25) < 1e-12 and 0 < fac < 1
