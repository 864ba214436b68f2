"""The C-ABI library loads and exports every entry point include/gamgpu.h
declares (no GPU work)."""
import ctypes as C
import os
import re

from mage_b200 import gamera

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(ROOT, "include", "gamgpu.h")).read()
    return sorted(set(re.findall(r"\b(?:int|const char\*)\s+(gam_\w+)\s*\(", src)))


def test_header_lists_all_python_bindings():
    assert set(declared()) == set(gamera.EXPORTED)


def test_library_exports_every_symbol():
    """Both builds: the product library and the bounds-check one."""
    for path in (gamera.LIB_PATH, gamera.CHECK_LIB_PATH):
        lib = C.CDLL(path)
        for name in declared():
            assert hasattr(lib, name), (path, name)


def test_default_params_match_reference():
    L = gamera.load_library()
    p = gamera._Params()
    assert L.gam_default_params(C.byref(p), 64, 64, 1) == 0
    assert abs(p.gamma - 5.0 / 3.0) < 1e-15 and p.pdmb == 0.75 and abs(p.CFL - 0.3) < 1e-15
    assert p.Vd0 == 0.5 and p.cHogH == 0.25 and p.dFloor == 1e-12 and p.do25D == 1 and p.nG == 4


def test_fortran_module_binds_every_entry_point():
    """mage_b200/fortran/gamgpu.F90 declares a bind(C) interface for every
    function of the header, and its gam_params type has the C struct's fields
    in the same order."""
    src = open(os.path.join(ROOT, "mage_b200", "fortran", "gamgpu.F90")).read()
    bound = set(re.findall(r'bind\(C, name="(gam_\w+)"\)', src))
    assert set(declared()) <= bound, sorted(set(declared()) - bound)
    body = src[src.index("type, bind(C) :: gam_params"):src.index("end type gam_params")]
    names = []
    for line in body.splitlines()[1:]:
        if "::" in line:
            names += [n.strip().split("(")[0] for n in line.split("::")[1].split(",") if n.strip()]
    assert names == [f for f, _ in gamera._Params._fields_], names


def test_whole_step_work_bytes_and_coverage():
    """gam_step_work_bytes (host arithmetic only): the work area of the
    whole-step adjoint is 413 box-sized arrays (66 of them the flux kernels'
    face states, 22 per face and direction, 30 the edge kernels' corner
    values, 10 per edge and direction, and 171 the scratch of the flux and
    edge adjoints' gathers), each started on 256 bytes, and
    14 more with non-periodic I boundaries (the update's result, its field
    and that field's adjoint); the entry points refuse what the adjoint does
    not cover (one I side periodic and the other not, Boris, 7UP)."""
    L = gamera.load_library()
    nb = C.c_int64()
    N = (16, 24, 8)
    box = (N[0] + 9) * (N[1] + 9) * (N[2] + 9)
    nc = [5, 5, 1, 3, 3, 3, 3, 3, 9, 3, 3, 15, 9, 66, 30, 5, 5, 1, 3, 3, 3, 3, 3, 3, 3, 15, 9, 3, 5, 3, 3, 5, 3, 3,
          171]
    assert sum(nc) == 413
    for fp32, es in ((0, 8), (1, 4)):
        p = gamera.GamParams(*N).to_c()
        assert L.gam_step_work_bytes(C.byref(p), fp32, C.byref(nb)) == 0
        assert nb.value == sum((c * box * es + 255) // 256 * 256 for c in nc)
    p = gamera.GamParams(*N, bc=(0, 0, 2, 2, 0, 0)).to_c()
    assert L.gam_step_work_bytes(C.byref(p), 0, C.byref(nb)) == 0
    for bc in ((6, 2, 2, 2, 0, 0), (3, 4, 2, 2, 0, 0), (6, 2, 0, 0, 0, 0)):
        p = gamera.GamParams(*N, bc=bc).to_c()
        assert L.gam_step_work_bytes(C.byref(p), 0, C.byref(nb)) == 0
        assert nb.value == sum((c * box * 8 + 255) // 256 * 256 for c in nc + [5, 3, 3, 3])
    for kw in ({"bc": (6, 0, 2, 2, 0, 0)}, {"bc": (0, 4, 0, 0, 0, 0)}, {"doBoris": True, "Ca": 1.0},
               {"rmeth": gamera.RECON_7UP}):
        p = gamera.GamParams(*N, **kw).to_c()
        assert L.gam_step_work_bytes(C.byref(p), 0, C.byref(nb)) == gamera.GAM_EINVAL, kw
