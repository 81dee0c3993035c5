"""C-ABI checks that need no GPU: the library loads, exports every entry point
declared in include/bosss_b200.h, and rejects bad or unsupported operators before
touching a device (the error behaviour of DifferentialOperator.cs:1022-1023 / 1590-1591)."""
import ctypes
import os
import re

import numpy as np
import pytest

from bosss_b200 import _capi as C
from bosss_b200 import operator as O
from bosss_b200 import problems as P

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_symbols():
    src = open(os.path.join(ROOT, "include", "bosss_b200.h")).read()
    return sorted(set(re.findall(r"\bint\s+(bosss_b200_\w+)\s*\(", src)))


def test_library_exports_every_header_symbol():
    L = C.lib()
    syms = _header_symbols()
    assert len(syms) >= 18
    for s in syms:
        assert hasattr(L, s), s
        assert s in C.SIGNATURES, s


def test_version():
    a, b, c = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
    C.check(C.lib().bosss_b200_version(ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
    assert (a.value, b.value) == (0, 3)


def _create(opd, gd, kernel=C.KERNEL_AUTO):
    h = ctypes.c_void_p()
    opt = C.Options()
    opt.kernel = kernel
    rc = C.lib().bosss_b200_create(ctypes.byref(opd), ctypes.byref(gd), ctypes.byref(opt), ctypes.byref(h))
    if rc == 0:
        C.lib().bosss_b200_destroy(h)
    return rc, C.last_error()


def test_unknown_component_is_rejected():
    pr = P.transport2d(n=4, k=2)
    opd, gd = pr.descs()
    opd.components[0].type = 99
    rc, msg = _create(opd, gd)
    assert rc == C.ERR_UNSUPPORTED_COMPONENT
    assert "no device functor" in msg


def test_mixed_degrees_rejected():
    pr = P.euler3d(n=2, k=2)
    opd, gd = pr.descs()
    opd.domain_degree[1] = 1
    rc, msg = _create(opd, gd)
    assert rc == C.ERR_BAD_ARG


def test_non_periodic_euler_accepted_on_generic_kernel_only():
    """HLLC with boundary faces (outer states from the boundary-state table) passes the
    operator checks (on a machine without a GPU create then stops at the device); the slab
    and face-once kernels, which do not read the table, are refused."""
    pr = P.euler3d(n=2, k=1)
    opd, gd = pr.descs()
    gd.periodic[0] = 0
    rc, msg = _create(opd, gd)
    assert rc in (C.OK, C.ERR_NO_DEVICE), msg
    for kern in (C.KERNEL_SLAB, C.KERNEL_FACES):
        rc, msg = _create(opd, gd, kern)
        assert rc == C.ERR_BAD_ARG, msg


def test_incomplete_hllc_set_rejected():
    pr = P.euler3d(n=2, k=1)
    opd, gd = pr.descs()
    opd.n_components = 4
    rc, _ = _create(opd, gd)
    assert rc == C.ERR_UNSUPPORTED_COMPONENT


def test_degree_out_of_range_rejected():
    pr = P.transport2d(n=4, k=2)
    opd, gd = pr.descs()
    opd.domain_degree[0] = opd.codomain_degree[0] = 6
    rc, _ = _create(opd, gd)
    assert rc == C.ERR_BAD_ARG


def test_bad_grid_rejected():
    pr = P.transport2d(n=4, k=2)
    opd, gd = pr.descs()
    gd.n[0] = 0
    rc, _ = _create(opd, gd)
    assert rc == C.ERR_BAD_ARG


def test_uncommitted_operator():
    op = O.DifferentialOperator(["u"], [], ["R"])
    op.EquationComponents["R"].Add(O.ScalarTransportFlux((1, 0), "u"))
    with pytest.raises(RuntimeError):
        op.descriptor([1], [1], 2)


def test_unknown_argument_name():
    op = O.DifferentialOperator(["u"], [], ["R"])
    op.EquationComponents["R"].Add(O.ScalarTransportFlux((1, 0), "w"))
    with pytest.raises(ValueError):
        op.Commit()


def test_nonuniform_grid_rejected():
    with pytest.raises(ValueError):
        O.Cartesian2DGrid([0, 0.1, 0.3], [0, 1])


def test_bsr_create_validates_on_host():
    rp = np.array([0, 1, 3], dtype=np.int64)
    ci = np.array([0, 5, 1], dtype=np.int32)   # 5 out of range
    v = np.zeros(3 * 4)
    A = ctypes.c_void_p()
    rc = C.lib().bosss_b200_bsr_create(2, 2, 2, 2, C.ptr(rp), C.ptr(ci), C.ptr(v), 0, ctypes.byref(A))
    assert rc == C.ERR_BAD_ARG


def test_cell_order_permutation_metadata():
    g1 = O.Cartesian3DGrid(np.linspace(0, 1, 3), np.linspace(0, 1, 4), np.linspace(0, 1, 5))
    g2 = O.Cartesian3DGrid(np.linspace(0, 1, 3), np.linspace(0, 1, 4), np.linspace(0, 1, 5),
                           cell_order=C.CELLS_GLOBALID)
    a, b = g1.cell_ijk(), g2.cell_ijk()
    # generator order: z fastest; GlobalID: x fastest (Grid3D.cs:232-249)
    assert tuple(a[1]) == (0, 0, 1) and tuple(b[1]) == (1, 0, 0)
    assert sorted(map(tuple, a)) == sorted(map(tuple, b))
