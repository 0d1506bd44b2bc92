"""The C-ABI library loads without a GPU and exports what the header declares."""

from __future__ import annotations

import ctypes as C

import numpy as np

from lithobat_b200 import _native as nat


def test_library_loads_and_reports_version():
    L = nat.lib()
    assert L.litho_version() >= 100


def test_every_declared_symbol_is_exported():
    L = nat.lib()
    names = nat.exported_symbols()
    assert "litho_abbe" in names and "litho_status_string" in names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_struct_sizes_match_the_python_layouts():
    L = nat.lib()
    L.litho_abi_sizes.restype = C.c_int
    out = (C.c_int32 * 16)()
    k = L.litho_abi_sizes(out, 16)
    sizes = list(out)[:k]
    assert sizes[:8] == [nat.PUPIL_DTYPE.itemsize, nat.JOB_DTYPE.itemsize, nat.ITEM_DTYPE.itemsize,
                         nat.NORM_DTYPE.itemsize, C.sizeof(nat.AbbePlan), nat.MIRROR_DTYPE.itemsize,
                         C.sizeof(nat.UnevenGroup), nat.QUEUE_TASK_DTYPE.itemsize]


def test_status_strings():
    L = nat.lib()
    assert L.litho_status_string(0) == b"ok"
    assert b"workspace" in L.litho_status_string(-3)
    assert L.litho_status_string(-99) == b"unknown status"


def test_bad_plans_are_rejected_before_any_launch():
    """Argument checks run on the host and need no device."""
    L = nat.lib()
    p = nat.AbbePlan(n=64, n_clips=1, n_out=1, n_jobs=1, n_items=1, n_pupils=1, h=3, bm=3, L=32,
                     mask_complex=0, ncomp_max=1, n_tab=1, pixel_size=4e-9)
    sz = C.c_size_t(0)
    assert L.litho_abbe_workspace(C.byref(p), C.byref(sz)) == 0 and sz.value > 0
    bad = nat.AbbePlan.from_buffer_copy(p); bad.h = 8          # 4h+1 > 32
    assert L.litho_abbe_workspace(C.byref(bad), C.byref(sz)) == -4
    bad = nat.AbbePlan.from_buffer_copy(p); bad.L = 48
    assert L.litho_abbe_workspace(C.byref(bad), C.byref(sz)) == -5
    bad = nat.AbbePlan.from_buffer_copy(p); bad.off_pupils = 8
    assert L.litho_abbe_workspace(C.byref(bad), C.byref(sz)) == -6
    bad = nat.AbbePlan.from_buffer_copy(p); bad.n = 0
    assert L.litho_abbe_workspace(C.byref(bad), C.byref(sz)) == -2
    bad = nat.AbbePlan.from_buffer_copy(p); bad.n_tab = 2       # more slots than jobs
    assert L.litho_abbe_workspace(C.byref(bad), C.byref(sz)) == -2
    # workspace too small / null pointers: rejected without touching the device
    assert L.litho_abbe(C.byref(p), None, None, None, None, None, 0, None) == -1
    buf = np.zeros(64, np.uint8)
    ptr = buf.ctypes.data
    assert L.litho_abbe(C.byref(p), ptr, ptr, ptr, ptr, ptr, 16, None) == -3
