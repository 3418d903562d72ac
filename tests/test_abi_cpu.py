"""C-ABI checks that need no GPU: the engine library loads, exports every
function declared in include/*.h, the NeighList container behaves like the
reference's nblist.c, and API misuse is reported with AGBNP_ERR before any
device work (agbnp3.c:138-141, 296-299, 504-511, 568-578)."""
import ctypes
import os
import re

import numpy as np
import pytest

import agbnp3_b200 as A
from conftest import ROOT

HEADERS = ["agbnp3.h", "nblist.h", "agbnp3_b200.h"]


def declared_functions():
    names = []
    for h in HEADERS:
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b([a-z_][a-z0-9_]*)\s*\(", src, flags=re.M):
            if not m.group(0).lstrip().startswith(("#", "typedef", "return")):
                names.append(m.group(1))
    return sorted(set(names))


def test_library_loads_and_exports_every_declared_symbol():
    L = A.lib()
    names = declared_functions()
    assert len(names) >= 34
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_readme_aliases_exported():
    L = A.lib()
    for n in ("agbnp_initialize", "agbnp_terminate", "agbnp_delete"):
        assert hasattr(L, n)


def test_nblist_container():
    L = A.lib()
    nl = A.NeighList()
    L.nblist_reset_neighbor_list(ctypes.byref(nl))
    assert nl.natoms == 0 and not nl.nne
    L.nblist_reallocate_neighbor_list.argtypes = [ctypes.POINTER(A.NeighList), ctypes.c_int, ctypes.c_int]
    assert L.nblist_reallocate_neighbor_list(ctypes.byref(nl), 4, 6) == 0
    assert nl.natoms == 4 and nl.neighl_size == 6
    for i, k in enumerate((1, 2, 2, 1)):
        nl.nne[i] = k
    L.nblist_reallocate_neighbor_list(ctypes.byref(nl), 4, 6)  # no change in size
    for k, j in enumerate([1, 0, 2, 1, 3, 2]):
        nl.neighl1[k] = j
    # growing the storage keeps contents and re-points neighl into it
    assert L.nblist_reallocate_neighbor_list(ctypes.byref(nl), 4, 100) == 0
    rows = [[nl.neighl[i][j] for j in range(nl.nne[i])] for i in range(4)]
    assert rows == [[1], [0, 2], [1, 3], [2]]
    L.nblist_delete_neighbor_list(ctypes.byref(nl))


def test_api_misuse_without_device():
    L = A.lib()
    L.agbnp3_terminate()  # not initialized: error message, no crash
    assert L.agbnp3_delete(0) == A.AGBNP_ERR
    assert L.agbnp3_ener_resident(0) == A.AGBNP_ERR
    assert L.agbnp3_initialize() == A.AGBNP_OK
    assert L.agbnp3_initialize() == A.AGBNP_OK  # idempotent
    assert L.agbnp3_delete(-1) == A.AGBNP_ERR
    assert L.agbnp3_delete(12345) == A.AGBNP_ERR
    s = A.make_globule(40, 1)
    with pytest.raises(A.AGBNPError, match="NULL connection table"):
        A.new(s, conntbl=False)
    bad = s.with_coords(s.coords())
    bad.ihydrogen = np.array([s.natoms + 3], np.int32)
    with pytest.raises(A.AGBNPError, match="out of range"):
        A.new(bad)
    assert L.agbnp3_set_device(-2) == A.AGBNP_ERR
    L.agbnp3_terminate()


def test_stage_names():
    L = A.lib()
    names = [L.agbnp3_stage_name(k).decode() for k in range(10)]
    assert names == ["prep", "nblist", "volumes", "scaling", "invb", "agb", "gbders", "ws", "treeders", "final"]
