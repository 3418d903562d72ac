"""The reference's float interface (float_i = float when a caller builds
with SINGLE_PREC_INTERFACE, agbnp3.h:44-50): libagbnp3_b200_sp.so exports
the same entry points with float arrays, converts them and runs the same
evaluation."""
import ctypes
import os

import numpy as np
import pytest

import agbnp3_b200 as A
from conftest import ENERGY_KEYS, load_golden, rms_rel
from test_abi_cpu import declared_functions

SP = os.path.join(os.path.dirname(A.__file__), "libagbnp3_b200_sp.so")
_fp = ctypes.POINTER(ctypes.c_float)
_ip = ctypes.POINTER(ctypes.c_int)


def _sp():
    L = ctypes.CDLL(SP)
    L.agbnp3_new.argtypes = ([_ip, ctypes.c_int] + [_fp] * 5 + [ctypes.c_float] * 2 + [_fp] * 4 +
                             [_ip, _fp, ctypes.c_int, _ip, ctypes.POINTER(A.NeighList), ctypes.c_int])
    L.agbnp3_ener.argtypes = ([ctypes.c_int, ctypes.c_int] + [_fp] * 17)
    L.agbnp3_delete.argtypes = [ctypes.c_int]
    return L


def test_float_library_exports_the_reference_api():
    L = ctypes.CDLL(SP)
    names = [n for n in declared_functions() if n.startswith(("agbnp3_initialize", "agbnp3_terminate", "agbnp3_new",
                                                               "agbnp3_delete", "agbnp3_ener", "nblist_"))]
    assert {"agbnp3_new", "agbnp3_ener", "nblist_reallocate_neighbor_list"} <= set(names)
    assert not [n for n in names + ["agbnp_initialize", "agbnp_terminate", "agbnp_delete"] if not hasattr(L, n)]


@pytest.mark.gpu
def test_float_interface_matches_double():
    """The 300-atom golden system through agbnp3_new / agbnp3_ener with float
    arrays (libagbnp3_b200_sp.so) against the double interface: the inputs
    differ by their rounding to float (relative 6e-8), so energies agree to
    1e-5 and per-atom outputs and forces to 1e-4 RMS (the tolerances of the
    mixed-precision parity tests)."""
    s, _ = load_golden("globule300_shuffled")
    A.initialize()
    R = A.Instance(s).ener()
    L = _sp()
    assert L.agbnp3_initialize() == A.AGBNP_OK
    f = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.float32))  # noqa: E731
    pf = lambda a: a.ctypes.data_as(_fp)  # noqa: E731
    x, y, z, r, q, ig, sg, ia, sa, hbc = (f(getattr(s, k)) for k in ("x", "y", "z", "r", "charge", "igamma", "sgamma",
                                                                      "ialpha", "salpha", "hbcorr"))
    hbt = np.ascontiguousarray(s.hbtype, dtype=np.int32)
    ih = np.ascontiguousarray(s.ihydrogen, dtype=np.int32)
    nl, keep = A.neighlist(s)
    tag = ctypes.c_int(-1)
    rc = L.agbnp3_new(ctypes.byref(tag), s.natoms, pf(x), pf(y), pf(z), pf(r), pf(q), s.eps_in, s.eps_out, pf(ig),
                      pf(sg), pf(ia), pf(sa), hbt.ctypes.data_as(_ip), pf(hbc), int(ih.shape[0]),
                      ih.ctypes.data_as(_ip), ctypes.byref(nl), 0)
    assert rc == A.AGBNP_OK
    n = s.natoms
    out = {k: np.zeros(n, np.float32) for k in ("sp", "br", "surf_area")}
    out.update({k: np.zeros((n, 3), np.float32) for k in ("dgbdr", "dvwdr", "decav", "dehb")})
    e = {k: ctypes.c_float() for k in ("mol_volume", "egb", "evdw", "ecorr_vdw", "ecav", "ecorr_cav", "ehb")}
    rc = L.agbnp3_ener(tag.value, 0, pf(x), pf(y), pf(z), pf(out["sp"]), pf(out["br"]), ctypes.byref(e["mol_volume"]),
                       pf(out["surf_area"]), ctypes.byref(e["egb"]), pf(out["dgbdr"]), ctypes.byref(e["evdw"]),
                       ctypes.byref(e["ecorr_vdw"]), pf(out["dvwdr"]), ctypes.byref(e["ecav"]),
                       ctypes.byref(e["ecorr_cav"]), pf(out["decav"]), ctypes.byref(e["ehb"]), pf(out["dehb"]))
    assert rc == A.AGBNP_OK
    for k in ENERGY_KEYS:
        assert abs(e[k].value - R[k]) <= 1e-5 * max(abs(R[k]), 10.0), (k, e[k].value, R[k])
    for k in ("sp", "br", "surf_area", "dgbdr", "dvwdr", "decav", "dehb"):
        assert rms_rel(out[k].astype(np.float64), R[k]) <= 1e-4, (k, rms_rel(out[k].astype(np.float64), R[k]))
    assert L.agbnp3_delete(tag.value) == A.AGBNP_OK
