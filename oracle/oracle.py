"""ctypes binding of the FP64 oracle and of the reference library.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py (cpu_baseline leg and reference arm).  The product package never
imports this module.

- :func:`oracle_eval` runs the FP64 C restatement (oracle/agbnp3_oracle.c)
  on a System and returns energies, outputs and intermediates.
- :class:`RefLib` drives the reference AGBNP3 library built unmodified from
  its sources (oracle/_ref/libagbnp3_refh.so, see oracle/Makefile) through
  its own public API (agbnp3.h:77-104) and exposes internals for parity
  tests.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "_build", "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libagbnp3_ref.so")
REFH_LIB = os.path.join(HERE, "_ref", "libagbnp3_refh.so")

MAX_ORDER = 5
NA = 512

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


class OrcIn(ctypes.Structure):
    _fields_ = [("natoms", ctypes.c_int), ("nheavy", ctypes.c_int),
                ("x", _dp), ("y", _dp), ("z", _dp), ("r", _dp), ("charge", _dp),
                ("igamma", _dp), ("sgamma", _dp), ("ialpha", _dp), ("salpha", _dp),
                ("hbtype", _ip), ("hbcorr", _dp), ("conn_offset", _ip), ("conn_list", _ip),
                ("eps_in", ctypes.c_double), ("eps_out", ctypes.c_double), ("compat", ctypes.c_int)]


class OrcOut(ctypes.Structure):
    _fields_ = [("egb", ctypes.c_double), ("evdw", ctypes.c_double), ("ecorr_vdw", ctypes.c_double),
                ("ecav", ctypes.c_double), ("ecorr_cav", ctypes.c_double), ("ehb", ctypes.c_double),
                ("mol_volume", ctypes.c_double),
                ("sp", _dp), ("br", _dp), ("surf_area", _dp), ("dgbdr", _dp), ("dvwdr", _dp),
                ("decav", _dp), ("dehb", _dp),
                ("volumep", _dp), ("surf_raw", _dp), ("spe", _dp), ("br1", _dp), ("dera", _dp),
                ("deru", _dp), ("derv", _dp), ("derh", _dp),
                ("q2ab", _dp), ("abrw", _dp), ("psvol", _dp), ("gammap", _dp), ("derus", _dp), ("dervs", _dp),
                ("nl_count", _ip), ("nl_list", _ip), ("nl_cap", ctypes.c_int), ("nl_total", ctypes.c_int),
                ("cand_cap", ctypes.c_int), ("cand_total", ctypes.c_int),
                ("cand_order", _ip), ("cand_parents", _ip), ("cand_gvol", _dp), ("cand_gvolp", _dp),
                ("n_kept", ctypes.c_int * (MAX_ORDER + 1)),
                ("ws_cap", ctypes.c_int), ("nws", ctypes.c_int),
                ("ws_pos", _dp), ("ws_sp", _dp), ("ws_parent0", _ip), ("ws_type", _ip),
                ("tab_cap", ctypes.c_int), ("ntypes", ctypes.c_int), ("tab_y", _dp), ("tab_y2", _dp),
                ("rtype", _ip)]


def _p(a, t):
    return a.ctypes.data_as(t)


_oracle = None


def _lib():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_LIB):
            raise RuntimeError(f"{ORACLE_LIB} missing; run `make -C oracle`")
        _oracle = ctypes.CDLL(ORACLE_LIB)
        _oracle.agbnp3_oracle_eval.argtypes = [ctypes.POINTER(OrcIn), ctypes.POINTER(OrcOut)]
        _oracle.agbnp3_oracle_eval.restype = ctypes.c_int
    return _oracle


def internal_arrays(system):
    """The system's inputs permuted to internal order (heavy first) with the
    radius increment of agbnp3.c:210 applied and the connection table
    remapped (agbnp3.c:308-317)."""
    int2ext, ext2int = system.internal_order()
    off, lst = system.conn_csr()
    cnt = np.diff(off)
    ioff = np.zeros(system.natoms + 1, dtype=np.int32)
    ioff[1:] = np.cumsum(cnt[int2ext])
    ilst = np.concatenate([ext2int[lst[off[e]:off[e + 1]]] for e in int2ext]).astype(np.int32) \
        if lst.size else np.zeros(0, np.int32)
    d = {k: np.ascontiguousarray(getattr(system, k)[int2ext], dtype=np.float64)
         for k in ("x", "y", "z", "charge", "igamma", "sgamma", "ialpha", "salpha", "hbcorr")}
    d["r"] = np.ascontiguousarray(system.r[int2ext] + 0.5)
    d["hbtype"] = np.ascontiguousarray(system.hbtype[int2ext], dtype=np.int32)
    d["conn_offset"], d["conn_list"] = ioff, np.ascontiguousarray(ilst)
    d["int2ext"], d["ext2int"] = int2ext, ext2int
    return d


def oracle_eval(system, compat: bool = True, internals: bool = False, cand_cap: int = 0):
    """FP64 evaluation.  Returns a dict with energies and per-atom outputs in
    EXTERNAL order (like agbnp3_ener), and, when `internals`, intermediates
    in internal order under key 'int'."""
    lib = _lib()
    a = internal_arrays(system)
    n, nh = system.natoms, system.nheavy
    ci = OrcIn()
    ci.natoms, ci.nheavy = n, nh
    for k in ("x", "y", "z", "r", "charge", "igamma", "sgamma", "ialpha", "salpha", "hbcorr"):
        setattr(ci, k, _p(a[k], _dp))
    ci.hbtype = _p(a["hbtype"], _ip)
    ci.conn_offset = _p(a["conn_offset"], _ip)
    ci.conn_list = _p(a["conn_list"], _ip) if a["conn_list"].size else _p(np.zeros(1, np.int32), _ip)
    ci.eps_in, ci.eps_out, ci.compat = system.eps_in, system.eps_out, int(compat)

    co = OrcOut()
    keep = {}

    def arr(name, size, dtype=np.float64):
        v = np.zeros(size, dtype=dtype)
        keep[name] = v
        setattr(co, name, _p(v, _dp if dtype == np.float64 else _ip))
        return v

    for k in ("sp", "br", "surf_area"):
        arr(k, n)
    for k in ("dgbdr", "dvwdr", "decav", "dehb"):
        arr(k, 3 * n)
    if internals:
        for k in ("volumep", "surf_raw", "spe", "br1", "dera", "deru", "derv", "derh", "q2ab", "abrw", "psvol",
                  "gammap", "derus", "dervs"):
            arr(k, n)
        arr("nl_count", max(nh, 1), np.int32)
        co.nl_cap = 64 * nh + 16
        arr("nl_list", co.nl_cap, np.int32)
        co.ws_cap = 4 * n + 4
        arr("ws_pos", 3 * co.ws_cap)
        arr("ws_sp", co.ws_cap)
        arr("ws_parent0", co.ws_cap, np.int32)
        arr("ws_type", co.ws_cap, np.int32)
        co.tab_cap = 64 * 64 * NA // 16
        arr("tab_y", co.tab_cap)
        arr("tab_y2", co.tab_cap)
        arr("rtype", n, np.int32)
    if cand_cap:
        co.cand_cap = cand_cap
        arr("cand_order", cand_cap, np.int32)
        arr("cand_parents", MAX_ORDER * cand_cap, np.int32)
        arr("cand_gvol", cand_cap)
        arr("cand_gvolp", cand_cap)
    rc = lib.agbnp3_oracle_eval(ctypes.byref(ci), ctypes.byref(co))
    int2ext = a["int2ext"]
    res = dict(rc=rc, egb=co.egb, evdw=co.evdw, ecorr_vdw=co.ecorr_vdw, ecav=co.ecav, ecorr_cav=co.ecorr_cav,
               ehb=co.ehb, mol_volume=co.mol_volume, n_kept=list(co.n_kept), nws=co.nws,
               cand_total=co.cand_total, nl_total=co.nl_total)
    for k in ("sp", "br", "surf_area"):
        v = np.empty(n)
        v[int2ext] = keep[k]
        res[k] = v
    for k in ("dgbdr", "dvwdr", "decav", "dehb"):
        v = np.empty((n, 3))
        v[int2ext] = keep[k].reshape(n, 3)
        res[k] = v
    if internals:
        it = {k: keep[k] for k in ("volumep", "surf_raw", "spe", "br1", "dera", "deru", "derv", "derh", "q2ab",
                                    "abrw", "psvol", "gammap", "derus", "dervs", "rtype")}
        it["nl_count"] = keep["nl_count"][:nh]
        it["nl_list"] = keep["nl_list"][: co.nl_total]
        w = co.nws
        it["ws_pos"] = keep["ws_pos"][: 3 * w].reshape(w, 3)
        it["ws_sp"], it["ws_parent0"], it["ws_type"] = keep["ws_sp"][:w], keep["ws_parent0"][:w], keep["ws_type"][:w]
        nt = co.ntypes
        it["tab_y"] = keep["tab_y"][: nt * nt * NA].reshape(nt * nt, NA)
        it["tab_y2"] = keep["tab_y2"][: nt * nt * NA].reshape(nt * nt, NA)
        it["ntypes"] = nt
        res["int"] = it
    if cand_cap:
        m = min(co.cand_total, cand_cap)
        res["cand"] = dict(order=keep["cand_order"][:m], parents=keep["cand_parents"][: MAX_ORDER * m].reshape(m, MAX_ORDER),
                           gvol=keep["cand_gvol"][:m], gvolp=keep["cand_gvolp"][:m])
    return res


# ---------------------------------------------------------------------------
# reference library (built from the reference sources by oracle/Makefile)
# ---------------------------------------------------------------------------
class NeighListC(ctypes.Structure):
    """NeighList of nblist.h:36-76."""
    _fields_ = [("natoms", ctypes.c_int), ("neighl_size", ctypes.c_int), ("nne", _ip), ("neighl1", _ip),
                ("neighl", ctypes.POINTER(_ip)), ("idx_remap", ctypes.c_int), ("int2ext", _ip), ("ext2int", _ip),
                ("pbc", ctypes.c_int), ("pbc_trans1", ctypes.c_void_p), ("pbc_trans", ctypes.c_void_p),
                ("data", ctypes.c_int), ("data_index1", ctypes.c_void_p), ("data_index", ctypes.c_void_p)]


def build_neighlist(system):
    """A NeighList connection table for `system` (external indices), kept
    alive by the returned tuple."""
    off, lst = system.conn_csr()
    n = system.natoms
    nne = np.ascontiguousarray(np.diff(off).astype(np.int32))
    neighl1 = np.ascontiguousarray(lst if lst.size else np.zeros(1, np.int32))
    ptrs = (_ip * n)()
    base = neighl1.ctypes.data
    for i in range(n):
        ptrs[i] = ctypes.cast(base + 4 * int(off[i]), _ip)
    nl = NeighListC()
    nl.natoms, nl.neighl_size = n, int(lst.size)
    nl.nne, nl.neighl1 = _p(nne, _ip), _p(neighl1, _ip)
    nl.neighl = ctypes.cast(ptrs, ctypes.POINTER(_ip))
    return nl, (nne, neighl1, ptrs)


class RefLib:
    """The reference library, called through its own public API."""

    def __init__(self, harness: bool = True):
        path = REFH_LIB if harness else REF_LIB
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing; run `make -C oracle ref` where the reference sources exist")
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.agbnp3_initialize.restype = ctypes.c_int
        L.agbnp3_new.argtypes = [ctypes.POINTER(ctypes.c_int), ctypes.c_int] + [_dp] * 5 + [ctypes.c_double] * 2 + \
            [_dp] * 4 + [_ip, _dp, ctypes.c_int, _ip, ctypes.POINTER(NeighListC), ctypes.c_int]
        L.agbnp3_new.restype = ctypes.c_int
        L.agbnp3_ener.argtypes = [ctypes.c_int, ctypes.c_int] + [_dp] * 3 + [_dp] * 2 + [_dp] * 2 + [_dp, _dp] + \
            [_dp, _dp, _dp] + [_dp, _dp, _dp] + [_dp, _dp]
        L.agbnp3_ener.restype = ctypes.c_int
        L.agbnp3_delete.argtypes = [ctypes.c_int]
        self.harness = harness
        if L.agbnp3_initialize() != 2:
            raise RuntimeError("agbnp3_initialize failed")

    def new(self, system):
        s = system
        self._keep = [np.ascontiguousarray(getattr(s, k), dtype=np.float64)
                      for k in ("x", "y", "z", "r", "charge", "igamma", "sgamma", "ialpha", "salpha", "hbcorr")]
        x, y, z, r, q, ig, sg, ia, sa, hbc = self._keep
        hbt = np.ascontiguousarray(s.hbtype, dtype=np.int32)
        ih = np.ascontiguousarray(s.ihydrogen, dtype=np.int32)
        nl, keep = build_neighlist(s)
        self._keep += [hbt, ih, nl, keep]
        tag = ctypes.c_int(-1)
        rc = self.lib.agbnp3_new(ctypes.byref(tag), s.natoms, _p(x, _dp), _p(y, _dp), _p(z, _dp), _p(r, _dp),
                                 _p(q, _dp), s.eps_in, s.eps_out, _p(ig, _dp), _p(sg, _dp), _p(ia, _dp),
                                 _p(sa, _dp), _p(hbt, _ip), _p(hbc, _dp), int(ih.shape[0]),
                                 _p(ih if ih.size else np.zeros(1, np.int32), _ip), ctypes.byref(nl), 0)
        if rc != 2:
            raise RuntimeError(f"reference agbnp3_new failed rc={rc}")
        return tag.value

    def ener(self, tag, system):
        n = system.natoms
        x = np.ascontiguousarray(system.x, dtype=np.float64)
        y = np.ascontiguousarray(system.y, dtype=np.float64)
        z = np.ascontiguousarray(system.z, dtype=np.float64)
        sp, br, sa = np.zeros(n), np.zeros(n), np.zeros(n)
        g = {k: np.zeros((n, 3)) for k in ("dgbdr", "dvwdr", "decav", "dehb")}
        e = {k: ctypes.c_double(0.0) for k in ("mol_volume", "egb", "evdw", "ecorr_vdw", "ecav", "ecorr_cav", "ehb")}
        rc = self.lib.agbnp3_ener(tag, 0, _p(x, _dp), _p(y, _dp), _p(z, _dp), _p(sp, _dp), _p(br, _dp),
                                  ctypes.byref(e["mol_volume"]), _p(sa, _dp), ctypes.byref(e["egb"]),
                                  _p(g["dgbdr"], _dp), ctypes.byref(e["evdw"]), ctypes.byref(e["ecorr_vdw"]),
                                  _p(g["dvwdr"], _dp), ctypes.byref(e["ecav"]), ctypes.byref(e["ecorr_cav"]),
                                  _p(g["decav"], _dp), ctypes.byref(e["ehb"]), _p(g["dehb"], _dp))
        res = {k: v.value for k, v in e.items()}
        res.update(rc=rc, sp=sp, br=br, surf_area=sa, **g)
        return res

    def delete(self, tag):
        return self.lib.agbnp3_delete(tag)

    # ---- internals (harness build only) ----------------------------------
    def near_list(self, tag, nheavy):
        cnt = np.zeros(nheavy, np.int32)
        cap = 64 * nheavy + 16
        nb = np.zeros(cap, np.int32)
        n = self.lib.refh_near_list(tag, _p(cnt, _ip), _p(nb, _ip), cap)
        return cnt, nb[:n]

    def gbuffers(self, tag, n):
        v3, v3p = np.zeros(n, np.float32), np.zeros(n, np.float32)
        fp = ctypes.POINTER(ctypes.c_float)
        m = self.lib.refh_gbuffers(tag, n, v3.ctypes.data_as(fp), v3p.ctypes.data_as(fp))
        return v3[:m], v3p[:m]

    def water_sites(self, tag):
        nws = self.lib.refh_nws(tag)
        fp = ctypes.POINTER(ctypes.c_float)
        pos, sp = np.zeros(3 * nws + 3, np.float32), np.zeros(nws + 1, np.float32)
        p0, ty = np.zeros(nws + 1, np.int32), np.zeros(nws + 1, np.int32)
        self.lib.refh_ws(tag, pos.ctypes.data_as(fp), sp.ctypes.data_as(fp), _p(p0, _ip), _p(ty, _ip), nws)
        return dict(pos=pos[: 3 * nws].reshape(nws, 3), sp=sp[:nws], parent0=p0[:nws], type=ty[:nws])

    def atom_array(self, tag, which, n):
        names = ["volumep", "surf_raw", "sp", "spe", "br", "br1", "dera", "deru", "derv", "derh", "q2ab", "abrw",
                 "psvol", "gammap", "derus", "dervs", "brw", "br1_swf_der"]
        idx = names.index(which)
        out = np.zeros(n, np.float32)
        self.lib.refh_atom_array(tag, idx, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
        return out

    def tables(self, tag, n):
        rt = np.zeros(n, np.int32)
        nt = self.lib.refh_rtypes(tag, _p(rt, _ip))
        fp = ctypes.POINTER(ctypes.c_float)
        y = np.zeros((nt * nt, NA), np.float32)
        y2 = np.zeros((nt * nt, NA), np.float32)
        for s in range(nt * nt):
            self.lib.refh_table(tag, s, y[s].ctypes.data_as(fp), y2[s].ctypes.data_as(fp))
        return rt, y, y2
