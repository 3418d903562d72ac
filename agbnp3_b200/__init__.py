"""AGBNP3 implicit-solvent engine for NVIDIA B200.

Python mirror of the reference's C API (agbnp3.h:77-104): :func:`initialize`,
:func:`new`, :func:`ener`, :func:`delete`, :func:`terminate`, with the same
argument meaning, return codes (AGBNP_OK = 2, AGBNP_ERR = -1) and caller atom
order, plus the engine's extensions (precision modes, device-resident
evaluation, batches, stage timers).  Every call goes through the C-ABI of
libagbnp3_b200.so; there is no CPU implementation behind it.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .system import System, make_globule  # noqa: F401

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libagbnp3_b200.so")

AGBNP_OK = 2
AGBNP_ERR = -1
PREC_FP64 = 0
PREC_MIXED = 1
ENERGY_KEYS = ("egb", "evdw", "ecorr_vdw", "ecav", "ecorr_cav", "ehb", "mol_volume")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p


class NeighList(ctypes.Structure):
    """The NeighList connection table of nblist.h:41-70."""
    _fields_ = [("natoms", ctypes.c_int), ("neighl_size", ctypes.c_int), ("nne", _ip), ("neighl1", _ip),
                ("neighl", ctypes.POINTER(_ip)), ("idx_remap", ctypes.c_int), ("int2ext", _ip), ("ext2int", _ip),
                ("pbc", ctypes.c_int), ("pbc_trans1", _vp), ("pbc_trans", _vp),
                ("data", ctypes.c_int), ("data_index1", _vp), ("data_index", _vp)]


class AGBNPError(RuntimeError):
    pass


_lib = None


def lib():
    """The loaded engine library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise AGBNPError(f"{LIB_PATH} is missing: build it with __graft_entry__.build() "
                             "(python -m agbnp3_b200.build)")
        L = ctypes.CDLL(LIB_PATH)
        L.agbnp3_initialize.restype = ctypes.c_int
        L.agbnp3_terminate.restype = None
        L.agbnp3_new.argtypes = [_ip, ctypes.c_int] + [_dp] * 5 + [ctypes.c_double] * 2 + [_dp] * 4 + \
            [_ip, _dp, ctypes.c_int, _ip, ctypes.POINTER(NeighList), ctypes.c_int]
        L.agbnp3_new.restype = ctypes.c_int
        L.agbnp3_delete.argtypes = [ctypes.c_int]
        L.agbnp3_ener.argtypes = [ctypes.c_int, ctypes.c_int] + [_dp] * 3 + [_dp] * 2 + [_dp] * 2 + [_dp, _dp] + \
            [_dp, _dp, _dp] + [_dp, _dp, _dp] + [_dp, _dp]
        L.agbnp3_ener.restype = ctypes.c_int
        L.agbnp3_set_mode.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.agbnp3_get_mode.argtypes = [ctypes.c_int, _ip, _ip]
        L.agbnp3_pair_order.argtypes = [ctypes.c_int, ctypes.c_int]
        L.agbnp3_batch_pair_order.argtypes = [ctypes.c_int, ctypes.c_int]
        L.agbnp3_set_nblist_skin.argtypes = [ctypes.c_int, ctypes.c_double]
        L.agbnp3_shard_unique_id.argtypes = [_vp, ctypes.c_int]
        L.agbnp3_shard.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int]
        L.agbnp3_shard_segment.argtypes = [ctypes.c_int, ctypes.c_int]
        L.agbnp3_shard_buffers.argtypes = [ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int]
        L.agbnp3_shard_buffers.restype = ctypes.c_longlong
        L.agbnp3_batch_set_nblist_skin.argtypes = [ctypes.c_int, ctypes.c_double]
        L.agbnp3_batch_stats.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_longlong), ctypes.c_int]
        L.agbnp3_set_device.argtypes = [ctypes.c_int]
        L.agbnp3_set_coords.argtypes = [ctypes.c_int, _dp, _dp, _dp]
        L.agbnp3_ener_resident.argtypes = [ctypes.c_int]
        L.agbnp3_get_results.argtypes = [ctypes.c_int] + [_dp] * 8
        L.agbnp3_stream.argtypes = [ctypes.c_int]
        L.agbnp3_stream.restype = _vp
        L.agbnp3_stage_timing.argtypes = [ctypes.c_int, ctypes.c_int]
        L.agbnp3_stage_times.argtypes = [ctypes.c_int, _dp, ctypes.c_int]
        L.agbnp3_stage_name.argtypes = [ctypes.c_int]
        L.agbnp3_stage_name.restype = ctypes.c_char_p
        L.agbnp3_stats.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_longlong), ctypes.c_int]
        L.agbnp3_debug_fetch.argtypes = [ctypes.c_int, ctypes.c_int, _vp, ctypes.c_longlong]
        L.agbnp3_debug_fetch.restype = ctypes.c_longlong
        L.agbnp3_last_error.restype = ctypes.c_char_p
        L.agbnp3_batch_new.argtypes = [_ip, ctypes.c_int, _ip]
        L.agbnp3_batch_delete.argtypes = [ctypes.c_int]
        L.agbnp3_batch_natoms.argtypes = [ctypes.c_int]
        L.agbnp3_batch_set_coords.argtypes = [ctypes.c_int, _dp, _dp, _dp]
        L.agbnp3_batch_ener_resident.argtypes = [ctypes.c_int]
        L.agbnp3_batches_ener_resident.argtypes = [ctypes.c_int, _ip]
        L.agbnp3_batch_get_results.argtypes = [ctypes.c_int] + [_dp] * 8
        L.agbnp3_batch_set_mode.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.agbnp3_batch_stream.argtypes = [ctypes.c_int]
        L.agbnp3_batch_stream.restype = _vp
        L.agbnp3_batch_stage_timing.argtypes = [ctypes.c_int, ctypes.c_int]
        L.agbnp3_batch_stage_times.argtypes = [ctypes.c_int, _dp, ctypes.c_int]
        L.agbnp3_autotune.argtypes = [ctypes.c_int, _ip, ctypes.c_int]
        L.agbnp3_batch_autotune.argtypes = [ctypes.c_int, _ip, ctypes.c_int]
        L.agbnp3_measure_peaks.argtypes = [ctypes.c_int, _dp, ctypes.c_int]
        L.agbnp3_ener_device.argtypes = [ctypes.c_int] + [_vp] * 12
        L.agbnp3_batch_ener_device.argtypes = [ctypes.c_int] + [_vp] * 12
        _lib = L
    return _lib


def last_error() -> str:
    return lib().agbnp3_last_error().decode()


def _check(rc, what):
    if rc != AGBNP_OK:
        raise AGBNPError(f"{what} failed: {last_error()}")


def _p(a, t=_dp):
    return a.ctypes.data_as(t)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def shard_unique_id() -> bytes:
    """NCCL unique id for a row-sharded instance (made on rank 0 and passed
    to every rank, agbnp3_shard_unique_id)"""
    buf = ctypes.create_string_buffer(512)
    n = lib().agbnp3_shard_unique_id(ctypes.cast(buf, _vp), 512)
    if n <= 0:
        raise AGBNPError(f"agbnp3_shard_unique_id failed: {last_error()}")
    return buf.raw[:n]


def measure_peaks(device: int = 0) -> dict:
    """FP32 / FP64 flop/s (FMA = 2 flops) and ex2 op/s of the GPU, measured
    by the library's own throughput kernels (agbnp3_measure_peaks)."""
    out = np.zeros(4)
    if lib().agbnp3_measure_peaks(device, _p(out), 4) != 4:
        raise AGBNPError("agbnp3_measure_peaks failed")
    return {"fp32_tflops": out[0] / 1e12, "fp64_tflops": out[1] / 1e12, "ex2_tops": out[2] / 1e12,
            "nominal_sm_mhz": out[3]}


def initialize():
    """agbnp3_initialize (agbnp3.h:77)."""
    _check(lib().agbnp3_initialize(), "agbnp3_initialize")


def terminate():
    """agbnp3_terminate (agbnp3.h:80)."""
    lib().agbnp3_terminate()


def neighlist(system: System):
    """A NeighList connection table for `system`; the returned tuple keeps
    the arrays it points to alive."""
    off, lst = system.conn_csr()
    n = system.natoms
    nne = np.ascontiguousarray(np.diff(off).astype(np.int32))
    neighl1 = np.ascontiguousarray(lst if lst.size else np.zeros(1, np.int32))
    ptrs = (_ip * n)()
    base = neighl1.ctypes.data
    for i in range(n):
        ptrs[i] = ctypes.cast(base + 4 * int(off[i]), _ip)
    nl = NeighList()
    nl.natoms, nl.neighl_size = n, int(lst.size)
    nl.nne, nl.neighl1 = _p(nne, _ip), _p(neighl1, _ip)
    nl.neighl = ctypes.cast(ptrs, ctypes.POINTER(_ip))
    return nl, (nne, neighl1, ptrs)


def new(system: System, verbose: int = 0, conntbl=True) -> int:
    """agbnp3_new (agbnp3.h:83-90): returns the instance tag."""
    s = system
    arrs = [_f64(getattr(s, k)) for k in ("x", "y", "z", "r", "charge", "igamma", "sgamma", "ialpha", "salpha",
                                          "hbcorr")]
    x, y, z, r, q, ig, sg, ia, sa, hbc = arrs
    hbt = np.ascontiguousarray(s.hbtype, dtype=np.int32)
    ih = np.ascontiguousarray(s.ihydrogen, dtype=np.int32)
    nl, keep = neighlist(s) if conntbl else (None, None)
    tag = ctypes.c_int(-1)
    rc = lib().agbnp3_new(ctypes.byref(tag), s.natoms, _p(x), _p(y), _p(z), _p(r), _p(q), s.eps_in, s.eps_out,
                          _p(ig), _p(sg), _p(ia), _p(sa), _p(hbt, _ip), _p(hbc), int(ih.shape[0]),
                          _p(ih if ih.size else np.zeros(1, np.int32), _ip),
                          ctypes.byref(nl) if nl is not None else None, int(verbose))
    _check(rc, "agbnp3_new")
    return tag.value


def delete(tag: int):
    """agbnp3_delete (agbnp3.h:93)."""
    _check(lib().agbnp3_delete(tag), "agbnp3_delete")


def ener(tag: int, x, y, z) -> dict:
    """agbnp3_ener (agbnp3.h:97-104): energies and gradients at the
    coordinates x, y, z (caller order)."""
    x, y, z = _f64(x), _f64(y), _f64(z)
    n = x.shape[0]
    sp, br, sa = np.empty(n), np.empty(n), np.empty(n)
    g = {k: np.empty((n, 3)) for k in ("dgbdr", "dvwdr", "decav", "dehb")}
    e = {k: ctypes.c_double(0.0) for k in ENERGY_KEYS}
    rc = lib().agbnp3_ener(tag, 0, _p(x), _p(y), _p(z), _p(sp), _p(br), ctypes.byref(e["mol_volume"]), _p(sa),
                           ctypes.byref(e["egb"]), _p(g["dgbdr"]), ctypes.byref(e["evdw"]),
                           ctypes.byref(e["ecorr_vdw"]), _p(g["dvwdr"]), ctypes.byref(e["ecav"]),
                           ctypes.byref(e["ecorr_cav"]), _p(g["decav"]), ctypes.byref(e["ehb"]), _p(g["dehb"]))
    _check(rc, "agbnp3_ener")
    out = {k: v.value for k, v in e.items()}
    out.update(sp=sp, br=br, surf_area=sa, **g)
    return out


class Instance:
    """One AGBNP3 instance (a tag) with the engine's extensions."""

    def __init__(self, system: System, precision: int = PREC_MIXED, compat: bool = True, verbose: int = 0):
        initialize()
        self.system = system
        self.natoms = system.natoms
        self.tag = new(system, verbose)
        self.set_mode(precision, compat)

    def set_mode(self, precision: int, compat: bool = True):
        _check(lib().agbnp3_set_mode(self.tag, int(precision), int(compat)), "agbnp3_set_mode")

    def pair_order(self, mode: int = 1):
        """1: pair passes over Hilbert-sorted atoms, taken from the next
        evaluation's coordinates; 0: the internal order"""
        _check(lib().agbnp3_pair_order(self.tag, int(mode)), "agbnp3_pair_order")

    def set_nblist_skin(self, skin: float):
        """Verlet skin (A) of the near list; 0 searches it at every evaluation"""
        _check(lib().agbnp3_set_nblist_skin(self.tag, float(skin)), "agbnp3_set_nblist_skin")

    def shard(self, rank: int, nranks: int, uid: bytes | None = None):
        """This instance as rank `rank` of `nranks` of a row-sharded
        evaluation (agbnp3_shard); uid from shard_unique_id() on rank 0, or
        None for segment-wise evaluation with caller-side sums."""
        if uid is None:
            _check(lib().agbnp3_shard(self.tag, int(rank), int(nranks), None, 0), "agbnp3_shard")
        else:
            buf = ctypes.create_string_buffer(bytes(uid), len(uid))
            _check(lib().agbnp3_shard(self.tag, int(rank), int(nranks), ctypes.cast(buf, _vp), len(uid)),
                   "agbnp3_shard")

    def shard_segment(self, k: int):
        _check(lib().agbnp3_shard_segment(self.tag, int(k)), "agbnp3_shard_segment")

    def shard_sums(self, k: int) -> np.ndarray:
        """partial sums of pair pass k on this rank, concatenated"""
        n = lib().agbnp3_shard_buffers(self.tag, int(k), None, 0)
        if n < 0:
            raise AGBNPError(last_error())
        out = np.empty(n)
        if lib().agbnp3_shard_buffers(self.tag, int(k), _p(out), 0) != n:
            raise AGBNPError(last_error())
        return out

    def set_shard_sums(self, k: int, sums: np.ndarray):
        sums = np.ascontiguousarray(sums, dtype=np.float64)
        if lib().agbnp3_shard_buffers(self.tag, int(k), _p(sums), 1) != sums.size:
            raise AGBNPError(last_error())

    def ener(self, xyz=None) -> dict:
        xyz = self.system.coords() if xyz is None else np.asarray(xyz)
        return ener(self.tag, xyz[:, 0], xyz[:, 1], xyz[:, 2])

    def set_coords(self, xyz):
        xyz = np.asarray(xyz, dtype=np.float64)
        x, y, z = (np.ascontiguousarray(xyz[:, k]) for k in range(3))
        _check(lib().agbnp3_set_coords(self.tag, _p(x), _p(y), _p(z)), "agbnp3_set_coords")

    def ener_resident(self):
        _check(lib().agbnp3_ener_resident(self.tag), "agbnp3_ener_resident")

    def results(self) -> dict:
        n = self.natoms
        e = np.empty(7)
        sp, br, sa = np.empty(n), np.empty(n), np.empty(n)
        g = {k: np.empty((n, 3)) for k in ("dgbdr", "dvwdr", "decav", "dehb")}
        _check(lib().agbnp3_get_results(self.tag, _p(e), _p(sp), _p(br), _p(sa), _p(g["dgbdr"]), _p(g["dvwdr"]),
                                        _p(g["decav"]), _p(g["dehb"])), "agbnp3_get_results")
        out = dict(zip(ENERGY_KEYS, e.tolist()))
        out.update(sp=sp, br=br, surf_area=sa, **g)
        return out

    def energies(self) -> dict:
        e = np.empty(7)
        _check(lib().agbnp3_get_results(self.tag, _p(e), None, None, None, None, None, None, None),
               "agbnp3_get_results")
        return dict(zip(ENERGY_KEYS, e.tolist()))

    @property
    def stream(self) -> int:
        return lib().agbnp3_stream(self.tag) or 0

    def stage_timing(self, enable=True):
        _check(lib().agbnp3_stage_timing(self.tag, int(enable)), "agbnp3_stage_timing")

    def stage_times(self) -> dict:
        ms = np.zeros(16)
        n = lib().agbnp3_stage_times(self.tag, _p(ms), 16)
        return {lib().agbnp3_stage_name(k).decode(): float(ms[k]) for k in range(n)}

    def stats(self) -> dict:
        a = (ctypes.c_longlong * 16)()
        lib().agbnp3_stats(self.tag, a, 16)
        return dict(near_pairs=a[0], kept=[a[1], a[2], a[3], a[4]], water_sites=a[6], error=a[7], launches=a[8],
                    near_builds=a[9])

    def debug_fetch(self, what: int, count: int, dtype=np.int32):
        out = np.zeros(max(count, 1), dtype=dtype)
        n = lib().agbnp3_debug_fetch(self.tag, what, out.ctypes.data_as(_vp), out.size)
        if n < 0:
            raise AGBNPError(f"debug_fetch({what}) needs {-n} elements")
        return out, int(n)

    def near_list(self):
        """(counts per internal atom, concatenated neighbour lists) of the
        last evaluation, internal order."""
        cnt, _ = self.debug_fetch(0, self.natoms)
        lst, n = self.debug_fetch(1, int(cnt.sum()) + 1)
        return cnt, lst[:n]

    def overlaps(self, order: int):
        """Parents of the kept overlaps of one order, shape (n, order)."""
        st = self.stats()
        n = st["kept"][order - 2]
        a, m = self.debug_fetch(2 + 16 * order, order * n + 1)
        return a[: order * m].reshape(order, m).T.copy()

    def water_sites(self):
        """(positions [nws, 3], volume scaling factors [nws]) of the water
        sites of the last evaluation, in the reference's site order."""
        n = self.stats()["water_sites"]
        sp, m = self.debug_fetch(200, n + 1, np.float64)
        pos, _ = self.debug_fetch(201, 3 * n + 3, np.float64)
        return pos[: 3 * m].reshape(m, 3), sp[:m]

    def atom_array(self, k: int):
        a, _ = self.debug_fetch(100 + k, self.natoms, np.float64)
        return a[: self.natoms]

    def pair_slots(self):
        """internal atom held by each pair slot"""
        a, _ = self.debug_fetch(202, self.natoms)
        return a[: self.natoms]

    def autotune(self) -> dict:
        """Times the pair-stage work decompositions at the current device
        coordinates and keeps the fastest (agbnp3_autotune)."""
        p = np.zeros(4, np.int32)
        _check(lib().agbnp3_autotune(self.tag, _p(p, _ip), 4), "agbnp3_autotune")
        return dict(desc_chunks=int(p[0]), sym_run=int(p[1]), invb_us=int(p[2]), pair_us=int(p[3]))

    def close(self):
        if self.tag is not None:
            delete(self.tag)
            self.tag = None


ATOM_ARRAYS = ("volumep", "surf_raw", "surf_area", "sp", "spe", "psvol", "gammap", "br1", "bder", "br", "brw",
               "dera", "q2ab", "abrw", "deru", "derv", "derh", "derus", "dervs", "desc_sum")


class Batch:
    """Several instances evaluated together in one launch sequence."""

    def __init__(self, instances):
        self.members = list(instances)
        tags = np.array([m.tag for m in self.members], dtype=np.int32)
        bt = ctypes.c_int(-1)
        _check(lib().agbnp3_batch_new(ctypes.byref(bt), len(tags), _p(tags, _ip)), "agbnp3_batch_new")
        self.btag = bt.value
        self.natoms = lib().agbnp3_batch_natoms(self.btag)
        self.offsets = np.cumsum([0] + [m.natoms for m in self.members])

    def set_mode(self, precision: int, compat: bool = True):
        _check(lib().agbnp3_batch_set_mode(self.btag, int(precision), int(compat)), "agbnp3_batch_set_mode")

    def pair_order(self, mode: int = 1):
        _check(lib().agbnp3_batch_pair_order(self.btag, int(mode)), "agbnp3_batch_pair_order")

    def set_nblist_skin(self, skin: float):
        _check(lib().agbnp3_batch_set_nblist_skin(self.btag, float(skin)), "agbnp3_batch_set_nblist_skin")

    def stats(self) -> dict:
        a = (ctypes.c_longlong * 16)()
        lib().agbnp3_batch_stats(self.btag, a, 16)
        return dict(near_pairs=a[0], kept=[a[1], a[2], a[3], a[4]], water_sites=a[6], error=a[7], launches=a[8],
                    near_builds=a[9])

    def set_coords(self, xyz):
        xyz = np.asarray(xyz, dtype=np.float64)
        x, y, z = (np.ascontiguousarray(xyz[:, k]) for k in range(3))
        _check(lib().agbnp3_batch_set_coords(self.btag, _p(x), _p(y), _p(z)), "agbnp3_batch_set_coords")

    def ener_resident(self):
        _check(lib().agbnp3_batch_ener_resident(self.btag), "agbnp3_batch_ener_resident")

    def results(self) -> dict:
        n, k = self.natoms, len(self.members)
        e = np.empty((k, 7))
        sp, br, sa = np.empty(n), np.empty(n), np.empty(n)
        g = {q: np.empty((n, 3)) for q in ("dgbdr", "dvwdr", "decav", "dehb")}
        _check(lib().agbnp3_batch_get_results(self.btag, _p(e), _p(sp), _p(br), _p(sa), _p(g["dgbdr"]),
                                              _p(g["dvwdr"]), _p(g["decav"]), _p(g["dehb"])),
               "agbnp3_batch_get_results")
        out = {key: e[:, i].copy() for i, key in enumerate(ENERGY_KEYS)}
        out.update(sp=sp, br=br, surf_area=sa, **g)
        return out

    @property
    def stream(self) -> int:
        return lib().agbnp3_batch_stream(self.btag) or 0

    def stage_timing(self, enable=True):
        _check(lib().agbnp3_batch_stage_timing(self.btag, int(enable)), "agbnp3_batch_stage_timing")

    def stage_times(self) -> dict:
        ms = np.zeros(16)
        n = lib().agbnp3_batch_stage_times(self.btag, _p(ms), 16)
        return {lib().agbnp3_stage_name(k).decode(): float(ms[k]) for k in range(n)}

    def autotune(self) -> dict:
        p = np.zeros(4, np.int32)
        _check(lib().agbnp3_batch_autotune(self.btag, _p(p, _ip), 4), "agbnp3_batch_autotune")
        return dict(desc_chunks=int(p[0]), sym_run=int(p[1]), invb_us=int(p[2]), pair_us=int(p[3]))

    def close(self):
        if self.btag is not None:
            lib().agbnp3_batch_delete(self.btag)
            self.btag = None


def ener_resident_many(batches):
    """Evaluates several distinct batches at once (agbnp3_batches_ener_resident):
    their captured evaluations run side by side, each on its own stream."""
    tags = np.array([b.btag for b in batches], dtype=np.int32)
    _check(lib().agbnp3_batches_ener_resident(len(tags), _p(tags, _ip)), "agbnp3_batches_ener_resident")
