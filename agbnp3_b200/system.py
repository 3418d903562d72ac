"""Molecular systems in the form agbnp3_new() takes them, and the seeded
synthetic-globule generator used by the benchmarks and tests.

A :class:`System` holds everything the reference's agbnp3_new()
(agbnp3.c:121-419) receives, in the caller's ("external") atom order, plus the
bond list from which the NeighList connection table is built.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
GLOBULE_LIB = os.path.join(_HERE, "libagbnp3_globule.so")

# HB types (agbnp3.h:61-74)
HB_INACTIVE = 0
HB_POLARH = 1
HB_TRIGONAL = 10
HB_TRIGONAL_S = 30
HB_TETRAHEDRAL = 20
HB_TRIGONAL1 = 11
HB_TRIGONAL2 = 12
HB_TRIGONAL_OOP = 13
HB_TETRAHEDRAL1 = 21
HB_TETRAHEDRAL2 = 22
HB_TETRAHEDRAL3 = 23

ELEMENTS = ("C", "N", "O", "S", "H")


@dataclass
class System:
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    r: np.ndarray
    charge: np.ndarray
    igamma: np.ndarray
    sgamma: np.ndarray
    ialpha: np.ndarray
    salpha: np.ndarray
    hbtype: np.ndarray
    hbcorr: np.ndarray
    ihydrogen: np.ndarray
    bonds: np.ndarray  # (nbonds, 2) external indices
    eps_in: float = 1.0
    eps_out: float = 80.0
    element: np.ndarray | None = None
    stats: dict = field(default_factory=dict)

    @property
    def natoms(self) -> int:
        return int(self.x.shape[0])

    @property
    def nheavy(self) -> int:
        return self.natoms - int(self.ihydrogen.shape[0])

    def coords(self) -> np.ndarray:
        return np.stack([self.x, self.y, self.z], axis=1)

    def with_coords(self, xyz: np.ndarray) -> "System":
        """Copy of this system with new coordinates (rounded to float, as the
        engine narrows them anyway)."""
        xyz = np.asarray(xyz, dtype=np.float32).astype(np.float64)
        s = System(**{k: getattr(self, k) for k in self.__dataclass_fields__})
        s.x, s.y, s.z = xyz[:, 0].copy(), xyz[:, 1].copy(), xyz[:, 2].copy()
        return s

    # ---- connection table -------------------------------------------------
    def conn_csr(self):
        """Connection table as CSR (offset[natoms+1], list) in external
        indices; each atom lists its bonded partners in bond order."""
        n = self.natoms
        nb = [[] for _ in range(n)]
        for a, b in self.bonds:
            nb[int(a)].append(int(b))
            nb[int(b)].append(int(a))
        off = np.zeros(n + 1, dtype=np.int32)
        off[1:] = np.cumsum([len(v) for v in nb])
        lst = np.array([j for v in nb for j in v], dtype=np.int32)
        return off, lst

    # ---- internal order (heavy atoms first, hydrogens last) -------------
    def internal_order(self):
        """int2ext / ext2int maps of agbnp3_atom_reorder (agbnp3.c:739-779):
        heavy atoms keep their relative order, hydrogens follow."""
        ish = np.zeros(self.natoms, dtype=bool)
        ish[self.ihydrogen] = True
        int2ext = np.concatenate([np.nonzero(~ish)[0], np.nonzero(ish)[0]]).astype(np.int32)
        ext2int = np.empty_like(int2ext)
        ext2int[int2ext] = np.arange(self.natoms, dtype=np.int32)
        return int2ext, ext2int

    def permuted(self, perm: np.ndarray) -> "System":
        """Same molecule with atoms renumbered: new atom k is old atom
        perm[k]."""
        perm = np.asarray(perm)
        inv = np.empty_like(perm)
        inv[perm] = np.arange(perm.shape[0])
        kw = {}
        for k in ("x", "y", "z", "r", "charge", "igamma", "sgamma", "ialpha", "salpha", "hbtype", "hbcorr"):
            kw[k] = getattr(self, k)[perm].copy()
        kw["ihydrogen"] = np.sort(inv[self.ihydrogen]).astype(np.int32)
        kw["bonds"] = inv[self.bonds].astype(np.int32)
        kw["eps_in"], kw["eps_out"] = self.eps_in, self.eps_out
        kw["element"] = None if self.element is None else self.element[perm].copy()
        return System(**kw)


def _globule_lib():
    if not os.path.exists(GLOBULE_LIB):
        raise RuntimeError(f"{GLOBULE_LIB} is missing; run __graft_entry__.build()")
    lib = ctypes.CDLL(GLOBULE_LIB)
    lib.agbnp3_globule_generate.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_double, ctypes.c_double] + [
        ctypes.c_void_p
    ] * 15
    lib.agbnp3_globule_generate.restype = ctypes.c_int
    return lib


def make_globule(natoms: int, seed: int, noise: float = 0.0, density: float = 0.05) -> System:
    """Seeded synthetic globule: ~natoms/2 heavy atoms on a branched
    self-avoiding walk (1.53 A bonds, >= 3.0 A between atoms that are not
    1-2 or 1-3 partners) in a sphere at `density` heavy atoms per A^3,
    C/N/O/S 62/17/19/2 %, 0-2 hydrogens per heavy atom at 1.0 A, charges
    N(0, 0.3) shifted to zero net charge, dielectrics 1/80, igamma 0.117 on
    heavy atoms, ialpha ~ U(-0.09, -0.02), hbcorr ~ U(-1, -0.5), polar
    hydrogens on N/O as donors and oxygens as tetrahedral acceptors.
    `noise` adds N(0, noise) A to every coordinate.  Coordinates are rounded
    to float."""
    lib = _globule_lib()
    n = int(natoms)
    f = lambda: np.zeros(n, dtype=np.float64)  # noqa: E731
    x, y, z, r, q, ig, sg, ia, sa, hbc = (f() for _ in range(10))
    hbt = np.zeros(n, dtype=np.int32)
    el = np.zeros(n, dtype=np.int32)
    bonds = np.zeros(4 * n, dtype=np.int32)
    nb = ctypes.c_int(0)
    stats = np.zeros(4)
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    rc = lib.agbnp3_globule_generate(
        n, ctypes.c_uint64(seed), density, noise, P(x), P(y), P(z), P(r), P(q), P(ig), P(sg), P(ia), P(sa),
        P(hbt), P(hbc), P(el), ctypes.byref(nb), P(bonds), P(stats))
    if rc != 0:
        raise RuntimeError(f"globule generator failed (rc={rc})")
    nbonds = nb.value
    return System(x=x, y=y, z=z, r=r, charge=q, igamma=ig, sgamma=sg, ialpha=ia, salpha=sa, hbtype=hbt,
                  hbcorr=hbc, ihydrogen=np.nonzero(el == 4)[0].astype(np.int32),
                  bonds=bonds[: 2 * nbonds].reshape(nbonds, 2).copy(), element=el,
                  stats=dict(density=stats[0], radius=stats[1], branches=int(stats[2]),
                             enlargements=int(stats[3]), seed=int(seed), noise=float(noise)))
