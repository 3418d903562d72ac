"""Generates the golden fixtures in this directory by running the reference
AGBNP3 library, built unmodified from the reference sources by
`make -C oracle ref`, through its public API (agbnp3_new / agbnp3_ener,
agbnp3.h:77-104) on seeded synthetic globules.

Run from the repository root where the reference sources are available:

    make -C oracle ref REF=<reference source tree> && python tests/golden/make_golden.py [names]

Each fixture (npz) holds the system in the caller's atom order, the
reference's outputs (energies, Born radii, volume scaling factors, surface
areas, the four gradient arrays) and internal state read by
oracle/ref_harness.c: the heavy-atom near list, the Gaussian-overlap
candidates of the overlap tree (raw/switched volumes in enumeration order),
the water sites and per-atom intermediates.

The large case (25,000 atoms) keeps digests of the index sets and a sample
of the per-atom outputs instead of whole arrays (see LARGE_CASES).

The reference runs with OMP_NUM_THREADS=1 (its HB energy depends on the
thread count) and with one instance per process: a second instance in the
same process reads an uninitialised table pointer (agbnp3_reset,
agbnp3.c:581-617, never clears f4c1table2dl), and agbnp3_delete frees
buffers twice (agbnp3.c:1007-1010), so instances are never deleted.
"""
import multiprocessing as mp
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
OUT = os.path.dirname(os.path.abspath(__file__))


def mixed_hb(s):
    """Relabels HB types by connectivity so that every water-site builder of
    the reference (agbnp3.c:1920-2012) is exercised."""
    off, lst = s.conn_csr()
    nne = np.diff(off)
    hb = s.hbtype.copy()
    ish = np.zeros(s.natoms, bool)
    ish[s.ihydrogen] = True
    c = {1: 0, 2: 0, 3: 0}
    for i in range(s.natoms):
        if ish[i]:
            continue
        nb = lst[off[i]:off[i + 1]]
        k = nne[i]
        if k == 1:
            p = nne[nb[0]]
            if p == 3:
                hb[i] = (10, 30)[c[1] % 2]
                c[1] += 1
            elif p == 4:
                hb[i] = 20
        elif k == 2:
            hb[i] = (10, 20, hb[i])[c[2] % 3]
            c[2] += 1
        elif k == 3:
            hb[i] = (13, 20, 0)[c[3] % 3]
            c[3] += 1
    s.hbtype = hb
    return s


CASES = [
    # name, natoms, seed, variant, candidate volumes stored, intermediates
    ("globule50", 50, 101, "plain", True, True),
    ("globule300_shuffled", 300, 102, "shuffled", True, True),
    ("globule2000_hbmix", 2000, 103, "hbmix", False, True),
]


def make_system(natoms, seed, variant):
    sys.path.insert(0, ROOT)
    from agbnp3_b200.system import make_globule
    s = make_globule(natoms, seed)
    if variant == "shuffled":
        s = s.permuted(np.random.default_rng(seed).permutation(natoms))
    elif variant == "hbmix":
        s = mixed_hb(s)
    return s


def run_case(args):
    name, natoms, seed, variant, want_cand, want_int = args
    os.environ["OMP_NUM_THREADS"] = "1"
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    s = make_system(natoms, seed, variant)
    ref = O.RefLib(harness=True)
    tag = ref.new(s)
    R = ref.ener(tag, s)
    assert R["rc"] == 2, R["rc"]
    # the candidate count comes from the oracle, whose enumeration order the
    # parity tests pin against these buffers
    Q = O.oracle_eval(s, internals=True, cand_cap=4_000_000)
    ncand = Q["cand_total"]
    v3, v3p = ref.gbuffers(tag, ncand)
    cnt, nb = ref.near_list(tag, s.nheavy)
    ws = ref.water_sites(tag)
    d = dict(
        natoms=natoms, seed=seed, variant=variant,
        x=s.x, y=s.y, z=s.z, r=s.r, charge=s.charge, igamma=s.igamma, sgamma=s.sgamma, ialpha=s.ialpha,
        salpha=s.salpha, hbtype=s.hbtype, hbcorr=s.hbcorr, ihydrogen=s.ihydrogen, bonds=s.bonds,
        eps=np.array([s.eps_in, s.eps_out]),
        energies=np.array([R[k] for k in ("egb", "evdw", "ecorr_vdw", "ecav", "ecorr_cav", "ehb", "mol_volume")]),
        sp=R["sp"], br=R["br"], surf_area=R["surf_area"], dgbdr=R["dgbdr"], dvwdr=R["dvwdr"], decav=R["decav"],
        dehb=R["dehb"], nl_count=cnt, nl_list=nb, ncand=np.array(ncand),
        cand_kept=np.packbits(v3p > np.float32(1.1754944e-38)),
        ws_pos=ws["pos"], ws_sp=ws["sp"], ws_parent0=ws["parent0"], ws_type=ws["type"],
    )
    if want_cand:
        d["cand_gvol"] = v3
    if want_int:
        for k in ("volumep", "surf_raw", "spe", "br1", "dera", "deru", "derv", "derh", "q2ab", "abrw", "psvol",
                  "gammap", "derus", "dervs"):
            d["int_" + k] = ref.atom_array(tag, k, natoms)
        rt, ty, ty2 = ref.tables(tag, natoms)
        d["rtype"], d["tab_y"], d["tab_y2"] = rt, ty, ty2
    np.savez_compressed(os.path.join(OUT, name + ".npz"), **d)
    return name, ncand, len(ws["sp"])


# large cases: too big to store whole, so the fixture holds digests of the
# index sets (tests/conftest.py index_set_digest), the reference's kept
# flags per candidate, the water sites, the energies and the per-atom
# outputs of a seeded sample of atoms; the system itself is regenerated
# from (natoms, seed) and pinned by a digest
LARGE_CASES = [
    # name, natoms, seed, sampled atoms
    ("globule25000", 25000, 1, 2000),
]


def run_large_case(args):
    name, natoms, seed, nsample = args
    os.environ["OMP_NUM_THREADS"] = "1"
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle as O
    from conftest import array_digest, index_set_digest
    from agbnp3_b200.system import make_globule
    s = make_globule(natoms, seed)
    ref = O.RefLib(harness=True)
    tag = ref.new(s)
    R = ref.ener(tag, s)
    assert R["rc"] == 2, R["rc"]
    Q = O.oracle_eval(s, internals=True, cand_cap=8_000_000)
    ncand = Q["cand_total"]
    v3, v3p = ref.gbuffers(tag, ncand)
    assert len(v3p) == ncand
    kept_ref = v3p > np.float32(1.1754944e-38)
    c = Q["cand"]
    kept_orc = c["gvolp"] > np.finfo(np.float32).tiny
    flips = np.nonzero(kept_ref != kept_orc)[0]
    cnt, nb = ref.near_list(tag, s.nheavy)
    ws = ref.water_sites(tag)
    idx = np.sort(np.random.default_rng(seed + 7).choice(natoms, nsample, replace=False))
    d = dict(
        natoms=natoms, seed=seed,
        system_digest=np.array(array_digest(np.concatenate([s.x, s.y, s.z, s.r, s.charge]), "f8")),
        energies=np.array([R[k] for k in ("egb", "evdw", "ecorr_vdw", "ecav", "ecorr_cav", "ehb", "mol_volume")]),
        nl_count=cnt, nl_total=np.array(len(nb)), nl_digest=np.array(array_digest(nb, "i4")),
        ncand=np.array(ncand), cand_kept=np.packbits(kept_ref),
        # candidates whose keep decision differs between the FP32 reference
        # and the FP64 oracle (volumes on the switch's lower edge)
        kept_flips=flips.astype(np.int32), kept_flips_gvol=c["gvol"][flips],
        ws_pos=ws["pos"], ws_sp=ws["sp"], ws_parent0=ws["parent0"], ws_type=ws["type"],
        sample=idx.astype(np.int32),
    )
    for m in range(2, 6):
        sel = (c["order"] == m) & kept_ref
        d[f"kept{m}_count"] = np.array(int(sel.sum()))
        d[f"kept{m}_digest"] = np.array(index_set_digest(c["parents"][sel, :m]))
        # the same set with the FP64 oracle's keep decisions
        sel64 = (c["order"] == m) & kept_orc
        d[f"kept{m}_fp64_digest"] = np.array(index_set_digest(c["parents"][sel64, :m]))
    for k in ("sp", "br", "surf_area", "dgbdr", "dvwdr", "decav", "dehb"):
        d["sample_" + k] = R[k][idx]
    np.savez_compressed(os.path.join(OUT, name + ".npz"), **d)
    return name, ncand, len(ws["sp"]), len(flips)


def _child(args):
    print("wrote", run_case(args), flush=True)


def _child_large(args):
    print("wrote", run_large_case(args), flush=True)


if __name__ == "__main__":
    ctx = mp.get_context("spawn")
    only = sys.argv[1:]
    jobs = [(_child, c) for c in CASES] + [(_child_large, c) for c in LARGE_CASES]
    for fn, case in jobs:
        if only and case[0] not in only:
            continue
        p = ctx.Process(target=fn, args=(case,))
        p.start()
        p.join(timeout=600)
        if p.is_alive():
            p.kill()
            raise SystemExit(f"{case[0]}: timed out")
        if p.exitcode != 0:
            raise SystemExit(f"{case[0]}: exit code {p.exitcode}")
