"""Parity of the CUDA engine (called through its C-ABI) with the FP64 oracle
and with the reference library's golden outputs.

Tolerances:
- plain FP64 path vs FP64 oracle: energies 1e-9 relative, per-atom outputs
  and forces 1e-9 RMS relative (only summation order differs);
- mixed path (float pair/overlap math, double accumulation) vs FP64 oracle:
  energies 1e-5 relative (or 1e-4 kcal/mol), forces 1e-4 RMS relative;
- both paths vs the reference's FP32 golden outputs: the FP32 tolerances of
  tests/test_oracle_golden.py;
- near lists and kept-overlap index sets: identical.
"""
import numpy as np
import pytest

import oracle as O
from conftest import ENERGY_KEYS, GOLDEN_CASES, load_golden, rms_rel

pytestmark = pytest.mark.gpu

A = pytest.importorskip("agbnp3_b200")

TOL = {A.PREC_FP64: dict(e=1e-9, g=1e-9), A.PREC_MIXED: dict(e=1e-5, g=1e-4)}
PREC_NAMES = {A.PREC_FP64: "fp64", A.PREC_MIXED: "mixed"}


def check_vs_oracle(R, Q, prec, label=""):
    t = TOL[prec]
    for k in ENERGY_KEYS:
        assert abs(R[k] - Q[k]) <= t["e"] * max(abs(Q[k]), 10.0), (label, k, R[k], Q[k])
    for k in ("sp", "br", "surf_area"):
        assert rms_rel(R[k], Q[k]) <= t["g"], (label, k, rms_rel(R[k], Q[k]))
    for k in ("dgbdr", "dvwdr", "decav", "dehb"):
        assert rms_rel(R[k], Q[k]) <= t["g"], (label, k, rms_rel(R[k], Q[k]))


@pytest.fixture(scope="module")
def engine():
    A.initialize()
    yield A
    A.terminate()


@pytest.mark.parametrize("prec", [A.PREC_FP64, A.PREC_MIXED], ids=["fp64", "mixed"])
@pytest.mark.parametrize("name", GOLDEN_CASES)
@pytest.mark.parametrize("compat", [True, False], ids=["compat", "exact"])
def test_engine_vs_oracle(engine, name, prec, compat):
    s, _ = load_golden(name)
    inst = A.Instance(s, precision=prec, compat=compat)
    try:
        R = inst.ener()
        check_vs_oracle(R, O.oracle_eval(s, compat=compat), prec, f"{name}/{PREC_NAMES[prec]}")
    finally:
        inst.close()


@pytest.mark.parametrize("prec", [A.PREC_FP64, A.PREC_MIXED], ids=["fp64", "mixed"])
@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_engine_vs_reference_golden(engine, name, prec):
    """Through agbnp3_ener, against the reference library's own outputs."""
    s, d = load_golden(name)
    inst = A.Instance(s, precision=prec, compat=True)
    try:
        R = inst.ener()
        for k, ref in zip(ENERGY_KEYS, d["energies"]):
            assert abs(R[k] - ref) <= 2e-5 * max(abs(ref), 1.0), (name, k, R[k], ref)
        for k in ("sp", "br", "surf_area"):
            assert rms_rel(R[k], d[k]) < 2e-5, (name, k)
        for k in ("dgbdr", "dvwdr", "decav", "dehb"):
            assert rms_rel(R[k], d[k]) < 1e-4, (name, k, rms_rel(R[k], d[k]))
    finally:
        inst.close()


@pytest.mark.parametrize("prec", [A.PREC_FP64, A.PREC_MIXED], ids=["fp64", "mixed"])
@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_near_list_bit_exact(engine, name, prec):
    """Heavy-atom near list: same pairs in the same (float d^2, index)
    order as the reference (agbnp3.c:4041-4066)."""
    s, d = load_golden(name)
    inst = A.Instance(s, precision=prec)
    try:
        inst.ener()
        cnt, lst = inst.near_list()
        assert np.array_equal(cnt[: s.nheavy], d["nl_count"])
        assert np.array_equal(lst, d["nl_list"])
    finally:
        inst.close()


def test_near_list_warp_search(engine, monkeypatch, large25k):
    """The near-list search used for large systems (a warp per 32 grid slots
    and neighbour direction, AGBNP3_NL_CELLS=1 forces it here) gives the
    reference's list too: the golden cases and the 25,000-atom globule
    (counts and the digest of the lists in the reference's order)."""
    from conftest import array_digest
    monkeypatch.setenv("AGBNP3_NL_CELLS", "1")
    for name in GOLDEN_CASES:
        s, d = load_golden(name)
        inst = A.Instance(s, precision=A.PREC_MIXED)
        try:
            inst.ener()
            cnt, lst = inst.near_list()
            assert np.array_equal(cnt[: s.nheavy], d["nl_count"]), name
            assert np.array_equal(lst, d["nl_list"]), name
        finally:
            inst.close()
    s, d, _ = large25k
    inst = A.Instance(s, precision=A.PREC_FP64)
    try:
        inst.ener()
        cnt, lst = inst.near_list()
        assert np.array_equal(cnt[: s.nheavy], d["nl_count"])
        assert len(lst) == int(d["nl_total"]) and array_digest(lst, "i4") == str(d["nl_digest"])
    finally:
        inst.close()


def canonical(parents):
    return {tuple(sorted(p)) for p in parents.tolist()}


@pytest.mark.parametrize("prec", [A.PREC_FP64, A.PREC_MIXED], ids=["fp64", "mixed"])
@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_overlap_sets(engine, name, prec):
    """Kept overlaps of every order: the same index sets as the oracle,
    whose candidates equal the reference's (test_oracle_golden).  Any
    difference may only involve overlaps whose volume sits on the switch's
    lower edge."""
    s, d = load_golden(name)
    n = int(d["ncand"])
    Q = O.oracle_eval(s, internals=True, cand_cap=n + 10)
    c = Q["cand"]
    int2ext, ext2int = s.internal_order()
    inst = A.Instance(s, precision=prec)
    try:
        inst.ener()
        for m in range(2, 6):
            sel = (c["order"] == m) & (c["gvolp"] > np.finfo(np.float32).tiny)
            want = canonical(c["parents"][sel, :m])
            got = canonical(inst.overlaps(m))
            diff = want ^ got
            if diff:
                border = {tuple(sorted(p)) for p, g in zip(c["parents"][c["order"] == m, :m].tolist(),
                                                          c["gvol"][c["order"] == m]) if abs(g - 0.01) < 1e-5}
                assert diff <= border, (m, len(diff))
    finally:
        inst.close()


def test_resident_graph_matches_direct(engine):
    """Graph replay of the device-resident path gives the same outputs as
    agbnp3_ener, and repeated replays are consistent."""
    s, _ = load_golden("globule300_shuffled")
    inst = A.Instance(s, precision=A.PREC_MIXED)
    try:
        R = inst.ener()
        inst.set_coords(s.coords())
        for _ in range(3):
            inst.ener_resident()
        G = inst.results()
        for k in ENERGY_KEYS:
            assert abs(G[k] - R[k]) <= 1e-9 * max(1.0, abs(R[k]))
        for k in ("dgbdr", "dehb"):
            assert rms_rel(G[k], R[k]) < 1e-9
    finally:
        inst.close()


@pytest.mark.parametrize("prec", [A.PREC_FP64, A.PREC_MIXED], ids=["fp64", "mixed"])
def test_batch_matches_members(engine, prec):
    """A batch of uneven instances evaluates each member as if alone (to
    summation order: the batch splits partner ranges differently, which in
    the mixed path regroups the float tile sums)."""
    systems = [A.make_globule(n, seed, noise=0.2) for n, seed in ((300, 1), (777, 2), (1500, 3), (420, 4))]
    insts = [A.Instance(x, precision=prec) for x in systems]
    B = A.Batch(insts)
    B.set_mode(prec, True)
    te, tg = (1e-9, 1e-9) if prec == A.PREC_FP64 else (1e-6, 1e-5)
    try:
        B.set_coords(np.concatenate([x.coords() for x in systems]))
        B.ener_resident()
        R = B.results()
        for k, (x, inst) in enumerate(zip(systems, insts)):
            S = inst.ener()
            o0, o1 = B.offsets[k], B.offsets[k + 1]
            for e in ENERGY_KEYS:
                assert abs(R[e][k] - S[e]) <= te * max(1.0, abs(S[e])), (k, e)
            for g in ("dgbdr", "dvwdr", "decav", "dehb"):
                assert rms_rel(R[g][o0:o1], S[g]) < tg, (k, g)
    finally:
        B.close()
        for i in insts:
            i.close()


@pytest.fixture(scope="module")
def batch64(engine):
    """64 instances of the batched configuration's distribution: atom counts
    log-uniform in [300, 5000], 0.2 A coordinate noise, distinct seeds; with
    the FP64 oracle of every member."""
    rng = np.random.default_rng(64)
    sizes = np.exp(rng.uniform(np.log(300), np.log(5000), 64)).astype(int)
    systems = [A.make_globule(int(n), 5000 + k, noise=0.2) for k, n in enumerate(sizes)]
    return systems, [O.oracle_eval(x, compat=True) for x in systems]


@pytest.mark.parametrize("prec", [A.PREC_FP64, A.PREC_MIXED], ids=["fp64", "mixed"])
def test_batch64_members_vs_oracle(batch64, prec):
    """One batched evaluation of 64 uneven instances: every member's
    energies, per-atom outputs and forces against its own FP64 oracle, at
    the tolerances of the single-instance parity tests."""
    systems, oracles = batch64
    insts = [A.Instance(x, precision=prec) for x in systems]
    B = A.Batch(insts)
    B.set_mode(prec, True)
    t = TOL[prec]
    try:
        B.set_coords(np.concatenate([x.coords() for x in systems]))
        B.ener_resident()
        R = B.results()
        for k, Q in enumerate(oracles):
            o0, o1 = B.offsets[k], B.offsets[k + 1]
            for e in ENERGY_KEYS:
                assert abs(R[e][k] - Q[e]) <= t["e"] * max(abs(Q[e]), 10.0), (k, e, R[e][k], Q[e])
            for g in ("sp", "br", "surf_area", "dgbdr", "dvwdr", "decav", "dehb"):
                assert rms_rel(R[g][o0:o1], Q[g]) <= t["g"], (k, g, rms_rel(R[g][o0:o1], Q[g]))
    finally:
        B.close()
        for i in insts:
            i.close()


def test_caller_order_and_permutation(engine):
    """Outputs follow the caller's atom order.  AGBNP3 itself depends on
    the atom numbering (the overlap tree is rooted at the lowest index and,
    with Gaussian prefactors above 1, a larger overlap can exceed a smaller
    one; the water-site order feeds the reference's free-volume index), so a
    renumbered molecule is checked against the oracle of that numbering, and
    its GB energy differs from the original only at the 1e-7 level."""
    s, _ = load_golden("globule300_shuffled")
    perm = np.random.default_rng(5).permutation(s.natoms)
    sp = s.permuted(perm)
    a, b = A.Instance(s, precision=A.PREC_FP64), A.Instance(sp, precision=A.PREC_FP64)
    try:
        Ra, Rb = a.ener(), b.ener()
        check_vs_oracle(Rb, O.oracle_eval(sp), A.PREC_FP64, "permuted")
        assert abs(Ra["egb"] - Rb["egb"]) <= 1e-6 * abs(Ra["egb"])
        assert rms_rel(Rb["br"], Ra["br"][perm]) < 1e-5
    finally:
        a.close()
        b.close()


def test_edge_cases(engine):
    """Two atoms, a molecule without hydrogens, and coincident atoms."""
    s = A.make_globule(60, 9)
    # no hydrogens: keep the heavy atoms only
    heavy = np.setdiff1d(np.arange(s.natoms), s.ihydrogen)
    keep = {int(h): i for i, h in enumerate(heavy)}
    bonds = np.array([[keep[a], keep[b]] for a, b in s.bonds if a in keep and b in keep], dtype=np.int32)
    sh = A.System(x=s.x[heavy], y=s.y[heavy], z=s.z[heavy], r=s.r[heavy], charge=s.charge[heavy],
                  igamma=s.igamma[heavy], sgamma=s.sgamma[heavy], ialpha=s.ialpha[heavy], salpha=s.salpha[heavy],
                  hbtype=np.where(s.hbtype[heavy] == 1, 0, s.hbtype[heavy]).astype(np.int32),
                  hbcorr=s.hbcorr[heavy], ihydrogen=np.zeros(0, np.int32), bonds=bonds)
    two = A.System(x=np.array([0.0, 3.0]), y=np.zeros(2), z=np.zeros(2), r=np.array([1.7, 1.52]),
                   charge=np.array([0.3, -0.3]), igamma=np.full(2, 0.117), sgamma=np.zeros(2),
                   ialpha=np.full(2, -0.05), salpha=np.zeros(2), hbtype=np.array([0, 20], np.int32),
                   hbcorr=np.full(2, -0.7), ihydrogen=np.zeros(0, np.int32), bonds=np.array([[0, 1]], np.int32))
    for sys_ in (sh, two):
        for prec in (A.PREC_FP64, A.PREC_MIXED):
            inst = A.Instance(sys_, precision=prec)
            try:
                check_vs_oracle(inst.ener(), O.oracle_eval(sys_), prec, "edge")
            finally:
                inst.close()
    # coincident heavy atoms: finite energies, pair excluded from GB
    c = A.make_globule(80, 11)
    c.x[1], c.y[1], c.z[1] = c.x[0], c.y[0], c.z[0]
    inst = A.Instance(c, precision=A.PREC_FP64)
    try:
        R = inst.ener()
        assert all(np.isfinite(R[k]) for k in ENERGY_KEYS)
        assert np.isfinite(R["dgbdr"]).all()
    finally:
        inst.close()


def test_api_errors_on_device(engine):
    s, _ = load_golden("globule50")
    with pytest.raises(A.AGBNPError):
        A.new(s, conntbl=False)
    tag = A.new(s)
    A.delete(tag)
    with pytest.raises(A.AGBNPError):
        A.ener(tag, s.x, s.y, s.z)
    with pytest.raises(A.AGBNPError):
        A.delete(tag)


@pytest.fixture(scope="module")
def large25k(engine):
    """The benchmark workload (25,000-atom globule, seed 1), its reference
    fixture (digests of the index sets, energies, water sites, sampled
    per-atom outputs) and the FP64 oracle with its overlap candidates."""
    from conftest import load_large_golden
    s, d = load_large_golden("globule25000")
    Q = O.oracle_eval(s, compat=True, internals=True, cand_cap=int(d["ncand"]) + 10)
    return s, d, Q


def test_large_fp64_vs_oracle(large25k):
    """25,000 atoms: plain FP64 path against the FP64 oracle, and the mixed
    path within the model's accuracy targets (energy 1e-4 relative, forces
    1e-3 RMS relative)."""
    s, d, Q = large25k
    a = A.Instance(s, precision=A.PREC_FP64)
    b = A.Instance(s, precision=A.PREC_MIXED)
    try:
        Ra, Rb = a.ener(), b.ener()
        check_vs_oracle(Ra, Q, A.PREC_FP64, "25k/fp64")
        et = lambda R: sum(R[k] for k in ("egb", "evdw", "ecav", "ehb"))  # noqa: E731
        assert abs(et(Rb) - et(Q)) <= 1e-4 * abs(et(Q))
        ft = lambda R: R["dgbdr"] + R["dvwdr"] + R["decav"] + R["dehb"]  # noqa: E731
        assert rms_rel(ft(Rb), ft(Q)) <= 1e-3
    finally:
        a.close()
        b.close()


@pytest.mark.parametrize("prec", [A.PREC_FP64, A.PREC_MIXED], ids=["fp64", "mixed"])
def test_large_vs_reference_golden(large25k, prec):
    """25,000 atoms, through agbnp3_ener, against the reference library run
    on the same input (tests/golden/globule25000.npz):
    - near list (agbnp3.c:3978-4115): bit-exact (counts, and the digest of
      the concatenated lists in the reference's order);
    - kept overlaps of orders 2-5 (agbnp3_cpu_simd_kernels.c:1064-1598): in
      FP64 the same sets as the FP64 oracle, whose sets the fixture pins
      (digest; they differ from the FP32 reference's only by the candidates
      on the switch's lower edge that the fixture lists); in the mixed mode
      the same sets up to candidates on that edge;
    - water sites (agbnp3.c:1837-3761): same count, positions 1e-4 A,
      scaling factors 1e-5;
    - energies within 2e-5 relative, sampled per-atom outputs at the FP32
      tolerances of the golden tests."""
    from conftest import array_digest, index_set_digest
    s, d, Q = large25k
    inst = A.Instance(s, precision=prec, compat=True)
    try:
        R = inst.ener()
        cnt, lst = inst.near_list()
        assert np.array_equal(cnt[: s.nheavy], d["nl_count"])
        assert len(lst) == int(d["nl_total"]) and array_digest(lst, "i4") == str(d["nl_digest"])
        c = Q["cand"]
        for m in range(2, 6):
            got = inst.overlaps(m)
            if prec == A.PREC_FP64:
                assert index_set_digest(got) == str(d[f"kept{m}_fp64_digest"]), m
            else:
                sel = (c["order"] == m) & (c["gvolp"] > np.finfo(np.float32).tiny)
                diff = canonical(c["parents"][sel, :m]) ^ canonical(got)
                if diff:
                    om = c["order"] == m
                    border = {tuple(sorted(p)) for p, g in zip(c["parents"][om, :m].tolist(), c["gvol"][om])
                              if abs(g - 0.01) < 1e-5}
                    assert diff <= border, (m, len(diff))
        pos, wsp = inst.water_sites()
        assert len(wsp) == len(d["ws_sp"])
        assert np.abs(pos - d["ws_pos"]).max() < 1e-4
        assert np.abs(wsp - d["ws_sp"]).max() < 1e-5
        for k, ref in zip(ENERGY_KEYS, d["energies"]):
            assert abs(R[k] - ref) <= 2e-5 * max(abs(ref), 1.0), (k, R[k], ref)
        idx = d["sample"]
        for k in ("sp", "br", "surf_area"):
            assert rms_rel(R[k][idx], d["sample_" + k]) < 2e-5, k
        for k in ("dgbdr", "dvwdr", "decav", "dehb"):
            assert rms_rel(R[k][idx], d["sample_" + k]) < 1e-4, (k, rms_rel(R[k][idx], d["sample_" + k]))
    finally:
        inst.close()


def test_mixed_100k_against_fp64(engine):
    """The 100,000-atom globule: the chosen mode against the plain FP64 path
    (which matches the oracle to 1e-9 at the sizes the oracle can run):
    every energy term within 1e-4 relative, forces within 1e-3 RMS relative,
    and the same near-list and overlap counts (the index sets use the same
    float tests in both modes)."""
    s = A.make_globule(100000, 3)
    a = A.Instance(s, precision=A.PREC_FP64)
    b = A.Instance(s, precision=A.PREC_MIXED)
    try:
        Ra, Rb = a.ener(), b.ener()
        for k in ("egb", "evdw", "ecav", "ehb", "mol_volume"):
            assert abs(Rb[k] - Ra[k]) <= 1e-4 * abs(Ra[k]), k
        ft = lambda R: R["dgbdr"] + R["dvwdr"] + R["decav"] + R["dehb"]  # noqa: E731
        assert rms_rel(ft(Rb), ft(Ra)) <= 1e-3
        sa, sb = a.stats(), b.stats()
        assert sa["near_pairs"] == sb["near_pairs"] and sa["error"] == sb["error"] == 0
    finally:
        a.close()
        b.close()


def test_mode_switch_on_one_instance(engine):
    """Precision and derivative convention switched back and forth on one
    instance (the captured graph and the pair-stage work lists are rebuilt
    for each mode) give the oracle's results every time."""
    s, _ = load_golden("globule2000_hbmix")
    q = {c: O.oracle_eval(s, compat=c) for c in (True, False)}
    inst = A.Instance(s, precision=A.PREC_MIXED)
    try:
        for prec, compat in [(A.PREC_MIXED, True), (A.PREC_FP64, True), (A.PREC_FP64, False),
                             (A.PREC_MIXED, False), (A.PREC_MIXED, True), (A.PREC_FP64, True)]:
            inst.set_mode(prec, compat)
            inst.set_coords(s.coords())
            inst.ener_resident()
            check_vs_oracle(inst.results(), q[compat], prec, f"switch/{PREC_NAMES[prec]}/{compat}")
    finally:
        inst.close()


def test_capacity_regrowth(engine, monkeypatch):
    """Near-list and overlap buffers that start far too small overflow, are
    detected through the device error word, regrown and the evaluation is
    repeated with identical results."""
    s, _ = load_golden("globule300_shuffled")
    q = O.oracle_eval(s)
    monkeypatch.setenv("AGBNP3_CAPACITY_SCALE", "0.001")
    inst = A.Instance(s, precision=A.PREC_FP64)
    try:
        check_vs_oracle(inst.ener(), q, A.PREC_FP64, "regrowth")
        assert inst.stats()["error"] == 0
    finally:
        inst.close()


@pytest.mark.parametrize("prec", [A.PREC_FP64, A.PREC_MIXED], ids=["fp64", "mixed"])
def test_regrowth_on_reused_device_memory(engine, monkeypatch, prec):
    """A first evaluation whose near-list sub-slabs and overlap buffers
    overflow, on device memory that held other data before (1 GB of -7
    written and handed back to the driver): the passes that run after the
    overflow was flagged must not take counts from what the memory held,
    and the repeated evaluation gives the oracle's results."""
    import torch
    junk = torch.full((256 * 1024 * 1024,), -7, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    del junk
    torch.cuda.empty_cache()
    s = A.make_globule(2500, 21, noise=0.2)
    q = O.oracle_eval(s)
    monkeypatch.setenv("AGBNP3_CAPACITY_SCALE", "0.01")
    inst = A.Instance(s, precision=prec)
    try:
        check_vs_oracle(inst.ener(), q, prec, "regrowth on reused memory")
        assert inst.stats()["error"] == 0
    finally:
        inst.close()


@pytest.mark.parametrize("prec", [A.PREC_FP64, A.PREC_MIXED], ids=["fp64", "mixed"])
def test_one_sided_pair_kernels(engine, monkeypatch, prec):
    """The one-sided tiled GB pair kernels (AGBNP3_PAIR_TILED=1, each
    ordered pair evaluated by its first atom) against the oracle, and in
    FP64 against the default symmetric kernels."""
    s, _ = load_golden("globule2000_hbmix")
    q = O.oracle_eval(s)
    base = A.Instance(s, precision=prec)
    monkeypatch.setenv("AGBNP3_PAIR_TILED", "1")
    inst = A.Instance(s, precision=prec)
    try:
        r = inst.ener()
        check_vs_oracle(r, q, prec, "tiled")
        if prec == A.PREC_FP64:
            b = base.ener()
            for k in ("egb", "evdw"):
                assert abs(r[k] - b[k]) <= 1e-10 * max(abs(b[k]), 1.0)
            assert rms_rel(r["dgbdr"], b["dgbdr"]) <= 1e-10
    finally:
        inst.close()
        base.close()


@pytest.mark.parametrize("gbd,desc", [("0", "0"), ("0", "1"), ("1", "0")],
                         ids=["both_global", "chain_rule_global", "descreening_global"])
def test_table_placement(engine, monkeypatch, gbd, desc):
    """The FP32 descreening and chain-rule passes read their Q4 tables from
    shared memory by default (the tables of the heavy descreener types,
    copied once per SM) and from global memory with AGBNP3_DESC_SMEM=0 /
    AGBNP3_GBD_SMEM=0: every placement against the oracle, and against the
    default one to within float summation order."""
    s, _ = load_golden("globule2000_hbmix")
    q = O.oracle_eval(s)
    base = A.Instance(s, precision=A.PREC_MIXED)
    monkeypatch.setenv("AGBNP3_GBD_SMEM", gbd)
    monkeypatch.setenv("AGBNP3_DESC_SMEM", desc)
    inst = A.Instance(s, precision=A.PREC_MIXED)
    try:
        r, b = inst.ener(), base.ener()
        check_vs_oracle(r, q, A.PREC_MIXED, f"gbd={gbd} desc={desc}")
        for k in ENERGY_KEYS:
            assert abs(r[k] - b[k]) <= 1e-6 * max(abs(b[k]), 1.0), (k, r[k], b[k])
        for k in ("br", "dgbdr", "dvwdr"):
            assert rms_rel(r[k], b[k]) <= 1e-5, (k, rms_rel(r[k], b[k]))
    finally:
        inst.close()
        base.close()


@pytest.mark.parametrize("prec", [A.PREC_FP64, A.PREC_MIXED], ids=["fp64", "mixed"])
def test_many_radius_types(engine, prec):
    """A 2,000-atom globule whose heavy atoms carry twelve distinct radii:
    the heavy-descreener tables (13 x 12 tables of 8 KB) do not fit in shared
    memory, so the FP32 passes fall back to tables in global memory; energies
    and forces against the oracle."""
    s = A.make_globule(2000, 5)
    heavy = np.setdiff1d(np.arange(s.natoms), s.ihydrogen)
    s.r = s.r.copy()
    s.r[heavy] = np.random.default_rng(3).choice(np.linspace(1.5, 2.05, 12), size=heavy.size)
    q = O.oracle_eval(s)
    inst = A.Instance(s, precision=prec)
    try:
        check_vs_oracle(inst.ener(), q, prec, "12 heavy radii")
    finally:
        inst.close()


@pytest.mark.parametrize("prec", [A.PREC_FP64, A.PREC_MIXED], ids=["fp64", "mixed"])
def test_pair_slot_order(engine, prec):
    """Hilbert-ordered pair slots (the default) against the internal order:
    the slots are a permutation that keeps the heavy atoms ahead of the
    hydrogens; both orders give the oracle's results and agree with each
    other up to summation order; after the atoms move, ordering again
    changes the slots and the results stay right."""
    s, _ = load_golden("globule2000_hbmix")
    q = O.oracle_eval(s)
    n, nh = s.natoms, s.nheavy
    inst = A.Instance(s, precision=prec)
    try:
        r1 = inst.ener()
        slots = inst.pair_slots()
        assert np.array_equal(np.sort(slots), np.arange(n))
        assert (slots[:nh] < nh).all()
        assert not np.array_equal(slots, np.arange(n))
        check_vs_oracle(r1, q, prec, "hilbert")
        inst.pair_order(0)
        r0 = inst.ener()
        assert np.array_equal(inst.pair_slots(), np.arange(n))
        check_vs_oracle(r0, q, prec, "identity")
        tol = 1e-11 if prec == A.PREC_FP64 else 1e-5
        for k in ENERGY_KEYS:
            assert abs(r1[k] - r0[k]) <= tol * max(abs(r0[k]), 10.0), (k, r1[k], r0[k])
        for k in ("br", "dgbdr", "dvwdr"):
            assert rms_rel(r1[k], r0[k]) <= 10 * tol, (k, rms_rel(r1[k], r0[k]))
        rng = np.random.default_rng(11)
        xyz = s.coords() + rng.normal(0.0, 0.5, (n, 3))
        s2 = s.with_coords(xyz)
        inst.pair_order(1)
        r2 = inst.ener(s2.coords())
        slots2 = inst.pair_slots()
        assert np.array_equal(np.sort(slots2), np.arange(n)) and not np.array_equal(slots2, slots)
        check_vs_oracle(r2, O.oracle_eval(s2), prec, "reordered")
    finally:
        inst.close()


@pytest.mark.parametrize("prec", [A.PREC_FP64, A.PREC_MIXED], ids=["fp64", "mixed"])
def test_descreening_range_culling(engine, prec):
    """A 3,000-atom globule spread to three times its size (most atom pairs
    lie beyond the Q4 tables' range, so the descreening pass skips most
    partner tiles by their bounding boxes): Born radii, energies and forces
    still equal the FP64 oracle's at the single-instance tolerances.  The
    spread water sites overlap nothing, so the HB gradient is ~1e-15 and is
    compared within the sum of all four gradients."""
    s0 = A.make_globule(3000, 11)
    s = s0.with_coords(3.0 * s0.coords())
    Q = O.oracle_eval(s, compat=True)
    inst = A.Instance(s, precision=prec)
    t = TOL[prec]
    try:
        R = inst.ener()
        for k in ENERGY_KEYS:
            assert abs(R[k] - Q[k]) <= t["e"] * max(abs(Q[k]), 10.0), (k, R[k], Q[k])
        for k in ("sp", "br", "surf_area", "dgbdr", "dvwdr", "decav"):
            assert rms_rel(R[k], Q[k]) <= t["g"], (k, rms_rel(R[k], Q[k]))
        tot = lambda X: X["dgbdr"] + X["dvwdr"] + X["decav"] + X["dehb"]  # noqa: E731
        assert rms_rel(tot(R), tot(Q)) <= t["g"]
    finally:
        inst.close()


def test_batches_side_by_side(engine):
    """agbnp3_batches_ener_resident: three batches launched together on
    their own streams give each batch's results from its own evaluation
    (the same kernels on the same data; summation order of the double
    atomics aside), on the first call (graphs captured one by one) and on
    replays (graphs launched side by side)."""
    groups = [[A.make_globule(n, 70 + 10 * q + k, noise=0.2) for k, n in enumerate(ns)]
              for q, ns in enumerate(((400, 1300), (2500,), (600, 350, 900)))]
    insts = [[A.Instance(x, precision=A.PREC_MIXED) for x in g] for g in groups]
    alone = [A.Batch(m) for m in insts]
    many = [A.Batch(m) for m in insts]
    try:
        for b, g in zip(alone + many, groups + groups):
            b.set_mode(A.PREC_MIXED, True)
            b.set_coords(np.concatenate([x.coords() for x in g]))
        for b in alone:
            b.ener_resident()
        for rep in range(3):
            A.ener_resident_many(many)
            for b, c in zip(alone, many):
                Ra, Rc = b.results(), c.results()
                for e in ENERGY_KEYS:
                    assert np.allclose(Rc[e], Ra[e], rtol=1e-12, atol=1e-12), (rep, e)
                for g in ("sp", "br", "surf_area", "dgbdr", "dvwdr", "decav", "dehb"):
                    assert rms_rel(Rc[g], Ra[g]) < 1e-12, (rep, g)
        with pytest.raises(A.AGBNPError):
            A.ener_resident_many([many[0], many[0]])
    finally:
        for b in alone + many:
            b.close()
        for m in insts:
            for i in m:
                i.close()
