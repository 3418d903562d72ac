"""The allocation-free GB energy entry point (agbnp3_gb_energy_static).

It is meant for callers that cannot call cudaMalloc (a host MD code that
owns all device memory through its own pool, a plugin with a fixed memory
budget).  Called through the C-ABI on device arrays, twice in
a row, it must agree with the engine's own GB pair stage of agbnp3_ener:
the GB energy (which depends only on coordinates, charges and Born radii)
and the A_i terms, within the mixed-precision tolerances of the parity
tests (energy 1e-5 relative, A_i 1e-4 RMS relative).  Its gradient at
constant Born radii is checked against central finite differences of the
FP64 GB energy (a NumPy evaluation of the same formula) on a sample of
atoms, within 1e-4 RMS relative.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
A = pytest.importorskip("agbnp3_b200")


def _fd_gradient(s, br, atoms, h=1e-4):
    """Central finite differences of the GB energy at fixed Born radii
    (agbnp3_cpu_simd_kernels.c:103-141: E = 332 [sum_i k q_i^2 / B_i +
    sum_{i<j} 2 k q_i q_j / f_ij], f = sqrt(d^2 + B_i B_j exp(-d^2 / 4 B_i B_j)),
    k = -(1/eps_in - 1/eps_out) / 2) with respect to the coordinates of the
    given atoms, in float64.  Only the pair terms of atom i move with x_i."""
    xyz = s.coords()
    q = np.asarray(s.charge, dtype=np.float64)
    df = -0.5 * (1.0 / s.eps_in - 1.0 / s.eps_out)
    out = np.zeros((len(atoms), 3))
    for n, i in enumerate(atoms):
        mask = np.arange(s.natoms) != i
        bb = br[i] * br[mask]

        def e_i(p):
            d2 = ((xyz[mask] - p) ** 2).sum(axis=1)
            f = np.sqrt(d2 + bb * np.exp(-d2 / (4.0 * bb)))
            return 332.0 * 2.0 * df * q[i] * (q[mask] / f).sum()

        for a in range(3):
            p, m = xyz[i].copy(), xyz[i].copy()
            p[a] += h
            m[a] -= h
            out[n, a] = (e_i(p) - e_i(m)) / (2 * h)
    return out


def test_gb_energy_static_matches_engine():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    L = A.lib()
    f = L.agbnp3_gb_energy_static
    f.argtypes = [ctypes.c_int] + [ctypes.c_void_p] * 5 + [ctypes.c_double] * 2 + [ctypes.c_void_p] * 4
    f.restype = ctypes.c_int
    A.initialize()
    s = A.make_globule(3000, 21, noise=0.1)
    inst = A.Instance(s, precision=A.PREC_MIXED)
    try:
        R = inst.ener()
        dera_int = inst.atom_array(A.ATOM_ARRAYS.index("dera"))
        int2ext, _ = s.internal_order()
        dera_ref = np.empty(s.natoms)
        dera_ref[int2ext] = dera_int
        dev = torch.device("cuda", 0)
        t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)  # noqa: E731
        x, y, z, q, br = t(s.x), t(s.y), t(s.z), t(s.charge), t(R["br"])
        for _ in range(2):
            egb = torch.zeros(1, dtype=torch.float64, device=dev)
            dera = torch.full((s.natoms,), np.nan, dtype=torch.float64, device=dev)
            grad = torch.full((s.natoms, 3), np.nan, dtype=torch.float64, device=dev)
            torch.cuda.synchronize()
            rc = f(s.natoms, x.data_ptr(), y.data_ptr(), z.data_ptr(), q.data_ptr(), br.data_ptr(), s.eps_in,
                   s.eps_out, egb.data_ptr(), dera.data_ptr(), grad.data_ptr(), None)
            torch.cuda.synchronize()
            assert rc == A.AGBNP_OK
            e = float(egb.item())
            assert abs(e - R["egb"]) <= 1e-5 * abs(R["egb"]), (e, R["egb"])
            d = dera.cpu().numpy()
            assert np.sqrt(((d - dera_ref) ** 2).sum() / (dera_ref ** 2).sum()) < 1e-4
            g = grad.cpu().numpy()
            assert np.isfinite(g).all()
            atoms = np.linspace(0, s.natoms - 1, 48).astype(int)
            fd = _fd_gradient(s, np.asarray(R["br"]), atoms)
            err = np.sqrt(((g[atoms] - fd) ** 2).sum() / (fd ** 2).sum())
            assert err < 1e-4, err
        # sizes beyond the static maximum are refused
        big = 40000
        assert f(big, x.data_ptr(), y.data_ptr(), z.data_ptr(), q.data_ptr(), br.data_ptr(), 1.0, 80.0,
                 egb.data_ptr(), dera.data_ptr(), grad.data_ptr(), None) == A.AGBNP_ERR
        assert "outside 1..32768" in A.last_error()
    finally:
        inst.close()
