"""The allocation-free GB energy entry point (agbnp3_gb_energy_static).

It is meant for callers that cannot call cudaMalloc (a host MD code that
owns all device memory, work recorded into a CUDA graph, a plugin with a
fixed memory budget).  Called through the C-ABI on device arrays, twice in
a row, it must agree with the engine's own GB pair stage of agbnp3_ener:
the GB energy (which depends only on coordinates, charges and Born radii)
and the A_i terms, within the mixed-precision tolerances of the parity
tests (energy 1e-5 relative, A_i 1e-4 RMS relative).
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
A = pytest.importorskip("agbnp3_b200")


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
            assert np.isfinite(grad.cpu().numpy()).all()
        # sizes beyond the static maximum are refused
        big = 40000
        assert f(big, x.data_ptr(), y.data_ptr(), z.data_ptr(), q.data_ptr(), br.data_ptr(), 1.0, 80.0,
                 egb.data_ptr(), dera.data_ptr(), grad.data_ptr(), None) == A.AGBNP_ERR
    finally:
        inst.close()
