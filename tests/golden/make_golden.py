"""Generate tests/golden/oracle_small.npz from the CPU oracle.

The reference itself (C# on .NET with MSolve NuGet packages) cannot be built
or run in this environment, so these fixtures are outputs of the oracle on
small cases, committed so that the oracle, which is pinned against the
reference's known-answer tests (tests/test_oracle_golden.py), stays fixed.
Run: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def compute(O):
    out = {}
    m = O.Model((6, 2, 2), (20, 1, 1))
    rp, ci, va = m.kff.arrays()
    out.update(kff_rowptr=rp, kff_col=ci, kff_val=va, rhs=m.rhs(), uf=m.uf())
    d = O.DuVi(m.kff).arrays()
    for k, v in d.items():
        out["duvi_" + k] = v
    u = O.Units.from_csr(m.kff).arrays()
    out["units_bytes"] = u["bytes"]
    out["units_vidx"] = u["vidx"]
    R, P = O.transfer((6, 2, 2), (3, 1, 1))
    for name, M in (("R", R), ("P", P)):
        a = M.arrays()
        out[name + "_rowptr"], out[name + "_col"], out[name + "_val"] = a
    g = O.Gmg((8, 2, 2), (20, 1, 1), gauss_seidel=True, duvi=False, max_cycles=500, coarse_relaxation=False,
              tol=1e-5, depth=2, level_iterations=2)
    x, st = g.solve()
    out["gmg_gs_x"] = x
    out["gmg_gs_cycles"] = np.array([st["cycles"]])
    x, it = O.pcg_jacobi(m.kff, m.rhs(), 2000, 1e-8)
    out["pcg_x"] = x
    out["pcg_it"] = np.array([it])
    return out


if __name__ == "__main__":
    sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
    import pyoracle
    pyoracle.build()
    np.savez_compressed(os.path.join(HERE, "oracle_small.npz"), **compute(pyoracle))
    print("wrote", os.path.join(HERE, "oracle_small.npz"))
