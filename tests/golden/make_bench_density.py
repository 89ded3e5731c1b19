"""Writes the density of the headline benchmark: (H2O)32 / cc-pVDZ, RHF after
12 SCF iterations with full FP64 builds (this library, on a GPU), stored as
the occupied MO coefficients in float32 (D = 2 C C^T) together with a hash of
the geometry and basis they belong to.

bench.py's two arms (the GPU build and the CPU reference build) both read
it, so that they time the same density; the parity tests use it as a
realistic density of the full-size plan.

    python tests/golden/make_bench_density.py [out.npz]
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

WORKLOAD = "h2o32_ccpvdz"
ITERATIONS = 12
DEFAULT_OUT = os.path.join(HERE, "h2o32_ccpvdz_scf12_cocc.npz")


def geometry_hash(bs) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(bs.molecule.coords, dtype=np.float64).tobytes())
    h.update(np.ascontiguousarray(bs.prim_exp, dtype=np.float64).tobytes())
    h.update(np.ascontiguousarray(bs.coef, dtype=np.float64).tobytes())
    return h.hexdigest()[:16]


def main(out=DEFAULT_OUT):
    from dalton_b200 import molecules
    from dalton_b200.basis import build_basis
    from dalton_b200.scf import rhf

    mol, basis = molecules.config(WORKLOAD)
    bs = build_basis(mol, basis)
    res = rhf(bs, maxiter=ITERATIONS, fixed_iterations=ITERATIONS, incremental=False)
    cocc = res["C"][:, :res["nocc"]].detach().cpu().numpy().astype(np.float32)
    np.savez_compressed(out, cocc=cocc, geometry_hash=geometry_hash(bs), workload=WORKLOAD,
                        iterations=ITERATIONS, energy=res["energy"])
    print(f"wrote {out}: C_occ {cocc.shape}, energy after {ITERATIONS} iterations {res['energy']:.10f}")


def load_density(bs, path=DEFAULT_OUT):
    """D = 2 C_occ C_occ^T (float64) from the stored coefficients, or None when
    the file is missing or belongs to another geometry or basis."""
    if not os.path.exists(path):
        return None
    z = np.load(path)
    if str(z["geometry_hash"]) != geometry_hash(bs):
        return None
    c = z["cocc"].astype(np.float64)
    return 2.0 * c @ c.T


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else DEFAULT_OUT)
