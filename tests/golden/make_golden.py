"""Generate golden vectors from the reference implementation (run in a container
that has the reference checked out; machines that only run the tests do not need this script).

    python tests/golden/make_golden.py REFERENCE_CHECKOUT

Writes ``tests/golden/reference_5pt.npz`` holding, from the reference's own
``nsrno.theranostic.wave`` module:

* ``matrix_*``  -- ``Solver.matrix`` (theranostic/wave.py:174-188) on a 30 x 26
  grid with a seeded random contrast, as COO triplets, plus the contrast;
* ``weights_*`` / ``fields`` / ``response`` -- the fixture of
  tests/test_theranostic.py:36-45 (81 x 81 nodes, 6 mm PML, 0.15 MHz, four
  finite-aperture elements): source weights, solved fields, response matrix;
* ``basis`` / ``jacobian`` / ``residual`` / ``gradient`` -- ``Solver.born_jacobian``
  with the three bump functions of tests/test_theranostic.py:48-55 and the
  seeded real gradient ``Re(J^H r)`` of tests/test_theranostic.py:108-114.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
from scipy import sparse


def main(reference_root):
    sys.path.insert(0, str(reference_root))
    from nsrno.theranostic.wave import Grid, Solver

    out = {}
    # (1) matrix on a small grid with contrast
    nz, nx, h_mm, pml = 30, 26, 0.1, 5
    z = np.arange(nz) * h_mm
    x = (np.arange(nx) - (nx - 1) / 2) * h_mm
    solver = Solver(Grid(x, z, pml_mm=pml * h_mm), c0_m_s=1540.0)
    rng = np.random.default_rng(0)
    inside = ~solver.grid.pml_mask
    mk = np.zeros((nz, nx))
    me = np.zeros((nz, nx))
    mk[inside] = rng.uniform(-0.2, 0.3, inside.sum())
    me[inside] = rng.uniform(-0.15, 0.2, inside.sum())
    m = solver.matrix(1.3, mk, me).tocoo()
    out.update(matrix_row=m.row.astype(np.int32), matrix_col=m.col.astype(np.int32), matrix_val=m.data,
               matrix_mk=mk, matrix_me=me, matrix_shape=np.array([nz, nx]), matrix_h_mm=h_mm,
               matrix_pml=pml, matrix_freq_mhz=1.3, matrix_c0=1540.0)

    # (2) the reference unit-test fixture
    axis = np.linspace(-16.0, 16.0, 81)
    solver = Solver(Grid(axis, axis, pml_mm=6.0))
    frequency = 0.15
    positions = np.array([[-6.4, -3.2], [-1.7, -3.1], [3.2, -3.2], [6.3, 1.7]])
    normals = np.array([[0.0, 1.0], [0.2, 1.0], [-0.15, 1.0], [-0.7, 0.7]])
    weights = solver.source_weights(positions, normals, np.array([0.8, 1.2, 0.6, 1.0])).tocoo()
    fields = solver.solve(frequency, weights.tocsc())
    response = solver.sample(fields, weights.tocsc())
    out.update(weights_row=weights.row.astype(np.int32), weights_col=weights.col.astype(np.int32),
               weights_val=weights.data, fields=fields, response=response, fixture_freq_mhz=frequency,
               fixture_axis_mm=axis, fixture_pml_mm=6.0, fixture_c0=1540.0)

    # (3) Born Jacobian and the seeded real gradient
    xx, zz = np.meshgrid(axis, axis)

    def bump(x0, z0, a, b):
        return np.maximum(1 - ((xx - x0) / a) ** 2 - ((zz - z0) / b) ** 2, 0) ** 2

    basis = np.column_stack([bump(-2.0, 1.0, 2.2, 1.7).ravel(), bump(2.0, 4.0, 1.6, 2.1).ravel(),
                             bump(-1.5, 6.5, 2.4, 1.3).ravel()])
    ports = np.arange(weights.shape[1])
    jac = solver.born_jacobian(frequency, fields, ports, ports, sparse.csr_matrix(basis), pair_chunk=3)
    rng = np.random.default_rng(42)
    target = response.ravel() + 0.02 * (rng.normal(size=response.size) + 1j * rng.normal(size=response.size))
    residual = response.ravel() - target
    gradient = np.real(jac.conj().T @ residual)
    out.update(basis=basis, jacobian=jac, residual=residual, gradient=gradient)

    path = Path(__file__).resolve().parent / "reference_5pt.npz"
    np.savez_compressed(path, **out)
    print(path, {k: np.shape(v) for k, v in out.items()})


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} REFERENCE_CHECKOUT")
    main(sys.argv[1])
