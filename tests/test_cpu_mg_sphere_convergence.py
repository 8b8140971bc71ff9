"""The oracle's multigrid with a subgrid conductor converges to an analytic
potential at second order, which pins the conductor stencil (condbndymg /
handlesubgrid2, f3d_mgrid.F:2426-3092, icndbndy = 2) by the physics rather
than by restatement: a sphere of radius 0.3 at 1 V, off the grid's symmetry
points, in the box [-1, 1]^3 with rho = 0 and the Dirichlet faces set to the
exterior solution u = V R / r. The error outside the sphere falls by about
4 each time the cell halves (16, 32, 64 cells a side). The product's solve
equals the oracle's bit for bit on conductor problems
(tests/test_gpu_mg.py)."""
import numpy as np

from oracle import oracle

V, R, C = 1.0, 0.3, (0.013, -0.021, 0.007)


def _max_error(n):
    h = 2.0 / n
    oc = oracle.Conductors(n, n, n, h, h, h, -1.0, -1.0, -1.0)
    oc.add_shape("Sphere", R, 0.0, V, *C)
    oc.finalize()
    xs = -1.0 + (np.arange(n + 3) - 1) * h
    X, Y, Z = np.meshgrid(xs, xs, xs, indexing="ij")
    r = np.sqrt((X - C[0]) ** 2 + (Y - C[1]) ** 2 + (Z - C[2]) ** 2)
    u = V * R / r
    phi = np.zeros((n + 3,) * 3, order="F")
    for ax in range(3):
        for s in (1, n + 1):
            idx = [slice(None)] * 3
            idx[ax] = s
            phi[tuple(idx)] = u[tuple(idx)]
    rho = np.zeros((n + 1,) * 3, order="F")
    it, err = oracle.mgsolve(phi, rho, h, h, h, (0,) * 6, conductors=oc, mgtol=1e-13)
    assert it < 100
    core = (slice(1, -1),) * 3
    outside = r[core] > R
    return np.abs(phi[core] - u[core])[outside].max()


def test_sphere_potential_converges_at_second_order():
    e = [_max_error(n) for n in (16, 32, 64)]
    assert e[0] / e[1] > 3.2 and e[1] / e[2] > 3.2, e
    assert e[2] < 6e-4
