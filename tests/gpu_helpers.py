"""Shared set-up for the GPU parity tests."""
import numpy as np

from oracle import oracle


def make_solver(nx, ny, nz, mins, maxs, bounds, **kw):
    from warp_b200.multigrid import MultiGridB200
    return MultiGridB200(nx, ny, nz, mins[0], maxs[0], mins[1], maxs[1], mins[2], maxs[2], bounds=bounds,
                         mgverbose=-1, **kw)


def oracle_conductors(s, shapes):
    """Oracle conductor data for the same shapes on the solver's grid."""
    oc = oracle.Conductors(s.nx, s.ny, s.nz, s.dx, s.dy, s.dz, s.xmmin, s.ymmin, s.zmmin)
    for sh in shapes:
        kind = {0: "ZCylinderOut", 1: "ZCylinder", 2: "Sphere"}[sh.kind]
        oc.add_shape(kind, sh.radius, sh.length, sh.voltage, sh.xcent, sh.ycent, sh.zcent, sh.condid)
    oc.finalize()
    return oc


def as_set(data):
    ii, iv, il = data["interior"]
    si, sd, sv, sl = data["subgrid"]
    interior = {(tuple(a), float(v), int(l)) for a, v, l in zip(ii, iv, il)}
    sub = {(tuple(a), tuple(d), tuple(v), int(l)) for a, d, v, l in zip(si, sd, sv, sl)}
    return interior, sub


def gaussian_blobs_rho(nx, ny, nz, mins, maxs, nblob, seed, eps0):
    rng = np.random.Generator(np.random.Philox(seed))
    x = np.linspace(mins[0], maxs[0], nx + 1)
    y = np.linspace(mins[1], maxs[1], ny + 1)
    z = np.linspace(mins[2], maxs[2], nz + 1)
    dx = (maxs[0] - mins[0]) / nx
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    rho = np.zeros((nx + 1, ny + 1, nz + 1))
    for _ in range(nblob):
        c = [rng.uniform(mins[k] + 0.2 * (maxs[k] - mins[k]), maxs[k] - 0.2 * (maxs[k] - mins[k])) for k in range(3)]
        sig = rng.uniform(2, 6) * dx
        amp = rng.uniform(-1, 1)
        rho += amp * np.exp(-((X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2) / (2 * sig * sig))
    return np.asfortranarray(rho * eps0 * 1e4)
