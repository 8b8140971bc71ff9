"""CPU-side checks of the product: the C-ABI library loads and exports every
symbol declared in include/warp_b200.h (no compute calls: no GPU here), and
the host-side set-up logic (lattice tables, beam loader) agrees with the
oracle."""
import ctypes
import os
import re

import numpy as np
import pytest

from oracle import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "warp_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(wg_\w+)\s*\(", txt, re.M)))


def test_library_exports_header_symbols():
    from warp_b200 import _lib
    syms = header_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(_lib.lib, s), s
    assert sorted(_lib.exported_symbols()) == syms


def test_library_is_sm100a_build():
    """The in-tree library exists and the build compiles every source under
    warp_b200/csrc for sm_100a only, with FMA contraction off."""
    from warp_b200 import _lib, build
    assert os.path.exists(_lib.LIBPATH) and _lib.LIBPATH == build.LIB
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    srcs = sorted(f for f in os.listdir(build.CSRC) if f.endswith((".cu", ".cpp")))
    assert sorted(build.SOURCES) == srcs
    import inspect
    body = inspect.getsource(build.build)
    assert "--fmad=false" in body and "-lineinfo" in body


def test_lattice_tables_match_oracle():
    from warp_b200.lattice import fodo
    lat = fodo(15.0, 0.10, 0.50)
    zs = np.array([q.zs for q in lat.quads])
    ze = np.array([q.ze for q in lat.quads])
    db = np.array([q.db for q in lat.quads])
    for (zlmin, dzl, nzl) in [(0.0, 1.0 / 64, 65), (0.0, 1.0 / 512, 513), (-0.3, 0.0071, 400)]:
        mine = lat.tables(zlmin, dzl, nzl)
        ref = oracle.quad_tables(zs, ze, db, lat.zlatperi, lat.zlatstrt, zlmin, dzl, nzl)
        for a, b in zip(mine, ref):
            assert np.array_equal(a, b)


def test_fodo_territories():
    from warp_b200.lattice import fodo
    lat = fodo(15.0, 0.10, 0.50)
    czs, cze, cdb = lat.tables(0.0, 0.01, 100)
    # cell centred at z = 0.0 -> focusing quad [-0.05, 0.05]
    assert (czs[0], cze[0], cdb[0]) == pytest.approx((-0.05, 0.05, 15.0))
    # z = 0.25 -> defocusing quad [0.20, 0.30]
    assert (czs[25], cze[25], cdb[25]) == pytest.approx((0.20, 0.30, -15.0))
    # z = 0.45 -> next period's focusing quad [0.45, 0.55]
    assert (czs[45], cze[45], cdb[45]) == pytest.approx((0.45, 0.55, 15.0))


def test_semigaussian_statistics():
    from warp_b200.particles import semigaussian
    p = semigaussian(200_000, seed=0, radius=2e-3, angle_rms=5e-3)
    r = np.hypot(p["x"], p["y"])
    assert r.max() <= 2e-3
    assert np.mean(r ** 2) == pytest.approx(0.5 * 2e-3 ** 2, rel=0.02)
    assert np.std(p["ux"] / p["uz"]) == pytest.approx(5e-3, rel=0.02)
    q = semigaussian(1000, seed=0)
    assert np.array_equal(q["x"], semigaussian(1000, seed=0)["x"])


def test_oracle_field_energy_matches_direct_sum():
    """or_ese (getese3dfromrhophi) equals dx dy dz / 2 * sum(rho * phi) on the
    nodes, to rounding."""
    import numpy as np
    from oracle import oracle
    rng = np.random.default_rng(4)
    rho = np.asfortranarray(rng.standard_normal((9, 7, 12)))
    phi = np.asfortranarray(rng.standard_normal((11, 9, 14)))
    e = oracle.ese(rho, phi, 0.1, 0.2, 0.05)
    ref = 0.1 * 0.2 * 0.05 * 0.5 * np.sum(rho * phi[1:-1, 1:-1, 1:-1])
    assert abs(e - ref) <= 1e-12 * np.sum(np.abs(rho * phi[1:-1, 1:-1, 1:-1]))


def test_product_never_imports_the_oracle():
    """The oracle is test infrastructure: no module of the warp_b200 package
    imports it, so no product path can route through it."""
    import ast
    pkg = os.path.join(ROOT, "warp_b200")
    for name in sorted(os.listdir(pkg)):
        if not name.endswith(".py"):
            continue
        tree = ast.parse(open(os.path.join(pkg, name)).read())
        for node in ast.walk(tree):
            if isinstance(node, ast.Import):
                mods = [a.name for a in node.names]
            elif isinstance(node, ast.ImportFrom):
                mods = [node.module or ""]
            else:
                continue
            assert not any(m == "oracle" or m.startswith("oracle.") for m in mods), (name, mods)
