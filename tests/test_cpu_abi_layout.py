"""The ctypes mirror of the C-ABI (warp_b200/_lib.py) against the header
include/warp_b200.h, compiled here with gcc: every struct has the same size
and field offsets, and every status code, solve flag, centre and profiling
kind has the same value. A mismatch would pass wrong arguments across the
boundary without any error."""
import ctypes
import json
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

STRUCTS = {
    "wg_grid": "Grid",
    "wg_solve_opts": "SolveOpts",
    "wg_solve_stats": "SolveStats",
    "wg_particles": "Particles",
    "wg_particles_f32": "ParticlesF32",
    "wg_push_params": "PushParams",
}
CONSTANTS = {
    "WG_OK": "WG_OK", "WG_SOLVE_GRAPH": "SOLVE_GRAPH", "WG_SOLVE_PDL": "SOLVE_PDL",
    "WG_CENTER_FULLV": "CENTER_FULLV", "WG_CENTER_HALFV": "CENTER_HALFV", "WG_CENTER_SYNCHV": "CENTER_SYNCHV",
    "WG_PROF_SOR0": "PROF_SOR0", "WG_PROF_DEPOSIT": "PROF_DEPOSIT", "WG_PROF_ADVANCE": "PROF_ADVANCE",
    "WG_PROF_RESID0": "PROF_RESID0", "WG_PROF_RESTRICT0": "PROF_RESTRICT0", "WG_PROF_EXPAND0": "PROF_EXPAND0",
    "WG_PROF_CORR": "PROF_CORR", "WG_PROF_COARSE": "PROF_COARSE",
}
ERRORS = ["WG_EINVAL", "WG_ECUDA", "WG_ESTATE", "WG_EOVERFLOW", "WG_ENODEV", "WG_ENOMEM", "WG_ETOOLARGE"]


def _c_layout(tmp_path):
    from warp_b200 import _lib
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "warp_b200.h"', "int main(void) {",
             'printf("{");']
    first = True
    for cname, pname in STRUCTS.items():
        fields = [f[0] for f in getattr(_lib, pname)._fields_]
        parts = ['\\"size\\": %zu']
        args = ["sizeof(%s)" % cname]
        for f in fields:
            parts.append('\\"%s\\": %%zu' % f)
            args.append("offsetof(%s, %s)" % (cname, f))
        fmt = ("" if first else ", ") + '\\"%s\\": {%s}' % (cname, ", ".join(parts))
        lines.append('printf("%s", %s);' % (fmt, ", ".join(args)))
        first = False
    for name in list(CONSTANTS) + ERRORS:
        lines.append('printf(", \\"%s\\": %%d", (int)(%s));' % (name, name))
    lines += ['printf("}\\n");', "return 0; }"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    return json.loads(subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout)


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_ctypes_mirror_matches_the_header(tmp_path):
    from warp_b200 import _lib
    c = _c_layout(tmp_path)
    for cname, pname in STRUCTS.items():
        cls = getattr(_lib, pname)
        assert ctypes.sizeof(cls) == c[cname]["size"], cname
        for f in cls._fields_:
            assert getattr(cls, f[0]).offset == c[cname][f[0]], (cname, f[0])
    for cname, pname in CONSTANTS.items():
        assert getattr(_lib, pname) == c[cname], cname
    for name in ERRORS:
        assert _lib.ERRORS[c[name]] == name


def _c_kind(param):
    """Coarse class of one C parameter declaration."""
    p = " ".join(param.replace("const", " ").split())
    if "*" in p:
        base = p.split("*")[0].strip()
        depth = p.count("*")
        return ("ptr", base if depth == 1 else "void")
    typ = p.rsplit(" ", 1)[0] if " " in p else p
    return {"double": ("double",), "int64_t": ("i64",), "int": ("i32",), "int32_t": ("i32",)}[typ]


def _py_kind(t):
    from warp_b200 import _lib
    if t is ctypes.c_void_p:
        return ("ptr", None)
    if isinstance(t, type) and issubclass(t, ctypes._Pointer):
        target = t._type_
        names = {ctypes.c_double: "double", ctypes.c_int32: "int32_t", ctypes.c_int64: "int64_t",
                 ctypes.c_void_p: "void"}
        for cname, pname in STRUCTS.items():
            if target is getattr(_lib, pname):
                return ("ptr", cname)
        return ("ptr", names.get(target, "?"))
    if t is ctypes.c_double:
        return ("double",)
    if t is ctypes.c_int64:
        return ("i64",)
    if t is ctypes.c_int:
        return ("i32",)
    raise AssertionError(t)


def test_ctypes_argtypes_match_the_prototypes():
    import re
    from warp_b200 import _lib
    text = open(os.path.join(ROOT, "include", "warp_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    protos = {m.group(1): m.group(2) for m in re.finditer(r"\bint\s+(wg_\w+)\s*\(([^;]*)\)\s*;", text, re.S)}
    assert set(protos) == set(_lib.SIGNATURES), set(protos) ^ set(_lib.SIGNATURES)
    for name, args in _lib.SIGNATURES.items():
        params = [s for s in (x.strip() for x in protos[name].split(",")) if s and s != "void"]
        assert len(params) == len(args), name
        for c, t in zip(params, args):
            ck, pk = _c_kind(c), _py_kind(t)
            assert ck[0] == pk[0], (name, c)
            # typed ctypes pointers must point at the declared type; c_void_p takes any pointer
            if ck[0] == "ptr" and pk[1] is not None:
                same = pk[1] == ck[1] or (pk[1] == "int32_t" and ck[1] == "int") or \
                    (pk[1] == "void" and ck[1] in ("wg_ctx", "void"))
                assert same, (name, c, pk)
