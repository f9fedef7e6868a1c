"""The C ABI library loads and exports every entry point include/abd_b200.h declares
(no compute calls: these run without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "abd_b200.h")
LIB = os.path.join(ROOT, "abd_warp_b200", "libabd_b200.so")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(abd_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "abd_step" in names and "abd_sim_create" in names
    assert len(names) >= 15


def test_library_exports_every_declared_symbol():
    if not os.path.exists(LIB):
        pytest.skip("libabd_b200.so not built")
    lib = ctypes.CDLL(LIB)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_matches_header():
    from abd_warp_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libabd_b200.so not built")
    assert set(_lib.exported_symbols()) <= set(declared_functions())


def test_status_strings():
    from abd_warp_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libabd_b200.so not built")
    L = _lib.load()
    assert L.abd_status_string(0) == b"ok"
    assert L.abd_status_string(3) == b"capacity could not be grown"


def test_create_rejects_mixed_precision():
    """precision 1 (FP32 Krylov inside FP64 refinement) is refused before any device work:
    the refinement diverges on contact systems (tests/test_mixed_precision.py)."""
    import numpy as np
    from abd_warp_b200 import _lib, scenes
    from abd_warp_b200.params import PRECISION_MIXED, SimParams
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libabd_b200.so not built")
    L = _lib.load()
    bodies, prm, _ = scenes.make_config(0)
    f = scenes.flatten_bodies(bodies)
    host = {k: np.ascontiguousarray(f[k], dtype=np.int32 if k in ("voff", "toff", "eoff", "tris", "edges", "fixed")
                                    else np.float64)
            for k in ("voff", "toff", "eoff", "x0", "tris", "edges", "mass", "I0", "fixed")}
    hp = {k: v.ctypes.data_as(ctypes.c_void_p) for k, v in host.items()}
    desc = _lib.SceneDesc(len(bodies), hp["voff"], hp["toff"], hp["eoff"], hp["x0"], hp["tris"], hp["edges"],
                          hp["mass"], hp["I0"], hp["fixed"])
    cprm = SimParams(precision=PRECISION_MIXED).to_c()
    h = ctypes.c_void_p()
    rc = L.abd_sim_create(ctypes.byref(desc), ctypes.byref(cprm), None, ctypes.byref(h))
    assert rc == _lib.ABD_ERR_INVALID and not h.value


def test_create_rejects_malformed_scenes():
    """A malformed scene is refused with ABD_ERR_INVALID before any device work: no bodies,
    offsets not starting at 0 or decreasing, a triangle or edge index outside its body, a
    non-finite rest position, a free body without positive mass or I0."""
    import numpy as np
    from abd_warp_b200 import _lib, scenes
    from abd_warp_b200.params import SimParams
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libabd_b200.so not built")
    L = _lib.load()
    bodies, prm, _ = scenes.make_config(0)
    f = scenes.flatten_bodies(bodies)
    ints = ("voff", "toff", "eoff", "tris", "edges", "fixed")
    base = {k: np.ascontiguousarray(f[k], dtype=np.int32 if k in ints else np.float64)
            for k in ("voff", "toff", "eoff", "x0", "tris", "edges", "mass", "I0", "fixed")}
    free = int(np.flatnonzero(base["fixed"] == 0)[0])

    def create(mod, n=None, prm=None):
        host = {k: v.copy() for k, v in base.items()}
        mod(host)
        hp = {k: v.ctypes.data_as(ctypes.c_void_p) for k, v in host.items()}
        desc = _lib.SceneDesc(len(bodies) if n is None else n, hp["voff"], hp["toff"], hp["eoff"], hp["x0"],
                              hp["tris"], hp["edges"], hp["mass"], hp["I0"], hp["fixed"])
        cprm = (prm or SimParams()).to_c()
        h = ctypes.c_void_p()
        rc = L.abd_sim_create(ctypes.byref(desc), ctypes.byref(cprm), None, ctypes.byref(h))
        return rc, h.value

    def setter(key, idx, val):
        def f_(h):
            h[key].reshape(-1)[idx] = val
        return f_

    cases = [
        (lambda h: None, 0),                                   # no bodies
        (setter("voff", 0, 1), None),                           # offsets start past 0
        (setter("toff", 1, int(base["toff"][0]) - 1), None),    # decreasing offsets
        (setter("tris", 0, int(base["voff"][-1])), None),       # triangle index out of range
        (setter("edges", 1, -1), None),                         # edge index out of range
        (setter("x0", 4, float("nan")), None),                  # non-finite rest position
        (setter("mass", free, 0.0), None),                      # free body without mass
        (setter("I0", free, float("inf")), None),               # non-finite I0
    ]
    def empty_body(h):  # body 0 loses its vertices (they go to body 1), keeps no primitives
        h["voff"][1] = 0
        h["toff"][1] = 0
        h["eoff"][1] = 0

    cases.append((empty_body, None))                            # a body without vertices
    for mod, n in cases:
        rc, h = create(mod, n)
        assert rc == _lib.ABD_ERR_INVALID and not h
    rc, h = create(lambda h: None, prm=SimParams(min_capacity=-1))  # negative injected capacity
    assert rc == _lib.ABD_ERR_INVALID and not h


def _c_layout(tmp_path, struct, fields):
    """sizeof and field offsets of a struct of include/abd_b200.h, from a C program built here."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    src = tmp_path / "layout.c"
    lines = ['#include <stddef.h>', '#include <stdio.h>', f'#include "{HEADER}"', "int main(void) {",
             f'  printf("%zu\\n", sizeof({struct}));']
    lines += [f'  printf("%zu\\n", offsetof({struct}, {f}));' for f in fields]
    lines += ["  return 0;", "}"]
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-o", str(exe), str(src)], check=True)
    out = [int(v) for v in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    return out[0], out[1:]


def test_ctypes_structs_match_the_header(tmp_path):
    """The Python mirrors of abd_params, abd_scene_desc, abd_states and abd_step_info have the
    C header's field offsets and sizes (the library reads them by the C layout)."""
    from abd_warp_b200 import _lib
    from abd_warp_b200.params import CParams
    for struct, cls in (("abd_params", CParams), ("abd_scene_desc", _lib.SceneDesc), ("abd_states", _lib.States),
                        ("abd_step_info", _lib.StepInfo)):
        names = [f[0] for f in cls._fields_]
        size, offs = _c_layout(tmp_path, struct, names)
        assert ctypes.sizeof(cls) == size, struct
        assert [getattr(cls, n).offset for n in names] == offs, struct
