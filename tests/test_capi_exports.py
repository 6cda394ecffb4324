"""The C-ABI library loads without a GPU and exports every symbol the header declares."""

import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "topo3d_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b(tp3d_\w+)\s*\(", src)
    return sorted(set(n for n in names if not n.startswith("tp3d_solver_opts")))


@pytest.fixture(scope="module")
def libpath():
    from pytopo3d_b200 import _build

    return _build.build()


def test_header_declares_the_expected_entry_points():
    names = _declared()
    for n in ["tp3d_filter_project", "tp3d_filter_transpose", "tp3d_filter_rowsum", "tp3d_heaviside",
              "tp3d_element_compliance", "tp3d_sensitivity", "tp3d_oc_update", "tp3d_solver_create",
              "tp3d_solver_solve", "tp3d_solver_apply_f64", "tp3d_solver_apply_f32"]:
        assert n in names


def test_library_exports_every_declared_symbol(libpath):
    L = ctypes.CDLL(libpath)
    missing = [n for n in _declared() if not hasattr(L, n)]
    assert not missing, missing


def test_python_binding_covers_the_header(libpath):
    from pytopo3d_b200 import _lib

    assert set(_declared()) <= set(_lib.SIGNATURES), set(_declared()) - set(_lib.SIGNATURES)
    L = _lib.lib()
    assert L.tp3d_abi_version() == 1
    # host-only entry points work without a device
    assert L.tp3d_sensitivity_scratch_bytes(4, 3, 2) >= 2 * 24 * 8
    assert L.tp3d_oc_scratch_bytes(4, 3, 2, 1.5) >= 24 * 8
    o = _lib.SolverOpts()
    L.tp3d_solver_default_opts(ctypes.byref(o))
    assert o.precision == 0 and o.rtol == pytest.approx(1e-10)


def test_bad_arguments_are_rejected_on_the_host(libpath):
    from pytopo3d_b200 import _lib

    L = _lib.lib()
    assert L.tp3d_filter_project(0, 1, 1, 1.5, None, None, 1.0, 0.5, None, None, None, None, None,
                                 None) == _lib.TP3D_ERR_ARG
    assert L.tp3d_heaviside(None, 4, 1.0, 0.5, None, None, None) == _lib.TP3D_ERR_ARG
    assert L.tp3d_oc_update(2, 2, 2, 1.5, None, None, None, None, None, None, 0.2, 1.0, 1.0, 0.5, 80,
                            1e-8, None, None, None, None, None) == _lib.TP3D_ERR_ARG
    with pytest.raises(ValueError):
        _lib.check(_lib.TP3D_ERR_ARG, "x")


@pytest.mark.parametrize("cname,pyname", [("tp3d_solver_opts", "SolverOpts"), ("tp3d_stage_desc", "StageDesc")])
def test_ctypes_structs_mirror_the_header(tmp_path, cname, pyname):
    """The Python mirror of each struct the header passes by pointer has the C
    layout: a C program built with the header prints every field's offset and
    the struct's size, and ctypes must agree on each of them."""
    import shutil
    import subprocess

    from pytopo3d_b200 import _lib

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    mirror = getattr(_lib, pyname)
    lines = [f'printf("%zu\\n", sizeof({cname}));']
    lines += [f'printf("%zu\\n", offsetof({cname}, {n}));' for n, _ in mirror._fields_]
    src = tmp_path / "layout.c"
    src.write_text("#include <stddef.h>\n#include <stdio.h>\n#include \"topo3d_b200.h\"\n"
                   "int main(void) {\n" + "\n".join(lines) + "\nreturn 0;\n}\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    assert got[0] == ctypes.sizeof(mirror)
    assert got[1:] == [getattr(mirror, n).offset for n, _ in mirror._fields_]
