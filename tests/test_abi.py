"""C-ABI boundary checks that need no GPU: the library loads, exports every
entry point declared in include/rsg.h, and its host-only calls behave."""
import ctypes as C
import os
import subprocess

import pytest

from rsg import _lib


def test_library_exports_every_header_symbol():
    lib = _lib.load()
    names = _lib.header_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"declared in include/rsg.h but not exported: {missing}"


def test_python_binding_covers_header():
    names = set(_lib.header_symbols())
    assert names <= set(_lib.SIGNATURES), sorted(names - set(_lib.SIGNATURES))


def test_exports_are_plain_c_symbols():
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    for n in _lib.header_symbols():
        assert n in exported  # unmangled: extern "C"


def test_conf_default_and_status_strings():
    lib = _lib.load()
    c = _lib.SolverConf()
    lib.rsg_conf_default(C.byref(c))
    assert c.solver_type == _lib.SOLVER_CG and c.n_outer == 1000 and c.n_inner == 30
    assert c.cvg == 1e-13 and c.output_frequency == 0 and c.scale_equations == 1
    assert lib.rsg_status_string(_lib.OK) == b"ok"
    assert b"converged" in lib.rsg_status_string(_lib.NOT_CONVERGED)


def test_no_device_is_an_error_not_a_crash():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    lib = _lib.load()
    h = C.c_void_p()
    assert lib.rsg_context_create(0, C.byref(h)) != _lib.OK
    assert not h.value


def test_rsg_package_fails_loudly_without_library(tmp_path, monkeypatch):
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "missing.so"))
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        _lib.load()


def test_struct_layouts_match_header(tmp_path):
    """The ctypes mirrors of the public structs have the C compiler's size and field offsets."""
    structs = {"rsg_solver_conf": _lib.SolverConf, "rsg_stats": _lib.Stats, "rsg_time": _lib.Time,
               "rsg_tune_info": _lib.TuneInfo, "rsg_model_groups": _lib.ModelGroups, "rsg_amg_info": _lib.AmgInfo}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "rsg.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'printf("{cname}.{f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(_lib.REPO, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    got = dict(line.rsplit(" ", 1) for line in out.splitlines() if line)
    for cname, py in structs.items():
        assert int(got[cname]) == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert int(got[f"{cname}.{f}"]) == getattr(py, f).offset, f"{cname}.{f}"
