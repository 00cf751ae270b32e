"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute calls: these run without a GPU)."""
import ctypes
import glob
import os
import re

import pytest

from conftest import ROOT, pkg


def declared_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*[A-Za-z_][\w\s\*]*?\b(eaf_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("eaf_cg_create", "eaf_cg_solve_f64", "eaf_cg_destroy",
                 "eaf_cg_solve_mixed"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = pkg().load()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_ctypes_signatures_cover_header():
    from importlib import import_module
    sigs = {n for n, _, _ in import_module("hornofusion-full3d_b200._lib").SIGNATURES}
    missing = [n for n in declared_functions() if n not in sigs]
    assert not missing, missing


def test_status_strings():
    lib = pkg().load()
    assert lib.eaf_status_string(0) == b"EAF_OK"
    assert lib.eaf_status_string(4) == b"EAF_ETIMEOUT"
    assert lib.eaf_status_string(99) == b"EAF_UNKNOWN"
    assert b"sm_100a" in lib.eaf_version()


def test_invalid_arguments_without_gpu():
    eaf = pkg()
    lib = eaf.load()
    h = ctypes.c_void_p()
    assert lib.eaf_cg_create(None, 4, 4, 4, 0) == eaf._lib.EAF_EINVAL
    assert lib.eaf_cg_create_mesh(ctypes.byref(h), 4, 4, 4, 1, 0) == \
        eaf._lib.EAF_EUNSUPPORTED
    assert lib.eaf_cg_destroy(None) == eaf._lib.EAF_EINVAL
    assert lib.eaf_selftest_barrier_timeout(0, -1.0) == eaf._lib.EAF_EINVAL


def test_struct_layouts_match_header(tmp_path):
    """ctypes mirrors of the public structs have the C compiler's sizes and
    field offsets."""
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    from importlib import import_module
    L = import_module("hornofusion-full3d_b200._lib")
    structs = {"eaf_pcorr_fields_t": L.PcorrFieldsC,
               "eaf_assembly_fields_t": L.AssemblyFieldsC,
               "eaf_phase_state_t": L.PhaseState,
               "eaf_phase_fields_t": L.PhaseFields}
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "eafcg.h"',
             "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["return 0; }"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o",
                    str(exe)], check=True)
    got = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    for line in got.splitlines():
        cname, field, val = line.split()
        py = structs[cname]
        want = ctypes.sizeof(py) if field == "size" else getattr(py, field).offset
        assert int(val) == want, (cname, field)
