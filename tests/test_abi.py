"""The C ABI surface without a GPU: the library loads, exports every entry
point include/pcc.h declares, and rejects bad arguments before touching a
device."""
import ctypes
import re

import pytest

from conftest import PKG, REPO


def declared():
    src = (REPO / "include" / "pcc.h").read_text()
    return sorted(set(re.findall(r"^(?:pcc_status|const char\*|int)\s+(pcc_[a-z0-9_]+)\(", src, re.M)))


def test_library_exports_every_declared_symbol():
    import pcc

    lib = pcc.load()
    names = declared()
    assert len(names) >= 19
    for name in names:
        assert hasattr(lib, name), name
    assert sorted(pcc.EXPORTS) == names


def test_status_strings():
    import pcc

    lib = pcc.load()
    for i, name in enumerate(pcc.STATUS):
        assert lib.pcc_status_string(i).decode() == name
    assert lib.pcc_status_string(999).decode() == "PCC_UNKNOWN"


def test_null_arguments_rejected_without_device():
    import pcc

    lib = pcc.load()
    assert lib.pcc_ctx_create(0, None, None) == 1
    assert lib.pcc_solve_create(None, None, None) == 1
    assert lib.pcc_shoot(None, None, None, None) == 1
    assert lib.pcc_jacobian(None, None, None, None, None) == 1
    assert lib.pcc_lu_solve(None, 0, None, None, None, 0, None) == 1
    assert lib.pcc_rhs_eval(None, 128, 4.0, 1, None, None, None) == 1
    assert lib.pcc_ctx_destroy(None) == 1
    assert lib.pcc_jacobian_batch(None, 1, None, None, None, None, None) == 1
    assert lib.pcc_newton_begin(None, None) == 1
    assert lib.pcc_newton_iterate(None, 1, None, 0, None, None) == 1
    assert lib.pcc_newton_result(None, None, None) == 1
    assert lib.pcc_newton_solve(None, 1, None, None, 0, None, None) == 1
    assert lib.pcc_serve_start(None, None) == 1
    assert lib.pcc_submit(None, None, None) == 1
    assert lib.pcc_poll(None, 1, None, None) == 1
    assert lib.pcc_wait(None, 1, 0.0, None, None) == 1
    assert lib.pcc_serve_stats(None, None) == 1
    assert lib.pcc_serve_stop(None) == 1


def test_struct_layouts_match_header(tmp_path):
    """ctypes mirrors of the pcc.h structs agree with the C compiler's layout."""
    import shutil
    import subprocess

    import pcc

    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    structs = {"pcc_solve_desc": pcc.SolveDesc, "pcc_stats": pcc.Stats, "pcc_refine_report": pcc.RefineReport,
               "pcc_newton_state": pcc.NewtonState, "pcc_serve_opts": pcc.ServeOpts, "pcc_request": pcc.Request,
               "pcc_result": pcc.Result, "pcc_serve_info": pcc.ServeInfo}
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "pcc.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'printf("{cname}.{f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I" + str(REPO / "include"), str(src), "-o", str(exe)], check=True)
    got = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True).stdout.splitlines())
    for cname, py in structs.items():
        assert int(got[cname]) == ctypes.sizeof(py), cname
        for f, _ in py._fields_:
            assert int(got[f"{cname}.{f}"]) == getattr(py, f).offset, (cname, f)


def test_library_built_for_sm100a():
    so = PKG / "libpcc_b200.so"
    data = so.read_bytes()
    assert b"sm_100a" in data or b"sm_100" in data
