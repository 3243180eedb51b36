"""The ctypes mirrors of the C-ABI structs (simox_b200/_abi.py) have the
layout the compiler gives include/simox_gpu.h: same size and the same offset
for every field.  Compiles a small C program with the system C compiler; no
GPU needed."""
import ctypes as C
import os
import shutil
import subprocess

import pytest

from simox_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PAIRS = [("simox_metl", _abi.Metl), ("simox_potn", _abi.Potn), ("simox_oxid", _abi.Oxid),
         ("simox_potential", _abi.Potential), ("simox_setup", _abi.Setup), ("simox_energies", _abi.Energies),
         ("simox_ctip_report", _abi.CtipReport), ("simox_md_opts", _abi.MdOpts), ("simox_tuning", _abi.Tuning),
         ("simox_eam_spline", _abi.EamSpline), ("simox_adjoint_report", _abi.AdjointReport),
         ("simox_oxidation", _abi.Oxidation)]

# ctypes names that differ from the C member (Python keywords)
RENAME = {("simox_metl", "lambda_"): "lambda"}


def _cfield(cname, fname):
    return RENAME.get((cname, fname), fname)


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "simox_gpu.h"', "int main(void) {"]
    for cname, cls in PAIRS:
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {_cfield(cname, fname)}));')
    lines += ["  return 0;", "}"]
    d = tmp_path_factory.mktemp("abi")
    src, exe = d / "layout.c", d / "layout"
    src.write_text("\n".join(lines) + "\n")
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)], check=True,
                   capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    table = {}
    for line in out.splitlines():
        cname, field, value = line.split()
        table[(cname, field)] = int(value)
    return table


@pytest.mark.parametrize("cname,cls", PAIRS, ids=[p[0] for p in PAIRS])
def test_struct_layout_matches_header(c_layout, cname, cls):
    assert C.sizeof(cls) == c_layout[(cname, "size")], cname
    for fname, _ in cls._fields_:
        assert getattr(cls, fname).offset == c_layout[(cname, fname)], (cname, fname)


@pytest.mark.parametrize("lang", ["c99", "c++11"])
def test_header_compiles_strict(tmp_path, lang):
    """include/simox_gpu.h is plain C (and C++) for any caller: no warnings
    under -std=c99 / -std=c++11 -Wall -Wextra -pedantic."""
    cc = shutil.which("gcc" if lang == "c99" else "g++")
    if cc is None:
        pytest.skip("no compiler")
    src = tmp_path / "h.c"
    src.write_text('#include "simox_gpu.h"\nint main(void) { return 0; }\n')
    cmd = [cc, f"-std={lang}", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", os.path.join(ROOT, "include"),
           "-c", str(src), "-o", str(tmp_path / "h.o")]
    if lang != "c99":
        cmd[1:1] = ["-x", "c++"]
    subprocess.run(cmd, check=True, capture_output=True)
