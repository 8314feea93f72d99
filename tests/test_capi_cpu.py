"""CPU checks of the C ABI: the library loads without a GPU, exports every
function include/*.h declares, and its structures have the reference layout."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

from obit_b200 import _lib

ROOT = Path(__file__).resolve().parent.parent
HEADERS = sorted((ROOT / "include").glob("*.h"))


def declared_functions():
    names = []
    for h in HEADERS:
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"([A-Za-z_][\w\s\*]*?)\b([A-Za-z_]\w*)\s*\(([^;{]*?)\)\s*;", text):
            ret, name = m.group(1).strip(), m.group(2)
            if ret.startswith("typedef") or name in ("if", "while", "for", "return", "sizeof"):
                continue
            names.append(name)
    return names


def test_headers_declare_api():
    names = declared_functions()
    for must in ("ObitCUDASkyModelDFTInit", "ObitCUDASkyModelDFTSetMod", "ObitCUDASkyModelDFTCalc",
                 "ObitCUDASkyModelDFTShutdown", "obit_dft_calc", "obit_gpu_skymodel_dft_calc"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.lib_path())], capture_output=True,
                         text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing
    for n in declared_functions():
        getattr(lib, n)


def test_bindings_cover_declarations():
    assert set(declared_functions()) == set(_lib.SIGNATURES)


def test_version_and_error_string_without_gpu():
    lib = _lib.load()
    assert lib.obit_dft_version() >= 100
    assert isinstance(lib.obit_dft_last_error(), bytes)


def test_null_gpuinfo_is_an_error_not_a_crash():
    lib = _lib.load()
    assert lib.obit_dft_calc(None) == 1
    assert b"NULL" in lib.obit_dft_last_error()
    assert lib.obit_dft_shutdown(None) == 1


# Byte offsets of the reference structures on LP64 (x86-64), from
# ObitCUDASkyModelInfoDef.h:66-195 compiled with gcc (tests/golden/make_struct_offsets.py).
def test_struct_layout_matches_reference():
    import json

    ref = json.loads((ROOT / "tests" / "golden" / "struct_offsets.json").read_text())
    for sname, cls in (("GPUVisInfo", _lib.GPUVisInfo), ("GPUModelInfo", _lib.GPUModelInfo),
                       ("GPUInfo", _lib.GPUInfo)):
        assert C.sizeof(cls) == ref[sname]["sizeof"], sname
        for fname, off in ref[sname]["offsets"].items():
            assert getattr(cls, fname).offset == off, (sname, fname)


def test_c_header_layout_matches_bindings(tmp_path):
    """Compile a probe against include/obit_dft.h and compare with ctypes."""
    import json

    src = tmp_path / "probe.c"
    fields = {
        "GPUVisInfo": [f[0] for f in _lib.GPUVisInfo._fields_],
        "GPUModelInfo": [f[0] for f in _lib.GPUModelInfo._fields_],
        "GPUInfo": [f[0] for f in _lib.GPUInfo._fields_],
        "ObitDFTBeamImages": [f[0] for f in _lib.ObitDFTBeamImages._fields_],
    }
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "obit_dft.h"', "int main(void){"]
    lines.append('printf("{");')
    first = True
    for s, fl in fields.items():
        lines.append(f'printf("{"," if not first else ""}\\"{s}\\": {{\\"sizeof\\": %zu, \\"offsets\\": {{", sizeof({s}));')
        for i, f in enumerate(fl):
            sep = "," if i else ""
            lines.append(f'printf("{sep}\\"{f}\\": %zu", offsetof({s}, {f}));')
        lines.append('printf("}}");')
        first = False
    lines.append('printf("}\\n"); return 0; }')
    src.write_text("\n".join(lines))
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    got = json.loads(subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout)
    for s, cls in (("GPUVisInfo", _lib.GPUVisInfo), ("GPUModelInfo", _lib.GPUModelInfo),
                   ("GPUInfo", _lib.GPUInfo), ("ObitDFTBeamImages", _lib.ObitDFTBeamImages)):
        assert got[s]["sizeof"] == C.sizeof(cls)
        for f, off in got[s]["offsets"].items():
            assert getattr(cls, f).offset == off
