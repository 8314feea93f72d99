"""Regenerate struct_offsets.json: byte offsets of GPUVisInfo, GPUModelInfo and
GPUInfo as the reference header declares them
(ObitSystem/Obit/include/ObitCUDASkyModelInfoDef.h:66-195), compiled with gcc
on this LP64 host.  Needs the reference tree: its Obit include directory as the
first argument, else $OBIT_REFERENCE/ObitSystem/Obit/include, else the
reference checked out beside this repository (../reference).  The JSON is
committed."""
import json
import os
import subprocess
import sys
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "struct_offsets.json"


def ref_include() -> Path:
    if len(sys.argv) > 1:
        return Path(sys.argv[1])
    root = os.environ.get("OBIT_REFERENCE") or str(HERE.parent.parent.parent / "reference")
    return Path(root) / "ObitSystem" / "Obit" / "include"

FIELDS = {
    "GPUVisInfo": ["nvis", "nprod", "nrparm", "lenvis", "nchan", "ilocu", "ilocv", "ilocw", "iloct",
                   "ilocb", "ilocsu", "chanb", "chane", "incf", "nIF", "IFb", "IFe", "incif",
                   "nstok", "stokb", "stoke", "incs", "stype", "kincif", "kincf", "freqRat",
                   "d_freqRat", "freqScale"],
    "GPUModelInfo": ["nterm", "size", "doSwap", "type", "opType", "specIndex", "d_specIndex",
                     "nmodel", "model", "stokFact"],
    "GPUInfo": ["nvis", "nchan", "nrparm", "lenvis", "modelSize", "nstream", "prtLv",
                "oldnVisPIO", "cuda_device", "bufferSize", "nmodel", "d_model", "d_freq",
                "h_data", "d_data", "d_visInfo", "h_visInfo", "d_modelInfo", "h_modelInfo",
                "stream", "cycleDone"],
}


def main():
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "ObitCUDASkyModelInfoDef.h"',
             "int main(void){"]
    for s, fl in FIELDS.items():
        lines.append(f'printf("{s} sizeof %zu\\n", sizeof({s}));')
        for f in fl:
            lines.append(f'printf("{s} {f} %zu\\n", offsetof({s}, {f}));')
    lines.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        src = Path(d) / "p.c"
        src.write_text("\n".join(lines))
        subprocess.run(["gcc", "-I", str(ref_include()), str(src), "-o", str(Path(d) / "p")], check=True)
        out = subprocess.run([str(Path(d) / "p")], capture_output=True, text=True, check=True).stdout
    res = {s: {"sizeof": 0, "offsets": {}} for s in FIELDS}
    for ln in out.splitlines():
        s, f, v = ln.split()
        if f == "sizeof":
            res[s]["sizeof"] = int(v)
        else:
            res[s]["offsets"][f] = int(v)
    res["_source"] = "ObitSystem/Obit/include/ObitCUDASkyModelInfoDef.h:66-195, gcc x86-64"
    OUT.write_text(json.dumps(res, indent=1) + "\n")
    print(OUT)


if __name__ == "__main__":
    main()
