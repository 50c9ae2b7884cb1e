"""The C-ABI library loads here (no GPU) and exports every function that
include/*.h declares, with C linkage."""
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(snapmrf_\w+)\s*\(", text, re.M):
            names.append(m.group(1))
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    for required in ["snapmrf_mrf_dict", "snapmrf_mrf_match", "snapmrf_last_error", "snapmrf_ra_read",
                     "snapmrf_parse_params", "snapmrf_trans_params", "snapmrf_normalize"]:
        assert required in names


@pytest.mark.parametrize("name", declared_functions())
def test_symbol_exported(snap, name):
    assert hasattr(snap.lib(), name)


def test_exports_are_c_linkage(snap):
    out = subprocess.run(["nm", "-D", "--defined-only", str(snap.api.LIB_PATH)], capture_output=True,
                         text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    for name in declared_functions():
        assert name in exported, name


def test_header_compiles_as_c(tmp_path):
    src = tmp_path / "t.c"
    src.write_text('#include "snapmrf.h"\nint main(void){ return snapmrf_version() == 0; }\n')
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-fsyntax-only", f"-I{ROOT / 'include'}",
                    str(src)], check=True)


STRUCTS = {"DictOpts": "snapmrf_dict_opts", "MatchOpts": "snapmrf_match_opts", "SvdOpts": "snapmrf_svd_opts",
           "RA": "snapmrf_ra"}


@pytest.mark.parametrize("py_name", sorted(STRUCTS))
def test_ctypes_structs_match_the_header(snap, tmp_path, py_name):
    """Every ctypes mirror of an option / RA struct has the header's size and
    field offsets (a field added on one side only would shift the rest)."""
    import ctypes
    cls = getattr(snap.api, py_name)
    c_name = STRUCTS[py_name]
    fields = [f[0] for f in cls._fields_]
    lines = [f'printf("sizeof() %zu\\n", sizeof({c_name}));']
    lines += [f'printf("{f} %zu\\n", offsetof({c_name}, {f}));' for f in fields]
    src = tmp_path / "s.c"
    src.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "snapmrf.h"\nint main(void){\n'
                   + "\n".join(lines) + "\nreturn 0; }\n")
    exe = tmp_path / "s"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", f"-I{ROOT / 'include'}", str(src), "-o", str(exe)],
                   check=True)
    out = dict(ln.split() for ln in subprocess.run([str(exe)], capture_output=True, text=True,
                                                   check=True).stdout.splitlines())
    assert int(out["sizeof()"]) == ctypes.sizeof(cls)
    for f in fields:
        assert int(out[f]) == getattr(cls, f).offset, f
