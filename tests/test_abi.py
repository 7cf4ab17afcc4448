"""The C-ABI library: loads on CPU and exports every entry point that
include/dmrg2_b200.h declares (no compute calls without a GPU)."""
import ctypes
import re
import subprocess
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parent.parent
HEADER = REPO / "include" / "dmrg2_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dmrg2_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    import dmrg2
    return dmrg2.load_library()


def test_header_declares_entry_points():
    names = declared_functions()
    assert "dmrg2_create" in names and "dmrg2_op_heff" in names
    assert len(names) >= 18


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_mirror_binds_every_declared_symbol():
    import dmrg2
    assert sorted(dmrg2.EXPORTED) == declared_functions()


def test_abi_version(lib):
    assert lib.dmrg2_abi_version() == 7


def test_null_arguments_are_rejected_without_touching_the_gpu(lib):
    h = ctypes.c_void_p()
    assert lib.dmrg2_create(None, ctypes.byref(h)) == 1
    assert b"null" in lib.dmrg2_last_error(None)
    assert lib.dmrg2_run(None, None, 1, None, 0, None) == 1


def test_invalid_shapes_are_rejected(lib):
    import dmrg2
    # dtype 7 is not a valid dmrg2_dtype; the call fails before any device work
    rc = lib.dmrg2_op_heff(7, 1, 1, 2, 1, 1, 1, None, None, None, None, None, None)
    assert rc == 1
    assert b"dtype" in lib.dmrg2_last_error(None)
    rc = lib.dmrg2_op_svd(0, 0, 3, None, 1, 0.0, b"R", None, None, None, None, None)
    assert rc == 1


def test_cli_binary_built():
    cli = REPO / "dmrg-implementations_b200" / "bin" / "dmrg2_gpu"
    assert cli.exists()
    r = subprocess.run([str(cli), "8", "16", "2", "--bogus"], capture_output=True, text=True)
    assert r.returncode == 1 and "Unknown flag" in r.stderr


def _c_layout(struct, fields, tmp_path):
    """sizeof and field offsets of a header struct, from a C program compiled with gcc."""
    prog = ["#include <stddef.h>", "#include <stdio.h>", f'#include "{HEADER}"', "int main(void) {",
            f'  printf("%zu\\n", sizeof({struct}));']
    prog += [f'  printf("%zu\\n", offsetof({struct}, {f}));' for f in fields]
    prog += ["  return 0;", "}"]
    src = tmp_path / f"{struct}.c"
    exe = tmp_path / f"{struct}.out"
    src.write_text("\n".join(prog) + "\n")
    subprocess.run(["gcc", "-std=c11", "-o", str(exe), str(src)], check=True, capture_output=True)
    vals = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    return vals[0], vals[1:]


@pytest.mark.parametrize("name,struct", [("Config", "dmrg2_config"), ("SweepReport", "dmrg2_sweep_report"),
                                         ("PdmrgOptions", "dmrg2_pdmrg_options"),
                                         ("ServerConfig", "dmrg2_server_config"), ("Request", "dmrg2_request"),
                                         ("Result", "dmrg2_result")])
def test_python_structs_match_the_header_layout(name, struct, tmp_path):
    """Every ctypes mirror of a header struct has the C compiler's size and field offsets
    (a field added on one side only, or in another order, fails here without a GPU)."""
    import dmrg2
    cls = getattr(dmrg2, name)
    fields = [f[0] for f in cls._fields_]
    size, offsets = _c_layout(struct, fields, tmp_path)
    assert ctypes.sizeof(cls) == size, (name, ctypes.sizeof(cls), size)
    assert [getattr(cls, f).offset for f in fields] == offsets, name


@pytest.mark.parametrize("compiler,std", [("gcc", "-std=c99"), ("gcc", "-std=c11"), ("g++", "-std=c++17")])
def test_header_compiles_cleanly(compiler, std, tmp_path):
    """include/dmrg2_b200.h is a plain C header: it compiles as C99, C11 and C++17 with
    -Wall -Wextra -pedantic -Werror (what a cgo, JNI or C++ caller builds it with)."""
    src = tmp_path / ("h.c" if compiler == "gcc" else "h.cpp")
    src.write_text(f'#include "{HEADER}"\nint main(void) {{ return (int)(sizeof(dmrg2_config) + '
                   f'sizeof(dmrg2_sweep_report) + sizeof(dmrg2_request) + sizeof(dmrg2_result)) == 0; }}\n')
    r = subprocess.run([compiler, std, "-Wall", "-Wextra", "-pedantic", "-Werror", "-fsyntax-only", str(src)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
