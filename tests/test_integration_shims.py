"""The C++ shims that the integration guide gives the reference's callers (DMRG2GPU<Scalar>
and PDMRGGPU<Scalar> over the C ABI) compile against include/dmrg2_b200.h, for double and
std::complex<double>: the code blocks are extracted from the guide and every member is
instantiated (compile only; nothing runs, no GPU)."""
import re
import shutil
import subprocess
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parent.parent


def shim_blocks():
    text = (REPO / "INTEGRATION.md").read_text()
    blocks = re.findall(r"```cpp\n(.*?)```", text, flags=re.S)
    return [b for b in blocks if "class DMRG2GPU" in b or "class PDMRGGPU" in b]


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_integration_shims_compile(tmp_path):
    blocks = shim_blocks()
    assert len(blocks) == 2, "expected the DMRG2GPU and PDMRGGPU shims"
    src = tmp_path / "shims.cpp"
    src.write_text("\n".join(blocks) + """
template class DMRG2GPU<double>;
template class DMRG2GPU<std::complex<double>>;
template class PDMRGGPU<double>;
template class PDMRGGPU<std::complex<double>>;
""")
    r = subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-fsyntax-only", f"-I{REPO / 'include'}", str(src)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_integration_python_snippets_name_real_entry_points():
    """The guide's Python snippets use names and signatures the package and the header
    have: the op-level drop-ins, dmrg2_op_heff's 7 ints and 6 pointers, and the Server's
    submit / result."""
    import inspect

    import dmrg2
    text = (REPO / "INTEGRATION.md").read_text()
    snippets = "\n".join(re.findall(r"```python\n(.*?)```", text, flags=re.S))
    imported = re.search(r"from dmrg2 import ([\w, ]+)", snippets).group(1)
    for name in (n.strip() for n in imported.split(",")):
        assert hasattr(dmrg2, name), name
    header = (REPO / "include" / "dmrg2_b200.h").read_text()
    params = re.search(r"int dmrg2_op_heff\((.*?)\);", header, flags=re.S).group(1).split(",")
    kinds = ["int" if p.split()[0] == "int" else "ptr" for p in params]
    assert kinds == ["int"] * 7 + ["ptr"] * 6
    assert "[ctypes.c_int] * 7 + [ctypes.c_void_p] * 6" in snippets
    assert "max_active" in inspect.signature(dmrg2.Server.__init__).parameters
    sub = inspect.signature(dmrg2.Server.submit).parameters
    assert list(sub)[1:3] == ["mpo", "schedule"] and "mps" in sub
    assert hasattr(dmrg2.Server, "result")
