"""The C++ shims that INTEGRATION.md gives the reference's callers (DMRG2GPU<Scalar> and
PDMRGGPU<Scalar> over the C ABI) compile against include/dmrg2_b200.h, for double and
std::complex<double>: the code blocks are extracted from the document and every member
is instantiated (compile only; nothing runs, no GPU)."""
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
