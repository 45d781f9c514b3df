"""CPU checks of the drop-in boundary: the library loads without a GPU and
exports every function declared in include/*.h; the Python host mirror has
pyqcu's surface (python/PyQuda/pyquda/pyqcu.pyi:1-32)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:void|int|void\s*\*)\s*\*?\s*([A-Za-z_]\w*)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_headers_declare_the_reference_abi():
    names = _declared("qcu.h")
    assert names == sorted(["dslashQcu", "dslashCloverQcu", "mpiDslashQcu", "mpiBistabCgQcu", "ncclDslashQcu",
                            "ncclBistabCgQcu"])


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(os.path.join(ROOT, "qcu_b200", "libqcu.so"))
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not h.endswith(".h"):
            continue
        for name in _declared(h):
            assert hasattr(lib, name), f"{name} declared in {h} but not exported"


def test_python_mirror_has_pyqcu_surface():
    import qcu_b200 as q

    for name in ["QcuParam", "dslashQcu", "dslashCloverQcu", "mpiDslashQcu", "mpiBistabCgQcu", "ncclDslashQcu",
                 "ncclBistabCgQcu"]:
        assert hasattr(q, name)
    p = q.QcuParam()
    p.lattice_size = [8, 8, 8, 16]
    assert p.lattice_size == [8, 8, 8, 16]
    assert ctypes.sizeof(q.QcuParam) == 16
    with pytest.raises(ValueError):
        p.lattice_size = [1, 2, 3]


def test_struct_layouts_match_header(tmp_path):
    """ctypes mirrors of the C structs have the C compiler's size and offsets."""
    import shutil
    import subprocess

    import qcu_b200 as q

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    src = tmp_path / "layout.c"
    src.write_text(
        "#include <stdio.h>\n#include <stddef.h>\n#include \"qcu.h\"\n#include \"qcu_ext.h\"\n"
        "int main(void){printf(\"%zu %zu %zu %zu %zu %zu\\n\", sizeof(QcuParam), sizeof(qcuInvertParam),"
        " offsetof(qcuInvertParam, x0_seed), offsetof(qcuInvertParam, inner_tol), sizeof(qcuInvertResult),"
        " offsetof(qcuInvertResult, seconds)); return 0;}\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert got == [ctypes.sizeof(q.QcuParam), ctypes.sizeof(q.QcuInvertParam), q.QcuInvertParam.x0_seed.offset,
                   q.QcuInvertParam.inner_tol.offset, ctypes.sizeof(q.QcuInvertResult),
                   q.QcuInvertResult.seconds.offset]


def test_error_path_without_gpu():
    """Calls fail cleanly (recorded error, no exit) when no device is usable."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("needs a machine without a GPU")
    import qcu_b200 as q

    q.dslashQcu(0, 0, 0, q.QcuParam([4, 4, 4, 4]), 0)
    code, msg = q.last_error()
    assert code != 0 and msg
