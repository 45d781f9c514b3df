"""Builds qcu's own Python binding -- PyQuda's `pyquda.pointer` and
`pyquda.pyqcu` Cython modules (python/PyQuda/pyquda/src/pointer.pyx,
python/PyQuda/pyquda/src/pyqcu.pyx, python/PyQuda/setup.py:28-58) -- from the
reference tree, unchanged, against THIS repository's include/qcu.h and
qcu_b200/libqcu.so.  TEST INFRASTRUCTURE ONLY: it shows that the binding
PyQuda ships for qcu drops in on this library; tests/test_gpu_pyqcu.py calls
the hot path through it.

Reads the reference tree (read-only), writes only under oracle/_ref/:
    oracle/_ref/pyquda/{__init__.py, pointer*.so, pyqcu*.so}
The pyqcu module links libqcu.so with an rpath to qcu_b200/ of this checkout.

    python oracle/pyqcu_build.py [--ref <qcu source tree>]   (default: $QCU_REFERENCE, else ../reference)
"""
import argparse
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
OUT = os.path.join(HERE, "_ref")


def build(ref: str) -> str:
    import numpy
    from Cython.Build import cythonize
    from setuptools import Extension
    from setuptools.dist import Distribution

    pyq = os.path.join(ref, "python", "PyQuda")
    src = os.path.join(pyq, "pyquda", "src")
    if not os.path.exists(os.path.join(src, "pyqcu.pyx")):
        raise FileNotFoundError(f"PyQuda sources not found under {pyq}")
    lib_dir = os.path.join(REPO, "qcu_b200")
    if not os.path.exists(os.path.join(lib_dir, "libqcu.so")):
        raise FileNotFoundError("qcu_b200/libqcu.so is not built (make -C qcu_b200)")
    tmp = os.path.join(OUT, "pyqcu_build")
    pkg = os.path.join(OUT, "pyquda")
    os.makedirs(pkg, exist_ok=True)
    with open(os.path.join(pkg, "__init__.py"), "w") as f:
        f.write("# PyQuda's qcu binding, built from the reference sources against libqcu.so of this repository\n")
    exts = [
        Extension("pyquda.pointer", [os.path.join(src, "pointer.pyx")], include_dirs=[numpy.get_include()],
                  define_macros=[("NPY_NO_DEPRECATED_API", "NPY_1_7_API_VERSION")], language="c"),
        Extension("pyquda.pyqcu", [os.path.join(src, "pyqcu.pyx")],
                  include_dirs=[os.path.join(REPO, "include"), numpy.get_include()],
                  define_macros=[("NPY_NO_DEPRECATED_API", "NPY_1_7_API_VERSION")],
                  library_dirs=[lib_dir], libraries=["qcu"], runtime_library_dirs=[lib_dir], language="c"),
    ]
    exts = cythonize(exts, build_dir=os.path.join(tmp, "c"), include_path=[pyq, src], language_level="3",
                     quiet=True)
    dist = Distribution({"name": "pyquda_qcu_binding", "ext_modules": exts})
    cmd = dist.get_command_obj("build_ext")
    cmd.build_lib = OUT
    cmd.build_temp = os.path.join(tmp, "obj")
    cmd.ensure_finalized()
    cmd.run()
    shutil.rmtree(tmp, ignore_errors=True)
    return pkg


def main():
    ap = argparse.ArgumentParser()
    sys.path.insert(0, REPO)
    from oracle import reference_root

    ap.add_argument("--ref", default=reference_root())
    a = ap.parse_args()
    print(build(a.ref))


if __name__ == "__main__":
    sys.exit(main())
