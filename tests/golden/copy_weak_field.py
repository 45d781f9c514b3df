"""Copy PyQuda's own test gauge configuration, python/PyQuda/tests/weak_field.lime
of the reference tree (a 4^3 x 8 FP64 SU(3) field in ILDG/LIME format with a
SciDAC checksum), next to this script, so that the tests -- the GPU ones
included, which run where the reference tree is absent -- read a gauge file
this project did not write.  The copy is checked against the SHA-256 below.

    python tests/golden/copy_weak_field.py      (reads $QCU_REFERENCE, else ../reference)
"""
import hashlib
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
SHA256 = "de4de48d80869ed537432e237e7cdd99aae36b31f05e2e6f6b4d0b0bc3b28576"


def main():
    sys.path.insert(0, ROOT)
    from oracle import reference_root

    src = os.path.join(reference_root(), "python", "PyQuda", "tests", "weak_field.lime")
    dst = os.path.join(HERE, "weak_field.lime")
    shutil.copyfile(src, dst)
    with open(dst, "rb") as f:
        digest = hashlib.sha256(f.read()).hexdigest()
    if digest != SHA256:
        os.remove(dst)
        raise SystemExit(f"unexpected content of {src}: sha256 {digest}")
    print(dst)


if __name__ == "__main__":
    main()
