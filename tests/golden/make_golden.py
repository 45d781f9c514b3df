"""Generate the golden vectors under tests/golden/ by running qcu itself.

qcu's library is compiled from its own sources into oracle/_ref/libqcu_ref.so
(`make -C oracle ref`, a one-rank stub replaces MPI) and called through its C
ABI exactly as PyQuda's pyqcu would (src/draft.cu:3-28,
src/nccl_wilson_dslash.cu:3-19, src/nccl_clover_dslash.cu:3-79,
src/nccl_wilson_bistabcg.cu:7-27).  The inputs are this project's seeded
fields (oracle generators) and are stored next to the outputs, so the tests
need neither the reference nor a GPU to use the fixtures.

Needs a GPU:   python tests/golden/make_golden.py [outdir]
"""
import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402


class QcuParam(ctypes.Structure):
    _fields_ = [("lattice_size", ctypes.c_int * 4)]


def param(v):
    p = QcuParam()
    for i in range(4):
        p.lattice_size[i] = v[i]
    return p


def main(outdir):
    import torch

    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libqcu_ref.so"))
    vp = ctypes.c_void_p
    P = ctypes.POINTER(QcuParam)
    lib.dslashQcu.argtypes = [vp, vp, vp, P, ctypes.c_int]
    lib.dslashCloverQcu.argtypes = [vp, vp, vp, P, ctypes.c_int]
    lib.ncclDslashQcu.argtypes = [vp, vp, vp, P, ctypes.c_int, P]
    lib.ncclBistabCgQcu.argtypes = [vp, vp, vp, P, P]

    def d(a):
        return torch.from_numpy(np.ascontiguousarray(a)).cuda()

    out = {}
    grid = param([1, 1, 1, 1])
    # Wilson hopping term, hot (Haar) links
    for tag, latt, seed in (("w4", [4, 4, 4, 4], 1), ("w8", [8, 4, 4, 8], 2)):
        U = O.gauge_haar(latt, seed)
        psi = O.fermion_gauss(O.full_shape(latt), 100 + seed)
        out[f"{tag}_latt"] = np.array(latt)
        out[f"{tag}_U"] = U
        out[f"{tag}_psi"] = psi
        for p in (0, 1):
            for api in ("dslashQcu", "ncclDslashQcu"):
                dU, din = d(U), d(psi[1 - p])
                dout = torch.zeros(O.half_shape(latt), dtype=torch.complex128, device="cuda")
                if api == "dslashQcu":
                    lib.dslashQcu(dout.data_ptr(), din.data_ptr(), dU.data_ptr(), ctypes.byref(param(latt)), p)
                else:
                    lib.ncclDslashQcu(dout.data_ptr(), din.data_ptr(), dU.data_ptr(), ctypes.byref(param(latt)), p,
                                      ctypes.byref(grid))
                torch.cuda.synchronize()
                out[f"{tag}_{api}_p{p}"] = dout.cpu().numpy()
    # clover (qcu's unit normalisation), smooth and hot links
    for tag, latt, kind, seed in (("c4s", [4, 4, 4, 4], "smooth", 3), ("c4h", [4, 4, 4, 4], "haar", 4)):
        U = O.gauge_smooth(latt, 0.3, seed) if kind == "smooth" else O.gauge_haar(latt, seed)
        psi = O.fermion_gauss(O.full_shape(latt), 100 + seed)
        out[f"{tag}_latt"] = np.array(latt)
        out[f"{tag}_U"] = U
        out[f"{tag}_psi"] = psi
        for p in (0, 1):
            dU, din = d(U), d(psi[1 - p])
            dout = torch.zeros(O.half_shape(latt), dtype=torch.complex128, device="cuda")
            lib.dslashCloverQcu(dout.data_ptr(), din.data_ptr(), dU.data_ptr(), ctypes.byref(param(latt)), p)
            torch.cuda.synchronize()
            out[f"{tag}_dslashCloverQcu_p{p}"] = dout.cpu().numpy()
    # solver: b = 1 (test/test.nccl.bistabcg.qcu-np1.py:30), kappa 0.125 fixed inside qcu
    latt = [4, 4, 4, 8]
    U = O.gauge_haar(latt, 6)
    b = np.ones(O.full_shape(latt), complex)
    dx = torch.zeros(O.full_shape(latt), dtype=torch.complex128, device="cuda")
    db, dU = d(b), d(U)  # keep the tensors alive across the call
    lib.ncclBistabCgQcu(dx.data_ptr(), db.data_ptr(), dU.data_ptr(), ctypes.byref(param(latt)),
                        ctypes.byref(grid))
    torch.cuda.synchronize()
    out["s_latt"] = np.array(latt)
    out["s_U"] = U
    out["s_b"] = b
    out["s_x"] = dx.cpu().numpy()
    os.makedirs(outdir, exist_ok=True)
    path = os.path.join(outdir, "qcu_ref_golden.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, sum(v.nbytes for v in out.values()), "bytes")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__)))
