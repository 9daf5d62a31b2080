"""Generate golden hop vectors from the reference's own CUDA kernels.

Runs on a GPU with oracle/_ref/libqcu_ref_kernels.so (built from the reference's
sources by oracle/ref_build.sh).  For each case it builds seeded fields with
qcu_mrhs_b200.fields, runs the reference's wmma hop (the one its solver uses) and its
SIMT hop (the one start_dslash/mat_Qcu use) in FP64, and writes one .npz per case:

  L, nc, m, seeds, gauge, psi (gathered [Vh][4][N][m]), and for every (parity, dagger)
  run: out_wmma_p{p}_d{d}, out_simt_p{p}_d{d}
  (the 8^4 configuration-1 case stores 64 seeded random projections of each output
  instead of the full vectors, plus the full inputs' checksums).

  python tests/golden/make_golden.py OUTDIR
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from qcu_mrhs_b200 import fields as F  # noqa: E402

CASES = [
    # name, L, nc, m, gauge kind, runs [(parity, dagger)], full vectors
    ("l4444_n3_m4", (4, 4, 4, 4), 3, 4, "haar", [(0, 0), (1, 0), (0, 1), (1, 1)], True),
    ("l6424_n3_m12", (6, 4, 2, 4), 3, 12, "haar", [(0, 0), (1, 1)], True),
    ("l4244_n4_m8", (4, 2, 4, 4), 4, 8, "haar", [(1, 0)], True),
    ("l2242_n5_m5", (2, 2, 4, 2), 5, 5, "haar", [(0, 0), (1, 1)], True),
    ("l2222_n2_m3", (2, 2, 2, 2), 2, 3, "haar", [(0, 1)], True),
    ("l8888_n3_m4", (8, 8, 8, 8), 3, 4, "haar", [(0, 0), (1, 0)], False),
]
SEED_GAUGE, SEED_PSI, SEED_PROJ = 1000, 2000, 3000
NPROJ = 64


def projections(vec: np.ndarray, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    flat = vec.reshape(-1)
    r = rng.standard_normal((NPROJ, flat.size)) + 1j * rng.standard_normal((NPROJ, flat.size))
    return r @ flat


def main(outdir: str) -> None:
    import torch
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libqcu_ref_kernels.so"))
    for fn in (lib.ref_wmma_hop_f64, lib.ref_simt_hop_f64):
        fn.restype = ctypes.c_int
        fn.argtypes = [ctypes.c_void_p] * 3 + [ctypes.POINTER(ctypes.c_int)] + [ctypes.c_int] * 4
    os.makedirs(outdir, exist_ok=True)
    for ci, (name, L, nc, m, kind, runs, full) in enumerate(CASES):
        gauge = F.gauge_field(L, nc, SEED_GAUGE + ci, kind=kind)
        psi = F.to_mrhs(F.gaussian_fermions(L, nc, m, SEED_PSI + ci, parities=1)[:, 0])
        dg = torch.from_numpy(np.ascontiguousarray(gauge).view(np.float64).copy()).cuda()
        dp = torch.from_numpy(np.ascontiguousarray(psi).view(np.float64).copy()).cuda()
        Lc = (ctypes.c_int * 4)(*L)
        rec = {"L": np.array(L), "nc": nc, "m": m, "seed_gauge": SEED_GAUGE + ci, "seed_psi": SEED_PSI + ci,
               "gauge_kind": kind}
        if full:
            rec["gauge"] = gauge
            rec["psi"] = psi
        else:
            rec["gauge_sum"] = np.array([gauge.sum(), (np.abs(gauge) ** 2).sum()])
            rec["psi_sum"] = np.array([psi.sum(), (np.abs(psi) ** 2).sum()])
        for parity, dagger in runs:
            for kname, fn in (("wmma", lib.ref_wmma_hop_f64), ("simt", lib.ref_simt_hop_f64)):
                out = torch.full_like(dp, float("nan"))
                rc = fn(out.data_ptr(), dp.data_ptr(), dg.data_ptr(), Lc, nc, m, parity, dagger)
                if rc != 0:
                    raise RuntimeError(f"{name} {kname}: CUDA error {rc}")
                o = out.cpu().numpy().view(np.complex128).reshape(psi.shape)
                key = f"out_{kname}_p{parity}_d{dagger}"
                rec[key] = o if full else projections(o, SEED_PROJ + ci)
        np.savez_compressed(os.path.join(outdir, f"hop_{name}.npz"), **rec)
        print("wrote", name, flush=True)


if __name__ == "__main__":
    # default: next to this script (the committed fixtures); pass another directory to
    # write a fresh set elsewhere for comparison
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__)))
