"""Generate the golden vectors in tests/golden/ from the reference's own CPU code.

Runs the reference (nishadtardalkar/vectorcache) flat path, compiled in place
into oracle/_ref/libtqref.so by oracle/Makefile, on small seeded inputs and
stores its outputs: codebooks, rotation tables, TQ+ calibration, bit-plane
codes, codes_flat, alpha, prepared-query state (q_rot, bias_corr, LUT bytes,
scale, bias) and top-k scores/ids of search_flat under the AVX2 PERM0 backend.

    make -C oracle ref && python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.oracle import Reference, ReferenceIndex  # noqa: E402
from vectorcache_b200.synthetic import gaussian_mixture, power_law  # noqa: E402

OUT = Path(__file__).resolve().parent

# (name, generator, dim, n_db, n_q, bits, tqplus, k)
CASES = [
    ("mix128_b4", "mix", 128, 520, 9, 4, False, 10),
    ("mix128_b2_tq", "mix", 128, 520, 9, 2, True, 10),
    ("pl256_b3_tq", "pl", 256, 300, 7, 3, True, 64),
    ("pl1536_b4_tq", "pl", 1536, 96, 4, 4, True, 10),
    ("pl768_b2", "pl", 768, 160, 5, 2, False, 17),
    ("mix104_b4_tq", "mix", 104, 333, 5, 4, True, 10),
]

CODEBOOK_DIMS = [8, 16, 104, 128, 200, 256, 384, 768, 1024, 1536, 2048, 4096, 16384]


def make_case(ref, name, gen, dim, n_db, n_q, bits, tq, k, seed):
    if gen == "mix":
        db, q = gaussian_mixture(n_db, n_q, dim, seed=seed)
    else:
        db = power_law(n_db, dim, seed=seed)
        q = power_law(n_q, dim, seed=seed + 100)
    n_calib = min(len(db), 256) if tq else 0
    calib = db[:n_calib] if tq else None
    shift = scale = None
    if tq:
        shift, scale = ref.fit_calibration(calib, bits)
    packed, alpha = ref.encode(db, bits, shift, scale)
    flat = ref.codes_flat(packed, bits, dim)
    prep = ref.prepare_queries(q, bits, shift, scale)
    idx = ReferenceIndex(ref, db, bits, calib_rows=calib)
    top_s, top_i = idx.search(q, k)
    idx.close()
    arrays = dict(db=db, q=q, packed=packed, codes_flat=flat, alpha=alpha, top_scores=top_s,
                  top_ids=top_i, meta=np.array([dim, bits, int(tq), k, n_calib], np.int64), **prep)
    if tq:
        arrays.update(shift=shift, scale=scale)
    np.savez_compressed(OUT / f"{name}.npz", **arrays)


def main():
    ref = Reference()
    for j, (name, gen, dim, n_db, n_q, bits, tq, k) in enumerate(CASES):
        make_case(ref, name, gen, dim, n_db, n_q, bits, tq, k, seed=100 + j)
    cb = {}
    for bits in (2, 3, 4):
        for dim in CODEBOOK_DIMS:
            b, c = ref.codebook(bits, dim)
            cb[f"b{bits}_d{dim}_boundaries"] = b
            cb[f"b{bits}_d{dim}_centroids"] = c
    rot = {}
    for dim in (8, 104, 128, 1536):
        s, p = ref.rotation(dim)
        rot[f"d{dim}_signs"] = s
        rot[f"d{dim}_perm"] = p
    beta = np.array([[a, t, ref.beta_cdf_aa(a, t)] for a in (3.5, 51.5, 63.5, 767.5, 8191.5)
                     for t in np.linspace(0.01, 0.99, 13)], np.float64)
    np.savez_compressed(OUT / "tables.npz", beta_cdf=beta, **cb, **rot)
    print("wrote", sorted(p.name for p in OUT.glob("*.npz")))


if __name__ == "__main__":
    main()
