"""Regenerate ``pf_gpu_baseline.json`` from the reference's performance table.

Reads ops-blas/test/gemm/cgemm3m/arch35/gpu_baseline.csv under the reference
checkout, given as the first argument or in CG3M_REFERENCE: the 200
performance shapes of the reference's case table (alpha = 1, beta = 0, fills
RANDOM_NORM_5_5) with the per-call time of the reference's GPU baseline, which
its own performance gate divides by the NPU time.  Kept per row: id, ops,
m, n, k, leading dimensions and gpu_ms; the sha256 of the source is recorded.

Run from the repository root:  python tests/golden/make_pf_baseline.py <reference checkout>
"""
import csv
import hashlib
import json
import os
import sys

def _source():
    """The reference's table: argv[1] or CG3M_REFERENCE names the checkout."""
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CG3M_REFERENCE")
    if not ref:
        sys.exit("usage: python %s <reference checkout>  (or set CG3M_REFERENCE)" % sys.argv[0])
    return os.path.join(ref, "ops-blas/test/gemm/cgemm3m/arch35/gpu_baseline.csv")


OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "pf_gpu_baseline.json")
OPS = {"ACLBLAS_OP_N": "N", "ACLBLAS_OP_T": "T", "ACLBLAS_OP_C": "C"}


def main():
    with open(_source(), "rb") as f:
        raw = f.read()
    rows = []
    for r in csv.DictReader(raw.decode().splitlines()):
        rows.append({"id": r["id"], "transa": OPS[r["transa"]], "transb": OPS[r["transb"]], "m": int(r["m"]),
                     "n": int(r["n"]), "k": int(r["k"]), "lda": int(r["lda"]), "ldb": int(r["ldb"]),
                     "ldc": int(r["ldc"]), "gpu_ms": float(r["gpu_ms"])})
    doc = {"source": "ops-blas/test/gemm/cgemm3m/arch35/gpu_baseline.csv",
           "source_sha256": hashlib.sha256(raw).hexdigest(), "count": len(rows), "cases": rows}
    with open(OUT, "w") as f:
        json.dump(doc, f, indent=0)
        f.write("\n")
    print(f"{len(rows)} rows -> {OUT}")


if __name__ == "__main__":
    main()
