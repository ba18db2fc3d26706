"""Regenerate ``cgemm3m_cases.json`` from the reference's case table.

Reads ops-blas/test/gemm/cgemm3m/arch35/cgemm3m_test.csv under the reference
checkout, given as the first argument or in CG3M_REFERENCE and keeps, per
row, the fields that pin behaviour: shapes, ops, scalars (``null`` kept as
None), fill kinds, leading dimensions, expected status and seed.  The legacy
``mere_threshold`` / ``mare_multiplier`` columns are dropped (the reference's
own test README says they are unused).  Matrix values are not part of the
table -- the reference generates them with an unshipped RNG -- so tests
regenerate their own seeded values from the same seeds.

Run from the repository root:  python tests/golden/make_cases.py <reference checkout>
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
    return os.path.join(ref, "ops-blas/test/gemm/cgemm3m/arch35/cgemm3m_test.csv")


OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cgemm3m_cases.json")

OPS = {"ACLBLAS_OP_N": "N", "ACLBLAS_OP_T": "T", "ACLBLAS_OP_C": "C", "999": 999}
STATUS = {
    "ACLBLAS_STATUS_SUCCESS": "SUCCESS",
    "ACLBLAS_STATUS_INVALID_VALUE": "INVALID_VALUE",
    "ACLBLAS_STATUS_HANDLE_IS_NULLPTR": "HANDLE_IS_NULLPTR",
}


def scalar(value):
    return None if value == "null" else float(value)


def main():
    with open(_source(), "rb") as f:
        raw = f.read()
    rows = list(csv.DictReader(raw.decode().splitlines()))
    cases = []
    for r in rows:
        cases.append({
            "name": r["case_name"],
            "desc": r["description"],
            "transa": OPS[r["transa"]],
            "transb": OPS[r["transb"]],
            "m": int(r["m"]), "n": int(r["n"]), "k": int(r["k"]),
            "alpha": [scalar(r["alpha_real"]), scalar(r["alpha_imag"])],
            "beta": [scalar(r["beta_real"]), scalar(r["beta_imag"])],
            "a_fill": r["a_fill"], "lda": int(r["lda"]),
            "b_fill": r["b_fill"], "ldb": int(r["ldb"]),
            "c_fill": r["c_fill"], "ldc": int(r["ldc"]),
            "expect": STATUS[r["expect_result"]],
            "seed": int(r["random_seed"]),
        })
    doc = {
        "source": "ops-blas/test/gemm/cgemm3m/arch35/cgemm3m_test.csv",
        "source_sha256": hashlib.sha256(raw).hexdigest(),
        "count": len(cases),
        "cases": cases,
    }
    with open(OUT, "w") as f:
        json.dump(doc, f, separators=(",", ":"))
        f.write("\n")
    print(f"wrote {len(cases)} cases to {OUT}")


if __name__ == "__main__":
    main()
