"""Golden values of the reference's flop counter (jaxqft/fermions/wilson.py:349-437).

Imports the reference's own ``WilsonDiracOperator`` (under the numpy JAX shim,
see ``reference_loader.py``) and records its counts over a grid of arguments in
``golden_flops.json`` beside this script.  Usage:
    python tests/golden/make_golden_flops.py --ref /path/to/jaxQFT
"""

from __future__ import annotations

import argparse
import itertools
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="root of the jaxQFT source tree")
    args = ap.parse_args()
    from reference_loader import load_reference

    R = load_reference(args.ref)
    import numpy as np

    gam = R.gamma.build_euclidean_gamma(4, dtype=np.complex128)
    op = R.wilson.WilsonDiracOperator(ndim=4, mass=0.1, wilson_r=1.0, gamma=gam, dtype=np.complex128)
    rows = []
    for nc, sparse, diag in itertools.product((1, 2, 3, 4), (True, False), (True, False)):
        rows.append({"nc": nc, "sparse": sparse, "diag": diag,
                     "dslash": int(op.flops_per_site_dslash(nc=nc, use_sparse_gamma=sparse)),
                     "matvec": int(op.flops_per_site_matvec(nc=nc, use_sparse_gamma=sparse, include_diagonal=diag)),
                     "call_V4096_B2": int(op.flops_per_matvec_call(nc=nc, volume=4096, batch=2,
                                                                   use_sparse_gamma=sparse, include_diagonal=diag))})
    with open(os.path.join(HERE, "golden_flops.json"), "w") as f:
        json.dump(rows, f, indent=1)
    print(f"wrote {len(rows)} rows")


if __name__ == "__main__":
    main()
