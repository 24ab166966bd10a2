"""Generates the committed golden fixtures under tests/golden/.

Run where a checkout of the reference (eozd/bnmf-algs) is available, giving
its root directory:

    python tests/golden/make_golden.py --reference <path to the reference checkout>

Fixtures:
  kat_8x10.json   the 8x10 count matrix of the reference's known-answer test
                  (test/bld/bld_mult/test_bld_mult.cpp:50-55, parsed from the
                  file's text), its parameters and thresholds (:58-84), and the
                  oracle's S after 2000 iterations from the seeded initial S
                  (seed 0) in both digamma modes.
  psi_points.json digamma at fixed points, evaluated with mpmath at 40 digits.
  plain_small.npz the 64x48x8 workload (X, seeded S0) and the oracle's S after
                  200 psi_appr iterations.
"""

import argparse
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def load_pkg():
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "bnmf_algs_b200_workloads", os.path.join(ROOT, "bnmf-algs_b200", "workloads.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def parse_kat_matrix(reference):
    path = os.path.join(reference, "test", "bld", "bld_mult", "test_bld_mult.cpp")
    text = open(path).read()
    m = re.search(r"matrixd X\(x, y\);\s*X <<(.*?);", text, re.S)
    vals = [float(v) for v in re.findall(r"[-+]?\d+\.?\d*", m.group(1))]
    sizes = re.search(r"size_t x = (\d+), y = (\d+), z = (\d+);\s*shape<3> tensor_shape\{x, y, z\};\s*"
                      r"SECTION\(\"Zero matrix", text, re.S)
    x, y, z = (int(sizes.group(i)) for i in (1, 2, 3))
    assert len(vals) == x * y, (len(vals), x, y)
    return np.array(vals).reshape(x, y), z


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True,
                    help="root directory of a checkout of the reference (eozd/bnmf-algs)")
    args = ap.parse_args()
    import oracle as O
    import mpmath

    X, z = parse_kat_matrix(args.reference)
    x, y = X.shape
    alpha, beta = np.ones(x), np.ones(z)
    kat = {"source": "test/bld/bld_mult/test_bld_mult.cpp:33-86",
           "X": X.tolist(), "z": z, "a": 40.0, "b": 1.0, "iters": 2000,
           "log_marginal_min": -262.0, "sparseness_min": 0.64,
           "rowsum_isapprox_exact": 1e-10, "rowsum_isapprox_appr": 1e-4,
           "init_seed": 0}
    S0 = O.init_S(X, z, 0)
    for name, mode in (("exact", O.PSI_EXACT), ("appr", O.PSI_APPR)):
        S = O.bld_mult(X, z, alpha, beta, 2000, mode, 1e-50, S0=S0)
        kat[f"S_{name}"] = S.reshape(-1).tolist()
        kat[f"log_marginal_{name}"] = O.log_marginal_S(S, alpha, beta, 40.0, 1.0)
        kat[f"sparseness_{name}"] = O.sparseness(S)
    with open(os.path.join(HERE, "kat_8x10.json"), "w") as f:
        json.dump(kat, f)

    mpmath.mp.dps = 40
    pts = sorted(set([1e-8, 1e-5, 1e-3, 0.1, 0.25, 0.5, 0.75, 0.999, 1.0, 1.4616321449683622,
                      1.5, 2.0, 2.5, 3.0, 4.5, 5.0, 5.999, 6.0, 6.5, 9.5, 10.0, 17.25, 33.0,
                      100.0, 1234.5, 1e5, 3.7e7, 1e12]))
    psi = {"points": pts, "digamma": [float(mpmath.digamma(mpmath.mpf(p))) for p in pts],
           "psi_appr_oracle": [O.psi_appr(p) for p in pts]}
    with open(os.path.join(HERE, "psi_points.json"), "w") as f:
        json.dump(psi, f, indent=1)

    W = load_pkg()
    prob = W.plain_small(0)
    S0 = O.init_S(prob["X"], prob["z"], 0)
    S = O.bld_mult(prob["X"], prob["z"], prob["alpha"], prob["beta"], prob["iters"], O.PSI_APPR,
                   1e-50, S0=S0)
    np.savez_compressed(os.path.join(HERE, "plain_small.npz"), X=prob["X"], S0=S0, S=S,
                        alpha=prob["alpha"], beta=prob["beta"], iters=prob["iters"])
    print("wrote kat_8x10.json psi_points.json plain_small.npz")


if __name__ == "__main__":
    main()
