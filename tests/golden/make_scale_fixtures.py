"""Run the at-scale parity cases through the CPU oracle and store the results.

TEST INFRASTRUCTURE.  Usage (from the repository root; one case per process,
so the cases can run side by side):

    OPENBLAS_NUM_THREADS=1 python tests/golden/make_scale_fixtures.py <case>
    python tests/golden/make_scale_fixtures.py --merge

Each run writes ``tests/golden/scale/<case>.json``; ``--merge`` combines them
into ``tests/golden/scale_levels.json``, which the ``-m gpu`` tests read, and
records a fingerprint of every case's initial states beside its results.
One BLAS thread per process: the site problems are small (n = chi^2 d =
8192 at chi=64), and a multi-threaded BLAS spends its time spinning.
"""
import glob
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, HERE)

import scale_cases  # noqa: E402


def main():
    out_dir = os.path.join(HERE, "scale")
    if sys.argv[1:] == ["--merge"]:
        merged = {}
        for p in sorted(glob.glob(os.path.join(out_dir, "*.json"))):
            with open(p) as f:
                d = json.load(f)
            # pins the initial states that the GPU tests replay to the ones the
            # oracle started from
            d["initial_states_fingerprint"] = scale_cases.fingerprint(scale_cases.initial_states(d["case"]))
            merged[d["case"]] = d
        with open(os.path.join(HERE, "scale_levels.json"), "w") as f:
            json.dump(merged, f, indent=1)
        return
    name = sys.argv[1]
    t0 = time.time()
    res = scale_cases.run_oracle(name)
    _, n, chi, levels, seed = scale_cases.CASES[name]
    res.update({"case": name, "sites": n, "chi": chi, "levels": levels, "seed": seed,
                "arpack_ncv": scale_cases.ARPACK_NCV, "thresholds": "reference defaults (1e-12)",
                "oracle_seconds": time.time() - t0})
    os.makedirs(out_dir, exist_ok=True)
    with open(os.path.join(out_dir, name + ".json"), "w") as f:
        json.dump(res, f, indent=1)
    print(json.dumps(res)[:400])


if __name__ == "__main__":
    main()
