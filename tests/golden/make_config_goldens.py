"""Oracle goldens at the benchmark workloads' own sizes (test infrastructure).

The CPU oracle (dense FP64, OpenMP) solves, on this machine's host cores:
  - config1: the long pair (2 x 200,000-point 3D spline paths, seed 1), the plain method to
    2^-33 relative: endpoint bound, DFD, VE-FD, every probe radius and its decision, the
    final distance; and the decision at the stop threshold over VE-FD, the first probe of
    the bracketed (learned) search;
  - config2: a fixed sample of the 4096-pair uneven batch (seed 2): every 16th pair plus
    every pair with a curve of 30,000 points or more (the batch's longest, up to the 50,000
    clip), the plain method as for config1, plus the threshold decision;
  - config4: the first two of the 512 large 3D pairs (seed 5; 383,833 x 378,296 and
    157,660 x 190,084 points): endpoint bound, DFD, VE-FD and the decision at the stop
    threshold over VE-FD (a full plain search of pair 0 is about 5e12 dense cells, beyond a
    CPU run of reasonable length).
The inputs come from the seeded generator (the same source compiled into liboracle.so and
librfd.so).  Results are written to tests/golden/config_goldens.json after every case, so a
long run can be resumed (cases already present are skipped).

    python tests/golden/make_config_goldens.py [--threads N] [--only config1,config2,config4]

About 80 minutes on 8 cores (config1: about 50).
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
import oracle  # noqa: E402

OUT = os.path.join(HERE, "config_goldens.json")
REL = 2.0 ** -33


def threshold(vefd):
    """The bracketed search's first probe: the stop threshold over the VE-FD lower bound
    (lb * (1 + 0.999 tol), relative stop rule), as the engine computes it."""
    return vefd * (1.0 + 0.999 * REL)


def cfg2_sample():
    dims, n1, n2, _, _, _ = oracle.gen_batch_spec(2, 4096, 2)
    m = np.maximum(n1, n2)
    return sorted(set(range(0, 4096, 16)) | set(np.nonzero(m >= 30000)[0].tolist()))


def solve_plain(P, Q, threads):
    t0 = time.time()
    r = oracle.distance(P, Q, stop_mode=1, quirks=False, threads=threads)
    t = threshold(r["vefd"])
    reach, ub = oracle.decide(P, Q, t, threads)
    return {
        "n1": len(P), "n2": len(Q), "dims": int(P.shape[1]),
        "endpoint": r["endpoint"], "dfd": r["dfd"], "vefd": r["vefd"],
        "distance": r["distance"], "lb": r["lb"], "ub": r["ub"], "probes": r["probes"],
        "probe_eps": r["probe_eps"], "probe_dec": r["probe_dec"],
        "threshold": t, "threshold_reach": bool(reach), "threshold_right_ub": ub,
        "cpu_seconds": time.time() - t0, "threads": threads,
    }


def solve_bounds(P, Q, threads):
    t0 = time.time()
    ep = oracle.endpoint(P, Q)
    dfd = float(np.sqrt(oracle.dfd_sq(P, Q, threads)))
    vefd = float(np.sqrt(oracle.vefd_sq(P, Q, ep, threads)))
    t = threshold(vefd)
    reach, ub = oracle.decide(P, Q, t, threads)
    return {
        "n1": len(P), "n2": len(Q), "dims": int(P.shape[1]),
        "endpoint": ep, "dfd": dfd, "vefd": vefd,
        "threshold": t, "threshold_reach": bool(reach), "threshold_right_ub": ub,
        "cpu_seconds": time.time() - t0, "threads": threads,
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=oracle.max_threads())
    ap.add_argument("--only", default="config2,config1,config4")
    a = ap.parse_args()
    data = json.load(open(OUT)) if os.path.exists(OUT) else {"cases": {}}
    data["note"] = ("CPU oracle (dense FP64) results at the benchmark workloads' sizes; "
                    "made by tests/golden/make_config_goldens.py")

    def save():
        tmp = OUT + ".tmp"
        with open(tmp, "w") as f:
            json.dump(data, f, indent=0, sort_keys=True)
        os.replace(tmp, OUT)

    jobs = []
    for part in a.only.split(","):
        if part == "config1":
            jobs.append(("config1/0", 1, 0, solve_plain))
        elif part == "config2":
            jobs += [(f"config2/{k}", 2, k, solve_plain) for k in cfg2_sample()]
        elif part == "config4":
            jobs += [(f"config4/{k}", 4, k, solve_bounds) for k in (1, 0)]
    for name, cfg, k, fn in jobs:
        if name in data["cases"]:
            continue
        P, Q = oracle.gen_config_pair(cfg, k)
        rec = fn(P, Q, a.threads)
        rec.update({"config": cfg, "index": k})
        data["cases"][name] = rec
        save()
        print(f"{name}: {len(P)}x{len(Q)} {rec['cpu_seconds']:.1f} s", flush=True)


if __name__ == "__main__":
    main()
