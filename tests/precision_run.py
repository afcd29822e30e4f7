"""The end-to-end precision measurement of tests/test_precision.py over a longer run, as a
measurement (one JSON line, no pass/fail): the 128^3 configuration (200 Mpc/h, ng 256, int8
ZIPX, PP on, device ICs at z=49) for `--steps` KDK steps of equal code time to `--z-end`,
in the GPU's chosen and plain forms and the oracle's FP32 and FP64 arms; each arm's final
positions and velocities and its P(k) on the 512^3 grid against the FP64 arm, with the
P(k) differences for k < k_Nyq/2, k < k_Nyq/4, k < 1 and k < 0.5 h/Mpc.  The oracle arms run on all host cores
(about 13 minutes for 100 steps on 16 cores).  Needs a GPU.

    python tests/precision_run.py --steps 100 --z-end 0
"""
import argparse
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from tests import test_precision as TP  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--z-end", type=float, default=0.0)
    ap.add_argument("--save", default="", help="also write every arm's P(k) table to this .npz")
    args = ap.parse_args()
    from oracle import oracle

    oracle.build()
    runs = TP.make_runs(oracle, args.steps, args.z_end)
    p = runs["p"]
    ref = runs["oracle64"]
    nw = 2 * p.ng
    pk_ref = TP._power(p, ref, nw)
    knyq = np.pi * nw / p.box
    out = {"workload": "128^3 CDM, 200 Mpc/h, ng 256, int8 ZIPX, z=49 -> %g in %d KDK steps" % (args.z_end, args.steps),
           "pk_grid": nw, "k_nyq_hmpc": float(knyq)}
    tables = {"oracle64": pk_ref}
    for arm in ("gpu_fixed", "gpu_plain", "oracle32"):
        e = TP._pos_vel_errors(p, runs[arm], ref)
        xi = TP._power(p, runs[arm], nw)
        tables[arm] = xi
        ranges = [("k_lt_knyq_2", knyq / 2), ("k_lt_knyq_4", knyq / 4), ("k_lt_1", 1.0), ("k_lt_0.5", 0.5)]
        for key, kmax in ranges:
            sel = (pk_ref[:, 0] > 0) & (pk_ref[:, 1] > 0) & (pk_ref[:, 1] < kmax)
            rel = np.abs(xi[sel, 2] / pk_ref[sel, 2] - 1)
            e["dP_over_P_max_" + key] = float(rel.max())
            e["dP_over_P_rms_" + key] = float(np.sqrt((rel ** 2).mean()))
        out[arm + "_vs_fp64"] = e
    if args.save:
        np.savez_compressed(args.save, **tables)
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
