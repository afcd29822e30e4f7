"""Fixture for the expansion table (s_a_tau_H.txt rows t and a) made by the reference's own
code: the recursion of neutrinos/Pk.py:263-277 is read from the reference source and executed
here, with the analytic flat LCDM + radiation H(a) of cube_nu_b200.cosmology standing in for
CAMB's hubble_parameter (CAMB is not installed) and omHsq as Pk.py:153 defines it, for the
cosmology of the benchmark runs.  cosmology.expansion_table must reproduce t and a bit for
bit (tests/test_host.py): the fixture holds every 97th entry and the last few, and the
SHA-256 of the whole a array.  The reference's H column is set to one value after the loop
(Pk.py:279) and is not part of the fixture.

    python tests/golden/make_expansion_golden.py /path/to/reference
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from cube_nu_b200 import cosmology  # noqa: E402
from cube_nu_b200.params import Params  # noqa: E402


def main(ref: str) -> None:
    src = open(os.path.join(ref, "neutrinos", "Pk.py")).read().splitlines()
    first = next(i for i, l in enumerate(src) if l.strip().startswith("n_a = int(istep_max)"))
    last = next(i for i, l in enumerate(src) if i > first and l.strip().startswith("i_end = i"))
    omhsq_line = next(l for l in src if l.strip().startswith("omHsq ="))
    block = "\n".join([omhsq_line.strip()] + src[first:last + 1])
    p = Params()
    om, orad = p.omega_m, p.omega_r
    ol = 1.0 - om - orad
    ns = {"np": np, "istep_max": cosmology.ISTEP_MAX, "H0": 100.0 * p.h0, "omega_m": om,
          "Ha": lambda a: float(cosmology.hubble(a, p.h0, om, orad, ol))}
    exec(compile(block, "Pk.py:%d-%d" % (first + 1, last + 1), "exec"), ns)
    i_end = int(ns["i_end"])
    n = i_end + 2  # the entries the loop wrote: a_ex[0 .. i_end+1]
    a = np.ascontiguousarray(ns["a_ex"][:n], dtype=np.float64)
    idx = np.unique(np.concatenate([np.arange(0, n, 97), np.arange(max(0, n - 8), n)]))
    np.savez_compressed(os.path.join(HERE, "expansion_table_ref.npz"), n=n, i_end=i_end, idx=idx, a_sample=a[idx],
                        t_sample=ns["t"][idx], a_sha256=hashlib.sha256(a.tobytes()).hexdigest(), h0=p.h0,
                        omega_m=om, omega_r=orad)
    print("wrote expansion_table_ref.npz: %d entries (%d sampled), a_end = %.6g" % (n, idx.size, a[-1]))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
