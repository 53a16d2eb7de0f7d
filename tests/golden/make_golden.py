"""Convert HORMONE's golden test dumps into compressed numpy fixtures.

Reads ``tests/<simtype>[_flat].bin`` of the reference tree (the files that
src/main/tests.f90:46-182 compares a finished test run against) with
``hormone_b200.binio.readbin`` and writes ``<simtype>[_flat].npz`` beside this
script.  Run once where the reference tree is present, giving its root as the
argument or in the environment variable HORMONE_REF:

    python tests/golden/make_golden.py /path/to/HORMONE
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from hormone_b200 import binio, config  # noqa: E402

CASES = [f"{k}_{d}" for k in ("sodshock", "briowushock") for d in "xyz"] + \
        [f"orszagtang_{p}" for p in ("xy", "yz", "xz")] + ["KHinstability", "sedov_default"]


def main(ref_root):
    for st in CASES:
        cfg = config.resolve(st + " test")
        for flat in (False, True):
            name = st + ("_flat" if flat else "")
            data = binio.readbin(os.path.join(ref_root, "tests", name + ".bin"), cfg["n"], cfg["mag_on"],
                                 cfg["gravswitch"], cfg["compswitch"])
            arrays = {k: v for k, v in data.items() if isinstance(v, np.ndarray)}
            if "spc" in arrays:  # (nz, ny, nx, spn) as stored -> (spn, nz, ny, nx)
                arrays["spc"] = np.ascontiguousarray(np.moveaxis(arrays["spc"], -1, 0))
            np.savez_compressed(os.path.join(HERE, name + ".npz"), tn=data["tn"], time=data["time"], **arrays)
            print(name, data["tn"], data["time"])


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("HORMONE_REF")
    if not root:
        sys.exit("usage: make_golden.py <HORMONE tree> (or set HORMONE_REF)")
    main(root)
