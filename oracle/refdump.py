"""Reader for the record files that ``oracle/_ref/ref_dump`` writes.

Test infrastructure only (the checker side): each line is
``<name> <count> v0 ... v(count-1)``.
"""
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DUMP = os.path.join(HERE, "_ref", "ref_dump")


def read_records(path):
    out = {}
    with open(path) as f:
        for line in f:
            parts = line.split()
            if not parts:
                continue
            name, n = parts[0], int(parts[1])
            out[name] = np.array([float(x) for x in parts[2:2 + n]], np.float64)
    return out


def run_ref(case_dir, *args, out="out.txt", timeout=3600):
    """Runs ref_dump inside ``case_dir`` and returns its records."""
    if not os.path.exists(REF_DUMP):
        raise FileNotFoundError("oracle/_ref/ref_dump is not built (make -C oracle)")
    cmd = [REF_DUMP, *[str(a) for a in args], out]
    r = subprocess.run(cmd, cwd=case_dir, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"ref_dump failed: {r.stderr[-2000:]}")
    return read_records(os.path.join(case_dir, out))
