"""Writes the golden fixtures of the parity suite: oracle (CPU FP64
restatement) outputs of the small seeded SH and P-SV cases.

    python tests/golden/make_golden.py

The fixtures pin the oracle against regressions and give the GPU tests a
reference that needs no oracle run.  They are not reference-Fortran output
(no Fortran compiler is available), so parity with the reference itself
stays unpinned."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "dsm-kernel_b200"))
sys.path.insert(0, os.path.join(REPO, "tests"))
sys.path.insert(0, REPO)

CASES = {
    "sh_small_seed0": ("sh", "sh_small", {}, [1, 7, 16, 31]),
    "psv_small_seed0": ("psv", "psv_small", {}, [1, 17, 50]),
    "psv_deep_seed1": ("psv", "psv_small", {"seed": 1, "r0": 5771.0}, [3, 40]),
}


def compute(name):
    """The oracle on its own set-up of the case's job."""
    import cases
    from oracle import driver_setup, oracle as orc
    mode, fn, kw, freqs = CASES[name]
    s = driver_setup.setup(getattr(cases, fn)(**kw), mode)
    t, r, y, llog = orc.run(s, freqs, threads=os.cpu_count() or 1)
    return s, freqs, t, r, y, llog


def main():
    for name in CASES:
        _, freqs, t, r, y, llog = compute(name)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), freqs=np.asarray(freqs, np.int32),
                            tsgt=t, rsgt=r, synn=y, llog=llog)
        print(name, t.shape, r.shape, y.shape, list(llog))


if __name__ == "__main__":
    main()
