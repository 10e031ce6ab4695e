"""Exit tests of the reference loop (spread_3d.py:3413-3437) on two variants
of the 32 x 8 x 12 case, run with the reference's own ``run_3d_spread``
through ``refharness``:

* ``extinct``: no ignition (solid-phase ignition off, ignition window 0 s),
  so no cell ever holds an active flame; the loop leaves once the flame body
  has been empty for more than 50 consecutive steps past the ignition window
  plus the 2 s bootstrap.
* ``front``: the bed ends right after the ignition strip (bed_x_end 0.75 m),
  so the level-set front (x = 0.7 m) already lies within one cell of the bed's
  end and the loop leaves in its first step.

Writes ``ref_exits.npz``: for each variant the number of outer steps the
reference started before leaving and the simulated time it had reached.

    python tests/golden/make_exits.py
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parents[1]))

CAP = 400


def main():
    from firewebapp_b200.cases import EXIT_CASES
    from refharness import run_reference
    out = {}
    for name, case in EXIT_CASES.items():
        init, snaps, trace = run_reference(case, CAP, capture_steps=[])
        n = len(trace["dt"])
        assert n < CAP, f"{name}: the reference did not leave within {CAP} steps"
        out[f"{name}/steps"] = np.int64(n)
        out[f"{name}/t"] = np.float64(np.sum(trace["dt"][:n - 1]))
        print(name, "left in step", n)
    np.savez_compressed(HERE / "ref_exits.npz", **out)


if __name__ == "__main__":
    main()
