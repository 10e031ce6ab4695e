"""Generate the committed golden fixtures under ``tests/golden/``.

Run here (the reference is importable in this container, not on the GPU box):

    python tests/golden/make_fixtures.py            # all fixtures
    python tests/golden/make_fixtures.py vectors    # only the kernel vectors

Outputs
-------
``kernel_vectors.npz``
    The reference's committed per-kernel golden vectors
    (``docs/data/kernel_vectors.json``, written by
    ``scripts/gen_kernel_vectors.py``) re-packed as arrays: key
    ``"<section>/<case>/<field>"``.  Lists become float64 arrays; ``None``
    values are dropped.
``ref_tiny.npz``
    Reference solver states for the 32 x 8 x 12 ``TINY`` case (see
    ``firewebapp_b200/cases.py``): the initial state and the full state after
    outer steps 1, 2, 9 and 10 (fields, particles, DOM intensities, warm-start
    pressure, level set), plus the per-step dt / projection / DOM-sweep trace.
    Key ``"s<step>/<name>"``; ``"init/<name>"``; ``"trace/<name>"``.
``ref_smoke.npz``
    Same for the 24 x 8 x 10 ``SMOKE`` case after steps 1 and 3 (used by the
    GPU smoke check).
``ref_cfg2_slice.npz``
    The 40 x 16 x 60 ``CFG2_SLICE`` case (the 400 x 120 x 60 workload's
    dz = 0.0625 m, four bed layers, 16 particles per surface cell, S8
    quadrature injected into the reference) after steps 1, 2 and 10, without
    the DOM intensities (80 ordinates would dominate the file).
``ref_cfg1_10.npz``
    The 64 x 24 x 20 ``CFG1`` case after steps 1 and 10, without the DOM
    intensities.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))
sys.path.insert(0, str(HERE))

REF_ROOT = Path("/root/reference")


def pack_vectors():
    src = REF_ROOT / "docs" / "data" / "kernel_vectors.json"
    d = json.loads(src.read_text())
    out = {}
    for sec, body in d.items():
        if sec.startswith("_"):
            continue
        for case in body.get("cases", []):
            name = case["name"]
            for k, v in case.items():
                if k == "name" or v is None:
                    continue
                if isinstance(v, str):
                    continue
                if isinstance(v, dict):
                    for k2, v2 in v.items():
                        if v2 is not None and not isinstance(v2, str):
                            out[f"{sec}/{name}/{k}.{k2}"] = np.asarray(v2, dtype=np.float64)
                    continue
                out[f"{sec}/{name}/{k}"] = np.asarray(v, dtype=np.float64)
        if isinstance(body.get("helpers"), dict):
            for k, v in body["helpers"].items():
                try:
                    out[f"{sec}/_helpers/{k}"] = np.asarray(v, dtype=np.float64)
                except (TypeError, ValueError):
                    pass
    np.savez_compressed(HERE / "kernel_vectors.npz", **out)
    print("kernel_vectors.npz:", len(out), "arrays")


def ref_run(case_name, n_steps, steps, out_name, intensities=True):
    from refharness import run_reference
    from firewebapp_b200.cases import CASES
    case = CASES[case_name]
    init, snaps, trace = run_reference(case, n_steps, capture_steps=steps)
    out = {}
    for k, v in init.items():
        out[f"init/{k}"] = np.asarray(v)
    for n, snap in snaps.items():
        for k, v in snap.items():
            if k == "I_set" and not intensities:
                continue
            out[f"s{n}/{k}"] = np.asarray(v)
    for k, v in trace.items():
        out[f"trace/{k}"] = np.asarray(v, dtype=np.float64)
    np.savez_compressed(HERE / out_name, **out)
    print(out_name, "steps", sorted(snaps), "trace", {k: v[:12] for k, v in trace.items()})


if __name__ == "__main__":
    what = sys.argv[1:] or ["vectors", "tiny", "smoke"]
    if "vectors" in what:
        pack_vectors()
    if "tiny" in what:
        ref_run("tiny", 10, [1, 2, 9, 10], "ref_tiny.npz")
    if "smoke" in what:
        ref_run("smoke", 3, [1, 3], "ref_smoke.npz")
    if "cfg2_slice" in what:
        ref_run("cfg2_slice", 10, [1, 2, 10], "ref_cfg2_slice.npz", intensities=False)
    if "cfg1_10" in what:
        ref_run("cfg1", 10, [1, 10], "ref_cfg1_10.npz", intensities=False)
