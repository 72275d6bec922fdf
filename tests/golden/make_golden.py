"""Record the reference's own outputs on the seeded parity cases (tests/golden/cases.py).

Runs the reference's ParticleDynamics, compiled from its unmodified sources for
sm_100a by oracle/build.py into oracle/_ref/libref_world.so, on a B200:

    python tests/golden/make_golden.py [OUT_DIR [CASE ...]]  # writes OUT_DIR/<case>.npz
                                              # (default: tests/golden, every case)

Per case it stores the initial state, the state and rhs after the case's steps, the
candidate set of every grain (the reference's device_neighbors rows, sorted: the
reference fills cells with atomicAdd slots, so only the sets are defined), the
total energy and the CIC field of the initial state, the overflow count, and the
state after a second, independent run of the same step (the reference's own
run-to-run spread, used to size the parity tolerances).
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from cases import CASES, case_inputs, csr_from_sets, write_state  # noqa: E402
from oracle.oracle import ReferenceSim  # noqa: E402


def run_case(name: str, tmp: str) -> dict:
    c = CASES[name]
    state_path = os.path.join(tmp, f"{name}.bin")
    text, state = case_inputs(name, state_path)
    yaml_path = os.path.join(tmp, f"{name}.yaml")
    if text is None:
        yaml_path = os.path.join(tmp, "no_such_file.yaml")   # reference defaults
    else:
        write_state(state_path, state)
        with open(yaml_path, "w") as f:
            f.write(text)

    def one_run():
        ref = ReferenceSim(yaml_path)
        s0 = ref.state()
        e0 = ref.energy()
        d0 = ref.density()
        ref.step(c["steps"])
        out = dict(state0=s0, energy0=np.float32(e0), density0=d0, state1=ref.state(),
                   rhs=ref.rhs(), sets=ref.neighbor_sets(), overflow=np.int32(ref.overflow()))
        if c["kind"] == "cube":
            ref.step(50 - c["steps"])
            out["state50"] = ref.state()
        ref.close()
        return out

    a = one_run()
    b = one_run()
    offsets, ids = csr_from_sets(a["sets"])
    rec = dict(yaml=np.array(text or ""), state0=a["state0"], state1=a["state1"], rhs=a["rhs"],
               nbr_offsets=offsets, nbr_ids=ids, energy0=a["energy0"], density0=a["density0"],
               overflow=a["overflow"], state1_rerun=b["state1"], rhs_rerun=b["rhs"])
    if "state50" in a:
        rec["state50"] = a["state50"]
    return rec


def main() -> int:
    out_dir = sys.argv[1] if len(sys.argv) > 1 else HERE
    os.makedirs(out_dir, exist_ok=True)
    if not ReferenceSim.available():
        print("oracle/_ref/libref_world.so missing: run python oracle/build.py where the "
              "reference tree is present", file=sys.stderr)
        return 1
    names = sys.argv[2:] or list(CASES)
    with tempfile.TemporaryDirectory() as tmp:
        for name in names:
            rec = run_case(name, tmp)
            path = os.path.join(out_dir, f"{name}.npz")
            np.savez_compressed(path, **rec)
            spread = float(np.abs(rec["state1"] - rec["state1_rerun"]).max())
            print(f"{name}: n={rec['state0'].size // 6} candidates={rec['nbr_ids'].size} "
                  f"rerun spread={spread:.3e} -> {path}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
