"""Regenerate tests/golden/golden.json from the reference's own sources.

Runs the reference build (oracle/_ref, compiled from the reference tree by
`make -C oracle ref`) on the library's synthetic scenes and records final-state
FNV-1a hashes and pair / contact counts. The GPU and CPU tests compare against
this file, so they need nothing from the reference tree at run time.

    python tests/golden/make_golden.py
"""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from dyphur_b200 import scenes  # noqa: E402
from oracle import oracle  # noqa: E402

CASES = [
    # name, scene builder, frames, solver mode
    ("determinism_8_f20", lambda: scenes.determinism(), 20, oracle.SOLVER_REFERENCE),
    ("blocks_1025_f60_reference", lambda: scenes.stress_blocks(), 60, oracle.SOLVER_REFERENCE),
    ("blocks_1025_f300_reference", lambda: scenes.stress_blocks(), 300, oracle.SOLVER_REFERENCE),
    ("blocks_1025_f300_serial", lambda: scenes.stress_blocks(), 300, oracle.SOLVER_SERIAL),
    ("pile_4096_f120_reference", lambda: scenes.random_pile(4096, seed=7), 120, oracle.SOLVER_REFERENCE),
]


def main() -> None:
    if not oracle.ref_available():
        raise SystemExit("the reference build is missing: run `make -C oracle ref` first")
    out = {"generator": "tests/golden/make_golden.py", "source": "reference sources on the host SYCL shim",
           "cases": {}}
    for name, make, frames, mode in CASES:
        s = make()
        w = oracle.World(s, which="ref")
        assert w.step(frames, mode) == 0
        pairs, n_pairs = w.pairs()
        ab, _ = w.contacts()
        out["cases"][name] = {"frames": frames, "mode": mode, "n_bodies": int(s.n_bodies),
                              "hash": f"{w.hash():#018x}", "pairs": int(n_pairs), "contacts": int(len(ab))}
        print(name, out["cases"][name])
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
