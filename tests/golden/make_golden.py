"""Regenerate tests/golden/oracle_small.json from the FP64 oracle.

The reference ships no golden vectors for its timestep path, so these
fixtures are the oracle's own outputs on small seeded cases: they pin the
oracle against later edits (tests/test_oracle.py) and give the device path a
fixed target that needs no oracle run (tests/test_gpu_parity.py).

    python tests/golden/make_golden.py
"""
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
import pipeflow_oracle as O  # noqa: E402

CASES = [
    dict(cfg=dict(N=16, K=4, M=4, Mp=1, Re=2000.0, alpha=1.25, dt=0.01), seed=1, energy=1e-3, steps=3),
    dict(cfg=dict(N=24, K=6, M=5, Mp=2, Re=3000.0, alpha=0.8, dt=0.005), seed=2, energy=1e-2, steps=2),
    dict(cfg=dict(N=20, K=5, M=6, Mp=1, Re=1800.0, alpha=1.6, dt=0.01, const_flux=False), seed=3, energy=1e-3,
         steps=2),
]


def run_case(case):
    p = O.Pipe(O.PipeConfig(**case["cfg"]))
    p.vel_matrices()
    p.set_state(*O.seeded_state(p, case["seed"], case["energy"]))
    ncorr = [p.timestep() for _ in range(case["steps"])]
    ur, ut, uz = p.state()
    out = dict(case)
    out["ncorr"] = ncorr
    out["energy_after"] = p.energy()
    out["checksums"] = {n: [float(np.sum(f.re)), float(np.sum(f.im))] for n, f in (("ur", ur), ("ut", ut), ("uz", uz))}
    # the k=0, m=0 axial profile and the (k=1, m=1) mode, full precision
    nh11 = 1 * (2 * p.cfg.K - 1) + (p.cfg.K - 1) + 1
    out["uz_mean_profile"] = [float(x) for x in uz.re[:, 0]]
    out["ur_mode11"] = [[float(a), float(b)] for a, b in zip(ur.re[:, nh11], ur.im[:, nh11])]
    return out


def main():
    gold = {"generator": "tests/golden/make_golden.py (FP64 oracle)", "cases": [run_case(c) for c in CASES]}
    path = Path(__file__).with_name("oracle_small.json")
    path.write_text(json.dumps(gold, indent=1))
    print(f"wrote {path}")


if __name__ == "__main__":
    main()
