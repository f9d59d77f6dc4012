"""Generates tests/golden/config1_ladder16_m256.json (run from the repository root).

    python tests/golden/make_config1.py

The oracle's run of the plain method on the 2x16 t-J ladder (open ends,
t = 1, J = 1/3, t' = 0, 28 electrons = 4 holes, total S = 0): the reference's
schedule Get_Ground_State (main.f90:96-187) -- warm-up, the two start
half-sweeps, 10 full sweeps at Lanczos tolerance 1e-10, the closing
half-sweep to the measurement point -- keeping m = 256 multiplets, start
vectors from a seeded generator (seed 7), every step on the oracle (the C
restatement of the reference's routines, FP64).  Then the correlators of
Measurement (main.f90:191-332).  The file holds every step's energy,
Lanczos iterations, kept multiplets and truncation error, and the
correlators; the GPU test runs the same schedule on the device and compares.
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from grand_sql_tj_b200.lattice import Geometry  # noqa: E402
from grand_sql_tj_b200.measure import measurement  # noqa: E402
from grand_sql_tj_b200.sweep import Dmrg, DmrgParams  # noqa: E402

NX, NY, ELECTRONS, M, SWEEPS, SEED = 16, 2, 28, 256, 10, 7
LANZERO = 1e-10


def config1_run(backend, sweeps=SWEEPS):
    """The schedule above on `backend`; returns (Dmrg, correlators)."""
    geo = Geometry(NX, NY, t=1.0, J=1.0 / 3.0, t2=0.0, esite=0.0, up_bias=1)
    p = DmrgParams(n_elec=ELECTRONS, kept_min=M, kept_max=M, lanzero=LANZERO, lanzero_warm=LANZERO * 1000,
                   seed=SEED)
    d = Dmrg(geo, backend, p)
    d.ground_state(sweeps, final_half=True)
    return d, measurement(backend, d)


def as_json(d, cors):
    return {
        "lattice": "%dx%d ladder" % (NY, NX), "electrons": ELECTRONS, "m": M, "sweeps": SWEEPS, "seed": SEED,
        "lanzero": LANZERO,
        "steps": [[r.phase, r.sys_len, r.env_len, r.energy, r.iters, r.num_state, r.trunc_err] for r in d.records],
        "correlators": {k: [[*key, v] for key, v in sorted(c.items())] for k, c in cors.items()},
    }


def main():
    from oracle import oracle
    from oracle.oracle import OracleBackend
    oracle.set_threads(os.cpu_count() or 1)
    t = time.perf_counter()
    d, cors = config1_run(OracleBackend())
    out = as_json(d, cors)
    out["oracle_seconds"] = time.perf_counter() - t
    with open(os.path.join(HERE, "config1_ladder16_m256.json"), "w") as f:
        json.dump(out, f, indent=0)
    print("steps", len(d.records), "E", d.records[-1].energy, "s", out["oracle_seconds"])


if __name__ == "__main__":
    main()
