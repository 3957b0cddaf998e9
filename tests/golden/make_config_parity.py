"""Digests of the oracle's results at the configurations' own sizes, for the
full-size GPU parity tests (tests/test_gpu_config_parity.py).

The correctly rounded oracle build (particle transcendentals from
libquadmath rounded to double) runs ~7x slower than the glibc build, too slow
to run at 10k-20k particles x 1000 turns inside the GPU test suite; its
results are recorded here once as SHA-256 digests.  The GPU result must have
the same digest (bit-identical).  The glibc build runs in the test itself;
its comparison with the correctly rounded build is recorded here too (the
particles whose plain per-coordinate relative error exceeds the bound), so
the test can show that the GPU differs from glibc on exactly those particles.

    python tests/golden/make_config_parity.py [config0 config1 ...]

Deterministic: the beams are seeded numpy Philox Gaussians and the oracle's
particle-major OpenMP loop gives the same bits for any thread count.
"""
import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT / "bmad-ecosystem_b200"))
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

from bgt import lattice as L  # noqa: E402
from helpers import (CONFIG_PARITY_CASES, config_parity_inputs, exceed_digest, oracle_track_elements,  # noqa: E402
                     plain_rel_err, result_digest)

OUT = HERE / "config_parity.json"
BOUNDS = {"1": 1e-13, "1000": 1e-9}


def case(name):
    c = CONFIG_PARITY_CASES[name]
    lat, v0 = config_parity_inputs(name)
    rec = {"n": c["n"], "turns": c["turns"], "apertures": c["apertures"], "beam": c["beam"]}
    for turns in (1, c["turns"]):
        t = time.time()
        cr = oracle_track_elements(lat, v0, 0, len(lat), turns, variant="cr")
        t_cr = time.time() - t
        t = time.time()
        gl = oracle_track_elements(lat, v0, 0, len(lat), turns, variant="glibc")
        t_gl = time.time() - t
        both = (cr[2] == L.ALIVE) & (gl[2] == L.ALIVE)
        err = plain_rel_err(cr[0], gl[0])
        bound = BOUNDS["1" if turns == 1 else "1000"]
        idx = np.nonzero(both & (err > bound))[0]
        rec[str(turns)] = {
            "digest_cr": result_digest(cr[0], cr[1], cr[2], cr[3], cr[4]),
            "lost_cr": int(np.sum(cr[2] != L.ALIVE)),
            "states_equal_glibc": bool(np.array_equal(cr[2], gl[2])),
            "loss_records_equal_glibc": bool(np.array_equal(cr[3], gl[3]) and np.array_equal(cr[4], gl[4])),
            "bound": bound,
            "exceed_count": int(idx.size),
            "exceed_digest": exceed_digest(idx),
            "max_plain_rel_err": float(np.max(err[both])) if both.any() else 0.0,
            "oracle_s": {"cr": round(t_cr, 1), "glibc": round(t_gl, 1)},
        }
        print(name, turns, rec[str(turns)], flush=True)
    return rec


def main(names):
    out = json.loads(OUT.read_text()) if OUT.exists() else {}
    for n in names:
        out[n] = case(n)
        OUT.write_text(json.dumps(out, indent=1, sort_keys=True) + "\n")


if __name__ == "__main__":
    main(sys.argv[1:] or list(CONFIG_PARITY_CASES))
