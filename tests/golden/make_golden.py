"""Build ``tests/golden/plan01_ug.npz`` from the reference's own golden file.

The reference stores the outputs of its fixed-seed capture
(``tests/test_data/plan01_ug_reference.npz``, written by
``tests/test_data/plan01_ug_capture.py:40-108``) but not the input potential,
which it draws as ``jax.random.uniform(PRNGKey(42), (32, 32, 2), float64) * 10``.
This script regenerates that input with the Threefry restatement in
``oracle/jax_prng.py`` and stores it next to the reference outputs and the
capture's scalar parameters, so the tests need neither JAX nor the reference
tree at run time.

Run from the repository root (needs the reference checkout):
    python tests/golden/make_golden.py REFERENCE_ROOT
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.jax_prng import prng_key, uniform_f64  # noqa: E402


def main() -> None:
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <reference project root>")
    ref_root = sys.argv[1]
    ref = np.load(os.path.join(ref_root, "tests/test_data/plan01_ug_reference.npz"))
    pot = uniform_f64(prng_key(42), (32, 32, 2)) * 10.0
    out = {
        "pot": pot,
        "cbed": ref["cbed"],
        "stem4d": ref["stem4d"],
        "stem4d_sharded": ref["stem4d_sharded"],
        "grad_pot": ref["grad_pot"],
        # plan01_ug_capture.py:34-38, 45-66
        "voltage_kv": np.float64(100.0),
        "aperture_mrad": np.float64(20.0),
        "calib_ang": np.float64(0.2),
        "slice_thickness_ang": np.float64(2.0),
        "positions_px": np.array([[12.0, 12.0], [12.0, 20.0], [20.0, 12.0], [20.0, 20.0]]),
    }
    path = os.path.join(HERE, "plan01_ug.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: " + ", ".join(f"{k}{np.shape(v)}" for k, v in out.items()))


if __name__ == "__main__":
    main()
