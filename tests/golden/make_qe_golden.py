"""Generates tests/golden/qe_refgpu.npz: throughput curves of the reference's
cuda_engine.

Runs oracle/_ref/harness_refgpu in its `qe` mode -- the reference's Surface
and Grating classes (SetRuleParams, ApplyQE) and ComputeQE's loop over the
reference's surface_QE and grating_energy_distr compiled for sm_100a -- on
every case of tests/qe_cases.py with single-value QE curves (the reference's
parallel spline_init makes tabulated curves irreproducible), and stores
<case>_lambda and <case>_qe (n_rows x n_lambda).  Needs a GPU; the fixture is
committed so that the CPU tests pin the oracle's blaze function to the
reference's kernel without one.

  python tests/golden/make_qe_golden.py [out.npz]
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]

import qe_cases as Q  # noqa: E402
import refharness as H  # noqa: E402


def main(out: str) -> None:
    arrays = {}
    for name, (specs, rows, n_lambda) in sorted(Q.cases().items()):
        rc, blocks = H.run_qe("refgpu", Q.scalar_qe(specs), rows, n_lambda)
        if rc != 0:
            raise SystemExit(f"{name}: harness_refgpu exited {rc}")
        arrays[name + "_lambda"] = np.stack([b[0] for b in blocks])
        arrays[name + "_qe"] = np.stack([b[1] for b in blocks])
        print(name, arrays[name + "_qe"].shape, flush=True)
    np.savez_compressed(out, **arrays)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "qe_refgpu.npz"))
