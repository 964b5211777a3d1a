#!/usr/bin/env python3
"""Per-step error of the binary32 path against the reference's FP64 NumPy oracle.

Test infrastructure only; run where the reference sources are available
(see oracle.build_ref.reference_root).  For each workload configuration, orientation
updates are drawn at random voxels of that configuration's synthetic field
with uniformly random orientations, and one orientation update is computed

  * in binary32 by the CPU oracle, whose results equal the CUDA kernels' bit
    for bit (tests/test_gpu_parity.py), and
  * in float64 by the reference's own NumPy implementation
    (algorithm.py:119-156 Transport, :243-269 Diffusion with zero noise, i.e.
    its drift) on the same float32 inputs widened to float64.

The error of a step is the largest absolute component difference of the
updated unit orientation, i.e. radians for small errors; a 0.1-voxel step
turns it into a position error of step_size x error.  Writes the table to
profiles/step_error_fp64.md.

Usage: python oracle/step_error.py [--reference DIR] [--samples 20000]
"""

from __future__ import annotations

import argparse
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
from oracle.build_ref import reference_root  # noqa: E402


def sample(field_values, rng, n):
    X, Y, Z, _ = field_values.shape
    vox = np.stack([rng.integers(0, X, n), rng.integers(0, Y, n), rng.integers(0, Z, n)], -1)
    params = field_values[vox[:, 0], vox[:, 1], vox[:, 2]].astype(np.float32)
    keep = np.any(params != 0, axis=1)
    o = rng.normal(size=(n, 3))
    o /= np.linalg.norm(o, axis=1, keepdims=True)
    return params[keep], o.astype(np.float32)[keep]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=str(reference_root()))
    ap.add_argument("--samples", type=int, default=20000)
    args = ap.parse_args()
    from oracle.refstubs import install_stubs

    install_stubs(Path(args.reference))
    import tractography as ref  # the reference package

    from oracle import oracle as O
    from oracle import reference as R
    from tractography_b200 import synthetic

    rng = np.random.default_rng(11)
    rows = []

    def measure(name, values, model, algorithm, step, gamma, note):
        params, o = sample(values, rng, args.samples)
        C = params.shape[1]
        local = ref.local.DiffusionTensorImaging() if model == O.MODEL_DTI else \
            ref.local.RealSymmetricSphericalHarmonics(C)
        if algorithm == O.ALGO_TRANSPORT:
            alg = ref.algorithm.Transport(local, step_size=step, gamma=gamma)
        else:
            alg = ref.algorithm.Diffusion(local, step_size=step, gamma=gamma, noise_variance=0.0, seed=0)
        exact = alg.update_orientation(params.astype(np.float64), o.astype(np.float64))
        got = O.Case(model=model, algorithm=algorithm, step_size=step, gamma=gamma, noise_variance=0.0
                     ).update_orientation(params, o)
        err = np.abs(got.astype(np.float64) - exact).max(axis=1)
        kind = "dti" if model == O.MODEL_DTI else "sh"
        ref32 = R.update_orientation(kind, C, "transport" if algorithm == O.ALGO_TRANSPORT else "diffusion", step,
                                     gamma, 0.0, 0, params, o) if R.available() else None
        e_ref = np.abs(ref32.astype(np.float64) - exact).max(axis=1) if ref32 is not None else np.full(1, np.nan)
        rows.append((name, note, len(err), np.median(err), np.percentile(err, 99), err.max(),
                     step * np.median(err), step * np.percentile(err, 99), np.median(e_ref),
                     np.percentile(e_ref, 99)))
        print(rows[-1], flush=True)

    fod0, _ = synthetic.config0()
    measure("config 0", np.asarray(fod0.dataobj), O.MODEL_SH, O.ALGO_TRANSPORT, 0.2, 1.0,
            "SH lmax 8, Transport, step 0.2 mm")
    fod1 = synthetic.config1(shape=(72, 88, 72))
    measure("config 1", np.asarray(fod1.dataobj), O.MODEL_SH, O.ALGO_DIFFUSION, 0.001, 1.0,
            "SH lmax 8, Diffusion drift (noise 0), step 0.001 mm; generator at half size")
    fod2 = synthetic.dti_field(shape=(96, 96, 60))
    measure("config 2", np.asarray(fod2.dataobj), O.MODEL_DTI, O.ALGO_TRANSPORT, 0.2, 1.0,
            "DTI, Transport, step 0.2 mm")
    for lmax in (4, 6):
        fod, _ = synthetic.bundle_field((64, 64, 64), lmax=lmax, seed=lmax)
        measure(f"config 3 (lmax {lmax})", np.asarray(fod.dataobj), O.MODEL_SH, O.ALGO_TRANSPORT, 0.2, 1.0,
                f"SH lmax {lmax}, Transport, step 0.2 mm")

    out = ROOT_PROFILES / "step_error_fp64.md"
    lines = [
        "# Per-step orientation error of the binary32 path vs the reference's FP64 NumPy update",
        "",
        "Command: `python oracle/step_error.py --samples %d` (needs the reference sources;" % args.samples,
        "the binary32 side is the CPU oracle, bit-identical to the CUDA kernels).",
        "",
        "One orientation update at random voxels of each configuration's synthetic field with random",
        "unit orientations; error = max |component| of (binary32 - float64) updated orientation",
        "(radians for small errors); position error per step = step_size x error.",
        "",
        "The last two columns give the same error for the reference's own OpenCL kernel source compiled",
        "as C++ on the CPU (oracle/_ref, g++ libm transcendentals): the binary32 error of the reference",
        "itself.  The p99 tails come from voxels where the model value is near the 1e-6 floor of the",
        "drift's denominator (ill-conditioned in any binary32 evaluation).",
        "",
        "| config | case | samples | median | p99 | max | position median (mm) | position p99 (mm) "
        "| reference kernel median | reference kernel p99 |",
        "|---|---|---|---|---|---|---|---|---|---|",
    ]
    for r in rows:
        lines.append("| %s | %s | %d | %.3g | %.3g | %.3g | %.3g | %.3g | %.3g | %.3g |" % r)
    lines.append("")
    out.write_text("\n".join(lines))
    print("wrote", out)


ROOT_PROFILES = HERE.parent / "profiles"

if __name__ == "__main__":
    main()
