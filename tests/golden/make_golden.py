#!/usr/bin/env python3
"""Generate golden vectors from the reference's own NumPy implementations.

Run on a machine where the reference sources are available
(oracle.build_ref.reference_root); writes tests/golden/reference_numpy.npz.  The reference
imports pyopencl, nibabel, trimesh and nimesh at module level; none of their
functionality is used by the functions called here, so minimal stand-ins are
registered in sys.modules first (pyopencl.cltypes dtypes, nibabel's
apply_affine and an in-memory image, a mesh with face areas).

Every array stored is either an input we generate (seeded) or the output of a
reference function on it, so the tests compare our code with the reference's
results without needing the reference at test time.
"""

from __future__ import annotations

import argparse
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

from oracle.build_ref import reference_root  # noqa: E402
from oracle.refstubs import install_stubs  # noqa: E402


def orientations(rng, n):
    phi = rng.uniform(0, 2 * np.pi, n)
    theta = np.arccos(rng.uniform(-1, 1, n))
    o = np.stack([np.sin(theta) * np.cos(phi), np.sin(theta) * np.sin(phi), np.cos(theta)], -1)
    o[:4] = [[0, 0, 1], [0, 0, -1], [1, 0, 0], [0.6, 0.8, 0.0]]
    return o


def quadratic_fod(tg, base, eps, C):
    d = tg.core.fibonacci_sphere(1000)
    az, co, _ = tg.core.cart2sph(*d.T)
    Y, _ = tg.core.ishtmtx(az, co, C)
    return np.linalg.lstsq(Y, base + eps * d[:, 0] * d[:, 2], rcond=None)[0]


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=str(reference_root()))
    args = ap.parse_args()
    install_stubs(Path(args.reference))
    import tractography as ref  # noqa: E402  (the reference package)

    rng = np.random.default_rng(20261203)
    out = {}

    # local models (local.py:123-189, 233-262)
    for C in (15, 28, 45):
        o = orientations(rng, 400)
        p = np.stack([quadratic_fod(ref, b, e, C) for b, e in rng.uniform([0.05, 0.1], [0.3, 0.6], (8, 2))])
        p = p[rng.integers(0, 8, 400)] + rng.normal(0, 0.01, (400, C))
        out[f"sh{C}_params"] = p.astype(np.float32)
        out[f"sh{C}_orient"] = o.astype(np.float32)
        out[f"sh{C}_value"] = ref.local.RealSymmetricSphericalHarmonics(C).evaluate(
            p.astype(np.float32).astype(np.float64), o.astype(np.float32).astype(np.float64))
    pd = np.abs(rng.normal(1e-3, 5e-4, (300, 6)))
    pd[:, 3:] = rng.normal(0, 2e-4, (300, 3))
    od = orientations(rng, 300)
    out["dti_params"], out["dti_orient"] = pd.astype(np.float32), od.astype(np.float32)
    out["dti_value"] = ref.local.DiffusionTensorImaging().evaluate(pd.astype(np.float32).astype(np.float64),
                                                                   od.astype(np.float32).astype(np.float64))

    # Transport / zero-noise Diffusion one-step updates (algorithm.py:119-156, 243-269)
    p = out["sh45_params"].astype(np.float64)
    o = out["sh45_orient"].astype(np.float64)
    for name, alg in (("transport", ref.algorithm.Transport(ref.local.RealSymmetricSphericalHarmonics(45),
                                                             step_size=0.01, gamma=1.5)),
                      ("diffusion0", ref.algorithm.Diffusion(ref.local.RealSymmetricSphericalHarmonics(45),
                                                              step_size=0.02, gamma=0.7, noise_variance=0.0))):
        out[f"{name}_update"] = alg.update_orientation(p, o)
    dti_alg = ref.algorithm.Transport(ref.local.DiffusionTensorImaging(), step_size=0.1, gamma=10.0)
    out["dti_transport_update"] = dti_alg.update_orientation(out["dti_params"].astype(np.float64),
                                                             out["dti_orient"].astype(np.float64))
    out["exps2_p"], out["exps2_x"] = o[:50], rng.normal(0, 0.3, (50, 3))
    out["exps2_out"] = ref.algorithm.exps2(out["exps2_p"], out["exps2_x"], 1.0)

    # field and domain nearest-voxel sampling (field.py:124-141, domain.py:400-430)
    img = rng.normal(size=(5, 6, 7, 3)).astype(np.float32)
    affine = np.array([[2.0, 0.1, 0, -3], [0, 1.5, 0.2, 1], [0.1, 0, 1.8, 2], [0, 0, 0, 1]])
    fimg = ref.field.Image(sys.modules["nibabel.nifti1"].Nifti1Image(img, affine))
    pts = rng.uniform(-6, 14, (2000, 3))
    vox = np.round(rng.uniform(-1, 7, (200, 3)) * 2) / 2          # exact half-voxel ties
    pts[:200] = vox @ affine[:3, :3].T + affine[:3, 3]
    out["field_img"], out["field_affine"], out["field_points"] = img, affine, pts.astype(np.float32)
    out["field_inv_affine"] = fimg.inverse_affine
    out["field_value"] = fimg.evaluate(pts.astype(np.float32))
    mask = (rng.uniform(size=(6, 5, 4)) > 0.4).astype(np.uint8)
    dimg = ref.domain.Image(sys.modules["nibabel.nifti1"].Nifti1Image(mask, affine))
    out["mask"], out["mask_inv_affine"] = mask, dimg.inverse_affine
    out["mask_points"] = pts.astype(np.float32)
    out["mask_contains"] = dimg.contains(pts.astype(np.float32))

    # core helpers (core.py)
    az, co = rng.uniform(0, 2 * np.pi, 200), rng.uniform(0, np.pi, 200)
    Y, dY = ref.core.ishtmtx(az, co, 45)
    out["ishtmtx_az"], out["ishtmtx_co"], out["ishtmtx_Y"], out["ishtmtx_dY"] = az, co, Y, dY
    out["fibonacci1000"] = ref.core.fibonacci_sphere(1000)
    cart = np.array([[2.0, 0, 0], [0, -3, 0], [0, 0, -4], [0, 0, 0], [1, 1, 1], [-1, 0.5, -0.2]])
    out["cart2sph_in"] = cart
    out["cart2sph_out"] = np.stack(ref.core.cart2sph(*cart.T), -1)

    # host seeding with NumPy's legacy generator (seeds.py:114-142, 218-240)
    smask = np.zeros((6, 7, 5))
    smask[1:4, 2:6, 1:4] = 1
    np.random.seed(7)
    out["from_mask"] = ref.seeds.from_mask(sys.modules["nibabel.nifti1"].Nifti1Image(smask, affine), 300)
    out["from_mask_input"] = smask
    fod = np.zeros((3, 2, 2, 45))
    for idx in np.ndindex(3, 2, 2):
        fod[idx] = quadratic_fod(ref, 0.2 + 0.1 * idx[0], 0.5, 45)
    fod[1, 1, 1] = 0
    np.random.seed(11)
    out["from_fod_numpy"] = ref.seeds.from_fod(sys.modules["nibabel.nifti1"].Nifti1Image(fod, affine), 120,
                                               use_opencl=False)
    out["from_fod_input"] = fod
    out["affine"] = affine
    np.savez_compressed(HERE / "reference_numpy.npz", **out)
    print(f"wrote {HERE / 'reference_numpy.npz'} with {len(out)} arrays")


if __name__ == "__main__":
    main()
