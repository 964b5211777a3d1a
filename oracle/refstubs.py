"""Stand-ins for the reference's import-time dependencies (test infrastructure only).

The reference package imports pyopencl, nibabel, trimesh, nimesh and
platformdirs at module level.  To call its NumPy reference functions and to
capture the OpenCL source it assembles, this module registers minimal
stand-ins in sys.modules: pyopencl.cltypes dtypes and mem_flags, nibabel's
apply_affine with an in-memory image and a Tractogram holder, and a triangle
mesh that computes face areas.  Nothing here runs OpenCL.
"""

from __future__ import annotations

import sys
import types
from pathlib import Path

import numpy as np


def install_stubs(reference_root: Path) -> None:
    cl = types.ModuleType("pyopencl")

    class mem_flags:  # noqa: N801 - mirrors the pyopencl name
        READ_ONLY, WRITE_ONLY, READ_WRITE, COPY_HOST_PTR = 1, 2, 4, 8

    cl.mem_flags = mem_flags
    for name in ("Device", "Context", "CommandQueue", "Program", "Buffer", "Event", "Kernel"):
        setattr(cl, name, type(name, (), {}))
    clt = types.ModuleType("pyopencl.cltypes")
    clt.float, clt.uint, clt.int = np.float32, np.uint32, np.int32
    cl.cltypes = clt
    sys.modules["pyopencl"] = cl
    sys.modules["pyopencl.cltypes"] = clt

    class Image:
        def __init__(self, data, affine=None, header=None):
            self._data = np.asarray(data)
            self.affine = np.eye(4) if affine is None else np.asarray(affine, dtype=float)
            self.header = header
            self.shape, self.ndim, self.dataobj = self._data.shape, self._data.ndim, self._data

        def get_fdata(self):
            return np.asarray(self._data, dtype=np.float64)

    class Tractogram:
        def __init__(self, streamlines, affine_to_rasmm=None):
            self.streamlines = list(streamlines)
            self.affine_to_rasmm = affine_to_rasmm

    nib = types.ModuleType("nibabel")
    aff = types.ModuleType("nibabel.affines")
    aff.apply_affine = lambda a, p: np.dot(np.asarray(p), np.asarray(a)[:3, :3].T) + np.asarray(a)[:3, 3]
    nib.affines = aff
    modules = {"nibabel": nib, "nibabel.affines": aff}
    for name in ("nibabel.nifti1", "nibabel.spatialimages", "nibabel.streamlines",
                 "nibabel.streamlines.tractogram"):
        modules[name] = types.ModuleType(name)
    modules["nibabel.nifti1"].Nifti1Image = Image
    modules["nibabel.spatialimages"].SpatialImage = Image
    modules["nibabel.streamlines.tractogram"].Tractogram = Tractogram
    nib.nifti1 = modules["nibabel.nifti1"]
    sys.modules.update(modules)

    class Trimesh:
        def __init__(self, vertices, faces, process=False):
            self.vertices = np.asarray(vertices, float)
            self.faces = np.asarray(faces)
            t = self.vertices[self.faces]
            self.area_faces = 0.5 * np.linalg.norm(np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0]), axis=1)

    tm = types.ModuleType("trimesh")
    tm.Trimesh = Trimesh
    sys.modules["trimesh"] = tm
    nm = types.ModuleType("nimesh")
    nm.Mesh = object
    sys.modules["nimesh"] = nm
    pd = types.ModuleType("platformdirs")
    pd.user_cache_path = lambda *a, **k: Path("/tmp")
    sys.modules["platformdirs"] = pd
    sys.path.insert(0, str(reference_root))
