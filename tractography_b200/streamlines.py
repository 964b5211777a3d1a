"""Streamline containers and the MRtrix ``.tck`` format.

``tracking.tractogram`` in the reference returns a
``nibabel.streamlines.Tractogram`` built from a Python list of per-seed array
views (tractography/tracking.py:178), and the command line writes it with
``nibabel.streamlines.TckFile`` (tractography/cli/tractogram.py:68-78).
Here streamlines are kept packed -- one (total_points, 3) float32 array plus
per-streamline offsets and lengths -- which is what the GPU produces, and
``ArraySequence`` exposes them as a sequence of (n, 3) views without copying.
When nibabel is installed, :func:`to_nibabel` converts to its classes.

TCK layout (MRtrix3 file format, public): a text header starting with
``mrtrix tracks`` and ending with ``END``; ``file: . <offset>`` gives the
byte offset of the binary data; points are little-endian float32 triplets;
each streamline is terminated by a (NaN, NaN, NaN) triplet and the file by
an (Inf, Inf, Inf) triplet.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np


class ArraySequence:
    """Sequence of (n_i, 3) float32 arrays stored in one packed buffer."""

    def __init__(self, data=None, offsets=None, lengths=None):
        if data is None:
            data = np.empty((0, 3), dtype=np.float32)
        self._data = np.asarray(data, dtype=np.float32).reshape(-1, 3)
        self._offsets = np.asarray(offsets if offsets is not None else [], dtype=np.int64)
        self._lengths = np.asarray(lengths if lengths is not None else [], dtype=np.int64)
        if self._offsets.shape != self._lengths.shape:
            raise ValueError("offsets and lengths must have the same shape")

    @classmethod
    def from_arrays(cls, arrays):
        arrays = [np.asarray(a, dtype=np.float32).reshape(-1, 3) for a in arrays]
        lengths = np.array([len(a) for a in arrays], dtype=np.int64)
        offsets = np.zeros(len(arrays), dtype=np.int64)
        if len(arrays) > 1:
            np.cumsum(lengths[:-1], out=offsets[1:])
        data = np.concatenate(arrays, axis=0) if arrays else np.empty((0, 3), np.float32)
        return cls(data, offsets, lengths)

    @property
    def data(self) -> np.ndarray:
        return self._data

    @property
    def offsets(self) -> np.ndarray:
        return self._offsets

    @property
    def lengths(self) -> np.ndarray:
        return self._lengths

    def get_data(self) -> np.ndarray:
        """Points of all streamlines, in streamline order."""
        if len(self) == 0:
            return np.empty((0, 3), dtype=np.float32)
        if self._is_contiguous():
            return self._data[: int(self._lengths.sum())]
        return np.concatenate([self[i] for i in range(len(self))], axis=0)

    def _is_contiguous(self) -> bool:
        if len(self) == 0:
            return True
        expected = np.zeros_like(self._offsets)
        if len(self) > 1:
            np.cumsum(self._lengths[:-1], out=expected[1:])
        return bool(self._offsets[0] == 0 and np.array_equal(expected, self._offsets))

    def __len__(self) -> int:
        return len(self._lengths)

    def __getitem__(self, index):
        if isinstance(index, (int, np.integer)):
            i = int(index)
            if i < 0:
                i += len(self)
            if not 0 <= i < len(self):
                raise IndexError("streamline index out of range")
            o = int(self._offsets[i])
            return self._data[o: o + int(self._lengths[i])]
        sel = np.arange(len(self))[index]
        return ArraySequence(self._data, self._offsets[sel], self._lengths[sel])

    def __iter__(self):
        for i in range(len(self)):
            yield self[i]

    def copy(self) -> "ArraySequence":
        lengths = self._lengths.copy()
        offsets = np.zeros_like(lengths)
        if len(lengths) > 1:
            np.cumsum(lengths[:-1], out=offsets[1:])
        return ArraySequence(self.get_data().copy(), offsets, lengths)


class Tractogram:
    """Streamlines with the affine that maps them to RAS+ mm.

    Mirrors the parts of ``nibabel.streamlines.Tractogram`` the reference's
    API returns: ``streamlines`` and ``affine_to_rasmm``.
    """

    def __init__(self, streamlines=None, affine_to_rasmm=None):
        if streamlines is None:
            streamlines = ArraySequence()
        elif not isinstance(streamlines, ArraySequence):
            streamlines = ArraySequence.from_arrays(list(streamlines))
        self.streamlines = streamlines
        self.affine_to_rasmm = None if affine_to_rasmm is None else np.asarray(affine_to_rasmm)
        self.data_per_streamline = {}
        self.data_per_point = {}

    def __len__(self) -> int:
        return len(self.streamlines)


def to_nibabel(tractogram: Tractogram):  # pragma: no cover - needs nibabel
    """Convert to ``nibabel.streamlines.Tractogram`` (nibabel must be installed)."""
    from nibabel.streamlines import ArraySequence as NibSeq
    from nibabel.streamlines import Tractogram as NibTractogram

    seq = NibSeq()
    seq._data = tractogram.streamlines.data
    seq._offsets = tractogram.streamlines.offsets
    seq._lengths = tractogram.streamlines.lengths
    return NibTractogram(seq, affine_to_rasmm=tractogram.affine_to_rasmm)


_TCK_MAGIC = b"mrtrix tracks\n"


def save_tck(filename, tractogram) -> None:
    """Write streamlines (RAS+ mm) to an MRtrix ``.tck`` file."""
    streamlines = tractogram.streamlines if hasattr(tractogram, "streamlines") else tractogram
    if not isinstance(streamlines, ArraySequence):
        streamlines = ArraySequence.from_arrays(list(streamlines))
    affine = getattr(tractogram, "affine_to_rasmm", None)
    n = len(streamlines)
    header_fields = [
        b"count: %010d\n" % n,
        b"datatype: Float32LE\n",
    ]
    body = b"".join(header_fields)
    # The offset line's own length depends on the offset: iterate to a fix point.
    offset = len(_TCK_MAGIC) + len(body) + len(b"file: . 0\nEND\n")
    while True:
        line = b"file: . %d\n" % offset
        total = len(_TCK_MAGIC) + len(body) + len(line) + len(b"END\n")
        if total <= offset:
            break
        offset = total
    header = _TCK_MAGIC + body + (b"file: . %d\n" % offset) + b"END\n"
    header = header + b" " * (offset - len(header))
    lengths = streamlines.lengths
    out = np.empty((int(lengths.sum()) + n + 1, 3), dtype="<f4")
    pos = 0
    for i in range(n):
        pts = streamlines[i]
        if affine is not None and not np.array_equal(affine, np.eye(4)):
            pts = pts @ affine[:3, :3].T + affine[:3, 3]
        out[pos: pos + len(pts)] = pts
        pos += len(pts)
        out[pos] = np.nan
        pos += 1
    out[pos] = np.inf
    with open(filename, "wb") as f:
        f.write(header)
        f.write(out.tobytes())


def load_tck(filename) -> Tractogram:
    """Read an MRtrix ``.tck`` file written with float32 little-endian data."""
    raw = Path(filename).read_bytes()
    if not raw.startswith(_TCK_MAGIC):
        raise ValueError(f"{filename} is not an MRtrix tracks file")
    end = raw.index(b"\nEND\n")
    fields = {}
    for line in raw[len(_TCK_MAGIC): end].split(b"\n"):
        if b":" in line:
            k, v = line.split(b":", 1)
            fields[k.strip().decode()] = v.strip().decode()
    if fields.get("datatype", "Float32LE") != "Float32LE":
        raise ValueError("only Float32LE .tck files are supported")
    offset = int(fields["file"].split()[1])
    pts = np.frombuffer(raw[offset:], dtype="<f4")
    pts = pts[: len(pts) // 3 * 3].reshape(-1, 3)
    inf_rows = np.where(np.all(np.isinf(pts), axis=1))[0]
    if len(inf_rows):
        pts = pts[: inf_rows[0]]
    nan_rows = np.where(np.all(np.isnan(pts), axis=1))[0]
    arrays = []
    start = 0
    for r in nan_rows:
        arrays.append(pts[start:r])
        start = r + 1
    if start < len(pts):
        arrays.append(pts[start:])
    return Tractogram(ArraySequence.from_arrays(arrays), affine_to_rasmm=np.eye(4))
