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


def _packed_rows(points, lengths, offsets):
    """Rows of packed streamlines laid end to end, each followed by a NaN row.

    ``points`` is (P, 3); streamline i is points[offsets[i] : offsets[i] +
    lengths[i]] (consecutive when ``offsets`` is None).  One gather, no
    per-streamline Python work.
    """
    lengths = np.asarray(lengths, dtype=np.int64)
    n = len(lengths)
    total = int(lengths.sum())
    out = np.empty((total + n, 3), dtype="<f4")
    if n == 0:
        return out
    ends = np.cumsum(lengths + 1)                   # one past each NaN row
    starts = ends - lengths - 1                     # first output row of each streamline
    src0 = np.cumsum(lengths) - lengths if offsets is None else np.asarray(offsets, dtype=np.int64)
    # output row r of streamline i takes points[src0[i] + (r - starts[i])]
    rows = np.arange(total, dtype=np.int64) + np.repeat(starts - (np.cumsum(lengths) - lengths), lengths)
    src = np.repeat(src0 - (np.cumsum(lengths) - lengths), lengths) + np.arange(total, dtype=np.int64)
    out[rows] = np.asarray(points, dtype=np.float32).reshape(-1, 3)[src]
    out[ends - 1] = np.nan
    return out


class TckWriter:
    """Streaming writer of MRtrix ``.tck`` files from packed batches.

    The reference writes through nibabel's ``TckFile`` from a Python list of
    streamlines (tractography/cli/tractogram.py:68-78).  Here each batch is
    appended as the packed (points, lengths, offsets) arrays the GPU produces;
    the header's ``count`` field has a fixed width and is rewritten on
    ``close``, so the file is written in one pass and no per-streamline
    Python objects are made.  ``affine`` (voxel-to-RAS, default identity) is
    applied to every point before it is written.
    """

    def __init__(self, filename, affine=None):
        self.filename = Path(filename)
        self.affine = None if affine is None or np.array_equal(affine, np.eye(4)) else \
            np.asarray(affine, dtype=np.float64)
        self.n_streamlines = 0
        self._f = open(self.filename, "wb")
        self._f.write(self._header(0))

    @staticmethod
    def _header(count: int) -> bytes:
        body = b"count: %010d\n" % count + b"datatype: Float32LE\n"
        # The offset line's own length depends on the offset: iterate to a fix point.
        offset = len(_TCK_MAGIC) + len(body) + len(b"file: . 0\nEND\n")
        while True:
            total = len(_TCK_MAGIC) + len(body) + len(b"file: . %d\n" % offset) + len(b"END\n")
            if total <= offset:
                break
            offset = total
        header = _TCK_MAGIC + body + (b"file: . %d\n" % offset) + b"END\n"
        return header + b" " * (offset - len(header))

    def append(self, points, lengths, offsets=None) -> None:
        """Append streamlines given as packed points (P, 3) (or (P, 4); the
        fourth column is dropped) with per-streamline lengths and optional
        offsets into points (default: consecutive)."""
        points = np.asarray(points, dtype=np.float32)
        points = points.reshape(-1, points.shape[-1])[:, :3] if points.size else points.reshape(0, 3)
        out = _packed_rows(points, lengths, offsets)
        if self.affine is not None and len(out):
            out = (out.astype(np.float64) @ self.affine[:3, :3].T + self.affine[:3, 3]).astype("<f4")
        self._f.write(out.tobytes())
        self.n_streamlines += len(lengths)

    def append_tractogram(self, tractogram) -> None:
        seq = tractogram.streamlines if hasattr(tractogram, "streamlines") else tractogram
        if not isinstance(seq, ArraySequence):
            seq = ArraySequence.from_arrays(list(seq))
        self.append(seq.data, seq.lengths, seq.offsets)

    def close(self) -> None:
        if self._f is None:
            return
        self._f.write(np.full((1, 3), np.inf, dtype="<f4").tobytes())
        self._f.seek(0)
        self._f.write(self._header(self.n_streamlines))
        self._f.close()
        self._f = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def save_tck(filename, tractogram) -> None:
    """Write streamlines (RAS+ mm) to an MRtrix ``.tck`` file."""
    with TckWriter(filename, getattr(tractogram, "affine_to_rasmm", None)) as w:
        w.append_tractogram(tractogram)


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


# ---------------------------------------------------------------------- TRX

class TrxWriter:
    """Streaming writer of the TRX tractography format (the batch writer of
    cli/tractogram.py:81-139, which the reference builds on trx-python).

    TRX layout (public format): a ZIP archive, stored uncompressed, holding
    ``header.json`` (``VOXEL_TO_RASMM`` 4x4, ``DIMENSIONS``, ``NB_VERTICES``,
    ``NB_STREAMLINES``), ``positions.3.float32`` (all points, little-endian
    float32 triplets) and ``offsets.uint64`` (index of each streamline's first
    point).  Batches are appended to spooled files as packed arrays -- the
    GPU's output layout -- so no per-streamline Python objects are made.
    """

    def __init__(self, filename, affine=None, dimensions=(1, 1, 1)):
        import tempfile

        self.filename = Path(filename)
        self.affine = np.eye(4) if affine is None else np.asarray(affine, dtype=np.float64)
        self.dimensions = [int(d) for d in dimensions]
        self._dir = tempfile.TemporaryDirectory()
        self._pos = open(Path(self._dir.name) / "positions", "wb")
        self._off = open(Path(self._dir.name) / "offsets", "wb")
        self.n_vertices = 0
        self.n_streamlines = 0

    def append(self, points, lengths, offsets=None) -> None:
        """Append streamlines given as packed points (P, 3) with per-streamline
        lengths (and offsets into points; default: consecutive)."""
        points = np.asarray(points, dtype="<f4").reshape(-1, 3)
        lengths = np.asarray(lengths, dtype=np.int64)
        if offsets is None:
            data = points[: int(lengths.sum())]
        else:
            offsets = np.asarray(offsets, dtype=np.int64)
            data = points[np.concatenate([np.arange(o, o + n) for o, n in zip(offsets, lengths)])] \
                if len(lengths) else points[:0]
        starts = self.n_vertices + np.concatenate([[0], np.cumsum(lengths)[:-1]]) if len(lengths) else lengths
        np.ascontiguousarray(data, dtype="<f4").tofile(self._pos)
        np.asarray(starts, dtype="<u8").tofile(self._off)
        self.n_vertices += int(lengths.sum())
        self.n_streamlines += len(lengths)

    def append_tractogram(self, tractogram) -> None:
        seq = tractogram.streamlines if hasattr(tractogram, "streamlines") else tractogram
        if isinstance(seq, ArraySequence):
            self.append(seq.data, seq.lengths, seq.offsets)
        else:
            arrays = [np.asarray(s, dtype=np.float32).reshape(-1, 3) for s in seq]
            self.append(np.concatenate(arrays) if arrays else np.empty((0, 3), np.float32),
                        np.array([len(a) for a in arrays], dtype=np.int64))

    def close(self) -> None:
        import json
        import zipfile

        if self._pos is None:
            return
        self._pos.close()
        self._off.close()
        header = {"VOXEL_TO_RASMM": self.affine.tolist(), "DIMENSIONS": self.dimensions,
                  "NB_VERTICES": self.n_vertices, "NB_STREAMLINES": self.n_streamlines}
        with zipfile.ZipFile(self.filename, "w", compression=zipfile.ZIP_STORED, allowZip64=True) as z:
            z.writestr("header.json", json.dumps(header))
            z.write(Path(self._dir.name) / "positions", "positions.3.float32")
            z.write(Path(self._dir.name) / "offsets", "offsets.uint64")
        self._pos = None
        self._dir.cleanup()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def save_trx(filename, tractogram, affine=None, dimensions=(1, 1, 1)) -> None:
    """Write a Tractogram (or sequence of (n, 3) arrays) as a TRX archive."""
    with TrxWriter(filename, affine, dimensions) as w:
        w.append_tractogram(tractogram)


def load_trx(filename):
    """Read a TRX archive written with float32 positions and uint32/uint64
    offsets; returns (Tractogram, header dict)."""
    import json
    import zipfile

    with zipfile.ZipFile(filename) as z:
        header = json.loads(z.read("header.json"))
        names = z.namelist()
        pos_name = next(n for n in names if n.startswith("positions.3."))
        off_name = next(n for n in names if n.startswith("offsets."))
        positions = np.frombuffer(z.read(pos_name), dtype="<" + _TRX_DTYPES[pos_name.rsplit(".", 1)[1]]).reshape(-1, 3)
        offsets = np.frombuffer(z.read(off_name), dtype="<" + _TRX_DTYPES[off_name.rsplit(".", 1)[1]]).astype(np.int64)
    n = int(header["NB_STREAMLINES"])
    lengths = np.diff(np.concatenate([offsets[:n], [int(header["NB_VERTICES"])]]))
    seq = ArraySequence(positions.astype(np.float32), offsets[:n], lengths)
    return Tractogram(seq, affine_to_rasmm=np.eye(4)), header


_TRX_DTYPES = {"float16": "f2", "float32": "f4", "float64": "f8", "uint32": "u4", "uint64": "u8"}
