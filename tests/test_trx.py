"""TRX output: streaming batches of packed arrays, round trip and archive layout."""

import json
import zipfile

import numpy as np

from tractography_b200 import streamlines as S


def test_trx_round_trip_in_batches(tmp_path):
    rng = np.random.default_rng(0)
    lengths = [rng.integers(1, 20, 30), rng.integers(1, 20, 0), rng.integers(1, 20, 17)]
    batches = [rng.normal(size=(int(L.sum()), 3)).astype(np.float32) for L in lengths]
    path = tmp_path / "out.trx"
    affine = np.diag([2.0, 2.0, 2.0, 1.0])
    with S.TrxWriter(path, affine, (32, 32, 32)) as w:
        for pts, L in zip(batches, lengths):
            w.append(pts, L)
    t, header = S.load_trx(path)
    want = [a for pts, L in zip(batches, lengths) for a in np.split(pts, np.cumsum(L)[:-1]) if len(L)]
    assert len(t.streamlines) == 47 == header["NB_STREAMLINES"]
    assert header["NB_VERTICES"] == sum(int(L.sum()) for L in lengths)
    assert header["DIMENSIONS"] == [32, 32, 32] and np.allclose(header["VOXEL_TO_RASMM"], affine)
    for a, b in zip(t.streamlines, want):
        assert np.array_equal(a, b)
    with zipfile.ZipFile(path) as z:
        assert sorted(z.namelist()) == ["header.json", "offsets.uint64", "positions.3.float32"]
        assert all(i.compress_type == zipfile.ZIP_STORED for i in z.infolist())
        assert json.loads(z.read("header.json"))["NB_STREAMLINES"] == 47


def test_trx_from_packed_sequence_with_gaps(tmp_path):
    data = np.arange(30, dtype=np.float32).reshape(10, 3)
    seq = S.ArraySequence(data, np.array([7, 0, 3]), np.array([2, 3, 1]))
    S.save_trx(tmp_path / "g.trx", S.Tractogram(seq))
    t, _ = S.load_trx(tmp_path / "g.trx")
    assert [len(s) for s in t.streamlines] == [2, 3, 1]
    assert np.array_equal(t.streamlines[0], data[7:9]) and np.array_equal(t.streamlines[2], data[3:4])
