"""Database file (bp_dbfile_*): the host-side writer and reader need no GPU.
Round trips in stored order, multi-volume splits, length-sorted files with
their oid map, and rejected inputs and damaged files."""
import numpy as np
import pytest

from blastp_b200 import BpError, read_database_file, synth, write_database_file


def _db(seed, n=700):
    rng = np.random.default_rng(seed)
    lens = rng.integers(0, 900, size=n)
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    return synth.residues(rng, int(off[-1])), off


@pytest.mark.parametrize("volume", [0, 4096, 50_000, 1])
def test_round_trip_in_order(tmp_path, volume):
    res, off = _db(1)
    p = tmp_path / "db.bpdb"
    write_database_file(p, res, off, volume_residues=volume)
    r2, o2, oids, nv = read_database_file(p)
    assert (r2 == res).all() and (o2 == off).all() and (oids == np.arange(len(off) - 1)).all()
    if volume == 4096:
        assert nv > 10
    if volume == 1:          # every volume holds one subject of residues (empty ones join it)
        assert nv == np.count_nonzero(np.diff(off))


def test_sorted_by_length_with_oid_map(tmp_path):
    res, off = _db(2)
    p = tmp_path / "sorted.bpdb"
    write_database_file(p, res, off, volume_residues=100_000, sort_by_length=True)
    r2, o2, oids, nv = read_database_file(p)
    lens = np.diff(o2)
    assert (lens[:-1] >= lens[1:]).all()                      # longest first
    assert sorted(oids.tolist()) == list(range(len(off) - 1))
    for i in range(0, len(oids), 37):
        o = oids[i]
        assert (r2[o2[i]:o2[i + 1]] == res[off[o]:off[o + 1]]).all()


def test_empty_database(tmp_path):
    p = tmp_path / "empty.bpdb"
    write_database_file(p, np.zeros(0, np.uint8), np.zeros(1, np.int64))
    r2, o2, oids, nv = read_database_file(p)
    assert len(r2) == 0 and o2.tolist() == [0] and nv == 0


def test_rejected_inputs_and_damaged_files(tmp_path):
    res, off = _db(3, n=50)
    with pytest.raises(BpError):
        write_database_file(tmp_path / "x", res, off[:-1])                 # offsets do not end at n_residues
    bad = res.copy()
    bad[5] = 40
    with pytest.raises(BpError):
        write_database_file(tmp_path / "x", bad, off)                      # residue code >= 28
    p = tmp_path / "ok.bpdb"
    write_database_file(p, res, off)
    raw = p.read_bytes()
    (tmp_path / "magic.bpdb").write_bytes(b"XXXX" + raw[4:])
    (tmp_path / "short.bpdb").write_bytes(raw[: len(raw) // 2])
    for name in ("magic.bpdb", "short.bpdb", "missing.bpdb"):
        with pytest.raises(BpError):
            read_database_file(tmp_path / name)
