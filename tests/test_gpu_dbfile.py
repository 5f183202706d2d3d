"""GPU check of bp_db_open: a database file streamed into HBM through the
pinned staging buffers searches exactly like the same subjects uploaded from
memory -- in file order, across volume and staging-buffer boundaries, and for
a length-sorted file (results map back through the oid map)."""
import numpy as np
import pytest

from blastp_b200 import BpError, read_database_file, synth, write_database_file
from helpers import assert_same

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("volume,sort", [(0, False), (3_000_000, False), (1 << 20, True)])
def test_open_matches_memory(engine, matrix, tmp_path, volume, sort):
    w = synth.shape2(matrix, n_subjects=250_000)      # ~90M residues: several 64 MiB staging rounds
    p = tmp_path / "db.bpdb"
    write_database_file(p, w.db.residues, w.db.offsets, volume_residues=volume, sort_by_length=sort)
    res, off, oids, nv = read_database_file(p)
    q = engine.query(w.queries[0])
    from_file = engine.open_database(p)
    assert from_file.n_subjects == w.db.n_subjects and from_file.n_residues == w.db.n_residues
    got = engine.search(from_file, q).fetch()
    ref = engine.search(engine.database(res, off), q).fetch()
    assert_same(got, (ref.counters, ref.hsp_off, ref.hsps_as_array()), "file vs memory")
    if sort:
        # the same subjects in their original order give the same per-subject results
        orig = engine.search(engine.database(w.db.residues, w.db.offsets), q).fetch()
        assert (orig.counters[oids] == got.counters).all()
        for i in range(0, len(oids), 997):
            a = got.hsps_as_array()[got.hsp_off[i]:got.hsp_off[i + 1]]
            o = oids[i]
            b = orig.hsps_as_array()[orig.hsp_off[o]:orig.hsp_off[o + 1]]
            assert (a == b).all()


def test_open_rejects_bad_residue_codes(engine, tmp_path):
    p = tmp_path / "bad.bpdb"
    write_database_file(p, np.array([1, 2, 3, 4], np.uint8), np.array([0, 4], np.int64))
    raw = bytearray(p.read_bytes())
    at = raw.index(bytes([1, 2, 3, 4]))
    raw[at + 2] = 99                                   # damage a residue after writing
    p.write_bytes(bytes(raw))
    with pytest.raises(BpError):
        engine.open_database(p)
