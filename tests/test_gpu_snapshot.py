"""GPU tests of tree snapshots (hm_snapshot_save / hm_snapshot_load) and of
building a tree from a reference insert file, checked against the oracle."""
import numpy as np
import pytest

from harmonia_b200 import BPlusTree, HarmoniaError, datagen as dg
from harmonia_b200.files import write_keys
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def test_snapshot_round_trip_after_upserts(tmp_path):
    keys = dg.gen_keys(1 << 18, 21)
    with BPlusTree.bulk_load(keys, dg.values_for(keys), leaf_fill=12) as t:
        bk, bv = dg.gen_upserts(keys, 4000, 0.5, seed=22)
        t.upsert(bk, bv)
        ek, ev = t.export()
        p = str(tmp_path / "tree.hmb")
        t.save(p)
    with BPlusTree.load(p) as t2:  # the saved configuration
        k2, v2 = t2.export()
        assert (k2 == ek).all() and (v2 == ev).all()
        assert t2.config()["leaf_fill"] == 12
        q = dg.gen_point_queries(ek, 1 << 16, 0.8, seed=23)
        assert (t2.search(q) == po.PortTree(ek, ev).search(q)).all()
    with BPlusTree.load(p, fanout=128, leaf_cap=64) as t3:  # another shape, same contents
        k3, v3 = t3.export()
        assert (k3 == ek).all() and (v3 == ev).all()
        assert t3.info().fanout == 128


def test_snapshot_rejects_damaged_files(tmp_path):
    keys = dg.gen_keys(5000, 24)
    p = tmp_path / "t.hmb"
    with BPlusTree.bulk_load(keys, dg.values_for(keys)) as t:
        t.save(str(p))
    raw = bytearray(p.read_bytes())
    for name, data in (("flipped", raw[:100] + bytes([raw[100] ^ 1]) + raw[101:]),
                       ("truncated", raw[:-9]), ("header", b"HMBTSNP2" + raw[8:])):
        bad = tmp_path / f"{name}.hmb"
        bad.write_bytes(bytes(data))
        with pytest.raises(HarmoniaError) as e:
            BPlusTree.load(str(bad))
        assert e.value.code == -12, name
    with pytest.raises(HarmoniaError) as e:
        BPlusTree.load(str(tmp_path / "missing.hmb"))
    assert e.value.code == -12


def test_empty_tree_snapshot(tmp_path):
    e = np.empty(0, np.int64)
    with BPlusTree.bulk_load(e, e) as t:
        t.save(str(tmp_path / "e.hmb"))
    with BPlusTree.load(str(tmp_path / "e.hmb")) as t2:
        assert t2.size == 0
        assert (t2.search(np.array([1, 2], np.int64)) == -1).all()


def test_tree_from_reference_insert_file(tmp_path):
    # the reference's main() inserts every key of the insert file with value = key
    keys = dg.gen_keys(1 << 16, 25)
    p = tmp_path / "insert64_0m.txt"
    write_keys(str(p), keys)
    with BPlusTree.from_reference_file(str(p)) as t:
        sk = np.sort(keys)
        q = dg.gen_point_queries(keys, 1 << 15, 0.5, seed=26)
        assert (t.search(q) == po.PortTree(sk, sk).search(q)).all()
