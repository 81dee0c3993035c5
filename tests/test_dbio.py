"""DG vector on-disk format (``bosss_b200.dbio``): the BSON codec against the known answers
of the BSON 1.1 specification, the GUID byte order of ``Guid.ToByteArray``, the
``CellFieldDataSet`` byte layout, part splitting, and save/load round trips (GlobalID
resorting, degree changes, missing fields, several ranks over gloo). No stored vector of
the reference exists to compare a file against byte for byte, so the file layout follows
the reference's serialisation code (cited in the module)."""
import gzip
import os
import socket
import struct
import uuid

import numpy as np
import pytest
import torch.multiprocessing as mp

from bosss_b200 import _capi as C
from bosss_b200 import dbio
from bosss_b200 import operator as O


def test_bson_specification_examples():
    # the two examples of the BSON specification's front page
    assert dbio.encode_document({"hello": "world"}) == (
        b"\x16\x00\x00\x00\x02hello\x00\x06\x00\x00\x00world\x00\x00")
    doc = {"BSON": ["awesome", 5.05, 1986]}
    raw = (b"\x31\x00\x00\x00\x04BSON\x00\x26\x00\x00\x00\x020\x00\x08\x00\x00\x00awesome\x00"
           b"\x011\x00\x33\x33\x33\x33\x33\x33\x14\x40\x102\x00\xc2\x07\x00\x00\x00\x00")
    assert dbio.encode_document(doc) == raw
    assert dbio.decode_document(raw) == doc


def test_bson_round_trip_of_every_supported_type():
    g = uuid.UUID("00112233-4455-6677-8899-aabbccddeeff")
    doc = {"d": -1.5, "s": "x", "o": {"a": 1}, "a": [1, 2], "b": dbio.Binary(b"\x01\x02", 0),
           "g": g, "t": True, "f": False, "n": None, "i": 7, "l": dbio.Int64(2 ** 40)}
    back = dbio.decode_document(dbio.encode_document(doc))
    assert back == doc
    assert isinstance(back["l"], dbio.Int64) and not isinstance(back["i"], dbio.Int64)
    with pytest.raises(ValueError):
        dbio.decode_document(dbio.encode_document(doc)[:-1])


def test_guid_bytes_follow_dotnet_to_byte_array():
    # Guid.ToByteArray: the first three groups little-endian, the last two as written
    g = uuid.UUID("00112233-4455-6677-8899-aabbccddeeff")
    el = dbio.encode_document({"m_Guid": g})
    assert el[4:4 + 1 + 7 + 5] == b"\x05m_Guid\x00\x10\x00\x00\x00\x04"
    assert el[17:33] == bytes.fromhex("33221100554477668899aabbccddeeff")


def test_cell_field_data_set_layout():
    c = dbio.CellFieldDataSet(42)
    assert c.NoOfFields == 0
    a, b = np.array([1.0, 2.0, 3.0]), np.array([-4.0])
    c.AppendDGCoordinates(a)
    c.AppendDGCoordinates(b)
    assert c.NoOfFields == 2
    assert c.DGData == struct.pack("<3i", 2, 3, 1) + struct.pack("<4d", 1, 2, 3, -4)
    assert np.array_equal(c.GetDGCoordinates(0), a) and np.array_equal(c.GetDGCoordinates(1), b)
    with pytest.raises(IndexError):
        c.GetDGCoordinates(2)


def test_repartition_rule():
    thr = dbio.SPLIT_UP_THRESHOLD
    assert dbio.repartition(1000, 100) == [(0, 1000)]
    n = 3 * thr // 100 + 7
    parts = dbio.repartition(n, 100)
    assert len(parts) == 4 and parts[0][0] == 0 and parts[-1][1] == n
    assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
    # the byte total is a 32-bit product: past 2^31 it wraps negative -> one part
    assert dbio.repartition(2 ** 22, 2 ** 10) == [(0, 2 ** 22)]


def _fields(grid, degrees=(2, 1), names=("rho", "u")):
    return [O.DGField(grid, k, n) for k, n in zip(degrees, names)]


def _grid3(order=C.CELLS_GENERATOR):
    return O.Cartesian3DGrid(np.linspace(0, 1, 4), np.linspace(0, 2, 3), np.linspace(0, 1, 6),
                             cell_order=order)


def test_save_writes_the_reference_part_layout(tmp_path):
    g = _grid3()
    fs = _fields(g)
    per = sum(f.Np for f in fs)
    x = np.random.default_rng(1).standard_normal(g.NoOfCells * per)
    vid = dbio.SaveFieldData(str(tmp_path), fs, x)
    files = sorted(os.listdir(tmp_path / "data"))
    assert files == ["%s.1.data" % vid]
    doc = dbio.decode_document(gzip.decompress((tmp_path / "data" / files[0]).read_bytes()))
    assert list(doc) == ["Item1", "Item2"]
    assert list(doc["Item1"]) == ["m_Guid", "Partitioning", "UseGzip"]
    assert doc["Item1"]["m_Guid"] == vid and doc["Item1"]["UseGzip"] is True
    assert doc["Item1"]["Partitioning"] == [0, g.NoOfCells]
    assert doc["Item2"]["$type"] == dbio.CELL_FIELD_DATA_SET_ARRAY
    items = doc["Item2"]["$values"]
    assert list(items[0]) == ["GlobalID", "DGData"]
    # items in local order, GlobalID = ix + iy*nX + iz*nX*nY (Grid3D.cs:248)
    ijk = g.cell_ijk()
    for j in (0, 1, 7, g.NoOfCells - 1):
        ix, iy, iz = ijk[j]
        assert items[j]["GlobalID"] == ix + 3 * iy + 3 * 2 * iz
        c = dbio.CellFieldDataSet(items[j]["GlobalID"], items[j]["DGData"])
        assert c.NoOfFields == 2
        row = x.reshape(g.NoOfCells, per)[j]
        assert np.array_equal(np.concatenate([c.GetDGCoordinates(0), c.GetDGCoordinates(1)]), row)


def test_2d_global_ids_are_the_generator_order():
    g = O.Cartesian2DGrid(np.linspace(0, 1, 4), np.linspace(0, 1, 6))
    assert np.array_equal(g.global_ids(), np.arange(g.NoOfCells))   # Grid2D.cs:182
    g2 = O.Cartesian2DGrid(np.linspace(0, 1, 4), np.linspace(0, 1, 6), cell_order=C.CELLS_GLOBALID)
    assert np.array_equal(g2.cell_ijk(), g.cell_ijk())


def test_load_resorts_by_global_id_and_adapts_degrees(tmp_path, capsys):
    g = _grid3()
    fs = _fields(g)
    per = sum(f.Np for f in fs)
    x = np.random.default_rng(2).standard_normal(g.NoOfCells * per)
    vid = dbio.SaveFieldData(tmp_path, fs, x)
    # the same fields on a grid numbered in GlobalID order: values follow the cells
    g2 = _grid3(C.CELLS_GLOBALID)
    y = dbio.LoadFieldData(tmp_path, vid, _fields(g2), ["rho", "u"])
    a = x.reshape(g.NoOfCells, per)
    b = y.reshape(g2.NoOfCells, per)
    pos = {tuple(t): j for j, t in enumerate(g.cell_ijk())}
    for j2, t in enumerate(g2.cell_ijk()):
        assert np.array_equal(b[j2], a[pos[tuple(t)]])
    # degree up (zero padding), degree down (cut), a field that was not stored (zeros)
    fs3 = [O.DGField(g, 3, "u"), O.DGField(g, 1, "rho"), O.DGField(g, 1, "p")]
    z = dbio.LoadFieldData(tmp_path, vid, fs3, ["rho", "u"]).reshape(g.NoOfCells, -1)
    np1, np2 = fs[0].Np, fs[1].Np
    assert np.array_equal(z[:, :np2], a[:, np1:np1 + np2]) and not z[:, np2:20].any()
    assert np.array_equal(z[:, 20:24], a[:, :4])
    assert not z[:, 24:].any()
    assert "Unable to load field 'p'; initializing with zeros." in capsys.readouterr().err


def test_split_parts_and_partial_loads(tmp_path, monkeypatch):
    g = _grid3()
    fs = _fields(g)
    per = sum(f.Np for f in fs)
    x = np.random.default_rng(3).standard_normal(g.NoOfCells * per)
    items = dbio.cell_data_sets(fs, x, g.global_ids())
    size = dbio.item_size(items)
    monkeypatch.setattr(dbio, "SPLIT_UP_THRESHOLD", 3 * size)   # 30 cells -> 10 parts
    db = dbio.DatabaseDriver(tmp_path)
    vid = db.SaveVector(items)
    files = sorted(os.listdir(tmp_path / "data"), key=lambda s: int(s.split(".")[1]))
    assert len(files) == 10 and files[0] == "%s.1.data" % vid
    hdr = db.LoadHeader(vid)
    assert hdr["Partitioning"] == [0] + [3 * (p + 1) for p in range(10)]
    second = dbio.decode_document(gzip.decompress((tmp_path / "data" / files[1]).read_bytes()))
    assert "Item1" not in second                     # header in part 0 only
    assert db.LoadVector(vid) == items
    for i0, n in ((0, 0), (5, 1), (4, 20), (27, 3)):
        with pytest.raises(ValueError):              # one process must load all of it
            db.LoadVector(vid, (i0, n))
    # a rank's slice crossing parts (the check on the total uses every rank's length)
    monkeypatch.setattr(dbio, "_allgather", lambda obj, group: [obj, 30 - obj]
                        if isinstance(obj, int) else [obj])
    assert db.LoadVector(vid, (4, 20)) == items[4:24]
    assert db.LoadVector(vid, (27, 3)) == items[27:30]
    y = dbio.LoadFieldData(db, vid, fs, ["rho", "u"])
    assert np.array_equal(y, x)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _x_global(g, per):
    return np.random.default_rng(4).standard_normal(g.NoOfCells * per)


def _rank_main(rank, world, port, path, vid, q):
    import torch.distributed as dist
    from datetime import timedelta
    from bosss_b200.distributed import SlabPartition
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        g = _grid3()
        fs = _fields(g)
        per = sum(f.Np for f in fs)
        x = _x_global(g, per)
        part = SlabPartition(g, world, rank, per)
        own = x[part.global_slice()]
        if vid is None:       # save this rank's slab, then load it back
            vid = dbio.SaveFieldData(path, fs, own, part=part)
        y = dbio.LoadFieldData(path, vid, fs, ["rho", "u"], part=part)
        q.put((rank, str(vid), bool(np.array_equal(y, own))))
    finally:
        dist.destroy_process_group()


def _spawn(world, path, vid):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, path, vid, q)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        out = sorted(q.get(timeout=240) for _ in range(world))
    finally:
        for p in procs:
            p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    return out


def test_several_ranks_save_and_load_over_gloo(tmp_path):
    out = _spawn(2, str(tmp_path), None)
    vids = {v for _, v, _ in out}
    assert len(vids) == 1 and all(ok for _, _, ok in out)
    vid = vids.pop()
    # the two ranks' parts form one vector: a single process reads all of it
    g = _grid3()
    fs = _fields(g)
    per = sum(f.Np for f in fs)
    hdr = dbio.DatabaseDriver(tmp_path).LoadHeader(vid)
    assert hdr["Partitioning"] == [0, 20, 30]     # x-planes of 10 cells: 2 + 1
    assert np.array_equal(dbio.LoadFieldData(tmp_path, vid, fs, ["rho", "u"]), _x_global(g, per))
    # three ranks read the vector two ranks wrote (slices cross the stored parts)
    out3 = _spawn(3, str(tmp_path), vid)
    assert all(ok for _, _, ok in out3)


def test_2d_round_trip(tmp_path):
    g = O.Cartesian2DGrid(np.linspace(0, 1, 5), np.linspace(0, 1, 4))
    fs = [O.DGField(g, 3, "T")]
    x = np.random.default_rng(6).standard_normal(g.NoOfCells * fs[0].Np)
    vid = dbio.SaveFieldData(tmp_path, fs, x)
    items = dbio.DatabaseDriver(tmp_path).LoadVector(vid)
    assert [it.GlobalID for it in items] == list(range(g.NoOfCells))   # ix*nY + iy
    assert np.array_equal(dbio.LoadFieldData(tmp_path, vid, fs, ["T"]), x)
