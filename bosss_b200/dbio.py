"""DG vector on-disk format of the BoSSS database: save and load the DG coordinates of a
time step in the files the reference writes and reads.

The reference stores the DG coordinates of a time step as one distributed vector of
``CellFieldDataSet`` items, one per cell (``DatabaseDriver_TimeStep.cs:92-114``):

* item ``j`` carries the cell's ``GlobalID`` and a byte buffer ``DGData`` holding the int32
  number of fields ``Q``, the Q int32 coordinate counts, then the doubles of every field's
  coordinates back to back (``CellFieldDataSet.cs:38-80``; little-endian, as the reference
  writes through raw pointers on x86);
* the vector is cut into parts of at most 64 MiB of serialised items
  (``DatabaseDriver_VectorData.cs:80-121``) and part ``p`` goes to
  ``<db>/data/<guid>.<p+1>.data`` (``StandardFsDriver.cs:357-361``);
* every part is a gzip stream of one BSON document, the serialisation of
  ``Tuple<DistributedVectorHeader, IList<T>>`` (``DatabaseDriver_VectorData.cs:168-196``):
  ``Item1`` is the header (vector GUID, part partitioning, ``UseGzip``) in part 0 only and is
  left out of the others (null values are ignored, ``DatabaseDriver_Serializer.cs:116-120``);
  ``Item2`` is the part's items, written with their array type name because the declared
  type is an interface (``TypeNameHandling.Auto``).

Loading reads the header from part 0, takes the rank's slice of the stored vector
(``DatabaseDriver_VectorData.cs:221-304``), sorts the items by GlobalID into the local cell
order (``DatabaseDriver_TimeStep.cs:262-307``) and copies every field's coordinates, cut or
zero-padded to the field's degree (``DGField.cs:1186-1203``).

The BSON subset (double, string, document, array, binary, bool, null, int32, int64) is
written here from the BSON 1.1 specification. GUIDs are BSON binary subtype 4 holding the
16 bytes of ``Guid.ToByteArray()`` (``uuid.UUID.bytes_le``).

This is host-side IO around the device path: a device coordinate vector crosses PCIe once
each way (one device-to-host copy before a save, one host-to-device copy after a load).
"""
import gzip
import io
import os
import struct
import sys
import uuid

import numpy as np

from .operator import CoordinateVector, DGField

DIST_VECTOR_DATA_DIR = "data"                 # StandardFsDriver.DistVectorDataDir
SPLIT_UP_THRESHOLD = 64 * 1024 * 1024         # DatabaseDriver_VectorData.RepartitionVector
CELL_FIELD_DATA_SET_ARRAY = "BoSSS.Foundation.IO.CellFieldDataSet[], BoSSS.Foundation"


# ----------------------------------------------------------------------------- BSON

class Int64(int):
    """An integer written as BSON int64 (C# ``long``)."""


class Binary(bytes):
    """Bytes written as BSON binary with a given subtype (0: generic, C# ``byte[]``)."""

    def __new__(cls, data, subtype=0):
        o = super().__new__(cls, data)
        o.subtype = int(subtype)
        return o


def _cstring(s):
    b = s.encode("utf-8")
    if b"\x00" in b:
        raise ValueError("BSON keys cannot contain NUL")
    return b + b"\x00"


def _element(key, v):
    k = _cstring(key)
    if isinstance(v, bool):
        return b"\x08" + k + (b"\x01" if v else b"\x00")
    if isinstance(v, Int64):
        return b"\x12" + k + struct.pack("<q", int(v))
    if isinstance(v, (int, np.integer)):
        v = int(v)
        if -2 ** 31 <= v < 2 ** 31:
            return b"\x10" + k + struct.pack("<i", v)
        return b"\x12" + k + struct.pack("<q", v)
    if isinstance(v, (float, np.floating)):
        return b"\x01" + k + struct.pack("<d", float(v))
    if isinstance(v, str):
        b = v.encode("utf-8") + b"\x00"
        return b"\x02" + k + struct.pack("<i", len(b)) + b
    if isinstance(v, uuid.UUID):
        return b"\x05" + k + struct.pack("<iB", 16, 4) + v.bytes_le
    if isinstance(v, (bytes, bytearray, memoryview)):
        sub = getattr(v, "subtype", 0)
        v = bytes(v)
        return b"\x05" + k + struct.pack("<iB", len(v), sub) + v
    if isinstance(v, dict):
        return b"\x03" + k + encode_document(v)
    if isinstance(v, (list, tuple)):
        return b"\x04" + k + encode_document({str(i): x for i, x in enumerate(v)})
    if v is None:
        return b"\x0a" + k
    raise TypeError("no BSON encoding for %r" % type(v))


def encode_document(doc):
    """BSON bytes of a mapping (insertion order kept). ``None`` values are written as
    BSON null; drop them first where the writer ignores nulls."""
    body = b"".join(_element(k, v) for k, v in doc.items())
    return struct.pack("<i", len(body) + 5) + body + b"\x00"


def _read_cstring(buf, o):
    e = buf.index(b"\x00", o)
    return buf[o:e].decode("utf-8"), e + 1


def _decode_at(buf, o, as_array=False):
    n = struct.unpack_from("<i", buf, o)[0]
    end = o + n
    if n < 5 or end > len(buf) or buf[end - 1] != 0:
        raise ValueError("malformed BSON document at offset %d" % o)
    o += 4
    out = {}
    while o < end - 1:
        t = buf[o]
        key, o = _read_cstring(buf, o + 1)
        if t == 0x01:
            v = struct.unpack_from("<d", buf, o)[0]; o += 8
        elif t == 0x02:
            ln = struct.unpack_from("<i", buf, o)[0]
            v = buf[o + 4:o + 4 + ln - 1].decode("utf-8"); o += 4 + ln
        elif t in (0x03, 0x04):
            v, o = _decode_at(buf, o, t == 0x04)
        elif t == 0x05:
            ln, sub = struct.unpack_from("<iB", buf, o)
            raw = bytes(buf[o + 5:o + 5 + ln]); o += 5 + ln
            v = uuid.UUID(bytes_le=raw) if sub in (3, 4) and ln == 16 else Binary(raw, sub)
        elif t == 0x07:
            v = bytes(buf[o:o + 12]); o += 12
        elif t == 0x08:
            v = buf[o] != 0; o += 1
        elif t == 0x09:
            v = Int64(struct.unpack_from("<q", buf, o)[0]); o += 8
        elif t == 0x0a:
            v = None
        elif t == 0x10:
            v = struct.unpack_from("<i", buf, o)[0]; o += 4
        elif t == 0x12:
            v = Int64(struct.unpack_from("<q", buf, o)[0]); o += 8
        else:
            raise ValueError("unsupported BSON element type 0x%02x (key %r)" % (t, key))
        out[key] = v
    if o != end - 1:
        raise ValueError("BSON document overruns its length")
    if as_array:
        return [out[str(i)] for i in range(len(out))], end
    return out, end


def decode_document(buf):
    """Mapping of one BSON document (arrays as lists, int64 as :class:`Int64`, subtype-3/4
    binaries of 16 bytes as ``uuid.UUID``, other binaries as :class:`Binary`)."""
    buf = memoryview(buf).cast("B") if not isinstance(buf, (bytes, bytearray)) else buf
    doc, end = _decode_at(bytes(buf), 0)
    if end != len(buf):
        raise ValueError("trailing bytes after the BSON document")
    return doc


# ----------------------------------------------------------------------------- CellFieldDataSet

class CellFieldDataSet:
    """DG coordinates of several fields in one cell (``CellFieldDataSet.cs:29-130``):
    ``DGData`` = int32 Q, Q int32 coordinate counts, then the doubles of every field."""

    __slots__ = ("GlobalID", "DGData")

    def __init__(self, GlobalID=0, DGData=None):
        self.GlobalID = int(GlobalID)
        self.DGData = None if DGData is None else bytes(DGData)

    @property
    def NoOfFields(self):
        if not self.DGData:
            return 0
        return struct.unpack_from("<i", self.DGData, 0)[0]

    def AppendDGCoordinates(self, coords):
        """Append one field's coordinates (``CellFieldDataSet.cs:50-80``)."""
        c = np.ascontiguousarray(coords, dtype="<f8")
        q = self.NoOfFields
        counts = list(struct.unpack_from("<%di" % q, self.DGData, 4)) if q else []
        old = self.DGData[4 * (q + 1):] if q else b""
        self.DGData = struct.pack("<%di" % (q + 2), q + 1, *counts, c.size) + old + c.tobytes()

    def GetDGCoordinates(self, ifld):
        """Coordinates of field ``ifld`` (``CellFieldDataSet.cs:103-130``)."""
        q = self.NoOfFields
        if not 0 <= ifld < q:
            raise IndexError("field index %d out of range (%d fields)" % (ifld, q))
        counts = struct.unpack_from("<%di" % q, self.DGData, 4)
        off = 4 * (q + 1) + 8 * sum(counts[:ifld])
        return np.frombuffer(self.DGData, dtype="<f8", count=counts[ifld], offset=off).copy()

    def to_bson_fields(self):
        d = {"GlobalID": Int64(self.GlobalID)}
        if self.DGData is not None:           # null values are not written
            d["DGData"] = Binary(self.DGData, 0)
        return d

    def __eq__(self, other):
        return (isinstance(other, CellFieldDataSet) and self.GlobalID == other.GlobalID
                and self.DGData == other.DGData)

    def __repr__(self):
        return "CellFieldDataSet(GlobalID=%d, fields=%d)" % (self.GlobalID, self.NoOfFields)


def _items_array_bytes(items):
    """BSON array document of CellFieldDataSet items, assembled without per-element dicts."""
    parts = []
    for i, it in enumerate(items):
        key = str(i).encode() + b"\x00"
        body = b"\x12GlobalID\x00" + struct.pack("<q", it.GlobalID)
        if it.DGData is not None:
            body += b"\x05DGData\x00" + struct.pack("<iB", len(it.DGData), 0) + it.DGData
        parts.append(b"\x03" + key + struct.pack("<i", len(body) + 5) + body + b"\x00")
    body = b"".join(parts)
    return struct.pack("<i", len(body) + 5) + body + b"\x00"


def _typed_array_doc(items):
    """``{"$type": "...CellFieldDataSet[], ...", "$values": [...]}``: the form the writer
    uses for an array whose declared type is ``IList<T>`` (or ``T``, in the size probe)."""
    t = CELL_FIELD_DATA_SET_ARRAY.encode() + b"\x00"
    inner = (b"\x02$type\x00" + struct.pack("<i", len(t)) + t
             + b"\x04$values\x00" + _items_array_bytes(items))
    return struct.pack("<i", len(inner) + 5) + inner + b"\x00"


def _typed_array_bytes(key, items):
    return b"\x03" + _cstring(key) + _typed_array_doc(items)


def _part_document(header, items):
    body = b""
    if header is not None:
        body += _element("Item1", header)
    body += _typed_array_bytes("Item2", items)
    return struct.pack("<i", len(body) + 5) + body + b"\x00"


def _items_from_bson(v):
    if isinstance(v, dict) and "$values" in v:
        v = v["$values"]
    if not isinstance(v, list):
        raise ValueError("vector part holds no item list")
    out = []
    for d in v:
        if isinstance(d, dict) and "$type" in d:
            d = {k: x for k, x in d.items() if k != "$type"}
        dg = d.get("DGData")
        out.append(CellFieldDataSet(d.get("GlobalID", 0), None if dg is None else bytes(dg)))
    return out


def item_size(items):
    """Average serialised size of the first (at most 10) items, rounded half to even
    (``DatabaseDriver_VectorData.cs:80-92``)."""
    n = min(10, len(items))
    if n == 0:
        return 0
    return int(round(len(_typed_array_doc(items[:n])) / n))


def repartition(n_items, itm_size):
    """Bounds of the parts a rank's vector is cut into (``DatabaseDriver_VectorData.cs:
    99-121``). The byte total is the reference's 32-bit product, wrapped as it is."""
    tot = (n_items * itm_size + 2 ** 31) % 2 ** 32 - 2 ** 31
    if tot < SPLIT_UP_THRESHOLD:
        return [(0, n_items)]
    nparts = -(-tot // SPLIT_UP_THRESHOLD)
    return [((n_items * p) // nparts, (n_items * (p + 1)) // nparts) for p in range(nparts)]


# ----------------------------------------------------------------------------- ranks

def _rank_size(group):
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(group), dist.get_world_size(group)
    return 0, 1


def _allgather(obj, group):
    """Every rank's ``obj`` in rank order (``MPIAllGather`` / ``MPIAllGatherv``)."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size(group) == 1:
        return [obj]
    out = [None] * dist.get_world_size(group)
    dist.all_gather_object(out, obj, group=group)
    return out


def _barrier(group):
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.barrier(group=group)


# ----------------------------------------------------------------------------- vectors

class DatabaseDriver:
    """Vector IO of a BoSSS database directory (``DatabaseDriver.cs:232-259``).

    ``group`` is a ``torch.distributed`` process group (default: the world group when one
    is initialised, else a single process); every rank passes its own slice of the vector,
    as every MPI process does in the reference.
    """

    def __init__(self, path, group=None):
        self.path = os.fspath(path)
        self.group = group

    def _part_file(self, vid, part):
        return os.path.join(self.path, DIST_VECTOR_DATA_DIR, "%s.%d.data" % (vid, part + 1))

    # -- SaveVector (DatabaseDriver_VectorData.cs:64-72, 136-211)
    def SaveVector(self, vector, id=None):
        """Save this rank's slice of a vector of :class:`CellFieldDataSet`; returns the
        vector's GUID (a new one, broadcast from rank 0, unless ``id`` is given; ``id`` must
        be the same on every rank)."""
        rank, size = _rank_size(self.group)
        if id is None:
            id = _allgather(uuid.uuid4(), self.group)[0]
        id = uuid.UUID(str(id))
        if len(set(str(g) for g in _allgather(id, self.group))) != 1:
            raise ValueError("Guid differs at least on one process")
        vector = list(vector)
        bounds = repartition(len(vector), item_size(vector))
        parts_per_rank = _allgather(len(bounds), self.group)
        lengths = [ln for r in _allgather([b - a for a, b in bounds], self.group) for ln in r]
        my_first = sum(parts_per_rank[:rank])
        os.makedirs(os.path.join(self.path, DIST_VECTOR_DATA_DIR), exist_ok=True)
        for ip, (a, b) in enumerate(bounds):
            header = None
            if rank == 0 and ip == 0:
                offsets = np.concatenate([[0], np.cumsum(lengths, dtype=np.int64)])
                header = {"m_Guid": id, "Partitioning": [Int64(x) for x in offsets],
                          "UseGzip": True}
            doc = _part_document(header, vector[a:b])
            with open(self._part_file(id, my_first + ip), "wb") as f:
                f.write(gzip.compress(doc, mtime=0))
        _barrier(self.group)
        return id

    def _read_part(self, vid, part):
        with open(self._part_file(vid, part), "rb") as f:
            doc = decode_document(gzip.decompress(f.read()))
        return doc.get("Item1"), doc.get("Item2")

    def LoadHeader(self, id):
        """Header of a stored vector (GUID, partitioning, gzip flag), from part 0."""
        header, _ = self._read_part(uuid.UUID(str(id)), 0)
        if not header or "Partitioning" not in header:
            raise IOError("vector %s: part 0 carries no header" % id)
        return header

    # -- LoadVector (DatabaseDriver_VectorData.cs:221-304)
    def LoadVector(self, id, part=None):
        """This rank's slice of a stored vector: ``part`` = (first index, length); by default
        the even split ``[L*rank/size, L*(rank+1)/size)`` of the stored length L."""
        rank, size = _rank_size(self.group)
        vid = uuid.UUID(str(id))
        hdr = self.LoadHeader(vid) if rank == 0 else None
        hdr = _allgather(hdr, self.group)[0]
        offsets = [int(x) for x in hdr["Partitioning"]]
        L = offsets[-1]
        if part is None:
            i0 = (L * rank) // size
            part = (i0, (L * (rank + 1)) // size - i0)
        i0, n = int(part[0]), int(part[1])
        total = sum(_allgather(n, self.group))
        if total != L:
            raise ValueError("IO error: length of vector to load differs from total length of list.")
        out = []
        if n == 0:
            return out
        p = 0
        while offsets[p] <= i0:
            p += 1
        p -= 1
        d = 0
        while d < n:
            _, items = self._read_part(vid, p)
            items = _items_from_bson(items)
            src = i0 + d - offsets[p]
            take = min(len(items) - src, n - d)
            out.extend(items[src:src + take])
            d += take
            p += 1
        return out


# ----------------------------------------------------------------------------- DG fields

def _host_rows(coords, n_cells, per_cell):
    """(n_cells, per_cell) float64 host array of a coordinate vector (numpy, torch on any
    device -- one device-to-host copy -- or :class:`CoordinateVector`)."""
    if isinstance(coords, CoordinateVector):
        coords = coords.data
    if hasattr(coords, "detach"):
        coords = coords.detach().to("cpu").numpy()
    a = np.ascontiguousarray(np.asarray(coords, dtype=np.float64))
    if a.size != n_cells * per_cell:
        raise ValueError("coordinate vector has %d entries, expected %d cells x %d"
                         % (a.size, n_cells, per_cell))
    return a.reshape(n_cells, per_cell)


def _local_cells(grid, part):
    """GlobalIDs of this rank's cells in local order and the rank's first index in the
    cell partitioning (ranks own consecutive ranges, ``grdDat.CellPartitioning``)."""
    gids = grid.global_ids()
    if part is None:
        return gids, 0
    a = part.first * part.plane_cells
    return gids[a:a + part.count * part.plane_cells], a


def cell_data_sets(fields, coords, global_ids):
    """One :class:`CellFieldDataSet` per cell, fields in the given order
    (``DatabaseDriver_TimeStep.cs:92-110``)."""
    nps = [f.Np for f in fields]
    rows = _host_rows(coords, len(global_ids), sum(nps))
    head = struct.pack("<%di" % (len(nps) + 1), len(nps), *nps)
    data = rows.astype("<f8", copy=False)
    return [CellFieldDataSet(g, head + data[j].tobytes()) for j, g in enumerate(global_ids)]


def SaveFieldData(db, fields, coords, id=None, part=None):
    """Save the DG coordinates of ``fields`` (one grid; the coordinate vector in the
    cell-major layout, host or device) as the time-step vector of the reference; returns
    its GUID (``TimestepInfo.StorageID``). With a :class:`~bosss_b200.distributed.
    SlabPartition` every rank passes its owned coordinates."""
    if isinstance(db, (str, os.PathLike)):
        db = DatabaseDriver(db)
    grid = fields[0].grid
    if any(f.grid is not grid for f in fields):
        raise ValueError("mismatch in GridData object.")
    gids, _ = _local_cells(grid, part)
    return db.SaveVector(cell_data_sets(fields, coords, gids), id)


def LoadFieldData(db, id, fields, stored_fields, part=None, device=None):
    """Load a stored time-step vector into ``fields`` (``DatabaseDriver_TimeStep.cs:
    262-307``). ``stored_fields`` names the stored fields in their stored order (the time
    step's field initialisers); a field not among them is set to zero with the reference's
    message. Coordinates are cut or zero-padded to each field's degree. Returns the
    cell-major coordinate vector of ``fields`` (numpy, or a torch tensor on ``device`` --
    one host-to-device copy)."""
    if isinstance(db, (str, os.PathLike)):
        db = DatabaseDriver(db)
    grid = fields[0].grid
    gids, i0 = _local_cells(grid, part)
    J = len(gids)
    items = db.LoadVector(id, (i0, J))
    # resort by GlobalID: the loaded slice may hold other ranks' cells, so every rank's slice
    # is gathered on every rank (host memory of the whole vector per rank; the reference
    # exchanges only the permuted items)
    pairs = [(it.GlobalID, it.DGData) for it in items]
    everything = _allgather(pairs, db.group)
    where = {int(g): j for j, g in enumerate(gids)}
    mine = [None] * J
    for chunk in everything:
        for g, blob in chunk:
            j = where.get(int(g))
            if j is not None:
                mine[j] = blob
    missing = sum(b is None for b in mine)
    if missing:
        raise IOError("vector %s holds no data for %d local cells" % (id, missing))
    nps = [f.Np for f in fields]
    offs = np.concatenate([[0], np.cumsum(nps)])
    out = np.zeros((J, int(offs[-1])))
    stored = list(stored_fields)
    src = []
    for f in fields:
        if f.name in stored:
            src.append(stored.index(f.name))
        else:
            print("Unable to load field '%s'; initializing with zeros." % f.name, file=sys.stderr)
            src.append(-1)
    uniform = len({len(b) if b is not None else -1 for b in mine}) == 1 and mine[0] is not None
    if uniform and len(set(b[:4 * (1 + struct.unpack_from("<i", b, 0)[0])] for b in mine)) == 1:
        # every cell has the same field sizes: one strided view of all the doubles
        q = struct.unpack_from("<i", mine[0], 0)[0]
        counts = struct.unpack_from("<%di" % q, mine[0], 4)
        hb = 4 * (q + 1)
        blob = np.frombuffer(b"".join(mine), dtype=np.uint8).reshape(J, -1)[:, hb:]
        vals = np.ascontiguousarray(blob).view("<f8").reshape(J, -1)
        coff = np.concatenate([[0], np.cumsum(counts)])
        for fi, s in enumerate(src):
            if s < 0:
                continue
            if s >= q:
                raise IndexError("stored field %d out of range (%d fields)" % (s, q))
            n = min(counts[s], nps[fi])
            out[:, offs[fi]:offs[fi] + n] = vals[:, coff[s]:coff[s] + n]
    else:
        for j, b in enumerate(mine):
            cell = CellFieldDataSet(0, b)
            for fi, s in enumerate(src):
                if s < 0:
                    continue
                c = cell.GetDGCoordinates(s)
                n = min(c.size, nps[fi])
                out[j, offs[fi]:offs[fi] + n] = c[:n]
    out = out.reshape(-1)
    if device is not None:
        import torch
        return torch.from_numpy(out).to(device)
    return out
