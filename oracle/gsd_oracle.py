"""GSD file-layer oracle (test infrastructure only; nothing in the package imports it).

An independent restatement, with Python's ``struct`` and numpy, of the GSD 2.0 file layer that the
reference's snapshot I/O drives through GSDFiles.jl (a third-party package pinned as
GSDFiles = "0.1, 0.2" in Project.toml:16; it is not in the reference's sources).  The layout
follows the published GSD 2.0 specification and the parts of it the reference itself spells out:

- the 256-byte header read field by field in src/io/GSDIO.jl:110-135 (magic, index location and
  allocated entries, name-block location and allocated bytes, schema and file-layer versions,
  64-byte application and schema names, 80 reserved bytes);
- the name block rebuilt in GSDIO.jl:145-149 (the names, each followed by a zero byte);
- the index-entry fields used by src/io/RestartIO.jl:41-52 and test/test_io_gsd.jl:117-130
  (frame, N, location, M, id, type), in the specification's 32-byte packing
  (uint64, uint64, int64, uint32, uint16, uint8, uint8);
- the type codes of RestartIO.jl:27-39; data stored row-major (RestartIO.jl:50-51: an N x M chunk
  is read as M*N values and reshaped (M, N)').

Parity is pinned by the reference's own GSD tests as far as they go (frame contents, append,
type codes of the virial chunks) and by the specification for the byte layout; no GSD file
written by the reference exists in its repository, so byte-level parity with GSDFiles.jl itself
is unpinned.

The writer here deliberately places blocks differently from libpdb200's writer (data first, the
index and name blocks at the end, sized exactly), so a reader that follows the header's pointers
reads both files and one that assumes a fixed layout does not.
"""
from __future__ import annotations

import struct

import numpy as np

MAGIC = 0x65DF65DF65DF65DF
HEADER = struct.Struct("<QQQQQII64s64s80s")
ENTRY = struct.Struct("<QQqIHBB")
assert HEADER.size == 256 and ENTRY.size == 32

TYPES = {1: np.uint8, 2: np.uint16, 3: np.uint32, 4: np.uint64, 5: np.int8, 6: np.int16, 7: np.int32, 8: np.int64,
         9: np.float32, 10: np.float64, 11: np.uint8}
CODES = {np.dtype(v): k for k, v in TYPES.items() if k != 11}


def version(major: int, minor: int) -> int:
    return (major << 16) | minor


def write(path, frames, application="oracle", schema="hoomd", schema_version=(1, 4), gsd_version=(2, 0),
          spare_entries=3):
    """Write ``frames`` (a list of {name: array}) as a GSD 2.0 file: chunk data first, then the index
    (sorted by frame, then by name id, plus ``spare_entries`` zero entries) and the name block."""
    names, ids = [], {}
    blobs, entries = [], []
    pos = HEADER.size
    for f, chunks in enumerate(frames):
        rows = []
        for name, arr in chunks.items():
            a = np.ascontiguousarray(arr)
            if a.ndim == 0:
                a = a.reshape(1)
            code = CODES[a.dtype]
            if name not in ids:
                ids[name] = len(names)
                names.append(name)
            n = a.shape[0]
            m = 1 if a.ndim == 1 else a.shape[1]
            rows.append((f, n, pos, m, ids[name], code, 0))
            blobs.append(a.tobytes())
            pos += a.nbytes
        entries.extend(sorted(rows, key=lambda e: e[4]))
    index_location = pos
    nalloc = len(entries) + spare_entries
    index = b"".join(ENTRY.pack(*e) for e in entries) + bytes(ENTRY.size * spare_entries)
    pos += len(index)
    name_block = b"".join(n.encode() + b"\0" for n in names) + b"\0"
    namelist_location = pos
    header = HEADER.pack(MAGIC, index_location, nalloc, namelist_location, len(name_block),
                         version(*schema_version), version(*gsd_version), application.encode(), schema.encode(),
                         bytes(80))
    with open(path, "wb") as fh:
        fh.write(header)
        for b in blobs:
            fh.write(b)
        fh.write(index)
        fh.write(name_block)


class Reader:
    """Reads a GSD 2.0 file from its bytes: header, names, used index entries, chunks."""

    def __init__(self, path):
        with open(path, "rb") as fh:
            self.raw = fh.read()
        h = HEADER.unpack_from(self.raw, 0)
        if h[0] != MAGIC:
            raise ValueError("invalid GSD magic")
        self.header = dict(index_location=h[1], index_allocated_entries=h[2], namelist_location=h[3],
                           namelist_allocated_entries=h[4], schema_version=(h[5] >> 16, h[5] & 0xFFFF),
                           gsd_version=(h[6] >> 16, h[6] & 0xFFFF),
                           application=h[7].split(b"\0", 1)[0].decode(), schema=h[8].split(b"\0", 1)[0].decode())
        blk = self.raw[h[3]:h[3] + h[4]]
        self.names = []
        o = 0
        while o < len(blk) and blk[o] != 0:
            end = blk.index(b"\0", o)
            self.names.append(blk[o:end].decode())
            o = end + 1
        self.index = []
        for k in range(h[2]):
            e = ENTRY.unpack_from(self.raw, h[1] + 32 * k)
            if e[2] == 0:
                break
            self.index.append(dict(frame=e[0], N=e[1], location=e[2], M=e[3], id=e[4], type=e[5], flags=e[6]))
        self.nframes = (self.index[-1]["frame"] + 1) if self.index else 0

    def entry(self, frame, name):
        if name not in self.names:
            return None
        cid = self.names.index(name)
        for e in self.index:
            if e["frame"] == frame and e["id"] == cid:
                return e
        return None

    def chunk(self, frame, name):
        e = self.entry(frame, name)
        if e is None:
            return None
        t = TYPES[e["type"]]
        a = np.frombuffer(self.raw, t, count=e["N"] * e["M"], offset=e["location"]).copy()
        return a if e["M"] == 1 else a.reshape(e["N"], e["M"])
