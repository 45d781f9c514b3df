"""ILDG gauge configurations in LIME files: read and write.

LIME, the USQCD record container, is a sequence of records.  Each record has
a 144-byte big-endian header -- magic 0x456789ab, format version 1, the
message-begin / message-end flags, the 64-bit data length and a 128-byte
NUL-padded type string -- followed by the data, padded to a multiple of 8
bytes.  An ILDG configuration holds:
  * an `ildg-format` record: XML with the field type, the precision (32 or 64
    bits) and the lattice extents lx, ly, lz, lt;
  * an `ildg-binary-data` record: the links as big-endian complex numbers in
    the order [t][z][y][x][mu][row][col] (python/PyQuda/pyquda/utils/gauge_utils.py:13-57
    reads the same record).
SciDAC writers add a `scidac-checksum` record (suma, sumb): for every site,
the CRC-32 of its bytes, rotated left by (lexicographic rank mod 29) resp.
(rank mod 31), XOR-ed over the lattice.  `read_ildg` verifies it when the file
has one; `write_ildg` writes one.

Gauge fields returned and accepted here are numpy complex128 arrays in
PyQuda's even-odd layout [mu][parity][t][z][y][x/2][3][3], the layout of the
library's gauge argument.  The links are returned as stored (no boundary
phase); the antiperiodic time boundary is the t_boundary argument of
qcu_b200.Gauge.
"""
from __future__ import annotations

import re
import struct
import zlib
from xml.etree import ElementTree as ET

import numpy as np

LIME_MAGIC = 0x456789AB
LIME_VERSION = 1
_HDR = struct.Struct(">IHHQ")


def read_lime(path):
    """All records of a LIME file: list of (type, data bytes, flags)."""
    recs = []
    with open(path, "rb") as f:
        while True:
            head = f.read(16)
            if not head:
                break
            if len(head) < 16:
                raise ValueError(f"{path}: truncated LIME header")
            magic, version, flags, length = _HDR.unpack(head)
            if magic != LIME_MAGIC or version != LIME_VERSION:
                raise ValueError(f"{path}: not a LIME file (magic {magic:#x}, version {version})")
            rtype = f.read(128).rstrip(b"\0").decode("utf-8")
            data = f.read(length)
            if len(data) != length:
                raise ValueError(f"{path}: record {rtype!r} is truncated")
            f.read((-length) % 8)  # padding
            recs.append((rtype, data, flags))
    return recs


def write_lime(path, records):
    """records: list of (type, data bytes); message begin/end flags set on
    the first/last record."""
    with open(path, "wb") as f:
        for i, (rtype, data) in enumerate(records):
            flags = (0x8000 if i == 0 else 0) | (0x4000 if i == len(records) - 1 else 0)
            f.write(_HDR.pack(LIME_MAGIC, LIME_VERSION, flags, len(data)))
            f.write(rtype.encode("utf-8").ljust(128, b"\0"))
            f.write(data)
            f.write(b"\0" * ((-len(data)) % 8))


def _rotl32(v, n):
    n %= 32
    return ((v << n) | (v >> (32 - n))) & 0xFFFFFFFF if n else v


def scidac_checksum(binary: bytes, site_bytes: int):
    """(suma, sumb) of a lexicographically ordered lattice of `site_bytes`-byte sites."""
    suma = sumb = 0
    nsite = len(binary) // site_bytes
    mv = memoryview(binary)
    for rank in range(nsite):
        crc = zlib.crc32(mv[rank * site_bytes:(rank + 1) * site_bytes]) & 0xFFFFFFFF
        suma ^= _rotl32(crc, rank % 29)
        sumb ^= _rotl32(crc, rank % 31)
    return suma, sumb


def _xml_values(xml: str, names):
    root = ET.fromstring(xml.strip("\0 \n"))
    out = {}
    for el in root.iter():
        tag = re.sub(r"^\{.*\}", "", el.tag)
        if tag in names and el.text is not None:
            out[tag] = el.text.strip()
    return out


def lexico_to_eo(lex, latt):
    """[t][z][y][x][mu][3][3] -> [mu][parity][t][z][y][x/2][3][3] (parity of x+y+z+t)."""
    Lx, Ly, Lz, Lt = latt
    g = np.moveaxis(lex, 4, 0)  # [mu][t][z][y][x][3][3]
    t, z, y, xh = np.meshgrid(np.arange(Lt), np.arange(Lz), np.arange(Ly), np.arange(Lx // 2), indexing="ij")
    out = np.empty((4, 2, Lt, Lz, Ly, Lx // 2, 3, 3), dtype=np.complex128)
    for p in (0, 1):
        x = 2 * xh + ((t + z + y + p) & 1)
        out[:, p] = g[:, t, z, y, x]
    return out


def eo_to_lexico(gauge, latt):
    """inverse of lexico_to_eo"""
    Lx, Ly, Lz, Lt = latt
    g = np.asarray(gauge).reshape(4, 2, Lt, Lz, Ly, Lx // 2, 3, 3)
    t, z, y, xh = np.meshgrid(np.arange(Lt), np.arange(Lz), np.arange(Ly), np.arange(Lx // 2), indexing="ij")
    lex = np.empty((4, Lt, Lz, Ly, Lx, 3, 3), dtype=g.dtype)
    for p in (0, 1):
        x = 2 * xh + ((t + z + y + p) & 1)
        lex[:, t, z, y, x] = g[:, p]
    return np.moveaxis(lex, 0, 4)  # [t][z][y][x][mu][3][3]


def read_ildg(path, verify: bool = True):
    """Returns (gauge [mu][parity][t][z][y][x/2][3][3] complex128, [Lx, Ly, Lz, Lt], info).
    verify: check the SciDAC checksum when the file carries one."""
    recs = {t: d for t, d, _ in read_lime(path)}
    if "ildg-format" not in recs or "ildg-binary-data" not in recs:
        raise ValueError(f"{path}: no ildg-format / ildg-binary-data records")
    fmt = _xml_values(recs["ildg-format"].decode("utf-8", "replace"), {"field", "precision", "lx", "ly", "lz", "lt"})
    latt = [int(fmt[k]) for k in ("lx", "ly", "lz", "lt")]
    prec = int(fmt["precision"])
    if prec not in (32, 64):
        raise ValueError(f"{path}: unsupported precision {prec}")
    if latt[0] % 2:
        raise ValueError(f"{path}: Lx must be even for the even-odd layout")
    binary = recs["ildg-binary-data"]
    vol = latt[0] * latt[1] * latt[2] * latt[3]
    site_bytes = 4 * 9 * 2 * prec // 8
    if len(binary) != vol * site_bytes:
        raise ValueError(f"{path}: binary record holds {len(binary)} bytes, expected {vol * site_bytes}")
    info = {"field": fmt.get("field"), "precision": prec, "checksum": None}
    if verify and "scidac-checksum" in recs:
        ck = _xml_values(recs["scidac-checksum"].decode("utf-8", "replace"), {"suma", "sumb"})
        want = (int(ck["suma"], 16), int(ck["sumb"], 16))
        got = scidac_checksum(binary, site_bytes)
        if got != want:
            raise ValueError(f"{path}: SciDAC checksum mismatch (file {want[0]:08x} {want[1]:08x}, "
                             f"data {got[0]:08x} {got[1]:08x})")
        info["checksum"] = "ok"
    lex = np.frombuffer(binary, dtype=f">c{2 * prec // 8}").astype(np.complex128)
    lex = lex.reshape(latt[3], latt[2], latt[1], latt[0], 4, 3, 3)
    return lexico_to_eo(lex, latt), latt, info


def write_ildg(path, gauge, latt, precision: int = 64):
    """Write a gauge field ([mu][parity][t][z][y][x/2][3][3]) as an ILDG
    configuration with a SciDAC checksum."""
    if precision not in (32, 64):
        raise ValueError("precision must be 32 or 64")
    lex = eo_to_lexico(gauge, latt)
    binary = np.ascontiguousarray(lex).astype(f">c{2 * precision // 8}").tobytes()
    Lx, Ly, Lz, Lt = latt
    fmt = ('<?xml version="1.0" encoding="UTF-8"?><ildgFormat xmlns="http://www.lqcd.org/ildg">'
           f"<version>1.0</version><field>su3gauge</field><precision>{precision}</precision>"
           f"<lx>{Lx}</lx><ly>{Ly}</ly><lz>{Lz}</lz><lt>{Lt}</lt></ildgFormat>")
    suma, sumb = scidac_checksum(binary, 4 * 9 * 2 * precision // 8)
    ck = ('<?xml version="1.0" encoding="UTF-8"?><scidacChecksum><version>1.0</version>'
          f"<suma>{suma:08x}</suma><sumb>{sumb:08x}</sumb></scidacChecksum>")
    write_lime(path, [("ildg-format", fmt.encode()), ("ildg-binary-data", binary), ("scidac-checksum", ck.encode())])
