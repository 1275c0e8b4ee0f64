"""Minimal FITS binary-table reader and writer (FITS Standard 4.0, sections 4 and 7.3).

The reference reads survey catalogs with ``fitsio`` (src/cosmonpc/catalog_processor.py:128-183):
HDU 1 if the file has more than one HDU, else HDU 0, the requested columns that
exist, all rows, files of a list concatenated in order.  This module keeps the
table in its on-disk form -- big-endian rows of ``NAXIS1`` bytes -- so that the
rows can be copied to the GPU unchanged and decoded there; ``read_columns``
gives host arrays for callers that want them.

Supported column types (repeat count 1): L (bool), B (uint8), I (int16),
J (int32), K (int64), E (float32), D (float64), with ``TSCALn``/``TZEROn``.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np

BLOCK = 2880
CARD = 80

# FITS TFORM code -> (numpy big-endian dtype, bytes per element)
_TFORM = {
    "L": (">i1", 1), "B": (">u1", 1), "I": (">i2", 2), "J": (">i4", 4),
    "K": (">i8", 8), "E": (">f4", 4), "D": (">f8", 8), "A": ("S1", 1),
    "X": (">u1", 1), "C": (">c8", 8), "M": (">c16", 16), "P": (">i4", 8), "Q": (">i8", 16),
}
NUMERIC = "LBIJKED"


@dataclass
class Column:
    name: str
    code: str          # TFORM type letter
    repeat: int
    offset: int        # byte offset within a row
    nbytes: int
    scale: float = 1.0
    zero: float = 0.0


@dataclass
class Table:
    path: str
    nrows: int
    row_bytes: int
    data_offset: int   # file offset of the first row
    columns: dict = field(default_factory=dict)

    def colnames(self):
        return list(self.columns)

    def rows(self):
        """The raw big-endian rows as a read-only (nrows, row_bytes) uint8 memmap."""
        if self.nrows == 0 or self.row_bytes == 0:
            return np.zeros((0, self.row_bytes), dtype=np.uint8)
        return np.memmap(self.path, dtype=np.uint8, mode="r", offset=self.data_offset,
                         shape=(self.nrows, self.row_bytes))

    def scalar_column(self, name):
        c = self.columns[name]
        if c.repeat != 1 or c.code not in NUMERIC:
            raise ValueError(f"column {name}: unsupported FITS form {c.repeat}{c.code}")
        return c

    def read_columns(self, names, rows=None):
        """Structured array with the given columns (host decode, native byte order)."""
        raw = self.rows() if rows is None else self.rows()[rows]
        dt = []
        for nm in names:
            c = self.scalar_column(nm)
            scaled = c.scale != 1.0 or c.zero != 0.0
            base = "?" if c.code == "L" else np.dtype(_TFORM[c.code][0]).newbyteorder("=").str
            dt.append((nm, "f8" if scaled else base))
        out = np.empty(raw.shape[0], dtype=dt)
        for nm in names:
            c = self.columns[nm]
            base, size = _TFORM[c.code]
            v = np.ascontiguousarray(raw[:, c.offset:c.offset + size]).view(base).reshape(-1)
            if c.code == "L":
                v = v == ord("T")
            if c.scale != 1.0 or c.zero != 0.0:
                v = c.zero + c.scale * v.astype(np.float64)
            out[nm] = v
        return out


def _parse_value(text):
    t = text.strip()
    if t.startswith("'"):
        i = 1
        out = []
        while i < len(t):
            if t[i] == "'":
                if i + 1 < len(t) and t[i + 1] == "'":
                    out.append("'")
                    i += 2
                    continue
                break
            out.append(t[i])
            i += 1
        return "".join(out).rstrip()
    t = t.split("/")[0].strip()
    if t in ("T", "F"):
        return t == "T"
    try:
        return int(t)
    except ValueError:
        pass
    try:
        return float(t.replace("D", "E"))
    except ValueError:
        return t


def _read_header(f):
    cards = {}
    nbytes = 0
    while True:
        block = f.read(BLOCK)
        if len(block) < BLOCK:
            if not block:
                return None, 0
            raise ValueError("truncated FITS header")
        nbytes += BLOCK
        for i in range(0, BLOCK, CARD):
            card = block[i:i + CARD].decode("ascii", errors="replace")
            key = card[:8].strip()
            if key == "END":
                return cards, nbytes
            if card[8:10] == "= ":
                cards[key] = _parse_value(card[10:])


def _data_bytes(h):
    naxis = int(h.get("NAXIS", 0))
    if naxis == 0:
        return 0
    size = abs(int(h.get("BITPIX", 8))) // 8
    for i in range(1, naxis + 1):
        size *= int(h.get(f"NAXIS{i}", 0))
    return int(h.get("GCOUNT", 1)) * (size + int(h.get("PCOUNT", 0)))


def _parse_tform(s):
    s = s.strip()
    j = 0
    while j < len(s) and s[j].isdigit():
        j += 1
    repeat = int(s[:j]) if j else 1
    code = s[j:j + 1].upper()
    if code not in _TFORM:
        raise ValueError(f"unsupported TFORM {s!r}")
    return code, repeat


def hdu_list(path):
    """[(header dict, data file offset), ...] for every HDU of a FITS file."""
    out = []
    with open(path, "rb") as f:
        pos = 0
        while True:
            f.seek(pos)
            h, hbytes = _read_header(f)
            if h is None:
                break
            if not out and h.get("SIMPLE") is not True:
                raise ValueError(f"{path}: not a FITS file")
            data_off = pos + hbytes
            out.append((h, data_off))
            pos = data_off + (_data_bytes(h) + BLOCK - 1) // BLOCK * BLOCK
    return out


def open_table(path):
    """The table fitsio would read: HDU 1 if the file has more than one HDU, else HDU 0."""
    hdus = hdu_list(path)
    if not hdus:
        raise ValueError(f"{path}: no HDU")
    h, off = hdus[1] if len(hdus) > 1 else hdus[0]
    if h.get("XTENSION") != "BINTABLE":
        raise ValueError(f"{path}: HDU is not a binary table")
    nrows = int(h.get("NAXIS2", 0))
    row_bytes = int(h.get("NAXIS1", 0))
    cols = {}
    pos = 0
    for i in range(1, int(h.get("TFIELDS", 0)) + 1):
        code, repeat = _parse_tform(h[f"TFORM{i}"])
        nb = (repeat + 7) // 8 if code == "X" else repeat * _TFORM[code][1]
        name = str(h.get(f"TTYPE{i}", f"COL{i}")).strip()
        cols[name] = Column(name, code, repeat, pos, nb, float(h.get(f"TSCAL{i}", 1.0)),
                            float(h.get(f"TZERO{i}", 0.0)))
        pos += nb
    if pos != row_bytes:
        raise ValueError(f"{path}: column widths ({pos}) != NAXIS1 ({row_bytes})")
    return Table(os.fspath(path), nrows, row_bytes, off, cols)


def _card(key, value):
    if isinstance(value, bool):
        v = f"{'T' if value else 'F':>20}"
    elif isinstance(value, (int, np.integer)):
        v = f"{int(value):>20d}"
    elif isinstance(value, (float, np.floating)):
        v = f"{float(value):>20.16G}"
    else:
        s = "'" + str(value).replace("'", "''").ljust(8) + "'"
        v = f"{s:<20}"
    return f"{key:<8}= {v}"[:CARD].ljust(CARD)


def _header_bytes(cards):
    body = "".join(cards) + "END".ljust(CARD)
    return (body + " " * ((-len(body)) % BLOCK)).encode("ascii")


_CODE_OF = {np.dtype("f8"): "D", np.dtype("f4"): "E", np.dtype("i8"): "K",
            np.dtype("i4"): "J", np.dtype("i2"): "I", np.dtype("u1"): "B"}


def write_table(path, columns):
    """Write ``{name: 1-D array}`` as a FITS file with one BINTABLE extension."""
    names = list(columns)
    arrs = [np.asarray(columns[nm]) for nm in names]
    nrows = len(arrs[0]) if arrs else 0
    if any(len(a) != nrows for a in arrs):
        raise ValueError("columns differ in length")
    codes = []
    for nm, a in zip(names, arrs):
        dt = np.dtype(a.dtype).newbyteorder("=")
        if dt not in _CODE_OF:
            raise ValueError(f"column {nm}: unsupported dtype {a.dtype}")
        codes.append(_CODE_OF[dt])
    rec = np.empty(nrows, dtype=[(nm, _TFORM[c][0]) for nm, c in zip(names, codes)])
    for nm, a in zip(names, arrs):
        rec[nm] = a
    primary = _header_bytes([_card("SIMPLE", True), _card("BITPIX", 8), _card("NAXIS", 0),
                             _card("EXTEND", True)])
    cards = [_card("XTENSION", "BINTABLE"), _card("BITPIX", 8), _card("NAXIS", 2),
             _card("NAXIS1", rec.dtype.itemsize), _card("NAXIS2", nrows), _card("PCOUNT", 0),
             _card("GCOUNT", 1), _card("TFIELDS", len(names))]
    for i, (nm, c) in enumerate(zip(names, codes), 1):
        cards += [_card(f"TTYPE{i}", nm), _card(f"TFORM{i}", c)]
    data = rec.tobytes()
    with open(path, "wb") as f:
        f.write(primary)
        f.write(_header_bytes(cards))
        f.write(data)
        f.write(b"\0" * ((-len(data)) % BLOCK))
