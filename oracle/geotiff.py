"""CPU restatement of the reference's GeoTIFF writer, and a reader for the tests.

Test infrastructure only: the product never imports this module.

write() follows WriteGeoTiff (src/raster/geotiff/geotiff_write.cpp:256-297): tiles in order
(band, tile row, tile column) padded with the no-data value (or 0); compressed tiles through the
floating-point predictor (EncodeFloatPredictor, tiff_codecs.cpp:354) then LZW (EncodeLzw,
tiff_codecs.cpp:269) or Deflate (zlib here at level 6; the reference's miniz gives other bytes
for the same data); each tile at an even offset after the header; the IFD (IfdWriter,
geotiff_write.cpp:23) after the last tile. read() parses the files the tests compare, decoding
None, LZW and Deflate tiles.
"""

from __future__ import annotations

import math
import struct
import zlib

import numpy as np

COMPRESSION_CODE = {"none": 1, "lzw": 5, "deflate": 8}
CLEAR, END, FIRST, MAX_CODE = 256, 257, 258, 4096


def predict(tile: np.ndarray) -> bytes:
    """EncodeFloatPredictor on a tile x tile float32 block: each row's bytes in planes, most
    significant first, then each byte minus the one before it."""
    t = tile.shape[1]
    b = np.ascontiguousarray(tile, "<f4").view(np.uint8).reshape(-1, t, 4)
    planes = b[:, :, ::-1].transpose(0, 2, 1).reshape(-1, 4 * t)
    out = planes.copy()
    out[:, 1:] = planes[:, 1:] - planes[:, :-1]
    return out.tobytes()


def unpredict(data: bytes, tile: int) -> np.ndarray:
    rows = np.frombuffer(data, np.uint8).reshape(-1, 4 * tile)
    planes = np.cumsum(rows, axis=1, dtype=np.uint64).astype(np.uint8)
    b = planes.reshape(-1, 4, tile).transpose(0, 2, 1)[:, :, ::-1]
    return np.ascontiguousarray(b).view("<f4").reshape(-1, tile)


def lzw_encode(data: bytes) -> bytes:
    """The reference's TIFF LZW: greedy longest match, MSB-first codes of 9 to 12 bits with the
    early width change, Clear when the next code reaches 4094, EndOfInfo at the end."""
    out = bytearray()
    acc = 0
    count = 0

    def put(code, width):
        nonlocal acc, count
        acc = (acc << width) | code
        count += width
        while count >= 8:
            count -= 8
            out.append((acc >> count) & 0xFF)
        acc &= (1 << count) - 1

    width, nxt = 9, FIRST
    put(CLEAR, width)
    table: dict = {}
    cur = -1
    for byte in data:
        if cur < 0:
            cur = byte
            continue
        key = (cur << 8) | byte
        found = table.get(key)
        if found is not None:
            cur = found
            continue
        table[key] = nxt
        put(cur, width)
        nxt += 1
        if nxt >= (1 << width) and width < 12:
            width += 1
        if nxt >= MAX_CODE - 2:
            put(CLEAR, width)
            width, nxt = 9, FIRST
            table.clear()
        cur = byte
    if cur >= 0:
        put(cur, width)
        nxt += 1
        if nxt >= (1 << width) and width < 12:
            width += 1
    put(END, width)
    if count > 0:
        out.append((acc << (8 - count)) & 0xFF)
    return bytes(out)


def lzw_decode(data: bytes, size: int) -> bytes:
    out = bytearray()
    pos, acc, count = 0, 0, 0
    width = 9
    strings = [bytes([i]) for i in range(256)] + [b"", b""]
    prev = None
    while len(out) < size:
        while count < width:
            if pos >= len(data):
                return bytes(out[:size])
            acc = (acc << 8) | data[pos]
            pos += 1
            count += 8
        count -= width
        code = (acc >> count) & ((1 << width) - 1)
        acc &= (1 << count) - 1
        if code == END:
            break
        if code == CLEAR:
            strings = strings[:FIRST]
            width = 9
            prev = None
            continue
        if prev is None:
            s = strings[code]
        else:
            s = strings[code] if code < len(strings) else prev + prev[:1]
            strings.append(prev + s[:1])
        out += s
        prev = s
        if len(strings) + 1 >= (1 << width) and width < 12:
            width += 1
    return bytes(out[:size])


def _tiles(bands, tile: int, fill: float):
    h, w = bands[0].shape
    across, down = math.ceil(w / tile), math.ceil(h / tile)
    for band in bands:
        padded = np.full((down * tile, across * tile), fill, np.float32)
        padded[:h, :w] = band
        for ty in range(down):
            for tx in range(across):
                yield padded[ty * tile:(ty + 1) * tile, tx * tile:(tx + 1) * tile]


def _pixel_is_point(directory) -> bool:
    d = list(directory)
    if len(d) < 4:
        return False
    for k in range(d[3]):
        at = 4 + 4 * k
        if at + 3 < len(d) and d[at] == 1025 and d[at + 1] == 0:
            return d[at + 3] == 2
    return False


def write(bands, transform, nodata=None, directory=(), doubles=(), ascii: str = "",
          compression: str = "lzw", tile_size: int = 256, big_tiff: bool = False) -> bytes:
    """The bytes WriteGeoTiff writes (Deflate through zlib: other bytes, the same data)."""
    bands = [np.ascontiguousarray(b, np.float32) for b in bands]
    h, w = bands[0].shape
    across, down = math.ceil(w / tile_size), math.ceil(h / tile_size)
    total = across * down * len(bands)
    tile_bytes = tile_size * tile_size * 4
    big = big_tiff or total * tile_bytes + (1 << 20) >= (1 << 32)
    start = 16 if big else 8
    fill = 0.0 if nodata is None else nodata
    stream = bytearray()
    offsets, counts = [], []
    for t in _tiles(bands, tile_size, fill):
        if compression == "none":
            data = np.ascontiguousarray(t, "<f4").tobytes()
        elif compression == "lzw":
            data = lzw_encode(predict(t))
        else:
            data = zlib.compress(predict(t), 6)
        offsets.append(start + len(stream))
        counts.append(len(data))
        stream += data
        if len(stream) % 2:
            stream.append(0)
    end = start + len(stream)
    nb = len(bands)
    entries = {256: (4, [w]), 257: (4, [h]), 258: (3, [32] * nb),
               259: (3, [COMPRESSION_CODE[compression]]), 262: (3, [1]), 277: (3, [nb]),
               284: (3, [1 if nb == 1 else 2]), 322: (4, [tile_size]), 323: (4, [tile_size]),
               324: (16 if big else 4, offsets), 325: (16 if big else 4, counts),
               339: (3, [3] * nb)}
    if compression != "none":
        entries[317] = (3, [3])
    if nb > 1:
        entries[338] = (3, [0] * (nb - 1))
    t = list(transform)
    if len(directory) > 0 or t != [0.0, 1.0, 0.0, 0.0, 0.0, 1.0]:
        ox, pw, rr, oy, cr, ph = t
        if _pixel_is_point(directory):
            ox += 0.5 * (pw + rr)
            oy += 0.5 * (cr + ph)
        if rr == 0.0 and cr == 0.0:
            entries[33550] = (12, [pw, -ph, 0.0])
            entries[33922] = (12, [0.0, 0.0, 0.0, ox, oy, 0.0])
        else:
            entries[34264] = (12, [pw, rr, 0.0, ox, cr, ph, 0.0, oy] + [0.0] * 7 + [1.0])
    if len(directory) > 0:
        entries[34735] = (3, list(directory))
        if len(doubles) > 0:
            entries[34736] = (12, list(doubles))
        if ascii:
            entries[34737] = (2, ascii.encode() + b"\0")
    if nodata is not None:
        entries[42113] = (2, ("%.9g" % float(np.float32(nodata))).encode() + b"\0")
    return bytes(_header(big, end)) + bytes(stream) + _ifd(entries, big, end)


_PACK = {2: "B", 3: "H", 4: "I", 12: "d", 16: "Q"}
_SIZE = {2: 1, 3: 2, 4: 4, 12: 8, 16: 8}


def _header(big: bool, ifd: int) -> bytes:
    if big:
        return b"II" + struct.pack("<HHHQ", 43, 8, 0, ifd)
    return b"II" + struct.pack("<HI", 42, ifd)


def _ifd(entries: dict, big: bool, offset: int) -> bytes:
    word = 8 if big else 4
    count_size = 8 if big else 2
    entry_size = 4 + 2 * word
    table_size = count_size + len(entries) * entry_size + word
    table = bytearray(table_size)
    extra = bytearray()
    table[0:count_size] = len(entries).to_bytes(count_size, "little")
    at = count_size
    for tag in sorted(entries):
        ftype, values = entries[tag]
        raw = bytes(values) if ftype == 2 else struct.pack("<" + _PACK[ftype] * len(values),
                                                          *values)
        n = len(values)
        table[at:at + 2] = tag.to_bytes(2, "little")
        table[at + 2:at + 4] = ftype.to_bytes(2, "little")
        table[at + 4:at + 4 + word] = n.to_bytes(word, "little")
        v = at + 4 + word
        if len(raw) <= word:
            table[v:v + len(raw)] = raw
        else:
            if len(extra) % 2:
                extra.append(0)
            table[v:v + word] = (offset + table_size + len(extra)).to_bytes(word, "little")
            extra += raw
        at += entry_size
    return bytes(table + extra)


def read(data: bytes) -> dict:
    """The first IFD's tags ({tag: (type, values)}) and the bands it holds, decoded."""
    assert data[:2] == b"II"
    magic = struct.unpack_from("<H", data, 2)[0]
    big = magic == 43
    word = 8 if big else 4
    ifd = struct.unpack_from("<Q", data, 8)[0] if big else struct.unpack_from("<I", data, 4)[0]
    n = int.from_bytes(data[ifd:ifd + (8 if big else 2)], "little")
    at = ifd + (8 if big else 2)
    tags = {}
    for _ in range(n):
        tag, ftype = struct.unpack_from("<HH", data, at)
        count = int.from_bytes(data[at + 4:at + 4 + word], "little")
        size = _SIZE[ftype] * count
        v = at + 4 + word
        if size > word:
            v = int.from_bytes(data[v:v + word], "little")
        raw = data[v:v + size]
        values = raw if ftype == 2 else list(struct.unpack("<" + _PACK[ftype] * count, raw))
        tags[tag] = (ftype, values)
        at += 4 + 2 * word
    w, h = tags[256][1][0], tags[257][1][0]
    tile = tags[322][1][0]
    code = tags[259][1][0]
    nb = tags[277][1][0]
    across, down = math.ceil(w / tile), math.ceil(h / tile)
    offsets, counts = tags[324][1], tags[325][1]
    bands = []
    k = 0
    for _ in range(nb):
        full = np.zeros((down * tile, across * tile), np.float32)
        for ty in range(down):
            for tx in range(across):
                chunk = data[offsets[k]:offsets[k] + counts[k]]
                size = tile * tile * 4
                if code == 1:
                    block = np.frombuffer(chunk, "<f4").reshape(tile, tile)
                else:
                    raw = lzw_decode(chunk, size) if code == 5 else zlib.decompress(chunk)
                    block = unpredict(raw, tile)
                full[ty * tile:(ty + 1) * tile, tx * tile:(tx + 1) * tile] = block
                k += 1
        bands.append(full[:h, :w])
    return {"tags": tags, "bands": bands, "big": big}
