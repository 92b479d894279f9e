"""PNG files for the headless slice pictures (RGBA8, rows top to bottom).

The reference shows its slices on a canvas; without a graphics API the
picture is a buffer, and this writes it as a standard PNG (8-bit RGBA,
filter 0 per row, one zlib stream) or reads one back.
"""
import struct
import zlib

import numpy as np

_SIG = b"\x89PNG\r\n\x1a\n"


def _chunk(tag: bytes, data: bytes) -> bytes:
    return struct.pack(">I", len(data)) + tag + data + struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF)


def png_bytes(rgba: np.ndarray) -> bytes:
    img = np.ascontiguousarray(rgba, np.uint8)
    if img.ndim != 3 or img.shape[2] != 4:
        raise ValueError("expected an (height, width, 4) uint8 array")
    h, w = img.shape[:2]
    raw = b"".join(b"\x00" + img[y].tobytes() for y in range(h))
    ihdr = struct.pack(">IIBBBBB", w, h, 8, 6, 0, 0, 0)
    return _SIG + _chunk(b"IHDR", ihdr) + _chunk(b"IDAT", zlib.compress(raw, 6)) + _chunk(b"IEND", b"")


def write_png(path, rgba: np.ndarray) -> None:
    with open(path, "wb") as f:
        f.write(png_bytes(rgba))


def read_png(data: bytes) -> np.ndarray:
    """Decodes what png_bytes writes (8-bit RGBA, filter type 0 rows)."""
    if data[:8] != _SIG:
        raise ValueError("not a PNG")
    pos, idat, w, h = 8, b"", 0, 0
    while pos < len(data):
        n = struct.unpack(">I", data[pos:pos + 4])[0]
        tag, body = data[pos + 4:pos + 8], data[pos + 8:pos + 8 + n]
        if tag == b"IHDR":
            w, h, depth, ctype = struct.unpack(">IIBB", body[:10])
            if depth != 8 or ctype != 6:
                raise ValueError("only 8-bit RGBA is read")
        elif tag == b"IDAT":
            idat += body
        pos += 12 + n
    raw = zlib.decompress(idat)
    rows = np.frombuffer(raw, np.uint8).reshape(h, 1 + 4 * w)
    if np.any(rows[:, 0] != 0):
        raise ValueError("only filter type 0 rows are read")
    return rows[:, 1:].reshape(h, w, 4).copy()
