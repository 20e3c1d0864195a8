"""Film output: the reference HDRBitmapFilm's save path (hdrfilm.cpp:199-304)
without FreeImage.

* Path rules of HDRBitmapFilm::RescaleAndSave: an empty path becomes
  "result.hdr"; a path without extension gets ".hdr" or ".exr" from the
  film's image type; an extension that does not match the type becomes
  "result.hdr"; a missing parent directory is created.
* Row order: the film's row y = 0 is the image's bottom row (FreeImage
  scanline 0), so top-down formats write row H - 1 first.
* Radiance HDR (".hdr"): "#?RADIANCE" header, FORMAT=32-bit_rle_rgbe,
  "-Y H +X W", then flat RGBE pixels (Ward's shared-exponent encoding,
  Graphics Gems II, "Real Pixels"); readers accept flat and run-length
  scanlines alike, and `read_hdr` reads both.
* OpenEXR (".exr"): single-part scanline file, channels B, G, R as 32-bit
  float, no compression (FreeImage's default stores half floats with PIZ
  compression; this keeps full float precision).
* PFM (".pfm"), a plain float format, for tests and tools.
"""
from __future__ import annotations

import os
import struct
from typing import Optional

import numpy as np

RADIANCE_HDR = "radiancehdr"
OPEN_EXR = "openexr"


def resolve_output_path(path: str, image_type: str = RADIANCE_HDR) -> str:
    """HDRBitmapFilm::RescaleAndSave's choice of the file name (hdrfilm.cpp:204-240)."""
    ext = {RADIANCE_HDR: ".hdr", OPEN_EXR: ".exr"}
    if image_type not in ext:
        raise ValueError(f"unknown image type '{image_type}'")
    if not path:
        return "result.hdr"
    root, e = os.path.splitext(path)
    if e:
        return path if e == ext[image_type] else "result.hdr"
    return path + ext[image_type]


def save_film(film: np.ndarray, path: str, image_type: str = RADIANCE_HDR, weight: float = 1.0) -> str:
    """Writes film (H, W, 3), row y = 0 first, scaled by `weight`; returns the
    path written."""
    out = resolve_output_path(path, image_type)
    parent = os.path.dirname(out)
    if parent and not os.path.exists(parent):
        os.makedirs(parent)
    img = np.asarray(film, np.float32).reshape(film.shape[0], film.shape[1], 3) * np.float32(weight)
    if out.endswith(".exr"):
        write_exr(out, img)
    else:
        write_hdr(out, img)
    return out


# ------------------------------------------------------------- Radiance ----

def rgbe_encode(img: np.ndarray) -> np.ndarray:
    """(..., 3) float -> (..., 4) uint8 RGBE: the largest component v sets the
    shared exponent e with v = m * 2^e, m in [0.5, 1); each channel is stored
    as floor(c * m * 256 / v); v < 1e-32 encodes as zero."""
    c = np.maximum(np.asarray(img, np.float64), 0.0)
    v = c.max(axis=-1)
    m, e = np.frexp(v)
    out = np.zeros(c.shape[:-1] + (4,), np.uint8)
    ok = v >= 1e-32
    scale = np.where(ok, m * 256.0 / np.where(ok, v, 1.0), 0.0)
    out[..., :3] = np.where(ok[..., None], np.floor(c * scale[..., None]), 0).astype(np.uint8)
    out[..., 3] = np.where(ok, e + 128, 0).astype(np.uint8)
    return out


def rgbe_decode(rgbe: np.ndarray) -> np.ndarray:
    """(..., 4) uint8 -> (..., 3) float32: (c + 0.5) * 2^(e - 136), zero for e = 0."""
    q = np.asarray(rgbe)
    e = q[..., 3].astype(np.int32)
    f = np.where(e > 0, np.ldexp(1.0, e - 136), 0.0)
    return ((q[..., :3].astype(np.float64) + 0.5) * f[..., None] * (e > 0)[..., None]).astype(np.float32)


def write_hdr(path: str, film: np.ndarray) -> None:
    H, W = film.shape[:2]
    top_down = film[::-1]                       # film row 0 is the bottom row
    with open(path, "wb") as f:
        f.write(b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n")
        f.write(f"-Y {H} +X {W}\n".encode())
        f.write(rgbe_encode(top_down).tobytes())


def read_hdr(path: str) -> np.ndarray:
    """Reads a Radiance HDR file ("-Y H +X W", flat or run-length scanlines);
    returns the film (H, W, 3), row y = 0 = the image's bottom row."""
    data = open(path, "rb").read()
    pos = 0
    header = []
    while True:
        nl = data.index(b"\n", pos)
        line = data[pos:nl].decode("latin-1")
        pos = nl + 1
        if line.startswith("-Y") or line.startswith("+Y"):
            break
        header.append(line)
    if not header or not header[0].startswith("#?"):
        raise ValueError("not a Radiance HDR file")
    parts = line.split()
    if parts[0] != "-Y" or parts[2] != "+X":
        raise ValueError("only -Y H +X W images are supported")
    H, W = int(parts[1]), int(parts[3])
    out = np.zeros((H, W, 4), np.uint8)
    for y in range(H):
        if 8 <= W < 32768 and data[pos] == 2 and data[pos + 1] == 2 and (data[pos + 2] << 8 | data[pos + 3]) == W:
            pos += 4
            for ch in range(4):                 # run-length: one component at a time
                x = 0
                while x < W:
                    n = data[pos]
                    pos += 1
                    if n > 128:
                        n -= 128
                        out[y, x:x + n, ch] = data[pos]
                        pos += 1
                    else:
                        out[y, x:x + n, ch] = np.frombuffer(data, np.uint8, n, pos)
                        pos += n
                    x += n
        else:
            out[y] = np.frombuffer(data, np.uint8, 4 * W, pos).reshape(W, 4)
            pos += 4 * W
    return rgbe_decode(out)[::-1].copy()


# -------------------------------------------------------------- OpenEXR ----

def _attr(name: str, type_name: str, value: bytes) -> bytes:
    return name.encode() + b"\0" + type_name.encode() + b"\0" + struct.pack("<i", len(value)) + value


def write_exr(path: str, film: np.ndarray) -> None:
    H, W = film.shape[:2]
    top_down = np.ascontiguousarray(film[::-1], np.float32)
    chans = b"".join(c.encode() + b"\0" + struct.pack("<iB3xii", 2, 0, 1, 1) for c in "BGR") + b"\0"
    box = struct.pack("<iiii", 0, 0, W - 1, H - 1)
    header = (struct.pack("<ii", 20000630, 2)
              + _attr("channels", "chlist", chans)
              + _attr("compression", "compression", b"\0")
              + _attr("dataWindow", "box2i", box)
              + _attr("displayWindow", "box2i", box)
              + _attr("lineOrder", "lineOrder", b"\0")
              + _attr("pixelAspectRatio", "float", struct.pack("<f", 1.0))
              + _attr("screenWindowCenter", "v2f", struct.pack("<ff", 0.0, 0.0))
              + _attr("screenWindowWidth", "float", struct.pack("<f", 1.0))
              + b"\0")
    line_bytes = 3 * 4 * W
    table_start = len(header)
    first = table_start + 8 * H
    offsets = struct.pack(f"<{H}Q", *[first + y * (8 + line_bytes) for y in range(H)])
    with open(path, "wb") as f:
        f.write(header)
        f.write(offsets)
        for y in range(H):
            row = top_down[y]
            f.write(struct.pack("<ii", y, line_bytes))
            for c in (2, 1, 0):                 # channels in name order: B, G, R
                f.write(row[:, c].astype("<f4").tobytes())


def read_exr(path: str) -> np.ndarray:
    """Reads an uncompressed 32-bit-float scanline OpenEXR file with B, G, R
    channels (as write_exr writes them); returns the film (H, W, 3)."""
    data = open(path, "rb").read()
    magic, version = struct.unpack_from("<ii", data, 0)
    if magic != 20000630:
        raise ValueError("not an OpenEXR file")
    pos = 8
    attrs = {}
    while data[pos] != 0:
        n0 = data.index(b"\0", pos)
        name = data[pos:n0].decode()
        t0 = data.index(b"\0", n0 + 1)
        size = struct.unpack_from("<i", data, t0 + 1)[0]
        attrs[name] = data[t0 + 5:t0 + 5 + size]
        pos = t0 + 5 + size
    pos += 1
    if attrs["compression"] != b"\0":
        raise ValueError("only uncompressed files are supported")
    x0, y0, x1, y1 = struct.unpack("<iiii", attrs["dataWindow"])
    W, H = x1 - x0 + 1, y1 - y0 + 1
    offsets = struct.unpack_from(f"<{H}Q", data, pos)
    img = np.zeros((H, W, 3), np.float32)
    for y, off in enumerate(offsets):
        yy, size = struct.unpack_from("<ii", data, off)
        row = np.frombuffer(data, "<f4", 3 * W, off + 8).reshape(3, W)
        img[yy - y0, :, 2], img[yy - y0, :, 1], img[yy - y0, :, 0] = row[0], row[1], row[2]
    return img[::-1].copy()


# ------------------------------------------------------------------ PFM ----

def write_pfm(path: str, film: np.ndarray) -> None:
    """PFM stores rows bottom-up, like the film."""
    H, W = film.shape[:2]
    with open(path, "wb") as f:
        f.write(f"PF\n{W} {H}\n-1.0\n".encode())
        f.write(np.ascontiguousarray(film, "<f4").tobytes())


def read_pfm(path: str) -> np.ndarray:
    with open(path, "rb") as f:
        if f.readline().strip() != b"PF":
            raise ValueError("not a colour PFM file")
        W, H = map(int, f.readline().split())
        scale = float(f.readline())
        dt = "<f4" if scale < 0 else ">f4"
        return np.frombuffer(f.read(), dt, H * W * 3).reshape(H, W, 3).astype(np.float32)
