"""Headless frame output: binary PPM and PNG writers (standard library only).

The reference presents frames through a Vulkan swapchain
(src/vulkan_context.cpp:617-688); without a graphics stack the frame stays
in a device buffer and is written to a file on request.
"""
import struct
import zlib

import numpy as np


def write_ppm(path, rgba):
    """RGBA8 (H, W, 4) -> binary P6 (alpha dropped)."""
    a = np.ascontiguousarray(np.asarray(rgba, dtype=np.uint8)[..., :3])
    h, w = a.shape[:2]
    with open(path, "wb") as f:
        f.write(b"P6\n%d %d\n255\n" % (w, h))
        f.write(a.tobytes())


def read_ppm(path):
    with open(path, "rb") as f:
        data = f.read()
    parts = data.split(maxsplit=4)
    assert parts[0] == b"P6" and parts[3] == b"255", "binary 8-bit PPM expected"
    w, h = int(parts[1]), int(parts[2])
    px = np.frombuffer(parts[4][: w * h * 3], dtype=np.uint8).reshape(h, w, 3)
    return px


def write_png(path, rgba):
    """RGBA8 (H, W, 4) -> PNG (colour type 6, no filtering, zlib level 6)."""
    a = np.ascontiguousarray(np.asarray(rgba, dtype=np.uint8))
    h, w = a.shape[:2]
    raw = np.concatenate([np.zeros((h, 1), dtype=np.uint8), a.reshape(h, w * 4)], axis=1).tobytes()

    def chunk(tag, body):
        return struct.pack(">I", len(body)) + tag + body + struct.pack(">I", zlib.crc32(tag + body) & 0xFFFFFFFF)

    with open(path, "wb") as f:
        f.write(b"\x89PNG\r\n\x1a\n")
        f.write(chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 6, 0, 0, 0)))
        f.write(chunk(b"IDAT", zlib.compress(raw, 6)))
        f.write(chunk(b"IEND", b""))


def write_image(path, rgba):
    if path.lower().endswith(".png"):
        write_png(path, rgba)
    else:
        write_ppm(path, rgba)
