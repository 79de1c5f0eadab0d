"""Radiance .hdr (RGBE) reading, as the viewer's environment loader does
(decodeHDR, src/env.js:5-77): the header must say 32-bit_rle_rgbe, the resolution
line must be "-Y h +X w", and scanlines are either new-style run-length encoded
(a 2 2 hi lo marker, then each of the four channels as runs) or flat RGBE pixels
with the old repeat markers (1 1 1 n). A pixel is (r, g, b) * 2^(e - 136), or 0 when
e = 0. The result feeds Sim.set_environment.

    rgb = load_hdr("sky.hdr")          # float32 [height, width, 3]
    sim.set_environment(rgb)
"""
import numpy as np


def decode_hdr(data):
    """The decoded float32 image [height, width, 3] of an .hdr file's bytes."""
    u8 = np.frombuffer(bytes(data), np.uint8)
    p = 0

    def line():
        nonlocal p
        end = p
        while end < len(u8) and u8[end] != 10:
            end += 1
        s = u8[p:end].tobytes().decode("latin-1")
        p = end + 1
        return s

    if not line().startswith("#?"):
        raise ValueError("not a Radiance .hdr file")
    while True:
        ln = line()
        if ln == "":
            break
        if ln.startswith("FORMAT=") and "32-bit_rle_rgbe" not in ln:
            raise ValueError("unsupported .hdr format: " + ln)
    dim = line().split()
    if len(dim) != 4 or dim[0] != "-Y" or dim[2] != "+X":
        raise ValueError("unsupported .hdr resolution line: " + " ".join(dim))
    h, w = int(dim[1]), int(dim[3])
    out = np.empty((h, w, 3), np.float32)
    rgbe = np.zeros((w, 4), np.uint8)
    for y in range(h):
        if p + 4 > len(u8):
            raise ValueError(".hdr ended early")
        r, g, b, e = (int(v) for v in u8[p:p + 4])
        if r == 2 and g == 2 and ((b << 8) | e) == w and 8 <= w < 32768:
            p += 4
            for c in range(4):
                x = 0
                while x < w:
                    n = int(u8[p])
                    p += 1
                    if n > 128:
                        n -= 128
                        rgbe[x:x + n, c] = u8[p]
                        p += 1
                    else:
                        rgbe[x:x + n, c] = u8[p:p + n]
                        p += n
                    x += n
        else:
            x = shift = 0
            while x < w:
                rr, gg, bb, ee = (int(v) for v in u8[p:p + 4])
                p += 4
                if rr == 1 and gg == 1 and bb == 1:
                    n = ee << (shift * 8)
                    rgbe[x:x + n] = rgbe[x - 1]
                    x += n
                    shift += 1
                else:
                    rgbe[x] = (rr, gg, bb, ee)
                    x += 1
                    shift = 0
        ex = rgbe[:, 3].astype(np.float64)
        f = np.where(ex > 0, np.exp2(ex - 136), 0.0)
        out[y] = (rgbe[:, :3] * f[:, None]).astype(np.float32)
    return out


def load_hdr(path):
    """decode_hdr of a file."""
    with open(path, "rb") as fh:
        return decode_hdr(fh.read())
