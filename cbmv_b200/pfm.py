"""PFM disparity files, as the reference reads and writes them
(pylibs/pfmutil.py:11-61): a text header "Pf" (grey) or "PF" (colour),
"width height", then the scale whose sign gives the byte order (negative =
little-endian), then float32 rows from the bottom of the image up."""
import re
import sys

import numpy as np


def load(path):
    """(image float32 [H,W] or [H,W,3], scale) -- pfmutil.py:11-42."""
    with open(path, "rb") as f:
        header = f.readline().rstrip()
        if header == b"PF":
            color = True
        elif header == b"Pf":
            color = False
        else:
            raise ValueError("not a PFM file: %s" % path)
        m = re.match(rb"^(\d+)\s(\d+)\s$", f.readline())
        if not m:
            raise ValueError("malformed PFM header: %s" % path)
        width, height = (int(v) for v in m.groups())
        scale = float(f.readline().rstrip())
        endian = "<" if scale < 0 else ">"
        data = np.fromfile(f, endian + "f4")
    shape = (height, width, 3) if color else (height, width)
    return np.flipud(data.reshape(shape)).astype(np.float32), abs(scale)


def save(path, image, scale=1):
    """pfmutil.py:44-66: float32 [H,W], [H,W,1] or [H,W,3]."""
    image = np.asarray(image)
    if image.dtype != np.float32:
        raise ValueError("image dtype must be float32")
    if image.ndim == 3 and image.shape[2] == 3:
        color = True
    elif image.ndim == 2 or (image.ndim == 3 and image.shape[2] == 1):
        color = False
    else:
        raise ValueError("image must be H x W x 3, H x W x 1 or H x W")
    endian = image.dtype.byteorder
    if endian == "<" or (endian == "=" and sys.byteorder == "little"):
        scale = -scale
    with open(path, "wb") as f:
        f.write(b"PF\n" if color else b"Pf\n")
        f.write(b"%d %d\n" % (image.shape[1], image.shape[0]))
        f.write(b"%f\n" % scale)
        np.flipud(image).tofile(f)
