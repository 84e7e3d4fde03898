"""Reconstructed-slice files as the reference's driver writes them.

* Raw float32 slices (RECON_IMAGE_TYPE_BIN, gridrec/GPU/tomo_recon.cpp:2177-2244):
  one file per slice, rows of float32 in host byte order, the slice number spliced
  into the base name just before the extension; with a crop radius also a
  "<name>_crop.bin" copy whose pixels outside the circle are 0 (the BIN writer
  keeps pixels with (x - w/2)^2 + (y - h/2)^2 <= r^2).
* NRRD volumes (RECON_IMAGE_TYPE_NRRD, :2120-2147, written there through ITK): a
  plain NRRD0004 header (type float, dimension 3, sizes x y z, raw encoding) and
  the float32 voxels, x fastest.
HDF5 (DataExchange) and 8-bit BMP/TIFF files need libraries this package does
not carry; their pixel arithmetic is in gr_to_u8 / gridrec.to_u8.
"""
from __future__ import annotations

import os
import sys

import numpy as np


def slice_file_name(base_name: str, index: int, ext: str = ".bin") -> str:
    """The reference's naming rule (tomo_recon.cpp:2191-2197): the decimal slice
    number overwrites as many characters of the base name as it has digits,
    ending just before the extension; "_crop" variants insert that before it."""
    if not base_name.endswith(ext):
        raise ValueError(f"base name must end with {ext}")
    digits = str(int(index))
    pos = len(base_name) - len(ext) - len(digits)
    if pos < 0:
        raise ValueError("slice number longer than the base name")
    return base_name[:pos] + digits + base_name[pos + len(digits):]


def crop_name(name: str, ext: str = ".bin") -> str:
    return name[:len(name) - len(ext)] + "_crop" + name[len(name) - len(ext):]


def circle_keep(rows: int, cols: int, radius: int) -> np.ndarray:
    """Mask of the BIN/8-bit writers' crop: (x - cols/2)^2 + (y - rows/2)^2 <= r^2."""
    y = np.arange(rows)[:, None] - rows // 2
    x = np.arange(cols)[None, :] - cols // 2
    return x * x + y * y <= radius * radius


def write_bin_slices(directory: str, base_name: str, images, first_index: int,
                     crop_radius: int = 0) -> list:
    """Writes images (S, rows, cols) as float32 .bin files numbered first_index + s
    (and their cropped copies); returns the paths written."""
    imgs = np.asarray(images, np.float32)
    paths = []
    keep = circle_keep(imgs.shape[1], imgs.shape[2], crop_radius) if crop_radius > 0 else None
    for s in range(imgs.shape[0]):
        name = os.path.join(directory, slice_file_name(base_name, first_index + s))
        imgs[s].astype("=f4").tofile(name)
        paths.append(name)
        if keep is not None:
            cname = crop_name(name)
            np.where(keep, imgs[s], np.float32(0)).astype("=f4").tofile(cname)
            paths.append(cname)
    return paths


def write_nrrd(path: str, volume) -> None:
    """float32 volume (z, y, x) as a raw NRRD file."""
    vol = np.ascontiguousarray(volume, np.float32)
    if vol.ndim == 2:
        vol = vol[None]
    z, y, x = vol.shape
    endian = "little" if sys.byteorder == "little" else "big"
    header = (f"NRRD0004\ntype: float\ndimension: 3\nsizes: {x} {y} {z}\n"
              f"endian: {endian}\nencoding: raw\n\n")
    with open(path, "wb") as f:
        f.write(header.encode("ascii"))
        f.write(vol.tobytes())


def read_nrrd(path: str) -> np.ndarray:
    """Reads back what write_nrrd writes (raw float32), as (z, y, x)."""
    with open(path, "rb") as f:
        data = f.read()
    head, _, body = data.partition(b"\n\n")
    fields = dict(line.split(": ", 1) for line in head.decode("ascii").splitlines()[1:])
    if fields.get("type") != "float" or fields.get("encoding") != "raw":
        raise ValueError("only raw float NRRD files")
    x, y, z = (int(v) for v in fields["sizes"].split())
    dt = "<f4" if fields.get("endian", "little") == "little" else ">f4"
    return np.frombuffer(body, dtype=dt, count=x * y * z).reshape(z, y, x).astype(np.float32)
