"""Output side of the slice pipeline on the host: the 8-bit threshold oracle's
rules (tomo_recon.cpp:2282-2361) and the raw/NRRD slice files (:2120-2244)."""
import numpy as np

from oracle import oracle as O
from projects_b200 import slice_io as S


def test_threshold_oracle_rules():
    img = np.array([[[0.0, 1.0, 2.0, np.nan],
                     [3.0, 4.0, -1.0, 5.0]]], np.float32)
    u, (lo, hi) = O.port_to_u8(img)
    assert (lo, hi) == (-1.0, 5.0)                      # NaN skipped by the min/max
    assert u[0, 0, 3] == 0                              # NaN pixel -> 0
    assert u[0, 1, 3] == 255 and u[0, 1, 2] == 0        # the extremes
    # interior value: (unsigned char)(255 * (p - lo) / (hi - lo)) in float
    assert u[0, 0, 1] == int(np.float32(255) * np.float32(2.0) / np.float32(6.0))
    u, (lo, hi) = O.port_to_u8(img, lower_clamp=0.5, upper_clamp=3.5)
    assert (lo, hi) == (0.5, 3.5)                       # clamps tighten the range
    assert u[0, 0, 0] == 0 and u[0, 1, 1] == 255
    flat = np.full((1, 3, 3), 2.0, np.float32)
    u, _ = O.port_to_u8(flat)
    assert np.all(u == 0)                               # hi == lo: 0/0 -> 0


def test_threshold_crop_keeps_the_boundary_circle():
    img = np.ones((1, 9, 9), np.float32)
    img[0, 0, 0] = 0.0
    u, _ = O.port_to_u8(img, radius=3)
    keep = S.circle_keep(9, 9, 3)
    assert keep[4, 7] and not keep[4, 8]                # distance 3 kept, 4 not
    assert np.all(u[0][~keep] == 0) and np.all(u[0][keep & (img[0] == 1)] == 255)


def test_slice_names():
    assert S.slice_file_name("recon_00000.bin", 12) == "recon_00012.bin"
    assert S.slice_file_name("rec_0000.bin", 1234) == "rec_1234.bin"
    assert S.crop_name("rec_0012.bin") == "rec_0012_crop.bin"


def test_bin_and_nrrd_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    vol = rng.normal(size=(3, 6, 8)).astype(np.float32)
    paths = S.write_bin_slices(str(tmp_path), "slice_0000.bin", vol, 7, crop_radius=2)
    assert [p.rsplit("/", 1)[1] for p in paths[:2]] == ["slice_0007.bin", "slice_0007_crop.bin"]
    back = np.fromfile(paths[0], dtype=np.float32).reshape(6, 8)
    assert np.array_equal(back, vol[0])
    crop = np.fromfile(paths[1], dtype=np.float32).reshape(6, 8)
    keep = S.circle_keep(6, 8, 2)
    assert np.array_equal(crop[keep], vol[0][keep]) and np.all(crop[~keep] == 0)
    S.write_nrrd(str(tmp_path / "v.nrrd"), vol)
    assert np.array_equal(S.read_nrrd(str(tmp_path / "v.nrrd")), vol)
    head = open(tmp_path / "v.nrrd", "rb").read(64).decode("ascii", "replace")
    assert head.startswith("NRRD0004\ntype: float\ndimension: 3\nsizes: 8 6 3\n")
