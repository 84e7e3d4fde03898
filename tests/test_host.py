"""CPU tests: the C-ABI library, its host-side logic and the phantom generator."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from oracle import oracle as O
from projects_b200 import gridrec as G
from projects_b200 import phantom as ph

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            src = open(os.path.join(inc, f)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(gr_\w+)\s*\(", src, re.M))
    return names


def test_library_exports_every_declared_symbol():
    lib = G.lib()
    declared = _declared_functions()
    assert declared, "no declarations parsed"
    for name in declared:
        assert hasattr(lib, name), f"{name} declared in include/ but not exported"
    assert set(G.EXPORTS) <= declared


def test_filter_codes():
    codes = {n: G.filter_code(n) for n in
             ["shlo", "shepp", "hann", "hamm", "hamming", "ramp", "ramlak", "none", "bogus"]}
    assert codes == {"shlo": 1, "shepp": 1, "hann": 2, "hamm": 3, "hamming": 3, "ramp": 4,
                     "ramlak": 4, "none": 0, "bogus": 1}


def test_params_default():
    th = np.zeros(10, np.float32)
    p, _ = G.make_params(64, 10, th)
    assert (p.n_det, p.n_ang, p.filter, p.ltbl, p.max_pairs) == (64, 10, 1, 512, 1)
    assert p.center < 0 and abs(p.pswf_c - 6.0) < 1e-6 and abs(p.sampl - 1.0) < 1e-6


@pytest.mark.parametrize("bad,code", [
    (dict(pswf_c=5.5), -2),       # not in the PSWF database
    (dict(n_det=8), -1),          # below the smallest FFT
    (dict(ltbl=0), -1),
    (dict(sampl=0.5), -1),
])
def test_parameter_errors(bad, code):
    kw = dict(n_det=64, n_ang=10, pswf_c=6.0, sampl=1.0, ltbl=512)
    kw.update(bad)
    p, th = G.make_params(kw["n_det"], kw["n_ang"], np.zeros(kw["n_ang"], np.float32),
                          pswf_c=kw["pswf_c"], sampl=kw["sampl"], ltbl=kw["ltbl"])
    ni = C.c_int()
    rc = G.lib().gr_worklist_export(C.byref(p), C.byref(ni), None, None, None, None, None, 0, 0)
    assert rc == code
    assert G.last_error()


def _emulate_gather(n, a, theta, sampl=1.0, pswf_c=6.0):
    """Numpy float64 execution of the gridding kernel's gather over the
    exported work list, compared with the oracle's scatter (gridrec.cu:540-576)."""
    p = O.params(n, a, None, None, 1, pswf_c, sampl)
    sz = O.port_sizes(p)
    rng = np.random.default_rng(n + a)
    spec = O.port_spectra(p, rng.random((a, n)), rng.random((a, n)))
    href = O.port_grid(p, theta, spec)
    items, runs, splits, tiles_v = G.worklist(n, a, theta, sampl=sampl, pswf_c=pswf_c)
    M, L2 = sz.M, sz.L / 2
    ts = 2 * 512 / sz.L
    wtbl, _ = O.port_tables(p)
    H = np.zeros((M, M), complex)
    T = 32
    seen = np.zeros(len(runs), int)
    for tile, rb, re_, slot in items:
        tu, tv = divmod(tile, tiles_v)
        p0, q0 = tu * T, tv * T
        seen[rb:re_] += 1
        for d, jlo, jhi, _ in runs[rb:re_]:
            nn, h = divmod(d, 2)
            t = np.deg2rad(float(theta[nn]))
            sg = -1.0 if h else 1.0
            js = np.arange(jlo, jhi + 1)
            U = M / 2 + sg * sz.scale * js * np.cos(t)
            V = M / 2 + sg * sz.scale * js * np.sin(t)
            for k, j in enumerate(js):
                for iu in range(max(int(np.ceil(U[k] - L2)), p0, 1),
                                min(int(np.floor(U[k] + L2)), p0 + T - 1, M - 1) + 1):
                    wu = wtbl[int(abs(U[k] - iu) * ts + 0.5)]
                    for iv in range(max(int(np.ceil(V[k] - L2)), q0, 1),
                                    min(int(np.floor(V[k] + L2)), q0 + T - 1, M - 1) + 1):
                        H[iu, iv] += wu * wtbl[int(abs(V[k] - iv) * ts + 0.5)] * spec[nn, h, j]
    assert np.all(seen == 1), "every run belongs to exactly one item"
    # split tiles: slots of a tile are consecutive and counted
    for tile, rb, re_, slot in items:
        if slot >= 0:
            sp = splits[tile]
            assert sp[1] <= slot < sp[1] + sp[2]
    return np.linalg.norm(H - href) / np.linalg.norm(href)


@pytest.mark.parametrize("n,a,sampl,C_", [(64, 48, 1.0, 6.0), (100, 37, 1.2, 6.0),
                                          (72, 30, 1.0, 4.0), (90, 25, 1.2, 7.0)])
def test_worklist_gather_equals_scatter(n, a, sampl, C_):
    th = ph.angles_deg(a)
    assert _emulate_gather(n, a, th, sampl, C_) < 1e-14


def test_worklist_gather_arbitrary_angles():
    th = np.array([-30.0, 0.0, 12.5, 90.0, 179.9, 200.0, 359.0, 45.0], np.float32)
    assert _emulate_gather(48, len(th), th) < 1e-14


def _emulate_wide(n, a, theta, sampl=1.0, pswf_c=6.0):
    """Float64 execution of grid_wide_kernel's scheme over the exported 4 x 8 list:
    every sample weights all rows and columns of the sub-tile by w(|d|), zero for
    |d| > L/2, and adds the outer product; compared with the oracle's scatter."""
    p = O.params(n, a, None, None, 1, pswf_c, sampl)
    sz = O.port_sizes(p)
    rng = np.random.default_rng(n + a)
    spec = O.port_spectra(p, rng.random((a, n)), rng.random((a, n)))
    href = O.port_grid(p, theta, spec)
    items, runs, splits, tiles_v = G.worklist(n, a, theta, sampl=sampl, pswf_c=pswf_c, wide=True)
    assert np.all(runs[:, 3] == 1) and np.all(runs[:, 2] - runs[:, 1] < 16)
    M, L2 = sz.M, sz.L / 2
    ts = 2 * 512 / sz.L
    wtbl, _ = O.port_tables(p)
    TR, TC = 4, 8
    assert tiles_v == M // TC
    rows, cols = np.arange(TR), np.arange(TC)
    wt = lambda d: np.where(d <= L2, wtbl[np.minimum((d * ts + 0.5).astype(int), 512)], 0.0)
    H = np.zeros((M, M), complex)
    seen = np.zeros(len(runs), int)
    for tile, rb, re_, slot in items:
        tu, tv = divmod(tile, tiles_v)
        p0, q0 = tu * TR, tv * TC
        seen[rb:re_] += 1
        for d, jlo, jhi, _ in runs[rb:re_]:
            nn, h = divmod(d, 2)
            t = np.deg2rad(float(theta[nn]))
            sg = -1.0 if h else 1.0
            for j in range(jlo, jhi + 1):
                u = M / 2 + sg * sz.scale * j * np.cos(t) - p0
                v = M / 2 + sg * sz.scale * j * np.sin(t) - q0
                H[p0:p0 + TR, q0:q0 + TC] += np.outer(wt(np.abs(u - rows)),
                                                      wt(np.abs(v - cols))) * spec[nn, h, j]
    assert np.all(seen == 1), "every run belongs to exactly one item"
    H[0, :] = 0
    H[:, 0] = 0
    return np.linalg.norm(H - href) / np.linalg.norm(href)


@pytest.mark.parametrize("n,a,sampl,C_", [(64, 48, 1.0, 6.0), (100, 37, 1.2, 6.0),
                                          (72, 30, 1.0, 4.0), (90, 25, 1.2, 7.0)])
def test_wide_worklist_gather_equals_scatter(n, a, sampl, C_):
    th = ph.angles_deg(a)
    assert _emulate_wide(n, a, th, sampl, C_) < 1e-14


def test_wide_worklist_arbitrary_angles():
    th = np.array([-30.0, 0.0, 12.5, 90.0, 179.9, 200.0, 359.0, 45.0], np.float32)
    assert _emulate_wide(48, len(th), th) < 1e-14


def _steps(n, P, spw=8):
    return sum(min(P, n - b) for b in range(0, n, spw * P))


def test_worklist_splits_heavy_tiles():
    items, runs, splits, tiles_v = G.worklist(2048, 1500, ph.angles_deg(1500))
    n = runs[:, 2] - runs[:, 1] + 1
    slots = np.array([_steps(int(k), int(P)) * 8 + 4 for k, P in zip(n, runs[:, 3])])
    cost = np.array([slots[b:e].sum() for _, b, e, _ in items])
    assert cost.max() <= 2048 + 1024       # kItemCap (+ one run)
    assert (items[:, 3] >= 0).sum() > 0     # the centre tiles are split
    assert np.all(np.diff(cost) <= 0)       # heaviest first
    # samples visited ~ 2 * n_ang * (pdim/2 - 1) plus the tile halo
    assert 1.0 < n.sum() / (2 * 1500 * 1023) < 1.6
    # footprints of one step are disjoint: P * max(|du|,|dv|) > L
    th = np.deg2rad(ph.angles_deg(1500).astype(np.float64))[runs[:, 0] // 2]
    step = np.maximum(np.abs(np.cos(th)), np.abs(np.sin(th))) * 2048 / 2047
    assert np.all(runs[:, 3] * step > 2 * 6.0 * (2048 / 2047) / np.pi)


def _morton(u, v):
    """Interleaved bits of (u, v), u in the even bits."""
    key = np.zeros_like(u, dtype=np.int64)
    for b in range(16):
        key |= ((u >> b) & 1).astype(np.int64) << (2 * b)
        key |= ((v >> b) & 1).astype(np.int64) << (2 * b + 1)
    return key


def test_wide_worklist_items_in_morton_order():
    """The 4 x 8 list is queued in eight cost classes, heaviest first (no heavy item
    starts late), and in Morton order of the sub-tiles within a class (neighbours run
    at the same time and share the spectra quads of the rays crossing them); an
    unsplit sub-tile is one item, and a split sub-tile's items, taken in slot order,
    cover its runs in order.  An item's cost: its samples plus 6 per run."""
    items, runs, splits, tiles_v = G.worklist(2048, 1500, ph.angles_deg(1500), wide=True)
    per_run = runs[:, 2] - runs[:, 1] + 1 + 6
    cum = np.concatenate([[0], np.cumsum(per_run)])
    cost = cum[items[:, 2]] - cum[items[:, 1]]
    cls = np.minimum(7, cost * 8 // (cost.max() + 1))
    assert np.all(np.diff(cls) <= 0) and len(np.unique(cls)) > 1
    tu, tv = items[:, 0] // tiles_v, items[:, 0] % tiles_v
    key = _morton(tu, tv)
    same = np.diff(cls) == 0
    assert np.all(np.diff(key)[same] >= 0)
    whole = items[items[:, 3] < 0, 0]
    assert len(np.unique(whole)) == len(whole)  # an unsplit sub-tile is one item
    assert items[:, 2].max() == len(runs) and np.all(items[:, 1] <= items[:, 2])
    split = items[items[:, 3] >= 0]
    for t in np.unique(split[:, 0])[:50]:
        rows = np.nonzero(items[:, 0] == t)[0]
        part = items[rows[np.argsort(items[rows, 3])]]  # in slot order
        assert np.all(np.diff(part[:, 3]) == 1)
        assert np.all(part[:-1, 2] == part[1:, 1])  # the parts cover the tile's runs in order


def test_phantom_line_integrals():
    # a centred disk of radius r: p(t) = 2 sqrt(r^2 - t^2) (in units of n/2)
    e = np.array([[1.0, 0.5, 0.5, 0.0, 0.0, 0.0]])
    n = 64
    p = ph.line_integrals(e, n, np.array([0.0, 33.0]), n / 2)
    t = (np.arange(n) - n / 2) / (n / 2)
    expect = np.where(np.abs(t) < 0.5, 2 * np.sqrt(np.clip(0.25 - t * t, 0, None)), 0) * (n / 2)
    np.testing.assert_allclose(p[0], expect, atol=1e-9)
    np.testing.assert_allclose(p[1], expect, atol=1e-9)
    s = ph.shepp_logan_sinogram(128, 90, center=64.3, noise_seed=1)
    assert s.shape == (90, 128) and s.dtype == np.float32
    assert 1.5 < s.max() < 3.0


def test_raw_counts_roundtrip():
    p = ph.line_integrals(ph.random_ellipses(4), 64, ph.angles_deg(20), 32.0) / 32.0
    raw, flat, dark = ph.raw_counts(p, seed=1)
    assert raw.dtype == np.uint16
    v = raw.astype(np.float64) - dark
    est = np.log((flat - dark) / v)
    assert np.abs(est - p).mean() < 0.05


def _build_shim(tmp_path):
    import shutil
    import subprocess
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    exe = str(tmp_path / "shim_demo")
    lib_dir = os.path.join(ROOT, "projects_b200")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cxx", "shim_demo.cpp"), "-L", lib_dir,
                    "-lgridrec_b200", f"-Wl,-rpath,{lib_dir}", "-o", exe], check=True)
    return exe


def _build_demo(tmp_path, name):
    """Builds tests/cxx/<name> (C or C++) against include/ and the library."""
    import shutil
    import subprocess
    src = os.path.join(ROOT, "tests", "cxx", name)
    cc = "gcc" if name.endswith(".c") else "g++"
    if shutil.which(cc) is None:
        pytest.skip(f"{cc} not available")
    exe = str(tmp_path / name.split(".")[0])
    lib_dir = os.path.join(ROOT, "projects_b200")
    std = ["-std=c11"] if cc == "gcc" else ["-std=c++17"]
    subprocess.run([cc, "-O2", *std, "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), src,
                    "-L", lib_dir, "-lgridrec_b200", f"-Wl,-rpath,{lib_dir}", "-lm", "-o", exe],
                   check=True)
    return exe


def test_gridrec_cpp_api_exports_and_callers_build(tmp_path):
    """The GridrecCPP calling sequence (include/gridrec_cpp_b200.h): its functions and
    row-pointer globals are exported, and a C caller and a find_shift-style C++
    caller build against include/ and the library."""
    lib = G.lib()
    for name in ("recon_init", "do_recon", "recon_free", "get_pswf", "get_filter",
                 "gr_gridrec_cpp_status", "gr_gridrec_cpp_set_device"):
        assert hasattr(lib, name), name
    for name in ("G1", "G2", "S1", "S2"):
        assert C.c_void_p.in_dll(lib, name).value is None  # null until a caller sets them
    assert C.c_long.in_dll(lib, "imgsiz").value == 0
    assert os.path.exists(_build_demo(tmp_path, "gridrec_cpp_demo.c"))
    assert os.path.exists(_build_demo(tmp_path, "find_shift_demo.cpp"))


class _PswfStruct(C.Structure):
    _fields_ = [("C", C.c_float), ("nt", C.c_int), ("lmbda", C.c_float),
                ("coefs", C.c_float * 15)]


def test_gridrec_cpp_pswf_and_filters_host():
    """get_pswf / get_filter (Gridrec5.2/pswf.cpp:36-47, filters.cpp:26-48): database
    entries by C, an unknown C reported instead of exit(2); the filter formulas,
    and an unknown name giving Shepp-Logan with the name overwritten."""
    lib = G.lib()
    lib.get_pswf.argtypes = [C.c_float, C.POINTER(C.POINTER(_PswfStruct))]
    ptr = C.POINTER(_PswfStruct)()
    lib.get_pswf(6.0, C.byref(ptr))
    assert lib.gr_gridrec_cpp_status() == 0
    assert ptr.contents.nt == 18 and abs(ptr.contents.lmbda - 0.9990188) < 1e-7
    assert abs(ptr.contents.coefs[0] - 24.95593) < 1e-4
    lib.get_pswf(5.5, C.byref(ptr))
    assert not ptr and lib.gr_gridrec_cpp_status() == -2
    FN = C.CFUNCTYPE(C.c_float, C.c_float)
    lib.get_filter.restype = FN
    lib.get_filter.argtypes = [C.c_char_p]
    x = 0.3
    want = {"shlo": abs(np.sin(np.pi * x) / np.pi), "hann": x * 0.5 * (1 + np.cos(2 * np.pi * x)),
            "hamming": x * (0.54 + 0.46 * np.cos(2 * np.pi * x)), "ramlak": x}
    for name, v in want.items():
        buf = C.create_string_buffer(name.encode(), 16)
        assert abs(lib.get_filter(buf)(x) - v) < 1e-7, name
    buf = C.create_string_buffer(b"bogus", 16)
    assert abs(lib.get_filter(buf)(x) - want["shlo"]) < 1e-7
    assert buf.value == b"shlo"


def test_cxx_shim_compiles_against_the_c_abi(tmp_path):
    """include/gridrec_b200.hpp (the GridRec-compatible class) builds and links."""
    assert os.path.exists(_build_shim(tmp_path))


def test_geom_recurrence_needs_no_angle_list():
    """geom 1 (GridrecCPP's uniform angles from its FP32 recurrence) takes no theta list;
    geom 3 is rejected.  Host-only (the work-list export)."""
    ni, nr, tv = C.c_int(), C.c_int(), C.c_int()
    p, _ = G.make_params(64, 30, np.zeros(30, np.float32))
    p.theta_deg = None
    p.geom = 1
    assert G.lib().gr_worklist_export(C.byref(p), C.byref(ni), C.byref(nr), C.byref(tv), None,
                                      None, None, 0, 0) == 0
    assert ni.value > 0 and nr.value > 0
    p.geom = 3
    assert G.lib().gr_worklist_export(C.byref(p), C.byref(ni), C.byref(nr), C.byref(tv), None,
                                      None, None, 0, 0) == -1


def test_wide_worklist_has_empty_items_past_the_runs():
    """Tiles that no sample reaches (the grid's corners) get empty items whose
    run_begin can equal the run count: the 16-pair kernel must read no run record
    for them (the GPU goldens run such a case)."""
    items, runs, splits, tv = G.worklist(120, 72, ph.angles_deg(72), sampl=1.2, pswf_c=7.0,
                                         wide=True)
    empty = items[items[:, 1] == items[:, 2]]
    assert len(empty) > 0 and (empty[:, 1] == len(runs)).any()


@pytest.mark.parametrize("seed", [11, 12, 13])
def test_wide_worklist_random_geometries(seed):
    """Seeded random geometries (width, angle count, irregular angle list,
    oversampling, PSWF parameter): the 16-pair kernel's 4 x 8 work list covers
    exactly the oracle's scatter, in float64."""
    rng = np.random.default_rng(seed)
    n = int(rng.integers(40, 110))
    a = int(rng.integers(12, 40))
    th = np.sort(rng.uniform(-20.0, 200.0, a)).astype(np.float32)
    sampl = float(rng.choice([1.0, 1.2, 1.5]))
    C_ = float(rng.choice([4.0, 5.0, 6.0, 7.0]))
    assert _emulate_wide(n, a, th, sampl, C_) < 1e-14


@pytest.mark.parametrize("n,a,sampl,C_", [(2048, 1500, 1.0, 6.0), (120, 72, 1.2, 7.0),
                                          (64, 9, 1.0, 4.0)])
def test_wide_worklist_runs_fit_the_precomputed_weights(n, a, sampl, C_):
    """The 16-pair kernel's weights are computed once per list, one 48-byte
    record per run sample, each run tagged with the sub-tile of its item: every
    run belongs to exactly one item, runs hold 1..16 samples (the kernel's
    staging and weight buffers), and the record count fits an int."""
    items, runs, splits, tv = G.worklist(n, a, ph.angles_deg(a), sampl=sampl, pswf_c=C_,
                                         wide=True)
    owner = np.zeros(len(runs), np.int64)
    for it in items:
        owner[it[1]:it[2]] += 1
    assert (owner == 1).all()
    lens = runs[:, 2] - runs[:, 1] + 1
    assert lens.min() >= 1 and lens.max() <= 16
    assert (runs[:, 3] == 1).all()
    assert int(lens.sum()) < 2**31 - 1


def test_no_gpu_means_an_error_not_a_fallback():
    """Without a usable GPU every compute entry point fails loudly: plan creation
    returns GR_ERR_CUDA (there is no CPU path to fall back to)."""
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(G.GrError) as err:
        G.Plan(64, 32, ph.angles_deg(32))
    assert "GR_ERR_CUDA" in str(err.value)


def test_on_stream_leaves_the_current_stream_for_none_and_raw_handles():
    """Raw int stream handles and None keep the caller's current stream (no torch
    stream context is entered); torch streams are entered (checked on the GPU)."""
    import contextlib

    from projects_b200 import gridrec as G
    assert isinstance(G._on_stream(None), contextlib.nullcontext)
    assert isinstance(G._on_stream(0), contextlib.nullcontext)
    assert isinstance(G._on_stream(12345), contextlib.nullcontext)
