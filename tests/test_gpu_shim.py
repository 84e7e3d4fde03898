"""GPU test of the header-only C++ GridRec class (include/gridrec_b200.hpp)."""
import subprocess

import numpy as np
import pytest

from oracle import oracle as O
from projects_b200 import phantom as ph
from tests.test_host import _build_shim

pytestmark = pytest.mark.gpu


def test_cxx_gridrec_class_matches_oracle(tmp_path):
    n, a = 256, 180
    s1 = ph.shepp_logan_sinogram(n, a, center=128.0, noise_seed=7)
    s2 = ph.shepp_logan_sinogram(n, a, center=128.0, noise_seed=8)
    np.stack([s1, s2]).astype(np.float32).tofile(tmp_path / "in.bin")
    exe = _build_shim(tmp_path)
    subprocess.run([exe, str(tmp_path / "in.bin"), str(tmp_path / "out.bin"), str(n), str(a), "2"],
                   check=True)
    out = np.fromfile(tmp_path / "out.bin", np.float32).reshape(2, n, n)
    o1, o2 = O.port_gridrec_pair(s1, s2, ph.angles_deg(a), filter=2)
    m = o1.shape[0]
    assert ph.rel_l2(out[0, :m, :m], o1[:, :m]) < 1e-3
    assert ph.rel_l2(out[1, :m, :m], o2[:, :m]) < 1e-3
    assert np.all(out[:, m:, :] == 0) and np.all(out[:, :, m:] == 0)
