"""Copies between pageable host arrays and the device go through pinned
staging buffers in chunks (hos_b200/csrc/hos_stage.cu).  Each case runs in a
child process with a small chunk (so that an array spans many chunks and ends
in a partial one) and again with staging off; the state, a step and the RHS
must come back bitwise the same, and a round trip must return the input."""
import os
import subprocess
import sys

import numpy as np
import pytest

from .conftest import ROOT

pytestmark = pytest.mark.gpu

CHILD = r"""
import sys
import numpy as np
from hos_b200.field import HosField
out = sys.argv[1]
nx, ny = 256, 1024
f = HosField(nx, ny, order=4)
rng = np.random.default_rng(7)
shape = (2, ny // 2 + 1, nx)  # two fields, ky rows of kx lines
u = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) * 1e-3
f.set_state_spectral(u, 0.0)
back, t = f.state_spectral()
eta = rng.standard_normal((nx, ny)) * 1e-2
phi = rng.standard_normal((nx, ny)) * 1e-2
r = f.rhs(back, 0.0)
f.set_state_physical(eta, phi, 0.0)
pe, pp = f.state_physical()
f.set_state_spectral(back, 0.0)
f.step(0.01, 3)
s3, t3 = f.state_spectral()
np.savez(out, u=u, back=back, r=r, pe=pe, pp=pp, s3=s3)
"""


def run_child(tmp_path, name, env_extra):
    out = os.path.join(str(tmp_path), name + ".npz")
    env = dict(os.environ, PYTHONPATH=ROOT, **env_extra)
    p = subprocess.run([sys.executable, "-c", CHILD, out], env=env, cwd=ROOT, capture_output=True, text=True,
                       timeout=300)
    assert p.returncode == 0, p.stderr[-2000:]
    return np.load(out)


def test_staged_copies_match_direct_copies(tmp_path):
    staged = run_child(tmp_path, "staged", {"HOS_STAGE_CHUNK_KB": "64", "HOS_COPY_THREADS": "3"})
    direct = run_child(tmp_path, "direct", {"HOS_STAGE": "0"})
    # 2 x 256 x 513 complex doubles = 4,202,496 bytes: 64 full chunks of 64 KB and a partial one
    assert staged["u"].nbytes % (64 << 10) != 0
    np.testing.assert_array_equal(staged["back"], staged["u"])
    for k in ("back", "r", "pe", "pp", "s3"):
        np.testing.assert_array_equal(staged[k], direct[k], err_msg=k)


CHILD_LARGE = r"""
import sys
import numpy as np
from hos_b200.field import HosField
out = sys.argv[1]
n = 2048  # the packed state is 67 MB: more than one window of the 64 MB staging buffer
f = HosField(n, n, order=3)
rng = np.random.default_rng(11)
shape = (2, n // 2 + 1, n)
u = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
f.set_state_spectral(u, 0.0)
back, _ = f.state_spectral()
np.savez(out, ok=np.array([np.array_equal(back, u)]))
"""


def test_staged_copies_longer_than_the_staging_buffer(tmp_path):
    out = os.path.join(str(tmp_path), "large.npz")
    p = subprocess.run([sys.executable, "-c", CHILD_LARGE, out], env=dict(os.environ, PYTHONPATH=ROOT), cwd=ROOT,
                       capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr[-2000:]
    assert bool(np.load(out)["ok"][0])
