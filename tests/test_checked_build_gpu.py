"""The S3TTMc and Tucker GPU suites rerun against the bounds-checked build of
the library (libsymprop_b200_checked.so, `make -C symprop_b200 checked`):
every index the S3TTMc kernels derive from the tensor (chunk ranges, owner
ids, level and tile offsets, output and partial-row offsets, split-row
slots, unpack positions) is tested on the device there, and a failed check
is a SYMPROP_ERR_CUDA status naming the site.  The suites passing means no
check fired on any of their shapes."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
pytestmark = pytest.mark.gpu


def test_s3ttmc_and_tucker_suites_under_the_checked_build(gpu):
    lib = os.path.join(ROOT, "symprop_b200", "libsymprop_b200_checked.so")
    assert os.path.exists(lib), "build it with: make -C symprop_b200 checked"
    env = dict(os.environ, SYMPROP_B200_LIB=lib)
    probe = subprocess.run([sys.executable, "-c", "import symprop_b200 as s; s.lib(); print(s.LIB_PATH)"],
                           cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert probe.returncode == 0 and probe.stdout.strip() == lib, probe.stderr
    r = subprocess.run([sys.executable, "-m", "pytest", "tests/test_s3ttmc_gpu.py", "tests/test_tucker_gpu.py",
                        "tests/test_failures_gpu.py", "-m", "gpu", "-q", "-x", "-p", "no:cacheprovider"],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=1200)
    assert r.returncode == 0, r.stdout[-4000:] + r.stderr[-2000:]
    assert " passed" in r.stdout.splitlines()[-1]
