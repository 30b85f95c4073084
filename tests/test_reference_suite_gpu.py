"""The reference's own hot-path tests, run against this library.

With $PIVTOOLS_REF naming a checkout of the reference, its tree is copied to a
scratch directory, the GPU libraries are dropped into the copy's
pivtools_cli/lib/ under the reference's names (libbulkxcorr2d.so,
libfusedwarp.so, libkspacefit.so), and the reference's own tests of the path run
unmodified through the reference's own loaders (ctypes.CDLL of those paths,
kspace_lm_fitting._load_kspace_lib with its staleness guard, the
pivtools_cpu_supported check):

  unit-tests/test_instantaneous_peaks.py   fitter and bulkxcorr2d entry points
  unit-tests/test_peakfit_batch.py         batch fitter vs scalar
  unit-tests/test_fused_warp.py            warp vs cv2 / NumPy references
  unit-tests/test_kspace_c_fit.py          k-space C vs the NumPy oracle
  unit-tests/test_kspace_c_constants.py    constant-drift guard
  unit-tests/test_cpu_supported.py         loader guard

Without $PIVTOOLS_REF the test is skipped.  Outcomes the GPU library cannot
share with the reference's CPU build are listed in EXPECTED_FAILURES with the
reason.
"""

import os
import shutil
import subprocess
import sys

import pytest

from pivtools_b200 import _lib

pytestmark = pytest.mark.gpu

SUITE = ["unit-tests/test_instantaneous_peaks.py", "unit-tests/test_peakfit_batch.py",
         "unit-tests/test_fused_warp.py", "unit-tests/test_kspace_c_fit.py",
         "unit-tests/test_kspace_c_constants.py", "unit-tests/test_cpu_supported.py"]

# node id -> why the GPU library's result differs from the reference CPU build's
EXPECTED_FAILURES: dict[str, str] = {}


def test_reference_suite_against_gpu_libraries(tmp_path):
    ref = os.environ.get("PIVTOOLS_REF", "")
    if not ref or not os.path.isdir(os.path.join(ref, "unit-tests")):
        pytest.skip("set PIVTOOLS_REF to a reference checkout to run its own tests against this library")
    tree = tmp_path / "ref"
    shutil.copytree(ref, tree, ignore=shutil.ignore_patterns("*.so", "*.dll", "*.exe", "__pycache__", ".git",
                                                             "pivtools_gui"))
    libdir = tree / "pivtools_cli" / "lib"
    for name in ("libbulkxcorr2d.so", "libfusedwarp.so", "libkspacefit.so"):
        shutil.copy2(_lib.lib_path(name), libdir / name)
        os.utime(libdir / name)          # newer than the sources beside it (the loader's staleness guard)
    env = dict(os.environ, PYTHONPATH=str(tree), PYTHONDONTWRITEBYTECODE="1")
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-rfE", "-p", "no:cacheprovider", *SUITE],
                       cwd=tree, env=env, capture_output=True, text=True, timeout=1800)
    print(r.stdout[-6000:])
    print(r.stderr[-2000:])
    failed = [ln.split()[1] for ln in r.stdout.splitlines() if ln.startswith(("FAILED", "ERROR"))]
    unexpected = [f for f in failed if f not in EXPECTED_FAILURES]
    assert not unexpected, unexpected
    assert " passed" in r.stdout
