import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built CUDA library")


def testdata(*parts):
    """A file of the reference's test data (the nickel scan, the nickel and GaN masters, kikuchipy's
    orientations of the scan): under $ZEBSDSOLVE_TESTDATA, else tests/data/ (filled by
    tests/golden/copy_testdata.sh); None where absent."""
    from pathlib import Path

    for base in (os.environ.get("ZEBSDSOLVE_TESTDATA"), os.path.join(ROOT, "tests", "data")):
        if base and Path(base, *parts).is_file():
            return Path(base, *parts)
    return None
