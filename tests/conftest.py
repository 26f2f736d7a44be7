import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
for p in (ROOT, ROOT / "treams-rs_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


def read_table(name):
    """Rows `key: values` of a golden table, comments skipped."""
    rows = []
    for line in (GOLDEN / name).read_text().splitlines():
        line = line.strip()
        if not line or line.startswith("#"):
            continue
        key, _, vals = line.partition(":")
        rows.append((key.split(), vals.split()))
    return rows


@pytest.fixture(scope="session")
def ctx():
    import treams_b200 as t
    c = t.Context(0)
    yield c
    c.close()
