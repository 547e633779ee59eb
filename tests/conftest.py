import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built native library")


def _cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


def pytest_terminal_summary(terminalreporter):
    """After a run with GPU parity tests: per test and output, how many entries pass at plain
    1e-12 relative (no floor) and how many needed one of the tolerance floors. Written as JSON to
    the path in $PARITY_REPORT when that is set."""
    gp = sys.modules.get("tests.gpu_parity")
    log = getattr(gp, "STRICT_LOG", None)
    if not log:
        return
    import json

    rows = []
    terminalreporter.write_sep("-", "parity: entries within plain 1e-12 relative (rest needed a floor)")
    for test, strict in log:
        for key, (tot, ok, idx, cls) in sorted(strict.items()):
            rows.append({"test": test, "output": key, "entries": tot, "strict": ok, "needed_floor": tot - ok,
                         "fraction_needed_floor": (tot - ok) / max(1, tot), "first_floor_indices": idx,
                         "floor_needed": {"summation_order": cls[0], "cancellation": cls[1], "libm_ulp": cls[2]}})
            terminalreporter.write_line(f"{test} {key}: {ok}/{tot} strict, {tot - ok} needed a floor "
                                        f"({(tot - ok) / max(1, tot):.2e}; summation order {cls[0]}, "
                                        f"cancellation {cls[1]}, libm ulp {cls[2]})")
    path = os.environ.get("PARITY_REPORT")
    if path:
        with open(path, "w") as f:
            json.dump(rows, f, indent=1)
