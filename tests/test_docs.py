"""The binding a maintainer would add (the ctypes stub printed in INTEGRATION.md) runs as written
against the built library: its struct definitions and calls are valid.  Without a device the
calls report errors through nmlmc_last_error instead of exiting, so the stub's final check is
replaced by a print."""
import os
import re
import subprocess
import sys

from conftest import ROOT


def test_integration_ctypes_stub_runs():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    code = re.findall(r"```python\n(.*?)```", text, re.S)[0]
    assert "ctypes.CDLL" in code and "model_sample" in code
    code = code.replace("assert lib.nmlmc_last_error() == 0", "print('status', lib.nmlmc_last_error())")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr[-2000:]
    assert "status" in out.stdout
