"""The mini-app executable's host-only paths (no GPU needed): the usage text
of Source/main.cpp's driver and the rejection of max_level > 0."""
from __future__ import annotations

import os
import subprocess


def test_miniapp_usage_and_rejections(pkg):
    exe = os.path.join(os.path.dirname(pkg.castro.lib_path(False)), "castro_b200.ex")
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and "n_cell: The number of zones per dimension" in out.stdout
    out = subprocess.run([exe, "n_cell=16", "max_level=1"], capture_output=True, text=True, timeout=120)
    assert out.returncode == 1 and "max_level" in out.stderr
