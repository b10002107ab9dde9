"""The mini-app executable (the counterpart of Source/main.cpp's driver): its
runtime keys, its report lines, and the blast radius it prints against the
oracle's level driver on the same problem (16^3 reference problem, 13 species,
periodic, eight 8^3 boxes)."""
from __future__ import annotations

import os
import re
import subprocess

import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", ["batched", "persistent", "plain", "plain_box"])
def test_miniapp_report_and_blast_radius(pkg, table, oracle, mode):
    exe = os.path.join(os.path.dirname(pkg.castro.lib_path(False)), "castro_b200.ex")
    assert os.path.exists(exe), exe
    out = subprocess.run([exe, "n_cell=16", "max_box_size=8", "max_step=4", "diagnostic_interval=2",
                          f"table={table}", f"mode={mode}"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    txt = out.stdout
    assert "Starting mini-Castro..." in txt
    assert "n_cell = 16" in txt and "max_box_size = 8" in txt
    assert "Number of timesteps taken: 4" in txt
    fom = re.search(r"Figure of Merit \(zones / usec\): ([0-9.eE+-]+)", txt)
    assert fom and float(fom.group(1)) > 0
    lines = re.findall(r"Blast radius at step (\d+), time ([0-9.eE+-]+): ([0-9.eE+-]+) km", txt)
    assert [int(s) for s, _, _ in lines] == [2, 4]

    cfg = pkg.configs.reference(scale=8, max_box=64)
    oracle.network_init(*cfg["network"])
    oracle.eos_init(table)
    inst = cfg["instances"][0]
    lev, _ = oracle.level_from_instance(inst, pkg.configs.nvar(cfg))
    for step, t, r in lines:
        while lev.steps < int(step):
            lev.coarse_step(-1.0)
        ro, _ = lev.blast_radius()
        assert float(t) == pytest.approx(lev.time, rel=1e-6)
        assert abs(float(r) - ro / 1e5) <= 1.5e-3, (step, r, ro / 1e5)
