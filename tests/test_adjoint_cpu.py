"""Reverse-mode stages on the CPU: the host build of castro_adjoint.cuh
(lib/castro_adjoint_selftest) checks every stage adjoint -- EOS (implicit
function derivative of the Newton root), clean_state, ctoprim, estdt, PPM
trace with flattening, CGF Riemann, trans1/trans2 -- against central finite
differences of its forward stage on seeded random inputs."""
from __future__ import annotations

import os
import subprocess


def test_stage_adjoints_match_finite_differences(pkg, table):
    exe = os.path.join(os.path.dirname(pkg.castro.lib_path(False)), "castro_adjoint_selftest")
    assert os.path.exists(exe), "build with mini-castro_b200/build.py"
    r = subprocess.run([exe, table, "300"], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ALL OK" in r.stdout
    stages = [l.split()[0] for l in r.stdout.splitlines() if " cases " in l]
    for s in ("riemann_cgf", "trans1_state", "trans2_state", "trace_zone", "trace+uflatten", "eos_vjp", "ctoprim",
              "clean_state", "estdt"):
        assert s in stages, s
