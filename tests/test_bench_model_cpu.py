"""The measurement model behind the bench line, on CPU: the compulsory HBM bytes
per launch that the roofline divides by the kernel time, and the autotuner's
candidate labels (its timing table must tell every knob apart)."""
from __future__ import annotations

import importlib.util
import os
import sys

from conftest import PKG_DIR, ROOT, load_package

NS = 2
NV, NQF, NQS, NTF = 7 + NS, 8 + NS, 6 + NS, 7 + NS


def _bench():
    spec = importlib.util.spec_from_file_location("bench_model", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_kernel_bytes_headline():
    pkg = load_package()
    kb = _bench().kernel_bytes(pkg.configs.sedov128_pert(), NS)
    assert set(kb) == {"front", "ghost", "trace", "trace2", "riemann1", "riemann2", "riemann3", "riemann23", "update"}
    n = 128
    vd, g1d, g4d = n ** 3, (n + 2) ** 3, (n + 8) ** 3
    # ghost fills the domain halo of Q (grow 4) and Sborder (grow 1), read and written once
    assert kb["ghost"] == 8 * ((g4d - vd) * NQF * 2 + (g1d - vd) * NV * 2)
    # the face boxes of the domain: tbx[d][d] is (n+1) x (n+2)^2, ebx[d] is (n+1) x n^2
    tdd = 3 * (n + 1) * (n + 2) ** 2
    tab = 6 * (n + 1) * (n + 2) * n
    eb = 3 * (n + 1) * n * n
    assert kb["riemann1"] == 8 * (tdd * 2 * NQS + g4d * 2 + tdd * NTF)
    assert kb["riemann2"] == 8 * (tdd * 2 * NQS + tdd * NTF + g4d * 2 + tab * NTF)
    assert kb["riemann3"] == 8 * (eb * 2 * NQS + tab * NTF + g1d * NV + g1d + g4d * 2 + eb * (NV + 1))
    # the fused kernel reads what both read, less the cross-flux records the pair passes through HBM
    assert kb["riemann23"] == kb["riemann2"] + kb["riemann3"] - 8 * (2 * tab * NTF + g4d * 2 + eb * 2 * NQS)
    # the two trace kernels write the 2 x NQS face-state components between them
    assert kb["trace"] + kb["trace2"] == 8 * (g4d * (9 + NS) + tdd * 2 * NQS + 2 * g1d)
    # front and update walk the 64 boxes of 32^3: the per-box terms add up to the domain's
    assert kb["front"] == 8 * vd * (NV * 3 + NQF)
    assert kb["update"] == 8 * (vd * NV * 2 + eb * (NV + 1))


def test_kernel_bytes_scale_with_instances():
    pkg = load_package()
    b = _bench()
    one = b.kernel_bytes(pkg.configs.sedov128_pert(), NS)
    cfg = pkg.configs.sedov128_pert()
    two = dict(cfg, instances=cfg["instances"] * 2)
    assert b.kernel_bytes(two, NS) == {k: 2 * v for k, v in one.items()}


def test_autotune_labels_distinct():
    sys.path.insert(0, PKG_DIR)
    import autotune as A

    labels = set()
    for knob, values in A.KNOBS:
        for v in values:
            labels.add(A.key(dict(A.DEFAULTS, **{knob: v})))
    n = 1 + sum(len([v for v in vals if v != A.DEFAULTS[k]]) for k, vals in A.KNOBS)
    assert len(labels) == n
    assert set(A.DEFAULTS) == {k for k, _ in A.KNOBS}


def test_reference_algorithm_fp64_fraction():
    """The FP64 fraction on the reference algorithm's counted operations
    (profiles/fp64_ops_reference_algorithm.json, oracle/count_ops.py):
    zone-updates/s x counted flops / peak, beside the executed-work figure."""
    b = _bench()
    ops = b.reference_algorithm_ops("sedov128_pert")
    assert ops and ops["zones"] == 128 ** 3 and ops["boxes"] == 64
    per = ops["per_zone_update"]
    assert abs(per["add"] + per["mul"] + per["div"] + per["sqrt"] + per["transcendental"]
               - ops["flops_per_zone_update"]) < 1.0
    zones, ms, peak = 128 ** 3, 3.4, 33.8
    r = b.path_roofline(zones, ms, 144, 6500.0, 13000.0, peak, ops["flops_per_zone_update"])
    want = zones * ops["flops_per_zone_update"] / (ms * 1e-3) / 1e12
    assert abs(r["fp64_reference_algorithm"]["achieved"] - want) < 1e-9 * want
    assert abs(r["fp64_reference_algorithm"]["frac"] - want / peak) < 1e-12
    assert r["fp64"]["flops_per_zone_update"] == 13000.0
