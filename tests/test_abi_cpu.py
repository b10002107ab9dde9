"""CPU tests of the product's host side: the C-ABI library loads and exports
every symbol of include/castro_b200.h, the table writer matches the reader's
format, and the workload generators produce valid BoxArrays.  No GPU calls."""
from __future__ import annotations

import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "castro_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*[A-Za-z_][\w ]*?[\s*]+([A-Za-z_]\w*)\s*\(", src, flags=re.M)
    return sorted(set(n for n in names if n not in ("if", "while", "for", "return", "sizeof")))


@pytest.fixture(scope="module")
def built(pkg):
    return pkg.build.build() if hasattr(pkg, "build") else __import__("build")


def test_header_and_binding_agree(pkg):
    decl = declared_functions()
    assert len(decl) >= 50
    assert sorted(pkg.castro.ABI_SYMBOLS) == decl


def test_enum_constants_agree(pkg):
    """The binding's mode and boundary-condition constants are the header's enum values."""
    src = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    enums = {k: int(v) for k, v in re.findall(r"(CASTRO_(?:MODE|BC)_\w+)\s*=\s*(\d+)", src)}
    assert enums["CASTRO_MODE_PLAIN"] == pkg.castro.MODE_PLAIN
    assert enums["CASTRO_MODE_BATCHED"] == pkg.castro.MODE_BATCHED
    assert enums["CASTRO_MODE_PLAIN_BOX"] == pkg.castro.MODE_PLAIN_BOX
    assert enums["CASTRO_MODE_PERSISTENT"] == pkg.castro.MODE_PERSISTENT
    assert len({v for k, v in enums.items() if k.startswith("CASTRO_MODE_")}) == 4


@pytest.mark.parametrize("exact", [False, True])
def test_library_exports_every_symbol(pkg, exact):
    import importlib

    b = importlib.import_module("mini_castro_b200.build")
    b.build()
    L = pkg.castro.load(exact)
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing
    assert L.castro_exact_build() == (1 if exact else 0)
    assert L.castro_version() >= 100


def test_library_reports_errors_without_gpu(pkg, table, tmp_path_factory):
    """Entry points report a clean error (no crash) when CUDA is unavailable or
    the table has not been loaded."""
    from conftest import cuda_available

    if cuda_available():
        pytest.skip("a GPU is present; covered by the gpu tests")
    L = pkg.castro.load(False)
    L.castro_clear_error()
    L.castro_eos_init_path(table.encode())
    assert L.castro_last_error() == 1     # the table parses; the device upload fails (CASTRO_ERR_CUDA)
    assert L.castro_error_string()
    L.castro_clear_error()
    # host-side table faults are found before any CUDA call (CASTRO_ERR_TABLE_IO)
    with open(table) as fp:
        lines = fp.readlines()
    d = tmp_path_factory.mktemp("tables")
    (d / "truncated.dat").write_text("".join(lines[:1000]))
    lines[7] = "1.0 x2.0\n"
    (d / "garbled.dat").write_text("".join(lines))
    del lines
    for name in ("truncated.dat", "garbled.dat", "absent.dat"):
        assert L.castro_eos_init_path(str(d / name).encode()) == 3, name
        L.castro_clear_error()
    lo = (0, 0, 0)
    L.compute_temp(pkg.castro.ivec(lo), pkg.castro.ivec(lo), None, pkg.castro.ivec(lo), pkg.castro.ivec(lo))
    assert L.castro_last_error() == 2   # CASTRO_ERR_NO_TABLE
    L.castro_clear_error()


def test_table_layout(pkg, table):
    d, t = pkg.helm_table.grid()
    assert d.shape == (541,) and t.shape == (201,)
    assert d[0] == 1e-12 and t[0] == 1e3
    with open(table) as fp:
        first = fp.readline().split()
    assert len(first) == 9
    nlines = sum(1 for _ in open(table))
    assert nlines == 541 * 201 * 4
    # thermodynamic consistency of the analytic table: p = d^2 df/dd = dpdf * d
    tabs = pkg.helm_table.ideal_nd_tables()
    f, fd = tabs[0][0], tabs[0][1]
    dpdf = tabs[1][0]
    D = d[None, :]
    np.testing.assert_allclose(D * D * fd, dpdf * D, rtol=1e-14)


def test_table_is_deterministic(pkg, table):
    # the generator is pure numpy; its output is pinned by this digest
    assert pkg.helm_table.sha256(table) == "ee3dde28879fac34c9f23ff7590b7158758a2762e4bff4d07d13f49da93f6f23"


@pytest.mark.parametrize("name", ["sedov64", "sedov128_pert", "batched", "large", "reference"])
def test_workload_boxarrays_tile_the_domain(pkg, name):
    cfg = pkg.configs.WORKLOADS[name](scale=4 if name != "batched" else 8)
    for inst in cfg["instances"]:
        n = [h - l + 1 for l, h in zip(inst["dom_lo"], inst["dom_hi"])]
        cover = np.zeros(n, dtype=np.int32)
        for lo, hi in inst["boxes"]:
            assert all(h >= l for l, h in zip(lo, hi))
            cover[lo[0]:hi[0] + 1, lo[1]:hi[1] + 1, lo[2]:hi[2] + 1] += 1
        assert (cover == 1).all()


def test_batched_workload_shape(pkg):
    cfg = pkg.configs.batched()
    insts = cfg["instances"]
    assert len(insts) == 33
    sizes = set()
    for lo, hi in insts[0]["boxes"]:
        sizes.update(h - l + 1 for l, h in zip(lo, hi))
    assert sizes <= {16, 24, 32, 48, 64}
    for inst in insts[1:]:
        n = inst["dom_hi"][0] + 1
        assert 32 <= n <= 96
        assert 1e49 <= inst["problem"]["exp_energy"] <= 1e51
        assert 0.1 <= inst["problem"]["dens_ambient"] <= 10


def test_perturbation_field(pkg):
    g = pkg.configs.gaussian_field((32, 32, 32), 4.0, 1)
    assert abs(g.mean()) < 1e-12 and abs(g.std() - 1) < 1e-12
    g2 = pkg.configs.gaussian_field((32, 32, 32), 4.0, 1)
    assert np.array_equal(g, g2)
    # smoothed over ~4 zones: neighbouring values strongly correlated
    c = np.corrcoef(g[:-1].ravel(), g[1:].ravel())[0, 1]
    assert c > 0.9
