"""Test set-up: the `gpu` marker (tests that need a CUDA device; the rest run on the CPU) and the golden fixtures.

Fixtures in tests/golden were made from the reference implementation by tests/golden/make_golden.py; nothing here
reads the reference itself.
"""
import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT))

CASES = ["diff_auto_trapezoid", "diff_midpoint_hat", "adj_0_180", "adj_0_360", "adj_0_90", "adj_180_0", "al5_small",
         "ti8_small"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def load_case(name):
    d = dict(np.load(GOLDEN / f"{name}.npz"))
    d["cfg"] = json.loads(str(d["cfg"]))
    d["material"] = json.loads(str(d["material"]))
    d["kernel"] = str(d["kernel"])
    d["quadrature"] = str(d["quadrature"])
    return d


@pytest.fixture(scope="session")
def golden():
    cache = {}

    def get(name):
        if name not in cache:
            cache[name] = load_case(name)
        return cache[name]
    return get


def case_inputs(d):
    """(cfg, Material, MatrixGrid) of a golden case, built with this package's own classes."""
    from diffractom_b200.grid import MatrixGrid
    from diffractom_b200.material import Material
    mat = Material.from_lattice_parameters(**d["material"])
    grid = MatrixGrid(d["rot"], d["sigma64"])
    return d["cfg"], mat, grid


def case_geometry(d):
    from diffractom_b200.geometry import OperatorGeometry
    cfg, mat, grid = case_inputs(d)
    return OperatorGeometry(cfg, mat, grid, normalized=True, quadrature=d["quadrature"], radon_kernel=d["kernel"])
