"""Shared test set-up: import paths, the `gpu` marker, case fixtures."""
import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libdalm.so")


def package():
    return importlib.import_module("3dalm_b200")


def casegen():
    return importlib.import_module("3dalm_b200.casegen")


@pytest.fixture
def make_case(tmp_path):
    """make_case(name, **overrides) -> (spec, mesh, case_dir, U0, profile)."""
    cg = casegen()

    def _make(name, **over):
        spec = cg.config(name, **over)
        d = tmp_path / spec.name
        mesh = cg.write_case(spec, str(d))
        return spec, mesh, str(d), cg.initial_velocity(spec, mesh), cg.inflow_profile(spec, mesh)

    return _make
