"""Shared pytest setup: the `gpu` marker, import paths and cached problems."""
import functools
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "parcel-legacy_b200"), os.path.join(ROOT, "oracle"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long-running CPU test")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@functools.lru_cache(maxsize=None)
def golden():
    import json
    with open(os.path.join(ROOT, "tests", "golden", "reference_templates.json")) as f:
        return json.load(f)


@functools.lru_cache(maxsize=4)
def poisson_reference(g: int):
    from parcel_b import problems
    return problems.poisson3d_reference(g, g, g)
