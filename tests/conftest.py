"""Test configuration: the ``gpu`` marker, import paths and shared fixtures.

Tests marked ``gpu`` need a B200 and the built libsoapb200.so; everything else
runs on the CPU (the FP64 oracle, host-side logic, the library's host-only
entry points and its exported symbols)."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libsoapb200.so")


def pytest_collection_modifyitems(config, items):
    # GPU tests cannot run without a device; report them as skipped instead of
    # failing the CPU suite when someone runs everything on a CPU-only host.
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:  # pragma: no cover
        has_gpu = False
    if has_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


def site_rel_err(a, b):
    """max_i |a_i - b_i|_inf / |b_i|_inf over sites (rows)."""
    a = np.asarray(a)
    b = np.asarray(b)
    return float((np.abs(a - b).max(axis=1) / np.abs(b).max(axis=1)).max())


def max_rel_err(a, b):
    """max |a - b| / max |b| over every element."""
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max())


# The accuracy gates of the mixed-precision path against the FP64 oracle.
SOAP_TOL = 1.0e-6   # max over sites of |soap - ref|_inf / |ref|_inf
VJP_TOL = 1.0e-5    # max |pair - ref| / max |ref|
FP64_TOL = 1.0e-8   # the plain FP64 path (W's conditioning amplifies ulp-level
                    # exp/erf differences to ~1e-10)
