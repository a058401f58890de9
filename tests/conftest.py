"""Shared fixtures.  GPU tests carry @pytest.mark.gpu and run only on a B200
box (python -m pytest tests -m gpu); everything else runs on the CPU."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

SEED = 0x9E3779B97F4A7C15  # the reference's regression seed (tests/measure_digit_bits.cpp:140)


def load_recipe(relpath: str):
    """Load a build recipe from its file.  Importing bigint_b200.build through
    the package would run the package's __init__, which needs the library the
    recipe builds."""
    import importlib.util

    name = "_recipe_" + relpath.replace("/", "_").replace(".", "_")
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(ROOT, relpath))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    sys.modules[name] = mod
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def port():
    from oracle.build import build_port
    from oracle.pyoracle import Port

    build_port()
    return Port()


@pytest.fixture(scope="session")
def reference():
    from oracle.pyoracle import Reference, have_reference

    if not have_reference():
        pytest.skip("oracle/_ref (the compiled reference) is not built on this machine")
    r = Reference()
    r.init_thread_pool(8)
    return r


@pytest.fixture(scope="session")
def reference_gpu():
    """The unmodified reference BigInt with ntt::mul / fft::mul hooked to the
    GPU engine (bigint_b200/hooks/reference_hook.cpp)."""
    from oracle.pyoracle import REF_GPU_SO, Reference, have_reference_gpu

    if not have_reference_gpu():
        pytest.skip("oracle/_ref/libbigint_ref_gpu.so (reference + GPU hook) is not built")
    r = Reference(REF_GPU_SO)
    r.init_thread_pool(1)  # the hook initializes the engine
    return r


@pytest.fixture(scope="session")
def golden():
    path = os.path.join(ROOT, "tests", "golden", "golden.npz")
    return dict(np.load(path, allow_pickle=False))


@pytest.fixture(scope="session")
def bb():
    """The CUDA engine, initialized on device 0 (GPU tests only)."""
    import bigint_b200

    bigint_b200.init(0)
    return bigint_b200


def rand_limbs(rng, n, top=True):
    x = rng.integers(0, 2**64, n, dtype=np.uint64, endpoint=False)
    if top and n:
        x[-1] |= np.uint64(1 << 63)
    return x


def rand_digits(rng, n):
    d = rng.integers(0, 1 << 28, n, dtype=np.uint32)
    if n and d[-1] == 0:
        d[-1] = 1
    return d


def golden_u64_cases(g):
    i = 0
    while f"u64_{i:03d}_a" in g:
        a, b, c = g[f"u64_{i:03d}_a"], g[f"u64_{i:03d}_b"], g[f"u64_{i:03d}_c"]
        yield str(g[f"u64_{i:03d}_kind"]), a, (None if b.size == 0 else b), c
        i += 1


def golden_digit_cases(g):
    j = 0
    while f"dig_{j:03d}_a" in g:
        a, b = g[f"dig_{j:03d}_a"], g[f"dig_{j:03d}_b"]
        yield (a, None if b.size == 0 else b, int(g[f"dig_{j:03d}_prec"]),
               int(g[f"dig_{j:03d}_pos"]), g[f"dig_{j:03d}_c"])
        j += 1
