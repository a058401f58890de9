"""Build recipe for the CPU oracle (test infrastructure only).

Two shared libraries come out of here:

* ``oracle/liboracle.so`` -- the plain-C restatement in ``bigint_oracle.c``.
* ``oracle/_ref/libbigint_ref.so`` -- the UNMODIFIED reference multiply path,
  compiled directly from its own sources where they lie (``src/mul/*.cpp``,
  ``src/bigint.cpp``) plus ``ref_shim.cpp``.  The reference targets MinGW; the
  force-included ``ref_compat.h`` supplies the overloads four of its call sites
  need on Linux (no source is copied or edited).  ``-flto`` from the
  reference's CMake release flags is left out: the LTO plugin cannot run here.

Usage: ``python oracle/build.py [port|ref|ref_gpu|all]`` (default ``all``).
The reference tree is only needed for ``ref`` and ``ref_gpu``: its root comes
from the ``BIGINT_REF_ROOT`` environment variable (or the ``ref_root``
argument of the build functions).  With no root given those two steps stop
with an error; with a root that holds no sources they are skipped and an
existing ``oracle/_ref`` build is kept.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_ROOT_ENV = "BIGINT_REF_ROOT"
REF_SOURCES = [
    "src/mul/ntt_multithread.cpp",
    "src/mul/fft.cpp",
    "src/mul/ssa.cpp",
    "src/bigint.cpp",
]
PORT_SO = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_SO = os.path.join(REF_DIR, "libbigint_ref.so")


def _run(cmd: list[str]) -> None:
    subprocess.run(cmd, check=True)


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build_port(force: bool = False) -> str:
    src = os.path.join(HERE, "bigint_oracle.c")
    hdr = os.path.join(HERE, "bigint_oracle.h")
    if force or _stale(PORT_SO, [src, hdr, __file__]):
        _run(["gcc", "-O2", "-std=c11", "-Wall", "-Wextra", "-fPIC", "-shared", src, "-o", PORT_SO])
    return PORT_SO


def ref_root(given: str | None = None) -> str:
    """The reference checkout to compile: `given`, else $BIGINT_REF_ROOT."""
    root = given or os.environ.get(REF_ROOT_ENV)
    if not root:
        raise RuntimeError(f"oracle/build.py: no reference root; set {REF_ROOT_ENV} to the "
                           "reference checkout (the directory holding include/ and src/)")
    return root


def build_ref(force: bool = False, ref_root_dir: str | None = None) -> str | None:
    REF_ROOT = ref_root(ref_root_dir)
    if not os.path.isdir(os.path.join(REF_ROOT, "src")):
        return REF_SO if os.path.exists(REF_SO) else None
    os.makedirs(REF_DIR, exist_ok=True)
    shim = os.path.join(HERE, "ref_shim.cpp")
    compat = os.path.join(HERE, "ref_compat.h")
    srcs = [os.path.join(REF_ROOT, s) for s in REF_SOURCES]
    if not (force or _stale(REF_SO, srcs + [shim, compat, __file__])):
        return REF_SO
    flags = ["-std=c++20", "-O3", "-DNDEBUG", "-mavx", "-mavx2", "-mfma", "-fPIC", "-pthread",
             "-include", compat, "-I", os.path.join(REF_ROOT, "include")]
    objs = []
    for s in srcs + [shim]:
        o = os.path.join(REF_DIR, os.path.basename(s).replace(".cpp", ".o"))
        _run(["g++", *flags, "-c", s, "-o", o])
        objs.append(o)
    _run(["g++", "-shared", "-pthread", *objs, "-o", REF_SO])
    for o in objs:
        os.remove(o)
    return REF_SO


HOOK_SRC = os.path.join(os.path.dirname(HERE), "bigint_b200", "hooks", "reference_hook.cpp")
ENGINE_DIR = os.path.join(os.path.dirname(HERE), "bigint_b200")
REF_GPU_SO = os.path.join(REF_DIR, "libbigint_ref_gpu.so")
# The reference without its CPU NTT and FFT translation units: those two
# functions (and init_thread_pool) come from the hook, which calls the engine.
REF_GPU_SOURCES = ["src/mul/ssa.cpp", "src/bigint.cpp"]


def build_ref_gpu(force: bool = False, ref_root_dir: str | None = None) -> str | None:
    """The unmodified reference BigInt with its multiplies on the GPU engine
    (bigint_b200/hooks/reference_hook.cpp), plus the same C-ABI shim as the
    reference oracle, linked against bigint_b200/libbigint_b200.so."""
    REF_ROOT = ref_root(ref_root_dir)
    engine = os.path.join(ENGINE_DIR, "libbigint_b200.so")
    if not os.path.isdir(os.path.join(REF_ROOT, "src")) or not os.path.exists(engine):
        return REF_GPU_SO if os.path.exists(REF_GPU_SO) else None
    os.makedirs(REF_DIR, exist_ok=True)
    shim = os.path.join(HERE, "ref_shim.cpp")
    compat = os.path.join(HERE, "ref_compat.h")
    srcs = [os.path.join(REF_ROOT, s) for s in REF_GPU_SOURCES]
    if not (force or _stale(REF_GPU_SO, srcs + [shim, compat, HOOK_SRC, engine, __file__])):
        return REF_GPU_SO
    flags = ["-std=c++20", "-O3", "-DNDEBUG", "-mavx", "-mavx2", "-mfma", "-fPIC", "-pthread",
             "-include", compat, "-I", os.path.join(REF_ROOT, "include"),
             "-I", os.path.join(os.path.dirname(HERE), "include")]
    objs = []
    for s in srcs + [shim, HOOK_SRC]:
        o = os.path.join(REF_DIR, "gpu_" + os.path.basename(s).replace(".cpp", ".o"))
        _run(["g++", *flags, "-c", s, "-o", o])
        objs.append(o)
    _run(["g++", "-shared", "-pthread", "-Wl,-Bsymbolic", *objs, "-o", REF_GPU_SO,
          "-L", ENGINE_DIR, "-lbigint_b200", "-Wl,-rpath,$ORIGIN/../../bigint_b200"])
    for o in objs:
        os.remove(o)
    return REF_GPU_SO


def main(argv: list[str]) -> int:
    what = argv[1] if len(argv) > 1 else "all"
    if what in ("port", "all"):
        print("oracle port:", build_port())
    if what in ("ref", "all"):
        print("oracle reference:", build_ref())
    if what in ("ref_gpu", "all"):
        print("reference on the GPU engine:", build_ref_gpu())
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
