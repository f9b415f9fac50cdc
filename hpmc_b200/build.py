"""Build recipe of the sm_100a extension library ``hpmc_b200/_lib/libhpmc_b200.so``.

Steps:
  1. import HPMC's case tables (``csrc/gen_tables.py``) from the HPMC source
     tree named by the ``HPMC_SRC`` environment variable (default: an HPMC
     checkout named ``reference`` beside this repository) into
     ``csrc/_gen/hpmc_case_tables.h`` (git-ignored; a prebuilt header is used
     when no tree is found);
  2. compile every ``csrc/*.cu`` with nvcc for ``sm_100a`` and link one shared
     library exposing the C ABI of ``include/hpmc.h``.

Run ``python -m hpmc_b200.build`` (or ``__graft_entry__.build()``).
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
GEN = os.path.join(CSRC, "_gen", "hpmc_case_tables.h")
OUT_DIR = os.path.join(PKG, "_lib")
OBJ_DIR = os.path.join(OUT_DIR, "obj")
LIB = os.path.join(OUT_DIR, "libhpmc_b200.so")
# The HPMC source tree: $HPMC_SRC, else a checkout named `reference` beside the repository.
DEFAULT_HPMC_SRC = os.path.normpath(os.path.join(ROOT, os.pardir, "reference"))

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "--expt-relaxed-constexpr",
    "-I" + os.path.join(ROOT, "include"), "-I" + CSRC,
]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found")
    return cand


def gen_tables() -> None:
    src = os.environ.get("HPMC_SRC", DEFAULT_HPMC_SRC)
    tables = os.path.join(src, "hpmc", "src", "tables.cpp")
    gen_script = os.path.join(CSRC, "gen_tables.py")
    if os.path.exists(tables):
        if (not os.path.exists(GEN) or os.path.getmtime(GEN) < os.path.getmtime(gen_script)
                or os.path.getmtime(GEN) < os.path.getmtime(tables)):
            subprocess.run([sys.executable, gen_script, src, GEN], check=True)
    elif not os.path.exists(GEN):
        raise RuntimeError(
            "HPMC case tables missing: set HPMC_SRC to an HPMC source tree "
            "(hpmc/src/tables.cpp) to generate csrc/_gen/hpmc_case_tables.h")


def _sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs.append(GEN)
    hs.append(os.path.join(ROOT, "include", "hpmc.h"))
    hs.append(os.path.join(ROOT, "include", "hpmc_types.h"))
    return hs


def _compile(src: str, extra: list[str]) -> str:
    obj = os.path.join(OBJ_DIR, os.path.basename(src)[:-3] + ".o")
    newest_dep = max([os.path.getmtime(src)] + [os.path.getmtime(h) for h in _headers() if os.path.exists(h)])
    if os.path.exists(obj) and os.path.getmtime(obj) >= newest_dep and not extra:
        return obj
    cmd = [nvcc(), *NVCC_FLAGS, *extra, "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(verbose_ptxas: bool = False) -> str:
    """Compile (incrementally) and return the path of the shared library."""
    gen_tables()
    os.makedirs(OBJ_DIR, exist_ok=True)
    extra = ["-Xptxas", "-v"] if verbose_ptxas else []
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, extra), _sources()))
    if not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        tmp = LIB + ".tmp"
        cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", tmp, *objs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
    return LIB


APPS_DIR = os.path.join(PKG, "apps")
APPS_OUT = os.path.join(OUT_DIR, "apps")
APPS = ["texture3d", "cayley", "metaballs", "transform_feedback", "custom_functor"]


def app_path(name: str) -> str:
    return os.path.join(APPS_OUT, "hpmc_" + name)


def build_apps() -> list[str]:
    """Headless ports of the reference's apps (C++ callers of the C ABI),
    linked against the library: ``_lib/apps/hpmc_<name>``."""
    lib = build()
    os.makedirs(APPS_OUT, exist_ok=True)
    cxx = shutil.which("g++") or "g++"
    cuda = os.path.dirname(os.path.dirname(os.path.realpath(nvcc())))
    out = []
    for name in APPS:
        cu = os.path.join(APPS_DIR, name + ".cu")
        src = cu if os.path.exists(cu) else os.path.join(APPS_DIR, name + ".cpp")
        dst = app_path(name)
        deps = [src, os.path.join(APPS_DIR, "app_common.hpp"), os.path.join(ROOT, "include", "hpmc.h"), lib]
        if src == cu:  # a caller with device code of its own (include/hpmc_functor.cuh)
            deps += [os.path.join(ROOT, "include", "hpmc_functor.cuh")] + _headers()
        if not os.path.exists(dst) or os.path.getmtime(dst) < max(os.path.getmtime(d) for d in deps):
            if src == cu:
                cmd = [nvcc(), *NVCC_FLAGS, src, "-o", dst, "-L" + OUT_DIR, "-lhpmc_b200",
                       "-Xlinker", "-rpath,$ORIGIN/.."]
            else:
                cmd = [cxx, "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"),
                       "-I" + os.path.join(cuda, "include"), src, "-o", dst, "-L" + OUT_DIR, "-lhpmc_b200",
                       "-L" + os.path.join(cuda, "lib64"), "-lcudart", "-Wl,-rpath,$ORIGIN/.."]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"app build failed for {name}:\n{r.stdout}\n{r.stderr}")
        out.append(dst)
    return out


if __name__ == "__main__":
    print(build(verbose_ptxas="-v" in sys.argv))
    for a in build_apps():
        print(a)
