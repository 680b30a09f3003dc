"""In-tree build of the native libraries (nvcc for sm_100a, g++ for host code).

Outputs go to ``pennsylvaniagpugraphclustering_b200/_build/``:

* ``libpggc_b200.so``   -- the CUDA kernels, the multilevel driver and the C ABI
                           declared in ``include/pggc.h``;
* ``libpggc_graphgen.so`` -- host-side seeded synthetic graph generators;
* ``plouvain``, ``pleiden``, ``pleiden+``, ``meme``, ``verify_obj`` -- the
  reference's command-line programs (app/CMakeLists.txt:3-7) over the C ABI.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
REPO = os.path.dirname(HERE)
INCLUDE = os.path.join(REPO, "include")

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _host_cxx() -> str:
    for c in ("/usr/bin/g++", shutil.which("g++") or ""):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("no host C++ compiler found")


def _nvcc() -> str:
    for c in (shutil.which("nvcc") or "", "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _stale(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build_graphgen(force: bool = False) -> str:
    os.makedirs(OUT, exist_ok=True)
    src = os.path.join(CSRC, "graphgen.cpp")
    out = os.path.join(OUT, "libpggc_graphgen.so")
    if force or _stale(out, [src]):
        cmd = [_host_cxx(), "-O3", "-std=c++17", "-fPIC", "-shared", "-pthread", "-o", out, src]
        subprocess.run(cmd, check=True)
    return out


def cuda_sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def build_cuda(force: bool = False, verbose_ptxas: bool = False) -> str:
    os.makedirs(OUT, exist_ok=True)
    srcs = cuda_sources()
    hdrs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))
    out = os.path.join(OUT, "libpggc_b200.so")
    if not (force or _stale(out, srcs + hdrs)):
        return out
    objs = []
    jobs = []
    for s in srcs:
        o = os.path.join(OUT, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            cmd = [_nvcc(), *ARCH_FLAGS, "-lineinfo", "-O3", "-std=c++17", "-ccbin", _host_cxx(),
                   "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", "--extended-lambda", "-fmad=false", "-I", INCLUDE, "-I", CSRC,
                   "-c", s, "-o", o]
            if verbose_ptxas:
                cmd[1:1] = ["-Xptxas", "-v"]
            jobs.append(subprocess.Popen(cmd))
    for j in jobs:
        if j.wait() != 0:
            raise RuntimeError("nvcc failed")
    cmd = [_nvcc(), *ARCH_FLAGS, "-shared", "-ccbin", _host_cxx(), "-o", out, *objs, "-cudart", "static"]
    subprocess.run(cmd, check=True)
    return out


APPS = {  # program: (source, extra defines); app/CMakeLists.txt:3-7, 17-19
    "plouvain": ("cluster_main.cpp", ["-DPGGC_APP_METHOD=0"]),
    "pleiden": ("cluster_main.cpp", ["-DPGGC_APP_METHOD=1"]),
    "pleiden+": ("cluster_main.cpp", ["-DPGGC_APP_METHOD=2"]),
    "meme": ("meme_main.cpp", []),
    "verify_obj": ("verify_main.cpp", []),
}


def build_apps(force: bool = False) -> list[str]:
    """Host programs linked against libpggc_b200.so (found next to them)."""
    apps_dir = os.path.join(HERE, "apps")
    lib = os.path.join(OUT, "libpggc_b200.so")
    hdrs = [os.path.join(apps_dir, "app_common.hpp"), os.path.join(INCLUDE, "pggc.h")]
    outs, jobs = [], []
    for name, (src, defs) in APPS.items():
        out = os.path.join(OUT, name)
        outs.append(out)
        srcp = os.path.join(apps_dir, src)
        if force or _stale(out, [srcp, lib] + hdrs):
            cmd = [_host_cxx(), "-O2", "-std=c++17", *defs, "-I", INCLUDE, "-I", apps_dir, srcp, "-o", out,
                   "-L", OUT, "-lpggc_b200", "-Wl,-rpath,$ORIGIN", "-pthread"]
            jobs.append(subprocess.Popen(cmd))
    for j in jobs:
        if j.wait() != 0:
            raise RuntimeError("building the command-line programs failed")
    return outs


def build_all(force: bool = False) -> None:
    build_graphgen(force)
    if cuda_sources():
        build_cuda(force)
        build_apps(force)


if __name__ == "__main__":
    import sys
    build_all(force="--force" in sys.argv)
