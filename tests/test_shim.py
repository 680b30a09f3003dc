"""The header-only C++ shim with the reference's names
(include/pggc_clustering_methods.hpp over include/pggc.h; the reference's
interface/clustering_methods.h:20-24).

A small C++ program (tests/native/shim_cluster.cpp) includes the shim, calls
clustering_methods::leiden_part<true,false>, leiden_part<true,true> and
louvain_part<false> on device label arrays the way the reference's
run_clustering does, and writes the labels and objectives.  On the CPU the
program must compile and link against libpggc_b200.so; on the GPU its results
must equal pggc_run_clustering bit for bit.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

import pennsylvaniagpugraphclustering_b200 as pg
from pennsylvaniagpugraphclustering_b200 import _lib, build as B

from . import graphs as G

SRC = os.path.join(os.path.dirname(os.path.abspath(__file__)), "native", "shim_cluster.cpp")
CUDA = "/usr/local/cuda"


def _compile(out_dir):
    lib = _lib.LIB_PATH if os.path.exists(_lib.LIB_PATH) else B.build_cuda()
    exe = os.path.join(str(out_dir), "shim_cluster")
    cxx = shutil.which("g++") or "/usr/bin/g++"
    cmd = [cxx, "-std=c++17", "-O1", "-Wall", "-Werror", "-I", B.INCLUDE, "-I", os.path.join(CUDA, "include"), SRC,
           "-o", exe, "-L", os.path.dirname(lib), "-lpggc_b200", "-Wl,-rpath," + os.path.dirname(lib),
           "-L", os.path.join(CUDA, "lib64"), "-lcudart", "-Wl,-rpath," + os.path.join(CUDA, "lib64")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def _write_graph(path, hg):
    with open(path, "wb") as f:
        np.array([hg.n, hg.nnz], np.int64).tofile(f)
        np.array([1 if hg.w is not None else 0], np.int32).tofile(f)
        hg.rowptr.astype(np.int64).tofile(f)
        hg.col.astype(np.int32).tofile(f)
        if hg.w is not None:
            hg.w.astype(np.float32).tofile(f)


def _read_runs(path, n, runs=3):
    raw = open(path, "rb").read()
    out = []
    off = 0
    for _ in range(runs):
        lab = np.frombuffer(raw, np.int32, n, off).copy()
        off += 4 * n
        q = float(np.frombuffer(raw, np.float64, 1, off)[0])
        off += 8
        out.append((lab, q))
    assert off == len(raw)
    return out


def test_shim_program_compiles_and_links(tmp_path):
    exe = _compile(tmp_path)
    assert os.access(exe, os.X_OK)


@pytest.mark.gpu
@pytest.mark.parametrize("name,make", [("sbm_mod", lambda: G.small_sbm(2)),
                                       ("dcsbm_wmod", lambda: G.small_dcsbm(3))])
def test_shim_matches_run_clustering(mem, tmp_path, name, make):
    hg = make()
    exe = _compile(tmp_path)
    gpath, opath = tmp_path / "g.bin", tmp_path / "out.bin"
    _write_graph(gpath, hg)
    seed = 17
    r = subprocess.run([exe, str(gpath), str(opath), str(seed)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    (l1, q1), (l2, q2), (l3, q3) = _read_runs(opath, hg.n)
    obj = pg.OBJ_WMOD if hg.w is not None else pg.OBJ_MOD
    wg = pg.weighted_graph(mem, hg.rowptr, hg.col, hg.w, objective=obj)
    # pass 0 of run_clustering is leiden_part<true,false> with the seed; pass 1
    # is leiden_part<true,true> from it with seed + 0x9E3779B97F4A7C15
    for ex, lab, q in ((0, l1, q1), (1, l2, q2)):
        cd = pg.get_objective(mem, wg, obj, 1.0)
        ref, st = pg.run_clustering(mem, wg, cd, method=pg.METHOD_LEIDEN_PLUS, ex_iters=ex, seed=seed)
        assert np.array_equal(lab, ref), f"leiden_part pass {ex}"
        assert q == st["objective"]
        cd.close()
    cd = pg.get_objective(mem, wg, obj, 1.0)
    ref, st = pg.run_clustering(mem, wg, cd, method=pg.METHOD_LOUVAIN, ex_iters=0, seed=seed)
    assert np.array_equal(l3, ref)
    assert q3 == st["objective"]
    cd.close()
    wg.close()
