"""The command-line programs (app/cluster_main.cpp, app/memetic_clustering.cpp,
app/verify_objective.cpp) -- option handling on the CPU (app/io/parse_args.cpp
rules: every option known, -i required, objective names, vertex weights only
with NLCC/LCC), whole runs on the GPU against the library's own entry points."""
import json
import os
import subprocess

import numpy as np
import pytest

import pennsylvaniagpugraphclustering_b200 as pg
from pennsylvaniagpugraphclustering_b200 import build as B

BIN = B.OUT


def _run(prog, *args, timeout=600):
    exe = os.path.join(BIN, prog)
    if not os.path.exists(exe):
        B.build_all()
    return subprocess.run([exe, *map(str, args)], capture_output=True, text=True, timeout=timeout)


@pytest.mark.parametrize("prog", ["plouvain", "pleiden", "pleiden+", "meme", "verify_obj"])
def test_unknown_option_is_fatal(prog):
    r = _run(prog, "-i", "g.mtx", "-bogus", "1")
    assert r.returncode == 255
    assert "Invalid option name: -bogus" in r.stderr


@pytest.mark.parametrize("args,msg", [
    (("-o", "x"), "Required graph input file not given"),
    (("-i",), "Value not provided for option '-i'"),
    (("-i", "g.mtx", "-objective", "Modularity"), "Invalid objective name 'Modularity'"),
    (("-i", "g.mtx", "-vtx_weights", "vw.txt"), "only supported with objectives Normalized LambdaCC"),
    (("-i", "g.mtx", "-objective", "WMod", "-vtx_weights", "vw.txt"), "only supported with objectives"),
])
def test_cluster_option_errors(args, msg):
    r = _run("pleiden+", *args)
    assert r.returncode == 255
    assert msg in r.stderr


def test_verify_needs_clusters():
    r = _run("verify_obj", "-i", "g.mtx")
    assert r.returncode == 255 and "Required clusters file not given" in r.stderr


def _mtx(tmp_path, n=3000, m=24000, seed=3, field="integer"):
    rng = np.random.default_rng(seed)
    blocks = rng.integers(0, 20, n)
    src = rng.integers(0, n, m)
    dst = rng.integers(0, n, m)
    # community structure: most edges stay inside a block
    same = rng.random(m) < 0.8
    order = np.argsort(blocks, kind="stable")
    starts = np.searchsorted(blocks[order], np.arange(21))
    for k in np.flatnonzero(same):
        b = blocks[src[k]]
        dst[k] = order[rng.integers(starts[b], starts[b + 1])]
    p = tmp_path / "g.mtx"
    lines = [f"%%MatrixMarket matrix coordinate {field} symmetric", f"{n} {n} {m}"]
    for k in range(m):
        lines.append(f"{src[k] + 1} {dst[k] + 1}" + (f" {rng.integers(1, 5)}" if field == "integer" else ""))
    p.write_text("\n".join(lines) + "\n")
    return p


@pytest.mark.gpu
@pytest.mark.parametrize("prog,method", [("plouvain", pg.METHOD_LOUVAIN), ("pleiden", pg.METHOD_LEIDEN),
                                         ("pleiden+", pg.METHOD_LEIDEN_PLUS)])
def test_cluster_program_matches_library(mem, tmp_path, prog, method):
    g = _mtx(tmp_path)
    out = tmp_path / "best.txt"
    met = tmp_path / "m.json"
    r = _run(prog, "-i", g, "-objective", "WMod", "-ex_iters", 2, "-trials", 2, "-metrics", met, "-o", out,
             "-seed", 11)
    assert r.returncode == 0, r.stderr
    recs = json.loads(met.read_text())
    assert len(recs) == 2
    for rec in recs:
        for key in ("edge-cut", "modularity", "total-nnz", "level-count", "coarsen-contract-duration-seconds",
                    "leiden-refine-duration-seconds", "total-duration-seconds", "iter-times-0", "iter-obj-2",
                    "number-coarse-levels"):
            assert key in rec
        assert rec["total-duration-seconds"] > 0
    # trial 0 is run_clustering with the same seed
    wg = pg.load_graph(mem, str(g), pg.OBJ_WMOD)
    cd = pg.get_objective(mem, wg, pg.OBJ_WMOD, 1.0)
    labels, st = pg.run_clustering(mem, wg, cd, method=method, ex_iters=2, seed=11)
    assert abs(recs[0]["modularity"] - st["objective"]) < 1e-6
    assert abs(recs[0]["iter-obj-2"] - st["objective"]) < 1e-6
    assert recs[0]["level-count"] == st["levels"]
    best = pg.load_view(wg.n, out, np.int32)
    q, _ = pg.verify_objective(mem, wg, best, pg.OBJ_WMOD)
    assert abs(q - max(r_["modularity"] for r_ in recs)) < 1e-6
    if recs[0]["modularity"] >= recs[1]["modularity"]:
        assert np.array_equal(best, labels)
    # verify_obj prints the same objective
    v = _run("verify_obj", "-i", g, "-objective", "WMod", "-clusters", out)
    assert v.returncode == 0, v.stderr
    assert abs(float(v.stdout.strip().split("Modularity: ")[-1]) - q) < 1e-8


@pytest.mark.gpu
def test_meme_program_matches_library(mem, tmp_path):
    g = _mtx(tmp_path, n=2000, m=12000, field="pattern")
    out = tmp_path / "best.txt"
    r = _run("meme", "-i", g, "-pop_size", 10, "-offspring", 3, "-time_limit", 600, "-seed", 4, "-o", out)
    assert r.returncode == 0, r.stderr
    wg = pg.load_graph(mem, str(g), pg.OBJ_MOD)
    labels, st = pg.meme_cluster(mem, wg, pg.OBJ_MOD, pop_size=10, offspring=3, seed=4)
    best = pg.load_view(wg.n, out, np.int32)
    assert np.array_equal(best, labels)
    assert "Final objective" in r.stdout


@pytest.mark.gpu
def test_vertex_weights_file_with_lcc(mem, tmp_path):
    g = _mtx(tmp_path, n=1500, m=9000, field="pattern")
    vwf = tmp_path / "vw.txt"
    vw = np.random.default_rng(2).integers(1, 4, 1500)
    pg.write_part(vw, vwf)
    out = tmp_path / "best.txt"
    r = _run("pleiden+", "-i", g, "-objective", "NLCC", "-vtx_weights", vwf, "-o", out, "-seed", 3)
    assert r.returncode == 0, r.stderr
    wg = pg.load_graph(mem, str(g), pg.OBJ_NLCC, vtx_w=vw.astype(np.int64))
    cd = pg.get_objective(mem, wg, pg.OBJ_NLCC, 1.0)
    labels, _ = pg.run_clustering(mem, wg, cd, method=pg.METHOD_LEIDEN_PLUS, ex_iters=0, seed=3)
    assert np.array_equal(pg.load_view(wg.n, out, np.int32), labels)


def test_metrics_records_are_one_json_array(tmp_path):
    """The -metrics writer (ExperimentLoggerUtil::log format): one object per
    trial appended to a single JSON array, keys and fixed-point numbers as the
    reference writes them."""
    import shutil
    src = os.path.join(os.path.dirname(os.path.abspath(__file__)), "native", "metrics_log.cpp")
    exe = tmp_path / "metrics_log"
    cxx = shutil.which("g++") or "/usr/bin/g++"
    subprocess.run([cxx, "-std=c++17", "-O1", "-I", B.INCLUDE, "-I", os.path.join(B.HERE, "apps"), src, "-o",
                    str(exe)], check=True)
    out = tmp_path / "m.json"
    subprocess.run([str(exe), str(out)], check=True)
    text = out.read_text()
    recs = json.loads(text)
    assert len(recs) == 3
    assert recs[0]["edge-cut"] == 1000 and recs[2]["edge-cut"] == 1002.0
    assert abs(recs[1]["modularity"] - 0.51) < 1e-9
    assert recs[2]["level-count"] == 6 and recs[0]["total-nnz"] == 123456
    for name in ("coarsen-contract", "coarsen", "leiden-refine", "free-graph", "total"):
        assert f"{name}-duration-seconds" in recs[0]
    assert "iter-times-2" in recs[2] and "iter-obj-2" in recs[2] and "iter-obj-1" not in recs[0]
    assert recs[1]["number-coarse-levels"] == 0
    # fixed notation with six decimals, as std::fixed writes them
    assert '"modularity":0.510000' in text


def test_option_clamping_printed_before_any_device_work(tmp_path):
    """parse_args.cpp clamps: -trials below 1 -> 1, -ex_iters below -1 -> -1,
    -pop_size below 10 -> 10 and -time_limit below 10 -> 10 (with warnings).
    The configuration is printed before the device is touched, so this runs
    anywhere (the missing graph file ends the run afterwards)."""
    missing = tmp_path / "absent.mtx"
    r = _run("pleiden+", "-i", missing, "-trials", "0", "-ex_iters", "-7")
    assert r.returncode == 255
    assert "-- Total trial count: 1" in r.stdout
    assert "-- Successive Iteration Count: -1" in r.stdout
    r = _run("meme", "-i", missing, "-pop_size", "3", "-time_limit", "2")
    assert r.returncode == 255
    assert "Setting population size to 10." in r.stdout
    assert "Setting time limit to 10s." in r.stdout
    assert "-- Population Size: 10" in r.stdout and "-- Time Limit Seconds: 10" in r.stdout
