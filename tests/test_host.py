"""Host-side logic on the CPU: the C ABI surface, error reporting without a
GPU, scene construction, and the multi-rank plumbing (gloo, world size 2)."""
import ctypes
import os
import re
import socket

import numpy as np
import pytest

import dist_util
import hfgrid
import scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not h.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"(?:HFG_API|MPHYSICS_API)\s+[\w\s\*]+?\b(\w+)\s*\(", src)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(hfgrid.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 50
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_the_c_api():
    """hfgrid.lib() binds a signature for every solver/operator entry point."""
    lib = hfgrid.lib()
    for n in declared_symbols():
        if n.startswith("hfg_"):
            assert getattr(lib, n).argtypes is not None, n


def test_errors_cross_the_abi_as_status_codes():
    import torch
    if torch.cuda.is_available():
        pytest.skip("needs a host without a CUDA device")
    lib = hfgrid.lib()
    assert lib.hfg_init(0) != 0
    assert "CUDA" in lib.hfg_last_error().decode() or "device" in lib.hfg_last_error().decode()
    h = ctypes.c_void_p()
    rc = lib.hfg_solver_create(ctypes.c_float(0.1), hfgrid._i3((4, 4, 4)), hfgrid._f3((0, 0, 0)),
                               hfgrid._f3((1, 1, 1)), ctypes.byref(h))
    assert rc < 0 and not h.value
    # invalid arguments are rejected before any CUDA call
    rc = lib.hfg_solver_create(ctypes.c_float(0.1), hfgrid._i3((0, 4, 4)), hfgrid._f3((0, 0, 0)),
                               hfgrid._f3((1, 1, 1)), ctypes.byref(h))
    assert rc == -1
    assert lib.hfg_solver_update(None) == -1
    assert lib.hfg_op_project(hfgrid._i3((4, 4, 4)), hfgrid._f3((1, 1, 1)), 0.1, None, None, None, None, None, None,
                              None, 0, 0, 1e-3, -1, None, None, None) == -1


def test_default_options_match_the_reference():
    o = hfgrid.default_options()
    assert o.precond == hfgrid.PRECOND_IDENTITY and o.tol_mode == hfgrid.TOL_REFERENCE
    assert o.tol == pytest.approx(1e-3) and o.max_iter == -1      # CuMatrixFreePCG.h:28, PressureSolver.cpp:151
    assert o.extrapolation_layers == 1000                           # GridFluidSolver.cpp:176
    assert o.clamp_mode == 1


def test_scene_sdfs():
    sc = scenes.dam_break_64()
    walls = scenes.sdf_walls(sc.res, sc.spacing)
    # the outermost cell layer is wall, everything inside is not
    assert (walls[0] < 0).all() and (walls[-1] < 0).all() and (walls[:, 0] < 0).all() and (walls[:, :, -1] < 0).all()
    assert (walls[1:-1, 1:-1, 1:-1] > 0).all()
    sph = scenes.solid_sdf(sc, sc.solids[0])
    assert sph.min() < 0 < sph.max()
    tot = scenes.total_solid(sc)
    assert set(np.unique(tot)) <= {-1.0, -2.0, np.finfo(np.float32).max}
    big = scenes.dam_break_256(n=32)
    b = scenes.boundaries(big)
    assert len(b) == 3 and all(s.dtype == np.float32 for s, _ in b)


def test_scene_assignment_respects_budget():
    fp = [100, 80, 60, 50, 40, 30, 20, 10, 500]
    placed, rejected = dist_util.assign_scenes(fp, 2, 200)
    assert rejected == [8]
    loads = [sum(fp[i] for i in p) for p in placed]
    assert all(l <= 200 for l in loads)
    assert sorted(i for p in placed for i in p) == list(range(8))
    assert dist_util.scene_bytes((256, 256, 256), 31_400_496) < 180e9


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        m = dist_util.max_over_ranks(10.0 + rank)
        # the library's own footprints of served scenes (hfg_scene_bytes)
        fp = [dist_util.scene_bytes((32 + 8 * i, 40, 48), 1000 * i) for i in range(7)]
        placed, rejected = dist_util.assign_scenes(fp, world, 10**9)
        same = dist_util.agree([i for p in placed for i in p] + [-1] + rejected)
        # each rank's server statistics, gathered and merged as bench.py does
        import bench
        mine = {"submitted": len(placed[rank]), "completed": len(placed[rank]), "failed": 0, "rejected": 0,
                "cell_steps": float(sum(fp[i] for i in placed[rank])), "peak_bytes": 1, "wall_s": 1.0 + rank,
                "step_ms_p50": 2.0 + rank, "step_ms_p99": 5.0 + rank, "request_ms_p50": 1.0, "request_ms_p99": 3.0,
                "failed_ids": [], "slots": 4}
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        merged = bench.merge_server_stats(gathered)
        out.put((rank, m, placed[rank], same, merged))
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=120) for _ in range(2)), key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][1] == res[1][1] == 11.0          # max over ranks
    assert res[0][3] and res[1][3]                 # identical assignment on both ranks
    assert sorted(res[0][2] + res[1][2]) == list(range(7))
    fp = [dist_util.scene_bytes((32 + 8 * i, 40, 48), 1000 * i) for i in range(7)]
    for merged in (res[0][4], res[1][4]):
        assert merged["completed"] == 7 and merged["ranks"] == 2
        assert merged["cell_steps"] == float(sum(fp))      # work adds up over ranks
        assert merged["wall_s"] == 2.0 and merged["step_ms_p99"] == 6.0  # the slowest rank
        assert merged["mcell_steps_per_s"] == merged["cell_steps"] / 2.0 / 1e6


def test_rank_plan_for_two_gpus():
    """`bench.py --gpus 2` outside torchrun starts two ranks of itself on
    this node, rendezvous on 127.0.0.1, with its own arguments."""
    import bench
    cmd = bench.rank_plan(2, 29512)
    assert cmd[1:3] == ["-m", "torch.distributed.run"]
    assert "--nproc-per-node=2" in cmd and "--nnodes=1" in cmd
    assert "--master-addr=127.0.0.1" in cmd and "--master-port=29512" in cmd
    assert cmd[cmd.index("--master-port=29512") + 1].endswith("bench.py")


def test_bench_starts_its_ranks(tmp_path):
    """The reference arm through the self-launch with --gpus 2: rank 0 prints
    the one line (n_gpus 2), rank 1 exits without work."""
    import json
    import subprocess
    import sys
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
           "--warmup", "3", "--cpu-sample-res", "16"]
    out = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.strip().startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["config"]["res"] == [16, 16, 16]


HOST_SRC = r"""
#include "mphysics.h"
#include "hfgrid.h"
#include <stdio.h>
int main(void) {
  hfg_options_t o;
  hfg_default_options(&o);
  %(ns)sloadScene("{ \"HybridSimulator\": 3 }");
  printf("%%s|%%d|%%u\n", %(ns)smphysics_last_error(), o.precond, %(ns)sgetParticleSize("none"));
#ifdef __cplusplus
  /* the reference's default arguments (MPhysics.h:49-67) */
  unsigned int inst = MPhysicsAPI::instanceRigidBoundary("none", 0);
  MPhysicsAPI::transformRigidBoundary("none", 0, inst);
#endif
  return 0;
}
"""


@pytest.mark.parametrize("cc,ns,ext", [("gcc", "", "c"), ("g++", "MPhysicsAPI::", "cpp")])
def test_headers_compile_and_link_from_c_and_cpp(tmp_path, cc, ns, ext):
    """A host written in C or C++ compiles against include/*.h and links
    libhfgrid.so; the reference's call form MPhysicsAPI::f() works in C++."""
    import shutil
    import subprocess
    if shutil.which(cc) is None:
        pytest.skip(f"{cc} not installed")
    src = tmp_path / f"host.{ext}"
    src.write_text(HOST_SRC % {"ns": ns})
    exe = tmp_path / "host"
    libdir = os.path.dirname(hfgrid.LIB_PATH)
    subprocess.run([cc, str(src), "-I", os.path.join(ROOT, "include"), "-L", libdir, "-lhfgrid",
                    f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True)
    env = dict(os.environ)
    import torch  # libcudart.so ships with torch's CUDA wheels; make it findable
    cudart = os.path.join(os.path.dirname(os.path.dirname(torch.__file__)), "nvidia", "cuda_runtime", "lib")
    env["LD_LIBRARY_PATH"] = cudart + os.pathsep + env.get("LD_LIBRARY_PATH", "")
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True, env=env).stdout.strip()
    assert out == "scene has no HybridSimulator array|0|0"
