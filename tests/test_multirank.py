"""Multi-rank host logic on CPU (gloo, world size 2): sharded partial sums
combine to the full result with one all-reduce, and a rank that fails before
the collective makes the other rank's collective end with an error (short
process-group timeout), not hang.  The per-rank partial sums come from the
oracle (CPU), split over lenses the way the library shards work items."""
import os
import socket
import subprocess
import sys
import textwrap

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


WORKER = textwrap.dedent(r'''
    import importlib, os, sys, json
    from datetime import timedelta
    import numpy as np
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    rank, world, mode = int(sys.argv[1]), int(sys.argv[2]), sys.argv[3]
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=8),
                            init_method=f"tcp://127.0.0.1:{PORT}")
    tpcf_dist = importlib.import_module("2pcf_b200.dist")
    tpcf = importlib.import_module("2pcf_b200")
    rng = np.random.default_rng(5)
    n = 1200
    f = lambda a: np.ascontiguousarray(a, np.float32)
    L = dict(x=f(rng.uniform(0, 100, n)), y=f(rng.uniform(0, 100, n)), z=np.zeros(n, np.float32),
             val=f(rng.normal(0, .02, n)), w=f(rng.uniform(.5, 1.5, n)))
    S = dict(x=f(rng.uniform(0, 100, n)), y=f(rng.uniform(0, 100, n)), z=np.ones(n, np.float32),
             e1=f(rng.normal(0, .26, n)), e2=f(rng.normal(0, .26, n)), w=np.ones(n, np.float32),
             m=np.zeros(n, np.float32))
    patch = (np.arange(n) % 3).astype(np.int32)
    e, e2 = O.canonical_edges(1.0, 30.0, 6)
    mine = np.arange(rank, n, world)            # this rank's share of the lenses
    def result(idx):
        c = O.canon_pairs(O.SHEAR, L, S, e2, lens_idx=idx)
        ps = np.zeros((3, 6, 6))
        for p in range(3):
            q = O.canon_pairs(O.SHEAR, L, S, e2, lens_idx=idx[patch[idx] == p])
            ps[p] = [q["sum_dw"], q["sum_gt"], q["sum_gx"], q["sum_w"], q["sum_K"], q["n_pairs"]]
        z = np.zeros(6, np.float32)
        return tpcf.Shear2pcfResults(n_bin=6, theta=z, mean_theta=z, g_t=z, g_x=z, weights=z,
                                     n_pairs=c["n_pairs"].astype(np.int64), sum_dw=c["sum_dw"],
                                     sum_gt=c["sum_gt"], sum_gx=c["sum_gx"], sum_w=c["sum_w"],
                                     sum_K=c["sum_K"], patch_sums=ps)
    if mode == "fail" and rank == 1:
        raise SystemExit(3)                       # leaves before the collective
    try:
        r = tpcf_dist.combine_shards([result(mine)])[0]
    except Exception as ex:
        print(json.dumps({"error": type(ex).__name__}), flush=True)
        sys.exit(0)
    full = result(np.arange(n))
    out = {"n_pairs_equal": bool(np.array_equal(r.n_pairs, full.n_pairs)),
           "gt_close": bool(np.allclose(r.sum_gt, full.sum_gt, rtol=1e-12, atol=1e-15)),
           "patch_close": bool(np.allclose(r.patch_sums, full.patch_sums, rtol=1e-12, atol=1e-15)),
           "g_t_close": bool(np.allclose(r.g_t, np.where(full.sum_K > 0, full.sum_gt / full.sum_K, 0), rtol=1e-6))}
    print(json.dumps(out), flush=True)
    dist.destroy_process_group()
''')


def run_ranks(mode):
    import json
    port = free_port()
    code = WORKER.replace("ROOT", repr(ROOT)).replace("{PORT}", str(port))
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", CUDA_VISIBLE_DEVICES="")
    procs = [subprocess.Popen([sys.executable, "-c", code, str(r), "2", mode], stdout=subprocess.PIPE,
                              stderr=subprocess.PIPE, text=True, env=env) for r in range(2)]
    outs = []
    for p in procs:
        try:
            o, e = p.communicate(timeout=120)
        except subprocess.TimeoutExpired:
            p.kill()
            raise
        outs.append((p.returncode, o.strip().splitlines()[-1] if o.strip() else "", e))
    return [(rc, json.loads(line) if line.startswith("{") else None, err) for rc, line, err in outs]


def test_sharded_sums_combine_to_full_result():
    res = run_ranks("ok")
    for rc, out, err in res:
        assert rc == 0, err[-2000:]
        assert out == {"n_pairs_equal": True, "gt_close": True, "patch_close": True, "g_t_close": True}, out


def test_failed_rank_ends_collective_with_error():
    res = run_ranks("fail")
    assert res[1][0] == 3                      # rank 1 left with its own status
    rc0, out0, err0 = res[0]
    assert rc0 == 0 and out0 is not None and "error" in out0, err0[-2000:]
