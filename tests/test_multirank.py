"""Multi-rank logic on CPU with gloo, world size 2.

The single-system step has no exchange, so N GPUs run N replicas; the only
cross-rank operations are the barrier around the timed region and the max of
the device times.  The batching ensemble splits over the ranks by work with
no exchange but the final gather of per-system results.  Covered here
without a GPU: Dist.max over two gloo ranks, the reference arm under torchrun
(rank 0 prints one JSON line, the other rank exits 0 without work), and the
ensemble split (partition, per-rank generation, gather) with the oracle's
reference step as each system's engine."""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench
    d = bench.Dist("gloo")
    d.barrier()
    m = d.max(10.0 * (rank + 1))
    d.close()
    with open(out + ".%d" % rank, "w") as f:
        f.write(repr(m))


def test_dist_max_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    out = str(tmp_path / "m")
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(2):
        assert float(open(out + ".%d" % r).read()) == 20.0


def test_reference_arm_under_torchrun_two_ranks():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--particles", "8192", "--steps", "1", "--warmup", "0"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["e2e"]["h2d_bytes_per_step"] == 0


def _per_system_forces(O, counts, pos, systems):
    """Per-system accelerations from the oracle's reference step, one system
    at a time (the CPU stand-in for the library's ensemble step)."""
    off = np.concatenate([[0], np.cumsum(counts)])
    out = []
    for s in systems:
        p = np.ascontiguousarray(pos[off[s]:off[s + 1]])
        S = O.OracleStep(p, theta=0.5, eps=0.01, nleaf=16, ncrit=64, level_split=5).build().multipoles().groups()
        S.forces()
        acc = np.zeros_like(p)
        acc[S.ph_perm] = S.acc
        out.append(acc)
    return out


def _split_rank_main(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import pickle

    import torch.distributed as dist

    from bonsai2_b200.ensemble import gather_systems, partition_systems, plummer_ensemble, system_sizes
    from oracle import oracle as O
    dist.init_process_group("gloo")
    counts = system_sizes(12, 32, 600, seed=11)
    parts = partition_systems(counts, world)
    mine = parts[rank]
    # each rank generates only its own systems, by their global seeds
    pos, _ = plummer_ensemble(counts[mine], seeds=100 + mine)
    local_off = np.concatenate([[0], np.cumsum(counts[mine])])
    accs = _per_system_forces(O, counts[mine], pos, range(len(mine)))
    # per-system result rows: a fixed-length checksum of each system's forces
    rows = np.array([[a[:, k].astype(np.float64).sum() for k in range(4)] for a in accs])
    assert local_off[-1] == pos.shape[0]
    allparts = [None] * world
    dist.all_gather_object(allparts, [p.tolist() for p in parts])
    full = gather_systems(dist, mine, rows, len(counts))
    dist.destroy_process_group()
    with open(out + ".%d" % rank, "wb") as f:
        pickle.dump({"parts": allparts, "full": full}, f)


def test_ensemble_split_two_gloo_ranks(tmp_path):
    """The batching ensemble split over two gloo ranks: both ranks compute the
    same partition, it covers every system once with balanced estimated work,
    and the per-system results gathered on rank 0 equal, bit for bit, those of
    one process running every system."""
    import pickle

    import torch.multiprocessing as mp

    from bonsai2_b200.ensemble import partition_systems, plummer_ensemble, system_sizes, system_work
    from oracle import oracle as O
    port = _free_port()
    out = str(tmp_path / "split")
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_split_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
        assert p.exitcode == 0
    res = [pickle.load(open(out + ".%d" % r, "rb")) for r in range(2)]
    assert res[0]["parts"] == res[1]["parts"]
    counts = system_sizes(12, 32, 600, seed=11)
    parts = partition_systems(counts, 2)
    assert sorted(np.concatenate(parts).tolist()) == list(range(len(counts)))
    w = system_work(counts)
    loads = [w[p].sum() for p in parts]
    assert max(loads) - min(loads) <= w.max()
    assert res[1]["full"] is None
    pos, _ = plummer_ensemble(counts, base_seed=100)
    one = _per_system_forces(O, counts, pos, range(len(counts)))
    ref = np.array([[a[:, k].astype(np.float64).sum() for k in range(4)] for a in one])
    assert np.array_equal(res[0]["full"], ref)


def test_partition_balance_and_determinism():
    from bonsai2_b200.ensemble import partition_systems, system_sizes, system_work
    counts = system_sizes(512, 1 << 10, 1 << 18, seed=2024)
    w = system_work(counts)
    for world in (1, 2, 3, 4, 8):
        parts = partition_systems(counts, world)
        assert sorted(np.concatenate(parts).tolist()) == list(range(512))
        loads = np.array([w[p].sum() for p in parts])
        assert loads.max() / loads.mean() < 1.01
        again = partition_systems(counts, world)
        assert all(np.array_equal(x, y) for x, y in zip(parts, again))
