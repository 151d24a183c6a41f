"""Multi-rank host logic of bench.py on CPU (gloo, world size 2)."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, values, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    out[rank] = bench.max_over_ranks(values[rank], dist)
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo():
    import torch.multiprocessing as mp
    port = _free_port()
    values = [3.5, 7.25]
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(2, port, values, out), nprocs=2, join=True)
        assert out[0] == out[1] == max(values)


def test_reference_arm_two_ranks_prints_once():
    """torchrun with 2 ranks: rank 0 prints one JSON line, rank 1 exits 0."""
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0", "--block", "1",
           "--therm-steps", "5"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["cpu_baseline"]["kind"] == "port"
    assert d["e2e"]["h2d_bytes_per_step"] == 0


# ---------------------------------------------------------------- replica exchange across ranks
NREP_LOCAL, ROUNDS = 3, 12


def _energy_table(world):
    """Potential energies (eV) per round and global replica, spread so that
    both accepted and rejected swaps occur."""
    rng = __import__("numpy").random.default_rng(11)
    return rng.normal(-300.0, 0.05, size=(ROUNDS + 1, NREP_LOCAL * world))


def _ladder(world):
    import numpy as np
    n = NREP_LOCAL * world
    return 200.0 * (900.0 / 200.0) ** (np.arange(n) / (n - 1))


def _remd_worker(rank, world, port, out):
    import numpy as np
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from gems_b200.remd import ReplicaExchange
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    table = _energy_table(world)
    lo = rank * NREP_LOCAL
    state = {"round": 0, "temps": {}}

    def energies():
        # each replica's energy this round: the table row of the round, at its global id
        return table[state["round"], lo:lo + NREP_LOCAL]

    def retemper(systems, temps):
        for s_, t in zip(systems, temps):
            state["temps"][s_] = float(t)

    rex = ReplicaExchange(None, list(range(NREP_LOCAL)), _ladder(world), seed=5,
                          energies=energies, retemper=retemper)
    accs = []
    for r in range(1, ROUNDS + 1):
        state["round"] = r
        accs.append(rex.exchange(r))
    out[rank] = {"label": rex.label.tolist(), "acc": accs, "local_t": rex.local_temperatures().tolist(),
                 "retempered": state["temps"]}
    dist.barrier()
    dist.destroy_process_group()


def test_replica_exchange_across_ranks_gloo():
    """Two ranks of three replicas each: every rank reaches the same labels,
    equal to one process swapping systems along the ladder with the same
    decisions, and each rank retempers exactly its own moved replicas."""
    import numpy as np
    import torch.multiprocessing as mp
    sys.path.insert(0, ROOT)
    from gems_b200.gemsgpu import remd_decide
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_remd_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    # one process, the formulation of gemsgpu_replica_exchange: a list of
    # replicas indexed by temperature, permuted by each round's partners
    table = _energy_table(world)
    temps = _ladder(world)
    at_temp = list(range(NREP_LOCAL * world))
    accs = []
    for r in range(1, ROUNDS + 1):
        part, acc = remd_decide(table[r, at_temp], temps, r, 5)
        at_temp = [at_temp[p] for p in part]
        accs.append(acc)
    label = [at_temp.index(rep) for rep in range(len(at_temp))]
    assert 0 < sum(accs) < len(accs) * (len(at_temp) // 2)   # both outcomes occur
    for rank in range(world):
        assert res[rank]["label"] == label
        assert res[rank]["acc"] == accs
        lo = rank * NREP_LOCAL
        np.testing.assert_array_equal(res[rank]["local_t"], temps[label[lo:lo + NREP_LOCAL]])
        # the last temperature each local replica was given is its current one
        for k, t in res[rank]["retempered"].items():
            assert t == temps[label[lo + k]]
