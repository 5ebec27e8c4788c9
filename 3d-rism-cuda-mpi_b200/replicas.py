"""Replicas: one process per GPU, each running its own independent solve.

A 3D-RISM solve does not exchange data with other solves, so N GPUs run N
replicas of a workload with no data-path collective (weak scaling).  The
process group exists only for the barrier around a timed region and for the
max over ranks of its device time.

    launch(n, argv)   starts n ranks of `argv` (a Python script and its
                      arguments) through torch.distributed.run on 127.0.0.1
    Group(backend)    joins the group those ranks form (RANK, WORLD_SIZE,
                      LOCAL_RANK, MASTER_ADDR/PORT from the environment; a
                      lone process with no WORLD_SIZE is a group of one)
    Group.timed(fn)   barrier, fn() -> (ms, units) on every rank, barrier;
                      the max of ms over ranks and the sum of units
"""
import datetime
import os
import socket
import subprocess
import sys


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def launch(nproc, argv, timeout_s=3600, env=None):
    """Runs `argv` (script path first) as nproc ranks on this node; returns
    the launcher's exit code.  The ranks find each other on 127.0.0.1."""
    cmd = ["timeout", "-k", "60", str(int(timeout_s)), sys.executable, "-m",
           "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={nproc}",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port())] + list(argv)
    return subprocess.run(cmd, env=dict(os.environ, **(env or {}))).returncode


class Group:
    """This process's place among the replicas.  backend: "nccl" (one GPU
    per rank, LOCAL_RANK selects it) or "gloo" (CPU)."""

    def __init__(self, backend="nccl", timeout_s=300):
        self.rank = int(os.environ.get("RANK", 0))
        self.world = int(os.environ.get("WORLD_SIZE", 1))
        self.local = int(os.environ.get("LOCAL_RANK", 0))
        self.backend = backend
        self.dist = None
        if self.world > 1:
            import torch.distributed as dist
            if backend == "nccl":
                import torch
                torch.cuda.set_device(self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def _tensor(self, x):
        import torch
        dev = f"cuda:{self.local}" if self.backend == "nccl" else "cpu"
        return torch.tensor([float(x)], dtype=torch.float64, device=dev)

    def barrier(self):
        if self.dist:
            self.dist.barrier()

    def allmax(self, x):
        if not self.dist:
            return float(x)
        t = self._tensor(x)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def allsum(self, x):
        if not self.dist:
            return float(x)
        t = self._tensor(x)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def timed(self, fn):
        """Barrier, fn() -> (device ms, units done) on every rank, barrier.
        Returns (max ms over ranks, units summed over ranks): the whole job's
        throughput is units / (ms * 1e-3)."""
        self.barrier()
        ms, units = fn()
        self.barrier()
        return self.allmax(ms), self.allsum(units)

    def close(self):
        if self.dist:
            self.dist.destroy_process_group()
            self.dist = None
