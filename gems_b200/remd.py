"""Replica exchange (parallel_tempering2, src/ReplicaExchange.f90:27-150)
over replicas spread across processes, one process per GPU.

The reference runs one replica per MPI rank and, on an accepted swap, sends
the configurations between the two ranks.  Here every rank holds a block of
replicas as systems of its own context and nothing but energies crosses
ranks: each round one all-gather of every replica's potential energy (one
float64 per replica), the same decision on every rank (host arithmetic in
gemsgpu_remd_decide, the same uniforms), and the swap applied as a change of
temperature labels with the velocity rescale, each rank on its own replicas.

Replica r (global id) lives on rank r // n_local.  `label[r]` is the index
into the temperature ladder that replica r currently runs at; at the start
replica r runs at temps[r].
"""
import numpy as np

from .gemsgpu import remd_decide


def _dist():
    try:
        import torch.distributed as dist
    except ImportError:
        return None
    return dist if dist.is_available() and dist.is_initialized() else None


class ReplicaExchange:
    """Exchange driver for this rank's replicas.

    ctx, systems: this rank's context and its n_local replicas (Ermak
        systems), in global-id order; rank q holds ids q*n_local ...
    temps: the whole temperature ladder (n_local * world entries).
    energies / retemper: overridable hooks (defaults: ctx.batch_energy and
        ctx.retemper) -- what a rank needs from its device.
    """

    def __init__(self, ctx, systems, temps, seed=1, group=None, energies=None, retemper=None):
        self.dist = _dist()
        self.group = group
        self.rank = self.dist.get_rank(group) if self.dist else 0
        self.world = self.dist.get_world_size(group) if self.dist else 1
        self.ctx = ctx
        self.systems = list(systems)
        self.n_local = len(self.systems)
        self.temps = np.ascontiguousarray(temps, dtype=np.float64)
        if len(self.temps) != self.n_local * self.world:
            raise ValueError("the ladder needs n_local * world = %d temperatures, got %d"
                             % (self.n_local * self.world, len(self.temps)))
        self.seed = int(seed)
        self.label = np.arange(len(self.temps))
        self._energies = energies or (lambda: ctx.batch_energy(self.systems)[0])
        self._retemper = retemper or (lambda sys, t: ctx.retemper(sys, t))
        self.accepted = 0

    def _all_energies(self):
        mine = np.ascontiguousarray(self._energies(), dtype=np.float64)
        if self.world == 1:
            return mine
        import torch
        dev = "cuda" if self.dist.get_backend(self.group) == "nccl" else "cpu"
        t = torch.from_numpy(mine).to(dev)
        parts = [torch.empty_like(t) for _ in range(self.world)]
        self.dist.all_gather(parts, t, group=self.group)
        return torch.cat(parts).cpu().numpy()

    def exchange(self, rnd, uniforms=None):
        """One round; returns the number of accepted swaps over all replicas."""
        e_rep = self._all_energies()                 # by global replica id
        owner = np.empty_like(self.label)
        owner[self.label] = np.arange(len(self.label))  # replica at each temperature index
        partner, acc = remd_decide(e_rep[owner], self.temps, rnd, self.seed, uniforms)
        new_owner = owner[partner]
        new_label = np.empty_like(self.label)
        new_label[new_owner] = np.arange(len(self.label))
        lo = self.rank * self.n_local
        changed = [k for k in range(self.n_local) if new_label[lo + k] != self.label[lo + k]]
        if changed:
            self._retemper([self.systems[k] for k in changed], self.temps[new_label[lo + np.array(changed)]])
        self.label = new_label
        self.accepted += acc
        return acc

    def local_temperatures(self):
        lo = self.rank * self.n_local
        return self.temps[self.label[lo:lo + self.n_local]]
