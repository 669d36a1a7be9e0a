"""One reconstruction split over several GPUs by views (strong scaling of a single job).

Every rank holds the whole FP32 iterate and a contiguous range of the views: its context
(``tomo_context_create_views``) carries that range's per-view geometry, sliced from the
whole acquisition's tables, and its real sinogram holds those views only. Per gradient
iteration (Iter3D_Algo_Gradient.cu:25-223):

1. ``PHASE_GRADIENT``: dJ_k = -2 H_k^T (g_k - H_k f) over the rank's views;
2. all-reduce (sum) of dJ over the ranks: the full gradient dJ = sum_k dJ_k;
3. ``PHASE_NORMS``: regulariser on dJ, ||dJ||^2 and ||L dJ||^2 of the summed dJ and the
   rank's ||H_k dJ||^2;
4. while the optimal step is computed, an all-reduce (sum) of the norm slots in which
   ||H_k dJ||^2 adds up over the ranks and the norms of the summed dJ count once (rank 0's;
   the others contribute 0). Those norms are FP64 sums whose last bits depend on the order
   of the device's atomics, so without this every rank could round alpha differently and
   the ranks' iterates would drift apart;
5. ``PHASE_UPDATE``: alpha and f += alpha dJ, bit-identical on every rank.

The exchange is one volume all-reduce (NCCL over NVLink between GPUs) and a few scalars
per iteration; the operators need none. Results equal the single-GPU solver's up to the order of
the FP32 sums over views (each rank accumulates its own views, then the partial volumes are
added), i.e. to within the FP32 parity tolerance, not bit for bit.

``bench.py --gpus N`` runs whole reconstructions as replicas (``replicas.py``); this module
is the form for one reconstruction too large or too urgent for one GPU.
"""
from __future__ import annotations

import os
from typing import Callable, List, Optional, Tuple

PHASE_GRADIENT, PHASE_NORMS, PHASE_UPDATE = 1, 2, 4


def view_ranges(views: int, world: int) -> List[Tuple[int, int]]:
    """Contiguous (begin, count) per rank; the first views % world ranks take one more."""
    if world < 1 or views < world:
        raise ValueError("need at least one view per rank")
    base, extra = divmod(views, world)
    out, b = [], 0
    for r in range(world):
        c = base + (1 if r < extra else 0)
        out.append((b, c))
        b += c
    return out


# norm slots of tomo_solver_buffers: [0] ||dJ||^2, [1] ||H_k dJ||^2, [2] ||L dJ||^2,
# [3] max|dJ| bits (FP16 storage; order-independent), [4] the Huber normdJProjReg
_GLOBAL_SLOTS = (0, 2, 4)


def iterate_exchange(phase: Callable[[int, int], None], dJ, norms, first: int, count: int, optimal_step_nb: int,
                     allreduce: Optional[Callable[[object], None]], rank: int = 0) -> None:
    """Runs iterations [first, first + count) of one rank: `phase(iteration, bits)` runs the
    solver's phases, `allreduce(tensor)` sums a tensor over the ranks in place (None on a
    single rank). dJ is the rank's gradient volume, norms its norm slots."""
    for it in range(first, first + count):
        phase(it, PHASE_GRADIENT)
        if allreduce is not None:
            allreduce(dJ)
        phase(it, PHASE_NORMS)
        if allreduce is not None and it < optimal_step_nb:
            if rank != 0:
                for k in _GLOBAL_SLOTS:
                    norms[k] = 0.0
            allreduce(norms[0:3])
            allreduce(norms[4:5])
        phase(it, PHASE_UPDATE)


def default_device(rank: int, device_count: Optional[int] = None) -> int:
    """The GPU of a process when none is given: one GPU per process, the node-local rank
    (torchrun's LOCAL_RANK, else the rank). A rank beyond this node's GPUs (a LOCAL_RANK
    inherited from an outer launcher, or a global rank of a multi-node run started without
    LOCAL_RANK) is an error rather than another process's GPU."""
    local = int(os.environ.get("LOCAL_RANK", rank))
    if device_count is None:
        import torch

        device_count = torch.cuda.device_count()
    if not 0 <= local < device_count:
        raise ValueError(f"local rank {local} has no GPU on this node ({device_count} visible); "
                         "pass device= explicitly or set LOCAL_RANK")
    return local


class ShardedSolver:
    """The simple gradient of one reconstruction over the ranks of the default process
    group (or `world`/`rank` given explicitly), one GPU per rank. `regularizer` is the
    argument tuple of Solver.set_regularizer (e.g. ("huber", 0.05) or ("gg", 0.0, 1.5));
    `weights`, a whole weight sinogram [P][v][u] (host array or tensor), makes it the
    weighted gradient, each rank keeping the weights of its own views."""

    def __init__(self, cfg, params, device: Optional[int] = None, rank: Optional[int] = None,
                 world: Optional[int] = None, regularizer: Optional[tuple] = None,
                 tuning: Optional[dict] = None, weights=None):
        import torch.distributed as dist

        from .operators import Context, Solver

        multi = dist.is_available() and dist.is_initialized()
        self.world = world if world is not None else (dist.get_world_size() if multi else 1)
        self.rank = rank if rank is not None else (dist.get_rank() if multi else 0)
        self.params = params
        self.begin, self.count = view_ranges(cfg.projection_nb, self.world)[self.rank]
        if device is None:
            device = default_device(self.rank)
        self.ctx = Context(cfg, device, views=(self.begin, self.count))
        if tuning:  # e.g. {"rs_layout": "hybrid"}; before the solver, which fixes its layout
            self.ctx.set_tuning(**tuning)
        self.solver = Solver(self.ctx, params)
        if regularizer is not None:
            self.solver.set_regularizer(*regularizer)
        if weights is not None:
            self.solver.set_weights(self.real_part(weights))
        self.dJ, self.norms = self.solver.buffers()

    def real_part(self, real_sinogram):
        """This rank's views of a whole real (or weight) sinogram [P][v][u]."""
        part = real_sinogram[self.begin:self.begin + self.count]
        return part.contiguous() if hasattr(part, "contiguous") else part.copy(order="C")

    def iterate(self, volume, real_part, first: int = 1, count: Optional[int] = None, allreduce=None) -> None:
        """Iterations [first, first + count) in place on the FP32 volume tensor (the same on
        every rank). `allreduce` defaults to torch.distributed's sum when world > 1."""
        import torch.distributed as dist

        count = self.params.gradient_iteration_nb - first + 1 if count is None else count
        if allreduce is None and self.world > 1:
            allreduce = lambda t: dist.all_reduce(t, op=dist.ReduceOp.SUM)  # noqa: E731

        def phase(it, bits):
            self.solver.phase(volume, real_part if bits & PHASE_GRADIENT else None, it, bits)

        iterate_exchange(phase, self.dJ, self.norms, first, count, self.params.optimal_step_iteration_nb, allreduce,
                         self.rank)

    def alphas(self):
        return self.solver.alphas()

    def close(self) -> None:
        self.solver.close()
        self.ctx.close()
