"""Sample decomposition over ranks and the end-of-job reduction.

The reference spreads samples over MPI ranks round-robin: in every round of
wSize configurations, rank r reads the r-th one (file offset
nrk * szCSet + wRank * szConf, Codes_Folder/smd_code.cpp:3128-3180), runs
get_dynSpectrum on it, and the root adds every rank's running sums of
|S(q,w)|^2 and of the autocorrelation into its own
(Codes_Folder/smd_code.cpp:3325-3397) before dividing by the sample count
(Codes_Folder/smd_code.cpp:3596-3611).

Here a rank is one GPU (one process, torch.distributed).  Samples are
independent, so there is no exchange during a job; the only collective is
one sum of the accumulators when the job ends.  ``reduce_sums`` takes any
process group: over NCCL the buffer goes to the rank's current GPU for the
collective, over gloo it stays on the host.
"""
from __future__ import annotations

from typing import Optional, Sequence, Tuple

import numpy as np


def rank_samples(n_samples: int, rank: int, world: int) -> np.ndarray:
    """Sample indices rank ``rank`` integrates: rank, rank + world, ...

    The reference's round-robin read order (Codes_Folder/smd_code.cpp:
    3128-3180).  Every sample lands on exactly one rank.
    """
    if world < 1 or not (0 <= rank < world):
        raise ValueError(f"rank {rank} outside a world of {world}")
    if n_samples < 0:
        raise ValueError("negative sample count")
    return np.arange(rank, n_samples, world, dtype=np.int64)


def reduce_sums(spec_sum: np.ndarray, qss_sum: np.ndarray, n_local: int,
                group=None, dst: Optional[int] = None) -> Tuple[np.ndarray, np.ndarray, int]:
    """Sum per-rank accumulators over the ranks of ``group``.

    spec_sum [3][Q][n_rec] and qss_sum [n_rec] are this rank's sums over its
    samples.  With dst = None every rank receives the totals (all-reduce);
    otherwise only rank dst does (reduce), as the reference's root.
    Returns (spec_total, qss_total, n_total) in FP64.
    """
    import torch
    import torch.distributed as dist

    spec = torch.from_numpy(np.ascontiguousarray(spec_sum, np.float64))
    qss = torch.from_numpy(np.ascontiguousarray(qss_sum, np.float64))
    cnt = torch.tensor([float(n_local)], dtype=torch.float64)
    flat = torch.cat([spec.reshape(-1), qss.reshape(-1), cnt])
    flat = flat.to(collective_device(group))
    if dst is None:
        dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    else:
        dist.reduce(flat, dst=dst, op=dist.ReduceOp.SUM, group=group)
    flat = flat.cpu()
    n_spec = spec.numel()
    out_spec = flat[:n_spec].reshape(spec.shape).numpy().copy()
    out_qss = flat[n_spec:n_spec + qss.numel()].reshape(qss.shape).numpy().copy()
    return out_spec, out_qss, int(round(float(flat[-1])))


def collective_device(group=None):
    """Where the collective's buffer must live: this rank's current CUDA
    device for an NCCL group (NCCL takes device tensors only), the host for
    gloo."""
    import torch
    import torch.distributed as dist

    if dist.get_backend(group) == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def average(spec_total: np.ndarray, qss_total: np.ndarray, n_total: int):
    """Sample averages of the reduced sums (Codes_Folder/smd_code.cpp:3596-3611)."""
    if n_total < 1:
        raise ValueError("no samples")
    f = 1.0 / n_total
    return spec_total * f, qss_total * f


def run_sharded(ctx, lattice_id: int, qset_id: int, spins: np.ndarray, dt: float, n_rec: int,
                rank: int, world: int, group=None, imp: Optional[np.ndarray] = None,
                **run_kw):
    """One job's samples spread over ranks; returns the all-sample averages.

    spins [S][N][3] (and imp [S][N]) hold every sample; this rank runs its
    share on its device through ``ctx.run`` and the sums are all-reduced.
    """
    idx = rank_samples(spins.shape[0], rank, world)
    Q = ctx.qset_size(qset_id)
    if len(idx):
        r = ctx.run(lattice_id, qset_id, spins[idx], dt, n_rec,
                    imp=None if imp is None else imp[idx], **run_kw)
        spec_sum, qss_sum = r.spec * len(idx), r.qss * len(idx)
    else:
        spec_sum, qss_sum = np.zeros((3, Q, n_rec)), np.zeros(n_rec)
    tot = reduce_sums(spec_sum, qss_sum, len(idx), group=group)
    return average(*tot)
