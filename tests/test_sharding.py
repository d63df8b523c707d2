"""Sample decomposition and the end-of-job reduction across ranks (host side,
world size 2 over gloo on the CPU).  Each rank's partial sums come from the
oracle on its own samples; the reduced averages must equal the
single-process average over all samples."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from classical_mc_and_smd_for_2d_heisenberg_models_b200 import sharding

N_SAMPLES, N_REC = 5, 16


@pytest.mark.parametrize("n,world", [(0, 1), (1, 2), (5, 2), (64, 3), (7, 8)])
def test_rank_samples_cover_every_sample_once(n, world):
    parts = [sharding.rank_samples(n, r, world) for r in range(world)]
    allv = np.sort(np.concatenate(parts)) if parts else np.array([])
    assert np.array_equal(allv, np.arange(n))
    for r, p in enumerate(parts):
        assert np.all(p % world == r)   # the reference's round-robin read order


def test_rank_samples_rejects_bad_ranks():
    with pytest.raises(ValueError):
        sharding.rank_samples(4, 2, 2)
    with pytest.raises(ValueError):
        sharding.rank_samples(4, 0, 0)


def _problem():
    from classical_mc_and_smd_for_2d_heisenberg_models_b200 import samples as smp, smd
    from classical_mc_and_smd_for_2d_heisenberg_models_b200.settings import SMDSettings
    s = SMDSettings(geom="square", L=4, J2=0.6, dtm=0.01, ntm=N_REC, window="hann1")
    spins, _ = smp.make_samples(s, N_SAMPLES, "stripe", 0.3, 11)
    return s, spins, smd.window("hann1", N_REC)


def _oracle_sums(s, spins, win, idx):
    import oracle
    m = oracle.Model(s, oracle.make_lattice(s.geom, s.L))
    spec, qss = 0.0, 0.0
    for k in idx:
        o = oracle.dyn_spectrum(m, spins[k], s.dtm, N_REC, stride=2, win=win)
        spec = spec + o["spec"]
        qss = qss + o["qss"]
    if len(idx) == 0:
        G = oracle.make_lattice(s.geom, s.L)["G"]
        return np.zeros((3, G * G, N_REC)), np.zeros(N_REC)
    return spec, qss


def _rank_main(rank, world, port, out_dir, use_reduce):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        s, spins, win = _problem()
        idx = sharding.rank_samples(N_SAMPLES, rank, world)
        spec, qss = _oracle_sums(s, spins, win, idx)
        tot = sharding.reduce_sums(spec, qss, len(idx), dst=0 if use_reduce else None)
        if rank == 0 or not use_reduce:
            a_spec, a_qss = sharding.average(*tot)
            np.savez(os.path.join(out_dir, f"r{rank}.npz"), spec=a_spec, qss=a_qss, n=tot[2])
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


@pytest.mark.parametrize("use_reduce", [False, True])
def test_two_rank_reduction_equals_single_process(tmp_path, oracle_mod, use_reduce):
    world = 2
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, str(tmp_path), use_reduce))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    for p in procs:
        if p.is_alive():
            p.kill()
        assert p.exitcode == 0
    s, spins, win = _problem()
    spec, qss = _oracle_sums(s, spins, win, range(N_SAMPLES))
    ref_spec, ref_qss = spec / N_SAMPLES, qss / N_SAMPLES
    ranks = [0] if use_reduce else [0, 1]
    for r in ranks:
        d = np.load(os.path.join(str(tmp_path), f"r{r}.npz"))
        assert int(d["n"]) == N_SAMPLES
        assert np.allclose(d["spec"], ref_spec, rtol=1e-13, atol=1e-15 * np.abs(ref_spec).max())
        assert np.allclose(d["qss"], ref_qss, rtol=1e-13, atol=1e-15)


@pytest.mark.gpu
def test_run_sharded_over_nccl_one_rank(ctx):
    """run_sharded over an NCCL process group (one rank: the GPU box has one
    GPU): the accumulators go through a device-tensor all-reduce and the
    averages equal the plain run's."""
    import torch
    import torch.distributed as dist
    from classical_mc_and_smd_for_2d_heisenberg_models_b200 import smd
    s, spins, win = _problem()
    lat = smd.build_lattice(s.geom, s.L)
    lid = ctx.lattice(s, lat)
    qid = ctx.qset(lid)
    direct = ctx.run(lid, qid, spins, s.dtm, N_REC, stride=2, win=win)
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0,
                            world_size=1)
    try:
        assert sharding.collective_device().type == "cuda"
        spec, qss = sharding.run_sharded(ctx, lid, qid, spins, s.dtm, N_REC, 0, 1, win=win,
                                         stride=2)
    finally:
        dist.destroy_process_group()
    assert np.allclose(spec, direct.spec, rtol=1e-14, atol=1e-16 * np.abs(direct.spec).max())
    assert np.allclose(qss, direct.qss, rtol=1e-14, atol=1e-16)
