"""The multi-rank path on the CPU: world size 2 over gloo.

Pixels are independent, so ranks share no data: each rank inverts its own
shard (here with the oracle, on the CPU) and the results meet only where one
process writes them.  With the LM chi^2 carry made irrelevant (no
regularisation, so no ratio test), the gathered shards equal one process's
inversion of the whole map bit for bit; the timing reduction is the max over
ranks.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import me_ranks

WORLD = 2


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank, port, out_dir):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path[:0] = [os.path.join(os.path.dirname(here), "milne-eddington_b200"), here]
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(WORLD), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import me_b200
    import me_maps
    import me_ranks
    import oracle_bind as ob
    dist = me_ranks.init("gloo", 120)
    r, w, local = me_ranks.rank_env()
    assert (r, w, local) == (rank, WORLD, rank)
    name = "fe15648_64x64"
    ctl = me_maps.control_text(name, precision="FP64",
                               extra={"Btheta_Regularization": "NO"})
    cfg = me_b200.parse_config_text(ctl)
    lam = me_maps.wavelengths(name)
    orc = ob.Oracle(cfg, lam)
    npix = 61
    par = me_maps.draw_parameters(name, npix, 5)
    prof = me_maps.add_noise(orc.synth_many(par), 1e-3, 5)
    start, count = me_ranks.shard(npix, rank, WORLD)
    mine = ob.Oracle(cfg, lam).invert(prof[start:start + count])
    allres = me_ranks.gather_rows(mine, dist, WORLD)
    t = me_ranks.max_over_ranks(1.5 + rank, dist)
    s = me_ranks.sum_over_ranks(count, dist)
    if rank == 0:
        np.save(os.path.join(out_dir, "gathered.npy"), allres)
        np.save(os.path.join(out_dir, "whole.npy"), orc.invert(prof))
        np.save(os.path.join(out_dir, "reduced.npy"), np.array([t, s]))
    dist.barrier()
    dist.destroy_process_group()


def test_shard_covers_every_pixel_once():
    for total in (0, 1, 7, 61, 1 << 20):
        for world in (1, 2, 3, 8):
            spans = [me_ranks.shard(total, r, world) for r in range(world)]
            assert spans[0][0] == 0
            for (a, n), (b, _) in zip(spans, spans[1:]):
                assert a + n == b
            assert sum(n for _, n in spans) == total
            assert max(n for _, n in spans) - min(n for _, n in spans) <= 1
    assert len({me_ranks.map_seed(r) for r in range(8)}) == 8


def test_two_ranks_over_gloo(tmp_path):
    port = free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=worker, args=(r, port, str(tmp_path))) for r in range(WORLD)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    for p in procs:
        if p.is_alive():
            p.kill()
            pytest.fail("rank did not finish")
        assert p.exitcode == 0
    gathered = np.load(tmp_path / "gathered.npy")
    whole = np.load(tmp_path / "whole.npy")
    np.testing.assert_array_equal(gathered, whole)
    t, s = np.load(tmp_path / "reduced.npy")
    assert t == 2.5 and s == 61
