"""Multi-process plumbing on CPU (gloo, world size 2): per-rank seeds and sector
shares, the maximum over ranks that every multi-GPU bench figure uses, and
sector sharding with real engine output: each rank opens host-only contexts
for its share of the g12 sectors and writes their row-mixing sidecars; the
union of the ranks' files equals one process's files byte for byte."""
import multiprocessing as mp
import os
import socket

import pytest

from prym_green_ancillary_b200 import sharding


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world_size, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world_size),
                      LOCAL_RANK=str(rank))
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world_size, timeout=timedelta(seconds=60))
    try:
        r, w, lr = sharding.world()
        got = sharding.max_over_ranks([1.0 + r, 10.0 - r])
        out.put((rank, (r, w, lr), got, sharding.assign_sectors(7, w, r), sharding.rank_seed(20, r)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, w0, max0, s0, seed0), (r1, w1, max1, s1, seed1) = results
    assert w0 == (0, 2, 0) and w1 == (1, 2, 1)
    assert max0 == max1 == [2.0, 10.0]              # element-wise maximum over the ranks
    assert sorted(s0 + s1) == list(range(7)) and not set(s0) & set(s1)   # disjoint, covering
    assert seed0 == 20 and seed1 == 1020


def test_single_process_is_identity():
    assert sharding.max_over_ranks([3.5]) == [3.5]
    assert sharding.assign_sectors(4, 1, 0) == [0, 1, 2, 3]



def _sidecar_worker(rank, world_size, port, out_dir, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world_size),
                      LOCAL_RANK=str(rank))
    import torch.distributed as dist
    from datetime import timedelta
    from pathlib import Path
    from prym_green_ancillary_b200 import CyclicEngine
    dist.init_process_group("gloo", rank=rank, world_size=world_size, timeout=timedelta(seconds=60))
    try:
        instance = Path(__file__).resolve().parent / "golden" / "g12_p661.json"
        written = []
        for sector in sharding.assign_sectors(6, world_size, rank):   # g12 has 6 sectors
            with CyclicEngine(instance, sector, device=-1) as eng:
                wdm = eng.output_path(out_dir)
                eng.write_sidecar(wdm)
                written.append(Path(wdm).name)
        dist.barrier()
        out.put((rank, written))
    finally:
        dist.destroy_process_group()


def _sidecars(directory):
    from pathlib import Path
    return {f.name: f.read_text().replace(str(directory), "<out>")
            for f in sorted(Path(directory).glob("*.rowmix.json"))}


def test_sector_shards_write_the_single_process_sidecars(tmp_path):
    from pathlib import Path
    from prym_green_ancillary_b200 import CyclicEngine
    instance = Path(__file__).resolve().parent / "golden" / "g12_p661.json"
    single = tmp_path / "single"
    for sector in range(6):
        with CyclicEngine(instance, sector, device=-1) as eng:
            eng.write_sidecar(eng.output_path(single))
    sharded = tmp_path / "sharded"
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_sidecar_worker, args=(r, 2, port, str(sharded), q)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, files0), (r1, files1) = results
    assert files0 and files1 and not set(files0) & set(files1)   # disjoint shares, both ranks did work
    want = _sidecars(single)
    assert len(want) == 6
    assert _sidecars(sharded) == want
