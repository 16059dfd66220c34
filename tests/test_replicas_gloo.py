"""CPU, world_size 2 over gloo: the replica path (frame sharding, max-over-ranks timing, gather) with
the oracle forming the frames, compared with one process forming all of them."""
import os
import socket

import numpy as np
import pytest

from pfa_b200 import replicas


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, ws, port, out_path):
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    sys.path[:0] = [str(root), str(root / "mpfs250t-sar-ifp_b200")]
    import json
    import time
    import torch.distributed as dist
    from datetime import timedelta
    from oracle import fixed_emulator as fe
    from pfa_b200 import geometry, replicas, synth
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=timedelta(seconds=60))
    frames = [(40 + 3 * k, 36 + 2 * k) for k in range(5)]           # uneven frame list
    local = {}
    t0 = time.perf_counter()
    for f in replicas.shard(len(frames), rank, ws):
        m, n = frames[f]
        sc = synth.make_scene(m, n, n_targets=3, seed=100 + f)
        img, _ = fe.form_image(sc.signal, geometry.prepare_tables_from_scene(sc), 64, True, True)
        local[f] = fe.frame_crc(img)
    elapsed = (time.perf_counter() - t0) * 1000.0 + 1000.0 * rank   # rank 1 pretends to be slower
    mpf = replicas.ms_per_frame(elapsed, len(frames))
    merged = replicas.gather_results(local)
    if rank == 0:
        Path(out_path).write_text(json.dumps({"crc": {str(k): v for k, v in merged.items()}, "mpf": mpf,
                                              "elapsed0": elapsed}))
    dist.destroy_process_group()


def test_shard_covers_every_frame_once():
    for ws in (1, 2, 3, 8):
        got = sorted(sum((replicas.shard(13, r, ws) for r in range(ws)), []))
        assert got == list(range(13))


def test_gloo_world2_replicas_match_single_process(tmp_path):
    import json
    import torch.multiprocessing as mp
    from oracle import fixed_emulator as fe
    from pfa_b200 import geometry, synth
    out = tmp_path / "res.json"
    mp.start_processes(_worker, args=(2, _free_port(), str(out)), nprocs=2, start_method="spawn", join=True)
    res = json.loads(out.read_text())
    frames = [(40 + 3 * k, 36 + 2 * k) for k in range(5)]
    for f, (m, n) in enumerate(frames):
        sc = synth.make_scene(m, n, n_targets=3, seed=100 + f)
        img, _ = fe.form_image(sc.signal, geometry.prepare_tables_from_scene(sc), 64, True, True)
        assert res["crc"][str(f)] == fe.frame_crc(img)
    # the slow rank (rank 1, +1000 ms) sets the whole-job time
    assert res["mpf"] >= 1000.0 / len(frames)
