"""CPU tests of the multi-rank host logic with real process groups (gloo, 127.0.0.1): the t-slab halo exchange of
kuqcd_b200/slab.py (which faces travel to which rank, in which order -- two ranks exercise the case where both
neighbours are the same peer), the reductions the distributed CG sums over ranks, and the bench launcher's
contract that under torchrun only rank 0 runs the reference arm."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from kuqcd_b200 import slab as SL
from oracle import oracle as O

ROOT = Path(__file__).resolve().parent.parent
GDIMS = (4, 2, 2, 24)


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _exchange_worker(rank, world, port, out_dir):
    import torch.distributed as dist

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        tr = SL.TorchTransport()
        glob = O.make_source(GDIMS, 0, 17)                      # global parity-0 field, host record
        loc = SL.slab_of_spinor(glob, GDIMS, rank, world).reshape(-1, 6)
        S = GDIMS[0] * GDIMS[1] * GDIMS[2] // 2
        lt = GDIMS[3] // world
        lo = torch.from_numpy(np.ascontiguousarray(loc[:3 * S]))           # slices 0..2
        hi = torch.from_numpy(np.ascontiguousarray(loc[(lt - 3) * S:]))    # slices lt-3..lt-1
        (glo, ghi), = tr.exchange([(lo, hi)])
        red = tr.allreduce([np.array([rank + 1.0, 2.0 ** rank])])[0]
        # the device-driven solver's in-place reduction of one slice of a state tensor
        state = torch.tensor([rank + 1.0, 10.0 * rank, -1.0], dtype=torch.float64)
        tr.allreduce_inplace([state[1:2]])
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), glo=glo.numpy(), ghi=ghi.numpy(), red=red,
                 state=state.numpy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3, 4])
def test_slab_halo_exchange_gloo(tmp_path, world):
    mp.spawn(_exchange_worker, args=(world, free_port(), str(tmp_path)), nprocs=world, join=True)
    glob = O.make_source(GDIMS, 0, 17).reshape(-1, 6)
    S = GDIMS[0] * GDIMS[1] * GDIMS[2] // 2
    nt, lt = GDIMS[3], GDIMS[3] // world
    for r in range(world):
        z = np.load(tmp_path / f"r{r}.npz")
        t0 = r * lt
        want_lo = np.concatenate([glob[((t0 - 3 + s) % nt) * S:((t0 - 3 + s) % nt + 1) * S] for s in range(3)])
        want_hi = np.concatenate([glob[((t0 + lt + s) % nt) * S:((t0 + lt + s) % nt + 1) * S] for s in range(3)])
        assert np.array_equal(z["glo"], want_lo), r
        assert np.array_equal(z["ghi"], want_hi), r
        assert np.allclose(z["red"], [world * (world + 1) / 2, 2.0 ** world - 1])
        assert np.array_equal(z["state"], [r + 1.0, 10.0 * world * (world - 1) / 2, -1.0])


def test_slab_record_slicing_round_trip():
    fat, lng = O.make_links(GDIMS, 0.3, 3)
    b = O.make_source(GDIMS, 1, 4)
    R = 3
    assert np.array_equal(SL.join_spinor([SL.slab_of_spinor(b, GDIMS, r, R) for r in range(R)]), b)
    # links: even halves then odd halves of the slabs reassemble the global record
    parts = [SL.slab_of_links(fat, GDIMS, r, R).reshape(2, -1) for r in range(R)]
    rebuilt = np.concatenate([np.concatenate([p[par] for p in parts]) for par in (0, 1)])
    assert np.array_equal(rebuilt, fat)
    # a slab of the links is the record of the local lattice: the oracle dslash of a 1-slab split is the global one
    assert np.array_equal(SL.slab_of_links(fat, GDIMS, 0, 1), fat)


def test_local_transport_is_periodic_ring():
    tr = SL.LocalTransport()
    faces = [(f"lo{r}", f"hi{r}") for r in range(4)]
    assert tr.exchange(faces) == [("hi3", "lo1"), ("hi0", "lo2"), ("hi1", "lo3"), ("hi2", "lo0")]
    assert [list(v) for v in tr.allreduce([[1.0, 2.0], [3.0, 4.0]])] == [[4.0, 6.0], [4.0, 6.0]]
    st = [torch.tensor([1.0, 2.0, 3.0], dtype=torch.float64), torch.tensor([4.0, 5.0, 6.0], dtype=torch.float64)]
    tr.allreduce_inplace([t[0:2] for t in st])
    assert [t.tolist() for t in st] == [[5.0, 7.0, 3.0], [5.0, 7.0, 6.0]]


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built here")
def test_bench_reference_arm_under_torchrun_rank0_only():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(free_port()), str(ROOT / "bench.py"), "--impl", "reference", "--gpus",
           "2", "--steps", "1", "--warmup", "0", "--cpu-sample-iters", "1", "--dims", "4", "4", "4", "4"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["e2e"]["h2d_bytes_per_step"] == 0


def _dead_peer_worker(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=5))
    if rank == 1:
        return  # leaves between steps, with nothing in flight: never joins the exchange
    tr = SL.TorchTransport()
    t = torch.zeros(16, dtype=torch.float64)
    try:
        tr.exchange([(t, t.clone())])
        outcome = "returned"
    except Exception as exc:  # the process group's timeout ends the wait with an error
        outcome = "error: " + type(exc).__name__
    with open(os.path.join(out_dir, "r0.txt"), "w") as f:
        f.write(outcome)


def test_slab_exchange_with_a_dead_peer_fails_with_an_error(tmp_path):
    """Failure detection on the host: a rank that never joins the halo exchange makes the others' exchange end
    with an error after the process group's (short) timeout instead of waiting for good."""
    mp.spawn(_dead_peer_worker, args=(2, free_port(), str(tmp_path)), nprocs=2, join=True)
    outcome = (tmp_path / "r0.txt").read_text()
    assert outcome.startswith("error"), outcome


def test_slab_relaxed_precision_schedule():
    """The slab mixed solver's precision schedule: FP64 until |r| < rho32 |b|, FP32 until rho16 |b|, then HALF, with
    the single-GPU solver's thresholds (target 1e-10: rho32 = 1e-4, rho16 = 3e-8); no HALF phase for sloppy FP32."""
    import kuqcd_b200 as K

    r32, r16 = SL.relaxed_thresholds(1e-10)
    assert np.isclose(r32, 1e-4) and np.isclose(r16, 3e-8)
    assert SL.relaxed_thresholds(1e-10, sloppy=K.KUQCD_SINGLE)[1] == 0.0
    pick = [SL.relaxed_precision(rel ** 2, r32, r16) for rel in (1.0, 2e-4, 9e-5, 1e-6, 4e-8, 2e-8, 1e-10)]
    assert pick == [K.KUQCD_DOUBLE] * 2 + [K.KUQCD_SINGLE] * 3 + [K.KUQCD_HALF] * 2
    assert SL.relaxed_precision(1e-20, r32, 0.0) == K.KUQCD_SINGLE
