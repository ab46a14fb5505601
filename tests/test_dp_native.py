"""The framework-free data-parallel path: NCCL's id handed from rank 0 to the other
ranks over a TCP socket (three spawned processes, no torch), the library making an NCCL
id (NCCL opened at run time; no GPU needed for the id), and the C-ABI argument checks."""
import ctypes
import importlib
import multiprocessing as mp
import socket

import pytest

DP = importlib.import_module("home-measure-privacy_b200.data_parallel")


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    payload = bytes(range(128)) if rank == 0 else None
    q.put((rank, DP.exchange_id(rank, world, "127.0.0.1", port, payload, timeout=30.0)))


def test_exchange_id_reaches_every_rank():
    port, world = free_port(), 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=60) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(got[r] == bytes(range(128)) for r in range(world))


def test_exchange_id_single_rank_and_bad_rank():
    assert DP.exchange_id(0, 1, "127.0.0.1", 0, b"abc") == b"abc"
    with pytest.raises(ValueError):
        DP.exchange_id(2, 2, "127.0.0.1", 0, b"abc")


def test_nccl_unique_id(native_lib):
    buf = ctypes.create_string_buffer(128)
    assert native_lib.gs_dp_unique_id(buf, 127) == -1  # too small
    rc = native_lib.gs_dp_unique_id(buf, 128)
    if rc == -7:
        pytest.skip("NCCL not available: " + native_lib.gs_last_error().decode())
    assert rc == 0
    assert any(buf.raw)  # an id was written
    assert native_lib.gs_dp_init(None, buf, 128, 0, 1) == -1  # no context
