"""Row bands of one 2D domain (the multi-GPU decomposition), on CPU: the band
arithmetic, and two gloo ranks each stepping its band with the FP64 oracle in
band mode and swapping edge rows through rapidsolid.bands.exchange, against
the single-domain oracle run, bit for bit (noise on, a pull-back from the
global coarse tip)."""
import os
import socket
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_split_rows_and_band_params():
    from rapidsolid import bands, configs
    assert bands.split_rows(10, 3) == [(1, 4), (5, 7), (8, 10)]
    p = configs.small(48, 64)
    q = bands.band_params(p, 1, 3)
    assert (q.ny_all, q.j_offset, q.band) == (21 + 2, 21, 1)  # 62 rows: 21, 21, 20
    assert (q.nx_all, q.dx, q.seed) == (p.nx_all, p.dx, p.seed)
    with pytest.raises(ValueError):
        bands.band_params(p, 0, 11)


def _params():
    from rapidsolid import configs
    p = configs.small(48, 40, i_tip_target=12)
    p.noise_amplitude = 0.02
    p.seed = 99
    return p


def _band_state(p, pb):
    import pyoracle
    from rapidsolid import configs
    return pyoracle.initial_planar(pb, configs.C_LIQUID_TI10NB, configs.C_SOLID_AT_TLIQ, 5)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


NSTEPS = 25


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "2d-rapid-solidification_b200"))
    import datetime
    import pyoracle
    from rapidsolid import bands
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    p = _params()
    pb = bands.band_params(p, rank, world)
    d = pyoracle.derive(pb)
    s = _band_state(p, pb)

    def fields(st):
        return [torch.from_numpy(st.psi), torch.from_numpy(st.phi), torch.from_numpy(st.c)]

    bands.exchange(fields(s), rank, world)
    hist = 0
    for n in range(NSTEPS):
        if n == 0:  # the moving frame: global coarse tip = max over the bands
            it = torch.tensor([pyoracle.itip(pb, s.psi)], dtype=torch.int64)
            dist.all_reduce(it, op=dist.ReduceOp.MAX)
            off = int(it.item()) - p.i_tip_target
            s = pyoracle.pull_back(pb, s, off)
            hist += off
        s = pyoracle.step(pb, d, s, n, i_offset_history=hist)
        bands.exchange(fields(s), rank, world)
    out = [np.ascontiguousarray(a[1:-1]) for a in (s.psi, s.c)]
    q.put((rank, out, hist))
    dist.barrier()
    dist.destroy_process_group()


def test_two_bands_with_gloo_equal_the_single_domain():
    import pyoracle
    p = _params()
    d = pyoracle.derive(p)
    from rapidsolid import configs
    s = pyoracle.initial_planar(p, configs.C_LIQUID_TI10NB, configs.C_SOLID_AT_TLIQ, 5)
    off = pyoracle.itip(p, s.psi) - p.i_tip_target
    s = pyoracle.pull_back(p, s, off)
    for n in range(NSTEPS):
        s = pyoracle.step(p, d, s, n, i_offset_history=off)
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    res = {}
    for _ in range(world):
        rank, out, hist = q.get(timeout=300)
        res[rank] = (out, hist)
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    assert res[0][1] == res[1][1] == off
    psi = np.concatenate([res[r][0][0] for r in range(world)])
    c = np.concatenate([res[r][0][1] for r in range(world)])
    assert np.array_equal(psi, s.psi[1:-1]) and np.array_equal(c, s.c[1:-1])
