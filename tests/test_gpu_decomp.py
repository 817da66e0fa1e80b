"""Mesh decomposition on the GPU: the ranks of a decomposed estuary, each a
model on its sub-mesh (all on this one GPU, halos exchanged through the
host after every internal step), give the bits of the undecomposed run on
every rank's own nodes and elements, in both precision forms."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# halo rings deep enough for one internal step of the estuary
# configuration (10 sub-steps, MUSCL tracers, filters, wetting / drying):
# 12 is the shallowest that is exact (8 is not); the library's default
# (decomp.DEFAULT_HALO) keeps a margin for the wider-stencil options
HALO = 12


def _case(fp32=0, **kw):
    from fesomc import cases
    c = cases.estuary_case("decomp", 160, 40, 300.0, 11, 2.0, 25.0, stress=(0.0, 0.05), **kw)
    c.params.fp32_form = fp32
    return c


def _whole(case, steps):
    from fesomc import model
    g = model.GpuModel(case)
    try:
        assert g.step(steps) == 0
        return g.state(), g.energy()
    finally:
        g.close()


@pytest.mark.parametrize("nranks,fp32", [(2, 0), (3, 0), (2, 1)])
def test_decomposed_run_gives_the_bits_of_the_whole_mesh(built, nranks, fp32):
    from fesomc import decomp
    steps = 12
    case = _case(fp32)
    ref, _ = _whole(case, steps)
    d = decomp.Decomposition(case, nranks, HALO)
    lr = decomp.LocalRanks(d)
    try:
        lr.step(steps)
        got = lr.assemble()
    finally:
        lr.close()
    for k, v in got.items():
        assert np.array_equal(v, ref[k]), (k, int(np.sum(v != ref[k])))


@pytest.mark.parametrize("opts", [
    {"bih_3D": 1, "bih_2D": 1},
    {"filt_bi_3D": 1, "filt_bi_2D": 1, "tracer_adv": 1},
])
def test_default_halo_covers_the_wider_stencils(built, opts):
    """The biharmonic and filter-2x viscosities reach further; the default
    halo depth still gives the whole-mesh bits."""
    from fesomc import decomp
    steps = 6
    case = _case(0, **opts)
    ref, _ = _whole(case, steps)
    d = decomp.Decomposition(case, 2, decomp.DEFAULT_HALO)
    lr = decomp.LocalRanks(d)
    try:
        lr.step(steps)
        got = lr.assemble()
    finally:
        lr.close()
    for k, v in got.items():
        assert np.array_equal(v, ref[k]), (k, int(np.sum(v != ref[k])))


def test_a_shallow_halo_departs(built):
    """With one ring the cut stencils reach the owned entities within a
    step: the test above is not passing by accident."""
    from fesomc import decomp
    case = _case(0)
    ref, _ = _whole(case, 2)
    d = decomp.Decomposition(case, 2, 1)
    lr = decomp.LocalRanks(d)
    try:
        lr.step(2)
        got = lr.assemble()
    finally:
        lr.close()
    assert any(not np.array_equal(v, ref[k]) for k, v in got.items())


def test_tracer_range_is_checked(built):
    import ctypes as C
    from fesomc import abi, model
    g = model.GpuModel(_case(0))
    try:
        bad = np.array([2.0, 1.0, 0.0, 1.0])
        assert g.lib.fesomc_gpu_set_tracer_range(g.h, abi.dptr(bad)) == 1
        nan = np.array([0.0, np.nan, 0.0, 1.0])
        assert g.lib.fesomc_gpu_set_tracer_range(g.h, abi.dptr(nan)) == 1
        # the model's own range given back: the same bits as without
        ref = model.GpuModel(_case(0))
        try:
            for _ in range(3):
                st = g.state()
                L = g.case.mesh.L
                t, s = st["TF"].reshape(-1, L), st["SF"].reshape(-1, L)
                rng = np.array([t.min(), t.max(), s.min(), s.max()])
                assert g.lib.fesomc_gpu_set_tracer_range(g.h, abi.dptr(rng)) == 0
                g.step(1)
                ref.step(1)
            a, b = g.state(), ref.state()
            for k in a:
                if not k.startswith("_"):
                    assert np.array_equal(a[k], b[k]), k
            assert g.lib.fesomc_gpu_set_tracer_range(g.h, None) == 0
        finally:
            ref.close()
    finally:
        g.close()


@pytest.mark.parametrize("fp32,sfc", [(0, 0), (1, 0), (0, 1)])
def test_device_halo_exchange_gives_the_same_bits(built, fp32, sfc):
    """The halos packed and unpacked on the device (fesomc_gpu_halo_*), the
    tracer range from the device: the bits of the whole-mesh run, also with
    every model storing its sub-mesh along the Hilbert curve (the plans'
    indices mapped to the storage order)."""
    from fesomc import decomp
    steps = 8
    case = _case(fp32)
    case.params.sfc_order = sfc
    ref, _ = _whole(case, steps)
    dr = decomp.DeviceRanks(decomp.Decomposition(case, 3, HALO))
    try:
        dr.step(steps)
        got = dr.assemble()
    finally:
        dr.close()
    for k, v in got.items():
        assert np.array_equal(v, ref[k]), (k, int(np.sum(v != ref[k])))


def _dist_rank(rank, world, port, path, steps):
    import os
    import torch.distributed as dist
    from fesomc import decomp
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        r = decomp.DistRank(_case(0), dist, HALO)
        try:
            r.step(steps)
            st = r.own_state()
            np.savez(os.path.join(path, "r%d.npz" % rank), **{k: v for k, v in st.items() if not k.startswith("_")})
        finally:
            r.close()
    finally:
        dist.destroy_process_group()


def test_one_rank_per_process(built, tmp_path):
    """Two processes (gloo between them; both on this one GPU, no kernel of
    one waits on the other), each a rank with its own model: the assembled
    owned state equals the whole-mesh run."""
    import socket
    import torch.multiprocessing as mp
    from fesomc import decomp
    steps = 6
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    mp.start_processes(_dist_rank, args=(2, port, str(tmp_path), steps), nprocs=2, join=True, start_method="spawn")
    case = _case(0)
    d = decomp.Decomposition(case, 2, HALO)
    states = [dict(np.load(tmp_path / ("r%d.npz" % r))) for r in range(2)]
    got = d.assemble(states)
    ref, _ = _whole(case, steps)
    for k, v in got.items():
        assert np.array_equal(v, ref[k]), (k, int(np.sum(v != ref[k])))

