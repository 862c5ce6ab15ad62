"""Instance sharding over ranks (world size 2, gloo on CPU): each rank runs the
oracle's IMEX steps on its block of a parameter sweep, rank 0 gathers, and
the result equals the unsharded sweep instance by instance."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from turing_sphere_b200.shard import shard_range

LMAX, NLAT, NPHI, NSTEPS = 7, 8, 16, 3
N = 5  # instances: shards of 3 and 2


def sweep_params(k):
    # linear model (c, D, dt): growth rate varies per instance
    return [-0.2 + 0.05 * k, 0.01, 0.1]


def start_state(k):
    rng = np.random.default_rng(100 + k)
    nlm = (LMAX + 1) * (LMAX + 2) // 2
    return rng.standard_normal((1, 2 * nlm))


def run_instances(ks):
    from oracle import oracle as O
    ref = O.ShtReference(LMAX, LMAX, NLAT, NPHI, threads=1)
    return np.stack([ref.model_step("linear", sweep_params(k), start_state(k), NSTEPS)[0]
                     for k in ks])


def worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    import torch.distributed as dist
    from turing_sphere_b200.shard import gather_instances, max_over_ranks
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        start, count = shard_range(N, rank, world)
        local = run_instances(range(start, start + count))
        full = gather_instances(local, N)
        worst = max_over_ranks(float(rank + 1))
        if rank == 0:
            np.save(out, full)
            np.save(out + ".max.npy", np.array([worst]))
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_range_partitions():
    for n in (0, 1, 5, 8, 257):
        for world in (1, 2, 3, 8):
            blocks = [shard_range(n, r, world) for r in range(world)]
            assert sum(c for _, c in blocks) == n
            assert all(blocks[r][0] + blocks[r][1] == blocks[r + 1][0] for r in range(world - 1))
            assert max(c for _, c in blocks) - min(c for _, c in blocks) <= 1
    with pytest.raises(ValueError):
        shard_range(4, 2, 2)


def test_two_rank_sweep_equals_serial(tmp_path):
    out = str(tmp_path / "gathered.npy")
    ctx = mp.get_context("spawn")
    port = free_port()
    procs = [ctx.Process(target=worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    full = np.load(out)
    assert full.shape[0] == N
    np.testing.assert_array_equal(full, run_instances(range(N)))
    assert float(np.load(out + ".max.npy")[0]) == 2.0


# ------------------------------------------------ the library, sharded (GPU)
GPU_LMAX, GPU_STEPS = 31, 20


def gpu_sweep(k):
    from turing_sphere_b200 import defaultParams, mModelByKey
    p = defaultParams(mModelByKey("schnakenberg"))
    return dict(p, b=p["b"] + 0.02 * k)


def gpu_run(ks):
    """Schnakenberg instances ks through the library (one batched model on a
    tensor-core plan), spectral seed 1 + k; returns their U states."""
    from tests.test_model_gpu import spectral_seed
    from turing_sphere_b200 import ModelSession, mModelByKey, requestShtDevice
    dev = requestShtDevice(0)
    model = mModelByKey("schnakenberg")
    sweep = [gpu_sweep(k) for k in ks]
    s = ModelSession.create(dev, model, sweep, GPU_LMAX, batch=len(ks), precision="tf32x3")
    seeds = [spectral_seed(GPU_LMAX, sweep[i], 1 + k) for i, k in enumerate(ks)]
    s.gpu.upload("U", np.stack([q[0] for q in seeds]))
    s.gpu.upload("V", np.stack([q[1] for q in seeds]))
    s.step(GPU_STEPS)
    U = s.read("U").reshape(len(ks), -1)
    s.destroy()
    return U


def gpu_worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    import torch.distributed as dist
    from turing_sphere_b200.shard import gather_instances
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        start, count = shard_range(N, rank, world)
        # one GPU stands in for the ranks' GPUs here: the ranks take turns on it
        # (in production each rank drives its own device)
        local = None
        for turn in range(world):
            if turn == rank:
                local = gpu_run(list(range(start, start + count)))
            dist.barrier()
        full = gather_instances(local, N)
        if rank == 0:
            np.save(out, full)
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_two_rank_library_sweep_equals_unsharded(tmp_path):
    """The sharded path of the library itself: two ranks (gloo for the gather;
    both on GPU 0, each with its own CUDA context and its own block of a
    5-instance Schnakenberg sweep, taking turns on the GPU) run their blocks
    through the C ABI; the gathered states match the f64 oracle stepping each
    instance alone, and the unsharded batch run in this process, instance by
    instance."""
    from tests.conftest import HAS_GPU
    if not HAS_GPU:
        pytest.skip("no CUDA device")
    from oracle import oracle as O
    from tests.test_model_gpu import spectral_seed
    from turing_sphere_b200 import gridForLmax
    out = str(tmp_path / "gathered_gpu.npy")
    ctx = mp.get_context("spawn")
    port = free_port()
    procs = [ctx.Process(target=gpu_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    full = np.load(out)
    nlat, nphi = gridForLmax(GPU_LMAX, 3)
    ref = O.ShtReference(GPU_LMAX, GPU_LMAX, nlat, nphi)
    want = []
    for k in range(N):
        p = gpu_sweep(k)
        st = np.stack(spectral_seed(GPU_LMAX, p, 1 + k)).astype(np.float64)
        want.append(ref.model_step("schnakenberg", [p[n] for n in ("a", "b", "D1", "D2", "dt")],
                                   st, GPU_STEPS)[0])
    here = gpu_run(list(range(N)))
    assert full.shape == here.shape
    e_sharded = [O.rel_l2(full[k], want[k]) for k in range(N)]
    e_here = [O.rel_l2(here[k], want[k]) for k in range(N)]
    if max(e_sharded) >= 1e-5 or max(e_here) >= 1e-5:
        # which neighbouring run each wrong row matches: one step fewer or
        # more, or another instance's parameters
        diag = {}
        for k in range(N):
            if e_sharded[k] < 1e-5:
                continue
            p = gpu_sweep(k)
            st = np.stack(spectral_seed(GPU_LMAX, p, 1 + k)).astype(np.float64)
            prm = [p[n] for n in ("a", "b", "D1", "D2", "dt")]
            d = {f"steps{n}": O.rel_l2(full[k], ref.model_step("schnakenberg", prm, st, n)[0])
                 for n in (GPU_STEPS - 1, GPU_STEPS + 1)}
            for j in range(N):
                q = gpu_sweep(j)
                d[f"params{j}"] = O.rel_l2(full[k], ref.model_step(
                    "schnakenberg", [q[n] for n in ("a", "b", "D1", "D2", "dt")], st, GPU_STEPS)[0])
            diag[k] = d
        raise AssertionError((e_sharded, e_here, diag))
    for k in range(N):
        assert O.rel_l2(full[k], here[k]) < 1e-6, k
