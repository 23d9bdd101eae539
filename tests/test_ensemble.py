"""Batched ensembles (many small shells stepped through one CUDA graph), the
tile autotuner, and the split of an ensemble over ranks.

CPU: the seeded shell study and the LPT bin-packing, including a 2-rank
gloo run that checks every member lands on exactly one rank.  GPU: an
ensemble step equals stepping each member alone, bit for bit (the graph
replays the very kernels css_step_rk4 launches), a member matches the
oracle, autotuning changes no result bit, and a non-finite member is
reported by index."""
import os

import numpy as np
import pytest

from css_b200 import ensemble as E


def test_shell_specs_follow_the_study_ranges():
    specs = E.shell_specs(48, seed=7)
    assert len(specs) == 48
    assert specs == E.shell_specs(48, seed=7)
    assert sum(s["magnetic"] for s in specs) == 24
    for s in specs:
        assert E.NR_RANGE[0] <= s["nr"] <= E.NR_RANGE[1]
        assert E.NTH_RANGE[0] <= s["nth"] <= E.NTH_RANGE[1] and s["nth"] % 16 == 0
        assert E.NPHI_RANGE[0] <= s["nphi"] <= E.NPHI_RANGE[1] and s["nphi"] % 16 == 0
        assert 1e4 <= s["ra"] <= 1e6 and 0.3 <= s["ro"] <= 3.0
        if s["magnetic"]:
            assert E.PM_RANGE[0] <= s["pm"] <= E.PM_RANGE[1]
        else:
            assert s["pm"] is None
        nnr, nnt, nnp = s["decomp"]
        assert nnr >= 2 and nnt >= 2 and nnp >= 3
        for n, nb in ((s["nr"], nnr), (s["nth"], nnt), (s["nphi"], nnp)):
            assert n % nb == 0 and (n // nb) % 2 == 0 and 10 <= n // nb <= 256


def test_lpt_partition_covers_each_member_once_and_balances():
    specs = E.shell_specs(48, seed=7)
    costs = [E.member_cost(s) for s in specs]
    for nranks in (1, 2, 3, 8):
        parts = E.lpt_partition(costs, nranks)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        # LPT: the most loaded rank exceeds the least loaded by at most one member
        assert max(loads) - min(loads) <= max(costs)


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    specs = E.shell_specs(48, seed=7)
    mine = E.lpt_partition([E.member_cost(s) for s in specs], world)[rank]
    got = [None] * world
    dist.all_gather_object(got, mine)
    if rank == 0:
        out.put(got)
    dist.barrier()
    dist.destroy_process_group()


def test_lpt_partition_over_two_gloo_ranks():
    import multiprocessing as mp
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    a, b = set(got[0]), set(got[1])
    assert not (a & b) and a | b == set(range(48))


TINY = [  # oracle-sized members: blocks of 10 points
    {"nr": 20, "nth": 20, "nphi": 30, "ra": 1e5, "ro": 0.5, "magnetic": False, "pm": None, "decomp": (2, 2, 3)},
    {"nr": 20, "nth": 20, "nphi": 30, "ra": 3e5, "ro": 1.5, "magnetic": True, "pm": 3.0, "decomp": (2, 2, 3)},
    {"nr": 20, "nth": 30, "nphi": 40, "ra": 1e4, "ro": 2.5, "magnetic": False, "pm": None, "decomp": (2, 3, 4)},
    {"nr": 30, "nth": 20, "nphi": 30, "ra": 2e4, "ro": 0.4, "magnetic": True, "pm": 1.2, "decomp": (3, 2, 3)},
]


def _oracle_rank_main(rank, world, port, out):
    """One rank of a CPU ensemble run: LPT share of TINY, each member stepped
    through the oracle; the final states gathered on rank 0."""
    import torch.distributed as dist
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    O.set_threads(2)
    mine = E.lpt_partition([E.member_cost(s) for s in TINY], world)[rank]
    states = {}
    for i in mine:
        p, prof, v0, dt = E.build_member(TINY[i], seed=100 + i)
        orc = O.Oracle(p, prof)
        states[i] = orc.step(v0, dt, 3)
        orc.close()
    got = [None] * world
    dist.all_gather_object(got, states)
    if rank == 0:
        out.put(got)
    dist.barrier()
    dist.destroy_process_group()


def test_ensemble_stepped_over_two_gloo_ranks_through_the_oracle():
    """Each of two gloo ranks steps its LPT share of the members (3 RK4
    steps, the FP64 oracle); every member comes back once and equals the
    same member stepped in one process."""
    import multiprocessing as mp
    import socket
    from oracle import oracle as O
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_oracle_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=600)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert not (set(got[0]) & set(got[1])) and set(got[0]) | set(got[1]) == set(range(len(TINY)))
    states = {**got[0], **got[1]}
    for i, spec in enumerate(TINY):
        p, prof, v0, dt = E.build_member(spec, seed=100 + i)
        want = O.Oracle(p, prof).step(v0, dt, 3)
        assert np.array_equal(states[i], want), i


# ---------------------------------------------------------------------------
SMALL = [
    {"nr": 24, "nth": 32, "nphi": 64, "ra": 1e5, "ro": 0.5, "magnetic": False, "decomp": (2, 2, 4)},
    {"nr": 32, "nth": 64, "nphi": 128, "ra": 3e5, "ro": 1.0, "magnetic": True, "decomp": (2, 2, 4)},
    {"nr": 52, "nth": 48, "nphi": 96, "ra": 1e4, "ro": 2.0, "magnetic": False, "decomp": (2, 3, 6)},
]


@pytest.mark.gpu
def test_ensemble_step_equals_members_stepped_alone(gpu_available):
    from css_b200.context import Simulation
    members = [E.build_member(s, seed=11 + i) for i, s in enumerate(SMALL)]
    alone = []
    for p, prof, v0, dt in members:
        sim = Simulation(p, prof)
        sim.upload(v0)
        sim.step_rk4(dt, 3)
        alone.append(sim.download())
        sim.close()
    sims = [Simulation(p, prof) for p, prof, _, _ in members]
    for sim, (_, _, v0, _) in zip(sims, members):
        sim.upload(v0)
    ens = E.Ensemble(sims)
    dts = [m[3] for m in members]
    ens.step(dts, 1)
    ens.step(dts, 2)  # replays the captured graph
    assert ens.launches() > 0
    for sim, ref in zip(sims, alone):
        assert np.array_equal(sim.download(), ref)
    ens.close()


@pytest.mark.gpu
def test_ensemble_member_matches_oracle(gpu_available):
    from css_b200.context import Simulation
    from oracle import oracle as O
    p, prof, v0, dt = E.build_member(SMALL[2], seed=3)
    sim = Simulation(p, prof)
    sim.upload(v0)
    ens = E.Ensemble([sim])
    ens.step([dt], 2)
    want = O.Oracle(p, prof).step(v0, dt, 2)
    got = sim.download()
    err = max(float(np.abs(got[i] - want[i]).max() / np.abs(want[i]).max()) for i in range(got.shape[0]))
    assert err < 1e-11, err


@pytest.mark.gpu
def test_ensemble_reports_the_non_finite_member(gpu_available):
    from css_b200._lib import CssError
    from css_b200.context import Simulation
    members = [E.build_member(s, seed=5) for s in SMALL[:2]]
    sims = [Simulation(p, prof) for p, prof, _, _ in members]
    for i, (sim, (_, _, v0, _)) in enumerate(zip(sims, members)):
        v = v0.copy()
        if i == 1:
            v[4, 5, 7, 9] = np.nan
        sim.upload(v)
    ens = E.Ensemble(sims)
    with pytest.raises(CssError) as ei:
        ens.step([m[3] for m in members], 1)
    assert ei.value.code == 4 and "member 1" in str(ei.value)


@pytest.mark.gpu
@pytest.mark.parametrize("spec", [SMALL[1], SMALL[2]])
def test_autotune_changes_no_result_bit(gpu_available, spec):
    from css_b200.context import Simulation
    p, prof, v0, dt = E.build_member(spec, seed=9)
    a = Simulation(p, prof)
    a.upload(v0)
    a.step_rk4(dt, 2)
    b = Simulation(p, prof)
    b.upload(v0)
    chosen = b.autotune(reps=2)
    assert all(t in (4, 8, 16) for t in chosen)
    assert np.array_equal(b.download(), v0)  # autotuning leaves the state alone
    b.step_rk4(dt, 2)
    assert np.array_equal(a.download(), b.download())


@pytest.mark.gpu
@pytest.mark.parametrize("spec", [SMALL[1], SMALL[2]])
def test_every_tile_variant_gives_the_same_bits(gpu_available, spec):
    from css_b200.context import Simulation
    p, prof, v0, dt = E.build_member(spec, seed=13)
    ref = Simulation(p, prof)
    ref.upload(v0)
    ref.step_rk4(dt, 2)
    want = ref.download()
    mt_phi = spec["nphi"] // spec["decomp"][2] in (16, 32)
    for tl in (8, 16):
        for pers in ((False, True) if mt_phi else (False,)):
            sim = Simulation(p, prof)
            sim.set_tiles(tl, tl, tl, pers)
            sim.upload(v0)
            sim.step_rk4(dt, 2)
            assert np.array_equal(sim.download(), want), (tl, pers)
            sim.close()


MIX = SMALL + [  # a member on 32^3 blocks (the two-pass stage for FP64)
    {"nr": 64, "nth": 64, "nphi": 96, "ra": 1e5, "ro": 0.8, "magnetic": True, "pm": 2.5, "decomp": (2, 2, 3)},
]


@pytest.mark.gpu
def test_ensemble_200_steps_fp64_and_mixed_against_each_member_alone(gpu_available):
    """200 steps of the ensemble, each member checked against its own
    unbatched FP64 run: the FP64 ensemble bit for bit, the mixed-precision
    ensemble (FP32 stage states) within the mixed form's bounds (rho and s
    1e-6, velocities and A 1e-3 of each field's size, tests/test_mixed.py)."""
    from css_b200.context import Simulation
    n = 200
    alone = []
    for i, spec in enumerate(MIX):
        p, prof, v0, dt = E.build_member(spec, seed=31 + i)
        sim = Simulation(p, prof)
        sim.upload(v0)
        sim.step_rk4(dt, n)
        alone.append(sim.download())
        sim.close()
    for precision in (0, 1):
        members = [E.build_member(spec, seed=31 + i, precision=precision) for i, spec in enumerate(MIX)]
        sims = [Simulation(p, prof) for p, prof, _, _ in members]
        for sim, (_, _, v0, _) in zip(sims, members):
            sim.upload(v0)
        ens = E.Ensemble(sims)
        ens.step([m[3] for m in members], n)
        for k, (sim, ref) in enumerate(zip(sims, alone)):
            got = sim.download()
            assert np.isfinite(got).all()
            if precision == 0:
                assert np.array_equal(got, ref), k
            else:
                for iv in range(got.shape[0]):
                    err = np.abs(got[iv] - ref[iv]).max() / np.abs(ref[iv]).max()
                    bar = 1e-6 if iv in (0, 4) else 1e-3
                    assert err < bar, (k, iv, err)
        ens.close()
        for sim in sims:
            sim.close()
