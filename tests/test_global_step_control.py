"""Global step control (micm's single step size for all cells,
include/micm/solver/rosenbrock.inl:12-304 with the NormalizedError of
:353-402) over one or several GPUs.

The error norm's sum over cells is formed in a fixed order that the GPU
reproduces: per cell in species order, a pairwise tree per 256-cell block, a
fixed reduction of the blocks per shard, and the shards' sums added in rank
order.  A job split over ranks exchanges one double per rank and attempt (an
all-gather), so every rank takes the same decisions.

CPU: the restatement's global solve follows micm's (identical statistics,
values to rounding); two gloo ranks, each solving its shard with the exchange,
equal the single-process solve of the same shards bit for bit.  GPU: the
library's plain global solve equals the restatement bit for bit, with and
without the exchange hook, and two ranks emulated by two host threads on one
GPU (each with its own state and stream; the exchange waits on the host, no
kernel waits on another) equal the two-shard restatement bit for bit."""
import ctypes
import os
import socket
import sys
import threading

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from micm_b200 import synthetic  # noqa: E402

pytestmark = pytest.mark.skipif(not oracle.restatement_available(), reason="oracle not built")
SHARDS = [300, 724]


def _case(n=1024):
    m = synthetic.synthetic_mechanism(60, 120, seed=601)
    return m, synthetic.cell_inputs(m, n, 5)


def _split(inp, sizes):
    out, start = [], 0
    for s in sizes:
        out.append({k: v[start:start + s] for k, v in inp.items()})
        start += s
    return out


@pytest.mark.skipif(not oracle.reference_available(), reason="oracle/_ref not built")
def test_restatement_follows_micms_global_solve():
    m, inp = _case(700)
    y, st = oracle.Restatement(m, 4).solve_global(inp, 600.0)
    y_micm, st_micm = oracle.Reference(m, tableau=4).solve_global(inp, 600.0)
    for q, key in enumerate(oracle.STATS_FIELDS[:7]):
        assert st[q] == st_micm[0][key], key
    np.testing.assert_allclose(y, y_micm, rtol=1e-10, atol=1e-30)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _dae_case():
    """two equilibrium constraints, inconsistent start: the constraint
    initialisation iterates, and its residual maximum crosses the ranks"""
    from dae_cases import equilibrium, equilibrium_inputs
    m = equilibrium(2.0, True)
    inp = equilibrium_inputs(m, 5, False, 0.2)
    inp["concentrations"][3:, 1] *= 3.0  # rank 1's cells start further from equilibrium
    return m, inp


def _dae_singular_case():
    """rank 1's cells start with the squared product at zero: dG/dF = 0, the
    initialisation's matrix is singular there, its update infinite, and the
    flag must reach rank 0 through the exchange (micm: InfDetected)"""
    from dae_cases import equilibrium, equilibrium_inputs
    m = equilibrium(2.0, True)
    inp = equilibrium_inputs(m, 4, False, 0.2)
    inp["concentrations"][2:, 5] = 0.0
    return m, inp


# kind: (case, shard sizes, tableau, dt)
KINDS = {"kinetic": (_case, SHARDS, 4, 600.0), "dae": (_dae_case, [2, 3], 40, 10.0),
         "dae_singular": (_dae_singular_case, [2, 2], 40, 10.0)}


def _rank_main(rank, world, port, out_path, kind="kinetic"):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        make_case, shards, tableau, dt = KINDS[kind]
        m, inp = make_case()
        mine = _split(inp, shards)[rank]

        def exchange(value, op):
            gathered = [torch.zeros(1, dtype=torch.float64) for _ in range(world)]
            dist.all_gather(gathered, torch.tensor([value], dtype=torch.float64))
            if op == oracle.EXCHANGE_MAX:
                return oracle.max_combine(g.item() for g in gathered)
            total = 0.0
            for g in gathered:  # rank order
                total += g.item()
            return total

        y, st = oracle.Restatement(m, tableau).solve_global(mine, dt, exchange=exchange, total_cells=sum(shards))
        np.savez(f"{out_path}.{rank}.npz", y=y, stats=st)
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("kind", ["kinetic", "dae", "dae_singular"])
def test_two_gloo_ranks_equal_the_single_process_solve(tmp_path, kind):
    out = str(tmp_path / "rank")
    mp.start_processes(_rank_main, args=(2, _free_port(), out, kind), nprocs=2, start_method="spawn")
    r0, r1 = (np.load(f"{out}.{r}.npz") for r in range(2))
    make_case, shards, tableau, dt = KINDS[kind]
    m, inp = make_case()
    y, st = oracle.Restatement(m, tableau).solve_global(inp, dt, shards=shards)
    if kind == "dae":
        assert st[9] >= 2 and st[7] == 2  # the initialisation iterated, and the solve converged
    if kind == "dae_singular":
        assert st[7] == 7  # InfDetected on both ranks, though only rank 1's cells are singular
    np.testing.assert_array_equal(np.concatenate([r0["y"], r1["y"]]), y)
    np.testing.assert_array_equal(r0["stats"], st)
    np.testing.assert_array_equal(r1["stats"], st)


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------
def _gpu_state(solver, inp, k):
    from gpu_helpers import make_state, upload_cols
    from micm_b200 import solver as sv
    st = make_state(solver, inp)
    upload_cols(st, sv.BUF_RATE_CONSTANTS, k)
    return st


class _DeviceArray:
    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def _dev(ptr, n):
    """torch view of n doubles at a device address"""
    return torch.as_tensor(_DeviceArray(ptr, n), device="cuda")


def _stats_equal(res, st):
    for q, key in enumerate(oracle.STATS_FIELDS[:7]):
        assert res.stats[key] == st[q], key
    assert res.state == st[7]


@pytest.mark.gpu
@pytest.mark.parametrize("L", [1, 32, 128])
def test_gpu_global_equals_restatement(cuda_device, L):
    from micm_b200 import Solver
    m, inp = _case()
    R = oracle.Restatement(m, 4, correctly_rounded=True)
    k = R._k(inp)
    y_ref, st_ref = R.solve_global(inp, 600.0, k=k)
    solver = Solver(m, 4, vector_length=L)
    st = _gpu_state(solver, inp, k)
    res = solver.solve(600.0, st, method="plain", step_control="global")
    st.sync_outputs_to_host()
    np.testing.assert_array_equal(st.concentrations(), y_ref)
    _stats_equal(res, st_ref)


@pytest.mark.gpu
def test_gpu_exchange_hook_with_one_rank_changes_nothing(cuda_device):
    from micm_b200 import Solver
    m, inp = _case()
    R = oracle.Restatement(m, 4, correctly_rounded=True)
    k = R._k(inp)
    y_ref, st_ref = R.solve_global(inp, 600.0, k=k)
    solver = Solver(m, 4, vector_length=32)
    st = _gpu_state(solver, inp, k)
    calls = []

    def identity(send, recv, world, stream):
        calls.append(world)
        with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
            _dev(recv, 1).copy_(_dev(send, 1))
        return 0
    st.set_global_exchange(identity, 1, len(inp["temperature"]))
    res = solver.solve(600.0, st, method="plain", step_control="global")
    st.sync_outputs_to_host()
    np.testing.assert_array_equal(st.concentrations(), y_ref)
    _stats_equal(res, st_ref)
    assert len(calls) >= res.stats["number_of_steps"]


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["kinetic", "dae"])
def test_gpu_two_ranks_on_host_threads_equal_two_shard_restatement(cuda_device, kind):
    """Two ranks as two host threads, each with its own state and stream on one
    GPU.  The exchange reads this rank's value on the host (after its stream is
    done), meets the other rank at a host barrier with a timeout, and writes
    both values back; no kernel ever waits on another rank's kernel.  "dae":
    the constraint initialisation's residual maxima and flags cross the ranks
    through the same hook."""
    from micm_b200 import Solver
    from micm_b200._native import check, lib
    from gpu_helpers import make_state
    make_case, shards, tableau, dt = KINDS[kind]
    m, inp = make_case()
    R = oracle.Restatement(m, tableau, correctly_rounded=True)
    k = R._k(inp)
    y_ref, st_ref = R.solve_global(inp, dt, k=k, shards=shards)
    solver = Solver(m, tableau, vector_length=32)
    parts = _split(inp, shards)
    if kind == "dae":
        states = [make_state(solver, p) for p in parts]
        for st in states:
            solver.update_state_parameters(st)
    else:
        kparts = np.split(k, np.cumsum(shards)[:-1])
        states = [_gpu_state(solver, p, kp) for p, kp in zip(parts, kparts)]
    streams = [torch.cuda.Stream() for _ in range(2)]
    for st, s in zip(states, streams):
        check(lib().micmb_state_set_stream(st.handle, ctypes.c_void_p(s.cuda_stream)))
    barrier = threading.Barrier(2, timeout=60)
    slots = [0.0, 0.0]
    results, errors = [None, None], []

    def make_exchange(rank):
        def exchange(send, recv, world, stream):
            streams[rank].synchronize()
            slots[rank] = float(_dev(send, 1).cpu().item())
            barrier.wait()
            both = torch.tensor(slots, dtype=torch.float64)
            barrier.wait()
            with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
                _dev(recv, 2).copy_(both)
            return 0
        return exchange

    def run(rank):
        try:
            torch.cuda.set_device(0)
            states[rank].set_global_exchange(make_exchange(rank), 2, sum(shards))
            results[rank] = solver.solve(dt, states[rank], method="plain", step_control="global")
        except Exception as e:  # reported below
            errors.append(e)
            barrier.abort()

    threads = [threading.Thread(target=run, args=(r,)) for r in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=600)
    assert not errors, errors
    y = []
    for st in states:
        st.sync_outputs_to_host()
        y.append(st.concentrations())
    np.testing.assert_array_equal(np.concatenate(y), y_ref)
    for res in results:
        _stats_equal(res, st_ref)
        assert res.stats["constraint_init_iterations"] == st_ref[9]


def test_max_combine_keeps_micms_order_of_checks():
    """The encoded residual maxima of the constraint initialisation combine
    with NaN first, then +Inf, else the largest: micm checks NaN before Inf
    (rosenbrock.inl:505-512, 564-571), so any rank's NaN wins."""
    nan, inf = float("nan"), float("inf")
    assert oracle.max_combine([1e-3, 2e-3]) == 2e-3
    assert oracle.max_combine([0.0, 0.0]) == 0.0
    assert oracle.max_combine([inf, 1.0]) == inf
    assert np.isnan(oracle.max_combine([inf, nan]))
    assert np.isnan(oracle.max_combine([nan, 1.0]))
    assert np.isnan(oracle.max_combine([1.0, inf, nan]))
