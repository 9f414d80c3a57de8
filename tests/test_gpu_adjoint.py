"""GPU discrete adjoint (micmb_solve_adjoint) against the FP64 CPU adjoint
oracle and against central finite differences of the fixed-step replay."""
import numpy as np
import pytest
import torch

import oracle
from micm_b200 import Solver, synthetic
from micm_b200.autograd import RosenbrockSolve

from gpu_helpers import make_state

pytestmark = pytest.mark.gpu


def _setup(mech_name, n, seed, fused_config=None):
    cfg = synthetic.CONFIGS[mech_name]
    mech = cfg["mech"]()
    inputs = synthetic.cell_inputs(mech, n, seed, **cfg["inputs"])
    solver = Solver(mech, cfg["stages"], vector_length=32)
    if fused_config:
        solver.set_fused_config(**fused_config)
    st = make_state(solver, inputs)
    solver.update_state_parameters(st)
    return cfg, mech, inputs, solver, st


def _significant(g, scale):
    return np.abs(g) > 1e-6 * scale


@pytest.mark.parametrize("name,n,config", [("c60_adjoint", 96, None),
                                           ("c60_adjoint", 64, dict(variant=1)),
                                           ("c60_adjoint", 64, dict(variant=2)),
                                           ("c210", 8, None),
                                           ("c600", 6, None)])
def test_adjoint_matches_oracle(cuda_device, name, n, config):
    cfg, mech, inputs, solver, st = _setup(name, n, 41, config)
    k = np.ascontiguousarray(st.rate_constants())        # the GPU's own rate constants
    rng = np.random.default_rng(5)
    ybar_sys = rng.normal(size=(n, mech.n_species)) * (rng.random((n, mech.n_species)) < 0.3)
    cols = solver.compiled.species_columns
    ybar_cols = np.zeros_like(ybar_sys)
    ybar_cols[:, cols] = ybar_sys
    g0_cols, gk, res = solver.solve_adjoint(cfg["dt"], st, ybar_cols, max_checkpoints=400)
    assert res.converged
    g0 = g0_cols[:, cols]
    R = oracle.Restatement(mech, tableau_kind=cfg["stages"])
    y_final, g0_ref, gk_ref = R.adjoint_per_cell(inputs, cfg["dt"], ybar_sys, k=k, max_steps=400)
    st.sync_outputs_to_host()
    np.testing.assert_allclose(st.concentrations(), y_final, rtol=1e-9, atol=1e-24)
    # per-cell initial-state gradients
    scale = np.abs(g0_ref).max(axis=1, keepdims=True)
    sig = _significant(g0_ref, scale)
    rel = np.abs(g0 - g0_ref)[sig] / np.abs(g0_ref)[sig]
    assert rel.max() < 1e-8
    assert np.all(np.abs(g0 - g0_ref) <= 1e-6 * scale + 1e-300)
    # rate-parameter gradients summed over cells
    gk_ref_sum = gk_ref.sum(axis=0)
    ks = np.abs(gk_ref_sum).max()
    np.testing.assert_allclose(gk, gk_ref_sum, rtol=1e-8, atol=1e-9 * ks)


@pytest.mark.parametrize("config", [None, dict(variant=2)])
def test_adjoint_chunks_and_recomputed_stages_change_nothing(cuda_device, config):
    """A memory limit that splits the cells into 32-cell chunks, with the
    stages recomputed in the sweep instead of stored, gives the same bits."""
    cfg, mech, inputs, solver, st = _setup("c60_adjoint", 100, 43, config)
    rng = np.random.default_rng(9)
    ybar = rng.normal(size=(100, mech.n_species))
    g0_a, gk_a, res_a = solver.solve_adjoint(cfg["dt"], st, ybar, max_checkpoints=300)
    st.sync_outputs_to_host()
    y_a = st.concentrations().copy()
    per_cell_y = 300 * (mech.n_species + 1) * 8
    solver.set_adjoint_memory_limit(32 * per_cell_y + 100)
    st.set_concentrations(inputs["concentrations"])
    st.sync_inputs_to_device()
    g0_b, gk_b, res_b = solver.solve_adjoint(cfg["dt"], st, ybar, max_checkpoints=300)
    st.sync_outputs_to_host()
    np.testing.assert_array_equal(st.concentrations(), y_a)
    np.testing.assert_array_equal(g0_b, g0_a)
    np.testing.assert_array_equal(gk_b, gk_a)
    assert res_b.stats["accepted"] == res_a.stats["accepted"]
    assert res_b.stats["number_of_steps"] == res_a.stats["number_of_steps"]


def test_adjoint_memory_limit_below_one_group(cuda_device):
    from micm_b200._native import MicmbError
    cfg, mech, inputs, solver, st = _setup("c60_adjoint", 40, 44)
    solver.set_adjoint_memory_limit(1000)
    with pytest.raises(MicmbError):
        solver.solve_adjoint(cfg["dt"], st, np.ones((40, mech.n_species)), max_checkpoints=300)
    solver.set_adjoint_memory_limit(0)
    st.set_concentrations(inputs["concentrations"])
    st.sync_inputs_to_device()
    _, _, res = solver.solve_adjoint(cfg["dt"], st, np.ones((40, mech.n_species)), max_checkpoints=300)
    assert res.converged


def test_adjoint_matches_finite_differences(cuda_device):
    cfg, mech, inputs, solver, st = _setup("c60_adjoint", 4, 7)
    k = np.ascontiguousarray(st.rate_constants())
    cols = solver.compiled.species_columns
    ybar_cols = np.zeros((4, mech.n_species))
    ybar_cols[:, cols[0]] = 1.0
    g0_cols, gk, _ = solver.solve_adjoint(cfg["dt"], st, ybar_cols, max_checkpoints=400)
    g0 = g0_cols[:, cols]
    R = oracle.Restatement(mech, tableau_kind=cfg["stages"])
    h, steps = R.step_sizes_per_cell(inputs, cfg["dt"], 400, k)
    y0 = inputs["concentrations"]

    def out(y, kk=k):
        return R.replay_per_cell(y, kk, h, steps)[:, 0]

    rel_h = 1e-6
    imp = np.abs(g0) * np.abs(y0)
    worst = 0.0
    for j in range(mech.n_species):
        e = rel_h * np.abs(y0[:, j])
        yp, ym = y0.copy(), y0.copy()
        yp[:, j] += e
        ym[:, j] -= e
        fd = (out(yp) - out(ym)) / (2 * e)
        sig = imp[:, j] > 1e-3 * imp.max(axis=1)
        if sig.any():
            worst = max(worst, (np.abs(fd - g0[:, j]) / np.abs(g0[:, j]))[sig].max())
    assert worst < 1e-5
    # summed log-k gradient against the finite difference of the summed output
    kimp = np.abs(gk)
    for r in np.argsort(-kimp)[:12]:
        c = R.reaction_columns[r]
        kp, km = k.copy(), k.copy()
        kp[:, c] *= np.exp(rel_h)
        km[:, c] *= np.exp(-rel_h)
        fd = (out(y0, kp).sum() - out(y0, km).sum()) / (2 * rel_h)
        assert abs(fd - gk[r]) <= 1e-5 * abs(gk[r])


def test_autograd_function(cuda_device):
    cfg, mech, inputs, solver, st = _setup("c60_adjoint", 16, 3)
    y0 = torch.tensor(inputs["concentrations"], dtype=torch.float64, device="cuda", requires_grad=True)
    logs = torch.zeros(mech.n_reactions, dtype=torch.float64, device="cuda", requires_grad=True)
    target = torch.rand(16, dtype=torch.float64, device="cuda") * 1e-9
    y = RosenbrockSolve.apply(y0, logs, solver, st, cfg["dt"])
    loss = ((y[:, 0] - target) ** 2).sum()
    loss.backward()
    # same gradient through the C ABI directly
    cols = solver.compiled.species_columns
    g = np.zeros((16, mech.n_species))
    g[:, cols[0]] = 2 * (y[:, 0] - target).detach().cpu().numpy()
    st.set_concentrations(inputs["concentrations"])
    st.sync_inputs_to_device()
    g0_cols, gk, _ = solver.solve_adjoint(cfg["dt"], st, g)
    np.testing.assert_array_equal(y0.grad.cpu().numpy(), g0_cols[:, cols])
    np.testing.assert_array_equal(logs.grad.cpu().numpy(), gk)


def test_adjoint_configuration_spot_check(cuda_device):
    """The adjoint configuration (60 species, 120 reactions, dt = 3600 s) at
    8,192 cells: the GPU's dL/dy0 on a seeded sample of 64 cells, and the
    per-cell rate-parameter gradients of those cells (through a loss that
    touches only them), against the FP64 CPU adjoint oracle."""
    n, n_check = 8192, 64
    cfg, mech, inputs, solver, st = _setup("c60_adjoint", n, 43)
    k = np.ascontiguousarray(st.rate_constants())
    rng = np.random.default_rng(9)
    pick = np.sort(rng.choice(n, n_check, replace=False))
    cols = solver.compiled.species_columns
    ybar_sys = np.zeros((n, mech.n_species))
    ybar_sys[pick] = rng.normal(size=(n_check, mech.n_species))
    ybar_cols = np.zeros_like(ybar_sys)
    ybar_cols[:, cols] = ybar_sys
    g0_cols, gk, res = solver.solve_adjoint(cfg["dt"], st, ybar_cols, max_checkpoints=400)
    assert res.converged
    g0 = g0_cols[:, cols]
    sub = {key: v[pick] for key, v in inputs.items()}
    R = oracle.Restatement(mech, tableau_kind=cfg["stages"])
    _, g0_ref, gk_ref = R.adjoint_per_cell(sub, cfg["dt"], ybar_sys[pick], k=k[pick], max_steps=400)
    scale = np.abs(g0_ref).max(axis=1, keepdims=True)
    sig = _significant(g0_ref, scale)
    assert (np.abs(g0[pick] - g0_ref)[sig] / np.abs(g0_ref)[sig]).max() < 1e-8
    assert np.all(g0[np.setdiff1d(np.arange(n), pick)] == 0.0)
    gk_ref_sum = gk_ref.sum(axis=0)
    np.testing.assert_allclose(gk, gk_ref_sum, rtol=1e-8, atol=1e-9 * np.abs(gk_ref_sum).max())
