"""The mechanisms and initial states of micm's own benchmark program
(test/benchmark/micm_bench.cpp): TS1 (MOZART-TS1: 209 state species, 547
reactions -- Arrhenius, Troe, user-defined photolysis and surface reactions
with a third body M; test/benchmark/ts1_mechanism.hpp) and Chapman (9
species, 7 reactions; test/benchmark/chapman_mechanism.hpp).  micm_bench
solves them with ThreeStageRosenbrockParameters and dt = 30 s by default.

Each mechanism and its initial state are read from
tests/golden/<name>_mechanism.json, which tests/golden/make_micm_bench.py
writes from micm itself (micm builds the mechanism from the benchmark's code
and the program prints it in this repository's JSON description; see
micm_b200.mechanism.mechanism_from_dict).
"""
from __future__ import annotations

import json
import os
from typing import Dict, Optional

import numpy as np

from .mechanism import Mechanism, ideal_air_density, mechanism_from_dict

GOLDEN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "golden")
NAMES = ("ts1", "chapman")
TABLEAU = 3          # micm_bench: RosenbrockSolverParameters::ThreeStageRosenbrockParameters()
DT = 30.0            # micm_bench's default time step [s]


def fixture(name: str) -> str:
    if name not in NAMES:
        raise ValueError(f"unknown micm_bench mechanism '{name}' (one of {NAMES})")
    return os.path.join(GOLDEN, f"{name}_mechanism.json")


def document(name: str, path: Optional[str] = None) -> dict:
    with open(path or fixture(name)) as f:
        return json.load(f)


def mechanism(name: str, path: Optional[str] = None, absolute_tolerance: Optional[float] = None) -> Mechanism:
    """The mechanism as micm builds it.  The absolute tolerance is micm's
    builder default (1e-3, what micm_bench runs with) unless one is given for
    every species."""
    m = mechanism_from_dict(document(name, path))
    if absolute_tolerance is not None:
        m.absolute_tolerance = np.full(m.n_species, float(absolute_tolerance))
    return m


def inputs(name: str, n_cells: int, seed: Optional[int] = None, path: Optional[str] = None) -> Dict[str, np.ndarray]:
    """micm_bench's initial state on every cell (its temperature, pressure and
    air density -- Chapman's InitState leaves the air density at 0 --, its
    concentrations and photolysis / aerosol parameters).  With a seed, each
    cell is varied: concentrations scaled by 10**U(-0.5, 0.5), T shifted by
    U(-30, 10) K (air density recomputed) and photolysis rates scaled by
    U(0, 1)."""
    doc = document(name, path)
    mech = mechanism_from_dict(doc)
    init = doc["init"]
    y = np.array([init["concentrations"][s] for s in mech.species], dtype=np.float64)
    labels = mech.custom_param_labels()
    p = np.array([init["custom_parameters"][l] for l in labels], dtype=np.float64)
    n = int(n_cells)
    T = np.full(n, float(init["temperature"]))
    P = np.full(n, float(init["pressure"]))
    rho = np.full(n, float(init["air_density"]))
    conc = np.tile(y, (n, 1))
    params = np.tile(p, (n, 1)).reshape(n, len(labels))
    if seed is not None:
        rng = np.random.default_rng(seed)
        conc *= 10.0 ** rng.uniform(-0.5, 0.5, size=conc.shape)
        T += rng.uniform(-30.0, 10.0, size=n)
        rho = ideal_air_density(P, T)
        photolysis = np.array([l.startswith("j") for l in labels], dtype=bool)
        params[:, photolysis] *= rng.uniform(0.0, 1.0, size=(n, int(photolysis.sum())))
    return dict(temperature=T, pressure=P, air_density=rho, concentrations=conc, custom_params=params)


def micm_columns(name: str, path: Optional[str] = None) -> Dict[str, Dict[str, int]]:
    """micm's own state columns for every species and custom parameter."""
    return document(name, path)["micm_columns"]


def golden(name: str):
    """micm's results on the fixture's 4-cell state (tests/golden/<name>_micm.npz)."""
    return np.load(os.path.join(GOLDEN, f"{name}_micm.npz"))
