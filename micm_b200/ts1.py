"""micm's TS1 benchmark mechanism (MOZART-TS1: 209 state species, 547
reactions) and micm_bench's initial state for it; the TS1 entries of
micm_b200.micm_bench (test/benchmark/ts1_mechanism.hpp)."""
from __future__ import annotations

from typing import Dict, Optional

import numpy as np

from . import micm_bench
from .mechanism import Mechanism

FIXTURE = micm_bench.fixture("ts1")
TABLEAU = micm_bench.TABLEAU
DT = micm_bench.DT


def mechanism(path: Optional[str] = None, absolute_tolerance: Optional[float] = None) -> Mechanism:
    """TS1 as micm builds it (absolute tolerance: micm's builder default, 1e-3, unless given)."""
    return micm_bench.mechanism("ts1", path, absolute_tolerance)


def inputs(n_cells: int, seed: Optional[int] = None, path: Optional[str] = None) -> Dict[str, np.ndarray]:
    """micm_bench's TS1 initial state on every cell (T = 287.45 K, P = 101319.9 Pa), varied per cell with a seed."""
    return micm_bench.inputs("ts1", n_cells, seed, path)


def micm_columns(path: Optional[str] = None) -> Dict[str, Dict[str, int]]:
    return micm_bench.micm_columns("ts1", path)
