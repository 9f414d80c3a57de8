"""Mechanisms shared by the tests."""
import numpy as np

from micm_b200 import mechanism as mk
from micm_b200 import synthetic


def all_rate_types():
    """One reaction of every rate-constant kind micm's GPU path evaluates,
    plus a parameterized third body (air density) and a surface reaction."""
    m = mk.Mechanism(species=["A", "B", "C", "D", "E"], reactions=[], name="all_kinds",
                     parameterized=[(0.0, 0.0, 0.0, 1.0)],  # M = air density
                     absolute_tolerance=np.full(5, 1e-12))
    m.add(mk.arrhenius(A=1.2e-3, B=1.6, C=-250.0, D=290.0, E=1.0e-6), [0], [(1, 0.7), (2, 0.3)])
    m.add(mk.troe(k0_A=3.4e-4, k0_B=-2.1, k0_C=120.0, kinf_A=2.3e-2, kinf_B=-0.4, kinf_C=-35.0, Fc=0.55, N=1.1),
          [1, 2], [(3, 1.0)])
    m.add(mk.ternary(k0_A=1.3e-1, k0_B=-1.0, kinf_A=4.0e0, Fc=0.6, N=1.0), [2, 3], [(4, 1.0)])
    m.add(mk.branched(0, 3.1e-1, 120.0, 0.15, 6), [3], [(0, 1.0)])
    m.add(mk.branched(1, 2.7e-1, 90.0, 0.2, 4), [4], [(0, 0.5)])
    m.add(mk.tunneling(A=2.0e-2, B=500.0, C=3.0e7), [4], [(1, 1.0)])
    m.add(mk.taylor_series(A=3.0e-3, B=0.5, C=-100.0, coefficients=(1.0, 2.0e-3, -1.0e-6)), [0, 1], [(4, 1.0)])
    m.add(mk.reversible(A=1.0e-2, C=-300.0, k_r=0.7), [2], [(0, 1.0)])
    m.add(mk.user_defined("PHOTO.A", 2.5), [0], [(3, 1.0)])
    m.add(mk.surface("SURF.B", diffusion_coefficient=2.3e-5, molecular_weight=0.046, reaction_probability=0.2),
          [1], [(2, 1.0)])
    m.add(mk.arrhenius(A=2.0e-7, C=40.0), [0, -1], [(2, 1.0)])  # A + M -> C
    m.add(mk.arrhenius(A=5.0e-6), [3, 3], [(4, 1.0)])             # 2 D -> E
    return m


def all_rate_types_inputs(n, seed):
    m = all_rate_types()
    rng = np.random.default_rng(seed)
    T = rng.uniform(220.0, 320.0, n)
    P = rng.uniform(5.0e4, 1.05e5, n)
    rho = mk.ideal_air_density(P, T)
    y = rng.uniform(0.1, 5.0, size=(n, m.n_species))
    params = np.stack([rng.uniform(1e-4, 1e-2, n), rng.uniform(1e-7, 1e-6, n), rng.uniform(1e8, 1e9, n)], axis=1)
    return dict(temperature=T, pressure=P, air_density=rho, concentrations=y, custom_params=params)


def mechanism_set():
    return {
        "readme": synthetic.readme_mechanism(),
        "abc": synthetic.abc_mechanism(),
        "all_kinds": all_rate_types(),
        "syn60": synthetic.synthetic_mechanism(60, 120, seed=601),
        "syn210": synthetic.synthetic_mechanism(210, 440, seed=2101),
    }
