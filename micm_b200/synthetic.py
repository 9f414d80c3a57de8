"""Seeded synthetic mechanisms and grid-cell inputs for the benchmark configurations.

The reference ships no mechanism of the benchmark's shape, so mechanisms are
generated here.  The generator keeps the structure of real gas-phase
chemistry that makes Markowitz ordering effective (TS1,
test/benchmark/ts1_mechanism.hpp, has 209 species and 2381 LU nonzeros): a
small set of *hub* species (oxidants and radicals, 5% of the species) that
react with almost everything -- partners drawn from a Zipf law, so a few
oxidants dominate as OH, O3 and NO3 do -- and *organic* species that degrade
into nearby downstream organics and hubs.  Products of an organic lie downstream of it, so the
organic block of the Jacobian is triangular and LU fill stays confined to the
hub rows and columns.  Hub yields per reaction are at most one hub, so no
reaction cycle can amplify, and the system never explodes.

Reaction mix (fractions of the reaction count):
  60% bimolecular Arrhenius, log10 A[cm3 molec-1 s-1] ~ U(-16,-10), converted
      to micm units (m3 mol-1 s-1) with N_A, C ~ U(-2000, 500) K;
  25% unimolecular Arrhenius, log10 A[s-1] ~ U(-6,-1), C ~ U(-2000, 500) K;
  10% Troe fall-off, k0_A log-uniform 1e-33..1e-29 cm6 molec-2 s-1,
      kinf_A log-uniform 1e-12..1e-10 cm3 molec-1 s-1, Fc = 0.6;
   5% photolysis, user-defined rates with base values log-uniform 1e-6..1e-2 s-1;
1-3 products per reaction with yields ~ U(0.1, 1.0).
"""
from __future__ import annotations

from typing import Dict, Optional

import numpy as np

from .mechanism import (AVOGADRO_CONSTANT, Mechanism, arrhenius, ideal_air_density,
                        troe, user_defined)

CM3_MOLEC = 1e-6 * AVOGADRO_CONSTANT          # cm3 molec-1 s-1 -> m3 mol-1 s-1
CM6_MOLEC2 = CM3_MOLEC * CM3_MOLEC            # cm6 molec-2 s-1 -> m6 mol-2 s-1


def readme_mechanism() -> Mechanism:
    """README.md:95-135: Foo -> 0.8 Bar + 0.2 Baz (A=1e-3); Foo + Bar -> Baz (A=1e-5, C=110)."""
    m = Mechanism(species=["Foo", "Bar", "Baz"], reactions=[], name="readme")
    m.add(arrhenius(A=1.0e-3), [0], [(1, 0.8), (2, 0.2)])
    m.add(arrhenius(A=1.0e-5, C=110.0), [0, 1], [(2, 1.0)])
    return m


def abc_mechanism(rate1=None, rate2=None) -> Mechanism:
    """A -k1-> B -k2-> C (test/integration/analytical_policy.hpp:138-276)."""
    m = Mechanism(species=["A", "B", "C"], reactions=[], name="abc")
    m.add(rate1 or arrhenius(A=4.0e-3, C=50.0), [0], [(1, 1.0)])
    m.add(rate2 or arrhenius(A=1.2e-4, B=2.5, C=75.0, D=50.0, E=0.5), [1], [(2, 1.0)])
    return m


def synthetic_mechanism(n_species: int, n_reactions: int, seed: int,
                        atol: float = 1e-12, hub_fraction: float = 0.05,
                        window: int = 8, hub_skew: float = 1.5) -> Mechanism:
    """Seeded gas-phase mechanism (see module docstring).

    The defaults are calibrated to micm's TS1 benchmark mechanism
    (test/benchmark/ts1_mechanism.hpp: 209 species, 2381 LU-filled nonzeros,
    6986 LU updates, 1244 multipliers): at 210 species / 440 reactions they
    give 2596 nonzeros, 7992 updates and 1155 multipliers."""
    rng = np.random.default_rng(seed)
    S, R = int(n_species), int(n_reactions)
    H = max(3, int(round(S * hub_fraction)))
    organics = np.arange(H, S)
    names = [f"H{i:03d}" if i < H else f"O{i:04d}" for i in range(S)]
    m = Mechanism(species=names, reactions=[], name=f"synthetic_{S}_{R}_{seed}",
                  absolute_tolerance=np.full(S, atol))

    n_bi = int(round(0.60 * R))
    n_uni = int(round(0.25 * R))
    n_troe = int(round(0.10 * R))
    n_photo = R - n_bi - n_uni - n_troe
    kinds = ["bi"] * n_bi + ["uni"] * n_uni + ["troe"] * n_troe + ["photo"] * n_photo
    kinds = list(rng.permutation(np.array(kinds)))

    # every organic gets at least one loss reaction: the first len(organics)
    # loss-capable reactions take organics as primary reactant, in order
    loss_capable = [i for i, k in enumerate(kinds) if k in ("bi", "uni", "photo")]
    primary = {}
    for j, o in enumerate(organics):
        if j < len(loss_capable):
            primary[loss_capable[j]] = int(o)

    # hub partners follow a Zipf law (weight 1/(rank+1)^hub_skew): as in real
    # mechanisms, a few oxidants (OH, O3, NO3, ...) take most of the reactions
    hub_w = 1.0 / np.arange(1, H + 1) ** hub_skew
    hub_w /= hub_w.sum()

    def hub() -> int:
        return int(rng.choice(H, p=hub_w))

    def downstream(x: int) -> int:
        lo = x + 1
        hi = min(S - 1, x + window)
        if lo > hi:
            return int(rng.integers(H, S))
        return int(rng.integers(lo, hi + 1))

    def products_for(reactants):
        n_prod = int(rng.integers(1, 4))
        orgs = [x for x in reactants if x >= H]
        prods = []
        used_hub = False
        for _ in range(n_prod):
            if (not used_hub) and (rng.random() < 0.3 or not orgs and rng.random() < 0.5):
                h = hub()
                used_hub = True
                prods.append(h)
            elif orgs:
                prods.append(downstream(max(orgs)))
            else:
                prods.append(int(rng.integers(H, min(S, H + window))))
        # merge duplicates (micm accepts them, but distinct species are more realistic)
        out = []
        for s in prods:
            if s not in [p for p, _ in out]:
                out.append((s, float(rng.uniform(0.1, 1.0))))
        return out

    photo_i = 0
    for i, kind in enumerate(kinds):
        if kind == "bi":
            if i in primary:
                reactants = [primary[i], hub()]
            elif rng.random() < 0.85:
                reactants = [int(rng.choice(organics)), hub()]
            else:
                reactants = [hub(), hub()]
            A = 10.0 ** rng.uniform(-16, -10) * CM3_MOLEC
            C = rng.uniform(-2000.0, 500.0)
            rate = arrhenius(A=A, C=C)
        elif kind == "uni":
            if i in primary:
                reactants = [primary[i]]
            elif rng.random() < 0.9:
                reactants = [int(rng.choice(organics))]
            else:
                reactants = [hub()]
            A = 10.0 ** rng.uniform(-6, -1)
            C = rng.uniform(-2000.0, 500.0)
            rate = arrhenius(A=A, C=C)
        elif kind == "troe":
            if rng.random() < 0.5:
                reactants = [hub(), hub()]
            else:
                reactants = [int(rng.choice(organics)), hub()]
            k0 = 10.0 ** rng.uniform(-33, -29) * CM6_MOLEC2
            kinf = 10.0 ** rng.uniform(-12, -10) * CM3_MOLEC
            rate = troe(k0_A=k0, k0_B=float(rng.uniform(-4.0, 0.0)), kinf_A=kinf,
                        kinf_B=float(rng.uniform(-1.0, 0.0)), Fc=0.6, N=1.0)
        else:  # photolysis
            if i in primary:
                reactants = [primary[i]]
            elif rng.random() < 0.7:
                reactants = [int(rng.choice(organics))]
            else:
                reactants = [hub()]
            rate = user_defined(f"PHOTO.j{photo_i:03d}", 1.0)
            photo_i += 1
        m.add(rate, reactants, products_for(reactants))
    # photolysis base rates, one per user-defined reaction, in input order
    m.photolysis_base = 10.0 ** rng.uniform(-6, -2, size=photo_i)
    return m


def cell_inputs(mech: Mechanism, n_cells: int, seed: int, t_range=(270.0, 310.0),
                p_range=(9.0e4, 1.02e5), log10_conc=(-14.0, -6.0), night_fraction=0.0,
                readme_foo: Optional[tuple] = None) -> Dict[str, np.ndarray]:
    """Per-cell seeded inputs in *system species order* (not state columns).

    Returns temperature, pressure, air_density [n], concentrations [n, S] and
    custom parameters [n, P] keyed by label order of ``mech.custom_param_labels()``.
    """
    rng = np.random.default_rng(seed)
    T = rng.uniform(*t_range, size=n_cells)
    P = rng.uniform(*p_range, size=n_cells)
    rho = ideal_air_density(P, T)
    S = mech.n_species
    if readme_foo is not None:
        y = np.zeros((n_cells, S))
        y[:, 0] = rng.uniform(*readme_foo, size=n_cells)
    else:
        y = 10.0 ** rng.uniform(*log10_conc, size=(n_cells, S))
    labels = mech.custom_param_labels()
    params = np.zeros((n_cells, len(labels)))
    base = getattr(mech, "photolysis_base", None)
    if base is not None and len(labels):
        # label order == sorted reaction order == input order of UD reactions here
        day = rng.uniform(0.5, 1.0, size=n_cells)
        night = rng.random(n_cells) < night_fraction
        day[night] = 0.0
        params[:, : len(base)] = day[:, None] * base[None, :]
    return dict(temperature=T, pressure=P, air_density=rho, concentrations=y,
                custom_params=params)


# Benchmark configurations (shapes of the benchmark suite; seeds recorded here).
CONFIGS = {
    "readme": dict(mech=lambda: readme_mechanism(), cells=1024, stages=3, dt=500.0,
                   solves=10, seed=11, inputs=dict(readme_foo=(1.0, 30.0))),
    "c210": dict(mech=lambda: synthetic_mechanism(210, 440, seed=2101), cells=16384,
                 stages=4, dt=600.0, solves=1, seed=2102, inputs={}),
    "c210_uneven": dict(mech=lambda: synthetic_mechanism(210, 440, seed=2101),
                        cells=1048576, stages=4, dt=600.0, solves=1, seed=2103,
                        inputs=dict(t_range=(200.0, 310.0), night_fraction=0.5)),
    "c60_adjoint": dict(mech=lambda: synthetic_mechanism(60, 120, seed=601), cells=131072,
                        stages=4, dt=3600.0, solves=1, seed=602, inputs={}),
    "c600": dict(mech=lambda: synthetic_mechanism(600, 1500, seed=6001), cells=262144,
                 stages=4, dt=600.0, solves=1, seed=6002, inputs={}),
}
