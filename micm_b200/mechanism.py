"""Mechanism description in micm's vocabulary, flattened for the C ABI.

A :class:`Mechanism` is what micm builds from ``System`` + ``std::vector<Process>``
(include/micm/system/system.hpp, include/micm/process/chemical_reaction_builder.hpp):
species in gas-phase order, reactions with a rate-constant kind and its
parameters, reactants (possibly parameterized, e.g. a third body M) and
products with yields.  :meth:`Mechanism.flat` turns it into the arrays of
``micmb_mechanism_desc`` (include/micmb.h).

Rate-constant kinds use micm's sort key (solver_builder.inl:274-329) so the
column order of ``rate_constants`` matches the reference solver.
"""
from __future__ import annotations

import dataclasses
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

ARRHENIUS = 0
TROE = 1
TERNARY_CHEMICAL_ACTIVATION = 2
BRANCHED = 3
TUNNELING = 4
TAYLOR_SERIES = 5
REVERSIBLE = 6
USER_DEFINED = 7
SURFACE = 8

RATE_PARAM_STRIDE = 24

# micm::constants (include/micm/util/constants.hpp)
BOLTZMANN_CONSTANT = 1.380649e-23
AVOGADRO_CONSTANT = 6.02214076e23
GAS_CONSTANT = BOLTZMANN_CONSTANT * AVOGADRO_CONSTANT


def arrhenius(A=1.0, B=0.0, C=0.0, D=300.0, E=0.0):
    """ArrheniusRateConstantParameters (arrhenius_rate_constant.hpp:9-22)."""
    return (ARRHENIUS, [A, B, C, D, E])


def troe(k0_A=1.0, k0_B=0.0, k0_C=0.0, kinf_A=1.0, kinf_B=0.0, kinf_C=0.0, Fc=0.6, N=1.0):
    """TroeRateConstantParameters (troe_rate_constant.hpp)."""
    return (TROE, [k0_A, k0_B, k0_C, kinf_A, kinf_B, kinf_C, Fc, N])


def ternary(k0_A=1.0, k0_B=0.0, k0_C=0.0, kinf_A=1.0, kinf_B=0.0, kinf_C=0.0, Fc=0.6, N=1.0):
    """TernaryChemicalActivationRateConstantParameters."""
    return (TERNARY_CHEMICAL_ACTIVATION, [k0_A, k0_B, k0_C, kinf_A, kinf_B, kinf_C, Fc, N])


def branched(branch, X, Y, a0, n):
    """BranchedRateConstantParameters; branch 0 = alkoxy, 1 = nitrate."""
    return (BRANCHED, [float(branch), X, Y, a0, float(n)])


def tunneling(A=1.0, B=0.0, C=0.0):
    """TunnelingRateConstantParameters."""
    return (TUNNELING, [A, B, C])


def taylor_series(A=1.0, B=0.0, C=0.0, D=300.0, E=0.0, coefficients=(1.0,)):
    """TaylorSeriesRateConstantParameters (up to 16 coefficients)."""
    coefficients = list(coefficients)
    if not 1 <= len(coefficients) <= 16:
        raise ValueError("TaylorSeries takes 1..16 coefficients")
    return (TAYLOR_SERIES, [A, B, C, D, E, float(len(coefficients))] + coefficients)


def reversible(A=1.0, C=0.0, k_r=0.0):
    """ReversibleRateConstantParameters."""
    return (REVERSIBLE, [A, C, k_r])


def user_defined(label, scaling_factor=1.0):
    """UserDefinedRateConstantParameters: k = custom parameter * scaling."""
    return (USER_DEFINED, [scaling_factor], label)


def surface(label, diffusion_coefficient, molecular_weight, reaction_probability=1.0):
    """SurfaceRateConstantParameters; custom parameters
    ``label.effective radius [m]`` and ``label.particle number concentration [# m-3]``."""
    return (SURFACE, [diffusion_coefficient, molecular_weight, reaction_probability], label)


@dataclasses.dataclass
class Reaction:
    kind: int
    params: List[float]
    reactants: List[int]                   # >=0 species, -(p+1) parameterized p
    products: List[Tuple[int, float]]      # (species, yield)
    label: Optional[str] = None            # custom parameter label (UD / surface)


CONSTRAINT_LINEAR = 0
CONSTRAINT_EQUILIBRIUM = 1


@dataclasses.dataclass
class Constraint:
    """An algebraic constraint replacing the ODE row of `species`
    (include/micm/constraint/types/linear_constraint.hpp,
    equilibrium_constraint.hpp)."""
    kind: int
    species: int                              # algebraic species (system index)
    terms: List[Tuple[int, float]]            # (species, coefficient or stoichiometry)
    n_reactants: int = 0                      # equilibrium: leading reactant terms
    params: Tuple[float, float, float, float] = (0.0, 0.0, 0.0, 0.0)
    name: str = "constraint"


def linear_constraint(species: int, terms: Sequence[Tuple[int, float]], constant: float, name="linear"):
    """LinearConstraint: sum coef * [species] - constant = 0, replacing the row of `species`."""
    return Constraint(CONSTRAINT_LINEAR, species, [(int(a), float(c)) for a, c in terms], 0,
                      (float(constant), 0.0, 0.0, 0.0), name)


def equilibrium_constraint(species: int, reactants: Sequence[Tuple[int, float]], products: Sequence[Tuple[int, float]],
                           K_HLC_ref: float, delta_H: float = 0.0, R: float = GAS_CONSTANT, T_ref: float = 298.15,
                           name="equilibrium"):
    """EquilibriumConstraint: K_eq(T) prod [reactants]^a - prod [products]^b = 0 with the
    Van't Hoff K_eq(T) = K_HLC_ref exp((delta_H / R)(1/T - 1/T_ref)), replacing the row of `species`."""
    terms = [(int(a), float(c)) for a, c in reactants] + [(int(a), float(c)) for a, c in products]
    return Constraint(CONSTRAINT_EQUILIBRIUM, species, terms, len(reactants),
                      (float(K_HLC_ref), float(delta_H), float(R), float(T_ref)), name)


@dataclasses.dataclass
class Mechanism:
    species: List[str]
    reactions: List[Reaction]
    parameterized: List[Tuple[float, float, float, float]] = dataclasses.field(default_factory=list)
    absolute_tolerance: Optional[np.ndarray] = None   # per species, system order
    relative_tolerance: float = 1e-6
    reorder_state: bool = True
    name: str = "mechanism"
    constraints: List[Constraint] = dataclasses.field(default_factory=list)

    @property
    def n_species(self) -> int:
        return len(self.species)

    @property
    def n_reactions(self) -> int:
        return len(self.reactions)

    def add(self, rate, reactants: Sequence[int], products: Sequence[Tuple[int, float]]):
        kind, params = rate[0], list(rate[1])
        label = rate[2] if len(rate) > 2 else None
        self.reactions.append(Reaction(kind, params, list(reactants), list(products), label))

    def custom_param_labels(self) -> List[str]:
        """Labels in micm's order: reactions stably sorted by kind, UD then
        surface labels in that order (solver_builder.inl:129-188)."""
        order = sorted(range(self.n_reactions), key=lambda r: self.reactions[r].kind)
        labels: List[str] = []
        for r in order:
            rx = self.reactions[r]
            if rx.kind == USER_DEFINED:
                labels.append(rx.label)
            elif rx.kind == SURFACE:
                labels.append(rx.label + ".effective radius [m]")
                labels.append(rx.label + ".particle number concentration [# m-3]")
        if len(set(labels)) != len(labels):
            raise ValueError("duplicate custom parameter labels")
        return labels

    def flat(self) -> Dict[str, np.ndarray]:
        """Arrays of micmb_mechanism_desc (include/micmb.h)."""
        R = self.n_reactions
        rate_type = np.array([rx.kind for rx in self.reactions], dtype=np.int32)
        rate_params = np.zeros((R, RATE_PARAM_STRIDE), dtype=np.float64)
        for r, rx in enumerate(self.reactions):
            rate_params[r, : len(rx.params)] = rx.params
        rstart = np.zeros(R + 1, dtype=np.int32)
        pstart = np.zeros(R + 1, dtype=np.int32)
        rs, ps, py = [], [], []
        for r, rx in enumerate(self.reactions):
            rs.extend(rx.reactants)
            for s, y in rx.products:
                ps.append(s)
                py.append(y)
            rstart[r + 1] = len(rs)
            pstart[r + 1] = len(ps)
        pc = np.array(self.parameterized, dtype=np.float64).reshape(-1)
        return dict(
            n_species=self.n_species,
            n_reactions=R,
            rate_type=rate_type,
            rate_params=rate_params.reshape(-1).copy(),
            reactant_start=rstart,
            reactant_species=np.array(rs, dtype=np.int32),
            product_start=pstart,
            product_species=np.array(ps, dtype=np.int32),
            product_yield=np.array(py, dtype=np.float64),
            n_parameterized=len(self.parameterized),
            parameterized_coef=pc if pc.size else np.zeros(1, dtype=np.float64),
            reorder_state=1 if self.reorder_state else 0,
            **self._constraint_arrays(),
        )

    def _constraint_arrays(self) -> Dict[str, np.ndarray]:
        n = len(self.constraints)
        if n == 0:
            return dict(n_constraints=0)
        start = np.zeros(n + 1, dtype=np.int32)
        tsp, tco = [], []
        for i, c in enumerate(self.constraints):
            for a, coef in c.terms:
                tsp.append(a)
                tco.append(coef)
            start[i + 1] = len(tsp)
        return dict(
            n_constraints=n,
            constraint_type=np.array([c.kind for c in self.constraints], dtype=np.int32),
            constraint_species=np.array([c.species for c in self.constraints], dtype=np.int32),
            constraint_term_start=start,
            constraint_term_species=np.array(tsp, dtype=np.int32),
            constraint_term_coef=np.array(tco, dtype=np.float64),
            constraint_n_reactants=np.array([c.n_reactants for c in self.constraints], dtype=np.int32),
            constraint_params=np.array([list(c.params) for c in self.constraints], dtype=np.float64).reshape(-1),
        )

    def atol(self) -> np.ndarray:
        if self.absolute_tolerance is None:
            return np.full(self.n_species, 1e-3)   # SolverBuilder default (solver_builder.inl:208)
        return np.asarray(self.absolute_tolerance, dtype=np.float64)


_KIND_BY_NAME = {"arrhenius": ARRHENIUS, "troe": TROE, "ternary_chemical_activation": TERNARY_CHEMICAL_ACTIVATION,
                 "branched": BRANCHED, "tunneling": TUNNELING, "taylor_series": TAYLOR_SERIES,
                 "reversible": REVERSIBLE, "user_defined": USER_DEFINED, "surface": SURFACE}


def mechanism_from_dict(d: dict) -> Mechanism:
    """A mechanism from its JSON description:

    ``species``: names in gas-phase order (the state's system order);
    ``parameterized``: ``[{"name", "coefficients": [c0, c_T, c_P, c_rho]}]``
    (third bodies and other parameterized reactants, value c0 + c_T T + c_P P +
    c_rho rho as micm's ParameterizedFunction, parameterized_function.hpp:26-49);
    ``reactions``: ``[{"kind", "params", "reactants": [names], "products":
    [[name, yield]], "label"?}]`` in input order, ``params`` as the rate
    helpers of this module take them; optional ``absolute_tolerance`` (one
    value or one per species; micm's builder default 1e-3 otherwise),
    ``relative_tolerance`` and ``reorder_state`` (micm's SetReorderState,
    default true); optional ``constraints`` (micm's SetConstraints):
    ``[{"type": "linear", "name", "algebraic_species", "terms": [[name,
    coefficient]], "constant"}]`` or ``[{"type": "equilibrium", "name",
    "algebraic_species", "reactants": [[name, stoichiometry]], "products":
    [[name, stoichiometry]], "K_HLC_ref", "delta_H"?, "R"?, "T_ref"?}]``."""
    species = list(d["species"])
    index = {n: i for i, n in enumerate(species)}
    params = d.get("parameterized", [])
    pindex = {p["name"]: i for i, p in enumerate(params)}
    atol = d.get("absolute_tolerance")
    if atol is not None:
        atol = np.broadcast_to(np.asarray(atol, dtype=np.float64), (len(species),)).copy()
    m = Mechanism(species=species, reactions=[], name=d.get("name", "mechanism"),
                  parameterized=[tuple(float(c) for c in p["coefficients"]) for p in params],
                  absolute_tolerance=atol, relative_tolerance=float(d.get("relative_tolerance", 1e-6)),
                  reorder_state=bool(d.get("reorder_state", True)))

    def reactant(name):
        if name in index:
            return index[name]
        if name in pindex:
            return -(pindex[name] + 1)
        raise ValueError(f"unknown reactant '{name}'")

    for rx in d["reactions"]:
        kind = _KIND_BY_NAME[rx["kind"]]
        products = []
        for name, y in rx["products"]:
            if name in pindex:
                continue        # a parameterized product is no state variable (process_set.hpp:299-303)
            if name not in index:
                raise ValueError(f"unknown product '{name}'")
            products.append((index[name], float(y)))
        m.reactions.append(Reaction(kind, [float(v) for v in rx["params"]],
                                    [reactant(n) for n in rx["reactants"]], products, rx.get("label")))

    def species_index(name):
        if name not in index:
            raise ValueError(f"unknown constraint species '{name}'")
        return index[name]

    for c in d.get("constraints", []):
        row = species_index(c["algebraic_species"])
        if c["type"] == "linear":
            m.constraints.append(linear_constraint(row, [(species_index(n), float(v)) for n, v in c["terms"]],
                                                   float(c["constant"]), name=c.get("name", "linear")))
        elif c["type"] == "equilibrium":
            m.constraints.append(equilibrium_constraint(
                row, [(species_index(n), float(v)) for n, v in c["reactants"]],
                [(species_index(n), float(v)) for n, v in c["products"]], float(c["K_HLC_ref"]),
                float(c.get("delta_H", 0.0)), float(c.get("R", GAS_CONSTANT)), float(c.get("T_ref", 298.15)),
                name=c.get("name", "equilibrium")))
        else:
            raise ValueError(f"unknown constraint type '{c['type']}'")
    return m


_NAME_BY_KIND = {v: k for k, v in _KIND_BY_NAME.items()}


def mechanism_to_dict(m: Mechanism, parameterized_names: Optional[Sequence[str]] = None) -> dict:
    """The JSON description mechanism_from_dict reads (parameterized reactants
    are named param0, param1, ... unless names are given)."""
    pnames = list(parameterized_names) if parameterized_names else [f"param{i}" for i in range(len(m.parameterized))]

    def reactant(i):
        return m.species[i] if i >= 0 else pnames[-i - 1]

    reactions = []
    for rx in m.reactions:
        d = {"kind": _NAME_BY_KIND[rx.kind], "params": [float(v) for v in rx.params],
             "reactants": [reactant(i) for i in rx.reactants],
             "products": [[m.species[s], float(y)] for s, y in rx.products]}
        if rx.label is not None:
            d["label"] = rx.label
        reactions.append(d)
    out = {"name": m.name, "species": list(m.species),
           "parameterized": [{"name": n, "coefficients": [float(c) for c in coef]}
                             for n, coef in zip(pnames, m.parameterized)],
           "reactions": reactions, "relative_tolerance": float(m.relative_tolerance)}
    if m.absolute_tolerance is not None:
        out["absolute_tolerance"] = [float(v) for v in m.absolute_tolerance]
    if not m.reorder_state:
        out["reorder_state"] = False
    constraints = []
    for c in m.constraints:
        terms = [[m.species[i], float(v)] for i, v in c.terms]
        if c.kind == CONSTRAINT_LINEAR:
            constraints.append({"type": "linear", "name": c.name, "algebraic_species": m.species[c.species],
                                "terms": terms, "constant": float(c.params[0])})
        else:
            constraints.append({"type": "equilibrium", "name": c.name, "algebraic_species": m.species[c.species],
                                "reactants": terms[:c.n_reactants], "products": terms[c.n_reactants:],
                                "K_HLC_ref": float(c.params[0]), "delta_H": float(c.params[1]),
                                "R": float(c.params[2]), "T_ref": float(c.params[3])})
    if constraints:
        out["constraints"] = constraints
    return out


def save_mechanism_json(m: Mechanism, path: str):
    """mechanism_to_dict written to a JSON file."""
    import json
    with open(path, "w") as f:
        json.dump(mechanism_to_dict(m), f, indent=1)


def load_mechanism_json(path: str) -> Mechanism:
    """mechanism_from_dict of a JSON file."""
    import json
    with open(path) as f:
        return mechanism_from_dict(json.load(f))


def ideal_air_density(pressure, temperature):
    """Conditions::CalculateIdealAirDensity (include/micm/system/conditions.hpp:20-23)."""
    return np.asarray(pressure) / (GAS_CONSTANT * np.asarray(temperature))


# --------------------------------------------------------------------------
# Vector-ordered layout helpers (include/micm/util/vector_matrix.hpp:254-345)
# --------------------------------------------------------------------------

def padded_cells(n_cells: int, L: int) -> int:
    return -(-n_cells // L) * L


def to_vector_layout(a: np.ndarray, L: int) -> np.ndarray:
    """[cell][col] -> flat vector-ordered array with groups of L cells."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    n, m = a.shape
    npad = padded_cells(n, L)
    buf = np.zeros((npad, m), dtype=np.float64)
    buf[:n] = a
    return buf.reshape(npad // L, L, m).transpose(0, 2, 1).reshape(-1).copy()


def from_vector_layout(buf: np.ndarray, n_cells: int, n_cols: int, L: int) -> np.ndarray:
    npad = padded_cells(n_cells, L)
    a = np.asarray(buf).reshape(npad // L, n_cols, L).transpose(0, 2, 1).reshape(npad, n_cols)
    return a[:n_cells].copy()
