"""Physics/grid parameters with the reference's defaults and inputs-deck keys.

Defaults follow ``InitializeCommonNamespace`` (common_functions.cpp:332-550) and
``InitializeCompressibleNamespace`` (compressible_functions.cpp:15-88): k_B,
Runiv, e0 = 0, visc_type 1, advection_type 0, stoch_stress_form 1,
transport_type 1.  ``parse_inputs`` reads an FHDeX inputs deck (``key = values``
with ``#`` comments) using the same key names.
"""
from __future__ import annotations

import dataclasses
import math
from dataclasses import dataclass, field

from .capi import MAX_REACTIONS, MAX_SPECIES, FhdParams

K_B = 1.38064852e-16
RUNIV = 8.314462175e7


@dataclass
class Params:
    nspecies: int = 2
    n_cells: tuple = (32, 32, 32)
    prob_lo: tuple = (0.0, 0.0, 0.0)
    prob_hi: tuple = (3.2e-5, 3.2e-5, 3.2e-5)
    molmass: tuple = (39.95, 39.95)
    diameter: tuple = (3.66e-8, 3.66e-8)
    dof: tuple = (3.0, 3.0)
    e0: tuple = (0.0, 0.0)
    hcv: tuple = (-1.0, -1.0)
    hcp: tuple = (-1.0, -1.0)
    k_B: float = K_B
    Runiv: float = RUNIV
    grav: tuple = (0.0, 0.0, 0.0)
    zeta_ratio: float = -1.0
    algorithm_type: int = 2
    visc_type: int = 2
    advection_type: int = 2
    transport_type: int = 1
    stoch_stress_form: int = 1
    precision: int = 0
    seed: int = 1
    # chemistry (chemistry_functions.cpp:45-124): stoich_R/stoich_P one tuple of
    # nspecies coefficients per reaction; avogadro <= 0 means Runiv / k_B
    nreaction: int = 0
    reaction_type: int = 0
    stoich_R: tuple = ()
    stoich_P: tuple = ()
    rate_const: tuple = ()
    alpha_param: tuple = ()
    beta_param: tuple = ()
    T0_chem: float = 0.0
    avogadro: float = 0.0
    # physical boundaries (boundaryStag.cpp; the reference's deck keys): walls = 0
    # fully periodic; else a direction with bc_vel_lo == bc_vel_hi == -1 is
    # periodic and the others have walls on both sides (bc_vel 1 slip / 2 no-slip,
    # bc_therm 1 adiabatic / 2 isothermal at t_lo / t_hi, bc_mass 1 impermeable /
    # 2 wall composition bc_Yk or bc_Xk, one tuple of nspecies values per direction)
    walls: int = 0
    bc_vel_lo: tuple = (-1, -1, -1)
    bc_vel_hi: tuple = (-1, -1, -1)
    bc_mass_lo: tuple = (-1, -1, -1)
    bc_mass_hi: tuple = (-1, -1, -1)
    bc_therm_lo: tuple = (-1, -1, -1)
    bc_therm_hi: tuple = (-1, -1, -1)
    t_lo: tuple = (0.0, 0.0, 0.0)
    t_hi: tuple = (0.0, 0.0, 0.0)
    bc_Yk_lo: tuple = ((), (), ())
    bc_Yk_hi: tuple = ((), (), ())
    bc_Xk_lo: tuple = ((), (), ())
    bc_Xk_hi: tuple = ((), (), ())
    # reservoirs (bc_mass 3): pressure (<= 0: the initial state's) and density
    # (<= 0: from p, t and the composition)
    p_lo: tuple = (0.0, 0.0, 0.0)
    p_hi: tuple = (0.0, 0.0, 0.0)
    rho_lo: tuple = (-1.0, -1.0, -1.0)
    rho_hi: tuple = (-1.0, -1.0, -1.0)
    # initial state (prob_type 1): not part of fhd_params
    rho0: float = 1.78e-3
    T_init: float = 273.0
    rhobar: tuple = (0.5, 0.5)
    ngc: int = 2
    # plot_cross's cell x* (common::cross_cell; statsStag.cpp:868-1105)
    cross_cell: int = 0
    # quasi-1-D / quasi-2-D runs (compressible::do_1D / do_2D): the step's noise only
    # in x (x and y), timeStepStag.cpp:172-323; transport on one ghost layer in 1-D
    do_1D: int = 0
    do_2D: int = 0
    # quasi-1-D statistics: correlate with five x* instead of cross_cell (compressible::all_correl)
    all_correl: int = 0

    @property
    def nvars(self):
        return 5 + self.nspecies

    @property
    def nprimvars(self):
        return 6 + 2 * self.nspecies

    @property
    def dx(self):
        return tuple((self.prob_hi[d] - self.prob_lo[d]) / self.n_cells[d] for d in range(3))

    def replace(self, **kw):
        return dataclasses.replace(self, **kw)

    def to_inputs(self) -> str:
        """This parameter set as an FHDeX inputs deck (see ``to_inputs``)."""
        return to_inputs(self)

    def hc(self):
        """(hcv, hcp) as GetHcGas derives them (compressible_functions.cpp:91-100)."""
        hcv, hcp = [], []
        for i in range(self.nspecies):
            v = self.hcv[i] if self.hcv[i] >= 0 else 0.5 * self.dof[i] * self.Runiv / self.molmass[i]
            p = self.hcp[i] if self.hcp[i] >= 0 else 0.5 * (2.0 + self.dof[i]) * self.Runiv / self.molmass[i]
            hcv.append(v)
            hcp.append(p)
        return hcv, hcp

    def to_c(self) -> FhdParams:
        p = FhdParams()
        p.nspecies = self.nspecies
        for d in range(3):
            p.n_cells[d] = self.n_cells[d]
            p.prob_lo[d] = self.prob_lo[d]
            p.prob_hi[d] = self.prob_hi[d]
            p.grav[d] = self.grav[d]
        for name in ("molmass", "diameter", "dof", "e0", "hcv", "hcp"):
            src = getattr(self, name)
            dst = getattr(p, name)
            for i in range(MAX_SPECIES):
                dst[i] = src[i] if i < len(src) else (0.0 if name in ("e0",) else (-1.0 if name in ("hcv", "hcp") else 1.0))
        p.k_B = self.k_B
        p.Runiv = self.Runiv
        p.zeta_ratio = self.zeta_ratio
        p.algorithm_type = self.algorithm_type
        p.visc_type = self.visc_type
        p.advection_type = self.advection_type
        p.transport_type = self.transport_type
        p.stoch_stress_form = self.stoch_stress_form
        p.precision = self.precision
        p.seed = self.seed & 0xFFFFFFFFFFFFFFFF
        p.nreaction = self.nreaction
        p.reaction_type = self.reaction_type
        for m in range(min(self.nreaction, MAX_REACTIONS)):
            for n in range(self.nspecies):
                p.stoich_R[m][n] = int(self.stoich_R[m][n])
                p.stoich_P[m][n] = int(self.stoich_P[m][n])
            p.rate_const[m] = self.rate_const[m]
            p.alpha_param[m] = self.alpha_param[m] if m < len(self.alpha_param) else 0.0
            p.beta_param[m] = self.beta_param[m] if m < len(self.beta_param) else 0.0
        p.T0_chem = self.T0_chem
        p.avogadro = self.avogadro
        p.walls = 1 if self.walls else 0
        for d in range(3):
            for name in ("bc_vel_lo", "bc_vel_hi", "bc_mass_lo", "bc_mass_hi", "bc_therm_lo", "bc_therm_hi",
                         "t_lo", "t_hi"):
                getattr(p, name)[d] = getattr(self, name)[d]
            for name in ("bc_Yk_lo", "bc_Yk_hi", "bc_Xk_lo", "bc_Xk_hi"):
                vals = getattr(self, name)[d]
                for i in range(MAX_SPECIES):
                    getattr(p, name)[d][i] = vals[i] if i < len(vals) else -1.0
            for name in ("p_lo", "p_hi", "rho_lo", "rho_hi"):
                getattr(p, name)[d] = getattr(self, name)[d]
        p.rho0 = self.rho0
        p.T_init = self.T_init
        p.cross_cell = self.cross_cell
        p.do_1D = self.do_1D
        p.do_2D = self.do_2D
        p.all_correl = self.all_correl
        for i in range(MAX_SPECIES):
            p.rhobar[i] = self.rhobar[i] if i < len(self.rhobar) else 0.0
        return p

    # -- thermodynamics on the host (for dt and theory) -------------------------------
    def sound_speed(self, T=None, Y=None):
        """GetSoundSpeed, compressible_functions.H:201-219."""
        T = self.T_init if T is None else T
        Y = self.rhobar if Y is None else Y
        hcv, hcp = self.hc()
        molmix = sum(Y[n] / self.molmass[n] for n in range(self.nspecies))
        molmix = 1.0 / molmix
        cv = sum(Y[n] * hcv[n] for n in range(self.nspecies))
        cp = sum(Y[n] * hcp[n] for n in range(self.nspecies))
        return math.sqrt(cp / cv * (self.Runiv / molmix) * T)


def argon(n=32, dx=1e-6, **kw) -> Params:
    """'Single-species' argon in the reference's parity form: two identical species
    (molmass 39.95, d = 3.66e-8 cm), rho0 = 1.78e-3 g/cm^3, T0 = 273 K."""
    n3 = (n, n, n) if isinstance(n, int) else tuple(n)
    base = Params(nspecies=2, n_cells=n3, prob_hi=tuple(dx * n3[d] for d in range(3)),
                  molmass=(39.95, 39.95), diameter=(3.66e-8, 3.66e-8), dof=(3.0, 3.0),
                  e0=(0.0, 0.0), hcv=(-1.0, -1.0), hcp=(-1.0, -1.0), rhobar=(0.5, 0.5))
    return base.replace(**kw)


def argon_single(n=32, dx=1e-6, **kw) -> Params:
    """Argon as one species (the single-gas fast path: no species flux; the
    reference itself cannot run nspecies = 1 and uses two identical species,
    ``argon``).  Same gas, same stable dt as ``argon``."""
    n3 = (n, n, n) if isinstance(n, int) else tuple(n)
    base = Params(nspecies=1, n_cells=n3, prob_hi=tuple(dx * n3[d] for d in range(3)),
                  molmass=(39.95,), diameter=(3.66e-8,), dof=(3.0,), e0=(0.0,), hcv=(-1.0,), hcp=(-1.0,),
                  rhobar=(1.0,))
    return base.replace(**kw)


def mixture4(n=32, dx=1e-6, **kw) -> Params:
    """4-species ideal-gas mixture (Ar/Ne/Kr/He), equal mass fractions."""
    n3 = (n, n, n) if isinstance(n, int) else tuple(n)
    base = Params(nspecies=4, n_cells=n3, prob_hi=tuple(dx * n3[d] for d in range(3)),
                  molmass=(39.95, 20.18, 83.80, 4.00),
                  diameter=(3.66e-8, 2.58e-8, 4.16e-8, 2.18e-8), dof=(3.0,) * 4,
                  e0=(0.0,) * 4, hcv=(-1.0,) * 4, hcp=(-1.0,) * 4, rhobar=(0.25,) * 4)
    return base.replace(**kw)


def no2_dimerization(n=16, dx=1e-5, **kw) -> Params:
    """2 NO2 <-> N2O4 with the reference's compressible chemistry: two species
    (NO2, N2O4), reaction 1 = 2 NO2 -> N2O4, reaction 2 = N2O4 -> 2 NO2, Arrhenius
    factors about T0 = 350 K, chemical Langevin noise (reaction_type 1); gas
    constants and composition of exec/compressible_stag/test_NO2_dimerization_eq
    (inputs_NO2_dimerization_eq), whose initial state is at chemical equilibrium."""
    n3 = (n, n, n) if isinstance(n, int) else tuple(n)
    base = Params(nspecies=2, n_cells=n3, prob_hi=tuple(dx * n3[d] for d in range(3)),
                  molmass=(46.0055, 92.0110), diameter=(3.765e-08, 4.621e-08), dof=(7.279586, 18.049072),
                  e0=(0.0, 0.0), hcv=(-1.0, -1.0), hcp=(-1.0, -1.0), k_B=1.38065e-16, Runiv=8.31446e7,
                  rho0=1.858338e-03, T_init=350.0, rhobar=(0.723969, 0.276031),
                  nreaction=2, reaction_type=1, stoich_R=((2, 0), (0, 1)), stoich_P=((0, 1), (2, 0)),
                  rate_const=(4.065753e+11, 6.236899e+07), alpha_param=(-5.337990e+10, 5.370000e+11),
                  beta_param=(0.644950, -1.100000), T0_chem=350.0)
    return base.replace(**kw)


def isomerization(p: Params) -> Params:
    """First-order A <-> B on the species of ``p`` (stoichiometric coefficients 0/1,
    no activation energy, no temperature power): the case in which every power and
    exponential of the chemistry source is exact."""
    return p.replace(nreaction=2, reaction_type=1, stoich_R=((1, 0), (0, 1)), stoich_P=((0, 1), (1, 0)),
                     rate_const=(2.0e5, 3.0e5), alpha_param=(0.0, 0.0), beta_param=(0.0, 0.0),
                     T0_chem=p.T_init)


def exchange_network(p: Params) -> Params:
    """A + B <-> C + D and A <-> C on the first four species of ``p`` (coefficients
    0/1, no activation energy, no temperature power): a four-species reaction
    network whose powers and exponentials are all exact.  A parity case for the
    four-species kernel, not a chemical system: the molar masses of the species it
    is applied to need not balance."""
    return p.replace(nreaction=3, reaction_type=1,
                     stoich_R=((1, 1, 0, 0), (0, 0, 1, 1), (1, 0, 0, 0)),
                     stoich_P=((0, 0, 1, 1), (1, 1, 0, 0), (0, 0, 1, 0)),
                     rate_const=(3.0e9, 2.0e9, 5.0e4), alpha_param=(0.0, 0.0, 0.0), beta_param=(0.0, 0.0, 0.0),
                     T0_chem=p.T_init)


def hard_sphere_single_gas(p: Params, T=None):
    """Closed-form first Chapman-Enskog hard-sphere viscosity and conductivity of a
    pure gas: eta = 5/(16 d^2) sqrt(m k T / pi), kappa = (75/64)(k/d^2) sqrt(kT/(pi m)).
    These are what the Giovangigli formulas (compressible_functions.H:1218-1326)
    reduce to for identical species."""
    T = p.T_init if T is None else T
    m = p.molmass[0] * p.k_B / p.Runiv
    d = p.diameter[0]
    eta = 5.0 / (16.0 * d * d) * math.sqrt(m * p.k_B * T / math.pi)
    kappa = 75.0 / 64.0 * p.k_B / (d * d) * math.sqrt(p.k_B * T / (math.pi * m))
    return eta, kappa


def with_walls(p: Params, **dirs) -> Params:
    """``p`` with physical walls on the directions named x, y, z (both sides),
    each a dict: vel (1 slip, 2 no-slip), therm (1 adiabatic, 2 isothermal), mass
    (1 impermeable, 2 held at a wall composition, 3 reservoir, 4 particle
    reservoir), t = (t_lo, t_hi)
    for isothermal walls and reservoirs, Yk or Xk = (lo, hi) compositions for
    concentration walls and reservoirs, p / rho = (lo, hi) reservoir pressure and
    density (defaults: the initial pressure; rho from p, t, Y).  The other
    directions stay periodic."""
    vl, vh, ml, mh, tl, th = ([-1] * 3 for _ in range(6))
    Tl, Th = [0.0] * 3, [0.0] * 3
    comp = {k: [(), (), ()] for k in ("bc_Yk_lo", "bc_Yk_hi", "bc_Xk_lo", "bc_Xk_hi")}
    Pl, Ph, Rl, Rh = [0.0] * 3, [0.0] * 3, [-1.0] * 3, [-1.0] * 3
    for ax, spec in dirs.items():
        d = "xyz".index(ax)
        vl[d] = vh[d] = int(spec.get("vel", 2))
        ml[d] = mh[d] = int(spec.get("mass", 1))
        tl[d] = th[d] = int(spec.get("therm", 1))
        Tl[d], Th[d] = (float(v) for v in spec.get("t", (p.T_init, p.T_init)))
        Pl[d], Ph[d] = (float(v) for v in spec.get("p", (0.0, 0.0)))
        Rl[d], Rh[d] = (float(v) for v in spec.get("rho", (-1.0, -1.0)))
        for key in ("Yk", "Xk"):
            if key in spec:
                comp[f"bc_{key}_lo"][d] = tuple(float(v) for v in spec[key][0])
                comp[f"bc_{key}_hi"][d] = tuple(float(v) for v in spec[key][1])
    return p.replace(walls=1, bc_vel_lo=tuple(vl), bc_vel_hi=tuple(vh), bc_mass_lo=tuple(ml),
                     bc_mass_hi=tuple(mh), bc_therm_lo=tuple(tl), bc_therm_hi=tuple(th), t_lo=tuple(Tl),
                     t_hi=tuple(Th), p_lo=tuple(Pl), p_hi=tuple(Ph), rho_lo=tuple(Rl), rho_hi=tuple(Rh),
                     **{k: tuple(v) for k, v in comp.items()})


def stable_dt(p: Params, cfl=0.2, diff=0.1):
    """dt = min(cfl*dx/(c+|u|), diff*dx^2/max(nu, chi)) at the initial state (|u| = 0).
    The configured acoustic CFL 0.2 alone violates the explicit diffusive limit at
    dx = 1e-6 cm, so the diffusive bound is applied too."""
    dx = min(p.dx)
    c = p.sound_speed()
    hcv, _ = p.hc()
    cv = sum(p.rhobar[n] * hcv[n] for n in range(p.nspecies))
    # bound the mixture's diffusivities by each species' pure-gas hard-sphere value
    # at the mixture's density and heat capacity (conservative for mixtures)
    dmax = 0.0
    for s in range(p.nspecies):
        q = p.replace(molmass=(p.molmass[s],), diameter=(p.diameter[s],))
        eta, kappa = hard_sphere_single_gas(q)
        dmax = max(dmax, eta / p.rho0, kappa / (p.rho0 * cv))
    return min(cfl * dx / c, diff * dx * dx / dmax)


def _fmt(v) -> str:
    return repr(float(v)) if isinstance(v, float) else str(v)


def to_inputs(p: "Params") -> str:
    """``p`` as an FHDeX inputs deck with the reference's key names
    (common_functions.cpp:257-1010, compressible_functions.cpp:15-88,
    chemistry_functions.cpp:45-124): fully periodic, two ghost cells,
    prob_type 1, nvars / nprimvars as main_driver.cpp:47-53 requires them.
    Floats are written in their shortest round-trip form, so a reader that
    parses decimal to the nearest double gets every value back exactly;
    ``parse_inputs`` reads the deck back into the same parameters."""
    ns = p.nspecies

    def row(key, vals):
        return f"{key} = " + " ".join(_fmt(float(x)) if not isinstance(x, int) else str(x) for x in vals)

    lines = [f"nspecies = {ns}", row("n_cells", [int(x) for x in p.n_cells]), row("prob_lo", p.prob_lo),
             row("prob_hi", p.prob_hi), f"ngc = {p.ngc} {p.ngc} {p.ngc}", f"nvars = {p.nvars}",
             f"nprimvars = {p.nprimvars}", row("molmass", p.molmass[:ns]), row("diameter", p.diameter[:ns]),
             row("dof", p.dof[:ns]), row("e0", p.e0[:ns]), row("hcv", p.hcv[:ns]), row("hcp", p.hcp[:ns]),
             row("rhobar", p.rhobar[:ns]), f"rho0 = {_fmt(float(p.rho0))}", f"T_init = {_fmt(float(p.T_init))}",
             f"k_B = {_fmt(float(p.k_B))}", f"Runiv = {_fmt(float(p.Runiv))}", row("grav", p.grav),
             f"algorithm_type = {p.algorithm_type}", f"visc_type = {p.visc_type}",
             f"advection_type = {p.advection_type}", f"transport_type = {p.transport_type}",
             f"stoch_stress_form = {p.stoch_stress_form}", f"seed = {p.seed}", "prob_type = 1",
             f"cross_cell = {p.cross_cell}", f"do_1D = {p.do_1D}", f"do_2D = {p.do_2D}",
             f"all_correl = {p.all_correl}"]
    if p.zeta_ratio >= 0:
        lines.append(f"zeta_ratio = {_fmt(float(p.zeta_ratio))}")
    for key in ("bc_vel_lo", "bc_vel_hi", "bc_mass_lo", "bc_mass_hi", "bc_therm_lo", "bc_therm_hi"):
        vals = getattr(p, key) if p.walls else (-1, -1, -1)
        lines.append(row(key, [int(x) for x in vals]))
    if p.walls:
        lines += [row("t_lo", p.t_lo), row("t_hi", p.t_hi), row("p_lo", p.p_lo), row("p_hi", p.p_hi),
                  row("rho_lo", p.rho_lo), row("rho_hi", p.rho_hi)]
        for name, key in (("bc_Yk_lo", "bc_Yk_{}_lo"), ("bc_Yk_hi", "bc_Yk_{}_hi"), ("bc_Xk_lo", "bc_Xk_{}_lo"),
                          ("bc_Xk_hi", "bc_Xk_{}_hi")):
            for d, ax in enumerate("xyz"):
                vals = getattr(p, name)[d]
                if len(vals):
                    lines.append(row(key.format(ax), [float(v) for v in vals]))
    if p.nreaction > 0:
        nr = p.nreaction
        lines += [f"nreaction = {nr}", f"reaction_type = {p.reaction_type}"]
        for m in range(nr):
            lines.append(row(f"stoich_{m + 1}R", [int(x) for x in p.stoich_R[m][:ns]]))
            lines.append(row(f"stoich_{m + 1}P", [int(x) for x in p.stoich_P[m][:ns]]))
        lines += [row("rate_const", p.rate_const[:nr]), row("alpha_param", (list(p.alpha_param) + [0.0] * nr)[:nr]),
                  row("beta_param", (list(p.beta_param) + [0.0] * nr)[:nr]), f"T0_chem = {_fmt(float(p.T0_chem))}"]
    if p.avogadro > 0:
        lines.append(f"avogadro = {_fmt(float(p.avogadro))}")
    return "\n".join(lines) + "\n"


_LIST_KEYS = ("n_cells", "prob_lo", "prob_hi", "molmass", "diameter", "dof", "e0", "hcv",
              "hcp", "rhobar", "grav", "T_init")


def parse_inputs(text: str, base: Params | None = None) -> Params:
    """Parse an FHDeX inputs deck (reference key names) into Params.  Keys outside
    this path (plot_int, struct_fact_int, ...) are ignored; reservoir boundaries
    are rejected."""
    kv = {}
    for line in text.splitlines():
        line = line.split("#", 1)[0].strip()
        if "=" not in line:
            continue
        k, v = line.split("=", 1)
        kv[k.strip()] = v.split()
    p = base or Params()
    upd = {}
    ns = int(kv["nspecies"][0]) if "nspecies" in kv else p.nspecies
    upd["nspecies"] = ns
    for key in _LIST_KEYS:
        if key in kv:
            vals = [float(x) for x in kv[key]]
            if key == "n_cells":
                vals = [int(x) for x in vals]
            if key == "T_init":
                upd["T_init"] = vals[0]
                continue
            upd[key] = tuple(vals)
    for key in ("rho0", "k_B", "Runiv", "zeta_ratio"):
        if key in kv:
            upd[key] = float(kv[key][0])
    for key in ("algorithm_type", "visc_type", "advection_type", "transport_type",
                "stoch_stress_form", "seed", "cross_cell", "do_1D", "do_2D", "all_correl"):
        if key in kv:
            upd[key] = int(kv[key][0])
    # chemistry keys (chemistry_functions.cpp:45-124); avogadro overrides Runiv
    # (common_functions.cpp:775-777)
    nr = int(kv["nreaction"][0]) if "nreaction" in kv else 0
    if nr > 0:
        upd["nreaction"] = nr
        upd["reaction_type"] = int(kv["reaction_type"][0])
        upd["stoich_R"] = tuple(tuple(int(x) for x in kv[f"stoich_{m + 1}R"][:ns]) for m in range(nr))
        upd["stoich_P"] = tuple(tuple(int(x) for x in kv[f"stoich_{m + 1}P"][:ns]) for m in range(nr))
        upd["rate_const"] = tuple(float(x) for x in kv["rate_const"][:nr])
        for key in ("alpha_param", "beta_param"):
            vals = [float(x) for x in kv.get(key, [])[:nr]]
            upd[key] = tuple(vals + [0.0] * (nr - len(vals)))
        if "T0_chem" in kv:
            upd["T0_chem"] = float(kv["T0_chem"][0])
    if "avogadro" in kv:
        upd["avogadro"] = float(kv["avogadro"][0])
        upd["Runiv"] = upd.get("k_B", p.k_B) * upd["avogadro"]
    # physical boundaries (boundaryStag.cpp): walls on the directions whose bc_vel is
    # not -1; reservoirs (bc_mass >= 3) are outside the implemented scope
    bck = ("bc_vel_lo", "bc_vel_hi", "bc_mass_lo", "bc_mass_hi", "bc_therm_lo", "bc_therm_hi")
    if any(k in kv and any(int(x) != -1 for x in kv[k]) for k in bck):
        upd["walls"] = 1
        for key in bck:
            if key in kv:
                upd[key] = tuple(int(x) for x in kv[key][:3])
        for key in ("bc_mass_lo", "bc_mass_hi"):
            if any(v >= 5 for v in upd.get(key, ())):
                raise ValueError(f"{key}: bc_mass values above 4 are not boundary conditions of this step")
        for key in ("t_lo", "t_hi", "p_lo", "p_hi", "rho_lo", "rho_hi"):
            if key in kv:
                upd[key] = tuple(float(x) for x in kv[key][:3])
        for name, pat in (("bc_Yk_lo", "bc_Yk_{}_lo"), ("bc_Yk_hi", "bc_Yk_{}_hi"), ("bc_Xk_lo", "bc_Xk_{}_lo"),
                          ("bc_Xk_hi", "bc_Xk_{}_hi")):
            upd[name] = tuple(tuple(float(x) for x in kv.get(pat.format(ax), [])[:ns]) for ax in "xyz")
    if "dof" in upd and "hcv" not in upd:
        upd["hcv"] = (-1.0,) * ns
        upd["hcp"] = (-1.0,) * ns
    return p.replace(**upd)
