"""Material properties (reference materials.py:23-160, material_tables.py,
physics/surfactant.py:27-65 and 177-194, the Heiple path).

A material is a set of constants plus optional temperature tables (knots
[T_K, value] for cp, k, mu and dgamma_dT).  With tables the coupled step
runs the reference's table path: per-cell rho*cp(T), alpha(T), tau(T) from
mu(T) and dgamma/dT(T), refreshed from T every step (gpu_tables.py).
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field


@dataclass
class MaterialTables:
    """Temperature-dependent properties as sorted (T_K, value) knot lists
    (material_tables.py:8-18)."""
    cp: list = field(default_factory=list)
    k: list = field(default_factory=list)
    mu: list = field(default_factory=list)
    dgamma_dT: list = field(default_factory=list)

    def has_any(self) -> bool:
        return bool(self.cp or self.k or self.mu or self.dgamma_dT)


def _parse_knots(raw) -> list:
    """material_tables.py:21-28: rows of two numbers, sorted by T; other rows dropped."""
    out = []
    for row in raw or []:
        if len(row) != 2:
            continue
        out.append((float(row[0]), float(row[1])))
    out.sort(key=lambda p: p[0])
    return out


def tables_from_yaml(data) -> MaterialTables:
    """material_tables.py:31-39."""
    if not data:
        return MaterialTables()
    return MaterialTables(cp=_parse_knots(data.get("cp", [])), k=_parse_knots(data.get("k", [])),
                          mu=_parse_knots(data.get("mu", [])),
                          dgamma_dT=_parse_knots(data.get("dgamma_dT", [])))


def interp_linear(T: float, knots: list, fallback: float) -> float:
    """material_tables.py:42-54: clamped piecewise-linear, first matching segment."""
    if not knots:
        return fallback
    if T <= knots[0][0]:
        return knots[0][1]
    if T >= knots[-1][0]:
        return knots[-1][1]
    for (t0, v0), (t1, v1) in zip(knots[:-1], knots[1:]):
        if t0 <= T <= t1:
            if t1 == t0:
                return v0
            w = (T - t0) / (t1 - t0)
            return v0 + w * (v1 - v0)
    return fallback


@dataclass
class MaterialProps:
    name: str
    k: float
    rho: float
    cp: float
    alpha: float
    T_solidus: float
    T_liquidus: float
    L_fusion: float
    gamma_0: float
    dgamma_dT: float
    T_ref_gamma: float
    mu: float
    beta_T: float = 1.2e-4
    contact_angle_deg: float = 80.0
    rho_e_ohm_m: float = 1.5e-7
    eta_stick: float = 0.85
    sulphur_ppm: float = 30.0
    status: str = "placeholder"
    source: str = ""
    high_sulphur: bool = False
    tables: MaterialTables = field(default_factory=MaterialTables)

    def __post_init__(self):
        if isinstance(self.tables, dict):
            self.tables = MaterialTables(**{k: _parse_knots(v) for k, v in self.tables.items()})

    @property
    def has_tables(self) -> bool:
        return self.tables.has_any()

    # materials.py:48-58
    def cp_at(self, T: float) -> float:
        return interp_linear(T, self.tables.cp, self.cp)

    def k_at(self, T: float) -> float:
        return interp_linear(T, self.tables.k, self.k)

    def mu_at(self, T: float) -> float:
        return interp_linear(T, self.tables.mu, self.mu)

    def dgamma_dT_at(self, T: float) -> float:
        return interp_linear(T, self.tables.dgamma_dT, self.dgamma_dT)


def from_constants(name: str, c: dict, status: str = "placeholder", **extra) -> MaterialProps:
    """MaterialProps from a constants dict (keys as the reference YAML ``constants``)."""
    rho, cp, k = float(c["rho"]), float(c["cp"]), float(c["k"])
    return MaterialProps(
        name=name, k=k, rho=rho, cp=cp, alpha=float(c.get("alpha", k / (rho * cp))),
        T_solidus=float(c["T_solidus"]), T_liquidus=float(c["T_liquidus"]),
        L_fusion=float(c["L_fusion"]), gamma_0=float(c["gamma_0"]),
        dgamma_dT=float(c["dgamma_dT"]), T_ref_gamma=float(c.get("T_ref_gamma", c["T_liquidus"])),
        mu=float(c["mu"]), beta_T=float(c.get("beta_T", 1.2e-4)), status=status, **extra)


# ER70S-6-like steel with the constants every benchmark configuration uses.
ER70S6_CONSTANTS = dict(rho=7800.0, cp=680.0, k=30.0, T_solidus=1723.0, T_liquidus=1783.0,
                        L_fusion=2.7e5, gamma_0=1.8, dgamma_dT=-4.3e-4, mu=0.0065, beta_T=1.2e-4)


def er70s6_constants(contact_angle_deg: float = 30.0) -> MaterialProps:
    return from_constants("ER70S-6-constants", ER70S6_CONSTANTS,
                          contact_angle_deg=contact_angle_deg)


# ---- surfactant: Heiple-Roper static sulphur scale (physics/surfactant.py:27-65) ----
def surfactant_dgamma_dT_scale(sulphur_ppm: float) -> float:
    """Multiplier of the base dgamma/dT: 1 up to 30 ppm S, -0.35 from 60 ppm,
    linear in between (the sign flip models the inward Marangoni flow)."""
    s = max(0.0, sulphur_ppm)
    if s <= 30.0:
        return 1.0
    if s >= 60.0:
        return -0.35
    return 1.0 - 1.35 * ((s - 30.0) / 30.0)


def effective_dgamma_dT(base: float, sulphur_ppm: float) -> float:
    scale = surfactant_dgamma_dT_scale(sulphur_ppm)
    if scale < 0:
        return -abs(base) * scale
    return base * scale


# ---- surfactant: Sahoo, DebRoy & McNallan (1988) Fe-S isotherm (physics/surfactant.py:66-174) ----
# gamma(T, a_S) = gamma_m - A (T - T_m) - R T Gamma_s ln(1 + K a_S),
# K = k1 exp(-dH0 / (R T)), a_S ~ wt% S = ppm / 1e4 (Metall. Trans. B 19 (1988) 483).
SAHOO_FE_S = dict(gamma_m=1.943, A=4.3e-4, T_m=1809.0, Gamma_s=1.3e-5, k1=0.00318,
                  delta_H0=-1.66e5, R=8.314462618)


def _sahoo_Ka(T, sulphur_ppm, p):
    T = max(float(T), 300.0)
    a_s = max(0.0, float(sulphur_ppm)) / 10000.0
    return T, p["k1"] * math.exp(-p["delta_H0"] / (p["R"] * T)) * a_s


def gamma_sahoo(T, sulphur_ppm, params=None, T_m=None):
    p = params or SAHOO_FE_S
    Tm = float(T_m) if T_m is not None else p["T_m"]
    T, Ka = _sahoo_Ka(T, sulphur_ppm, p)
    return p["gamma_m"] - p["A"] * (T - Tm) - p["R"] * T * p["Gamma_s"] * math.log(1.0 + Ka)


def dgamma_dT_sahoo(T, sulphur_ppm, params=None):
    """d gamma / dT of the isotherm (mixing enthalpy neglected):
    -A - R Gamma_s ln(1 + K a) - K a / (1 + K a) * Gamma_s dH0 / T."""
    p = params or SAHOO_FE_S
    T, Ka = _sahoo_Ka(T, sulphur_ppm, p)
    frac = Ka / (1.0 + Ka) if Ka > 0.0 else 0.0
    return (-p["A"] - p["R"] * p["Gamma_s"] * math.log(1.0 + Ka)
            - frac * p["Gamma_s"] * p["delta_H0"] / T)


def build_sahoo_dgamma_table(sulphur_ppm, T_min, T_max, n=25, params=None):
    n = max(2, int(n))
    lo = float(T_min)
    hi = max(lo + 1.0, float(T_max))
    return [(lo + (hi - lo) * i / (n - 1), dgamma_dT_sahoo(lo + (hi - lo) * i / (n - 1),
                                                            sulphur_ppm, params))
            for i in range(n)]


def apply_sahoo_to_material_props(props: MaterialProps) -> None:
    """An 8-knot dgamma/dT table from T_liquidus to max(T_liquidus + 800, 2600) K,
    the scalar dgamma/dT at T_liquidus + 50 K and gamma_0 at T_liquidus."""
    T_liq = float(props.T_liquidus)
    props.tables.dgamma_dT = build_sahoo_dgamma_table(props.sulphur_ppm, T_liq,
                                                      max(T_liq + 800.0, 2600.0), n=8)
    props.dgamma_dT = dgamma_dT_sahoo(T_liq + 50.0, props.sulphur_ppm)
    props.gamma_0 = gamma_sahoo(T_liq, props.sulphur_ppm, T_m=T_liq)
    props.T_ref_gamma = T_liq


def apply_surfactant_model(props: MaterialProps, model: str = "heiple") -> None:
    """physics/surfactant.py:177-194: "heiple" scales dgamma/dT (and its table)
    by the sulphur content; "sahoo" replaces them by the Fe-S isotherm."""
    key = (model or "heiple").lower().replace("-", "_")
    if key in ("sahoo", "sahoo_debroy", "debroy"):
        apply_sahoo_to_material_props(props)
        return
    scale = surfactant_dgamma_dT_scale(props.sulphur_ppm)
    props.dgamma_dT = effective_dgamma_dT(props.dgamma_dT, props.sulphur_ppm)
    if props.tables.dgamma_dT:
        props.tables.dgamma_dT = [(t, -abs(dg) * scale if scale < 0 else dg * scale)
                                  for t, dg in props.tables.dgamma_dT]


# Constants of the reference's built-in fallback library (materials.py:169-190),
# used when no material YAML is found for a name.
LEGACY_LIBRARY = {
    "ER70S-6": dict(k=30.0, rho=7000.0, cp=680.0, alpha=6.3e-6, T_solidus=1748.0,
                    T_liquidus=1793.0, L_fusion=272_000.0, gamma_0=1.8, dgamma_dT=-4.3e-4,
                    T_ref_gamma=1793.0, mu=6.5e-3),
    "SS316L": dict(k=16.3, rho=6900.0, cp=750.0, alpha=3.1e-6, T_solidus=1648.0,
                   T_liquidus=1723.0, L_fusion=285_000.0, gamma_0=1.6, dgamma_dT=-3.5e-4,
                   T_ref_gamma=1723.0, mu=5.5e-3),
    "AISI4043": dict(k=160.0, rho=2380.0, cp=900.0, alpha=74.0e-6, T_solidus=846.0,
                     T_liquidus=904.0, L_fusion=397_000.0, gamma_0=0.87, dgamma_dT=-1.55e-4,
                     T_ref_gamma=904.0, mu=1.3e-3, beta_T=2.5e-4),
}


def _material_dirs(materials_dir=None):
    dirs = []
    if materials_dir:
        dirs.append(materials_dir)
    dirs += [d for d in os.environ.get("WAAM_MATERIALS_DIR", "").split(os.pathsep) if d]
    return dirs


def resolve_material_path(name: str, materials_dir=None):
    """materials.py:150-165: an existing path, else <dir>/validated/<name>.yaml|.yml,
    then <dir>/placeholders/..., for each materials directory (the argument,
    then the WAAM_MATERIALS_DIR list)."""
    if os.path.exists(name):
        return name
    for base in _material_dirs(materials_dir):
        if os.path.exists(os.path.join(base, name)):
            return os.path.join(base, name)
        for sub in ("validated", "placeholders"):
            for ext in (".yaml", ".yml"):
                cand = os.path.join(base, sub, name + ext)
                if os.path.exists(cand):
                    return cand
            cand = os.path.join(base, sub, name)
            if os.path.exists(cand):
                return cand
    return None


def load_material_yaml(path: str) -> MaterialProps:
    """materials.py:127-147: constants, surface / electrical / surfactant
    sections, temperature tables, then the surfactant model."""
    import yaml
    with open(path) as fh:
        data = yaml.safe_load(fh)
    for key in ("name", "status", "constants"):
        if key not in data:
            raise ValueError("material %s: missing required key %r" % (path, key))
    surf = data.get("surface", {}) or {}
    elec = data.get("electrical", {}) or {}
    sact = data.get("surfactant", {}) or {}
    props = from_constants(data.get("name", os.path.splitext(os.path.basename(path))[0]),
                           data["constants"], status=data.get("status", "placeholder"),
                           source=data.get("source", ""),
                           contact_angle_deg=float(surf.get("contact_angle_deg", 80.0)),
                           rho_e_ohm_m=float(elec.get("rho_e_ohm_m", 1.5e-7)),
                           eta_stick=float(elec.get("eta_stick", 0.85)),
                           sulphur_ppm=float(sact.get("sulphur_ppm", 30.0)))
    props.tables = tables_from_yaml(data.get("tables"))
    apply_surfactant_model(props, str(sact.get("model", "heiple")))
    return props


def load_material(spec, high_sulphur: bool = False, materials_dir=None) -> MaterialProps:
    """MaterialProps from a MaterialProps, a constants dict (optionally with
    ``tables``), a material YAML path or a material name (materials.py:194-241:
    YAML under the materials directories, else the built-in library)."""
    if isinstance(spec, MaterialProps):
        props = spec
    elif isinstance(spec, dict):
        props = from_constants(spec.get("name", "material"), spec.get("constants", spec))
        props.tables = tables_from_yaml(spec.get("tables"))
    else:
        path = resolve_material_path(str(spec), materials_dir)
        if path is not None:
            props = load_material_yaml(path)
        else:
            key = next((k for k in LEGACY_LIBRARY if str(spec).upper().startswith(k.upper())),
                       None)
            if key is None:
                raise KeyError("Material '%s' not found: pass a YAML path, set "
                               "WAAM_MATERIALS_DIR, or use one of %s"
                               % (spec, sorted(LEGACY_LIBRARY)))
            props = from_constants(key, LEGACY_LIBRARY[key], status="placeholder",
                                   source="legacy constant")
    if high_sulphur:
        # materials.py:226-235
        props.sulphur_ppm = max(float(props.sulphur_ppm), 150.0)
        props.high_sulphur = True
        if len(props.tables.dgamma_dT) >= 10:
            apply_sahoo_to_material_props(props)
        else:
            props.dgamma_dT = abs(float(props.dgamma_dT))
    return props
