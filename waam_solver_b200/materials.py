"""Material properties (reference materials.py:23-80, constants path only)."""
from __future__ import annotations

from dataclasses import dataclass, field


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
    tables: dict = field(default_factory=dict)

    @property
    def has_tables(self) -> bool:
        return any(bool(v) for v in (self.tables or {}).values())


def from_constants(name: str, c: dict, status: str = "synthetic", **extra) -> MaterialProps:
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


def load_material(spec, high_sulphur: bool = False) -> MaterialProps:
    """MaterialProps from a MaterialProps, a constants dict or a YAML file with a
    ``constants`` section.  Temperature tables are rejected (constants path only)."""
    if isinstance(spec, MaterialProps):
        return spec
    if isinstance(spec, dict):
        return from_constants(spec.get("name", "material"), spec.get("constants", spec))
    if spec in ("ER70S-6", "er70s6"):
        return er70s6_constants(80.0)
    import yaml
    with open(spec) as fh:
        data = yaml.safe_load(fh)
    if data.get("tables"):
        raise ValueError("material %s has temperature tables; only constants-only materials "
                         "are supported" % spec)
    surf = data.get("surface", {}) or {}
    return from_constants(data.get("name", str(spec)), data["constants"],
                          status=data.get("status", "placeholder"),
                          contact_angle_deg=float(surf.get("contact_angle_deg", 80.0)))
