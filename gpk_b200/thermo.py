"""Thermodynamic-model descriptors: the Python face of ``gpk_thermo_desc``.

The reference plugs constitutive laws into ``GPKGrid`` through virtual
``ThermoModel`` callbacks (include/gpk_core.hpp:72-200) and its subclasses
(include/gpk_thermo.hpp:18-591).  Virtual calls cannot run on the device, so
this package describes a model by a tag plus its scalar parameters; the CUDA
kernels evaluate the same formulas.  The factory functions below take the
same constructor arguments, in the same order, as the reference subclasses.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field, fields
from typing import List

# field ids of include/gpk_b200.h
FIELD_IDS = {
    "phi": 0, "alpha": 1, "c": 2, "T": 3, "g": 4, "rho": 5,
    "nx_f": 6, "ny_f": 7, "nz_f": 8, "kappa_f": 9, "vn_f": 10, "E_el": 11,
    "phi_comp": 12, "g_comp": 13, "mask": 14,
}
INT_FIELDS = {"phi", "phi_comp"}
U8_FIELDS = {"mask"}
REAL_FIELDS = [k for k in FIELD_IDS if k not in INT_FIELDS and k not in U8_FIELDS]

MODEL_IDS = {
    "base": 0, "isotropic": 1, "anisotropic": 2, "solidification": 3,
    "recrystallisation": 4, "dislocation": 5, "ostwald": 6, "tensor_aniso": 7,
    "aniso_ostwald": 8, "precipitation": 9, "grooving": 10, "reduction": 11,
    "magnetic_anneal": 12, "magnetoelastic": 13, "ndfeb": 14,
}
NPARAM = 40
MAX_PHASES = 8


class CThermoDesc(C.Structure):
    """ctypes image of ``gpk_thermo_desc`` (include/gpk_b200.h)."""
    _fields_ = [
        ("model", C.c_int32),
        ("phase_selection", C.c_int32), ("grain_network", C.c_int32), ("stochastic", C.c_int32),
        ("solute_rejection", C.c_int32), ("elastic_enabled", C.c_int32),
        ("elastic_smooth_iters", C.c_int32),
        ("dislocation_enabled", C.c_int32), ("magnetic_enabled", C.c_int32),
        ("sigma0", C.c_float), ("eps4", C.c_float), ("M0", C.c_float), ("Q", C.c_float),
        ("Rgas", C.c_float),
        ("noise_scale", C.c_float), ("kB", C.c_float),
        ("k_partition", C.c_float),
        ("elastic_modulus", C.c_float), ("eigenstrain_coeff", C.c_float), ("c_ref", C.c_float),
        ("disloc_coeff", C.c_float), ("rho_rex", C.c_float), ("recovery_rate", C.c_float),
        ("Ku", C.c_float), ("Ms", C.c_float), ("H_ext", C.c_float), ("H_theta", C.c_float),
        ("g_easy_ref", C.c_float), ("lambda_s", C.c_float),
        ("p", C.c_float * NPARAM),
    ]


@dataclass
class ThermoDesc:
    """ThermoModel fields with the defaults of include/gpk_core.hpp:73-123."""
    model: str = "base"
    sigma0: float = 0.5
    eps4: float = 0.0
    M0: float = 1e-8
    Q: float = 0.0
    Rgas: float = 8.314
    phase_selection: bool = False
    grain_network: bool = False
    stochastic: bool = False
    noise_scale: float = 1.0
    kB: float = 1.380649e-23
    solute_rejection: bool = False
    k_partition: float = 1.0
    elastic_enabled: bool = False
    elastic_modulus: float = 0.0
    eigenstrain_coeff: float = 0.0
    c_ref: float = 0.0
    elastic_smooth_iters: int = 8
    dislocation_enabled: bool = False
    disloc_coeff: float = 0.0
    rho_rex: float = 0.0
    recovery_rate: float = 0.0
    magnetic_enabled: bool = False
    Ku: float = 0.0
    Ms: float = 0.0
    H_ext: float = 0.0
    H_theta: float = 0.0
    g_easy_ref: float = 0.0
    lambda_s: float = 0.0
    p: List[float] = field(default_factory=lambda: [0.0] * NPARAM)

    def to_c(self) -> CThermoDesc:
        d = CThermoDesc()
        for f in fields(self):
            v = getattr(self, f.name)
            if f.name == "model":
                d.model = MODEL_IDS[v]
            elif f.name == "p":
                for i, x in enumerate(v[:NPARAM]):
                    d.p[i] = float(x)
            elif isinstance(v, bool):
                setattr(d, f.name, int(v))
            else:
                setattr(d, f.name, v)
        return d

    def copy(self, **kw) -> "ThermoDesc":
        import copy as _copy
        t = _copy.deepcopy(self)
        for k, v in kw.items():
            setattr(t, k, v)
        return t


def _params(*vals) -> List[float]:
    p = [0.0] * NPARAM
    for i, v in enumerate(vals):
        p[i] = float(v)
    return p


# ---- factories: one per ThermoModel subclass (include/gpk_thermo.hpp) ----
def isotropic(M0, sigma0=0.5) -> ThermoDesc:
    """IsotropicGrowthThermo (include/gpk_thermo.hpp:18-27)."""
    return ThermoDesc("isotropic", M0=M0, sigma0=sigma0, eps4=0.0, grain_network=True)


def anisotropic(M0, sigma0, eps4) -> ThermoDesc:
    """AnisotropicGrowthThermo (include/gpk_thermo.hpp:33-45)."""
    return ThermoDesc("anisotropic", M0=M0, sigma0=sigma0, eps4=eps4, grain_network=True)


def solidification(M0=5e-8, sigma0=0.2, eps4=0.04, m_liq=-500.0, k_part=0.3,
                   T_melt=933.0, L=1e8) -> ThermoDesc:
    """SolidificationThermo (include/gpk_thermo.hpp:52-85)."""
    return ThermoDesc("solidification", M0=M0, sigma0=sigma0, eps4=eps4,
                      p=_params(m_liq, k_part, T_melt, L))


def recrystallisation(M0, sigma0, E_stored) -> ThermoDesc:
    """RecrystallisationThermo (include/gpk_thermo.hpp:90-110)."""
    return ThermoDesc("recrystallisation", M0=M0, sigma0=sigma0, p=_params(E_stored))


def dislocation(M0, sigma0, mu, b, alphaT=0.5, recovery_rate=0.0, rho_rex=0.0) -> ThermoDesc:
    """DislocationThermo (include/gpk_thermo.hpp:135-167)."""
    import numpy as np
    f32 = np.float32
    coeff = float(f32(f32(f32(f32(0.5) * f32(alphaT)) * f32(mu)) * f32(b)) * f32(b))
    return ThermoDesc("dislocation", M0=M0, sigma0=sigma0, dislocation_enabled=True,
                      disloc_coeff=coeff, recovery_rate=recovery_rate, rho_rex=rho_rex,
                      p=_params(mu, b, alphaT))


def ostwald(M0, sigma0, c_sat=0.15, Omega=5e8) -> ThermoDesc:
    """OstwaldThermo (include/gpk_thermo.hpp:172-207)."""
    return ThermoDesc("ostwald", M0=M0, sigma0=sigma0, p=_params(c_sat, Omega))


def tensor_aniso(M0, sigma0, bxx=1.0, byy=1.0, bzz=1.0, dG_bias=0.0) -> ThermoDesc:
    """TensorAnisotropyThermo (include/gpk_thermo.hpp:229-268)."""
    return ThermoDesc("tensor_aniso", M0=M0, sigma0=sigma0, p=_params(bxx, byy, bzz, dG_bias))


def aniso_ostwald(M0, sigma0, bxx, byy, bzz, c_sat, Omega) -> ThermoDesc:
    """AnisoOstwaldThermo (include/gpk_thermo.hpp:284-325)."""
    return ThermoDesc("aniso_ostwald", M0=M0, sigma0=sigma0, p=_params(bxx, byy, bzz, c_sat, Omega))


def precipitation(M0, sigma0, n_phases, a, b, c2, dT, T_ref=900.0) -> ThermoDesc:
    """PrecipitationThermo (include/gpk_thermo.hpp:333-387)."""
    if not (len(a) == len(b) == len(c2) == len(dT) == n_phases):
        raise ValueError("PrecipitationThermo: coefficient size mismatch")
    if n_phases > MAX_PHASES:
        raise ValueError(f"at most {MAX_PHASES} phases are supported on the device")
    p = [0.0] * NPARAM
    p[0], p[1] = float(n_phases), float(T_ref)
    for q in range(n_phases):
        p[2 + q], p[10 + q], p[18 + q], p[26 + q] = a[q], b[q], c2[q], dT[q]
    return ThermoDesc("precipitation", M0=M0, sigma0=sigma0, phase_selection=True, p=p)


def grooving(M0, sigma_gb, sigma_sv) -> ThermoDesc:
    """GroovingThermo (include/gpk_thermo.hpp:399-418)."""
    return ThermoDesc("grooving", M0=M0, sigma0=sigma_gb, p=_params(sigma_gb, sigma_sv))


def reduction(M0, sigma0, pH2_over_pH2O, dG0_J_per_mol, V_molar_metal) -> ThermoDesc:
    """ReductionThermo (include/gpk_thermo.hpp:431-463)."""
    return ThermoDesc("reduction", M0=M0, sigma0=sigma0,
                      p=_params(pH2_over_pH2O, dG0_J_per_mol, V_molar_metal))


def magnetic_anneal(M0, sigma0, Ku, Ms, H_ext, H_theta, g_easy_ref=0.0) -> ThermoDesc:
    """MagneticAnnealingThermo (include/gpk_thermo.hpp:472-495)."""
    return ThermoDesc("magnetic_anneal", M0=M0, sigma0=sigma0, magnetic_enabled=True,
                      Ku=Ku, Ms=Ms, H_ext=H_ext, H_theta=H_theta, g_easy_ref=g_easy_ref)


def magnetoelastic(M0, sigma0, elastic_modulus, lambda_s, H_theta, H_ext=0.0, Ku=0.0, Ms=0.0) -> ThermoDesc:
    """MagnetoelasticThermo (include/gpk_thermo.hpp:508-537)."""
    t = ThermoDesc("magnetoelastic", M0=M0, sigma0=sigma0, elastic_enabled=True,
                   elastic_modulus=elastic_modulus, eigenstrain_coeff=0.0, c_ref=0.0,
                   lambda_s=lambda_s, H_theta=H_theta)
    if Ku != 0.0 or Ms != 0.0:
        t.magnetic_enabled, t.Ku, t.Ms, t.H_ext = True, Ku, Ms, H_ext
    return t


def ndfeb(M0, sigma_gb, sigma_gbphase_0, k_Cu, c_sat, Omega) -> ThermoDesc:
    """NdFeBGrainBoundaryThermo (include/gpk_thermo.hpp:548-589)."""
    return ThermoDesc("ndfeb", M0=M0, sigma0=sigma_gb,
                      p=_params(sigma_gb, sigma_gbphase_0, k_Cu, c_sat, Omega))
