"""Named solve settings (mesh, physics constants, integrator, seeded initial state).

``surface32``  6 panels x 32^2 zones x 1 radial zone, 3 ghost layers, FP64,
               SSP-RK3, CFL 0.4: the CPU-runnable surface case (density
               1 + 0.1 Y from a seeded harmonic sum of degree <= 4, p = 1,
               solid-body rotation 0.5, vector potential amplitude 0.1).
``shell128``   6 x 128^2 x 64, r in [1, 2] with geometric radial stretch 1.02,
               4 ghost layers, FP64: hydrostatic 1/r^2 shell with seeded density
               and field perturbations of amplitude 0.05 under point-mass
               gravity, IMEX-RK2 (ARS(2,2,2), gravity implicit).
``shell256``   the same shell at 6 x 256^2 x 128 zones: the workload of the
               precision form's 200-step error statement.
``shell16`` / ``shell32``  the same shell at test sizes.
"""
from __future__ import annotations

PRESETS = {
    "surface32": dict(
        params=dict(ntp=32, nr=1, nghost=3, radial_mesh="uniform", rmin=1.0, rmax=1.05, gamma=5.0 / 3.0,
                    cfl_coef=0.4, rk_scheme=3, gm=0.0),
        init=dict(seed=2024, kind=0, lmax=4, rho_amp=0.1, a_amp=0.1, v_amp=0.5, p0=1.0),
        steps=100,
    ),
    "shell128": dict(
        params=dict(ntp=128, nr=64, nghost=4, radial_mesh="stretched", radial_ratio=1.02, rmin=1.0, rmax=2.0,
                    gamma=5.0 / 3.0, cfl_coef=0.4, rk_scheme=4, gm=1.0),
        init=dict(seed=2025, kind=1, lmax=4, rho_amp=0.05, a_amp=0.05, v_amp=0.0, p0=0.05),
        steps=50,
    ),
    "shell256": dict(
        params=dict(ntp=256, nr=128, nghost=4, radial_mesh="stretched", radial_ratio=1.02, rmin=1.0, rmax=2.0,
                    gamma=5.0 / 3.0, cfl_coef=0.4, rk_scheme=4, gm=1.0),
        init=dict(seed=2025, kind=1, lmax=4, rho_amp=0.05, a_amp=0.05, v_amp=0.0, p0=0.05),
        steps=200,
    ),
    "shell32": dict(
        params=dict(ntp=32, nr=16, nghost=4, radial_mesh="stretched", radial_ratio=1.02, rmin=1.0, rmax=2.0,
                    gamma=5.0 / 3.0, cfl_coef=0.4, rk_scheme=4, gm=1.0),
        init=dict(seed=2025, kind=1, lmax=4, rho_amp=0.05, a_amp=0.05, v_amp=0.0, p0=0.05),
        steps=10,
    ),
    "shell16": dict(
        params=dict(ntp=16, nr=8, nghost=4, radial_mesh="stretched", radial_ratio=1.02, rmin=1.0, rmax=2.0,
                    gamma=5.0 / 3.0, cfl_coef=0.4, rk_scheme=4, gm=1.0),
        init=dict(seed=2025, kind=1, lmax=4, rho_amp=0.05, a_amp=0.05, v_amp=0.0, p0=0.05),
        steps=4,
    ),
}


def preset(name: str) -> dict:
    p = PRESETS[name]
    return {"params": dict(p["params"]), "init": dict(p["init"]), "steps": p["steps"]}
