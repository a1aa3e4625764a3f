"""Algorithmic (compulsory) HBM bytes of each kernel of one step.

Every particle's own inputs are read once and its outputs written once at
their natural sizes (vector 12 B, float 4 B, phase/flags 1 B, id/key 4 B);
neighbour re-reads are assumed to be served on chip (cell-sorted order).  The
counts follow the fields each kernel reads and writes for the configuration
of the run (SolverConfig switches).  `kernel_bytes` returns bytes per launch.
"""
from __future__ import annotations

import math


def _flags(cfg):
    g = lambda k, d=0: getattr(cfg, k) if hasattr(cfg, k) else cfg.get(k, d)  # noqa: E731
    cont = int(g("density_mode")) == 1
    tvf = bool(g("transport_velocity", 1))
    return dict(
        cont=cont,
        tvf=tvf,
        thermal=bool(g("thermal", 1)),
        pc=bool(g("phase_change", 1)),
        st=int(g("surface_tension", 1)),
        wet=int(g("wetting_model", 0)),
        sps=bool(g("sps_turbulence", 0)),
        stress=bool(g("transport_stress", 0)),
    )


def per_particle(kernel: str, cfg, has_vapor: bool):
    """(fluid bytes, wall bytes) per particle for one launch of `kernel`."""
    f = _flags(cfg)
    csf = f["st"] == 1 and has_vapor
    if kernel == "k_kick_drift_keys":
        fl = 12 + 1 + 12 + 12 + 12 + 12 + 12 + 12 + 4 + (8 + 4 if f["cont"] else 0)
        return fl, 12 + 1 + 4
    if kernel == "k_gather":
        return 2 * 70 + 4, 2 * 70 + 4
    if kernel == "k_density":
        return 12 + 1 + 4 + 4 + 16, 1 + 8
    if kernel == "k_wall":
        return 1, 12 + 1 + 4 * 4 + 12 + 12
    if kernel == "k_interface":
        return 12 + 1 + 4 * 3 + 12 + 12 + (12 if csf else 0), 1
    if kernel == "k_forces":
        rd = 12 + 1 + 12 + 4 * 6 + 4  # x phase v | T m rho p sigma alpha | rmin
        if f["stress"] or (f["cont"] and f["tvf"]):
            rd += 12
        if csf:
            rd += 12 + (12 if f["wet"] else 0)
        if f["thermal"]:
            rd += 4
        wr = 4 * 12 + (4 if csf else 0) + (4 if f["cont"] else 0) + (4 if f["thermal"] else 0)
        wall = 1 + 4 * 12 + (4 if f["cont"] else 0) + (4 if f["thermal"] else 0)
        return rd + wr, wall
    if kernel == "k_kick":
        fl = 1 + 12 + 12 + 12 + (12 if f["thermal"] else 0)
        if f["pc"]:
            fl += 4 + 4 + 13
        return fl, 1 + (13 if f["pc"] else 0)
    if kernel == "k_saturation":
        return 9, 1
    if kernel == "k_rs_upsweep":
        return 4, 4
    if kernel == "k_rs_downsweep":
        return 16, 16
    if kernel == "k_cells":
        return 4, 4
    return 0, 0


def kernel_bytes(kernel: str, cfg, n_fluid: int, n_wall: int, has_vapor: bool, num_cells: int = 0) -> float:
    fl, wl = per_particle(kernel, cfg, has_vapor)
    extra = 4 * (num_cells + 1) if kernel == "k_cells" else 0
    return float(fl * n_fluid + wl * n_wall + extra)


def sort_passes(num_cells: int) -> int:
    bits = max(1, int(math.ceil(math.log2(num_cells + 1))))
    return (bits + 7) // 8
