"""Algorithmic byte model of the RK3 dycore step (float64).

Whole step (the reporting denominator): one cell-substep moves
``B_SUB = 336`` bytes (42 float64 arrays: 10 evolving arrays read and written
-- u, v, w, ph, t_2, t_2ave, p, pm1, al, ww -- and 22 stage-constant reads);
one RK stage moves ``B_STAGE`` = 328 (dry) / 472 (moist) bytes per cell and
the carry 72 bytes per cell per step, so a step moves
``cells * (3*B_STAGE + n_sub*B_SUB + B_CARRY)`` bytes with
``n_sub = 1 + ns//2 + ns`` substeps.

Per kernel (each logically touched array counted once per launch, halo
re-reads excluded):

* ``k_column`` -- advance_mu_t + advance_w + calc_p_rho on one column: reads
  dvdxi, theta flux divergence, theta_1, t_2, t_tend, ww_1, w, ph, ph_1+phb,
  ph_tend, c2a, alt, cqw, rw_tend, a, alpha, gamma, t_2ave, pm1 (19) [+ w_save
  with damp_opt 3], writes t_2, ww, w, ph, t_2ave, p, pm1, al (8): 216 (224)
  B/cell.
* ``k_advance_uv`` -- advance_uv on the u and v faces: per face reads u (v),
  u_tend (v_tend), cqu (cqv) and writes u (v): 32 B/face; per cell reads the
  mass-point planes ph, p, alt, al, pb, php once: 48 B/cell.
* ``k_div_h`` -- the column-coupling horizontal divergences: reads u, v, u_1,
  v_1, theta_1 (5), writes dvdxi and the theta flux divergence (2): 56 B/cell.
"""

from __future__ import annotations

B_SUB = 336
B_STAGE_DRY = 328
B_STAGE_MOIST = 472
B_CARRY = 72


def substeps_per_step(ns: int) -> int:
    return 1 + max(1, ns // 2) + ns


def step_bytes(nx: int, ny: int, nz: int, ns: int, moist: bool) -> float:
    cells = nx * ny * nz
    b_stage = B_STAGE_MOIST if moist else B_STAGE_DRY
    return float(cells) * (3 * b_stage + substeps_per_step(ns) * B_SUB + B_CARRY)


def kernel_bytes_per_launch(name: str, nx: int, ny: int, nz: int, damp_opt: int = 0) -> float | None:
    cells = nx * ny * nz
    if name == "k_column":
        return float(cells) * (224 if damp_opt == 3 else 216)
    if name == "k_advance_uv":
        faces = nz * ny * (nx + 1) + nz * (ny + 1) * nx
        return float(faces) * 32 + float(cells) * 48
    if name == "k_div_h":
        return float(cells) * 56
    return None
