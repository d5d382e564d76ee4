"""Transport systems in the form the reference's transport modules hand to
solve(): salinity (n=5) and one class of suspended sediment (n=4).

Test fixtures for the solve boundary, assembled on the host from a flow state
(flux, visk, hk, iwet, depths) as the reference assembles them:

- convection schemes: schemes/comp_lib.f90:54-109 (upwindcoef, hybridcoef,
  powerlawcoef, exponentialcoef);
- salinity: salinity/salinity.F90:713-768 (coeffsourcesink_sal, first-order
  time scheme ntsch=1), salinity/sal_bnd.f90:197-268 (bound_sal: dry rows,
  inflow/outflow at the boundary string), salinity/salinity.F90:575-620
  (sal_imp: su reset from susal0 before every solve, exit once
  rmom(5) < tolsal after more than 5 iterations, dry cells restored);
- sediment: sediment/sed_imp.f90:436-545 (coeffsourcesink_c with ntsch=1, the
  total-load correction factor btk=1 and the mixing-layer fraction rsk=1),
  sed_imp.f90:230-236 (solve, then the concentration is bounded to
  [0, Cteqmax]).

Arrays follow the solve() layout: acoef (ncellsD, nmaxfaces), cell arrays of
ncellsD values, cell2cell 1-based.
"""
from __future__ import annotations

import numpy as np


def upwindcoef(dk, fk):
    return dk + np.maximum(0.0, -fk)


def hybridcoef(dk, fk):
    peck = np.abs(fk) / np.maximum(dk, 1e-6)
    return dk * np.maximum(0.0, 1.0 - 0.5 * peck) + np.maximum(0.0, -fk)


def powerlawcoef(dk, fk):
    absfk = np.abs(fk)
    peck = absfk / np.maximum(np.maximum(dk, absfk), 1e-6)
    return dk * (1.0 - peck ** 5) + np.maximum(0.0, -fk)


def exponentialcoef(dk, fk):
    # With fk = 0 this is 0, not dk: peck = 0 and the denominator is the 1e-6 floor.
    absfk = np.abs(fk)
    peck = absfk / np.maximum(np.maximum(dk, 1e-6), absfk)
    return dk * peck / np.maximum(np.exp(peck) - 1.0, 1e-6) + np.maximum(0.0, -fk)


SCHEMES = {"upwind": upwindcoef, "hybrid": hybridcoef, "powerlaw": powerlawcoef, "exponential": exponentialcoef}


def flow_state(fl, h1):
    """The fields a transport assembly reads, from a FlowOracle after a step;
    h1 is the depth at the start of that step."""
    return {"flux": fl.get("flux"), "visk": fl.get("visk"), "hk": fl.get("hk"), "dsxy": fl.get("dsxy"),
            "areap": fl.get("areap"), "iwet": fl.get("iwet").astype(np.int32), "h": fl.get("h"),
            "h1": np.asarray(h1, np.float64)}


def _faces(g):
    n = g.ncells
    kmask = np.arange(g.nmaxfaces)[None, :] < g.ncface[:n, None]
    nb = np.where(kmask, g.cell2cell[:n], 1).astype(np.int64) - 1  # 0-based neighbour (valid where kmask)
    return kmask, nb


def _dry_rows(g, st, acoef, sp, su0):
    """Rows of dry cells average their wet neighbours (all neighbours when none
    is wet); ghosts drop out; no source and no time term."""
    n = g.ncells
    kmask, nb = _faces(g)
    iwet = st["iwet"]
    inb = iwet[nb] * kmask
    dry = iwet[:n] == 0
    idrym = (inb * (nb < n)).sum(axis=1)
    rows = np.where((idrym >= 1)[:, None], inb.astype(np.float64), st["dsxy"][:n])
    rows = np.where(kmask & (nb < n), rows, 0.0)
    acoef[:n][dry] = rows[dry]
    sp[:n][dry] = 0.0
    su0[:n][dry] = 0.0


def salinity_system(g, st, sal, sal1, dt, scheme="exponential", schmidt=1.0, str_cells=(), str_faces=(),
                    salbnd=35.0, ramp=1.0, salbnd0=None):
    """acoef, susal0, sp of one salinity solve; sets the ghost salinity of the
    boundary string in sal (inflow: the boundary value; outflow: the cell's)."""
    n, nmf = g.ncells, g.nmaxfaces
    schm = SCHEMES[scheme]
    kmask, nb = _faces(g)
    iwet = st["iwet"]
    acoef = np.zeros((g.ncellsD, nmf))
    sp = np.zeros(g.ncellsD)
    su0 = np.zeros(g.ncellsD)
    fac1 = iwet[:n] * st["areap"][:n] * st["h1"][:n] / dt
    sp[:n] = -fac1
    su0[:n] = fac1 * sal1[:n]
    ddk = st["visk"][:n] * st["hk"][:n] * st["dsxy"][:n] / schmidt
    acoef[:n] = np.where(kmask, schm(ddk, st["flux"][:n]), 0.0)
    # bound_sal: wet rows lose their dry faces, dry rows average
    wet = iwet[:n] == 1
    acoef[:n][wet] = (acoef[:n] * np.where(kmask, iwet[nb], 0))[wet]
    _dry_rows(g, st, acoef, sp, su0)
    if salbnd0 is None:
        salbnd0 = np.full(len(str_cells), salbnd)
    for j, (c, k) in enumerate(zip(str_cells, str_faces)):
        i, kk = int(c) - 1, int(k) - 1
        nck = int(g.cell2cell[i, kk]) - 1
        if st["flux"][i, kk] < 0.0:  # inflow
            sal[nck] = ramp * salbnd + (1.0 - ramp) * salbnd0[j]
            su0[i] += acoef[i, kk] * sal[nck]
            sp[i] -= acoef[i, kk]
        else:
            sal[nck] = sal[i]
        acoef[i, kk] = 0.0
    return acoef, su0, sp


def sediment_system(g, st, ctk, ctk1, dt, ctkstar, alphat, wsfall, scheme="exponential"):
    """acoef, su, sp of one suspended-sediment solve (one size class). Wet cells
    next to a dry one copy their concentration into it (as the assembly does)."""
    n, nmf = g.ncells, g.nmaxfaces
    schm = SCHEMES[scheme]
    kmask, nb = _faces(g)
    iwet = st["iwet"]
    acoef = np.zeros((g.ncellsD, nmf))
    sp = np.zeros(g.ncellsD)
    su = np.zeros(g.ncellsD)
    a0 = iwet[:n] * st["areap"][:n] / dt
    su[:n] = a0 * st["h1"][:n] * ctk1[:n]
    sp[:n] = -a0 * st["h1"][:n]
    aws = st["areap"][:n] * alphat[:n] * wsfall
    su[:n] += aws * ctkstar[:n]
    sp[:n] -= aws
    ddk = st["visk"][:n] * st["hk"][:n] * st["dsxy"][:n]
    acoef[:n] = np.where(kmask, schm(ddk, st["flux"][:n]), 0.0)
    for i in np.nonzero(iwet[:n] == 1)[0]:
        for k in range(int(g.ncface[i])):
            nck = int(nb[i, k])
            if iwet[nck] == 0:
                ctk[nck] = ctk[i]
                acoef[i, k] = 0.0
    _dry_rows(g, st, acoef, sp, su)
    return acoef, su, sp
