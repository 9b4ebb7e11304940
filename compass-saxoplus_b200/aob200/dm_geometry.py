"""Piezo-stack DM geometry with Gaussian influence functions (host side, once).

Restates the reference's square-pattern Gaussian DM set-up:
  shesha/shesha/init/dm_init.py      _dm_init :104-160, make_pzt_dm :453-625
  shesha/shesha/util/dm_util.py      dim_dm_support :32-50, createSquarePattern :93-112,
                                     select_actuators :240-298
  shesha/shesha/util/influ_util.py   makeGaussian :300-339
The output (influence cube, patch origins i1/j1, DM screen size) is what the
reference hands to SutraDm::pzt_loadarrays and what aob_dm_create takes.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


def gaussian_support(pitch: float, coupling: float) -> int:
    irc = 1.16136 + 2.97422 * coupling + (-13.2381) * coupling**2 + 20.4395 * coupling**3
    s = int(np.ceil(2 * irc * pitch + 10))
    return s + (s % 2)


def gaussian_influence(pitch: float, coupling: float, x, y):
    sig = pitch / np.sqrt(-2 * np.log(coupling))
    return np.exp(-0.5 * ((x / sig) ** 2 + (y / sig) ** 2))


def square_pattern(pitch: float, nxact: int):
    g = np.tile(np.arange(nxact) - (nxact - 1.0) / 2.0, (nxact, 1)).astype(np.float32)
    return np.float32(np.array([g.flatten(), g.T.flatten()]) * pitch)


def select_actuators(xc, yc, nxact, pitch, cobs, margin_in=0.0, margin_out=None):
    dis = np.sqrt(xc**2 + yc**2)
    rad_in = (((nxact - 1) / 2) * cobs - margin_in) * pitch
    if margin_out is None:
        margin_out = 1.44
    rad_out = ((nxact - 1.0) / 2.0 + margin_out) * pitch
    return np.where((dis <= rad_out) * (dis >= rad_in))[0]


@dataclass
class DmGeometry:
    nact: int
    pitch: float
    n1: int
    n2: int
    dim: int
    influsize: int
    xpos: np.ndarray
    ypos: np.ndarray
    i1: np.ndarray
    j1: np.ndarray
    influ: np.ndarray

    @property
    def ntotact(self) -> int:
        return int(self.xpos.size)


def pzt_dm_geometry(nact: int, pupdiam: int, cent: float, ssize: int, n_mpupil: int, cobs: float,
                    coupling: float = 0.3, unitpervolt: float = 1.0, margin_out=None, pzt_extent: float = 5.0):
    """Square-pattern Gaussian DM conjugated to the pupil (altitude 0, on-axis sensors)."""
    pitch = pupdiam / float(nact - 1)
    extent = pitch * (nact + pzt_extent)
    n1 = np.floor(cent - extent / 2)
    n2 = np.ceil(cent + extent / 2)
    n1 = int(max(n1, 1))
    n2 = int(min(n2, ssize))
    ss = gaussian_support(pitch, coupling)
    xy = square_pattern(pitch, nact + 4)
    valid = select_actuators(xy[0, :], xy[1, :], nact, pitch, np.float32(cobs), 0.0,
                             None if margin_out is None else np.float32(margin_out))
    xy = xy + cent
    xy = xy[:, valid]
    xpos, ypos = xy[0, :], xy[1, :]
    i1 = (xpos - ss / 2 - 0.5 - n1).astype(np.int32)
    j1 = (ypos - ss / 2 - 0.5 - n1).astype(np.int32)
    influ = np.zeros((ss, ss, xpos.size), dtype=np.float32)
    for a in range(xpos.size):
        x = np.tile(np.arange(i1[a], i1[a] + ss, dtype=np.float32), (ss, 1)).T
        x += n1
        x -= xpos[a]
        y = np.tile(np.arange(j1[a], j1[a] + ss, dtype=np.float32), (ss, 1))
        y += n1
        y -= ypos[a]
        influ[:, :, a] = gaussian_influence(pitch, coupling, x, y)
    influ = influ * float(unitpervolt / np.max(influ))
    dim = max(n2 - n1 + 1, n_mpupil)
    return DmGeometry(nact, pitch, n1, n2, dim, ss, xpos, ypos, i1, j1, influ)
