"""Network description consumed by the batched GGA solver.

`Net` mirrors the field names and meaning of the reference network object
(dgga/parse.py:206-310) so that a network parsed by the reference can be
handed to this package unchanged, and a network built here can be handed to
the reference.  Everything is stored in EPANET's internal units: lengths and
heads in ft, flows in cfs (dgga/CONTRACT.md:15-20).

Only the fields the hot path reads are required; the B2 extension fields
(tanks, pumps, controls) default to empty arrays exactly as the reference's
`__post_init__` does (dgga/parse.py:271-296).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

# EPANET link types (epanet2_enums.h order, as used by dgga/parse.py:64-75)
CVPIPE, PIPE, PUMP, PRV, PSV, PBV, FCV, TCV, GPV = range(9)
# node types (dgga/parse.py:212)
JUNCTION, RESERVOIR, TANK = 0, 1, 2
# pump curve kinds (dgga/parse.py:51-54)
CONST_HP, POWER_FUNC, CUSTOM, NOCURVE = 0, 1, 2, 3

# EPANET unit constants (types.h values as listed in dgga/units.py:12-27)
MperFT = 0.3048
LPSperCFS = 28.317
PSIperFT = 0.4333

_META_DEFAULTS = {
    "extra_iter": -1,
    "checkfreq": 2,
    "maxcheck": 10,
    "damp_limit": 0.0,
    "tstart_sec": 0,
    "report_step_sec": 3600,
    "report_start_sec": 0,
    "spgrav": 1.0,
    "press_units": "",
    "rule_step_sec": 0,
    "viscosity": 1.1e-5,
}

_EMPTY = {
    "tank_node": np.int32, "tank_h0": np.float64, "tank_hmin": np.float64,
    "tank_hmax": np.float64, "tank_area": np.float64, "tank_vmin": np.float64,
    "tank_v0": np.float64, "tank_vmax": np.float64, "tank_overflow": np.int8,
    "pump_link": np.int32, "pump_ptype": np.int8, "pump_h0": np.float64,
    "pump_r": np.float64, "pump_n": np.float64, "pump_q0": np.float64,
    "pump_qmax": np.float64, "pump_hmax": np.float64, "pump_upat": np.int32,
    "pump_curve_q": np.float64, "pump_curve_h": np.float64,
    "pump_curve_ptr": np.int32,
    "ctl_link": np.int32, "ctl_node": np.int32, "ctl_type": np.int8,
    "ctl_status": np.int8, "ctl_setting": np.float64, "ctl_grade": np.float64,
    "ctl_time": np.int64,
}


@dataclass
class Net:
    """Water network in EPANET internal units (ft, cfs), file order, 0-based."""

    node_id: list
    node_type: np.ndarray          # int8[N] 0 junction, 1 reservoir, 2 tank
    elev_ft: np.ndarray            # float64[N] (reservoir: fixed head)
    node_ke: np.ndarray            # float64[N] internal emitter coefficient
    res_head_pat: np.ndarray       # int32[N]
    link_id: list
    link_type: np.ndarray          # int8[L] EN link type
    link_n1: np.ndarray            # int32[L]
    link_n2: np.ndarray            # int32[L]
    diam_ft: np.ndarray            # float64[L]
    len_ft: np.ndarray             # float64[L]
    roughness: np.ndarray          # float64[L] Hazen-Williams C
    km_int: np.ndarray             # float64[L] 0.02517*K/D^4
    r_hw: np.ndarray               # float64[L] 4.727*L/C^1.852/D^4.871
    init_status: np.ndarray        # int8[L] 0 closed, 1 open, 2 active
    valve_setting_user: np.ndarray  # float64[L] user-unit setting; pumps: speed
    dem_node: np.ndarray           # int32[K]
    dem_base_cfs: np.ndarray       # float64[K]
    dem_pat: np.ndarray            # int32[K]
    pattern_ids: list
    patterns: list
    meta: dict
    controls_raw: list = field(default_factory=list)
    rules_raw: list = field(default_factory=list)
    tank_node: np.ndarray = None
    tank_h0: np.ndarray = None
    tank_hmin: np.ndarray = None
    tank_hmax: np.ndarray = None
    tank_area: np.ndarray = None
    tank_vmin: np.ndarray = None
    tank_v0: np.ndarray = None
    tank_vmax: np.ndarray = None
    tank_overflow: np.ndarray = None
    pump_link: np.ndarray = None
    pump_ptype: np.ndarray = None
    pump_h0: np.ndarray = None
    pump_r: np.ndarray = None
    pump_n: np.ndarray = None
    pump_q0: np.ndarray = None
    pump_qmax: np.ndarray = None
    pump_hmax: np.ndarray = None
    pump_upat: np.ndarray = None
    pump_curve_q: np.ndarray = None
    pump_curve_h: np.ndarray = None
    pump_curve_ptr: np.ndarray = None
    ctl_link: np.ndarray = None
    ctl_node: np.ndarray = None
    ctl_type: np.ndarray = None
    ctl_status: np.ndarray = None
    ctl_setting: np.ndarray = None
    ctl_grade: np.ndarray = None
    ctl_time: np.ndarray = None

    def __post_init__(self):
        for k, dt in _EMPTY.items():
            if getattr(self, k) is None:
                setattr(self, k, np.zeros(0, dtype=dt))
        for k, v in _META_DEFAULTS.items():
            self.meta.setdefault(k, v)

    @property
    def N(self) -> int:
        return len(self.node_id)

    @property
    def L(self) -> int:
        return len(self.link_id)

    # Pattern lookup: stair-step, no interpolation (dgga/parse.py:300-335).
    def _factors_at(self, t_sec):
        npat = len(self.patterns)
        fac = np.ones(npat + 1, dtype=np.float64)
        start = float(self.meta.get("pat_start_sec", 0))
        step = float(self.meta.get("pat_step_sec", 3600)) or 3600.0
        for i, pat in enumerate(self.patterns):
            pat = np.asarray(pat, dtype=np.float64)
            if pat.size:
                fac[i] = pat[int((t_sec + start) // step) % pat.size]
        return fac

    def demand_cfs_at(self, t_sec=0):
        """Nominal demand float64[N] (cfs) at time t: sum of categories times
        pattern factor times the global demand multiplier."""
        out = np.zeros(self.N, dtype=np.float64)
        if np.asarray(self.dem_node).size == 0:
            return out
        fac = self._factors_at(t_sec)
        pat = np.asarray(self.dem_pat)
        idx = np.where(pat < 0, len(self.patterns), pat)
        w = np.asarray(self.dem_base_cfs) * fac[idx] * float(
            self.meta.get("demand_multiplier", 1.0))
        return np.bincount(np.asarray(self.dem_node), weights=w,
                           minlength=self.N).astype(np.float64)

    def reservoir_head_ft_at(self, t_sec=0):
        """Reservoir heads float64[N] (ft); nan at every other node, tanks
        included (same contract as the reference)."""
        out = np.full(self.N, np.nan, dtype=np.float64)
        fac = self._factors_at(t_sec)
        nt = np.asarray(self.node_type)
        for i in np.flatnonzero(nt == RESERVOIR):
            p = int(self.res_head_pat[i])
            out[i] = self.elev_ft[i] * (fac[p] if p >= 0 else 1.0)
        return out

    def fixed_head_ft_at(self, t_sec=0):
        """Reservoir heads plus tank initial heads (a tank is a fixed head
        inside one steady solve); nan at junctions."""
        out = self.reservoir_head_ft_at(t_sec)
        tn = np.asarray(self.tank_node)
        if tn.size:
            out[tn] = np.asarray(self.tank_h0)
        return out

    def as_fields(self) -> dict:
        """Plain dict of every dataclass field (used to rebuild the network as
        another package's network object with the same field names)."""
        from dataclasses import fields
        return {f.name: getattr(self, f.name) for f in fields(self)}
