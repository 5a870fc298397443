"""Seeded synthetic water networks with the shapes of the benchmark workloads.

The public benchmark networks (L-TOWN and friends) are not available offline,
so every workload here is generated from a seed:

* `looped_network`  -- planar looped graph: jittered grid points, Delaunay
  triangulation, Euclidean minimum spanning tree, then a seeded set of chords.
  Optional pressure-reducing valves are placed on tree edges that feed a
  whole subtree ("pressure zone"), with no chord crossing the zone boundary,
  so that each PRV is its zone's only feed.  Pipes are sized from the tree
  flow of the base demand so that velocities stay near 1 m/s.
* `config1_network` -- 31 junctions, 1 reservoir at 100 m, 34 pipes
  (random spanning tree plus 3 chords), C in 80-140, D from a fixed set,
  lengths 100-3500 m, demands 0-0.4 m3/s.
* `config2_network` -- 782 junctions, 905 pipes, 3 PRVs (settings 30-50 m),
  2 reservoirs (80-120 m), about 12 % chords, 20 emitters.
* `config2_scenarios` -- per-scenario demand = base * lognormal(sigma=0.2).

Every quantity is converted to EPANET internal units (ft, cfs) with the same
conversion chain the reference parser uses: r = 4.727 L / C^1.852 / D^4.871
(dgga/parse.py:603), emitter Ke = (Ucf_flow^qexp / Ucf_pressure) / C^qexp
(dgga/parse.py:568), PRV setting stored in user pressure units (m).
"""
from __future__ import annotations

import numpy as np

from .net import (JUNCTION, RESERVOIR, TANK, PIPE, PRV, PSV, PUMP, TCV, FCV,
                  LPSperCFS, MperFT, Net)

_M3S_PER_CFS = LPSperCFS / 1000.0        # 0.028317 m3/s per cfs


def _meta(**over):
    meta = dict(flow_units="LPS", headloss="H-W", trials=200, accuracy=0.001,
                demand_model="DDA", emitter_exponent=0.5, qexp=2.0,
                duration_sec=0, hyd_step_sec=3600, pat_step_sec=3600,
                pat_start_sec=0, demand_multiplier=1.0)
    meta.update(over)
    return meta


def _r_hw(len_ft, c, d_ft):
    """Hazen-Williams resistance in internal units, reference operation order."""
    out = np.zeros_like(len_ft)
    for k in range(len_ft.size):
        if c[k] > 0 and d_ft[k] > 0 and len_ft[k] > 0:
            out[k] = 4.727 * len_ft[k] / (c[k] ** 1.852) / (d_ft[k] ** 4.871)
    return out


def emitter_ke(c_m3s, qexp=2.0, ucf_flow=LPSperCFS, ucf_pressure=MperFT):
    """Internal emitter coefficient from a user coefficient given in m3/s per
    m^(1/qexp) (converted to L/s, the LPS flow unit)."""
    c_user = np.asarray(c_m3s, dtype=np.float64) * 1000.0
    out = np.zeros_like(c_user)
    pos = c_user > 0
    out[pos] = (ucf_flow ** qexp / ucf_pressure) / c_user[pos] ** qexp
    return out


def _delaunay_edges(pts):
    from scipy.spatial import Delaunay
    tri = Delaunay(pts)
    e = set()
    for s in tri.simplices:
        for a, b in ((s[0], s[1]), (s[1], s[2]), (s[0], s[2])):
            e.add((min(a, b), max(a, b)))
    return np.array(sorted(e), dtype=np.int64)


def _spanning_tree(n, edges, weights):
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import minimum_spanning_tree
    w = coo_matrix((weights, (edges[:, 0], edges[:, 1])), shape=(n, n))
    t = minimum_spanning_tree(w).tocoo()
    te = np.stack([np.minimum(t.row, t.col), np.maximum(t.row, t.col)], 1)
    return te[np.lexsort((te[:, 1], te[:, 0]))]


def _root_tree(n, tree_edges, root):
    """parent[] and BFS order of the tree rooted at `root`."""
    adj = [[] for _ in range(n)]
    for a, b in tree_edges:
        adj[a].append(b)
        adj[b].append(a)
    parent = np.full(n, -1, dtype=np.int64)
    order = [root]
    seen = np.zeros(n, dtype=bool)
    seen[root] = True
    i = 0
    while i < len(order):
        u = order[i]
        i += 1
        for v in adj[u]:
            if not seen[v]:
                seen[v] = True
                parent[v] = u
                order.append(v)
    return parent, np.array(order, dtype=np.int64)


def looped_network(seed, n_junc, n_res, n_pipes, n_prv=0, res_head_m=(80, 120),
                   spacing_m=180.0, elev_m=(0.0, 40.0), base_lps=(0.2, 1.5),
                   c_range=(90.0, 140.0), n_emitters=0, emitter_c=(0.0, 1e-3),
                   prv_setting_m=(30.0, 50.0), zone_size=(25, 70),
                   diam_set_m=(0.1, 0.15, 0.2, 0.25, 0.3, 0.4, 0.5, 0.6, 0.75,
                               0.9, 1.0, 1.2), vmax=0.9):
    rng = np.random.default_rng(seed)
    N = n_junc + n_res
    side = int(np.ceil(np.sqrt(N)))
    gx, gy = np.meshgrid(np.arange(side), np.arange(side))
    grid = np.stack([gx.ravel(), gy.ravel()], 1)[:N].astype(np.float64)
    pts = (grid + rng.uniform(-0.35, 0.35, size=grid.shape)) * spacing_m
    edges = _delaunay_edges(pts)
    elen = np.linalg.norm(pts[edges[:, 0]] - pts[edges[:, 1]], axis=1)
    # drop the long hull edges Delaunay adds on the boundary
    keep = elen < 2.2 * spacing_m
    edges, elen = edges[keep], elen[keep]
    tree = _spanning_tree(N, edges, elen)
    # reservoirs: nodes nearest to opposite corners, heads high on one side
    corners = np.array([[0, 0], [side, side], [0, side], [side, 0]],
                       dtype=np.float64) * spacing_m
    res_nodes = []
    for c in corners[:n_res]:
        d = np.linalg.norm(pts - c, axis=1)
        d[res_nodes] = np.inf
        res_nodes.append(int(np.argmin(d)))
    res_nodes = np.array(res_nodes, dtype=np.int64)
    node_type = np.zeros(N, dtype=np.int8)
    node_type[res_nodes] = RESERVOIR
    # smooth elevation field, in m
    cx, cy = rng.uniform(0, side * spacing_m, 2)
    r2 = ((pts[:, 0] - cx) ** 2 + (pts[:, 1] - cy) ** 2) / (side * spacing_m) ** 2
    el = elev_m[0] + (elev_m[1] - elev_m[0]) * (
        0.5 + 0.35 * np.sin(2.5 * pts[:, 0] / (side * spacing_m) + rng.uniform(0, 6))
        * np.cos(1.7 * pts[:, 1] / (side * spacing_m)) - 0.3 * r2)
    el = np.clip(el, elev_m[0], elev_m[1])
    base = np.where(node_type == JUNCTION, rng.uniform(*base_lps, N), 0.0)  # L/s
    parent, order = _root_tree(N, tree, int(res_nodes[0]))
    # subtree demand and size
    sub_q = base.copy()
    sub_n = (node_type == JUNCTION).astype(np.int64)
    for v in order[::-1]:
        p = parent[v]
        if p >= 0:
            sub_q[p] += sub_q[v]
            sub_n[p] += sub_n[v]
    # PRV zones: disjoint subtrees fed only by their root edge
    zone = np.full(N, -1, dtype=np.int64)
    prv_edges = []
    if n_prv:
        cand = [v for v in order[1:]
                if zone_size[0] <= sub_n[v] <= zone_size[1]
                and node_type[v] == JUNCTION and node_type[parent[v]] == JUNCTION]
        rng.shuffle(cand)
        children = [[] for _ in range(N)]
        for v in order[1:]:
            children[parent[v]].append(v)

        def subtree(v):
            out, st = [], [v]
            while st:
                u = st.pop()
                out.append(u)
                st.extend(children[u])
            return out

        for v in cand:
            if len(prv_edges) == n_prv:
                break
            members = subtree(v)
            if any(node_type[m] != JUNCTION for m in members):
                continue
            if (zone[members] >= 0).any() or zone[parent[v]] >= 0:
                continue
            zone[members] = len(prv_edges)
            prv_edges.append((int(parent[v]), int(v)))
        if len(prv_edges) < n_prv:
            raise RuntimeError("could not place %d PRV zones" % n_prv)
        # the zone sits lower, so that the PRV must reduce pressure
        for z in range(n_prv):
            el[zone == z] = np.maximum(elev_m[0], el[zone == z] - 0.25 * (elev_m[1] - elev_m[0]))
    # chords: non-tree Delaunay edges that do not cross a zone boundary
    tset = {tuple(e) for e in tree.tolist()}
    n_links = n_pipes + n_prv
    n_chords = n_links - (N - 1)
    if n_chords < 0:
        raise ValueError("fewer links than a spanning tree needs")
    nontree = [tuple(e) for e in edges.tolist() if tuple(e) not in tset
               and zone[e[0]] == zone[e[1]]
               and not (node_type[e[0]] == RESERVOIR and node_type[e[1]] == RESERVOIR)]
    pick = rng.choice(len(nontree), size=n_chords, replace=False)
    chords = [nontree[i] for i in np.sort(pick)]
    # link list: tree edges oriented parent -> child, then chords
    links = []
    prv_set = set(prv_edges)
    for v in order[1:]:
        links.append((int(parent[v]), int(v)))
    links += chords
    n1 = np.array([a for a, _ in links], dtype=np.int64)
    n2 = np.array([b for _, b in links], dtype=np.int64)
    L = len(links)
    ltype = np.full(L, PIPE, dtype=np.int8)
    for k, e in enumerate(links):
        if e in prv_set:
            ltype[k] = PRV
    # pipe sizing from the tree flow (m3/s); chords small
    q_m3s = np.zeros(L)
    n_tree = N - 1
    q_m3s[:n_tree] = 0.6 * sub_q[n2[:n_tree]] / 1000.0
    dset = np.asarray(diam_set_m)
    diam_m = np.empty(L)
    for k in range(L):
        if k < n_tree:
            need = np.sqrt(4.0 * max(q_m3s[k], 1e-5) / (np.pi * vmax))
            ok = dset[dset >= need]
            diam_m[k] = ok[0] if ok.size else dset[-1]
        else:
            diam_m[k] = rng.choice(dset[:4])
    length_m = np.linalg.norm(pts[n1] - pts[n2], axis=1) * rng.uniform(1.0, 1.3, L)
    length_m = np.maximum(length_m, 20.0)
    c = rng.uniform(*c_range, L)
    is_prv = ltype == PRV
    length_m[is_prv] = 0.0
    c[is_prv] = 0.0
    # reservoir heads (stored as the reservoir's elevation, in ft)
    rh = rng.uniform(*res_head_m, n_res)
    el_ft = el / MperFT
    el_ft[res_nodes] = rh / MperFT
    setting = np.zeros(L)
    setting[is_prv] = rng.uniform(*prv_setting_m, int(is_prv.sum()))
    init_status = np.where(is_prv, 2, 1).astype(np.int8)
    ke = np.zeros(N)
    if n_emitters:
        junc = np.flatnonzero(node_type == JUNCTION)
        em = rng.choice(junc, size=n_emitters, replace=False)
        ke[em] = emitter_ke(rng.uniform(*emitter_c, n_emitters))
    diam_ft = diam_m / MperFT
    len_ft = length_m / MperFT
    junc = np.flatnonzero(node_type == JUNCTION)
    return Net(
        node_id=[f"n{i}" for i in range(N)],
        node_type=node_type, elev_ft=el_ft, node_ke=ke,
        res_head_pat=np.full(N, -1, dtype=np.int32),
        link_id=[f"l{k}" for k in range(L)],
        link_type=ltype, link_n1=n1.astype(np.int32), link_n2=n2.astype(np.int32),
        diam_ft=diam_ft, len_ft=len_ft, roughness=c,
        km_int=np.zeros(L), r_hw=_r_hw(len_ft, c, diam_ft),
        init_status=init_status, valve_setting_user=setting,
        dem_node=junc.astype(np.int32),
        dem_base_cfs=base[junc] / LPSperCFS,
        dem_pat=np.full(junc.size, -1, dtype=np.int32),
        pattern_ids=[], patterns=[], meta=_meta())


def config2_network(seed=2):
    """782 junctions, 2 reservoirs, 905 pipes + 3 PRVs, 20 emitters."""
    return looped_network(seed, n_junc=782, n_res=2, n_pipes=905, n_prv=3,
                          n_emitters=20)


def config1_network(seed=1):
    """31 junctions, 1 reservoir (100 m), 34 pipes; literal parameter ranges."""
    rng = np.random.default_rng(seed)
    N = 32
    pts = rng.uniform(0, 3000.0, size=(N, 2))
    edges = _delaunay_edges(pts)
    tree = _spanning_tree(N, edges, rng.uniform(0.1, 1.0, len(edges)))
    res = 0
    parent, order = _root_tree(N, tree, res)
    links = [(int(parent[v]), int(v)) for v in order[1:]]
    tset = {tuple(e) for e in tree.tolist()}
    nontree = [tuple(e) for e in edges.tolist() if tuple(e) not in tset]
    pick = rng.choice(len(nontree), size=3, replace=False)
    links += [nontree[i] for i in np.sort(pick)]
    L = len(links)
    n1 = np.array([a for a, _ in links], dtype=np.int32)
    n2 = np.array([b for _, b in links], dtype=np.int32)
    node_type = np.zeros(N, dtype=np.int8)
    node_type[res] = RESERVOIR
    el_ft = rng.uniform(0.0, 20.0, N) / MperFT
    el_ft[res] = 100.0 / MperFT
    c = rng.uniform(80.0, 140.0, L)
    diam_ft = rng.choice([0.3, 0.4, 0.5, 0.6, 0.75, 1.0], L) / MperFT
    len_ft = rng.uniform(100.0, 3500.0, L) / MperFT
    junc = np.flatnonzero(node_type == JUNCTION)
    dem = rng.uniform(0.0, 0.4, junc.size) / _M3S_PER_CFS
    return Net(
        node_id=[f"n{i}" for i in range(N)], node_type=node_type,
        elev_ft=el_ft, node_ke=np.zeros(N),
        res_head_pat=np.full(N, -1, dtype=np.int32),
        link_id=[f"l{k}" for k in range(L)],
        link_type=np.full(L, PIPE, dtype=np.int8), link_n1=n1, link_n2=n2,
        diam_ft=diam_ft, len_ft=len_ft, roughness=c, km_int=np.zeros(L),
        r_hw=_r_hw(len_ft, c, diam_ft), init_status=np.ones(L, dtype=np.int8),
        valve_setting_user=np.zeros(L), dem_node=junc.astype(np.int32),
        dem_base_cfs=dem, dem_pat=np.full(junc.size, -1, dtype=np.int32),
        pattern_ids=[], patterns=[], meta=_meta())


def config2_scenarios(net, B, seed=0, sigma=0.2):
    """Per-scenario demand [B,N] (cfs) = base * lognormal(0, sigma) per node,
    and reservoir heads [B,N] (nan off reservoirs)."""
    rng = np.random.default_rng(seed)
    d0 = net.demand_cfs_at(0)
    fac = rng.lognormal(0.0, sigma, size=(B, net.N))
    d = d0[None, :] * fac
    rh = np.broadcast_to(net.reservoir_head_ft_at(0), (B, net.N)).copy()
    return d, rh


def sensor_nodes(net, n=30, seed=0):
    """Seeded junction indices used by the sum-of-squared-heads loss."""
    rng = np.random.default_rng(seed)
    junc = np.flatnonzero(np.asarray(net.node_type) == JUNCTION)
    return np.sort(rng.choice(junc, size=n, replace=False))


def feature_network(seed=5, n_junc=60, tank_level=0.5, with_chp=False):
    """Small looped network that exercises every element the batched path
    handles: power-function, custom-curve and no-curve pumps (optionally a
    constant-horsepower pump), two TCVs (Km>0 and Km=0), a check-valve pipe,
    an initially closed pipe, an active PRV and a fixed-open PRV, one tank
    (a fixed head in a steady solve) and emitters."""
    base = looped_network(seed, n_junc=n_junc, n_res=1, n_pipes=n_junc + 10,
                          n_prv=1, zone_size=(5, 15), n_emitters=4,
                          emitter_c=(2e-4, 1e-3), spacing_m=150.0)
    rng = np.random.default_rng(seed + 100)
    N, L = base.N, base.L
    nt = base.node_type.copy()
    junc = np.flatnonzero(nt == JUNCTION)
    prv_k = np.flatnonzero(base.link_type == PRV)
    prv_nodes = set(base.link_n1[prv_k].tolist()) | set(base.link_n2[prv_k].tolist())
    res = int(np.flatnonzero(nt == RESERVOIR)[0])
    pipes = [k for k in range(L) if base.link_type[k] == PIPE
             and base.link_n1[k] not in prv_nodes and base.link_n2[k] not in prv_nodes
             and base.link_n1[k] != res and base.link_n2[k] != res]
    pipes = rng.permutation(pipes).tolist()
    ltype = base.link_type.copy()
    status = base.init_status.copy()
    setting = base.valve_setting_user.copy()
    km = base.km_int.copy()
    c = base.roughness.copy()
    length = base.len_ft.copy()
    diam = base.diam_ft.copy()
    # the reservoir feeds the network through a power-function pump
    k_res = [k for k in range(L) if base.link_n1[k] == res or base.link_n2[k] == res]
    pump_links = [k_res[0]]
    # elements on interior pipes
    k_custom, k_nocurve, k_tcv1, k_tcv0, k_cv, k_closed, k_fixprv = pipes[:7]
    pump_links += [k_custom, k_nocurve]
    if with_chp:
        pump_links.append(pipes[7])
    for k in pump_links:
        ltype[k] = PUMP
        if base.link_n2[k] == res:          # pump discharges away from the source
            base.link_n1[k], base.link_n2[k] = base.link_n2[k], base.link_n1[k]
    ltype[k_tcv1] = TCV
    status[k_tcv1] = 2
    setting[k_tcv1] = 5.0
    ltype[k_tcv0] = TCV
    status[k_tcv0] = 2
    setting[k_tcv0] = 0.0
    ltype[k_cv] = 0                          # CVPIPE
    status[k_closed] = 0
    ltype[k_fixprv] = PRV
    status[k_fixprv] = 1                     # fixed OPEN: setting is MISSING
    km[k_fixprv] = 0.02517 * 2.0 / diam[k_fixprv] ** 4
    for k in pump_links + [k_tcv1, k_tcv0, k_fixprv]:
        c[k] = 0.0
        length[k] = 0.0
    r = _r_hw(length, c, diam)
    d4 = diam ** 2 * diam ** 2
    # pumps: power function (shutoff 40 m, design 60 L/s), custom curve, no curve
    npump = len(pump_links)
    ptype = np.array([1, 2, 3] + ([0] if with_chp else []), dtype=np.int8)
    hs = 40.0 / MperFT
    q0 = 60.0 / LPSperCFS
    nexp = 1.85
    rr = (hs - 0.75 * hs) / q0 ** nexp          # 75 % head at design flow
    h0 = np.array([-hs, 0.0, 0.0] + ([0.0] if with_chp else []))
    pr = np.array([rr, 0.0, 0.0] + ([-8.814 * 20.0] if with_chp else []))
    pn = np.array([nexp, 1.0, 1.0] + ([-1.0] if with_chp else []))
    pq0 = np.array([q0, 10.0 / LPSperCFS, 1.0] + ([1.0] if with_chp else []))
    phmax = np.array([hs, 25.0 / MperFT, 1e10] + ([1e10] if with_chp else []))
    for i, k in enumerate(pump_links):
        setting[k] = 1.0
    # custom curve in user units (L/s, m): three points
    cq = np.array([0.0, 10.0, 30.0])
    ch = np.array([25.0, 20.0, 8.0])
    ptr = np.array([0, 0, 3, 3] + ([3] if with_chp else []), dtype=np.int32)
    # tank on a junction far from the reservoir
    far = int(junc[np.argmax(np.abs(junc - res))])
    nt[far] = TANK
    el = base.elev_ft.copy()
    tank_el = el[far]
    lo, hi = tank_el + 1.0 / MperFT, tank_el + 30.0 / MperFT
    h0t = lo + tank_level * (hi - lo)
    area = np.pi * (20.0 / MperFT) ** 2 / 4.0
    junc2 = np.flatnonzero(nt == JUNCTION)
    base_dem = base.demand_cfs_at(0)
    return Net(
        node_id=base.node_id, node_type=nt, elev_ft=el, node_ke=np.where(nt == JUNCTION, base.node_ke, 0.0),
        res_head_pat=base.res_head_pat, link_id=base.link_id, link_type=ltype,
        link_n1=base.link_n1, link_n2=base.link_n2, diam_ft=diam, len_ft=length,
        roughness=c, km_int=km, r_hw=r, init_status=status,
        valve_setting_user=setting, dem_node=junc2.astype(np.int32),
        dem_base_cfs=base_dem[junc2], dem_pat=np.full(junc2.size, -1, dtype=np.int32),
        pattern_ids=[], patterns=[], meta=_meta(),
        tank_node=np.array([far], dtype=np.int32), tank_h0=np.array([h0t]),
        tank_hmin=np.array([lo]), tank_hmax=np.array([hi]), tank_area=np.array([area]),
        tank_vmin=np.array([0.0]), tank_v0=np.array([(h0t - lo) * area]),
        tank_vmax=np.array([(hi - lo) * area]), tank_overflow=np.array([0], dtype=np.int8),
        pump_link=np.array(pump_links, dtype=np.int32), pump_ptype=ptype,
        pump_h0=h0, pump_r=pr, pump_n=pn, pump_q0=pq0,
        pump_qmax=np.full(npump, 1e10), pump_hmax=phmax,
        pump_upat=np.full(npump, -1, dtype=np.int32),
        pump_curve_q=cq, pump_curve_h=ch, pump_curve_ptr=ptr)


def eps_network(seed=7, n_junc=60, n_pipes=75, n_pumps=4, n_tanks=3, res_head_m=10.0,
                shutoff_m=(40.0, 60.0), tank_center_ft=None, tank_range_m=10.0,
                tank_diam_m=(15.0, 30.0), base_lps=(0.05, 0.4), spacing_m=150.0):
    """Extended-period network: one low reservoir feeding a looped network
    through power-function pumps h = a - b q^1.85 (shutoff a in `shutoff_m`,
    75 % of it at the design flow), and cylindrical tanks on junctions far
    from the source, starting at mid-range.  Reservoir-incident links become
    the pumps (parallel copies are added when there are fewer than
    `n_pumps`; surplus ones are closed).  `tank_center_ft` gives each tank's
    mid-range head (ft); the default is the reservoir head plus 60 % of the
    mean shutoff head, a rough grade-line estimate."""
    base = looped_network(seed, n_junc=n_junc + n_tanks, n_res=1, n_pipes=n_pipes,
                          res_head_m=(res_head_m, res_head_m), base_lps=base_lps,
                          spacing_m=spacing_m)
    rng = np.random.default_rng(seed + 1000)
    N = base.N
    nt = base.node_type.copy()
    res = int(np.flatnonzero(nt == RESERVOIR)[0])
    n1 = list(base.link_n1.tolist())
    n2 = list(base.link_n2.tolist())
    ltype = list(base.link_type.tolist())
    status = list(base.init_status.tolist())
    diam, length, c = list(base.diam_ft), list(base.len_ft), list(base.roughness)
    inc = [k for k in range(base.L) if n1[k] == res or n2[k] == res]
    pumps = inc[:n_pumps]
    for k in inc[n_pumps:]:
        status[k] = 0                                   # surplus source links closed
    while len(pumps) < n_pumps:                         # parallel copies
        k0 = pumps[len(pumps) % max(len(inc), 1)]
        n1.append(n1[k0]); n2.append(n2[k0]); ltype.append(PIPE); status.append(1)
        diam.append(diam[k0]); length.append(0.0); c.append(0.0)
        pumps.append(len(n1) - 1)
    for k in pumps:
        ltype[k] = PUMP
        if n2[k] == res:                                # discharge away from the source
            n1[k], n2[k] = n2[k], n1[k]
        length[k] = 0.0
        c[k] = 0.0
        status[k] = 1
    L = len(n1)
    diam, length, c = np.asarray(diam), np.asarray(length), np.asarray(c)
    # pump curves, internal units: h0 = -a (shutoff), r so that the head is 75 % of a
    # at the design flow (the peak demand shared by the pumps)
    d0 = base.demand_cfs_at(0)
    q_design = 1.6 * float(d0.sum()) / n_pumps
    a_ft = rng.uniform(*shutoff_m, n_pumps) / MperFT
    nexp = 1.85
    pr = 0.25 * a_ft / q_design ** nexp
    # tanks: junctions far from the source, spread out (greedy farthest points)
    pts_el = base.elev_ft
    junc = np.flatnonzero(nt == JUNCTION)
    dist = np.abs(junc - res).astype(np.float64)
    chosen = [int(junc[np.argmax(dist)])]
    while len(chosen) < n_tanks:
        dd = np.min(np.abs(junc[:, None] - np.asarray(chosen)[None, :]), axis=1)
        dd = np.minimum(dd, dist)
        chosen.append(int(junc[np.argmax(dd)]))
    tanks = np.asarray(chosen, dtype=np.int32)
    nt[tanks] = TANK
    if tank_center_ft is None:
        tank_center_ft = np.full(n_tanks, res_head_m / MperFT + 0.6 * float(a_ft.mean()))
    ctr = np.asarray(tank_center_ft, dtype=np.float64)
    half = 0.5 * tank_range_m / MperFT
    hmin, hmax = ctr - half, ctr + half
    el = pts_el.copy()
    el[tanks] = hmin
    area = np.pi * (rng.uniform(*tank_diam_m, n_tanks) / MperFT) ** 2 / 4.0
    h0 = 0.5 * (hmin + hmax)
    junc2 = np.flatnonzero(nt == JUNCTION)
    r = _r_hw(length, c, diam)
    ltype = np.asarray(ltype, dtype=np.int8)
    setting = np.zeros(L)
    setting[pumps] = 1.0
    return Net(
        node_id=base.node_id, node_type=nt, elev_ft=el, node_ke=np.zeros(N),
        res_head_pat=base.res_head_pat, link_id=[f"l{k}" for k in range(L)],
        link_type=ltype, link_n1=np.asarray(n1, dtype=np.int32),
        link_n2=np.asarray(n2, dtype=np.int32), diam_ft=diam, len_ft=length,
        roughness=c, km_int=np.zeros(L), r_hw=r,
        init_status=np.asarray(status, dtype=np.int8), valve_setting_user=setting,
        dem_node=junc2.astype(np.int32), dem_base_cfs=d0[junc2],
        dem_pat=np.full(junc2.size, -1, dtype=np.int32),
        pattern_ids=[], patterns=[], meta=_meta(duration_sec=0),
        tank_node=tanks, tank_h0=h0, tank_hmin=hmin, tank_hmax=hmax, tank_area=area,
        tank_vmin=np.zeros(n_tanks), tank_v0=(h0 - hmin) * area,
        tank_vmax=(hmax - hmin) * area, tank_overflow=np.zeros(n_tanks, dtype=np.int8),
        pump_link=np.asarray(pumps, dtype=np.int32),
        pump_ptype=np.ones(n_pumps, dtype=np.int8), pump_h0=-a_ft, pump_r=pr,
        pump_n=np.full(n_pumps, nexp), pump_q0=np.full(n_pumps, q_design),
        pump_qmax=np.full(n_pumps, 1e10), pump_hmax=a_ft,
        pump_upat=np.full(n_pumps, -1, dtype=np.int32),
        pump_curve_q=np.zeros(0), pump_curve_h=np.zeros(0),
        pump_curve_ptr=np.zeros(n_pumps + 1, dtype=np.int32))


def diurnal(t_hours):
    """Smooth 24-h demand multiplier in [0.5, 1.6], lowest at 00:00."""
    return 1.05 - 0.55 * np.cos(2.0 * np.pi * np.asarray(t_hours, dtype=np.float64) / 24.0)


def eps_demands(net, T, B, seed=0, sigma=0.15, t0_hours=0.0):
    """Demands [T,B,N] (cfs): base * diurnal(t) * lognormal(0, sigma) noise
    drawn per step, scenario and node."""
    rng = np.random.default_rng(seed)
    d0 = net.demand_cfs_at(0)
    m = diurnal(t0_hours + np.arange(T))
    noise = rng.lognormal(0.0, sigma, size=(T, B, net.N))
    return d0[None, None, :] * m[:, None, None] * noise


def chp_dead_end_network(demand_cfs=2e-4, seed=5):
    """The feature network with its constant-horsepower pump re-routed to
    feed a new dead-end junction of tiny demand: at convergence the pump
    carries only that demand, and its gradient -r/q^2 lies above CBIG (the
    clamp branch hloss = -CBIG q of hydcoeffs.c:748-752)."""
    net = feature_network(seed=seed, with_chp=True)
    k = int(net.pump_link[3])
    n1 = int(net.link_n1[k])
    x = net.N
    f = net.as_fields()
    f["node_id"] = list(net.node_id) + ["CHPX"]
    f["node_type"] = np.append(net.node_type, np.int8(JUNCTION)).astype(np.int8)
    f["elev_ft"] = np.append(net.elev_ft, net.elev_ft[n1])
    f["node_ke"] = np.append(net.node_ke, 0.0)
    f["res_head_pat"] = np.append(net.res_head_pat, -1).astype(np.int32)
    n2 = np.asarray(net.link_n2).copy()
    n2[k] = x
    f["link_n2"] = n2.astype(np.int32)
    f["dem_node"] = np.append(net.dem_node, x).astype(np.int32)
    f["dem_base_cfs"] = np.append(net.dem_base_cfs, demand_cfs)
    f["dem_pat"] = np.append(net.dem_pat, -1).astype(np.int32)
    return Net(**f)


def fcv_network(seed=5, links=(62, 22), settings_lps=(14.0, 70.0), km=0.5):
    """The feature network (PRVs, pumps, tank, emitters) with two junction-to-
    junction pipes turned into flow control valves with a setting: the first
    below its pipe's natural flow (an ACTIVE throttle), the second far above
    it (the network cannot push that much, so fcvstatus takes it to XFCV, an
    open valve).  Link orientation follows the natural flow."""
    net = feature_network(seed=seed)
    f = net.as_fields()
    lt = np.asarray(net.link_type).copy()
    st = np.asarray(net.init_status).copy()
    vs = np.asarray(net.valve_setting_user, dtype=np.float64).copy()
    kmi = np.asarray(net.km_int, dtype=np.float64).copy()
    d = np.asarray(net.diam_ft, dtype=np.float64)
    for k, q in zip(links, settings_lps):
        lt[k] = FCV
        st[k] = 2
        vs[k] = q
        kmi[k] = 0.02517 * km / (d[k] ** 2 * d[k] ** 2)
    f["link_type"] = lt.astype(np.int8)
    f["init_status"] = st.astype(np.int8)
    f["valve_setting_user"] = vs
    f["km_int"] = kmi
    return Net(**f)


def psv_network(seed=5, link=27, setting_m=72.0, km=0.5):
    """The feature network (with its ACTIVE PRV) plus a pressure sustaining
    valve on a junction-to-junction pipe whose upstream pressure (about 70 m)
    lies below the valve's setting: the PSV throttles (ACTIVE) to hold its
    upstream head at El[n1] + setting.  Link orientation follows the flow."""
    net = feature_network(seed=seed)
    f = net.as_fields()
    lt = np.asarray(net.link_type).copy()
    st = np.asarray(net.init_status).copy()
    vs = np.asarray(net.valve_setting_user, dtype=np.float64).copy()
    kmi = np.asarray(net.km_int, dtype=np.float64).copy()
    d = np.asarray(net.diam_ft, dtype=np.float64)
    lt[link] = PSV
    st[link] = 2
    vs[link] = setting_m
    kmi[link] = 0.02517 * km / (d[link] ** 2 * d[link] ** 2)
    f["link_type"] = lt.astype(np.int8)
    f["init_status"] = st.astype(np.int8)
    f["valve_setting_user"] = vs
    f["km_int"] = kmi
    return Net(**f)


def unrolled_network(seed=5):
    """The feature network with its PRVs and its no-curve pump turned into
    open pipes: power-function, custom-curve and constant-horsepower pumps,
    TCVs, a check-valve pipe, a closed pipe, a tank as a fixed head and
    emitters, and no control valve (the elements of the unrolled-K route; a
    no-curve pump makes the reference's unrolled autograd return NaN, its
    unselected power-function branch dividing by a zero slope)."""
    net = feature_network(seed=seed, with_chp=True)
    f = net.as_fields()
    lt = np.asarray(net.link_type).copy()
    st = np.asarray(net.init_status).copy()
    prv = lt == PRV
    lt[prv] = PIPE
    st[prv] = 1
    keep = np.asarray(net.pump_ptype) != 3
    lt[np.asarray(net.pump_link)[~keep]] = PIPE
    for key in ("pump_link", "pump_ptype", "pump_h0", "pump_r", "pump_n", "pump_q0",
                "pump_qmax", "pump_hmax", "pump_upat"):
        f[key] = np.asarray(f[key])[keep]
    ptr = np.asarray(net.pump_curve_ptr)
    f["pump_curve_ptr"] = np.concatenate([ptr[:1], ptr[1:][keep]]).astype(np.int32)
    f["link_type"] = lt.astype(np.int8)
    f["init_status"] = st.astype(np.int8)
    return Net(**f)


def config5_network(seed=5, tank_center_ft=None):
    """Extended-period workload shape: about 20 000 junctions and 23 000
    pipes, 4 power-function pumps (shutoff 40-60 m, exponent 1.85),
    3 cylindrical tanks (15-30 m diameter, starting at mid-range) and
    1 reservoir."""
    return eps_network(seed, n_junc=20000, n_pipes=23000, n_pumps=4, n_tanks=3,
                       tank_center_ft=tank_center_ft, base_lps=(0.02, 0.08),
                       spacing_m=120.0)


def tcv_network(seed=3, n_junc=542, n_links=554, n_tcv=79, km_range=(1.0, 20.0)):
    """Looped network whose `n_tcv` links are throttle control valves (Km in
    `km_range`, fully open TCVs for a quarter of them: Km = 0)."""
    base = looped_network(seed, n_junc=n_junc, n_res=2, n_pipes=n_links, spacing_m=160.0)
    rng = np.random.default_rng(seed + 300)
    L = base.L
    res = set(np.flatnonzero(base.node_type == RESERVOIR).tolist())
    cand = [k for k in range(L)
            if base.link_n1[k] not in res and base.link_n2[k] not in res]
    tcv = np.sort(rng.choice(cand, size=n_tcv, replace=False))
    ltype = base.link_type.copy()
    ltype[tcv] = TCV
    status = base.init_status.copy()
    status[tcv] = 2
    setting = base.valve_setting_user.copy()
    setting[tcv] = rng.uniform(*km_range, n_tcv)
    setting[tcv[: n_tcv // 4]] = 0.0
    c = base.roughness.copy()
    length = base.len_ft.copy()
    c[tcv] = 0.0
    length[tcv] = 0.0
    f = dict(base.as_fields())
    f.update(link_type=ltype, init_status=status, valve_setting_user=setting, roughness=c,
             len_ft=length, r_hw=_r_hw(length, c, base.diam_ft))
    return Net(**f)


def config3_networks(seed=3):
    """The four networks of the mixed-size workload: 100 junctions / 120
    pipes; 542 junctions / 554 links including 79 throttle control valves;
    782 junctions / 905 pipes / 3 PRVs (the config-2 network); 3000 junctions
    / 3600 pipes."""
    return [looped_network(seed, n_junc=100, n_res=1, n_pipes=120),
            tcv_network(seed + 1),
            config2_network(),
            looped_network(seed + 2, n_junc=3000, n_res=2, n_pipes=3600, spacing_m=150.0)]


def tanks_as_junctions(net):
    """The same network with every tank turned into a zero-demand junction
    (for a steady pre-solve that finds the grade line at the tank sites)."""
    f = dict(net.as_fields())
    tn = np.asarray(net.tank_node if net.tank_node is not None else [], dtype=np.int64)
    nt = np.asarray(f["node_type"]).copy()
    nt[tn] = JUNCTION
    junc = np.flatnonzero(nt == JUNCTION)
    d0 = net.demand_cfs_at(0)
    f.update(node_type=nt, dem_node=junc.astype(np.int32), dem_base_cfs=d0[junc],
             dem_pat=np.full(junc.size, -1, np.int32), tank_node=np.zeros(0, np.int32),
             tank_overflow=np.zeros(0, np.int8))
    for k in ("tank_h0", "tank_hmin", "tank_hmax", "tank_area", "tank_vmin", "tank_v0",
              "tank_vmax"):
        f[k] = np.zeros(0)
    return Net(**f)


def many_valves_network(seed=8, n_prv=8, psv_links=2, psv_margin_m=12.0,
                        psv_setting_m=(51.57, 48.71), psv_flip=(False, False),
                        psv_pick=(293, 316)):
    """Looped network with `n_prv` PRV zones (each a subtree fed only by its
    PRV) and `psv_links` pressure sustaining valves on junction-to-junction
    tree pipes of the main zone, oriented with the tree flow; each PSV's
    setting is the static pressure at its upstream junction (highest
    reservoir head minus elevation) less `psv_margin_m`, so that the
    headloss upstream makes it throttle in most scenarios, unless the
    settings (m, one per PSV in link order) are given; `psv_flip` (one bool
    per PSV) reverses a PSV's orientation, for one that carries its flow
    against the tree direction; `psv_pick` names the PSV links instead of
    the seeded choice.  The defaults place both PSVs where, with settings
    1 m above the pressure the pipe would see, they throttle (ACTIVE) in the
    seeded lognormal(0.3) scenarios, next to eight ACTIVE PRVs: ten
    constraint rows in the polish and the adjoint."""
    net = looped_network(seed, n_junc=520, n_res=2, n_pipes=600, n_prv=n_prv,
                         zone_size=(12, 40), prv_setting_m=(25.0, 40.0))
    f = net.as_fields()
    lt = np.asarray(net.link_type).copy()
    st = np.asarray(net.init_status).copy()
    vs = np.asarray(net.valve_setting_user, dtype=np.float64).copy()
    kmi = np.asarray(net.km_int, dtype=np.float64).copy()
    nt = np.asarray(net.node_type)
    n1, n2 = np.asarray(net.link_n1).copy(), np.asarray(net.link_n2).copy()
    el_m = np.asarray(net.elev_ft) * MperFT
    hres = float(el_m[nt == RESERVOIR].max())
    # nodes inside PRV zones: reachable from a PRV's downstream end without
    # crossing another PRV
    adj = [[] for _ in range(net.N)]
    for k in range(net.L):
        if lt[k] != PRV:
            adj[n1[k]].append(n2[k])
            adj[n2[k]].append(n1[k])
    inzone = np.zeros(net.N, bool)
    for k in np.flatnonzero(lt == PRV):
        stack = [int(n2[k])]
        while stack:
            u = stack.pop()
            if inzone[u]:
                continue
            inzone[u] = True
            stack.extend(adj[u])
    n_tree = net.N - 1
    rng = np.random.default_rng(seed + 77)
    cand = [k for k in range(n_tree) if lt[k] == PIPE and nt[n1[k]] == JUNCTION
            and nt[n2[k]] == JUNCTION and not inzone[n1[k]] and not inzone[n2[k]]
            and hres - el_m[n1[k]] > psv_margin_m + 20.0]
    rng.shuffle(cand)
    res0 = int(np.flatnonzero(nt == RESERVOIR)[0])

    def reaches_all(skip):  # the network stays connected without link `skip`
        nb = [[] for _ in range(net.N)]
        for k in range(net.L):
            if k != skip:
                nb[n1[k]].append(n2[k])
                nb[n2[k]].append(n1[k])
        seen = np.zeros(net.N, bool)
        stack = [res0]
        while stack:
            u = stack.pop()
            if not seen[u]:
                seen[u] = True
                stack.extend(nb[u])
        return bool(seen.all())

    pick = (sorted(int(k) for k in psv_pick) if psv_pick is not None
            else sorted([k for k in cand if reaches_all(k)][:psv_links]))
    for i, k in enumerate(pick):
        if psv_flip is not None and psv_flip[i]:
            n1[k], n2[k] = n2[k], n1[k]
        lt[k] = PSV
        st[k] = 2
        vs[k] = (hres - el_m[n1[k]] - psv_margin_m if psv_setting_m is None
                 else float(psv_setting_m[i]))
        d = float(net.diam_ft[k])
        kmi[k] = 0.02517 * 0.5 / (d ** 2 * d ** 2)
    f["link_type"] = lt.astype(np.int8)
    f["init_status"] = st.astype(np.int8)
    f["valve_setting_user"] = vs
    f["km_int"] = kmi
    f["link_n1"] = n1.astype(np.int32)
    f["link_n2"] = n2.astype(np.int32)
    return Net(**f)
