"""NumPy restatement of CerebroSim's lattice builder — TEST INFRASTRUCTURE (the oracle), never the product path.

Follows lbm.py:33-58 (D3Q27 constants), lbm.py:63-82 (`Units`), lbm.py:264-330 (`build_lattice`), lbm.py:333-338
(`scatter`) and lbm.py:398-416 (`Solver.set_sponge`). Pinned bit-exactly against tables the reference itself wrote
(tests/golden/tables_small.npz, tests/golden/tables_hash.json, tests/golden/sponge.npz).
"""
import numpy as np

# D3Q27 velocity set in the reference's order (lbm.py:34-40): rest, 6 axis links (+x,-x,+y,-y,+z,-z), 12 edge
# links in +- pairs, 8 corner links in +- pairs.
C = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1],
              [1, 1, 0], [-1, -1, 0], [1, -1, 0], [-1, 1, 0], [1, 0, 1], [-1, 0, -1], [1, 0, -1], [-1, 0, 1],
              [0, 1, 1], [0, -1, -1], [0, 1, -1], [0, -1, 1],
              [1, 1, 1], [-1, -1, -1], [1, 1, -1], [-1, -1, 1], [1, -1, 1], [-1, 1, -1], [-1, 1, 1], [1, -1, -1]],
             np.int32)
W = np.array([8 / 27] + [2 / 27] * 6 + [1 / 54] * 12 + [1 / 216] * 8)
Q = 27
OPP = np.array([int(np.flatnonzero((C == -c).all(1))[0]) for c in C], np.int32)
WALL, INLET, OUTLET0 = -1, -2, -3


class Units:
    """lbm.py:63-82: lattice <-> physical units."""

    def __init__(self, dx, dt, rho, nu):
        self.dx, self.dt, self.rho, self.nu = dx, dt, rho, nu
        self.nu_lu = nu * dt / dx ** 2
        self.tau = 3.0 * self.nu_lu + 0.5
        self.c = dx / dt

    def u(self, u_lu):
        return np.asarray(u_lu) * self.c

    def u_lu(self, u):
        return np.asarray(u) / self.c

    def p(self, p_lu):
        return np.asarray(p_lu) * self.rho * self.c ** 2

    def p_lu(self, p):
        return np.asarray(p) / (self.rho * self.c ** 2)


def _axial_lateral(points, centre, normal):
    """Signed distance along `normal` from the opening's plane, and distance from its axis (lbm.py:301-303)."""
    rel = points - centre
    ax = rel @ normal
    lat = np.linalg.norm(rel - ax[:, None] * normal, axis=1)
    return ax, lat


def build_lattice(phi, origin, dx, openings=(), periodic=(), opening_slack=1.0):
    """lbm.py:264-330. Fluid = phi < 0, numbered in C order; per link i the pull source x - c_i or a boundary code;
    wall fraction q from the SDF; inlet profile from the last inlet over every cell with an inlet link."""
    phi = np.asarray(phi, np.float32)
    dims = np.array(phi.shape)
    fluid = phi < 0
    coords = np.argwhere(fluid).astype(np.int32)
    n = len(coords)
    rank = np.full(phi.shape, -1, np.int32)
    rank[tuple(coords.T)] = np.arange(n, dtype=np.int32)
    origin = np.asarray(origin, float)
    nbr = np.empty((Q, n), np.int32)
    qw = np.full((Q, n), 0.5, np.float32)
    uin = np.zeros((n, 3), np.float32)
    phi_here = phi[tuple(coords.T)]
    inlets = [o for o in openings if o["kind"] == "inlet"]
    outlets = [o for o in openings if o["kind"] == "outlet"]
    # inlets are tested first, then outlets in list order; the first hit claims the link (lbm.py:298-305)
    claim_order = [(o, INLET) for o in inlets] + [(o, OUTLET0 - k) for k, o in enumerate(outlets)]
    counts = {"wall": 0, "inlet": 0, "outlet": [0] * len(outlets)}
    for i in range(Q):
        src_xyz = coords - C[i]
        for a in periodic:
            src_xyz[:, a] %= dims[a]
        in_grid = np.all((src_xyz >= 0) & (src_xyz < dims), axis=1)
        link = np.full(n, WALL, np.int32)
        link[in_grid] = rank[tuple(src_xyz[in_grid].T)]
        missing = np.flatnonzero(link < 0)
        if len(missing) == 0:
            nbr[i] = link
            continue
        pos = origin + src_xyz[missing] * dx
        code = np.full(len(missing), WALL, np.int32)
        for o, c in claim_order:
            ax, lat = _axial_lateral(pos, np.asarray(o["centre"], float), np.asarray(o["normal"], float))
            claim = (ax >= -1e-6) & (lat < o["radius"] + opening_slack * dx) & (code == WALL)
            code[claim] = c
        link[missing] = code
        walls = missing[code == WALL]
        if len(walls):
            sx = src_xyz[walls]
            ok = np.all((sx >= 0) & (sx < dims), axis=1)
            phi_src = np.full(len(walls), np.nan, np.float32)
            phi_src[ok] = phi[tuple(sx[ok].T)]
            with np.errstate(invalid="ignore", divide="ignore"):
                q = -phi_here[walls] / (phi_src - phi_here[walls])
            qw[i, walls] = np.where(np.isfinite(q), np.clip(q, 1e-3, 1.0), 0.5)
        counts["wall"] += int(np.count_nonzero(code == WALL))
        counts["inlet"] += int(np.count_nonzero(code == INLET))
        for k in range(len(outlets)):
            counts["outlet"][k] += int(np.count_nonzero(code == OUTLET0 - k))
        nbr[i] = link
    if inlets:
        cells = np.flatnonzero((nbr == INLET).any(0))
        o = inlets[-1]                      # every inlet pass rewrites all inlet cells: the last one stands
        nrm = np.asarray(o["normal"], float)
        _, lat = _axial_lateral(origin + coords[cells] * dx, np.asarray(o["centre"], float), nrm)
        prof = np.clip(2.0 * (1.0 - (lat / o["radius"]) ** 2), 0.0, None)
        uin[cells] = (-prof[:, None] * nrm[None]).astype(np.float32)
    return {"nbr": nbr, "q": qw, "uin": uin, "coords": coords, "origin": origin, "dx": dx, "shape": phi.shape,
            "n_outlets": len(outlets), "counts": counts, "openings": inlets + outlets}


def scatter(lat, values, fill=np.nan):
    """lbm.py:333-338: per-cell values onto the dense grid."""
    values = np.asarray(values)
    out = np.full(tuple(lat["shape"]) + values.shape[1:], fill, values.dtype if values.dtype.kind == "f" else float)
    out[tuple(lat["coords"].T)] = values
    return out


def sponge_tau(lat, tau, length, tau_max, kinds=("inlet", "outlet")):
    """lbm.py:398-416: per-cell tau raised smoothly towards the openings of the given kinds."""
    pos = lat["origin"] + lat["coords"] * lat["dx"]
    out = np.full(len(lat["coords"]), tau)
    for o in lat["openings"]:
        if o["kind"] not in kinds:
            continue
        c, nrm = np.asarray(o["centre"], float), np.asarray(o["normal"], float)
        rel = pos - c
        depth = -(rel @ nrm) / lat["dx"]
        near = np.linalg.norm(rel - (rel @ nrm)[:, None] * nrm, axis=1) < 1.5 * o["radius"]
        w = np.clip(1.0 - depth / length, 0.0, 1.0)
        w = w * w * (3.0 - 2.0 * w)
        out = np.maximum(out, np.where(near, tau + (tau_max - tau) * w, tau))
    return out
