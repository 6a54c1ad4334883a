"""SHiP magnet templates 1 to 4 without gmsh (``snoopy/SHiP_functions.py:282-2138``).

``get_vector_field_mag_1`` to ``_mag_4`` keep the reference drivers' arguments,
flow and return values:
the template's iron (``geometry_tools.py:133-392``, or with ``use_diluted_steel`` the core plus
a diluted return-yoke wing, ``geometry_tools.py:601-805``) in an air box, the racetrack
filament coil(s) around the core (template 1) or the return-yoke legs (template 3), the
reduced-potential Newton solve (``RedMVPSolver`` or
``RedMVPSolverDiluted``), B = curl A_r + B_coil at the quadrature points of every element,
optionally B at extra positions by nodal interpolation, and the iron mass, coil mass, power
and current density of the design.

The geometry is meshed by this module instead of gmsh's OCC kernel: every boundary of the
template is a plane x = c + m z or y = c + m z between the magnet's entrance and exit, so the
quarter model (x >= 0, y >= 0) is a tensor grid whose x and y grid lines follow those planes
(linear in z inside the magnet, constant in front of and behind it), split into 6 tetrahedra
per cell.  Cells inside iron get spacing ``0.2 lc`` across x and y (the reference's inner mesh
size) and ``lc`` along z; the plane y = 0 carries the natural boundary condition, every other
box face n x A = 0, as in the reference (``SHiP_functions.py:539-570``).  Plotting and the gmsh
GUI flags are accepted and ignored.
"""

import json
import os

import numpy as np

from . import mesh as M
from .materials import Dilution, Reluctance
from .racetrack_coil import RacetrackCoil

TAG_WING = 5  # the diluted return-yoke wing (templates 1 and 3)
TAG_YOKE = 6  # template 4's yoke (its core carries tag 1, the dilutable part)
TAG_NC = 7  # the normal-conducting magnet of the NC/SC model (the superconducting one is tag 1)


def compute_J_opt(conductor_material_data, kappa_elec):
    """Current density in A/mm^2 that balances conductor cost against the cost of its losses
    (``SHiP_functions.py:260-279``): sqrt(kappa_cu rho_mass / (kappa_elec rho_el))."""
    kappa_cu = conductor_material_data["material_cost(CHF/kg)"] + conductor_material_data["manufacturing_cost(CHF/kg)"]
    dens = conductor_material_data["density(g/m3)"]
    rho = conductor_material_data["resistivity(Ohm.m)"]
    return np.sqrt(kappa_cu * dens * 1e-3 / kappa_elec / rho) * 1e-6


def compute_area_polygon(kp, isclosed=True):
    """Signed shoelace area of a polygon kp [M, 2] (``geometry_tools.py:1121-1145``); a closed
    polygon repeats its first point last, otherwise ``isclosed=False`` adds the closing edge."""
    kp = np.asarray(kp, dtype=np.float64)
    area = float(np.sum(kp[:-1, 0] * kp[1:, 1] - kp[1:, 0] * kp[:-1, 1]))
    if not isclosed:
        area += kp[-1, 0] * kp[0, 1] - kp[0, 0] * kp[-1, 1]
    return 0.5 * area


def get_NI(B_goal, parameters_df, df_index, materials_directory="files/materials"):
    """Ampere-turns for a field B_goal from a magnetic-circuit estimate, and whether the
    geometry suits the template (``SHiP_functions.py:40-202``).

    The three flux-path areas are side views (x-z and y-z polygons over the magnet length) of
    the core (A1), the top yoke (A2) and the leg (A3), with the reference's polygons as they
    are (each starts at the origin); path lengths l1 = l3 = mean of Y_core and Y_yoke, l2 = mean
    leg-to-gap width.  Mag1 / Mag2: flux B_goal A1 through all three parts, valid when A1 < A3;
    Mag3: flux B_goal A3, valid when A1 > A3.  NI = sum of nu(B_i) B_i l_i, signed like B_goal.
    """
    reluctance = Reluctance(os.path.join(materials_directory, str(np.asarray(parameters_df["material"])[df_index])))
    v = lambda name: _value(parameters_df, name, df_index)
    Zl = v("Z_len(m)")

    def side(a1, b1, b2, a2):
        # (0, 0), (b1, 0), (b2, Z_len), (a2, Z_len), (a1, 0): the reference's five points
        return compute_area_polygon(np.array([[0.0, 0.0], [b1, 0.0], [b2, Zl], [a2, Zl], [a1, 0.0]]))

    A1 = side(v("Xmgap1(m)"), v("Xcore1(m)"), v("Xcore2(m)"), v("Xmgap2(m)"))
    A2 = side(v("Yvoid1(m)"), v("Yyoke1(m)"), v("Yyoke2(m)"), v("Yvoid2(m)"))
    A3 = side(v("Xvoid1(m)"), v("Xyoke1(m)"), v("Xyoke2(m)"), v("Xvoid2(m)"))
    kind = str(np.asarray(parameters_df["yoke_type"])[df_index])
    l1 = 0.25 * (v("Ycore1(m)") + v("Ycore2(m)") + v("Yyoke1(m)") + v("Yyoke2(m)"))
    l2 = (0.5 * (v("Xyoke1(m)") + v("Xyoke2(m)")) + 0.5 * (v("Xvoid1(m)") + v("Xvoid2(m)"))
          - 0.5 * (v("Xcore1(m)") + v("Xcore2(m)")) - 0.5 * (v("Xmgap1(m)") + v("Xmgap2(m)")))
    l3 = l1
    H = lambda B: float(reluctance.evaluate_nu(B)) * B
    NI, valid = 0.0, True
    if kind in ("Mag1", "Mag2"):
        Phi = abs(B_goal) * A1
        NI = H(B_goal) * l1 + H(Phi / A2) * l2 + H(Phi / A3) * l3
        valid = A1 < A3
    elif kind == "Mag3":
        Phi = abs(B_goal) * A3
        NI = H(Phi / A1) * l1 + H(Phi / A2) * l2 + H(Phi / A3) * l3
        valid = A1 > A3
    if kind in ("Mag1", "Mag2", "Mag3") and B_goal < 0.0:
        NI *= -1.0
    return NI, valid


def compute_prices(magnet_parameters, df_index, M_iron, M_coil, Q, electricity_costs=5.0 / 72000.0, runtime=72000,
                   materials_directory="files/materials", price_peanuts=0.5):
    """Costs of iron, coil and electricity (``SHiP_functions.py:204-257``): masses in g times
    (material + manufacturing cost per kg), power times electricity cost per Wh times runtime,
    all scaled by ``price_peanuts``."""
    with open(os.path.join(materials_directory, str(np.asarray(magnet_parameters["material"])[df_index]))) as f:
        iron = json.load(f)
    with open(os.path.join(materials_directory, str(np.asarray(magnet_parameters["coil_material"])[df_index]))) as f:
        coil = json.load(f)
    C_iron = 1e-3 * M_iron * (iron["material_cost(CHF/kg)"] + iron["manufacturing_cost(CHF/kg)"]) * price_peanuts
    C_coil = 1e-3 * M_coil * (coil["material_cost(CHF/kg)"] + coil["manufacturing_cost(CHF/kg)"]) * price_peanuts
    C_edf = Q * electricity_costs * runtime * price_peanuts
    return C_iron, C_coil, C_edf


def _value(parameters, name, df_index):
    return float(np.asarray(parameters[name])[df_index])


def mag_1_parameters(parameters, df_index=0):
    """The template's geometry and coil parameters from one row of the SHiP parameter table."""
    names = {"X_mgap": "Xmgap", "X_core": "Xcore", "X_void": "Xvoid", "X_yoke": "Xyoke", "Y_core": "Ycore",
             "Y_void": "Yvoid", "Y_yoke": "Yyoke"}
    g = {}
    for key, col in names.items():
        for e in (1, 2):
            name = f"{col}{e}(m)"
            # template 2's table has no magnet gap: its core starts at x = 0
            g[f"{key}_{e}"] = _value(parameters, name, df_index) if (key != "X_mgap" or name in parameters) else 0.0
    for key, col in (("Z_len", "Z_len(m)"), ("Z_pos", "Z_pos(m)"), ("delta_x", "delta_x(m)"),
                     ("delta_y", "delta_y(m)"), ("delta_z", "delta_z(m)"), ("current", "NI(A)"),
                     ("field_density", "field_density"), ("max_turns", "max_turns")):
        g[key] = _value(parameters, col, df_index)
    g["yoke_spacer"] = _value(parameters, "yoke_spacer(mm)", df_index) * 1e-3
    g["ins"] = _value(parameters, "insulation(mm)", df_index) * 1e-3
    g["coil_radius"] = 0.5 * _value(parameters, "coil_diam(mm)", df_index) * 1e-3
    g["lim_x"] = max(g["X_yoke_1"], g["X_yoke_2"]) + g["delta_x"]
    g["lim_y"] = max(g["Y_yoke_1"], g["Y_yoke_2"]) + g["delta_y"]
    g["z_min"] = g["Z_pos"] - g["delta_z"]
    g["z_max"] = g["Z_pos"] + g["Z_len"] + g["delta_z"]
    return g


def mag_4_parameters(parameters, df_index=0):
    """Template 4's parameters: its six x boundaries X_A..X_F come from two table rows
    (``SHiP_functions.py:1800-1815``): X_A, X_B, X_C = Xmgap, Xcore, Xvoid of row df_index and
    X_D, X_E, X_F = Xcore, Xvoid, Xyoke of row df_index + 1."""
    g = mag_1_parameters(parameters, df_index)
    for e in (1, 2):
        g[f"X_A_{e}"] = _value(parameters, f"Xmgap{e}(m)", df_index)
        g[f"X_B_{e}"] = _value(parameters, f"Xcore{e}(m)", df_index)
        g[f"X_C_{e}"] = _value(parameters, f"Xvoid{e}(m)", df_index)
        g[f"X_D_{e}"] = _value(parameters, f"Xcore{e}(m)", df_index + 1)
        g[f"X_E_{e}"] = _value(parameters, f"Xvoid{e}(m)", df_index + 1)
        g[f"X_F_{e}"] = _value(parameters, f"Xyoke{e}(m)", df_index + 1)
    g["lim_x"] = max(g["X_F_1"], g["X_F_2"]) + g["delta_x"]
    return g


def _axis(breaks_1, breaks_2, spacing, names):
    """Grid lines of one axis of the template.

    breaks_1 / breaks_2: breakpoints at the entrance / exit, spacing and names per interval.
    Intervals of zero width at both ends are dropped; a width that vanishes at one end only
    is rejected.  Returns, per grid line, its interval and fraction inside it, the interval
    name of every cell, and the entrance / exit breakpoints kept."""
    b1, b2, hs, nm = [breaks_1[0]], [breaks_2[0]], [], []
    for i in range(len(names)):
        w1 = breaks_1[i + 1] - breaks_1[i]
        w2 = breaks_2[i + 1] - breaks_2[i]
        if w1 == 0.0 and w2 == 0.0:
            continue
        if not (w1 > 0.0 and w2 > 0.0):
            raise ValueError(f"template interval {names[i]!r} is empty or inverted at one end ({w1}, {w2})")
        b1.append(breaks_1[i + 1])
        b2.append(breaks_2[i + 1])
        hs.append(spacing[i])
        nm.append(names[i])
    counts = [max(1, int(np.ceil(max(b1[i + 1] - b1[i], b2[i + 1] - b2[i]) / hs[i] - 1e-9))) for i in range(len(nm))]
    line_iv, line_f = [], []
    for i, c in enumerate(counts):
        line_iv += [i] * c
        line_f += [k / c for k in range(c)]
    line_iv.append(len(counts) - 1)
    line_f.append(1.0)
    cell_names = np.repeat(np.array(nm, dtype=object), counts)
    return np.array(line_iv), np.array(line_f), cell_names, np.array(b1), np.array(b2)


def mag_1_mesh(g, lc=0.2, use_diluted_steel=False, inner=0.2):
    """Quarter-model tetrahedral mesh of templates 1 and 3 (one iron geometry; tags: iron 1,
    air 2, diluted wing 5); ``inner`` x ``lc`` is the spacing across the iron."""
    return template_mesh(g, 1, lc, use_diluted_steel, inner)


def template_mesh(g, template=1, lc=0.2, use_diluted_steel=False, inner=0.2):
    """Quarter-model tetrahedral mesh of a template (tags: iron 1, air 2, diluted wing 5).

    Templates 1 and 3 (``geometry_tools.py:213-259``): core [X_mgap, X_core] x [0, Y_yoke],
    top [X_core, X_void] x [Y_core, Y_yoke] and leg [X_void, X_yoke] x [0, Y_yoke]; with the
    diluted wing (``geometry_tools.py:601-805``) the leg below Y_void is the wing.  Template 2
    (``geometry_tools.py:392-500, 305-345``): core [0, X_core] x [0, Y_core], yoke
    [0, X_yoke] x [Y_void, Y_yoke] and leg [X_void, X_yoke] x [0, Y_void]."""
    lci = inner * lc
    Z1, Z2 = g["Z_pos"], g["Z_pos"] + g["Z_len"]
    if template == 4:
        xb = lambda e: [0.0] + [g[f"X_{c}_{e}"] for c in "ABCDEF"] + [g["lim_x"]]
        xi, xf, xcell, xb1, xb2 = _axis(xb(1), xb(2), [lci] * 6 + [lc],
                                        ["gap", "legA", "slot1", "core", "slot2", "legF", "out"])
        yb = lambda e: [0.0, g[f"Y_core_{e}"], g[f"Y_yoke_{e}"], g["lim_y"]]
        yi, yf, ycell, yb1, yb2 = _axis(yb(1), yb(2), [lci, lci, lc], ["low", "top", "out"])
        return _finish(g, lc, xi, xf, xcell, xb1, xb2, yi, yf, ycell, yb1, yb2, template, use_diluted_steel)
    if template == 2:
        xb = lambda e: [0.0, g[f"X_core_{e}"], g[f"X_void_{e}"], g[f"X_yoke_{e}"], g["lim_x"]]
        xi, xf, xcell, xb1, xb2 = _axis(xb(1), xb(2), [lci, lci, lci, lc], ["core", "void", "leg", "out"])
        yb = lambda e: [0.0, g[f"Y_core_{e}"], g[f"Y_void_{e}"], g[f"Y_yoke_{e}"], g["lim_y"]]
        yi, yf, ycell, yb1, yb2 = _axis(yb(1), yb(2), [lci, lci, lci, lc], ["low", "mid", "top", "out"])
        return _finish(g, lc, xi, xf, xcell, xb1, xb2, yi, yf, ycell, yb1, yb2, template, use_diluted_steel)
    xb = lambda e: [0.0, g[f"X_mgap_{e}"], g[f"X_core_{e}"], g[f"X_void_{e}"], g[f"X_yoke_{e}"], g["lim_x"]]
    xi, xf, xcell, xb1, xb2 = _axis(xb(1), xb(2), [lci, lci, lci, lci, lc], ["gap", "core", "void", "leg", "out"])
    if use_diluted_steel:
        yb = lambda e: [0.0, g[f"Y_core_{e}"], g[f"Y_void_{e}"], g[f"Y_yoke_{e}"], g["lim_y"]]
        yi, yf, ycell, yb1, yb2 = _axis(yb(1), yb(2), [lci, lci, lci, lc], ["low", "mid", "top", "out"])
    else:
        yb = lambda e: [0.0, g[f"Y_core_{e}"], g[f"Y_yoke_{e}"], g["lim_y"]]
        yi, yf, ycell, yb1, yb2 = _axis(yb(1), yb(2), [lci, lci, lc], ["low", "top", "out"])
    return _finish(g, lc, xi, xf, xcell, xb1, xb2, yi, yf, ycell, yb1, yb2, template, use_diluted_steel)


def _finish(g, lc, xi, xf, xcell, xb1, xb2, yi, yf, ycell, yb1, yb2, template, use_diluted_steel):
    """z lines, cell materials and the mapped nodes of a template mesh."""
    Z1, Z2 = g["Z_pos"], g["Z_pos"] + g["Z_len"]
    zb = [g["z_min"], Z1, Z2, g["z_max"]]
    zi, zf, zcell, zb1, _ = _axis(zb, zb, [lc, lc, lc], ["front", "magnet", "back"])
    zs = zb1[zi] + zf * (zb1[np.minimum(zi + 1, len(zb1) - 1)] - zb1[zi])
    # cell materials
    nx, ny, nz = len(xcell), len(ycell), len(zcell)
    X, Y, Z = np.meshgrid(xcell, ycell, zcell, indexing="ij")
    inside = Z == "magnet"
    if template == 4:
        # core [X_C, X_D] x [0, Y_core]; yoke [X_A, X_F] x [0, Y_yoke] without [X_B, X_E] x [0, Y_core]
        iron = inside & (X == "core") & (Y == "low")
        wing = inside & (np.isin(X, ["legA", "legF"]) & (Y != "out") |
                         np.isin(X, ["slot1", "core", "slot2"]) & (Y == "top"))
        dom = np.full((nx, ny, nz), M.TAG_AIR, dtype=np.int32)
        dom[iron] = M.TAG_IRON
        dom[wing] = TAG_YOKE
        return _mapped(g, xi, xf, xb1, xb2, yi, yf, yb1, yb2, zs, nx, ny, nz, dom)
    if template == 2:
        iron = inside & ((X == "core") & (Y == "low") | (Y == "top") & (X != "out") |
                         (X == "leg") & (Y != "out"))
        wing = np.zeros_like(iron)
    elif use_diluted_steel:
        iron = inside & ((X == "core") & (Y != "out") | (X == "void") & np.isin(Y, ["mid", "top"]) |
                         (X == "leg") & (Y == "top"))
        wing = inside & (X == "leg") & np.isin(Y, ["low", "mid"])
    else:
        iron = inside & (np.isin(X, ["core", "leg"]) & (Y != "out") | (X == "void") & (Y == "top"))
        wing = np.zeros_like(iron)
    dom = np.full((nx, ny, nz), M.TAG_AIR, dtype=np.int32)
    dom[iron] = M.TAG_IRON
    dom[wing] = TAG_WING
    return _mapped(g, xi, xf, xb1, xb2, yi, yf, yb1, yb2, zs, nx, ny, nz, dom)


def _mapped(g, xi, xf, xb1, xb2, yi, yf, yb1, yb2, zs, nx, ny, nz, dom):
    """Split the reference grid into tetrahedra and move its nodes onto the template."""
    Z1, Z2 = g["Z_pos"], g["Z_pos"] + g["Z_len"]
    ref = M.tensor_grid_mesh(np.arange(nx + 1.0), np.arange(ny + 1.0), np.arange(nz + 1.0), dom)
    # map the reference grid onto the template: x and y lines follow their planes along z
    I = np.rint(ref.nodes[:, 0]).astype(np.int64)
    J = np.rint(ref.nodes[:, 1]).astype(np.int64)
    K = np.rint(ref.nodes[:, 2]).astype(np.int64)
    z = zs[K]
    t = np.clip((z - Z1) / (Z2 - Z1), 0.0, 1.0)

    def along(b1, b2, iv, f):
        lo = b1[iv] + t * (b2[iv] - b1[iv])
        hi_i = np.minimum(iv + 1, len(b1) - 1)
        hi = b1[hi_i] + t * (b2[hi_i] - b1[hi_i])
        return lo + f * (hi - lo)

    nodes = np.stack([along(xb1, xb2, xi[I], xf[I]), along(yb1, yb2, yi[J], yf[J]), z], axis=1)
    msh = M.TetMesh(nodes, ref.cells, ref.elem_domain)
    msh.natural_planes = [(1, 0.0)]
    return msh


class Magnet:
    """One magnet of a multi-magnet model: its z range, its x and y boundaries at the entrance
    and the exit (interior breakpoints, 0 and the box face are implied) with the names of the
    intervals between them, a spacing across its iron, and ``tag(X, Y)`` giving the volume tag
    (0 for air) of cells with interval names X, Y (arrays)."""

    def __init__(self, z1, z2, x_names, x1, x2, y_names, y1, y2, tag, inner):
        self.z1, self.z2 = float(z1), float(z2)
        self.x = (list(x_names), list(x1), list(x2))
        self.y = (list(y_names), list(y1), list(y2))
        self.tag = tag
        self.inner = inner


def _chain(names, b1, b2, lim):
    """A magnet's lines along one axis without zero-width intervals: entrance and exit
    positions of its interior lines and the names of its intervals (from 0 to the box face)."""
    k1, k2, nm = [0.0], [0.0], []
    for i in range(len(b1)):
        w1, w2 = b1[i] - k1[-1], b2[i] - k2[-1]
        if w1 == 0.0 and w2 == 0.0:
            continue
        if not (w1 > 0.0 and w2 > 0.0):
            raise ValueError(f"interval {names[i]!r} is empty or inverted at one end ({w1}, {w2})")
        k1.append(b1[i])
        k2.append(b2[i])
        nm.append(names[i])
    if not (lim > k1[-1] and lim > k2[-1]):
        raise ValueError("the box does not contain the magnet")
    nm.append(names[len(b1)])
    return np.array(k1[1:]), np.array(k2[1:]), nm


def _merged_axis(magnets, axis, lim, lc):
    """Grid lines of one axis shared by several magnets.

    Every magnet's lines take part; they are ordered by their mid-length positions (each
    magnet's own order is kept).  Inside a magnet's z range its lines lie on its planes and the
    other magnets' lines are spread evenly between their active neighbours; between magnets
    every line moves linearly from one arrangement to the next.  Returns a function giving,
    for a z value, the positions of the merged lines (0 and the box face included), the grid
    lines (merged interval, fraction), and per magnet the name of its interval holding each
    merged interval."""
    chains = [_chain(*getattr(m, axis), lim) for m in magnets]
    keys, owner = [], []
    for mi, (k1, k2, _) in enumerate(chains):
        for li in range(len(k1)):
            keys.append((0.5 * (k1[li] + k2[li]), mi, li))
            owner.append((mi, li))
    order = sorted(range(len(keys)), key=lambda i: keys[i])
    lines = [owner[i] for i in order]  # merged interior lines
    L = len(lines) + 2

    def arrangement(mi, t):
        k1, k2, _ = chains[mi]
        pos = np.full(L, np.nan)
        pos[0], pos[-1] = 0.0, lim
        for q, (m2, li) in enumerate(lines):
            if m2 == mi:
                pos[q + 1] = k1[li] + t * (k2[li] - k1[li])
        act = np.flatnonzero(~np.isnan(pos))
        for a, b in zip(act[:-1], act[1:]):
            for j in range(a + 1, b):
                pos[j] = pos[a] + (j - a) / (b - a) * (pos[b] - pos[a])
        return pos

    def positions(z):
        if z <= magnets[0].z1:
            return arrangement(0, 0.0)
        for mi, m in enumerate(magnets):
            if z <= m.z2:
                if z >= m.z1:
                    return arrangement(mi, (z - m.z1) / (m.z2 - m.z1))
                prev = magnets[mi - 1]
                s_ = (z - prev.z2) / (m.z1 - prev.z2)
                return (1.0 - s_) * arrangement(mi - 1, 1.0) + s_ * arrangement(mi, 0.0)
        return arrangement(len(magnets) - 1, 1.0)

    # per magnet: the name of its interval that holds merged interval q
    names = []
    for mi, (k1, _, nm) in enumerate(chains):
        count = 0
        per = []
        for q in range(L - 1):
            per.append(nm[count])
            if q < len(lines) and lines[q][0] == mi:
                count += 1
        names.append(np.array(per, dtype=object))
    # spacing: the finest of the magnets whose lateral extent holds the interval
    hs = np.full(L - 1, lc)
    for mi, m in enumerate(magnets):
        hs = np.where(names[mi] != "out", np.minimum(hs, m.inner), hs)
    arr = [arrangement(mi, t) for mi in range(len(magnets)) for t in (0.0, 1.0)]
    width = np.max([np.diff(a) for a in arr], axis=0)
    counts = np.maximum(1, np.ceil(width / hs - 1e-9).astype(np.int64))
    line_iv = np.concatenate([np.full(c, q) for q, c in enumerate(counts)] + [[L - 2]])
    line_f = np.concatenate([np.arange(c) / c for c in counts] + [[1.0]])
    cell_iv = np.repeat(np.arange(L - 1), counts)
    return positions, line_iv, line_f, cell_iv, names


def magnets_mesh(magnets, lim_x, lim_y, z_min, z_max, lc):
    """Tetrahedral mesh of an air box [0, lim_x] x [0, lim_y] x [z_min, z_max] holding magnets
    one after another along z (quarter model: y = 0 carries the natural condition)."""
    magnets = sorted(magnets, key=lambda m: m.z1)
    for a, b in zip(magnets[:-1], magnets[1:]):
        if b.z1 < a.z2:
            raise ValueError("magnets overlap along z")
    xpos, xi, xf, xcell, xnames = _merged_axis(magnets, "x", lim_x, lc)
    ypos, yi, yf, ycell, ynames = _merged_axis(magnets, "y", lim_y, lc)
    zb = [z_min]
    zseg = []
    for mi, m in enumerate(magnets):
        if m.z1 > zb[-1]:
            zb.append(m.z1)
            zseg.append(-1)
        zb.append(m.z2)
        zseg.append(mi)
    zb.append(z_max)
    zseg.append(-1)
    zcount = [max(1, int(np.ceil((zb[i + 1] - zb[i]) / lc - 1e-9))) for i in range(len(zseg))]
    zs = np.concatenate([zb[i] + (zb[i + 1] - zb[i]) * np.arange(c) / c for i, c in enumerate(zcount)] + [[z_max]])
    zcell = np.repeat(np.array(zseg), zcount)
    nx, ny, nz = len(xcell), len(ycell), len(zcell)
    dom = np.full((nx, ny, nz), M.TAG_AIR, dtype=np.int32)
    for mi, m in enumerate(magnets):
        ks = np.flatnonzero(zcell == mi)
        if len(ks) == 0:
            continue
        X, Y = np.meshgrid(xnames[mi][xcell], ynames[mi][ycell], indexing="ij")
        tag = np.asarray(m.tag(X, Y), dtype=np.int32)
        dom[:, :, ks] = np.where(tag[:, :, None] != 0, tag[:, :, None], M.TAG_AIR)
    ref = M.tensor_grid_mesh(np.arange(nx + 1.0), np.arange(ny + 1.0), np.arange(nz + 1.0), dom)
    I = np.rint(ref.nodes[:, 0]).astype(np.int64)
    J = np.rint(ref.nodes[:, 1]).astype(np.int64)
    K = np.rint(ref.nodes[:, 2]).astype(np.int64)
    PX = np.array([xpos(z) for z in zs])  # [nz + 1, merged lines]
    PY = np.array([ypos(z) for z in zs])
    x = PX[K, xi[I]] + xf[I] * (PX[K, np.minimum(xi[I] + 1, PX.shape[1] - 1)] - PX[K, xi[I]])
    y = PY[K, yi[J]] + yf[J] * (PY[K, np.minimum(yi[J] + 1, PY.shape[1] - 1)] - PY[K, yi[J]])
    msh = M.TetMesh(np.stack([x, y, zs[K]], axis=1), ref.cells, ref.elem_domain)
    msh.natural_planes = [(1, 0.0)]
    return msh


def _coils(g, J_tar, filling_factor, template=1):
    """The template's racetrack coils, turn positions and the coil's electrical figures
    (template 1: around the core, ``SHiP_functions.py:572-658``; template 3: around the
    return-yoke legs, ``SHiP_functions.py:1505-1562``)."""
    X_mgap_1, X_mgap_2 = g["X_mgap_1"], g["X_mgap_2"]
    X_core_1, X_core_2 = g["X_core_1"], g["X_core_2"]
    Z_pos, Z_len = g["Z_pos"], g["Z_len"]
    sp, ins, r = g["yoke_spacer"], g["ins"], g["coil_radius"]
    current = g["current"]
    slot_size = 2 * min(g["Y_core_1"], g["Y_core_2"])
    num_cond = min(int(slot_size / 2 / (r + ins)), int(g["max_turns"]))
    if num_cond < 1:
        raise ValueError("the slot holds no conductor")
    y = np.linspace(-0.5 * slot_size + r + ins, 0.5 * slot_size - r - ins, num_cond)
    slot_size_horz = min(g["X_void_1"] - X_core_1, g["X_void_2"] - X_core_2)
    A_geo = slot_size_horz * slot_size
    A_cu = abs(current) / J_tar
    A_coil = A_cu / filling_factor
    current_density = 0.0 if current == 0.0 else abs(current) / min(A_geo, A_coil) / filling_factor
    d = sp + ins + r
    if template == 2:
        X_mgap_1 = X_mgap_2 = 0.0  # one coil around the core
    if template == 4:
        # slots on both sides of the core (SHiP_functions.py:1975-1976)
        slot_size_horz = min(g["X_C_1"] - g["X_B_1"], g["X_C_2"] - g["X_B_2"], g["X_E_1"] - g["X_D_1"],
                             g["X_E_2"] - g["X_D_2"])
        A_geo = slot_size_horz * slot_size
        current_density = 0.0 if current == 0.0 else abs(current) / min(A_geo, A_coil) / filling_factor
        X_C_1, X_C_2, X_D_1, X_D_2 = g["X_C_1"], g["X_C_2"], g["X_D_1"], g["X_D_2"]
        kp_1 = np.array([[X_C_2 - d, Z_pos + Z_len], [X_C_2, Z_pos + Z_len + d], [X_D_2, Z_pos + Z_len + d],
                         [X_D_2 + d, Z_pos + Z_len], [X_D_1 + d, Z_pos], [X_D_1, Z_pos - d],
                         [X_C_1, Z_pos - d], [X_C_1 - d, Z_pos]])
        kp_2 = kp_1.copy()
        kp_2[:, 0] *= -1.0
        coils = [RacetrackCoil(kp_1, y, r, current / num_cond), RacetrackCoil(kp_2, y, r, current / num_cond)]
    elif template == 3:
        X_void_1, X_void_2, X_yoke_1, X_yoke_2 = g["X_void_1"], g["X_void_2"], g["X_yoke_1"], g["X_yoke_2"]
        kp_1 = np.array([[X_void_2 - d, Z_pos + Z_len], [X_void_2, Z_pos + Z_len + d], [X_yoke_2, Z_pos + Z_len + d],
                         [X_yoke_2 + d, Z_pos + Z_len], [X_yoke_1 + d, Z_pos], [X_yoke_1, Z_pos - d],
                         [X_void_1, Z_pos - d], [X_void_1 - d, Z_pos]])
        kp_2 = kp_1.copy()
        kp_2[:, 0] *= -1.0
        coils = [RacetrackCoil(kp_1, y, r, current / num_cond), RacetrackCoil(kp_2, y, r, current / num_cond)]
    elif X_mgap_1 == 0.0 or X_mgap_2 == 0.0:
        kp = np.array([[-X_core_2 - d, Z_pos + Z_len], [-X_core_2, Z_pos + Z_len + d], [X_core_2, Z_pos + Z_len + d],
                       [X_core_2 + d, Z_pos + Z_len], [X_core_1 + d, Z_pos], [X_core_1, Z_pos - d],
                       [-X_core_1, Z_pos - d], [-X_core_1 - d, Z_pos]])
        coils = [RacetrackCoil(kp, y, r, current / num_cond)]
    else:
        kp_1 = np.array([[X_mgap_2 - d, Z_pos + Z_len + r], [X_mgap_2, Z_pos + Z_len + d], [X_core_2, Z_pos + Z_len + d],
                         [X_core_2 + d, Z_pos + Z_len], [X_core_1 + d, Z_pos], [X_core_1, Z_pos - d],
                         [X_mgap_1, Z_pos - d], [X_mgap_1 - d, Z_pos]])
        kp_2 = kp_1.copy()
        kp_2[:, 0] *= -1.0
        coils = [RacetrackCoil(kp_1, y, r, current / num_cond), RacetrackCoil(kp_2, y, r, current / num_cond)]
    perimeter = sum(c.get_length() for c in coils)
    return coils, A_cu, A_coil, perimeter, current_density


def get_vector_field_mag_1(parameters, df_index=0, lc=0.2, geo_th=1e-5, run_gmsh=False, plot_geo=False,
                           plot_result=False, result_directory="none", result_spec="", eval_pos=np.zeros((0, 3)),
                           materials_directory="files/materials", quad_order=8, max_coil_size=0.05,
                           use_diluted_steel=False, kappa_elec=5.0):
    """B of SHiP magnet template 1 (``SHiP_functions.py:282-809``): coil around the core; see
    ``_template`` for the return values."""
    return _template(1, parameters, df_index, lc, result_directory, result_spec, eval_pos, materials_directory,
                     quad_order, use_diluted_steel, kappa_elec)


def get_vector_field_mag_3(parameters, df_index=0, lc=0.2, geo_th=1e-5, run_gmsh=False, plot_geo=False,
                           plot_result=False, result_directory="none", result_spec="", eval_pos=np.zeros((0, 3)),
                           materials_directory="files/materials", quad_order=8, max_coil_size=0.05,
                           use_diluted_steel=False, kappa_elec=5.0):
    """B of SHiP magnet template 3 (``SHiP_functions.py:1218-1711``): template 1's iron (and
    diluted wing), coils around the return-yoke legs."""
    return _template(3, parameters, df_index, lc, result_directory, result_spec, eval_pos, materials_directory,
                     quad_order, use_diluted_steel, kappa_elec)


def get_vector_field_mag_4(parameters, df_index=0, lc=0.2, geo_th=1e-5, run_gmsh=False, plot_geo=False,
                           plot_result=False, result_directory="none", result_spec="", eval_pos=np.zeros((0, 3)),
                           materials_directory="files/materials", quad_order=8, max_coil_size=0.05,
                           use_diluted_steel=False, kappa_elec=5.0):
    """B of SHiP magnet template 4 (``SHiP_functions.py:1712-2138``): a core [X_C, X_D] between
    the two legs of a yoke (its boundaries from rows df_index and df_index + 1, see
    ``mag_4_parameters``), coils around the core; ``use_diluted_steel`` dilutes the core."""
    return _template(4, parameters, df_index, lc, result_directory, result_spec, eval_pos, materials_directory,
                     quad_order, use_diluted_steel, kappa_elec)


def get_vector_field_mag_2(parameters, df_index=0, lc=0.4, geo_th=1e-5, run_gmsh=False, plot_geo=False,
                           plot_result=False, result_directory="none", result_spec="", eval_pos=np.zeros((0, 3)),
                           materials_directory="files/materials", quad_order=8, max_coil_size=0.05, kappa_elec=5.0):
    """B of SHiP magnet template 2, the superconducting one (``SHiP_functions.py:812-1217``):
    an iron core [0, X_core] x [0, Y_core] inside an L-shaped yoke, one coil around the core."""
    return _template(2, parameters, df_index, lc, result_directory, result_spec, eval_pos, materials_directory,
                     quad_order, False, kappa_elec)


def _template(template, parameters, df_index, lc, result_directory, result_spec, eval_pos, materials_directory,
              quad_order, use_diluted_steel, kappa_elec):
    """Templates 1 to 4.

    :return: ``[points, B, M_iron, M_coil, Q, current_density]``: the quadrature points of every
        element (``field_density`` order) and the total field there, the iron mass in g (the
        quarter model's iron volume x 4 x density), the coil mass in g, the ohmic power in W
        and the coil's current density in A/m^2.  With ``eval_pos``, B there (nodal
        interpolation per domain) is written to ``B<result_spec>.csv``.
    """
    from .evaluators import evaluate_fem_solution_node_interpolation
    from .red_mvp_solver import RedMVPSolver
    from .red_mvp_solver_diluted import RedMVPSolverDiluted

    reluctance_iron = Reluctance(os.path.join(materials_directory, str(np.asarray(parameters["material"])[df_index])))
    with open(os.path.join(materials_directory, str(np.asarray(parameters["material"])[df_index]))) as f:
        iron_material_data = json.load(f)
    with open(os.path.join(materials_directory, str(np.asarray(parameters["coil_material"])[df_index]))) as f:
        conductor_material_data = json.load(f)
    J_tar_mm2 = _value(parameters, "J_tar(A/mm2)", df_index)
    J_tar = (compute_J_opt(conductor_material_data, kappa_elec) if J_tar_mm2 < 0 else J_tar_mm2) * 1e6

    g = mag_4_parameters(parameters, df_index) if template == 4 else mag_1_parameters(parameters, df_index)
    # iron spacing: 0.2 lc, except 0.3 lc for template 2 and template 3's plain yoke and lc for
    # template 4 (SHiP_functions.py:944-969, 1435, 1871)
    if template == 4:
        inner = 1.0
    else:
        inner = 0.3 if (template == 2 or (template == 3 and not use_diluted_steel)) else 0.2
    msh = template_mesh(g, template, lc=lc, use_diluted_steel=use_diluted_steel, inner=inner)
    vol = M.tet_volumes6(msh.nodes, msh.cells) / 6.0
    if template == 4:
        iron_tags = [M.TAG_IRON, TAG_YOKE]
    else:
        iron_tags = [M.TAG_IRON, TAG_WING] if use_diluted_steel else [M.TAG_IRON]
    M_iron = 4 * float(vol[np.isin(msh.elem_domain, iron_tags)].sum()) * iron_material_data["density(g/m3)"]

    coils, A_cu, A_coil, perimeter, current_density = _coils(g, J_tar, conductor_material_data["filling_factor"],
                                                             template)
    M_coil = A_cu * perimeter * conductor_material_data["density(g/m3)"]
    current = g["current"]
    Q = 0.0 if current == 0 else abs(current * current) * perimeter * conductor_material_data["resistivity(Ohm.m)"] / A_cu

    max_newton = 150 if template == 4 else 25
    rels = [reluctance_iron] * len(iron_tags)
    if use_diluted_steel and template == 4:
        # template 4 dilutes its core (SHiP_functions.py:1850-1854, 2033-2038)
        dil = Dilution(g["X_A_1"] + g["X_E_1"], g["X_B_1"] + g["X_F_1"], g["X_C_1"], g["X_D_1"],
                       g["X_A_2"] + g["X_E_2"], g["X_B_2"] + g["X_F_2"], g["X_C_2"], g["X_D_2"], g["Z_pos"], g["Z_len"])
        solver = RedMVPSolverDiluted(msh, coils, iron_tags, [M.TAG_AIR], rels, [dil, None], quad_order=quad_order,
                                     max_newton_iterations=max_newton)
    elif use_diluted_steel:
        dilution_wing = Dilution(g["X_mgap_1"], g["X_core_1"], g["X_void_1"], g["X_yoke_1"], g["X_mgap_2"],
                                 g["X_core_2"], g["X_void_2"], g["X_yoke_2"], g["Z_pos"], g["Z_len"])
        solver = RedMVPSolverDiluted(msh, coils, iron_tags, [M.TAG_AIR], rels, [None, dilution_wing],
                                     quad_order=quad_order, max_newton_iterations=max_newton)
    else:
        solver = RedMVPSolver(msh, coils, iron_tags, [M.TAG_AIR], rels, quad_order=quad_order,
                              max_newton_iterations=max_newton)
    solver.verbose = False
    x = np.zeros(solver.num_dofs_mvp) if current == 0.0 else solver.solve()
    points, B_i = solver.curl_curl_factory.compute_B(x, quad_order=int(0.5 * g["field_density"]))
    B_coil = 0.0 * B_i
    for coil in coils:
        B_coil += coil.compute_B(points)
    if result_directory != "none":
        np.save(os.path.join(result_directory, "x" + result_spec + ".npy"), x)
        row = {k: np.asarray(v)[df_index] for k, v in dict(parameters).items()}
        with open(os.path.join(result_directory, "parameters" + result_spec + ".csv"), "w") as f:
            f.write(",".join(row) + "\n" + ",".join(str(v) for v in row.values()) + "\n")
    ret_vals = [points, B_i + B_coil, M_iron, M_coil, Q, current_density]
    eval_pos = np.asarray(eval_pos, dtype=np.float64).reshape(-1, 3)
    if eval_pos.shape[0] > 0:
        B_tot = evaluate_fem_solution_node_interpolation(msh, eval_pos, solver, coils, x, iron_tags + [M.TAG_AIR])
        name = "B" + result_spec + ".csv"
        out = os.path.join(result_directory, name) if result_directory != "none" else name
        header = "x(m),y(m),z(m),Bx(T),By(T),Bz(T)"
        np.savetxt(out, np.append(eval_pos, B_tot, axis=1), delimiter=",", header=header, comments="")
    return ret_vals


def _tag_type_1(X, Y):
    """Templates 1 and 3's iron (``geometry_tools.py:213-259``)."""
    return (np.isin(X, ["core", "leg"]) & (Y != "out")) | ((X == "void") & (Y == "top"))


def _tag_type_2(X, Y):
    """Template 2's core and L-shaped yoke (``geometry_tools.py:305-345, 392-500``)."""
    return ((X == "core") & (Y == "low")) | ((Y == "top") & (X != "out")) | ((X == "leg") & (Y != "out"))


def get_vector_field_ncsc(parameters, df_index=0, lc=0.2, geo_th=1e-5, run_gmsh=False, plot_geo=False,
                          plot_result=False, result_directory="none", result_spec="", eval_pos=np.zeros((0, 3)),
                          materials_directory="files/materials", quad_order=8):
    """B of the NC/SC model (``SHiP_functions.py:2139-2623``): a normal-conducting magnet with
    template 1's yoke (row df_index) followed along z by a superconducting one with template
    2's core and yoke (row df_index + 1), one coil around each core, in one air box.  The two
    magnets' boundaries share one grid (``magnets_mesh``).

    :return: ``[points, B, M_iron, M_coil, Q, J_tar]`` as the reference: the iron mass of the
        superconducting magnet only, the coil mass and power of its coil, and its target
        current density.
    """
    from .evaluators import evaluate_fem_solution_node_interpolation
    from .red_mvp_solver import RedMVPSolver

    row = df_index + 1
    material = str(np.asarray(parameters["material"])[row])
    reluctance_iron = Reluctance(os.path.join(materials_directory, material))
    with open(os.path.join(materials_directory, material)) as f:
        iron_material_data = json.load(f)
    with open(os.path.join(materials_directory, str(np.asarray(parameters["coil_material"])[row]))) as f:
        conductor_material_data = json.load(f)
    J_tar = _value(parameters, "J_tar(A/mm2)", row) * 1e6
    g1 = mag_1_parameters(parameters, df_index)
    g2 = mag_1_parameters(parameters, row)
    lim_x = max(g1["lim_x"], g2["lim_x"])
    lim_y = max(g1["lim_y"], g2["lim_y"])
    z_min, z_max = g1["z_min"], g2["z_max"]
    e1 = lambda g, keys: ([g[f"{k}_1"] for k in keys], [g[f"{k}_2"] for k in keys])
    x1 = e1(g1, ["X_mgap", "X_core", "X_void", "X_yoke"])
    y1 = e1(g1, ["Y_core", "Y_yoke"])
    x2 = e1(g2, ["X_core", "X_void", "X_yoke"])
    y2 = e1(g2, ["Y_core", "Y_void", "Y_yoke"])
    nc = Magnet(g1["Z_pos"], g1["Z_pos"] + g1["Z_len"], ["gap", "core", "void", "leg", "out"], *x1,
                ["low", "top", "out"], *y1, lambda X, Y: np.where(_tag_type_1(X, Y), TAG_NC, 0), lc)
    sc = Magnet(g2["Z_pos"], g2["Z_pos"] + g2["Z_len"], ["core", "void", "leg", "out"], *x2,
                ["low", "mid", "top", "out"], *y2, lambda X, Y: np.where(_tag_type_2(X, Y), M.TAG_IRON, 0), lc)
    msh = magnets_mesh([nc, sc], lim_x, lim_y, z_min, z_max, lc)
    vol = M.tet_volumes6(msh.nodes, msh.cells) / 6.0
    M_iron = 4 * float(vol[msh.elem_domain == M.TAG_IRON].sum()) * iron_material_data["density(g/m3)"]

    # coils (SHiP_functions.py:2427-2474): turns offset by spacer + insulation from each core
    coils = []
    for g in (g1, g2):
        slot = 2 * min(g["Y_core_1"], g["Y_core_2"])
        r, ins, sp = g["coil_radius"], g["ins"], g["yoke_spacer"]
        n = min(int(slot / 2 / (r + ins)), int(g["max_turns"]))
        if n < 1:
            raise ValueError("a slot holds no conductor")
        y = np.linspace(-0.5 * slot + r + ins, 0.5 * slot - r - ins, n)
        d = sp + ins
        X1, X2, Z1, Z2 = g["X_core_1"], g["X_core_2"], g["Z_pos"], g["Z_pos"] + g["Z_len"]
        kp = np.array([[-X2 - d, Z2], [-X2, Z2 + d], [X2, Z2 + d], [X2 + d, Z2], [X1 + d, Z1], [X1, Z1 - d],
                       [-X1, Z1 - d], [-X1 - d, Z1]])
        coils.append(RacetrackCoil(kp, y, r, g["current"] / n))
    perimeter = coils[1].get_length()
    current_2 = g2["current"]
    A_cu = abs(current_2) / J_tar
    M_coil = A_cu * perimeter * conductor_material_data["density(g/m3)"]
    Q = abs(current_2 * current_2) * perimeter * conductor_material_data["resistivity(Ohm.m)"] / A_cu

    iron_tags = [TAG_NC, M.TAG_IRON]
    solver = RedMVPSolver(msh, coils, iron_tags, [M.TAG_AIR], [reluctance_iron] * 2, quad_order=quad_order,
                          max_newton_iterations=50)
    solver.verbose = False
    x = solver.solve()
    field_density = int(max(0.5 * g1["field_density"], 0.5 * g2["field_density"]))
    points, B_i = solver.curl_curl_factory.compute_B(x, quad_order=field_density)
    B_coil = 0.0 * B_i
    for coil in coils:
        B_coil += coil.compute_B(points)
    if result_directory != "none":
        np.save(os.path.join(result_directory, "x" + result_spec + ".npy"), x)
    ret_vals = [points, B_i + B_coil, M_iron, M_coil, Q, J_tar]
    eval_pos = np.asarray(eval_pos, dtype=np.float64).reshape(-1, 3)
    if eval_pos.shape[0] > 0:
        B_tot = evaluate_fem_solution_node_interpolation(msh, eval_pos, solver, coils, x, iron_tags + [M.TAG_AIR])
        name = "B" + result_spec + ".csv"
        out = os.path.join(result_directory, name) if result_directory != "none" else name
        np.savetxt(out, np.append(eval_pos, B_tot, axis=1), delimiter=",", header="x(m),y(m),z(m),Bx(T),By(T),Bz(T)",
                   comments="")
    return ret_vals

