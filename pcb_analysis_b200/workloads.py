"""Seeded synthetic boards: the benchmark workloads of the steady thermal solve.

There is no public board dataset for this path; these generators stand in for
boards of the shape the reference's production producer builds
(src/geometry/cad_import/adapters.py:173-228 of pcb-analysis: copper slabs
whose conductivity follows a copper fill pattern, FR-4 between them, pads as
heat sources, Newton cooling on both faces).  Every draw comes from
numpy.random.default_rng(seed).

Common to all: 0.25 mm pitch, FR-4 k = 0.3 W/mK (isotropic), copper k = 385
W/mK, copper slabs 35 um, 1.6 mm of FR-4 split evenly over the FR-4 slabs,
ambient 298.15 K, sources spread over squares of top-face nodes.

* ``board_c1``: 128 x 128 cells x 8 slabs (Cu, 6 FR-4, Cu); copper fill by
  random rectangles (side 2..20 cells) to >= 60 %; four 2 x 2 mm pads of 1 W;
  h = 10 W/m^2K top and bottom.  149,769 nodes.
* ``board_c2``: 512 x 512 x 12 (Cu, 3 FR-4, Cu, 2 FR-4, Cu, 3 FR-4, Cu); inner
  planes ~85 % (full plane minus random voids), outer layers seeded traces
  (width 1..4 cells) plus pads; 16 sources of U(0.1, 2) W; h = 10 / 10.
  3,421,197 nodes.
* ``board_c3``: 2048 x 2048 x 16, six copper slabs interleaved with ten FR-4
  slabs, per-layer fill U(0.4, 0.9); 64 sources of U(0.05, 5) W; h = 25 top,
  5 bottom; bottom-face nodes of columns 0..40 (a 10 mm edge strip) held at
  298.15 K.  71,370,417 nodes.
* ``batch_c4``: 64 boards, sides log-uniform in [96, 768] cells (rows and
  columns drawn independently), slabs uniform in [4, 12], c2 rules scaled.
* ``request_c5``: one served request: sides log-uniform in [64, 1024], slabs
  in [4, 16], random stackup, sources, h in {5, 10, 25}, optional fixed strip.
* ``dc_power_net``: the layered DC workload (the electrical package's
  solve_pcb_dc): a four-layer power distribution net of 1024 x 1024 cells at
  0.25 mm (4.2 M nodes): four planes with rectangular voids (35, 35, 17.5 and
  70 um; fill 0.9, 0.95, 0.8, 0.85), each kept to its largest connected piece
  of copper so that no island floats; 2000 stitching vias between random layer
  pairs; a regulator pad held at 1 V on the first plane, a ground pad held at
  0 V on the second, 16 loads of 3 x 3 nodes drawing U(0.1, 2) A.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Any

import numpy as np

PITCH_M = 0.25e-3
K_FR4 = 0.3
K_CU = 385.0
CU_THICKNESS_M = 35e-6
FR4_TOTAL_M = 1.6e-3
AMBIENT_K = 298.15


def _namespace(ns: Any | None):
    if ns is None:
        import pcb_analysis_b200.thermal as ns_local

        return ns_local
    return ns


def rectangle_fill(rng: np.random.Generator, rows: int, cols: int, target: float,
                   side: tuple[int, int] = (2, 20)) -> np.ndarray:
    """Boolean copper mask painted with random axis-aligned rectangles until >= target."""

    mask = np.zeros((rows, cols), dtype=bool)
    mean_area = ((side[0] + side[1]) / 2.0) ** 2
    while mask.mean() < target:
        missing = (target - mask.mean()) * rows * cols
        count = max(16, int(1.5 * missing / mean_area))
        h = rng.integers(side[0], side[1] + 1, count)
        w = rng.integers(side[0], side[1] + 1, count)
        r0 = rng.integers(0, rows, count)
        c0 = rng.integers(0, cols, count)
        r1 = np.minimum(r0 + h, rows)
        c1 = np.minimum(c0 + w, cols)
        diff = np.zeros((rows + 1, cols + 1), dtype=np.int32)
        np.add.at(diff, (r0, c0), 1)
        np.add.at(diff, (r0, c1), -1)
        np.add.at(diff, (r1, c0), -1)
        np.add.at(diff, (r1, c1), 1)
        mask |= np.cumsum(np.cumsum(diff, axis=0), axis=1)[:rows, :cols] > 0
    return mask


def plane_with_voids(rng: np.random.Generator, rows: int, cols: int, fill: float) -> np.ndarray:
    """A full copper plane with random rectangular voids down to about ``fill``."""

    return ~rectangle_fill(rng, rows, cols, 1.0 - fill, side=(2, 12))


def traces(rng: np.random.Generator, rows: int, cols: int, target: float) -> np.ndarray:
    """Long thin rectangles (width 1..4 cells, length 10..cols/4) until >= target."""

    mask = np.zeros((rows, cols), dtype=bool)
    longest = max(11, min(rows, cols) // 4)
    while mask.mean() < target:
        horizontal = rng.random() < 0.5
        width = int(rng.integers(1, 5))
        length = int(rng.integers(10, longest + 1))
        if horizontal:
            r, c = int(rng.integers(0, rows)), int(rng.integers(0, cols))
            mask[r : r + width, c : c + length] = True
        else:
            r, c = int(rng.integers(0, rows)), int(rng.integers(0, cols))
            mask[r : r + length, c : c + width] = True
    return mask


def _pad_nodes(z: int, r: int, c: int, size: int) -> tuple[tuple[int, int, int], ...]:
    return tuple((z, r + i, c + j) for i in range(size + 1) for j in range(size + 1))


def _sources(ns, rng, rows, cols, slabs, count, power_low, power_high, pad_cells=None, fixed_power=None):
    sources = []
    for k in range(count):
        size = pad_cells if pad_cells is not None else int(rng.integers(2, 9))
        size = min(size, rows, cols)
        r = int(rng.integers(0, rows - size + 1))
        c = int(rng.integers(0, cols - size + 1))
        power = fixed_power if fixed_power is not None else float(rng.uniform(power_low, power_high))
        sources.append(ns.HeatSource(_pad_nodes(slabs, r, c, size), power, f"pad{k}"))
    return tuple(sources)


@dataclass(frozen=True)
class Stackup:
    copper: tuple[bool, ...]  # per slab, bottom to top

    @property
    def thickness_m(self) -> tuple[float, ...]:
        fr4 = sum(1 for c in self.copper if not c)
        t_fr4 = FR4_TOTAL_M / max(fr4, 1)
        return tuple(CU_THICKNESS_M if c else t_fr4 for c in self.copper)


def _board(ns, rows, cols, stackup: Stackup, layers: dict[int, np.ndarray], sources, h_top, h_bottom,
           fixed_mask=None):
    slabs = len(stackup.copper)
    k = np.full((slabs, rows, cols), K_FR4)
    for z, mask in layers.items():
        k[z] = np.where(mask, K_CU, K_FR4)
    mesh = ns.LayeredThermalMesh(
        slab_thickness_m=stackup.thickness_m,
        pitch_x_m=PITCH_M,
        pitch_y_m=PITCH_M,
        conductivity_w_per_m_k=k,
    )
    convection = []
    if h_top > 0:
        convection.append(ns.ConvectionBoundary("top", float(h_top), AMBIENT_K))
    if h_bottom > 0:
        convection.append(ns.ConvectionBoundary("bottom", float(h_bottom), AMBIENT_K))
    kwargs = {}
    if fixed_mask is not None:
        kwargs = dict(fixed_temperature_mask=fixed_mask, fixed_temperature_k=AMBIENT_K)
    return ns.ThermalConductionProblem(mesh, convection=tuple(convection), heat_sources=sources, **kwargs)


def board_c1(seed: int = 0, ns: Any | None = None, rows: int = 128, cols: int = 128):
    ns = _namespace(ns)
    rng = np.random.default_rng(seed)
    stackup = Stackup((True,) + (False,) * 6 + (True,))
    layers = {0: rectangle_fill(rng, rows, cols, 0.60), 7: rectangle_fill(rng, rows, cols, 0.60)}
    sources = _sources(ns, rng, rows, cols, 8, 4, 1.0, 1.0, pad_cells=8, fixed_power=1.0)
    return _board(ns, rows, cols, stackup, layers, sources, 10.0, 10.0)


def _c2_stackup() -> Stackup:
    c, f = True, False
    return Stackup((c, f, f, f, c, f, f, c, f, f, f, c))


def board_c2(seed: int = 0, ns: Any | None = None, rows: int = 512, cols: int = 512):
    ns = _namespace(ns)
    rng = np.random.default_rng(seed)
    stackup = _c2_stackup()
    slabs = len(stackup.copper)
    layers = {}
    for z, cu in enumerate(stackup.copper):
        if not cu:
            continue
        if z in (0, slabs - 1):
            layers[z] = traces(rng, rows, cols, 0.25) | rectangle_fill(rng, rows, cols, 0.10, side=(4, 12))
        else:
            layers[z] = plane_with_voids(rng, rows, cols, 0.85)
    sources = _sources(ns, rng, rows, cols, slabs, 16, 0.1, 2.0)
    return _board(ns, rows, cols, stackup, layers, sources, 10.0, 10.0)


def board_c3(seed: int = 0, ns: Any | None = None, rows: int = 2048, cols: int = 2048):
    ns = _namespace(ns)
    rng = np.random.default_rng(seed)
    slabs = 16
    cu_at = {0, 3, 6, 9, 12, 15}
    stackup = Stackup(tuple(z in cu_at for z in range(slabs)))
    layers = {z: rectangle_fill(rng, rows, cols, float(rng.uniform(0.4, 0.9))) for z in sorted(cu_at)}
    sources = _sources(ns, rng, rows, cols, slabs, 64, 0.05, 5.0)
    fixed = np.zeros((slabs + 1, rows + 1, cols + 1), dtype=bool)
    fixed[0, :, : min(41, cols + 1)] = True  # 10 mm strip on the bottom face
    return _board(ns, rows, cols, stackup, layers, sources, 25.0, 5.0, fixed_mask=fixed)


def _random_stackup(rng: np.random.Generator, slabs: int) -> Stackup:
    copper = [False] * slabs
    copper[0] = copper[-1] = True
    inner = [z for z in range(1, slabs - 1)]
    for z in inner:
        if rng.random() < 0.3:
            copper[z] = True
    return Stackup(tuple(copper))


def board_random(seed: int, ns: Any | None = None, *, side: tuple[int, int] = (96, 768), slabs: tuple[int, int] = (4, 12),
                 h_choices: tuple[float, ...] = (10.0,), fixed_strip: bool = False):
    """One board drawn by the c4 / c5 rules."""

    ns = _namespace(ns)
    rng = np.random.default_rng(seed)
    lo, hi = math.log(side[0]), math.log(side[1])
    rows = int(round(math.exp(rng.uniform(lo, hi))))
    cols = int(round(math.exp(rng.uniform(lo, hi))))
    nz = int(rng.integers(slabs[0], slabs[1] + 1))
    stackup = _random_stackup(rng, nz)
    layers = {}
    for z, cu in enumerate(stackup.copper):
        if not cu:
            continue
        if z in (0, nz - 1):
            layers[z] = traces(rng, rows, cols, 0.2) | rectangle_fill(rng, rows, cols, 0.10, side=(3, 10))
        else:
            layers[z] = plane_with_voids(rng, rows, cols, float(rng.uniform(0.75, 0.9)))
    area_scale = rows * cols / (512.0 * 512.0)
    count = max(2, int(round(16 * area_scale)))
    sources = _sources(ns, rng, rows, cols, nz, count, 0.1, 2.0)
    h_top = float(rng.choice(h_choices))
    h_bottom = float(rng.choice(h_choices))
    fixed = None
    if fixed_strip and rng.random() < 0.5:
        fixed = np.zeros((nz + 1, rows + 1, cols + 1), dtype=bool)
        fixed[0, :, : min(41, cols + 1)] = True
    return _board(ns, rows, cols, stackup, layers, sources, h_top, h_bottom, fixed_mask=fixed)


def batch_c4(seed: int = 0, count: int = 64, ns: Any | None = None):
    return [board_random(seed * 1000 + i, ns) for i in range(count)]


def request_c5(seed: int, ns: Any | None = None):
    return board_random(seed, ns, side=(64, 1024), slabs=(4, 16), h_choices=(5.0, 10.0, 25.0), fixed_strip=True)


def dc_power_net(seed: int = 0, ns: Any | None = None, rows: int = 1024, cols: int = 1024, vias: int = 2000):
    """The layered DC workload: a seeded four-layer power net (see the module notes)."""

    if ns is None:
        from . import electrical as ns  # noqa: N813
    from scipy import ndimage

    rng = np.random.default_rng(seed)
    planes = []
    for fill in (0.9, 0.95, 0.8, 0.85):
        plane = plane_with_voids(rng, rows, cols, fill)
        # elements sharing a corner node are coupled: 8-connected pieces
        labels, count = ndimage.label(plane, structure=np.ones((3, 3), dtype=int))
        sizes = np.bincount(labels.reshape(-1), minlength=count + 1)
        sizes[0] = 0
        planes.append(labels == int(np.argmax(sizes)))
    active = np.stack(planes)
    mesh = ns.LayeredPCBMesh(element_active=active, layer_thickness_m=(35e-6, 35e-6, 17.5e-6, 70e-6),
                             pitch_x_m=PITCH_M, pitch_y_m=PITCH_M)
    # terminals only on copper: nodes of active elements
    copper = np.zeros((4, rows + 1, cols + 1), dtype=bool)
    for dy in (0, 1):
        for dx in (0, 1):
            copper[:, dy : dy + rows, dx : dx + cols] |= active
    pad = 8
    regulator = tuple((0, y, x) for y in range(rows // 2 - pad, rows // 2 + pad) for x in range(0, pad)
                      if copper[0, y, x])
    ground = tuple((1, y, x) for y in range(0, pad) for x in range(cols + 1 - pad, cols + 1) if copper[1, y, x])
    taken = set(regulator) | set(ground)
    loads = []
    for k in range(16):
        while True:
            y0, x0 = int(rng.integers(pad, rows - 2 * pad)), int(rng.integers(pad, cols - 2 * pad))
            nodes = tuple((0, y, x) for y in range(y0, y0 + 3) for x in range(x0, x0 + 3))
            if not taken.intersection(nodes) and all(copper[node] for node in nodes):
                break
        taken.update(nodes)
        loads.append(ns.CurrentTerminal(nodes, -float(rng.uniform(0.1, 2.0)), f"load{k}"))
    links = []
    used = set(taken)
    while len(links) < vias:
        y, x = int(rng.integers(0, rows + 1)), int(rng.integers(0, cols + 1))
        lower, upper = sorted(rng.choice(4, size=2, replace=False).tolist())
        if (lower, y, x) in used or (upper, y, x) in used:
            continue
        if not (copper[lower, y, x] and copper[upper, y, x]):  # a via joins copper to copper
            continue
        used.update({(lower, y, x), (upper, y, x)})
        links.append(ns.ViaConnection((lower, y, x), (upper, y, x), float(rng.uniform(0.5e-3, 2e-3))))
    return ns.PCBConductionProblem(
        mesh=mesh, terminals=tuple(loads), vias=tuple(links),
        voltage_terminals=(ns.VoltageTerminal(regulator, 1.0, "vrm"), ns.VoltageTerminal(ground, 0.0, "gnd")),
    )
