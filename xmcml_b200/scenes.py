"""Synthetic tissue models in the reference's input format (XML model + binary .surface file).

The reference ships no benchmark inputs for its transport path, so the workloads are generated
here from their stated shapes: planar layer stacks, triangulated height fields
z = d + A sin(2 pi x / lam) sin(2 pi y / lam), and triangulated ellipsoids. Each Scene writes the
XML element set read by ParseInputFile (base/xmcml/xmcmlLauncher/parser.cpp:18-514) and the
.surface layout read by ParseSurfaceFile (parser.cpp:516-611).
"""
from __future__ import annotations

import math
import os
import struct
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

# speed of light in mm/ps: time bins are optical path length in mm (time += step * n)
C_MM_PER_PS = 0.299792458


@dataclass
class Layer:
    n: float
    mua: float = 0.0
    mus: float = 0.0
    g: float = 0.0
    surfaces: List[int] = field(default_factory=list)


@dataclass
class Ring:
    r0: float
    r1: float
    center: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    filter: Optional[List[int]] = None
    angle: Optional[float] = None


@dataclass
class Cube:
    center: Tuple[float, float, float]
    length: Tuple[float, float, float]
    filter: Optional[List[int]] = None
    angle: Optional[float] = None


@dataclass
class Scene:
    layers: List[Layer]
    surfaces: List[Tuple[np.ndarray, np.ndarray]]  # (vertices [N,3] f64, triangles [M,3] i32)
    area_corner: Tuple[float, float, float]
    area_length: Tuple[float, float, float]
    area_partitions: Tuple[int, int, int]
    photons: int = 1000
    min_weight: float = 1e-4
    rings: List[Ring] = field(default_factory=list)
    cubes: List[Cube] = field(default_factory=list)
    time_start: Optional[float] = None
    time_finish: Optional[float] = None
    time_bins: Optional[int] = None
    start_position: Optional[Tuple[float, float, float]] = None
    start_direction: Optional[Tuple[float, float, float]] = None
    target_layers: Optional[List[int]] = None
    # <Biasing>: attractive point (integers: the reference parses it with atoi) and weight integral
    bias_target: Optional[Tuple[int, int, int]] = None
    bias_factor: float = 1.0
    bias_integral_precision: int = 128
    bias_table_precision: int = 262144
    name: str = "scene"

    # ------------------------------------------------------------------ writers
    def xml(self) -> str:
        out = ['<?xml version="1.0"?>', "<Input>", f"    <NumberOfPhotons>{int(self.photons)}</NumberOfPhotons>",
               f"    <MinWeight>{self.min_weight!r}</MinWeight>"]
        if self.time_start is not None:
            out.append(f"    <TimeStart>{self.time_start!r}</TimeStart>")
        if self.time_finish is not None:
            out.append(f"    <TimeFinish>{self.time_finish!r}</TimeFinish>")
        if self.time_bins is not None:
            out.append(f"    <TimeScaleSize>{int(self.time_bins)}</TimeScaleSize>")
        if self.target_layers:
            out.append("    <TargetRange>")
            out += [f"        <Layer>{int(l)}</Layer>" for l in self.target_layers]
            out.append("    </TargetRange>")

        def xyz(tag, v, ind="    "):
            return [f"{ind}<{tag}>", f"{ind}    <X>{v[0]!r}</X>", f"{ind}    <Y>{v[1]!r}</Y>",
                    f"{ind}    <Z>{v[2]!r}</Z>", f"{ind}</{tag}>"]

        if self.bias_target is not None:
            out += ["    <Biasing>", "        <WeightIntegral>",
                    f"            <IntegralPrecision>{int(self.bias_integral_precision)}</IntegralPrecision>",
                    f"            <TablePrecision>{int(self.bias_table_precision)}</TablePrecision>",
                    f"            <AttractiveFactor>{float(self.bias_factor)!r}</AttractiveFactor>",
                    "        </WeightIntegral>", "        <TargetPoint>"]
            out += [f"            <{a}>{int(v)}</{a}>" for a, v in zip("XYZ", self.bias_target)]
            out += ["        </TargetPoint>", "    </Biasing>"]
        if self.start_position is not None:
            out += xyz("StartPosition", [float(x) for x in self.start_position])
        if self.start_direction is not None:
            out += xyz("StartDirection", [float(x) for x in self.start_direction])
        out.append("    <Area>")
        out += xyz("Corner", [float(x) for x in self.area_corner], "        ")
        out += xyz("Length", [float(x) for x in self.area_length], "        ")
        out += ["        <PartitionNumber>", f"            <X>{int(self.area_partitions[0])}</X>",
                f"            <Y>{int(self.area_partitions[1])}</Y>", f"            <Z>{int(self.area_partitions[2])}</Z>",
                "        </PartitionNumber>", "    </Area>"]
        out.append(f"    <NumberOfLayers>{len(self.layers)}</NumberOfLayers>")
        out.append("    <Layers>")
        for L in self.layers:
            out += ["        <Layer>", f"            <RefractiveIndex>{L.n!r}</RefractiveIndex>",
                    f"            <AbsorptionCoefficient>{L.mua!r}</AbsorptionCoefficient>",
                    f"            <ScatteringCoefficient>{L.mus!r}</ScatteringCoefficient>",
                    f"            <Anisotropy>{L.g!r}</Anisotropy>",
                    f"            <NumberOfSurfaces>{len(L.surfaces)}</NumberOfSurfaces>", "            <SurfaceIds>"]
            out += [f"                <Id>{int(s)}</Id>" for s in L.surfaces]
            out += ["            </SurfaceIds>", "        </Layer>"]
        out.append("    </Layers>")
        if self.cubes:
            out.append(f"    <NumberOfCubeDetectors>{len(self.cubes)}</NumberOfCubeDetectors>")
            out.append("    <CubeDetectors>")
            for c in self.cubes:
                out.append("        <CubeDetector>")
                out += xyz("Center", [float(x) for x in c.center], "            ")
                out += xyz("Length", [float(x) for x in c.length], "            ")
                if c.filter is not None:
                    out += ["            <Filter>"] + [f"                <Layer>{int(l)}</Layer>" for l in c.filter] + ["            </Filter>"]
                if c.angle is not None:
                    out.append(f"            <TargetAngle>{c.angle!r}</TargetAngle>")
                out.append("        </CubeDetector>")
            out.append("    </CubeDetectors>")
        if self.rings:
            out.append(f"    <NumberOfRingDetectors>{len(self.rings)}</NumberOfRingDetectors>")
            out.append("    <RingDetectors>")
            for r in self.rings:
                out.append("        <RingDetector>")
                out += xyz("Center", [float(x) for x in r.center], "            ")
                out += [f"            <SmallRadius>{r.r0!r}</SmallRadius>", f"            <BigRadius>{r.r1!r}</BigRadius>"]
                if r.filter is not None:
                    out += ["            <Filter>"] + [f"                <Layer>{int(l)}</Layer>" for l in r.filter] + ["            </Filter>"]
                if r.angle is not None:
                    out.append(f"            <TargetAngle>{r.angle!r}</TargetAngle>")
                out.append("        </RingDetector>")
            out.append("    </RingDetectors>")
        out.append(f"    <NumberOfSurfaces>{len(self.surfaces)}</NumberOfSurfaces>")
        out.append("</Input>")
        return "\n".join(out) + "\n"

    def surface_bytes(self) -> bytes:
        parts = [struct.pack("<Ii", 0x0100, len(self.surfaces))]
        for v, t in self.surfaces:
            v = np.ascontiguousarray(v, dtype="<f8")
            t = np.ascontiguousarray(t, dtype="<i4")
            parts.append(struct.pack("<i", v.shape[0]))
            parts.append(v.tobytes())
            parts.append(struct.pack("<i", t.shape[0]))
            parts.append(t.tobytes())
        return b"".join(parts)

    def write(self, directory: str, stem: Optional[str] = None) -> Tuple[str, str]:
        os.makedirs(directory, exist_ok=True)
        stem = stem or self.name
        xml_path = os.path.join(directory, stem + ".xml")
        surf_path = os.path.join(directory, stem + ".surface")
        with open(xml_path, "w") as f:
            f.write(self.xml())
        with open(surf_path, "wb") as f:
            f.write(self.surface_bytes())
        return xml_path, surf_path

    @property
    def n_triangles(self) -> int:
        return int(sum(t.shape[0] for _, t in self.surfaces))


# ---------------------------------------------------------------------- meshes

def plane(z: float, half: float = 100.0, cx: float = 0.0, cy: float = 0.0) -> Tuple[np.ndarray, np.ndarray]:
    """Square z = const made of two triangles."""
    v = np.array([[cx - half, cy - half, z], [cx + half, cy - half, z], [cx + half, cy + half, z],
                  [cx - half, cy + half, z]], dtype=np.float64)
    t = np.array([[0, 1, 2], [0, 2, 3]], dtype=np.int32)
    return v, t


def height_field(z0: float, amp: float, lam: float, n: int = 256, half: float = 10.0,
                 offset: float = 0.0) -> Tuple[np.ndarray, np.ndarray]:
    """n x n vertex grid over [-half, half]^2 (shifted by `offset`), z = z0 + amp sin(2 pi x/lam) sin(2 pi y/lam),
    2 (n-1)^2 triangles."""
    xs = np.linspace(-half, half, n) + offset
    X, Y = np.meshgrid(xs, xs, indexing="xy")
    Z = z0 + amp * np.sin(2 * np.pi * X / lam) * np.sin(2 * np.pi * Y / lam)
    v = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1).astype(np.float64)
    i = np.arange(n - 1)
    I, J = np.meshgrid(i, i, indexing="xy")
    a = (J * n + I).ravel()
    b = a + 1
    c = a + n + 1
    d = a + n
    t = np.concatenate([np.stack([a, b, c], 1), np.stack([a, c, d], 1)]).astype(np.int32)
    return v, t


def ellipsoid(center: Sequence[float], semi: Sequence[float], subdiv: int = 6) -> Tuple[np.ndarray, np.ndarray]:
    """Icosphere with `subdiv` midpoint subdivisions mapped to an ellipsoid (20 * 4^subdiv triangles)."""
    p = (1 + 5 ** 0.5) / 2
    verts = [(-1, p, 0), (1, p, 0), (-1, -p, 0), (1, -p, 0), (0, -1, p), (0, 1, p), (0, -1, -p), (0, 1, -p),
             (p, 0, -1), (p, 0, 1), (-p, 0, -1), (-p, 0, 1)]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
             (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    V = [np.array(v, dtype=np.float64) / np.linalg.norm(v) for v in verts]
    F = faces
    for _ in range(subdiv):
        cache = {}
        nf = []

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = V[a] + V[b]
                V.append(m / np.linalg.norm(m))
                cache[key] = len(V) - 1
            return cache[key]

        for a, b, c in F:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        F = nf
    v = np.array(V) * np.asarray(semi, dtype=np.float64) + np.asarray(center, dtype=np.float64)
    return v, np.array(F, dtype=np.int32)


# ---------------------------------------------------------------------- workloads

# Optical properties of the 3-layer tissue: (thickness mm, mua, mus, g, n)
THREE_LAYER = [(0.1, 0.3, 10.0, 0.8, 1.4), (1.0, 0.05, 20.0, 0.9, 1.4), (50.0, 0.02, 15.0, 0.85, 1.37)]


def rings(count: int, width: float) -> List[Ring]:
    return [Ring(i * width, (i + 1) * width) for i in range(count)]


def planar(props=THREE_LAYER, photons: int = 10 ** 6, ambient_n: float = 1.0, n_rings: int = 50,
           ring_width: float = 0.1, area_corner=(-5.0, -5.0, 0.0), area_length=(10.0, 10.0, 5.0),
           area_partitions=(100, 100, 100), time_bins=None, time_finish=None, min_weight: float = 1e-4,
           half: float = 100.0, name: str = "planar") -> Scene:
    """Pencil beam at normal incidence into a stack of planar layers (planes at the cumulative depths).

    With the default arguments this is the 3-layer configuration: L1 0.1 mm (mua 0.3, mus 10, g 0.8,
    n 1.4), L2 1.0 mm (0.05, 20, 0.9, 1.4), L3 50 mm (0.02, 15, 0.85, 1.37), absorption grid
    100x100x100 over a 10x10x5 mm box, 50 rings of 0.1 mm, 1e6 photons."""
    zs = np.concatenate([[0.0], np.cumsum([p[0] for p in props])])
    surfaces = [plane(float(z), half) for z in zs]
    nl = len(props)
    layers = [Layer(ambient_n, 0.0, 0.0, 0.0, [0, nl])]
    for i, (_, mua, mus, g, n) in enumerate(props):
        layers.append(Layer(n, mua, mus, g, [i, i + 1]))
    sc = Scene(layers, surfaces, area_corner, area_length, area_partitions, photons=photons,
               min_weight=min_weight, rings=rings(n_rings, ring_width), name=name)
    if time_bins is not None:
        sc.time_start, sc.time_finish, sc.time_bins = 0.0, float(time_finish), int(time_bins)
    return sc


def height_field_tissue(photons: int = 10 ** 7, grid: int = 256, half: float = 10.0, amp: float = 0.05,
                        lam: float = 2.0, n_rings: int = 50, ring_width: float = 0.1, time_bins: int = 200,
                        bin_ps: float = 5.0, area_partitions=(100, 100, 100), name: str = "heightfield") -> Scene:
    """The 3 layers with the top two boundaries triangulated height fields on a grid x grid vertex mesh
    over (2 half)^2 mm (2 (grid-1)^2 triangles each), z = d + amp sin(2 pi x/lam) sin(2 pi y/lam);
    the L2/L3 boundary and the bottom are planes. 50 rings of 0.1 mm and `time_bins` bins of `bin_ps`
    ps of optical path length (TimeFinish = bins * bin_ps * c). Area: inside the mesh footprint, from
    z = -0.1 to 9.9 mm."""
    d = [0.0, 0.1, 1.1, 51.1]
    # shift the vertex grid by half a cell for an even vertex count so the beam point (0, 0) is a
    # mesh vertex lying exactly on z = d0: otherwise the beam enters on a cell diagonal where the
    # triangulated surface is above z = 0 and the start point (z = 1e-8) lies outside the tissue
    cell = 2 * half / (grid - 1)
    off = cell / 2 if grid % 2 == 0 else 0.0
    surfaces = [height_field(d[0], amp, lam, grid, half, off), height_field(d[1], amp, lam, grid, half, off),
                plane(d[2], half + cell), plane(d[3], half + cell)]
    layers = [Layer(1.0, 0, 0, 0, [0, 3])]
    for i, (_, mua, mus, g, n) in enumerate(THREE_LAYER):
        layers.append(Layer(n, mua, mus, g, [i, i + 1]))
    inner = half - 2 * cell  # Area inside the mesh footprint
    sc = Scene(layers, surfaces, (-inner, -inner, -0.1), (2 * inner, 2 * inner, 10.0), area_partitions, photons=photons,
               min_weight=1e-4, rings=rings(n_rings, ring_width), name=name)
    sc.time_start = 0.0
    sc.time_finish = time_bins * bin_ps * C_MM_PER_PS
    sc.time_bins = time_bins
    return sc


def ellipsoid_target(photons: int = 10 ** 9, subdiv: int = 6, n_rings: int = 100, ring_width: float = 0.1,
                     time_bins: int = 200, bin_ps: float = 5.0, name: str = "ellipsoid") -> Scene:
    """3-layer planar tissue with an embedded triangulated ellipsoid target (semi-axes 2 x 2 x 1 mm,
    centre depth 2.5 mm, mua 0.5, mus 12, g 0.9, n 1.4) inside L3; absorption grid 256x256x128 over
    20x20x10 mm; 100 rings x 200 time bins. subdiv=6 gives 81,920 triangles (subdiv 5: 20,480)."""
    d = [0.0, 0.1, 1.1, 51.1]
    surfaces = [plane(z, 100.0) for z in d] + [ellipsoid((0.0, 0.0, 2.5), (2.0, 2.0, 1.0), subdiv)]
    layers = [Layer(1.0, 0, 0, 0, [0, 3])]
    for i, (_, mua, mus, g, n) in enumerate(THREE_LAYER):
        sids = [i, i + 1] + ([4] if i == 2 else [])
        layers.append(Layer(n, mua, mus, g, sids))
    layers.append(Layer(1.4, 0.5, 12.0, 0.9, [4]))
    sc = Scene(layers, surfaces, (-10.0, -10.0, 0.0), (20.0, 20.0, 10.0), (256, 256, 128), photons=photons,
               min_weight=1e-4, rings=rings(n_rings, ring_width), name=name)
    sc.time_start = 0.0
    sc.time_finish = time_bins * bin_ps * C_MM_PER_PS
    sc.time_bins = time_bins
    sc.target_layers = [4]
    return sc
