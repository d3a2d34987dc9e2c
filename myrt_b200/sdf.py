"""SDF programs: the reference's instruction tree (src/pathtracer/sdf.hpp:399-633)
serialised to the flat form the core evaluates.

The reference compiles an instruction tree into a GLSL map() per scene
(sdf.cpp:122-407). This core instead evaluates a flat post-order program per
SDF: modifier instructions move the position of the next primitive (innermost
modifier first), primitives push a distance and a material, operators pop two
and push one. Parameters live in one float buffer with the reference's block
layout per instruction type (float = 1 block, int = 1 block holding the value,
vec3 = 3 blocks).

    prog = smooth_union(translate(sphere(0.3, material=1), (0.2, 0, 0)), box((0.2, 0.1, 0.3)), k=0.1)
    lib = SdfLibrary(); idx = lib.add(prog)
    lib.instrs, lib.programs, lib.params   # -> Context.upload_sdf
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

SPHERE, BOX, TORUS, CAPSULE, MENGER = 1, 2, 3, 4, 5
UNION, SUBTRACTION, INTERSECTION, SMOOTH_UNION = 16, 17, 18, 19
TRANSLATE, MIRROR = 32, 33


@dataclass
class Node:
    op: int
    params: list
    children: list = field(default_factory=list)  # operators: [lhs, rhs]; primitives: []
    mods: list = field(default_factory=list)      # primitives: [(op, params)], innermost first


def sphere(radius: float = 1.0, material: int = 0) -> Node:
    return Node(SPHERE, [radius, material])


def box(size=(1.0, 1.0, 1.0), material: int = 0) -> Node:
    return Node(BOX, [*size, material])


def torus(radius_large: float = 1.0, radius_small: float = 0.2, material: int = 0) -> Node:
    return Node(TORUS, [radius_large, radius_small, material])


def vertical_capsule(height: float = 1.0, radius: float = 0.2, material: int = 0) -> Node:
    return Node(CAPSULE, [height, radius, material])


def menger_fractal(material: int = 0) -> Node:
    return Node(MENGER, [material])


def translate(prim: Node, offset) -> Node:
    """Evaluate `prim` at (p - offset). Applied after the modifiers already on it
    (the reference's `prim.child = translate(...)` chain, innermost first)."""
    prim.mods.insert(0, (TRANSLATE, list(offset)))
    return prim


def mirror_axis(prim: Node, axis: int) -> Node:
    prim.mods.insert(0, (MIRROR, [axis]))
    return prim


def union(a: Node, b: Node) -> Node:
    return Node(UNION, [], [a, b])


def subtraction(a: Node, b: Node) -> Node:
    return Node(SUBTRACTION, [], [a, b])


def intersection(a: Node, b: Node) -> Node:
    return Node(INTERSECTION, [], [a, b])


def smooth_union(a: Node, b: Node, k: float = 0.1) -> Node:
    return Node(SMOOTH_UNION, [k], [a, b])


class SdfLibrary:
    """Instructions, programs and parameters of a set of SDFs (sdf_index = order added)."""

    def __init__(self):
        self._instrs: list[tuple[int, int]] = []
        self._programs: list[tuple[int, int]] = []
        self._params: list[float] = []

    def _param(self, values) -> int:
        off = len(self._params)
        self._params.extend(float(v) for v in values)
        return off

    def _emit(self, root: Node):
        # post order without recursion (long folds nest thousands deep)
        todo = [(root, False)]
        while todo:
            n, expanded = todo.pop()
            if n.children and not expanded:
                todo.append((n, True))
                todo.append((n.children[1], False))
                todo.append((n.children[0], False))
                continue
            if not n.children:
                for op, params in n.mods:
                    self._instrs.append((op, self._param(params)))
            self._instrs.append((n.op, self._param(n.params)))

    def add(self, root: Node) -> int:
        first = len(self._instrs)
        self._emit(root)
        self._programs.append((first, len(self._instrs) - first))
        return len(self._programs) - 1

    @property
    def instrs(self) -> np.ndarray:
        return np.asarray(self._instrs, np.int32).reshape(-1, 2)

    @property
    def programs(self) -> np.ndarray:
        return np.asarray(self._programs, np.int32).reshape(-1, 2)

    @property
    def params(self) -> np.ndarray:
        return np.asarray(self._params, np.float32)


def sdf_drawables(transforms, sdf_indices) -> np.ndarray:
    """drawable_sdf_t records (src/pathtracer/scene.hpp:105-110) as float32 [N, 36]:
    column-major transformation, its inverse, sdf_index (int bits), 3 pad words."""
    out = np.zeros((len(sdf_indices), 36), np.float32)
    for i, (m, idx) in enumerate(zip(transforms, sdf_indices)):
        m = np.asarray(m, np.float64).reshape(4, 4)
        out[i, 0:16] = m.T.astype(np.float32).ravel()
        out[i, 16:32] = np.linalg.inv(m).T.astype(np.float32).ravel()
        out[i, 32:33] = np.array([idx], np.int32).view(np.float32)
    return out


def random_sdf_field(n_prims: int = 256, k: float = 0.1, seed: int = 3, extent: float = 1.0,
                     chain: bool = False) -> Node:
    """Smooth union of n seeded spheres, boxes and tori (the SDF + mesh hybrid
    configuration: 256 primitives, k = 0.1). chain=False folds them as a
    balanced tree, chain=True left to right (((p0 u p1) u p2) u ...), which
    lets the evaluator skip every primitive far from the point exactly."""
    rng = np.random.default_rng(seed)
    nodes = []
    for i in range(n_prims):
        kind = rng.integers(0, 3)
        c = rng.uniform(-extent, extent, 3)
        mat = int(rng.integers(0, 4))
        if kind == 0:
            p = sphere(float(rng.uniform(0.03, 0.12)), mat)
        elif kind == 1:
            p = box(tuple(rng.uniform(0.02, 0.1, 3)), mat)
        else:
            p = torus(float(rng.uniform(0.05, 0.12)), float(rng.uniform(0.01, 0.04)), mat)
        nodes.append(translate(p, c))
    if chain:
        acc = nodes[0]
        for nd in nodes[1:]:
            acc = smooth_union(acc, nd, k)
        return acc
    # balanced tree: depth log2(n), stack depth stays small
    while len(nodes) > 1:
        nxt = [smooth_union(nodes[i], nodes[i + 1], k) for i in range(0, len(nodes) - 1, 2)]
        if len(nodes) % 2:
            nxt.append(nodes[-1])
        nodes = nxt
    return nodes[0]
