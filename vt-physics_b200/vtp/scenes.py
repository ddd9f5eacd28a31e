"""Seeded synthetic particle scenes.

The lattice generators restate the arithmetic of the reference's scene
generators so that particle counts and unjittered coordinates are identical:

* ``cube``  follows ``ModelHandler::generateParticleCubeElements``
  (Simulator/Library/Source/Model/ModelHandler.cpp:43-67): FP32 running sums
  ``x += diameter`` starting at ``lb + r``, loop order z (outer), y, x (inner).
* ``box``   follows ``ModelHandler::generateParticleBoxElements``
  (ModelHandler.cpp:124-154): per-axis counts ``int((size + r) / (2.0 r))``,
  indices ``0..n`` inclusive, a particle is kept when it lies in the first
  ``layerNum`` or the last ``layerNum + 1`` index layers of any axis, loop
  order x (outer), y, z (inner), coordinates computed in double and rounded
  to float.

Jitter is the project's own: SplitMix64 per scene seed, one uniform draw per
component in generation order, ``(2u - 1) * a * spacing`` added in double and
rounded to float32.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

EPM_FLUID = 0
EPM_BOUNDARY = 1

_MASK64 = (1 << 64) - 1


def splitmix64_uniform(seed: int, count: int) -> np.ndarray:
    """``count`` doubles in [0, 1) from SplitMix64 started at ``seed``."""
    idx = np.arange(1, count + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = (np.uint64(seed & _MASK64) + idx * np.uint64(0x9E3779B97F4A7C15))
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def _f32_run(start: np.float32, limit: np.float32, step: np.float32) -> np.ndarray:
    vals = []
    v = np.float32(start)
    while v < limit:
        vals.append(v)
        v = np.float32(v + step)
    return np.array(vals, dtype=np.float32)


def cube(r: float, lb, size) -> np.ndarray:
    """Lattice cube, same count and coordinates as the reference generator."""
    r = np.float32(r)
    lb = [np.float32(v) for v in lb]
    size = [np.float32(v) for v in size]
    d = np.float32(2 * r)
    xs = _f32_run(np.float32(r + lb[0]), np.float32(lb[0] + size[0]), d)
    ys = _f32_run(np.float32(r + lb[1]), np.float32(lb[1] + size[1]), d)
    zs = _f32_run(np.float32(r + lb[2]), np.float32(lb[2] + size[2]), d)
    z, y, x = np.meshgrid(zs, ys, xs, indexing="ij")
    return np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1).astype(np.float32)


def box(r: float, lb, size, layer_num: int) -> np.ndarray:
    """Hollow box shell, same count and coordinates as the reference generator."""
    r32 = np.float32(r)
    lb = [np.float32(v) for v in lb]
    size = [np.float32(v) for v in size]
    n = [int(float(np.float32(size[a] + r32)) / (2.0 * float(r32))) for a in range(3)]
    axes = []
    for a in range(3):
        base = float(np.float32(lb[a] + r32))
        idx = np.arange(n[a] + 1, dtype=np.float64)
        axes.append((base + 2.0 * float(r32) * idx).astype(np.float32))
    I, J, K = np.meshgrid(np.arange(n[0] + 1), np.arange(n[1] + 1), np.arange(n[2] + 1), indexing="ij")
    L = layer_num
    keep = ((I < L) | (I >= n[0] - L) | (J < L) | (J >= n[1] - L) | (K < L) | (K >= n[2] - L))
    pts = np.stack([axes[0][I[keep]], axes[1][J[keep]], axes[2][K[keep]]], axis=1)
    return pts.astype(np.float32)


def jitter(pos: np.ndarray, amplitude: float, spacing: float, seed: int) -> np.ndarray:
    """Add SplitMix64 jitter of +-amplitude*spacing per component (double, then float32)."""
    if amplitude == 0.0:
        return pos.astype(np.float32).copy()
    u = splitmix64_uniform(seed, pos.size).reshape(pos.shape)
    return (pos.astype(np.float64) + (2.0 * u - 1.0) * amplitude * spacing).astype(np.float32)


@dataclass
class SceneObject:
    """One attached object: particles plus the reference's per-object configs."""
    name: str
    pos: np.ndarray                      # (n, 3) float32
    material: int                        # EPM_FLUID / EPM_BOUNDARY
    velocity_start: tuple = (0.0, 0.0, 0.0)
    color_start: tuple = (0.0, 0.0, 0.0)
    export_flag: bool = False
    phase_fraction: tuple | None = None  # IMM / IMM-CT only
    velocity: np.ndarray | None = None   # optional per-particle initial velocity (n, 3)

    @property
    def n(self) -> int:
        return int(self.pos.shape[0])


@dataclass
class Scene:
    solver: str                          # "PBF" | "DFSPH" | "IMM" | "IMMCT"
    config: dict
    objects: list = field(default_factory=list)

    @property
    def n_total(self) -> int:
        return sum(o.n for o in self.objects)

    @property
    def n_fluid(self) -> int:
        return sum(o.n for o in self.objects if o.material == EPM_FLUID)

    @property
    def n_boundary(self) -> int:
        return sum(o.n for o in self.objects if o.material == EPM_BOUNDARY)


def _export_block():
    return {"Common": {"exportTargetDir": "out", "exportFilePrefix": "obj", "exportFileType": "PLY"},
            "SolverRequired": {"enable": False, "exportFps": 35, "exportGroupPolicy": "MERGE"}}


def pbf_config(*, dt, r, lb, size, iterations=4, xsph_k=0.01, rho_f=1000.0, rho_b=1000.0,
               gravity=(0.0, -9.81, 0.0), max_nbr=60, animation_time=10.0):
    return {"PBF": {"Required": {"animationTime": animation_time, "timeStep": dt, "particleRadius": r,
                                 "simSpaceLB": list(lb), "simSpaceSize": list(size),
                                 "maxNeighborNum": max_nbr, "iterationNum": iterations, "XSPH_k": xsph_k,
                                 "fPartRestDensity": rho_f, "bPartRestDensity": rho_b},
                    "Optional": {"enable": True, "gravity": list(gravity)}},
            "EXPORT": _export_block()}


def dfsph_config(*, dt, r, lb, size, rho_f=1000.0, rho_b=1000.0, viscosity=1e-6, div_thr=1e-3,
                 incomp_thr=1e-3, tension=0.0, gravity=(0.0, -9.81, 0.0), max_nbr=60, animation_time=10.0):
    return {"DFSPH": {"Required": {"animationTime": animation_time, "timeStep": dt, "particleRadius": r,
                                   "simSpaceLB": list(lb), "simSpaceSize": list(size),
                                   "maxNeighborNum": max_nbr, "fPartRestDensity": rho_f,
                                   "bPartRestDensity": rho_b, "fPartRestViscosity": viscosity,
                                   "divFreeThreshold": div_thr, "incompThreshold": incomp_thr,
                                   "surfaceTensionCoefficient": tension},
                      "Optional": {"enable": True, "gravity": list(gravity)}},
            "EXPORT": _export_block()}


def pbf_dam_break(seed: int = 1001, jitter_amp: float = 0.1) -> Scene:
    """PBF dam break: 20x40x20 fluid lattice (16,000) in a 2-layer box (35,315), h = 0.04."""
    r = 0.01
    fluid = jitter(cube(r, (0.04, 0.04, 0.04), (0.4, 0.8, 0.4)), jitter_amp, 2 * r, seed)
    wall = box(r, (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), 2)
    cfg = pbf_config(dt=1.0 / 240.0, r=r, lb=(-0.1, -0.1, -0.1), size=(1.2, 1.2, 1.2))
    return Scene("PBF", cfg, [SceneObject("fluid", fluid, EPM_FLUID, export_flag=True, color_start=(0, 0, 1)),
                              SceneObject("box", wall, EPM_BOUNDARY)])


def pbf_dam_break_m1(seed: int = 1001, jitter_amp: float = 0.1) -> Scene:
    """The PBF dam break at the particle size of the reference's own PBF examples
    (particleRadius 0.05, so the particle mass rho0 (2r)^3 is 1): the same 20x40x20 block
    (16,000) in a 2-layer box, every length 5 times the benchmark's.  The reference's
    constraint gradients leave out the particle mass, which is consistent only for m = 1
    (PBFCudaImpl.cu:95-144); here its fluid stays in the box, where at r = 0.01 it passes
    through the floor."""
    r = 0.05
    fluid = jitter(cube(r, (0.2, 0.2, 0.2), (2.0, 4.0, 2.0)), jitter_amp, 2 * r, seed)
    wall = box(r, (0.0, 0.0, 0.0), (5.0, 5.0, 5.0), 2)
    cfg = pbf_config(dt=1.0 / 240.0, r=r, lb=(-0.5, -0.5, -0.5), size=(6.0, 6.0, 6.0))
    return Scene("PBF", cfg, [SceneObject("fluid", fluid, EPM_FLUID, export_flag=True, color_start=(0, 0, 1)),
                              SceneObject("box", wall, EPM_BOUNDARY)])


def dfsph_1m(seed: int = 2002, jitter_amp: float = 0.05) -> Scene:
    """DFSPH 1M: 100^3 fluid lattice at spacing 0.01 (x, y, z in [0.035, 1.025]) in a 3-layer box.

    The box is 2 x 1.5 x 1.06 (outer): a 1 m fluid cube does not fit inside a
    1 m box whose 3-layer walls are 0.03 m thick, so the z extent is widened until
    the far wall starts one spacing beyond the fluid (wall layers at z = 1.035 ...
    1.065).  The grid spans [-0.05, 2.05] x [-0.05, 1.55] x [-0.05, 1.15], leaving
    at least two empty cell layers beyond every wall.
    """
    r = 0.005
    fluid = jitter(cube(r, (0.03, 0.03, 0.03), (1.0, 1.0, 1.0)), jitter_amp, 2 * r, seed)
    wall = box(r, (0.0, 0.0, 0.0), (2.0, 1.5, 1.06), 3)
    cfg = dfsph_config(dt=1e-3, r=r, lb=(-0.05, -0.05, -0.05), size=(2.1, 1.6, 1.2))
    return Scene("DFSPH", cfg, [SceneObject("fluid", fluid, EPM_FLUID, export_flag=True, color_start=(0, 0, 1)),
                                SceneObject("box", wall, EPM_BOUNDARY)])


def dam_break(solver: str, n_target: int, seed: int, gravity_y: float = -9.81, jitter_amp: float = 0.05,
              spacing: float | None = None) -> Scene:
    """Dam break of about ``n_target`` particles: fluid block n x 2n x n in a cubic box of side n*spacing/0.4.

    Used for the small parity scenes and the batched scene mix; number density is constant
    because the box scales with the fluid block.  Spacing 0.02 for PBF and 0.01 for DFSPH
    unless given (0.1 gives PBF particles of mass 1, the reference examples' size).
    """
    spacing = spacing or (0.02 if solver == "PBF" else 0.01)
    r = spacing / 2
    n = max(2, int(round((n_target / 2.0) ** (1.0 / 3.0))))
    side = n * spacing / 0.4
    layers = 2 if solver == "PBF" else 3
    off = layers * spacing + spacing
    fluid = cube(r, (off, off, off), (n * spacing, 2 * n * spacing, n * spacing))
    fluid = jitter(fluid, jitter_amp, spacing, seed)
    wall = box(r, (0.0, 0.0, 0.0), (side, max(side, 2 * n * spacing + 2 * off), side), layers)
    ext = np.float32(max(side, 2 * n * spacing + 2 * off))
    lb = (-2 * spacing * 2.5,) * 3
    size = (float(side) + 5 * 2 * spacing * 2.5, float(ext) + 5 * 2 * spacing * 2.5, float(side) + 5 * 2 * spacing * 2.5)
    g = (0.0, gravity_y, 0.0)
    if solver == "PBF":
        cfg = pbf_config(dt=1.0 / 240.0, r=r, lb=lb, size=size, gravity=g)
    else:
        cfg = dfsph_config(dt=1e-3, r=r, lb=lb, size=size, gravity=g)
    return Scene(solver, cfg, [SceneObject("fluid", fluid, EPM_FLUID, export_flag=True),
                               SceneObject("box", wall, EPM_BOUNDARY)])


def colliding_blocks(seed: int = 41, tension: float = 0.001, speed: float = 1.5, n_side: int = 12,
                     jitter_amp: float = 0.05) -> Scene:
    """Two DFSPH fluid blocks (n_side^3 each, spacing 0.01) thrown at each other along x at
    +-speed inside a 3-layer box whose longest side is x, so that a decomposition into x slabs
    sees particles migrate between slabs within a few tens of substeps; surface tension on.
    Both fluid objects come before the box in attach order."""
    sp = 0.01
    r = sp / 2
    side = n_side * sp
    a = jitter(cube(r, (0.05, 0.05, 0.05), (side, side, side)), jitter_amp, sp, seed)
    b = jitter(cube(r, (0.1 + side, 0.06, 0.05), (side, side, side)), jitter_amp, sp, seed + 1)
    lx = 0.16 + 2 * side
    wall = box(r, (0.0, 0.0, 0.0), (lx, side + 0.13, side + 0.1), 3)
    cfg = dfsph_config(dt=1e-3, r=r, lb=(-0.05, -0.05, -0.05), size=(lx + 0.1, side + 0.23, side + 0.2),
                       tension=tension)
    return Scene("DFSPH", cfg, [SceneObject("left", a, EPM_FLUID, velocity_start=(speed, 0.0, 0.0)),
                                SceneObject("right", b, EPM_FLUID, velocity_start=(-speed, 0.0, 0.0)),
                                SceneObject("box", wall, EPM_BOUNDARY)])


def diff_pbf(seed: int = 5005) -> Scene:
    """The differentiable PBF scene: a 40^3 lattice (spacing 0.02, lb 0.2, no jitter) in a
    2-layer [0, 1.2]^3 box, initial fluid velocities N(0, 0.1^2) per component (SplitMix64
    stream ``seed``, Box-Muller), PBF parameters of the dam break, dt 1/240."""
    r = 0.01
    fluid = cube(r, (0.2, 0.2, 0.2), (0.8, 0.8, 0.8))
    wall = box(r, (0.0, 0.0, 0.0), (1.2, 1.2, 1.2), 2)
    u = splitmix64_uniform(seed, 2 * fluid.shape[0] * 3).reshape(2, -1)
    z = np.sqrt(-2.0 * np.log1p(-u[0])) * np.cos(2.0 * np.pi * u[1])
    v0 = (0.1 * z).reshape(-1, 3).astype(np.float32)
    cfg = pbf_config(dt=1.0 / 240.0, r=r, lb=(-0.1, -0.1, -0.1), size=(1.4, 1.4, 1.4))
    return Scene("PBF", cfg, [SceneObject("fluid", fluid, EPM_FLUID, export_flag=True, velocity=v0),
                              SceneObject("box", wall, EPM_BOUNDARY)])


def diff_dfsph(seed: int = 5005) -> Scene:
    """The differentiable DFSPH scene: a 40^3 lattice (spacing 0.01, lb 0.1, no jitter, 64,000
    fluid particles) in a 3-layer [0, 0.6]^3 box, initial fluid velocities N(0, 0.1^2) per
    component (SplitMix64 stream ``seed``, Box-Muller), DFSPH parameters of the dam break
    (dt 1 ms fixed, thresholds 0.1 %, viscosity 1e-6, no surface tension)."""
    r = 0.005
    fluid = cube(r, (0.1, 0.1, 0.1), (0.4, 0.4, 0.4))
    wall = box(r, (0.0, 0.0, 0.0), (0.6, 0.6, 0.6), 3)
    u = splitmix64_uniform(seed, 2 * fluid.shape[0] * 3).reshape(2, -1)
    z = np.sqrt(-2.0 * np.log1p(-u[0])) * np.cos(2.0 * np.pi * u[1])
    v0 = (0.1 * z).reshape(-1, 3).astype(np.float32)
    cfg = dfsph_config(dt=1e-3, r=r, lb=(-0.05, -0.05, -0.05), size=(0.7, 0.7, 0.7))
    return Scene("DFSPH", cfg, [SceneObject("fluid", fluid, EPM_FLUID, export_flag=True, velocity=v0),
                                SceneObject("box", wall, EPM_BOUNDARY)])


def batched_scenes(count: int = 64, n_pbf: int = 48, seed: int = 4242, gravity_seed: int = 4243,
                   n_min: float = 4e3, n_max: float = 2.56e5, pbf_spacing: float | None = None) -> list:
    """The batched mix: ``count`` dam breaks, the first ``n_pbf`` PBF and the rest DFSPH.

    Fluid counts are log-uniform in [n_min, n_max] (SplitMix64 stream ``seed``), gravity
    y is uniform in [-12, -8] (stream ``gravity_seed``), scene k is jittered with seed
    4000 + k.  Box size scales with the fluid block so number density is constant.
    ``pbf_spacing`` 0.1 makes the PBF scenes' particles of mass 1, where the reference's
    PBF formulation keeps the fluid in its box (the default 0.02 lets it through the floor).
    """
    u = splitmix64_uniform(seed, count)
    ns = np.round(np.exp(np.log(n_min) + u * (np.log(n_max) - np.log(n_min)))).astype(np.int64)
    g = -12.0 + 4.0 * splitmix64_uniform(gravity_seed, count)
    return [dam_break("PBF" if k < n_pbf else "DFSPH", int(ns[k]), seed=4000 + k, gravity_y=float(g[k]),
                      spacing=pbf_spacing if k < n_pbf else None)
            for k in range(count)]


def immct_config(*, dt, r, lb, size, rho=(1000.0, 1200.0), cf=1e-3, cd0=0.5, solvent_vis=0.01, vis_base=12.0,
                 vis_max=12.0, relax=0.05, thin=0.6, theta=0.4, div_thr=1e-4, incomp_thr=1e-4, tension=0.001,
                 colors=((255, 0, 0), (0, 0, 255)), gravity=(0.0, -9.81, 0.0), max_nbr=60, animation_time=5.0):
    return {"IMMCT": {"Required": {"animationTime": animation_time, "timeStep": dt, "particleRadius": r,
                                   "simSpaceLB": list(lb), "simSpaceSize": list(size), "maxNeighborNum": max_nbr,
                                   "divFreeThreshold": div_thr, "incompThreshold": incomp_thr,
                                   "surfaceTensionCoefficient": tension, "diffusionCoefficientCf": cf,
                                   "momentumExchangeCoefficientCd0": cd0, "solventViscosity": solvent_vis,
                                   "phaseRestDensity": list(rho), "phaseRestColor": [list(c) for c in colors],
                                   "solutionBasicViscosity": vis_base, "solutionMaxViscosity": vis_max,
                                   "relaxationTime": relax, "shearThinningBasicFactor": thin,
                                   "rheologicalThreshold": theta},
                      "Optional": {"enable": True, "gravity": list(gravity)}},
            "EXPORT": _export_block()}


def imm_config(*, dt, r, lb, size, rho=(1000.0, 1000.0, 1000.0), vis=(0.01, 0.01, 0.01), cf=0.1, cd=0.5,
               div_thr=1e-4, incomp_thr=1e-4, tension=0.001, colors=((255, 0, 0), (0, 255, 0), (0, 0, 255)),
               gravity=(0.0, -9.81, 0.0), max_nbr=60, animation_time=5.0):
    return {"IMM": {"Required": {"animationTime": animation_time, "timeStep": dt, "particleRadius": r,
                                 "simSpaceLB": list(lb), "simSpaceSize": list(size), "maxNeighborNum": max_nbr,
                                 "divFreeThreshold": div_thr, "incompThreshold": incomp_thr,
                                 "surfaceTensionCoefficient": tension, "diffusionCoefficientCf": cf,
                                 "momentumExchangeCoefficientCd": cd, "phaseRestDensity": list(rho),
                                 "phaseRestViscosity": list(vis), "phaseRestColor": [list(c) for c in colors]},
                    "Optional": {"enable": True, "gravity": list(gravity)}},
            "EXPORT": _export_block()}


def immct_500k(seed: int = 3003, jitter_amp: float = 0.05) -> Scene:
    """IMM-CT: two stacked 100 x 25 x 100 layers at spacing 0.01 (phase 1 below, phase 0 on top).

    Phase 1 (rho 1200) is the viscoelastic phase (the conformation-tensor terms read
    fraction index 1); relaxation time 0.05 s, thinning factor 0.6, Cf 1e-3,
    dt 0.5 ms.  Walls: 3-layer box 1.06 x 0.8 x 1.06.  Solver thresholds are 0.1 %.
    Solution viscosities are 8e-5 / 1.2e-4 (the example's 8 : 12 ratio): the
    reference's stress-divergence sum (add_phase_pct_acc_cuda) carries no neighbour
    volume, so its strength grows as 1 / V_j; at spacing 0.01 the template values
    (12) make the reference's own run explode within one substep.
    """
    r = 0.005
    bottom = cube(r, (0.03, 0.03, 0.03), (1.0, 0.25, 1.0))
    top = cube(r, (0.03, 0.28, 0.03), (1.0, 0.25, 1.0))
    both = jitter(np.concatenate([bottom, top]), jitter_amp, 2 * r, seed)
    wall = box(r, (0.0, 0.0, 0.0), (1.06, 0.8, 1.06), 3)
    cfg = immct_config(dt=5e-4, r=r, lb=(-0.05, -0.05, -0.05), size=(1.16, 0.9, 1.16), div_thr=1e-3,
                       incomp_thr=1e-3, vis_base=8e-5, vis_max=1.2e-4)
    nb = bottom.shape[0]
    return Scene("IMMCT", cfg, [
        SceneObject("bottom", both[:nb], EPM_FLUID, export_flag=True, phase_fraction=(0.0, 1.0)),
        SceneObject("top", both[nb:], EPM_FLUID, export_flag=True, phase_fraction=(1.0, 0.0)),
        SceneObject("box", wall, EPM_BOUNDARY, phase_fraction=(0.0, 1.0))])


def layered_mixture(solver: str, n_side: int, seed: int, jitter_amp: float = 0.05) -> Scene:
    """Small stratified mixture: two fluid layers of n x n/4 x n at spacing 0.01 in a 3-layer box."""
    r = 0.005
    sp = 2 * r
    off = 4 * sp
    hl = max(1, n_side // 4) * sp
    w = n_side * sp
    bottom = cube(r, (off, off, off), (w, hl, w))
    top = cube(r, (off, off + hl, off), (w, hl, w))
    both = jitter(np.concatenate([bottom, top]), jitter_amp, sp, seed)
    side = w + 2 * off
    height = 2 * hl + 2 * off + 0.1
    wall = box(r, (0.0, 0.0, 0.0), (side, height, side), 3)
    lb = (-0.05, -0.05, -0.05)
    size = (side + 0.1, height + 0.1, side + 0.1)
    nb = bottom.shape[0]
    if solver == "IMMCT":
        cfg = immct_config(dt=5e-4, r=r, lb=lb, size=size, vis_base=8e-5, vis_max=1.2e-4)
        fr_b, fr_t, fr_w = (0.0, 1.0), (1.0, 0.0), (0.0, 1.0)
    else:
        cfg = imm_config(dt=5e-4, r=r, lb=lb, size=size, rho=(1000.0, 1100.0, 1200.0), vis=(0.01, 0.02, 0.03))
        fr_b, fr_t, fr_w = (0.0, 0.3, 0.7), (0.6, 0.4, 0.0), (0.0, 0.0, 1.0)
    return Scene(solver, cfg, [
        SceneObject("bottom", both[:nb], EPM_FLUID, export_flag=True, phase_fraction=fr_b),
        SceneObject("top", both[nb:], EPM_FLUID, export_flag=True, phase_fraction=fr_t),
        SceneObject("box", wall, EPM_BOUNDARY, phase_fraction=fr_w)])


def grid_dims(cfg_block: dict, h: float):
    """Grid dimensions as ``UniformGirdNeighborSearcher::setConfig`` computes them (ceil(size / h))."""
    size = cfg_block["Required"]["simSpaceSize"]
    hh = np.float32(h)
    return tuple(int(math.ceil(float(np.float32(np.float32(s) / hh)))) for s in size)
