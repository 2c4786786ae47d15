"""Fitting a scene's materials and lights to a target image by gradient descent on the adjoint
(rtg_render_adjoint): the differentiable-render workload's loop.

The parameters are the base colours (RGB) and GGX alphas of the chosen materials and the powers of
the chosen lights. Each iteration writes them into the scene (rtg_scene_update with a file that
keeps the geometry, so no tree is rebuilt), renders the next range of samples with the adjoint,
and takes an Adam step: colours and alphas in their own units, powers in log space (their
gradients are scaled by the power), colours clamped to [0, 1] and alphas to [0.01, 1].
"""
from __future__ import annotations

import copy
import math
from dataclasses import dataclass, field
from typing import List, Sequence

import numpy as np

from . import scenes


@dataclass
class FitState:
    """Parameters as one vector: [colours (3 per material), alphas (1 per material), log powers]."""
    theta: np.ndarray
    m: np.ndarray
    v: np.ndarray
    step: int = 0
    losses: List[float] = field(default_factory=list)


class Fit:
    def __init__(self, scene, desc: scenes.Scene, target: np.ndarray, spp: int, materials: Sequence[int] = range(16),
                 lights: Sequence[int] = range(3), lr: float = 0.02, decay: float = 1.0):
        """scene: a loaded repackshot_b200.Scene of `desc`; target: h x w x 3 linear RGB. The step
        size is lr at the first step and shrinks by `decay` at every step: with noisy gradients,
        Adam's normalised steps let weakly constrained parameters wander by about lr per step, and
        a decaying step lets them settle."""
        self.scene, self.desc = scene, copy.deepcopy(desc)
        self.target = np.ascontiguousarray(target, np.float32)
        self.spp, self.lr, self.decay = spp, lr, decay
        self.materials, self.lights = list(materials), list(lights)
        self.film = scene.film()
        theta = np.concatenate([
            np.array([c for m in self.materials for c in desc.materials[m].base_color], np.float64),
            np.array([desc.materials[m].roughness ** 2 for m in self.materials], np.float64),
            np.array([math.log(max(desc.lights[j].power, 1e-12)) for j in self.lights], np.float64)])
        self.state = FitState(theta, np.zeros_like(theta), np.zeros_like(theta))

    def params(self):
        """(colours (k, 3), alphas (k,), powers (l,)) of the current parameters."""
        k, th = len(self.materials), self.state.theta
        return th[:3 * k].reshape(k, 3), th[3 * k:4 * k], np.exp(th[4 * k:])

    def _write(self):
        cols, alphas, powers = self.params()
        for i, m in enumerate(self.materials):
            self.desc.materials[m].base_color = tuple(float(c) for c in cols[i])
            self.desc.materials[m].roughness = float(math.sqrt(alphas[i]))
        for i, j in enumerate(self.lights):
            self.desc.lights[j].power = float(powers[i])
        self.scene.update(scenes.to_rsb(self.desc, meshes=False))

    def gradient(self):
        """(loss, gradient over theta) at the current parameters, on the next range of samples."""
        self._write()
        first = self.state.step * self.spp
        loss, grads, _ = self.scene.adjoint(self.film, self.target, first, self.spp)
        nm = len(self.desc.materials)
        G = grads[:4 * nm].reshape(nm, 4)
        _, _, powers = self.params()
        g = np.concatenate([G[self.materials, :3].reshape(-1), G[self.materials, 3],
                            grads[4 * nm + np.array(self.lights, int)] * powers])
        return loss, g.astype(np.float64)

    def step(self, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-12) -> float:
        """One Adam step; returns the loss before it."""
        loss, g = self.gradient()
        st = self.state
        st.step += 1
        st.m = b1 * st.m + (1 - b1) * g
        st.v = b2 * st.v + (1 - b2) * g * g
        mh, vh = st.m / (1 - b1 ** st.step), st.v / (1 - b2 ** st.step)
        st.theta = st.theta - self.lr * self.decay ** (st.step - 1) * mh / (np.sqrt(vh) + eps)
        k = len(self.materials)
        st.theta[:3 * k] = np.clip(st.theta[:3 * k], 0.0, 1.0)
        st.theta[3 * k:4 * k] = np.clip(st.theta[3 * k:4 * k], 0.01, 1.0)
        st.losses.append(loss)
        return loss
