"""CoreManager: the entry point of the reference (src/managers/core_manager.py).

Same constructor argument (the `simulation_parameters` dict of the demos),
same lifecycle (`initialization(fD, fN)`, `run()`, `kill()`).  The reference's
interactive GGUI window and video output (core_manager.py:58-139) need a
graphics stack and are not part of this build: `vis`, `make_video` and
`show_wireframe` are accepted and ignored.  What the window would draw stays
in device tensors: the per-vertex results (`BEMManager.solved`,
`.analytical_solved`) and the colour and position buffers that `run()` fills
as the reference's does (`.solved_vert_color`, `.analytical_vert_color`,
`.diff_vert_color`, `.solved_vertices`, `.analytical_vertices`,
`.diff_vertices`, each [nv, 3] float32).

Boundary-data callbacks are vectorised: fD(x[m,dim] float64 tensor[, sqrt_n])
and fN(x[m,dim], normal[m,dim][, sqrt_n]) return m real (Laplace) or complex
(Helmholtz) values (dim = 3, or 2 for the reference's 2D path on the
analytical disk).
"""
from __future__ import annotations

import logging

import torch

from .bem_manager import BEMManager
from .mesh_manager import MeshManager

log = logging.getLogger("bem_b200")


class _Log:
    """LogManager stand-in with the reference's method names
    (src/managers/log_manager.py:51-69), routed to `logging`."""
    initialized = True

    def InfoLog(self, s=""):
        log.info(s)

    def WarnLog(self, s=""):
        log.warning(s)

    def ErrorLog(self, s=""):
        log.error(s)

    def initialization(self):
        self.initialized = True

    def kill(self):
        pass


class CoreManager:
    def __init__(self, simulation_parameters):
        self._simulation_parameters = dict(simulation_parameters)
        p = self._simulation_parameters
        if "Helmholtz" not in p["kernel"]:
            p["k"] = 0
        self._is_transmission = 1 if ("Full" in p["boundary"] or "Transmission" in p["kernel"]) else 0
        if int(p.get("dim", 3)) not in (2, 3):
            raise NotImplementedError("dim must be 2 or 3")
        self._log_manager = _Log()
        self._mesh_manager = MeshManager(self)
        self._BEM_manager = BEMManager(self)
        self.initialized = False

    def initialization(self, analytical_function_Dirichlet, analytical_function_Neumann):
        self._log_manager.initialization()
        self._mesh_manager.initialization()
        self._BEM_manager.initialization(analytical_function_Dirichlet, analytical_function_Neumann)
        self.iteration = 0
        self.initialized = True

    def run(self):
        self._BEM_manager.run()
        b = self._BEM_manager
        a = b.raw_analytical_solved.abs()
        s = b.raw_solved.abs()
        d = (b.raw_solved - b.raw_analytical_solved).abs()
        self._log_manager.InfoLog("BEM has finished running")
        for name, t in (("analytical", a), ("solved", s), ("diff", d)):
            self._log_manager.InfoLog(f"{name}: min = {t.min().item():.6g}, max = {t.max().item():.6g}, "
                                      f"mean = {t.mean().item():.6g}")

    def kill(self):
        self.initialized = False
        self._BEM_manager.kill()
        self._mesh_manager.kill()
        self._log_manager.kill()
