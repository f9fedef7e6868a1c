"""Batched scenes: many independent scenes stepped together (``abd_batch_*`` in the C ABI).

The reference steps one scene per ``AffineBodySimulator``.  :class:`BatchSimulator` holds one
simulator per scene and steps them all with one CUDA graph launch: each scene's step (its
Newton iterations as a device loop) is a branch of the graph, so the scenes' iterations run
concurrently on the GPU while each keeps its own iteration counts, line search and
convergence -- every scene's result is the one its own ``step()`` gives.
"""
from __future__ import annotations

import ctypes

from . import _lib
from .params import SimParams
from .simulator import AffineBodySimulator


class BatchSimulator:
    """``scenes``: a list of body lists (one per scene, as ``scenes.config3`` returns them);
    ``params``: one :class:`SimParams` for all (or a list, one per scene)."""

    def __init__(self, scenes, params: SimParams | list | None = None, device: str = "cuda"):
        import torch
        prms = params if isinstance(params, list) else [params] * len(scenes)
        self.sims = [AffineBodySimulator(bodies=b, params=p, device=device) for b, p in zip(scenes, prms)]
        self.device = self.sims[0].device
        self._L = _lib.load()
        arr = (ctypes.c_void_p * len(self.sims))(*[s._h.value for s in self.sims])
        h = ctypes.c_void_p()
        stream = ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)
        _lib.check(self._L.abd_batch_create(len(self.sims), arr, stream, ctypes.byref(h)), "abd_batch_create")
        self._h = h
        self._states = (_lib.States * len(self.sims))(*[s._cstates() for s in self.sims])
        self._xview = (ctypes.c_void_p * len(self.sims))(*[s.x_view.data_ptr() for s in self.sims])

    def __len__(self):
        return len(self.sims)

    def step(self):
        """One step of every scene; returns the per-scene step infos."""
        infos = (_lib.StepInfo * len(self.sims))()
        _lib.check(self._L.abd_batch_step(self._h, self._states, self._xview, infos), "abd_batch_step")
        for s, inf in zip(self.sims, infos):
            s.last_info = inf.as_dict()
        return [inf.as_dict() for inf in infos]

    def step_sequential(self):
        """One step of every scene, one ``step()`` after another (the comparison)."""
        return [s.step() for s in self.sims]

    def reset(self):
        for s in self.sims:
            s.reset()

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            import torch
            torch.cuda.synchronize(self.device)
            self._L.abd_batch_destroy(self._h)
            self._h = None
        for s in getattr(self, "sims", []):
            s.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
