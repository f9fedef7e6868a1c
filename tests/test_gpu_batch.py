"""Batched scenes on the GPU (abd_batch_step through the C ABI, abd_warp_b200/batch.py): the
scenes of the batched configuration (independent scenes of 2 to 48 bodies over their own
ground boxes) stepped together by one graph launch give each scene exactly the result of its
own step: bit for bit against the same scenes stepped one by one, and against the oracle."""
import numpy as np
import pytest

import oracle
from abd_warp_b200 import scenes

pytestmark = pytest.mark.gpu

FIELDS = ("A0", "p0", "Adot", "pdot")
COUNTERS = ("newton_iters", "linear_iters", "ls_trials", "n_pt", "n_ee", "n_vg", "n_ij", "n_active")


def _scenes(n):
    sc, prm, _ = scenes.config3(n_scenes=n)
    return sc, prm


def test_batch_equals_scene_by_scene_and_the_oracle():
    from abd_warp_b200.batch import BatchSimulator
    sc, prm = _scenes(12)
    batch = BatchSimulator(sc, prm)
    alone = BatchSimulator(sc, prm)
    orcs = [oracle.Oracle(scenes.flatten_bodies(b), prm) for b in sc[:3]]
    contact = 0
    try:
        for step in range(40):
            got = batch.step()
            ref = alone.step_sequential()
            for i in range(len(sc)):
                for k in COUNTERS:
                    assert got[i][k] == ref[i][k], (step, i, k)
                assert got[i]["energy"] == ref[i]["energy"], (step, i)
                for f in FIELDS:
                    np.testing.assert_array_equal(getattr(batch.sims[i].states, f).cpu().numpy(),
                                                  getattr(alone.sims[i].states, f).cpu().numpy(), err_msg=f"{step} {i} {f}")
                contact += got[i]["n_active"]
            for i, o in enumerate(orcs):
                ri = o.step()
                for k in COUNTERS:
                    assert got[i][k] == ri[k], (step, i, k)
                st = o.get_state()
                for f in FIELDS:
                    np.testing.assert_array_equal(getattr(batch.sims[i].states, f).cpu().numpy(), st[f])
        assert contact > 0  # the scenes land on their ground boxes
    finally:
        batch.close()
        alone.close()


def test_batch_reruns_a_scene_whose_list_overflowed():
    """A scene created with tiny lists (min_capacity) overflows inside the batch graph; it is
    grown and stepped again alone, and its result still equals its own step's."""
    import dataclasses

    from abd_warp_b200.batch import BatchSimulator
    sc, prm = _scenes(4)
    prms = [prm, dataclasses.replace(prm, min_capacity=16), prm, prm]
    batch = BatchSimulator(sc, prms)
    alone = BatchSimulator(sc, prm)
    try:
        for step in range(30):
            got = batch.step()
            ref = alone.step_sequential()
            for i in range(len(sc)):
                for k in COUNTERS:
                    assert got[i][k] == ref[i][k], (step, i, k)
                for f in FIELDS:
                    np.testing.assert_array_equal(getattr(batch.sims[i].states, f).cpu().numpy(),
                                                  getattr(alone.sims[i].states, f).cpu().numpy())
    finally:
        batch.close()
        alone.close()
