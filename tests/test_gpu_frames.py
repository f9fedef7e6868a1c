"""The headless frame loop: a config in the reference's format (scene file, frame range,
save_sequence, output folder) run through AffineBodySimulator.run(), its frames written as
.npz files and read back with load_trajectory -- the stand-in for the reference's viewer loop
and bgeo export (abd/abd.py:364-416, simulator/base.py:70-75)."""
import json

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _config(tmp_path):
    scene = {"objects": [
        {"file": "box.bgeo", "folder": "assets/", "p": [0.0, 0.0, 0.0], "fixed": True},
        {"file": "box.bgeo", "folder": "assets/", "p": [0.05, 1.05, -0.03], "pdot": [0.0, -2.0, 0.0],
         "Adot": [[0.0, 0.3, 0.0], [-0.3, 0.0, 0.0], [0.0, 0.0, 0.0]]}]}
    (tmp_path / "scene.json").write_text(json.dumps(scene))
    cfg = {"scene": "scene.json", "frame_in": 0, "frame_out": 8, "save_sequence": True,
           "output_seq_folder": "frames", "dt": 0.01, "dhat": 1e-3, "mesh_map": {"box.bgeo": "cube:1.0"}}
    path = tmp_path / "config.json"
    path.write_text(json.dumps(cfg))
    return path


def test_run_exports_every_frame(tmp_path):
    from abd_warp_b200.simulator import AffineBodySimulator, load_trajectory
    cfg = _config(tmp_path)
    sim = AffineBodySimulator(str(cfg))
    assert sim.params.dhat == 1e-3 and sim.frame_out == 8 and sim.save_sequence
    infos = sim.run()
    assert len(infos) == 8 and all(i["status"] == 0 for i in infos)
    traj = load_trajectory(str(tmp_path / "frames"))
    np.testing.assert_array_equal(traj["frames"], np.arange(8))
    assert traj["x"].shape == (8, 16, 3)
    # a second simulator stepped frame by frame gives the same positions, bit for bit
    ref = AffineBodySimulator(str(cfg))
    for f in range(8):
        ref.step(f)
        np.testing.assert_array_equal(traj["x"][f], ref.x_view.cpu().numpy())
        np.testing.assert_array_equal(traj["p"][f], ref.states.p0.cpu().numpy())
    # the fixed body stays put; the other falls
    np.testing.assert_array_equal(traj["x"][-1][:8], traj["x"][0][:8])
    assert traj["p"][-1][1][1] < traj["p"][0][1][1]
    sim.close()
    ref.close()
