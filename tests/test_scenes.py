import numpy as np
import pytest

from abd_warp_b200 import meshes, scenes


@pytest.mark.parametrize("level,counts", [(2, (162, 320, 480)), (3, (642, 1280, 1920))])
def test_icosphere_counts(level, counts):
    V, F = meshes.icosphere_mesh(level, 0.3)
    E = meshes.unique_edges(F)
    assert (V.shape[0], F.shape[0], E.shape[0]) == counts


def test_cube_mass_properties():
    V, F = meshes.cube_mesh(0.5)
    m, com, I0 = meshes.mass_properties(V, F, 1000.0)
    assert m == pytest.approx(1000 * 0.125)
    assert np.allclose(com, 0)
    assert I0 == pytest.approx(1000 * 0.5 ** 5 / 12)
    assert meshes.unique_edges(F).shape[0] == 18


@pytest.mark.parametrize("idx,sizes", [(0, (2, 16, 24, 36)), (1, (65, 10376, 20492, 30738)),
                                       (4, (17, 2600, 5132, 7698))])
def test_config_sizes(idx, sizes):
    bodies, prm, steps = scenes.make_config(idx)
    f = scenes.flatten_bodies(bodies)
    assert (f["n"], f["voff"][-1], f["toff"][-1], f["eoff"][-1]) == sizes


def test_config0_initial_separation():
    bodies, prm, _ = scenes.make_config(0)
    assert bodies[1].vertices_world()[:, 1].min() > 0.5 + prm.dhat


def test_scene_json_with_mesh_map(tmp_path):
    """A scene in the reference's JSON format (objects with file / folder / p / Adot) whose
    .bgeo assets have no reader here loads once their names are mapped to procedural meshes."""
    import json
    from abd_warp_b200.affine_body import Scene
    scene = {"objects": [
        {"file": "box.bgeo", "folder": "assets/", "p": [0.0, 0.2, 0.0],
         "Adot": [[0.0, 0.5, 0.0], [-0.5, 0.0, 0.0], [0.0, 0.0, 0.0]]},
        {"file": "box.bgeo", "folder": "assets/", "p": [0.3, 2.0, 0.1]}]}
    path = tmp_path / "scene.json"
    path.write_text(json.dumps(scene))
    with pytest.raises(ValueError, match="mesh_map"):
        Scene(scene_config_file=str(path))
    s = Scene(scene_config_file=str(path), mesh_map={"box.bgeo": "cube:1.0"})
    assert len(s.kinetic_objects) == 2
    a, b = s.kinetic_objects
    assert a.V.shape == (8, 3) and a.F.shape == (12, 3) and a.edges.shape == (18, 2)
    np.testing.assert_array_equal(a.p, [0.0, 0.2, 0.0])
    np.testing.assert_array_equal(a.Adot[0], [0.0, 0.5, 0.0])
    np.testing.assert_array_equal(b.A, np.identity(3))
    assert abs(a.mass - 1000.0) < 1e-9  # unit cube, density 1000


def test_config3_batched_scenes():
    """Configuration 3 (the batched workload): independent scenes of 2..48 bodies over their
    own fixed ground box, deterministic for a seed, bodies apart (bounding spheres more than
    2 dhat apart) and above the ground."""
    import numpy as np
    from abd_warp_b200 import scenes

    sc, prm, steps = scenes.config3(n_scenes=12)
    again, _, _ = scenes.config3(n_scenes=12)
    assert steps == 100 and len(sc) == 12
    for bodies, other in zip(sc, again):
        assert 3 <= len(bodies) <= 49
        assert bodies[0].fixed and not any(b.fixed for b in bodies[1:])
        assert len(other) == len(bodies)
        for b, c in zip(bodies, other):
            np.testing.assert_array_equal(b.vertices_world(), c.vertices_world())
        centres = [b.vertices_world().mean(axis=0) for b in bodies[1:]]
        radii = [np.linalg.norm(b.vertices_world() - m, axis=1).max() for b, m in zip(bodies[1:], centres)]
        for i in range(len(centres)):
            assert bodies[1 + i].vertices_world()[:, 1].min() > 0.0
            for j in range(i):
                assert np.linalg.norm(centres[i] - centres[j]) > radii[i] + radii[j] + 2 * prm.dhat - 1e-9
